// grog_v6.cu -- fused GROG grid / degrid with operator-stationary slots.
//
// Work split.  A warp is cut into S "slots" of L = C / RPL lanes; a slot
// handles one replica at a time and lane l of the slot produces the RPL
// output coils l*RPL .. l*RPL+RPL-1.  The valid replicas of a brick are cut
// into sub-chunks of at most `sub_cap` replicas along the sample index, so a
// sub-chunk's source samples ("slots" of the staging buffer) are gathered
// with coalesced loads.  Inside a sub-chunk the replicas are ordered by
// (outer index, inner index, cell) and every warp takes a contiguous range,
// so the slots of one warp step mostly share the outer factor (a shared-
// memory broadcast).  Both factors (or the whole table when it is not
// factored) live in shared memory in a lane-chunk layout (chunk (j, l) = the
// RPL entries of column j that lane l needs, contiguous; operators start in
// different bank quads).
//
//   forward:  y = O[k] (I[q] x_src)      grid[:, cell] += w y
//   adjoint:  y = I^H[q] (O^H[k] g_cell) out[:, src]  += w y
//
// Scheduling.  The plan gives every CTA a fixed stream of sub-chunk
// descriptors (bricks assigned largest-first to the least loaded CTA), so a
// CTA knows its next sub-chunks in advance: the descriptors are prefetched
// three ahead, the staging-slot sample indices two ahead, and the sample
// coils, replica metadata and weights of the next sub-chunk are copied into
// the second shared-memory buffer with cp.async while the current one is
// computed.  Bricks with more than one item ("split") add into a
// pre-zeroed brick with global atomics.
#include "common.cuh"

namespace pgb {

struct Geom6 {
  int gz, gy, gx;
  int bz, by, bx;
  int lbx, lby;
  int nbz, nby, nbx;
};

constexpr int kT6 = 512;
constexpr int kW6 = kT6 / 32;

// stream-entry flags
constexpr int kFirst = 1, kLast = 2, kSplit = 4;

template <int C>
struct Map6 {
  static constexpr int RPL = (C % 2 == 0) ? 2 : 1;            // output rows per lane
  static constexpr int L = C / RPL;                           // lanes per slot
  static constexpr int S = 32 / L;                            // slots per warp
  static constexpr int OPS = C * C + ((C % 2 == 0) ? 2 : 1);  // float2 per staged operator
  static constexpr int XS = C + ((C % 2 == 0) ? 2 : 1);       // float2 per staged vector
};

__device__ __forceinline__ void origin6(const Geom6& g, int brick, int& z0, int& y0, int& x0) {
  const int bxy = g.nby * g.nbx;
  const int biz = brick / bxy;
  const int rem = brick - biz * bxy;
  const int biy = rem / g.nbx;
  z0 = biz * g.bz;
  y0 = biy * g.by;
  x0 = (rem - biy * g.nbx) * g.bx;
}

__device__ __forceinline__ bool flat6(const Geom6& g, int z0, int y0, int x0, int cl, int64_t& flat) {
  const int x = x0 + (cl & (g.bx - 1));
  const int y = y0 + ((cl >> g.lbx) & (g.by - 1));
  const int z = z0 + (cl >> (g.lbx + g.lby));
  if (z >= g.gz || y >= g.gy || x >= g.gx) return false;
  flat = (static_cast<int64_t>(z) * g.gy + y) * g.gx + x;
  return true;
}

__host__ __device__ constexpr int round_even(int v) { return (v + 1) & ~1; }

// Shared-memory carve-up in float2 units:
//   inner table | outer table | tile | xs[2] (sub_cap x XS) | meta[2] (sub_cap int2) | w[2] (sub_cap float, padded) | exchange rows
template <int C>
struct Smem6 {
  int tab, otab, tile, xs, ms, ws, ub, total;
  __host__ __device__ Smem6(int n_inner, int n_outer, int cells, int sub_cap, bool forward) {
    tab = 0;
    otab = n_inner * Map6<C>::OPS;
    tile = otab + (n_outer > 1 ? n_outer * Map6<C>::OPS : 0);
    const int tile_sz = forward ? C * (cells + 1) : cells * C;
    xs = tile + round_even(tile_sz);
    ms = xs + 2 * sub_cap * Map6<C>::XS;
    ws = ms + 2 * sub_cap;
    ub = ws + round_even(sub_cap);  // 2 * sub_cap floats
    total = ub + kW6 * Map6<C>::S * Map6<C>::XS;
  }
};

__device__ __forceinline__ void cp_async8z(void* smem_dst, const void* gsrc, int bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Stage the lane-chunk table: global (n, C*C) -> shared (n, OPS).
template <int C>
__device__ __forceinline__ void stage_tab6(float2* __restrict__ dst, const float2* __restrict__ src, int n) {
  constexpr int per = C * C;
  for (int t = threadIdx.x; t < n * per; t += kT6) {
    const int m = t / per;
    dst[m * Map6<C>::OPS + (t - m * per)] = __ldg(src + t);
  }
}

// acc[t] += sum_j tab_chunk(j, l)[t] * v[j]   (one operator, lane-chunk layout)
template <int C>
__device__ __forceinline__ void apply_lc(const float2* __restrict__ op, const float2* __restrict__ v, int l,
                                         float2 (&acc)[Map6<C>::RPL]) {
  using M = Map6<C>;
  if constexpr (M::RPL == 2) {
#pragma unroll
    for (int j = 0; j < C; j += 2) {
      const float4 vv = *reinterpret_cast<const float4*>(v + j);
      const float4 a0 = *reinterpret_cast<const float4*>(op + (j * M::L + l) * 2);
      const float4 a1 = *reinterpret_cast<const float4*>(op + ((j + 1) * M::L + l) * 2);
      cfma(acc[0], make_float2(a0.x, a0.y), make_float2(vv.x, vv.y));
      cfma(acc[1], make_float2(a0.z, a0.w), make_float2(vv.x, vv.y));
      cfma(acc[0], make_float2(a1.x, a1.y), make_float2(vv.z, vv.w));
      cfma(acc[1], make_float2(a1.z, a1.w), make_float2(vv.z, vv.w));
    }
  } else {
#pragma unroll
    for (int j = 0; j < C; ++j) cfma(acc[0], op[j * M::L + l], v[j]);
  }
}

struct Rep6 {
  int cell, slot, q, k;
  float w;
};

__device__ __forceinline__ bool decode6(int2 m, float w, int cells, int nu, int n_inner, int n_outer, Rep6& rp) {
  rp.cell = m.x & 0xFFFF;
  rp.slot = static_cast<int>(static_cast<unsigned>(m.x) >> 16);
  rp.q = m.y & 0xFFFF;
  rp.k = static_cast<int>(static_cast<unsigned>(m.y) >> 16);
  rp.w = w;
  return rp.cell < cells && rp.slot < nu && rp.q < n_inner && rp.k < n_outer;
}

// Sub-chunk stream of one CTA with descriptors prefetched three ahead.
struct Stream6 {
  const int4* sd;
  const int2* si;
  int p, p1;
  int4 d0, d1, d2, d3;
  int2 i0, i1, i2, i3;
  __device__ __forceinline__ int4 ld_d(int q) const {
    return q < p1 ? __ldg(sd + q) : make_int4(0, 0, 0, 0);
  }
  __device__ __forceinline__ int2 ld_i(int q) const { return q < p1 ? __ldg(si + q) : make_int2(0, 0); }
  __device__ __forceinline__ void init(const int4* sd_, const int2* si_, int p0_, int p1_) {
    sd = sd_;
    si = si_;
    p = p0_;
    p1 = p1_;
    d0 = ld_d(p);
    d1 = ld_d(p + 1);
    d2 = ld_d(p + 2);
    d3 = ld_d(p + 3);
    i0 = ld_i(p);
    i1 = ld_i(p + 1);
    i2 = ld_i(p + 2);
    i3 = ld_i(p + 3);
  }
  __device__ __forceinline__ void advance() {
    ++p;
    d0 = d1;
    d1 = d2;
    d2 = d3;
    i0 = i1;
    i1 = i2;
    i2 = i3;
    d3 = ld_d(p + 3);
    i3 = ld_i(p + 3);
  }
};

__device__ __forceinline__ int nslots(int4 d, int sub_cap) { return min(max(d.w - d.z, 0), sub_cap); }
__device__ __forceinline__ int nreps(int4 d, int sub_cap) { return min(max(d.y - d.x, 0), sub_cap); }

// Thread t: staging slot t (all C coils of sample u) and replica t (meta, weight).
template <int C, bool COILS>
__device__ __forceinline__ void issue_stage6(const float2* __restrict__ dat, int64_t N, const int2* __restrict__ meta,
                                             const float* __restrict__ wts, int4 d, int u, int sub_cap,
                                             float2* __restrict__ xs, int2* __restrict__ ms, float* __restrict__ ws) {
  const int t = threadIdx.x;
  if constexpr (COILS) {
    if (t < nslots(d, sub_cap)) {
      const bool ok = u >= 0 && u < N;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const float2* src = ok ? dat + static_cast<int64_t>(c) * N + u : dat;
        cp_async8z(xs + t * Map6<C>::XS + c, src, ok ? 8 : 0);
      }
    }
  }
  if (t < nreps(d, sub_cap)) {
    cp_async8z(ms + t, meta + d.x + t, 8);
    cp_async4(ws + t, wts + d.x + t);
  }
}

template <int C, bool OUTER>
__global__ void __launch_bounds__(kT6, 1) grog_grid_v6_kernel(
    const float2* __restrict__ data, int64_t N, float2* __restrict__ grid, int64_t G,
    const float2* __restrict__ inner_lc, int n_inner, const float2* __restrict__ outer_lc, int n_outer,
    const int4* __restrict__ sd, const int2* __restrict__ si, const int32_t* __restrict__ cta_ptr,
    const int32_t* __restrict__ uniq, const int2* __restrict__ meta, const float* __restrict__ wts, int sub_cap,
    Geom6 geom) {
  using M = Map6<C>;
  extern __shared__ float4 smem4[];
  const int p0 = cta_ptr[blockIdx.x], p1 = cta_ptr[blockIdx.x + 1];
  if (p0 >= p1) return;  // block-uniform
  const int cells = geom.bz * geom.by * geom.bx;
  const int TS = cells + 1;
  const Smem6<C> lay(n_inner, OUTER ? n_outer : 1, cells, sub_cap, true);
  float2* base = reinterpret_cast<float2*>(smem4);
  float2* tab = base + lay.tab;
  float2* otab = base + lay.otab;
  float2* tile = base + lay.tile;  // (C, TS)
  float2* xs0 = base + lay.xs;
  int2* ms0 = reinterpret_cast<int2*>(base + lay.ms);
  float* ws0 = reinterpret_cast<float*>(base + lay.ws);
  float2* ub = base + lay.ub;
  const int b = blockIdx.y;
  const float2* dat = data + static_cast<int64_t>(b) * C * N;
  float2* grd = grid + static_cast<int64_t>(b) * C * G;

  Stream6 st;
  st.init(sd, si, p0, p1);
  const int tid = threadIdx.x;
  int u0 = tid < nslots(st.d0, sub_cap) ? __ldg(uniq + st.d0.z + tid) : -1;
  int u1 = tid < nslots(st.d1, sub_cap) && st.p + 1 < p1 ? __ldg(uniq + st.d1.z + tid) : -1;
  issue_stage6<C, true>(dat, N, meta, wts, st.d0, u0, sub_cap, xs0, ms0, ws0);
  cp_commit();
  stage_tab6<C>(tab, inner_lc, n_inner);
  if (OUTER) stage_tab6<C>(otab, outer_lc, n_outer);
  for (int t = tid; t < C * TS; t += kT6) tile[t] = make_float2(0.f, 0.f);

  const int warp = tid >> 5, lane = tid & 31;
  const int slot = lane / M::L;
  const int l = lane - slot * M::L;
  const bool lane_on = slot < M::S;
  float2* ubw = ub + (warp * M::S + (lane_on ? slot : 0)) * M::XS;
  int buf = 0;
  while (true) {
    const bool more = st.p + 1 < p1;
    if (more) {
      const int nb = buf ^ 1;
      issue_stage6<C, true>(dat, N, meta, wts, st.d1, u1, sub_cap, xs0 + nb * sub_cap * M::XS, ms0 + nb * sub_cap,
                            ws0 + nb * sub_cap);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    // slot samples of the sub-chunk after next (consumed at the next iteration)
    const int u2 = st.p + 2 < p1 && tid < nslots(st.d2, sub_cap) ? __ldg(uniq + st.d2.z + tid) : -1;
    __syncthreads();  // buffer `buf` complete; tile zeroed
    {
      const int nu = nslots(st.d0, sub_cap);
      const int nr = nreps(st.d0, sub_cap);
      const float2* xs = xs0 + buf * sub_cap * M::XS;
      const int2* ms = ms0 + buf * sub_cap;
      const float* ws = ws0 + buf * sub_cap;
      const int per = (((nr + kW6 - 1) / kW6) + M::S - 1) / M::S * M::S;
      const int rb = warp * per;
      const int re = min(nr, rb + per);
      for (int r0 = rb; r0 < re; r0 += M::S) {  // warp-uniform trip count
        const int r = r0 + slot;
        Rep6 rp{0, 0, 0, 0, 0.f};
        bool on = lane_on && r < re;
        if (on) on = decode6(ms[r], ws[r], cells, nu, n_inner, OUTER ? n_outer : 1, rp);
        if (!on) rp = Rep6{0, 0, 0, 0, 0.f};
        float2 u[M::RPL];
#pragma unroll
        for (int t = 0; t < M::RPL; ++t) u[t] = make_float2(0.f, 0.f);
        apply_lc<C>(tab + rp.q * M::OPS, xs + rp.slot * M::XS, l, u);
        if constexpr (OUTER) {
          if (lane_on) {
#pragma unroll
            for (int t = 0; t < M::RPL; ++t) ubw[l * M::RPL + t] = u[t];
          }
          __syncwarp();
          float2 y[M::RPL];
#pragma unroll
          for (int t = 0; t < M::RPL; ++t) y[t] = make_float2(0.f, 0.f);
          apply_lc<C>(otab + rp.k * M::OPS, ubw, l, y);
          __syncwarp();
#pragma unroll
          for (int t = 0; t < M::RPL; ++t) u[t] = y[t];
        }
        if (on) {
#pragma unroll
          for (int t = 0; t < M::RPL; ++t) {
            float2* dst = tile + (l * M::RPL + t) * TS + rp.cell;
            atomicAdd(&dst->x, rp.w * u[t].x);
            atomicAdd(&dst->y, rp.w * u[t].y);
          }
        }
      }
    }
    __syncthreads();  // compute done: buffer `buf` and the tile are free
    if (st.i0.y & kLast) {
      int z0, y0, x0;
      origin6(geom, st.i0.x, z0, y0, x0);
      const bool split = (st.i0.y & kSplit) != 0;
      for (int t = tid; t < C * cells; t += kT6) {
        const int c = t / cells;
        const int cl = t - c * cells;
        int64_t flat;
        if (!flat6(geom, z0, y0, x0, cl, flat)) continue;
        const float2 v = tile[c * TS + cl];
        float2* dst = grd + static_cast<int64_t>(c) * G + flat;
        if (split) {
          if (v.x != 0.f || v.y != 0.f) {
            atomicAdd(&dst->x, v.x);
            atomicAdd(&dst->y, v.y);
          }
        } else {
          *dst = v;
        }
      }
      if (!more) break;
      __syncthreads();  // flush read the tile
      for (int t = tid; t < C * TS; t += kT6) tile[t] = make_float2(0.f, 0.f);
    } else if (!more) {
      break;
    }
    st.advance();
    u1 = u2;
    buf ^= 1;
  }
}

template <int C, bool OUTER, bool ACC>
__global__ void __launch_bounds__(kT6, 1) grog_degrid_v6_kernel(
    const float2* __restrict__ grid, int64_t G, float2* __restrict__ out, int64_t N,
    const float2* __restrict__ inner_h_lc, int n_inner, const float2* __restrict__ outer_h_lc, int n_outer,
    const int4* __restrict__ sd, const int2* __restrict__ si, const int32_t* __restrict__ cta_ptr,
    const int32_t* __restrict__ uniq, const int2* __restrict__ meta, const float* __restrict__ wts, int sub_cap,
    Geom6 geom) {
  using M = Map6<C>;
  extern __shared__ float4 smem4[];
  const int p0 = cta_ptr[blockIdx.x], p1 = cta_ptr[blockIdx.x + 1];
  if (p0 >= p1) return;
  const int cells = geom.bz * geom.by * geom.bx;
  const Smem6<C> lay(n_inner, OUTER ? n_outer : 1, cells, sub_cap, false);
  float2* base = reinterpret_cast<float2*>(smem4);
  float2* tab = base + lay.tab;
  float2* otab = base + lay.otab;
  float2* tile = base + lay.tile;  // (cells, C) cell-major
  float2* xs0 = base + lay.xs;     // per-slot results
  int2* ms0 = reinterpret_cast<int2*>(base + lay.ms);
  float* ws0 = reinterpret_cast<float*>(base + lay.ws);
  float2* ub = base + lay.ub;
  const int b = blockIdx.y;
  const float2* grd = grid + static_cast<int64_t>(b) * C * G;
  float2* o = out + static_cast<int64_t>(b) * C * N;

  Stream6 st;
  st.init(sd, si, p0, p1);
  const int tid = threadIdx.x;
  // brick tile of the first item, then the replica metadata of the first sub-chunk
  auto issue_tile = [&](int brick) {
    int z0, y0, x0;
    origin6(geom, brick, z0, y0, x0);
    for (int t = tid; t < C * cells; t += kT6) {
      const int c = t / cells;
      const int cl = t - c * cells;
      int64_t flat;
      const bool in = flat6(geom, z0, y0, x0, cl, flat);
      cp_async8z(tile + cl * C + c, in ? grd + static_cast<int64_t>(c) * G + flat : grd, in ? 8 : 0);
    }
  };
  issue_tile(st.i0.x);
  issue_stage6<C, false>(nullptr, N, meta, wts, st.d0, 0, sub_cap, nullptr, ms0, ws0);
  cp_commit();
  stage_tab6<C>(tab, inner_h_lc, n_inner);
  if (OUTER) stage_tab6<C>(otab, outer_h_lc, n_outer);
  int u0 = tid < nslots(st.d0, sub_cap) ? __ldg(uniq + st.d0.z + tid) : -1;

  const int warp = tid >> 5, lane = tid & 31;
  const int slot = lane / M::L;
  const int l = lane - slot * M::L;
  const bool lane_on = slot < M::S;
  float2* ubw = ub + (warp * M::S + (lane_on ? slot : 0)) * M::XS;
  int buf = 0;
  while (true) {
    const bool more = st.p + 1 < p1;
    if (more) {
      const int nb = buf ^ 1;
      issue_stage6<C, false>(nullptr, N, meta, wts, st.d1, 0, sub_cap, nullptr, ms0 + nb * sub_cap,
                             ws0 + nb * sub_cap);
      cp_commit();
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    const int u1 = more && tid < nslots(st.d1, sub_cap) ? __ldg(uniq + st.d1.z + tid) : -1;
    const int nu = nslots(st.d0, sub_cap);
    const int nr = nreps(st.d0, sub_cap);
    float2* xs = xs0 + buf * sub_cap * M::XS;
    if (ACC) {
      for (int t = tid; t < nu * M::XS; t += kT6) xs[t] = make_float2(0.f, 0.f);
    }
    __syncthreads();  // tile and metadata of this sub-chunk complete; xs cleared
    {
      const int2* ms = ms0 + buf * sub_cap;
      const float* ws = ws0 + buf * sub_cap;
      const int per = (((nr + kW6 - 1) / kW6) + M::S - 1) / M::S * M::S;
      const int rb = warp * per;
      const int re = min(nr, rb + per);
      for (int r0 = rb; r0 < re; r0 += M::S) {
        const int r = r0 + slot;
        Rep6 rp{0, 0, 0, 0, 0.f};
        bool on = lane_on && r < re;
        if (on) on = decode6(ms[r], ws[r], cells, nu, n_inner, OUTER ? n_outer : 1, rp);
        if (!on) rp = Rep6{0, 0, 0, 0, 0.f};
        const float2* gin = tile + rp.cell * C;
        if constexpr (OUTER) {
          float2 v[M::RPL];
#pragma unroll
          for (int t = 0; t < M::RPL; ++t) v[t] = make_float2(0.f, 0.f);
          apply_lc<C>(otab + rp.k * M::OPS, gin, l, v);
          if (lane_on) {
#pragma unroll
            for (int t = 0; t < M::RPL; ++t) ubw[l * M::RPL + t] = v[t];
          }
          __syncwarp();
          gin = ubw;
        }
        float2 y[M::RPL];
#pragma unroll
        for (int t = 0; t < M::RPL; ++t) y[t] = make_float2(0.f, 0.f);
        apply_lc<C>(tab + rp.q * M::OPS, gin, l, y);
        if constexpr (OUTER) __syncwarp();
        if (on) {
#pragma unroll
          for (int t = 0; t < M::RPL; ++t) {
            float2* dst = xs + rp.slot * M::XS + l * M::RPL + t;
            if (ACC) {
              atomicAdd(&dst->x, rp.w * y[t].x);
              atomicAdd(&dst->y, rp.w * y[t].y);
            } else {
              *dst = make_float2(rp.w * y[t].x, rp.w * y[t].y);
            }
          }
        }
      }
    }
    __syncthreads();  // results of this sub-chunk complete; tile no longer read
    // next item's tile (lands before the next iteration's wait)
    if ((st.i0.y & kLast) && more) {
      issue_tile(st.i1.x);
      cp_commit();
    }
    if (tid < nu && u0 >= 0 && u0 < N) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const float2 v = xs[tid * M::XS + c];
        float2* dst = o + static_cast<int64_t>(c) * N + u0;
        if (ACC) {
          atomicAdd(&dst->x, v.x);
          atomicAdd(&dst->y, v.y);
        } else {
          *dst = v;
        }
      }
    }
    if (!more) break;
    st.advance();
    u0 = u1;
    buf ^= 1;
  }
}

__global__ void zero_bricks_v6(float2* __restrict__ grid, int64_t G, int C, int B,
                               const int32_t* __restrict__ bricks, int n_bricks, Geom6 geom) {
  const int cells = geom.bz * geom.by * geom.bx;
  const int64_t total = static_cast<int64_t>(n_bricks) * cells;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / cells);
    const int cl = static_cast<int>(t - static_cast<int64_t>(i) * cells);
    int z0, y0, x0;
    origin6(geom, bricks[i], z0, y0, x0);
    int64_t flat;
    if (!flat6(geom, z0, y0, x0, cl, flat)) continue;
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < C; ++c) grid[(static_cast<int64_t>(b) * C + c) * G + flat] = make_float2(0.f, 0.f);
  }
}

__global__ void zero_samples_v6(float2* __restrict__ out, int64_t N, int C, int B,
                                const int32_t* __restrict__ src, int64_t n) {
  const int64_t total = n * C * B;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = t % n;
    const int64_t bc = t / n;
    const int64_t s = src[i];
    if (s >= 0 && s < N) out[bc * N + s] = make_float2(0.f, 0.f);
  }
}

#define PGB6_FOR_EACH_C(X) \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

static size_t v6_smem_c(int64_t C, int cells, int64_t n_inner, int64_t n_outer, int64_t sub_cap, bool forward) {
  switch (C) {
#define X(CC)                                                                                              \
  case CC:                                                                                                 \
    return static_cast<size_t>(Smem6<CC>(static_cast<int>(n_inner), static_cast<int>(n_outer), cells,      \
                                         static_cast<int>(sub_cap), forward).total) * sizeof(float2);
    PGB6_FOR_EACH_C(X)
#undef X
    default:
      return ~static_cast<size_t>(0);
  }
}

static int v6_geom(const pgb_v6_plan* p, Geom6& g, const char* who) {
  PGB_REQUIRE(p != nullptr, PGB_ERR_INVALID, "%s: null plan", who);
  auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
  PGB_REQUIRE(pow2(p->bz) && pow2(p->by) && pow2(p->bx) && p->gz >= 1 && p->gy >= 1 && p->gx >= 1,
              PGB_ERR_INVALID, "%s: brick extents must be powers of two", who);
  const int64_t cells = static_cast<int64_t>(p->bz) * p->by * p->bx;
  PGB_REQUIRE(cells <= 4096, PGB_ERR_RANGE, "%s: brick of %lld cells exceeds 4096", who, (long long)cells);
  PGB_REQUIRE(p->nbz == (p->gz + p->bz - 1) / p->bz && p->nby == (p->gy + p->by - 1) / p->by &&
                  p->nbx == (p->gx + p->bx - 1) / p->bx,
              PGB_ERR_INVALID, "%s: brick counts do not match the grid", who);
  PGB_REQUIRE(p->n_cta >= 0 && p->n_cta <= 65535 && p->sub_cap >= 1 && p->sub_cap <= kT6, PGB_ERR_INVALID,
              "%s: invalid CTA count or sub-chunk capacity (1..%d)", who, kT6);
  PGB_REQUIRE(p->n_cta == 0 || (p->cta_ptr && p->sd && p->si && p->uniq && p->meta && p->w), PGB_ERR_INVALID,
              "%s: null plan arrays", who);
  int lbx = 0, lby = 0;
  while ((1 << lbx) < p->bx) ++lbx;
  while ((1 << lby) < p->by) ++lby;
  g = Geom6{p->gz, p->gy, p->gx, p->bz, p->by, p->bx, lbx, lby, p->nbz, p->nby, p->nbx};
  return PGB_OK;
}

}  // namespace pgb

using namespace pgb;

extern "C" {

size_t pgb_grog_v6_smem_bytes(int64_t C, int64_t cells, int64_t n_inner, int64_t n_outer, int64_t sub_cap) {
  if (C < 1 || C > 16 || cells < 1 || cells > 4096 || n_inner < 1 || n_inner > 65535 || n_outer < 1 ||
      n_outer > 65535 || sub_cap < 1 || sub_cap > kT6)
    return ~static_cast<size_t>(0);
  const size_t a = v6_smem_c(C, static_cast<int>(cells), n_inner, n_outer, sub_cap, true);
  const size_t b = v6_smem_c(C, static_cast<int>(cells), n_inner, n_outer, sub_cap, false);
  return a > b ? a : b;
}

int pgb_grog_grid_v6(const void* data, int64_t N, void* grid, int64_t G, const void* inner_lc, int64_t n_inner,
                     const void* outer_lc, int64_t n_outer, int64_t C, int64_t B, const pgb_v6_plan* plan,
                     void* stream) {
  clear_error();
  Geom6 geom;
  int st = v6_geom(plan, geom, "grog_grid_v6");
  if (st) return st;
  PGB_REQUIRE(C >= 1 && C <= 16, PGB_ERR_UNSUPPORTED, "grog_grid_v6: ncoils must be 1..16, got %lld",
              (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 && n_inner <= 65535 &&
                  n_outer >= 1 && n_outer <= 65535,
              PGB_ERR_RANGE, "grog_grid_v6: invalid N/B/table sizes");
  PGB_REQUIRE(n_outer == 1 || outer_lc != nullptr, PGB_ERR_INVALID, "grog_grid_v6: null outer table");
  PGB_REQUIRE(G == static_cast<int64_t>(plan->gz) * plan->gy * plan->gx, PGB_ERR_INVALID,
              "grog_grid_v6: G does not match the plan grid");
  if (B == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(grid && inner_lc && (data || N == 0), PGB_ERR_INVALID, "grog_grid_v6: null pointer");
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = v6_smem_c(C, cells, n_inner, n_outer, plan->sub_cap, true);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "grog_grid_v6: table + tile + staging need %zu B of shared memory", smem);
  cudaStream_t s = as_stream(stream);
  if (plan->n_zero_bricks > 0) {
    PGB_REQUIRE(plan->zero_bricks != nullptr, PGB_ERR_INVALID, "grog_grid_v6: null zero-brick list");
    const int64_t tot = static_cast<int64_t>(plan->n_zero_bricks) * cells;
    zero_bricks_v6<<<grid_for(tot, 256, 148 * 16), 256, 0, s>>>(static_cast<float2*>(grid), G, static_cast<int>(C),
                                                               static_cast<int>(B), plan->zero_bricks,
                                                               plan->n_zero_bricks, geom);
    PGB_LAUNCH_CHECK("grog_grid_v6(zero bricks)");
  }
  if (plan->n_cta == 0) return PGB_OK;
  const bool has_outer = n_outer > 1;
  dim3 grd(plan->n_cta, static_cast<unsigned>(B));
  switch (C) {
#define X(CC)                                                                                               \
  case CC: {                                                                                                \
    auto k = has_outer ? grog_grid_v6_kernel<CC, true> : grog_grid_v6_kernel<CC, false>;                    \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                        \
    k<<<grd, kT6, smem, s>>>(static_cast<const float2*>(data), N, static_cast<float2*>(grid), G,             \
                             static_cast<const float2*>(inner_lc), static_cast<int>(n_inner),               \
                             static_cast<const float2*>(outer_lc), static_cast<int>(n_outer),               \
                             reinterpret_cast<const int4*>(plan->sd), reinterpret_cast<const int2*>(plan->si), \
                             plan->cta_ptr, plan->uniq, reinterpret_cast<const int2*>(plan->meta), plan->w,  \
                             plan->sub_cap, geom);                                                          \
  } break;
    PGB6_FOR_EACH_C(X)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK("grog_grid_v6");
  return PGB_OK;
}

int pgb_grog_degrid_v6(const void* grid, int64_t G, void* out, int64_t N, const void* inner_h_lc,
                       int64_t n_inner, const void* outer_h_lc, int64_t n_outer, int64_t C, int64_t B,
                       const pgb_v6_plan* primary, const pgb_v6_plan* secondary, const int32_t* zero_src,
                       int64_t n_zero, void* stream) {
  clear_error();
  Geom6 geom;
  int st = v6_geom(primary, geom, "grog_degrid_v6");
  if (st) return st;
  if (secondary != nullptr) {
    Geom6 g2;
    st = v6_geom(secondary, g2, "grog_degrid_v6(secondary)");
    if (st) return st;
    PGB_REQUIRE(secondary->bz == primary->bz && secondary->by == primary->by && secondary->bx == primary->bx &&
                    secondary->gz == primary->gz && secondary->gy == primary->gy && secondary->gx == primary->gx,
                PGB_ERR_INVALID, "grog_degrid_v6: primary and secondary plans differ in geometry");
  }
  PGB_REQUIRE(C >= 1 && C <= 16, PGB_ERR_UNSUPPORTED, "grog_degrid_v6: ncoils must be 1..16, got %lld",
              (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 && n_inner <= 65535 &&
                  n_outer >= 1 && n_outer <= 65535 && n_zero >= 0,
              PGB_ERR_RANGE, "grog_degrid_v6: invalid N/B/table sizes");
  PGB_REQUIRE(n_outer == 1 || outer_h_lc != nullptr, PGB_ERR_INVALID, "grog_degrid_v6: null outer table");
  PGB_REQUIRE(G == static_cast<int64_t>(primary->gz) * primary->gy * primary->gx, PGB_ERR_INVALID,
              "grog_degrid_v6: G does not match the plan grid");
  if (B == 0 || N == 0) return PGB_OK;
  PGB_REQUIRE(out && inner_h_lc && (grid || G == 0), PGB_ERR_INVALID, "grog_degrid_v6: null pointer");
  cudaStream_t s = as_stream(stream);
  if (n_zero > 0) {
    PGB_REQUIRE(zero_src != nullptr, PGB_ERR_INVALID, "grog_degrid_v6: null zero list");
    zero_samples_v6<<<grid_for(n_zero * C * B, 256, 148 * 8), 256, 0, s>>>(
        static_cast<float2*>(out), N, static_cast<int>(C), static_cast<int>(B), zero_src, n_zero);
    PGB_LAUNCH_CHECK("grog_degrid_v6(zero samples)");
  }
  const bool has_outer = n_outer > 1;
  const int cells = primary->bz * primary->by * primary->bx;
  for (int pass = 0; pass < 2; ++pass) {
    const pgb_v6_plan* p = pass == 0 ? primary : secondary;
    if (p == nullptr || p->n_cta == 0) continue;
    const size_t smem = v6_smem_c(C, cells, n_inner, n_outer, p->sub_cap, false);
    PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
                "grog_degrid_v6: table + tile + staging need %zu B of shared memory", smem);
    dim3 grd(p->n_cta, static_cast<unsigned>(B));
    switch (C) {
#define X(CC)                                                                                                 \
  case CC: {                                                                                                  \
    auto k = has_outer ? (pass ? grog_degrid_v6_kernel<CC, true, true> : grog_degrid_v6_kernel<CC, true, false>) \
                       : (pass ? grog_degrid_v6_kernel<CC, false, true> : grog_degrid_v6_kernel<CC, false, false>); \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                          \
    k<<<grd, kT6, smem, s>>>(static_cast<const float2*>(grid), G, static_cast<float2*>(out), N,                \
                             static_cast<const float2*>(inner_h_lc), static_cast<int>(n_inner),               \
                             static_cast<const float2*>(outer_h_lc), static_cast<int>(n_outer),               \
                             reinterpret_cast<const int4*>(p->sd), reinterpret_cast<const int2*>(p->si),      \
                             p->cta_ptr, p->uniq, reinterpret_cast<const int2*>(p->meta), p->w, p->sub_cap,   \
                             geom);                                                                           \
  } break;
      PGB6_FOR_EACH_C(X)
#undef X
      default:
        break;
    }
    PGB_LAUNCH_CHECK("grog_degrid_v6");
  }
  return PGB_OK;
}

}  // extern "C"
