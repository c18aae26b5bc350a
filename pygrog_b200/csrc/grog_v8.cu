// grog_v8.cu -- fused GROG grid / degrid, one lane per replica on balanced
// sub-chunk streams.
//
// Plan: the v6 plan (calib/_plan6.py) with sub-chunks of at most 256
// replicas = one replica per thread of the 256-thread CTA.  Inside a
// sub-chunk the replicas are ordered by (outer index k, inner index q, cell),
// so the eight lanes of a quarter-warp read eight consecutive inner operators
// (operator stride = an odd number of 16-byte bank quads: all eight land in
// different quads) and, mostly, one shared outer operator (broadcast): every
// 128-bit operator load of a warp costs the four wavefronts it must.  Each
// lane keeps its replica's source coils, intermediate and result in
// registers; the tables live in shared memory, row-major per operator.
//
//   forward:  y = O[k] (I[q] x_src); w y goes to the staging buffer, then one
//             owner thread per cell sums the cell's replicas (plan cell order)
//             and updates tile[:, cell] with plain loads and stores
//   adjoint:  y = I^H[q] (O^H[k] tile[cell]) result[:, slot] = w y
//
// Streams as in grog_v6.cu: every CTA walks its own list of sub-chunk
// descriptors; the next sub-chunk's sample coils (forward) are copied into a
// second coil-major staging buffer with cp.async during the current compute,
// per-lane metadata is prefetched two sub-chunks ahead in registers, and the
// adjoint loads the next brick's tile into the second tile buffer during the
// last sub-chunk of the current brick.
#include "common.cuh"

namespace pgb {

struct Geom8 {
  int gz, gy, gx;
  int bz, by, bx;
  int lbx, lby;
  int nbz, nby, nbx;
};

constexpr int kT8 = 256;
constexpr int kFirst8 = 1, kLast8 = 2, kSplit8 = 4;

template <int C>
struct Pad8 {
  static constexpr int OPS = C * C + (C % 2 == 0 ? 2 : 1);  // float2 per staged operator
};

__device__ __forceinline__ void origin8(const Geom8& g, int brick, int& z0, int& y0, int& x0) {
  const int bxy = g.nby * g.nbx;
  const int biz = brick / bxy;
  const int rem = brick - biz * bxy;
  const int biy = rem / g.nbx;
  z0 = biz * g.bz;
  y0 = biy * g.by;
  x0 = (rem - biy * g.nbx) * g.bx;
}

__device__ __forceinline__ bool flat8(const Geom8& g, int z0, int y0, int x0, int cl, int64_t& flat) {
  const int x = x0 + (cl & (g.bx - 1));
  const int y = y0 + ((cl >> g.lbx) & (g.by - 1));
  const int z = z0 + (cl >> (g.lbx + g.lby));
  if (z >= g.gz || y >= g.gy || x >= g.gx) return false;
  flat = (static_cast<int64_t>(z) * g.gy + y) * g.gx + x;
  return true;
}

__host__ __device__ constexpr int even8(int v) { return (v + 1) & ~1; }

// Shared memory in float2 units:
//   inner table | outer table | tiles[T] | staging / results (X buffers of C x sub_cap, coil-major) |
//   forward: cell-order words of the current sub-chunk (sub_cap int32)
template <int C>
struct Smem8 {
  int tin, tout, tile, tile_sz, xs, cw, total;
  __host__ __device__ Smem8(int n_inner, int n_outer, int cells, int sub_cap, bool forward) {
    tin = 0;
    tout = n_inner * Pad8<C>::OPS;
    tile = tout + (n_outer > 1 ? n_outer * Pad8<C>::OPS : 0);
    tile_sz = even8(forward ? C * (cells + 1) : cells * C);
    xs = tile + (forward ? 1 : 2) * tile_sz;
    cw = xs + (forward ? 2 : 1) * C * sub_cap;
    total = cw + (forward ? (sub_cap + 1) / 2 : 0);  // forward: cell-order words of the sub-chunk
  }
};

__device__ __forceinline__ void cp8_v8(void* smem_dst, const void* gsrc, int bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}
__device__ __forceinline__ void commit8() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait8() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Copy (n, C, C) row-major operators into the padded shared-memory layout.
template <int C, int NT>
__device__ __forceinline__ void stage_ops8(float2* __restrict__ dst, const float2* __restrict__ src, int n) {
  constexpr int per = C * C;
  for (int t = threadIdx.x; t < n * per; t += NT) {
    const int m = t / per;
    dst[m * Pad8<C>::OPS + (t - m * per)] = __ldg(src + t);
  }
}

// y = rows 0..NR-1 of M times x, M a row-major C x C operator (or the NR-row
// slice of one) in shared memory.
template <int C, int NR = C>
__device__ __forceinline__ void matvec8(const float2* __restrict__ M, const float2 (&x)[C], float2 (&y)[NR]) {
#pragma unroll
  for (int r = 0; r < NR; ++r) {
    float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
    const float2* row = M + r * C;
    if constexpr (C % 2 == 0) {
#pragma unroll
      for (int j = 0; j < C / 2; ++j) {
        const float4 v = reinterpret_cast<const float4*>(row)[j];
        cfma(a0, make_float2(v.x, v.y), x[2 * j]);
        cfma(a1, make_float2(v.z, v.w), x[2 * j + 1]);
      }
    } else {
#pragma unroll
      for (int j = 0; j < C; ++j) cfma((j & 1) ? a1 : a0, row[j], x[j]);
    }
    y[r] = make_float2(a0.x + a1.x, a0.y + a1.y);
  }
}

// Two threads per replica (lanes 2i, 2i + 1): each computed H = C / 2 rows of
// a product; returns the full vector in row order on both.
template <int C>
__device__ __forceinline__ void join_halves8(const float2 (&mine)[C / 2], int h, float2 (&full)[C]) {
#pragma unroll
  for (int i = 0; i < C / 2; ++i) {
    const float2 o = make_float2(__shfl_xor_sync(0xffffffffu, mine[i].x, 1), __shfl_xor_sync(0xffffffffu, mine[i].y, 1));
    full[i] = h ? o : mine[i];
    full[C / 2 + i] = h ? mine[i] : o;
  }
}

struct Stream8 {
  const int4* sd;
  const int2* si;
  int p, p1;
  int4 d0, d1, d2, d3;
  int2 i0, i1, i2, i3;
  __device__ __forceinline__ int4 ld_d(int q) const { return q < p1 ? __ldg(sd + q) : make_int4(0, 0, 0, 0); }
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

__device__ __forceinline__ int nsl8(int4 d, int cap) { return min(max(d.w - d.z, 0), cap); }
__device__ __forceinline__ int nrp8(int4 d, int cap) { return min(max(d.y - d.x, 0), cap); }

// This lane's replica of sub-chunk d: metadata and weight (zeros past the end).
__device__ __forceinline__ void ld_rep8(const int2* __restrict__ meta, const float* __restrict__ wts, int4 d,
                                        int cap, int t, int2& m, float& w) {
  if (t < nrp8(d, cap)) {
    m = __ldg(meta + d.x + t);
    w = __ldg(wts + d.x + t);
  } else {
    m = make_int2(-1, 0);
    w = 0.f;
  }
}

__device__ __forceinline__ int ld_uniq8(const int32_t* __restrict__ uniq, int4 d, int cap, bool valid) {
  const int t = threadIdx.x;
  return (valid && t < nsl8(d, cap)) ? __ldg(uniq + d.z + t) : -1;
}

// Stage the C coils of this thread's slot sample u into xs (coil-major, stride cap).
template <int C>
__device__ __forceinline__ void stage_x8(const float2* __restrict__ dat, int64_t N, int u, int4 d, int cap,
                                         float2* __restrict__ xs) {
  const int t = threadIdx.x;
  if (t < nsl8(d, cap)) {
    const bool ok = u >= 0 && u < N;
#pragma unroll
    for (int c = 0; c < C; ++c)
      cp8_v8(xs + c * cap + t, ok ? dat + static_cast<int64_t>(c) * N + u : dat, ok ? 8 : 0);
  }
}

template <int C, bool OUTER, int NT>
__global__ void __launch_bounds__(NT, 1) grog_grid_v8_kernel(
    const float2* __restrict__ data, int64_t N, float2* __restrict__ grid, int64_t G,
    const float2* __restrict__ inner, int n_inner, const float2* __restrict__ outer, int n_outer,
    const int4* __restrict__ sd, const int2* __restrict__ si, const int32_t* __restrict__ cta_ptr,
    const int32_t* __restrict__ uniq, const int2* __restrict__ meta, const float* __restrict__ wts,
    const int32_t* __restrict__ cword, int cap, Geom8 geom) {
  extern __shared__ float4 smem4[];
  constexpr int OPS = Pad8<C>::OPS;
  constexpr bool PAIR = NT > kT8;  // two threads per replica, H rows of each product
  constexpr int H = PAIR ? C / 2 : C;
  static_assert(!PAIR || (C % 2 == 0 && NT == 2 * kT8), "thread pairs need an even coil count");
  const int p0 = cta_ptr[blockIdx.x], p1 = cta_ptr[blockIdx.x + 1];
  if (p0 >= p1) return;  // block-uniform
  const int cells = geom.bz * geom.by * geom.bx;
  const int TS = cells + 1;
  const Smem8<C> lay(n_inner, OUTER ? n_outer : 1, cells, cap, true);
  float2* base = reinterpret_cast<float2*>(smem4);
  float2* tin = base + lay.tin;
  float2* tout = base + lay.tout;
  // tile as separate real / imaginary planes (C, TS) each
  float* tre = reinterpret_cast<float*>(base + lay.tile);
  float* tim = tre + C * TS;
  float2* xs0 = base + lay.xs;  // 2 x (C, cap): staged sample coils, then this sub-chunk's results
  int32_t* cws = reinterpret_cast<int32_t*>(base + lay.cw);
  const int b = blockIdx.y;
  const float2* dat = data + static_cast<int64_t>(b) * C * N;
  float2* grd = grid + static_cast<int64_t>(b) * C * G;
  const int tid = threadIdx.x;
  const int rr = PAIR ? tid >> 1 : tid;  // this thread's replica in the sub-chunk
  const int h = PAIR ? tid & 1 : 0;      // and which half of the rows it computes

  Stream8 st;
  st.init(sd, si, p0, p1);
  int u1 = ld_uniq8(uniq, st.d1, cap, st.p + 1 < p1);
  {
    const int u0 = ld_uniq8(uniq, st.d0, cap, true);
    stage_x8<C>(dat, N, u0, st.d0, cap, xs0);
    commit8();
  }
  int2 m0, m1;
  float w0, w1;
  ld_rep8(meta, wts, st.d0, cap, rr, m0, w0);
  ld_rep8(meta, wts, st.d1, cap, rr, m1, w1);
  auto ld_cw = [&](int4 d, bool valid) -> int32_t {
    return (valid && tid < nrp8(d, cap)) ? __ldg(cword + d.x + tid) : 0;
  };
  int32_t c0 = ld_cw(st.d0, true), c1 = ld_cw(st.d1, st.p + 1 < p1);
  stage_ops8<C, NT>(tin, inner, n_inner);
  if (OUTER) stage_ops8<C, NT>(tout, outer, n_outer);
  for (int t = tid; t < 2 * C * TS; t += NT) tre[t] = 0.f;

  int buf = 0;
  while (true) {
    const bool more = st.p + 1 < p1;
    if (more) {
      stage_x8<C>(dat, N, u1, st.d1, cap, xs0 + (buf ^ 1) * C * cap);
      commit8();
      wait8<1>();
    } else {
      wait8<0>();
    }
    // prefetch two ahead (consumed in later iterations)
    const int u2 = ld_uniq8(uniq, st.d2, cap, st.p + 2 < p1);
    int2 m2;
    float w2;
    ld_rep8(meta, wts, st.p + 2 < p1 ? st.d2 : make_int4(0, 0, 0, 0), cap, rr, m2, w2);
    const int32_t c2 = ld_cw(st.d2, st.p + 2 < p1);
    __syncthreads();  // staging buffer `buf` complete; tile zeroed
    {
      const int nr = nrp8(st.d0, cap);
      const int nu = nsl8(st.d0, cap);
      const int cell = m0.x & 0xFFFF;
      const int sl = static_cast<int>(static_cast<unsigned>(m0.x) >> 16);
      const int q = m0.y & 0xFFFF;
      const int k = static_cast<int>(static_cast<unsigned>(m0.y) >> 16);
      const bool on = m0.x >= 0 && cell < cells && sl < nu && q < n_inner && (OUTER ? k < n_outer : k == 0);
      float2* xs = xs0 + buf * C * cap;
      float2 y[H];
      if constexpr (PAIR) {
        // both threads of a pair run every step (the halves are exchanged with
        // shuffles); an idle pair works on operator 0 and slot 0, writes zeros
        const int slc = on ? sl : 0, qc = on ? q : 0, kc = on ? k : 0;
        float2 x[C];
#pragma unroll
        for (int c = 0; c < C; ++c) x[c] = xs[c * cap + slc];
        if constexpr (OUTER) {
          float2 uh[H], u[C];
          matvec8<C, H>(tin + qc * OPS + h * H * C, x, uh);
          join_halves8<C>(uh, h, u);
          matvec8<C, H>(tout + kc * OPS + h * H * C, u, y);
        } else {
          matvec8<C, H>(tin + qc * OPS + h * H * C, x, y);
        }
      } else if (on) {
        float2 x[C];
#pragma unroll
        for (int c = 0; c < C; ++c) x[c] = xs[c * cap + sl];
        if constexpr (OUTER) {
          float2 u[C];
          matvec8<C>(tin + q * OPS, x, u);
          matvec8<C, H>(tout + k * OPS, u, y);
        } else {
          matvec8<C, H>(tin + q * OPS, x, y);
        }
      }
      __syncthreads();  // every lane has read its staged coils: the buffer takes the results
      if (rr < nr) {
#pragma unroll
        for (int i = 0; i < H; ++i)
          xs[(h * H + i) * cap + rr] = on ? make_float2(w0 * y[i].x, w0 * y[i].y) : make_float2(0.f, 0.f);
      }
      if (tid < nr) cws[tid] = c0;
      __syncthreads();
      // one owner per segment (the head of at most a few entries of one cell
      // in cell order) sums the segment's results and updates the tile; only
      // segments of a cell with several add atomically
      if (tid < nr && ((c0 >> 21) & 1)) {
        const int cl = (c0 >> 9) & 4095;
        float2 acc[C];
#pragma unroll
        for (int c = 0; c < C; ++c) acc[c] = make_float2(0.f, 0.f);
        int j = tid, wj = c0;
        while (true) {
          const int pos = wj & 511;
          if (pos < nr) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
              const float2 v = xs[c * cap + pos];
              acc[c].x += v.x;
              acc[c].y += v.y;
            }
          }
          if (++j >= nr) break;
          wj = cws[j];
          if ((wj >> 21) & 1) break;
        }
        if (cl < cells) {
          if ((c0 >> 22) & 1) {
#pragma unroll
            for (int c = 0; c < C; ++c) {
              atomicAdd(tre + c * TS + cl, acc[c].x);
              atomicAdd(tim + c * TS + cl, acc[c].y);
            }
          } else {
#pragma unroll
            for (int c = 0; c < C; ++c) {
              tre[c * TS + cl] += acc[c].x;
              tim[c * TS + cl] += acc[c].y;
            }
          }
        }
      }
    }
    // every owner is done with the results (their buffer is refilled by the
    // next iteration's staging) and with the tile (flushed below)
    __syncthreads();
    if (st.i0.y & kLast8) {
      int z0, y0, x0;
      origin8(geom, st.i0.x, z0, y0, x0);
      const bool split = (st.i0.y & kSplit8) != 0;
      for (int t = tid; t < C * cells; t += NT) {
        const int c = t / cells;
        const int cl = t - c * cells;
        const float2 v = make_float2(tre[c * TS + cl], tim[c * TS + cl]);
        tre[c * TS + cl] = 0.f;  // this thread re-zeroes what it flushed
        tim[c * TS + cl] = 0.f;
        int64_t flat;
        if (!flat8(geom, z0, y0, x0, cl, flat)) continue;
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
    }
    if (!more) break;
    st.advance();
    u1 = u2;
    m0 = m1;
    w0 = w1;
    m1 = m2;
    w1 = w2;
    c0 = c1;
    c1 = c2;
    buf ^= 1;
  }
}

template <int C, bool OUTER, bool ACC, int NT>
__global__ void __launch_bounds__(NT, 1) grog_degrid_v8_kernel(
    const float2* __restrict__ grid, int64_t G, float2* __restrict__ out, int64_t N,
    const float2* __restrict__ inner_h, int n_inner, const float2* __restrict__ outer_h, int n_outer,
    const int4* __restrict__ sd, const int2* __restrict__ si, const int32_t* __restrict__ cta_ptr,
    const int32_t* __restrict__ uniq, const int2* __restrict__ meta, const float* __restrict__ wts, int cap,
    Geom8 geom) {
  extern __shared__ float4 smem4[];
  constexpr int OPS = Pad8<C>::OPS;
  constexpr bool PAIR = NT > kT8;  // two threads per replica, H rows of each product
  constexpr int H = PAIR ? C / 2 : C;
  static_assert(!PAIR || (C % 2 == 0 && NT == 2 * kT8), "thread pairs need an even coil count");
  const int p0 = cta_ptr[blockIdx.x], p1 = cta_ptr[blockIdx.x + 1];
  if (p0 >= p1) return;
  const int cells = geom.bz * geom.by * geom.bx;
  const Smem8<C> lay(n_inner, OUTER ? n_outer : 1, cells, cap, false);
  float2* base = reinterpret_cast<float2*>(smem4);
  float2* tin = base + lay.tin;
  float2* tout = base + lay.tout;
  float2* tiles = base + lay.tile;  // 2 x (cells, C) cell-major
  float2* res = base + lay.xs;      // (C, cap) per-slot results
  const int b = blockIdx.y;
  const float2* grd = grid + static_cast<int64_t>(b) * C * G;
  float2* o = out + static_cast<int64_t>(b) * C * N;
  const int tid = threadIdx.x;
  const int rr = PAIR ? tid >> 1 : tid;  // this thread's replica in the sub-chunk
  const int h = PAIR ? tid & 1 : 0;      // and which half of the rows it computes

  auto issue_tile = [&](int brick, float2* tl) {
    int z0, y0, x0;
    origin8(geom, brick, z0, y0, x0);
    for (int t = tid; t < C * cells; t += NT) {
      const int c = t / cells;
      const int cl = t - c * cells;
      int64_t flat;
      const bool in = flat8(geom, z0, y0, x0, cl, flat);
      cp8_v8(tl + cl * C + c, in ? grd + static_cast<int64_t>(c) * G + flat : grd, in ? 8 : 0);
    }
  };

  Stream8 st;
  st.init(sd, si, p0, p1);
  int par = 0;  // tile buffer of the current brick item
  issue_tile(st.i0.x, tiles);
  commit8();
  stage_ops8<C, NT>(tin, inner_h, n_inner);
  if (OUTER) stage_ops8<C, NT>(tout, outer_h, n_outer);
  for (int t = tid; t < C * cap; t += NT) res[t] = make_float2(0.f, 0.f);
  int u0 = ld_uniq8(uniq, st.d0, cap, true);
  int u1 = ld_uniq8(uniq, st.d1, cap, st.p + 1 < p1);
  int2 m0, m1;
  float w0, w1;
  ld_rep8(meta, wts, st.d0, cap, rr, m0, w0);
  ld_rep8(meta, wts, st.d1, cap, rr, m1, w1);

  while (true) {
    const bool more = st.p + 1 < p1;
    const bool last = (st.i0.y & kLast8) != 0;
    if (last && more) {  // next brick's tile into the other buffer during this compute
      issue_tile(st.i1.x, tiles + (par ^ 1) * lay.tile_sz);
      commit8();
      wait8<1>();
    } else {
      wait8<0>();
    }
    const int u2 = ld_uniq8(uniq, st.d2, cap, st.p + 2 < p1);
    int2 m2;
    float w2;
    ld_rep8(meta, wts, st.p + 2 < p1 ? st.d2 : make_int4(0, 0, 0, 0), cap, rr, m2, w2);
    __syncthreads();  // tile of this brick complete; previous results flushed and cleared
    {
      const int nu = nsl8(st.d0, cap);
      const int cell = m0.x & 0xFFFF;
      const int sl = static_cast<int>(static_cast<unsigned>(m0.x) >> 16);
      const int q = m0.y & 0xFFFF;
      const int k = static_cast<int>(static_cast<unsigned>(m0.y) >> 16);
      const bool on = m0.x >= 0 && cell < cells && sl < nu && q < n_inner && (OUTER ? k < n_outer : k == 0);
      if constexpr (PAIR) {
        // both threads of a pair run every step (the halves are exchanged with
        // shuffles); an idle pair works on cell 0 and operator 0, writes nothing
        const int cc = on ? cell : 0, qc = on ? q : 0, kc = on ? k : 0;
        const float2* gt = tiles + par * lay.tile_sz + cc * C;
        float2 g[C], r[H];
#pragma unroll
        for (int c = 0; c < C; c += 2) {
          const float4 v = *reinterpret_cast<const float4*>(gt + c);
          g[c] = make_float2(v.x, v.y);
          g[c + 1] = make_float2(v.z, v.w);
        }
        if constexpr (OUTER) {
          float2 yh[H], y[C];
          matvec8<C, H>(tout + kc * OPS + h * H * C, g, yh);
          join_halves8<C>(yh, h, y);
          matvec8<C, H>(tin + qc * OPS + h * H * C, y, r);
        } else {
          matvec8<C, H>(tin + qc * OPS + h * H * C, g, r);
        }
        if (on) {
#pragma unroll
          for (int i = 0; i < H; ++i) {
            float2* dst = res + (h * H + i) * cap + sl;
            if (ACC) {
              atomicAdd(&dst->x, w0 * r[i].x);
              atomicAdd(&dst->y, w0 * r[i].y);
            } else {
              *dst = make_float2(w0 * r[i].x, w0 * r[i].y);
            }
          }
        }
      } else if (on) {
        const float2* gt = tiles + par * lay.tile_sz + cell * C;
        float2 g[C], y[C];
        if constexpr (C % 2 == 0) {
#pragma unroll
          for (int c = 0; c < C; c += 2) {
            const float4 v = *reinterpret_cast<const float4*>(gt + c);
            g[c] = make_float2(v.x, v.y);
            g[c + 1] = make_float2(v.z, v.w);
          }
        } else {
#pragma unroll
          for (int c = 0; c < C; ++c) g[c] = gt[c];
        }
        if constexpr (OUTER) {
          matvec8<C>(tout + k * OPS, g, y);
          matvec8<C>(tin + q * OPS, y, g);
        } else {
          matvec8<C>(tin + q * OPS, g, y);
#pragma unroll
          for (int c = 0; c < C; ++c) g[c] = y[c];
        }
#pragma unroll
        for (int c = 0; c < C; ++c) {
          float2* dst = res + c * cap + sl;
          if (ACC) {
            atomicAdd(&dst->x, w0 * g[c].x);
            atomicAdd(&dst->y, w0 * g[c].y);
          } else {
            *dst = make_float2(w0 * g[c].x, w0 * g[c].y);
          }
        }
      }
    }
    __syncthreads();  // results complete; this brick's tile no longer read
    if (tid < nsl8(st.d0, cap)) {
      const bool ok = u0 >= 0 && u0 < N;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        float2* rv = res + c * cap + tid;
        const float2 v = *rv;
        if (ACC) *rv = make_float2(0.f, 0.f);  // this thread re-clears what it flushed
        if (!ok) continue;
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
    if (last) par ^= 1;
    st.advance();
    u0 = u1;
    u1 = u2;
    m0 = m1;
    w0 = w1;
    m1 = m2;
    w1 = w2;
  }
}

__global__ void zero_bricks_v8(float2* __restrict__ grid, int64_t G, int C, int B,
                               const int32_t* __restrict__ bricks, int n_bricks, Geom8 geom) {
  const int cells = geom.bz * geom.by * geom.bx;
  const int64_t total = static_cast<int64_t>(n_bricks) * cells;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / cells);
    const int cl = static_cast<int>(t - static_cast<int64_t>(i) * cells);
    int z0, y0, x0;
    origin8(geom, bricks[i], z0, y0, x0);
    int64_t flat;
    if (!flat8(geom, z0, y0, x0, cl, flat)) continue;
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < C; ++c) grid[(static_cast<int64_t>(b) * C + c) * G + flat] = make_float2(0.f, 0.f);
  }
}

__global__ void zero_samples_v8(float2* __restrict__ out, int64_t N, int C, int B,
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

#define PGB8_FOR_EACH_C(X) \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

static size_t v8_smem_c(int64_t C, int cells, int64_t n_inner, int64_t n_outer, int64_t cap, bool forward) {
  switch (C) {
#define X(CC)                                                                                              \
  case CC:                                                                                                 \
    return static_cast<size_t>(Smem8<CC>(static_cast<int>(n_inner), static_cast<int>(n_outer), cells,      \
                                         static_cast<int>(cap), forward).total) * sizeof(float2);
    PGB8_FOR_EACH_C(X)
#undef X
    default:
      return ~static_cast<size_t>(0);
  }
}

// The v8 kernels read the v6 plan; its sub-chunks must hold at most one replica
// and one staging slot per thread.
static int v8_geom(const pgb_v6_plan* p, Geom8& g, const char* who) {
  PGB_REQUIRE(p != nullptr, PGB_ERR_INVALID, "%s: null plan", who);
  auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
  PGB_REQUIRE(pow2(p->bz) && pow2(p->by) && pow2(p->bx) && p->gz >= 1 && p->gy >= 1 && p->gx >= 1,
              PGB_ERR_INVALID, "%s: brick extents must be powers of two", who);
  const int64_t cells = static_cast<int64_t>(p->bz) * p->by * p->bx;
  PGB_REQUIRE(cells <= 4096, PGB_ERR_RANGE, "%s: brick of %lld cells exceeds 4096", who, (long long)cells);
  PGB_REQUIRE(p->nbz == (p->gz + p->bz - 1) / p->bz && p->nby == (p->gy + p->by - 1) / p->by &&
                  p->nbx == (p->gx + p->bx - 1) / p->bx,
              PGB_ERR_INVALID, "%s: brick counts do not match the grid", who);
  PGB_REQUIRE(p->n_cta >= 0 && p->n_cta <= 65535 && p->sub_cap >= 1 && p->sub_cap <= kT8, PGB_ERR_INVALID,
              "%s: invalid CTA count or sub-chunk capacity (1..%d)", who, kT8);
  PGB_REQUIRE(p->n_cta == 0 || (p->cta_ptr && p->sd && p->si && p->uniq && p->meta && p->w), PGB_ERR_INVALID,
              "%s: null plan arrays", who);
  int lbx = 0, lby = 0;
  while ((1 << lbx) < p->bx) ++lbx;
  while ((1 << lby) < p->by) ++lby;
  g = Geom8{p->gz, p->gy, p->gx, p->bz, p->by, p->bx, lbx, lby, p->nbz, p->nby, p->nbx};
  return PGB_OK;
}

}  // namespace pgb

using namespace pgb;

extern "C" {

size_t pgb_grog_v8_smem_bytes(int64_t C, int64_t cells, int64_t n_inner, int64_t n_outer, int64_t sub_cap) {
  if (C < 1 || C > 16 || cells < 1 || cells > 4096 || n_inner < 1 || n_inner > 65535 || n_outer < 1 ||
      n_outer > 65535 || sub_cap < 1 || sub_cap > kT8)
    return ~static_cast<size_t>(0);
  const size_t a = v8_smem_c(C, static_cast<int>(cells), n_inner, n_outer, sub_cap, true);
  const size_t b = v8_smem_c(C, static_cast<int>(cells), n_inner, n_outer, sub_cap, false);
  return a > b ? a : b;
}

}  // extern "C"

namespace {

// `nt` threads per CTA (kT8: one thread per replica); `who` names the entry
// point in errors.
int grid_v8_launch(int nt, const char* who, const void* data, int64_t N, void* grid, int64_t G,
                   const void* inner, int64_t n_inner, const void* outer, int64_t n_outer, int64_t C, int64_t B,
                   const pgb_v6_plan* plan, void* stream) {
  Geom8 geom;
  int st = v8_geom(plan, geom, who);
  if (st) return st;
  PGB_REQUIRE(C >= 1 && C <= 16 && (nt == kT8 || C % 2 == 0), PGB_ERR_UNSUPPORTED,
              "%s: ncoils must be 1..16 (even for thread pairs), got %lld", who, (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 && n_inner <= 65535 &&
                  n_outer >= 1 && n_outer <= 65535,
              PGB_ERR_RANGE, "%s: invalid N/B/table sizes", who);
  PGB_REQUIRE(n_outer == 1 || outer != nullptr, PGB_ERR_INVALID, "%s: null outer table", who);
  PGB_REQUIRE(G == static_cast<int64_t>(plan->gz) * plan->gy * plan->gx, PGB_ERR_INVALID,
              "%s: G does not match the plan grid", who);
  if (B == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(grid && inner && (data || N == 0), PGB_ERR_INVALID, "%s: null pointer", who);
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = v8_smem_c(C, cells, n_inner, n_outer, plan->sub_cap, true);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "%s: tables + tile + staging need %zu B of shared memory", who, smem);
  cudaStream_t s = as_stream(stream);
  if (plan->n_zero_bricks > 0) {
    PGB_REQUIRE(plan->zero_bricks != nullptr, PGB_ERR_INVALID, "%s: null zero-brick list", who);
    const int64_t tot = static_cast<int64_t>(plan->n_zero_bricks) * cells;
    zero_bricks_v8<<<grid_for(tot, 256, 148 * 16), 256, 0, s>>>(static_cast<float2*>(grid), G, static_cast<int>(C),
                                                               static_cast<int>(B), plan->zero_bricks,
                                                               plan->n_zero_bricks, geom);
    PGB_LAUNCH_CHECK(who);
  }
  if (plan->n_cta == 0) return PGB_OK;
  PGB_REQUIRE(plan->cword != nullptr, PGB_ERR_INVALID, "%s: the plan has no cell order (cword)", who);
  const bool has_outer = n_outer > 1;
  dim3 grd(plan->n_cta, static_cast<unsigned>(B));
  switch (C) {
#define X(CC)                                                                                                 \
  case CC: {                                                                                                  \
    auto k = has_outer ? grog_grid_v8_kernel<CC, true, kT8> : grog_grid_v8_kernel<CC, false, kT8>;            \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                          \
    k<<<grd, nt, smem, s>>>(static_cast<const float2*>(data), N, static_cast<float2*>(grid), G,                \
                            static_cast<const float2*>(inner), static_cast<int>(n_inner),                     \
                            static_cast<const float2*>(outer), static_cast<int>(n_outer),                     \
                            reinterpret_cast<const int4*>(plan->sd), reinterpret_cast<const int2*>(plan->si),  \
                            plan->cta_ptr, plan->uniq, reinterpret_cast<const int2*>(plan->meta), plan->w,     \
                            plan->cword, plan->sub_cap, geom);                                                \
  } break;
    PGB8_FOR_EACH_C(X)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK(who);
  return PGB_OK;
}

}  // namespace

extern "C" {

int pgb_grog_grid_v8(const void* data, int64_t N, void* grid, int64_t G, const void* inner, int64_t n_inner,
                     const void* outer, int64_t n_outer, int64_t C, int64_t B, const pgb_v6_plan* plan,
                     void* stream) {
  clear_error();
  return grid_v8_launch(kT8, "grog_grid_v8", data, N, grid, G, inner, n_inner, outer, n_outer, C, B, plan, stream);
}

}  // extern "C"

namespace {

int degrid_v8_launch(int nt, const char* who, const void* grid, int64_t G, void* out, int64_t N,
                     const void* inner_h, int64_t n_inner, const void* outer_h, int64_t n_outer, int64_t C,
                     int64_t B, const pgb_v6_plan* primary, const pgb_v6_plan* secondary, const int32_t* zero_src,
                     int64_t n_zero, void* stream) {
  Geom8 geom;
  int st = v8_geom(primary, geom, who);
  if (st) return st;
  if (secondary != nullptr) {
    Geom8 g2;
    st = v8_geom(secondary, g2, who);
    if (st) return st;
    PGB_REQUIRE(secondary->bz == primary->bz && secondary->by == primary->by && secondary->bx == primary->bx &&
                    secondary->gz == primary->gz && secondary->gy == primary->gy && secondary->gx == primary->gx,
                PGB_ERR_INVALID, "%s: primary and secondary plans differ in geometry", who);
  }
  PGB_REQUIRE(C >= 1 && C <= 16 && (nt == kT8 || C % 2 == 0), PGB_ERR_UNSUPPORTED,
              "%s: ncoils must be 1..16 (even for thread pairs), got %lld", who, (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 && n_inner <= 65535 &&
                  n_outer >= 1 && n_outer <= 65535 && n_zero >= 0,
              PGB_ERR_RANGE, "%s: invalid N/B/table sizes", who);
  PGB_REQUIRE(n_outer == 1 || outer_h != nullptr, PGB_ERR_INVALID, "%s: null outer table", who);
  PGB_REQUIRE(G == static_cast<int64_t>(primary->gz) * primary->gy * primary->gx, PGB_ERR_INVALID,
              "%s: G does not match the plan grid", who);
  if (B == 0 || N == 0) return PGB_OK;
  PGB_REQUIRE(out && inner_h && (grid || G == 0), PGB_ERR_INVALID, "%s: null pointer", who);
  cudaStream_t s = as_stream(stream);
  if (n_zero > 0) {
    PGB_REQUIRE(zero_src != nullptr, PGB_ERR_INVALID, "%s: null zero list", who);
    zero_samples_v8<<<grid_for(n_zero * C * B, 256, 148 * 8), 256, 0, s>>>(
        static_cast<float2*>(out), N, static_cast<int>(C), static_cast<int>(B), zero_src, n_zero);
    PGB_LAUNCH_CHECK(who);
  }
  const bool has_outer = n_outer > 1;
  const int cells = primary->bz * primary->by * primary->bx;
  for (int pass = 0; pass < 2; ++pass) {
    const pgb_v6_plan* p = pass == 0 ? primary : secondary;
    if (p == nullptr || p->n_cta == 0) continue;
    const size_t smem = v8_smem_c(C, cells, n_inner, n_outer, p->sub_cap, false);
    PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
                "%s: tables + tiles + results need %zu B of shared memory", who, smem);
    dim3 grd(p->n_cta, static_cast<unsigned>(B));
    switch (C) {
#define X(CC)                                                                                                 \
  case CC: {                                                                                                  \
    auto k = has_outer ? (pass ? grog_degrid_v8_kernel<CC, true, true, kT8> : grog_degrid_v8_kernel<CC, true, false, kT8>) \
                       : (pass ? grog_degrid_v8_kernel<CC, false, true, kT8> : grog_degrid_v8_kernel<CC, false, false, kT8>); \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                          \
    k<<<grd, nt, smem, s>>>(static_cast<const float2*>(grid), G, static_cast<float2*>(out), N,                 \
                            static_cast<const float2*>(inner_h), static_cast<int>(n_inner),                   \
                            static_cast<const float2*>(outer_h), static_cast<int>(n_outer),                   \
                            reinterpret_cast<const int4*>(p->sd), reinterpret_cast<const int2*>(p->si),       \
                            p->cta_ptr, p->uniq, reinterpret_cast<const int2*>(p->meta), p->w, p->sub_cap,    \
                            geom);                                                                            \
  } break;
      PGB8_FOR_EACH_C(X)
#undef X
      default:
        break;
    }
    PGB_LAUNCH_CHECK(who);
  }
  return PGB_OK;
}

}  // namespace

extern "C" {

int pgb_grog_degrid_v8(const void* grid, int64_t G, void* out, int64_t N, const void* inner_h, int64_t n_inner,
                       const void* outer_h, int64_t n_outer, int64_t C, int64_t B, const pgb_v6_plan* primary,
                       const pgb_v6_plan* secondary, const int32_t* zero_src, int64_t n_zero, void* stream) {
  clear_error();
  return degrid_v8_launch(kT8, "grog_degrid_v8", grid, G, out, N, inner_h, n_inner, outer_h, n_outer, C, B, primary,
                          secondary, zero_src, n_zero, stream);
}

}  // extern "C"
