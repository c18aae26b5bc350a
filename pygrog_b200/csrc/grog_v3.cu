// grog_v3.cu -- latency-hiding fused GROG grid / degrid with a shared-memory
// shift table (whole table, or the inner factor of T = outer @ inner).
//
// Work decomposition as in grog_fused.cu (bricks of the Cartesian grid, valid
// replicas sorted by brick), plus:
//  * persistent CTAs (one per SM, 512 threads) walk their work items as one
//    flat stream of sub-chunks of kSC replicas;
//  * the metadata and the source samples of sub-chunk t+1 (t+2 for the
//    metadata) are loaded into registers by all 512 threads while sub-chunk t
//    is computed from shared memory, then parked in a double buffer: every
//    global load is independent and issued early, instead of two dependent
//    loads per replica inside one 12-lane slot;
//  * per-replica metadata is pre-split at plan time (no integer division):
//      meta = cell | inner << 11 | outer << 25
//    (cell < 2048, inner < 16384, outer < 128); bricks of at most 512 cells.
//  * forward: the outer factor is applied once per run of replicas sharing
//    (outer index, cell); adjoint: once per such run before the inner factor.
#include "common.cuh"

namespace pgb {

struct BrickGeom3 {
  int gz, gy, gx;
  int bz, by, bx;  // powers of two
  int lbx, lby;    // log2(bx), log2(by)
  int nbz, nby, nbx;
};

constexpr int kT3 = 512;
constexpr int kW3 = kT3 / 32;
constexpr int kSC = 128;  // replicas per staged sub-chunk

struct Chunk {
  int it;     // work item index (>= n_work: end of stream)
  int s, e;   // replica range of this sub-chunk
  int brick, split, item_end;
};

__device__ __forceinline__ Chunk chunk_at(const int4* __restrict__ work, int n_work, int it, int s) {
  Chunk c;
  c.it = it;
  if (it >= n_work) {
    c.s = c.e = 0;
    c.brick = c.split = c.item_end = 0;
    return c;
  }
  const int4 w = work[it];
  c.brick = w.x;
  c.split = w.w;
  c.item_end = w.z;
  c.s = s < 0 ? w.y : s;
  c.e = min(c.s + kSC, w.z);
  return c;
}

__device__ __forceinline__ Chunk chunk_next(const int4* __restrict__ work, int n_work, const Chunk& c) {
  if (c.it >= n_work) return c;
  if (c.e < c.item_end) return chunk_at(work, n_work, c.it, c.e);
  return chunk_at(work, n_work, c.it + gridDim.x, -1);
}

__device__ __forceinline__ bool cell_flat3(const BrickGeom3& g, int brick, int cl, int64_t& flat) {
  const int bxy = g.nby * g.nbx;
  const int biz = brick / bxy;
  const int rem = brick - biz * bxy;
  const int biy = rem / g.nbx;
  const int bix = rem - biy * g.nbx;
  const int lx = cl & (g.bx - 1);
  const int ly = (cl >> g.lbx) & (g.by - 1);
  const int lz = cl >> (g.lbx + g.lby);
  const int z = biz * g.bz + lz, y = biy * g.by + ly, x = bix * g.bx + lx;
  if (z >= g.gz || y >= g.gy || x >= g.gx) return false;
  flat = (static_cast<int64_t>(z) * g.gy + y) * g.gx + x;
  return true;
}

template <int C>
__device__ __forceinline__ void lds_row(const float2* __restrict__ row, float2 (&t)[C]) {
  if constexpr ((C % 2) == 0) {
    const float4* r4 = reinterpret_cast<const float4*>(row);
#pragma unroll
    for (int i = 0; i < C / 2; ++i) {
      const float4 v = r4[i];
      t[2 * i] = make_float2(v.x, v.y);
      t[2 * i + 1] = make_float2(v.z, v.w);
    }
  } else {
#pragma unroll
    for (int i = 0; i < C; ++i) t[i] = row[i];
  }
}

template <int C>
__device__ __forceinline__ void ldg_row(const float2* __restrict__ row, float2 (&t)[C]) {
  if constexpr ((C % 2) == 0) {
    const float4* r4 = reinterpret_cast<const float4*>(row);
#pragma unroll
    for (int i = 0; i < C / 2; ++i) {
      const float4 v = __ldg(r4 + i);
      t[2 * i] = make_float2(v.x, v.y);
      t[2 * i + 1] = make_float2(v.z, v.w);
    }
  } else {
#pragma unroll
    for (int i = 0; i < C; ++i) t[i] = __ldg(row + i);
  }
}

// sum_i a[i] * b[i] with four independent accumulator chains (the FFMA
// latency would otherwise serialise a 2C-deep dependency chain per output)
template <int C>
__device__ __forceinline__ float2 cdot(const float2 (&a)[C], const float2 (&b)[C]) {
  float2 acc[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) acc[q] = make_float2(0.f, 0.f);
#pragma unroll
  for (int i = 0; i < C; ++i) cfma(acc[i & 3], a[i], b[i]);
  return make_float2((acc[0].x + acc[1].x) + (acc[2].x + acc[3].x),
                     (acc[0].y + acc[1].y) + (acc[2].y + acc[3].y));
}

// brick origin (z0, y0, x0) of `brick`, decoded once per work item
struct BrickOrigin {
  int z0, y0, x0;
};
__device__ __forceinline__ BrickOrigin brick_origin(const BrickGeom3& g, int brick) {
  const int bxy = g.nby * g.nbx;
  const int biz = brick / bxy;
  const int rem = brick - biz * bxy;
  const int biy = rem / g.nbx;
  return BrickOrigin{biz * g.bz, biy * g.by, (rem - biy * g.nbx) * g.bx};
}
__device__ __forceinline__ bool cell_flat_o(const BrickGeom3& g, const BrickOrigin& o, int cl, int64_t& flat) {
  const int x = o.x0 + (cl & (g.bx - 1));
  const int y = o.y0 + ((cl >> g.lbx) & (g.by - 1));
  const int z = o.z0 + (cl >> (g.lbx + g.lby));
  if (z >= g.gz || y >= g.gy || x >= g.gx) return false;
  flat = (static_cast<int64_t>(z) * g.gy + y) * g.gx + x;
  return true;
}

// Validate and decode one replica's metadata at staging time so that the
// compute loop is branch-free: an invalid replica keeps weight 0, cell 0,
// row 0 and outer index 0 (it then adds exactly zero).
__device__ __forceinline__ void decode_meta(int src, uint32_t meta, float w, int64_t N, int cells,
                                            int n_inner, int n_outer, int C, int& o_src,
                                            uint32_t& o_ck, float& o_w, int& o_off) {
  const int cell = static_cast<int>(meta & 2047u);
  const int ii = static_cast<int>((meta >> 11) & 16383u);
  const int k = static_cast<int>(meta >> 25);
  const bool ok = src >= 0 && src < N && cell < cells && ii < n_inner && k < n_outer;
  o_src = ok ? src : -1;
  o_ck = ok ? (static_cast<uint32_t>(cell) | (static_cast<uint32_t>(k) << 16)) : 0u;
  o_w = ok ? w : 0.f;
  o_off = ok ? ii * C * C : 0;
}

// ---------------------------------------------------------------------------
// Forward
// ---------------------------------------------------------------------------
template <int C, bool OUTER>
__global__ void __launch_bounds__(kT3, 1) grog_grid_v3_kernel(
    const float2* __restrict__ data, int64_t N, float2* __restrict__ grid, int64_t G,
    const float2* __restrict__ inner, int n_inner, const float2* __restrict__ outer, int n_outer,
    const int32_t* __restrict__ rep_src, const uint32_t* __restrict__ rep_meta,
    const float* __restrict__ rep_w, const int4* __restrict__ work, int n_work, BrickGeom3 geom) {
  constexpr int S = 32 / C;
  constexpr int XPT = (C * kSC + kT3 - 1) / kT3;  // staged samples per thread
  extern __shared__ float4 smem4[];
  float2* inner_s = reinterpret_cast<float2*>(smem4);
  const int cells = geom.bz * geom.by * geom.bx;
  const int TS = cells + 1;
  float2* tile = inner_s + static_cast<int64_t>(n_inner) * C * C;
  float2* us = tile + C * TS;                 // (kW3, 32)
  float2* X = us + kW3 * 32;                  // (2, kSC, C)
  int* Msrc = reinterpret_cast<int*>(X + 2 * kSC * C);  // (2, kSC) source sample (-1: skip)
  uint32_t* Mmeta = reinterpret_cast<uint32_t*>(Msrc + 2 * kSC);  // (2, kSC) row offset | cell,k
  float* Mw = reinterpret_cast<float*>(Mmeta + 2 * kSC);         // (2, kSC) weight (0: skip)
  int* Moff = reinterpret_cast<int*>(Mw + 2 * kSC);              // (2, kSC) inner row offset

  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const float2* dat = data + static_cast<int64_t>(b) * C * N;
  float2* grd = grid + static_cast<int64_t>(b) * C * G;
  for (int64_t t = tid; t < static_cast<int64_t>(n_inner) * C * C; t += kT3) inner_s[t] = __ldg(inner + t);
  for (int t = tid; t < C * TS; t += kT3) tile[t] = make_float2(0.f, 0.f);

  const int warp = tid >> 5, lane = tid & 31;
  const int slot = lane / C;
  const int co = lane - slot * C;
  const unsigned smask = ((C == 32) ? 0xffffffffu : ((1u << C) - 1u)) << ((slot < S ? slot : 0) * C);
  float2* mysu = us + warp * 32 + slot * C;

  Chunk c0 = chunk_at(work, n_work, blockIdx.x, -1);
  Chunk c1 = chunk_next(work, n_work, c0);
  Chunk c2 = chunk_next(work, n_work, c1);

  const int n_out_eff = OUTER ? n_outer : 1;
  // prologue: meta(c0) -> buffer 0, meta(c1) -> regs, x(c0) -> buffer 0
  if (tid < kSC) {
    int a = -1, off = 0;
    uint32_t ck = 0;
    float ww = 0.f;
    if (c0.it < n_work && tid < c0.e - c0.s)
      decode_meta(__ldg(rep_src + c0.s + tid), __ldg(rep_meta + c0.s + tid), __ldg(rep_w + c0.s + tid), N,
                  cells, n_inner, n_out_eff, C, a, ck, ww, off);
    Msrc[tid] = a;
    Mmeta[tid] = ck;
    Mw[tid] = ww;
    Moff[tid] = off;
  }
  int mr_src = 0;
  uint32_t mr_meta = 0;
  float mr_w = 0.f;
  bool mr_has = false;
  if (c1.it < n_work && tid < c1.e - c1.s) {
    mr_src = __ldg(rep_src + c1.s + tid);
    mr_meta = __ldg(rep_meta + c1.s + tid);
    mr_w = __ldg(rep_w + c1.s + tid);
    mr_has = true;
  }
  __syncthreads();
  float2 xr[XPT];
  {
    const int n0 = c0.it < n_work ? c0.e - c0.s : 0;
#pragma unroll
    for (int q = 0; q < XPT; ++q) {
      const int el = tid + q * kT3;
      const int cc = el / kSC, r = el - (el / kSC) * kSC;
      xr[q] = make_float2(0.f, 0.f);
      if (cc < C && r < n0) {
        const int src = Msrc[r];
        if (src >= 0 && src < N) xr[q] = __ldg(dat + static_cast<int64_t>(cc) * N + src);
      }
    }
#pragma unroll
    for (int q = 0; q < XPT; ++q) {
      const int el = tid + q * kT3;
      const int cc = el / kSC, r = el - (el / kSC) * kSC;
      if (cc < C) X[r * C + cc] = xr[q];
    }
    if (tid < kSC) {
      int a = -1, off = 0;
      uint32_t ck = 0;
      float ww = 0.f;
      if (mr_has) decode_meta(mr_src, mr_meta, mr_w, N, cells, n_inner, n_out_eff, C, a, ck, ww, off);
      Msrc[kSC + tid] = a;
      Mmeta[kSC + tid] = ck;
      Mw[kSC + tid] = ww;
      Moff[kSC + tid] = off;
    }
  }
  __syncthreads();

  for (int t = 0; c0.it < n_work; ++t) {
    const int bf = t & 1;
    // prefetch x(c1) using meta buffer bf^1, and meta(c2) into registers
    const int n1 = c1.it < n_work ? c1.e - c1.s : 0;
#pragma unroll
    for (int q = 0; q < XPT; ++q) {
      const int el = tid + q * kT3;
      const int cc = el / kSC, r = el - (el / kSC) * kSC;
      xr[q] = make_float2(0.f, 0.f);
      if (cc < C && r < n1) {
        const int src = Msrc[(bf ^ 1) * kSC + r];
        if (src >= 0 && src < N) xr[q] = __ldg(dat + static_cast<int64_t>(cc) * N + src);
      }
    }
    const int n2 = c2.it < n_work ? c2.e - c2.s : 0;
    mr_has = tid < n2;
    if (mr_has) {
      mr_src = __ldg(rep_src + c2.s + tid);
      mr_meta = __ldg(rep_meta + c2.s + tid);
      mr_w = __ldg(rep_w + c2.s + tid);
    }

    // compute sub-chunk c0 from shared memory (branch-free per replica)
    if (slot < S) {
      const int n0 = c0.e - c0.s;
      const int gslot = warp * S + slot;
      const int nslots = kW3 * S;
      const int p0 = (n0 * gslot) / nslots;
      const int p1 = (n0 * (gslot + 1)) / nslots;
      const uint32_t* mm = Mmeta + bf * kSC;
      const float* mw = Mw + bf * kSC;
      const int* mo = Moff + bf * kSC;
      const float2* xb = X + bf * kSC * C;
      const float2* inner_lane = inner_s + co * C;
      float2* tile_lane = tile + co * TS;
      int cur_k = -1;
      float2 orow[C];
#pragma unroll
      for (int i = 0; i < C; ++i) orow[i] = make_float2(0.f, 0.f);
      for (int r = p0; r < p1; ++r) {
        const uint32_t ck = mm[r];
        const float w = mw[r];
        const int cell = static_cast<int>(ck & 0xFFFFu);
        float2 irow[C], xv[C];
        lds_row<C>(inner_lane + mo[r], irow);
        lds_row<C>(xb + r * C, xv);
        float2 u = cdot<C>(irow, xv);
        u.x *= w;
        u.y *= w;
        if constexpr (OUTER) {
          const int k = static_cast<int>(ck >> 16);
          if (k != cur_k) {
            ldg_row<C>(outer + (static_cast<int64_t>(k) * C + co) * C, orow);
            cur_k = k;
          }
          __syncwarp(smask);
          mysu[co] = u;
          __syncwarp(smask);
          float2 uv[C];
          lds_row<C>(mysu, uv);
          u = cdot<C>(orow, uv);
        }
        atomicAdd(&tile_lane[cell].x, u.x);
        atomicAdd(&tile_lane[cell].y, u.y);
      }
    }
    __syncthreads();
    const bool item_done = !(c1.it < n_work) || c1.it != c0.it;
    if (item_done) {
      const BrickOrigin org = brick_origin(geom, c0.brick);
      for (int t2 = tid; t2 < C * cells; t2 += kT3) {
        const int c = t2 / cells;
        const int cl = t2 - c * cells;
        int64_t flat;
        if (!cell_flat_o(geom, org, cl, flat)) continue;
        const float2 v = tile[c * TS + cl];
        float2* dst = grd + static_cast<int64_t>(c) * G + flat;
        if (c0.split) {
          if (v.x != 0.f || v.y != 0.f) {
            atomicAdd(&dst->x, v.x);
            atomicAdd(&dst->y, v.y);
          }
        } else {
          *dst = v;
        }
      }
      __syncthreads();
      for (int t2 = tid; t2 < C * TS; t2 += kT3) tile[t2] = make_float2(0.f, 0.f);
    }
    // park the prefetched sub-chunks
#pragma unroll
    for (int q = 0; q < XPT; ++q) {
      const int el = tid + q * kT3;
      const int cc = el / kSC, r = el - (el / kSC) * kSC;
      if (cc < C) X[(bf ^ 1) * kSC * C + r * C + cc] = xr[q];
    }
    if (tid < kSC) {
      int a = -1, off = 0;
      uint32_t ck = 0;
      float ww = 0.f;
      if (mr_has) decode_meta(mr_src, mr_meta, mr_w, N, cells, n_inner, n_out_eff, C, a, ck, ww, off);
      Msrc[bf * kSC + tid] = a;
      Mmeta[bf * kSC + tid] = ck;
      Mw[bf * kSC + tid] = ww;
      Moff[bf * kSC + tid] = off;
    }
    __syncthreads();
    c0 = c1;
    c1 = c2;
    c2 = chunk_next(work, n_work, c2);
  }
}

// ---------------------------------------------------------------------------
// Adjoint.  pass 0 stores (first valid replica of each sample), pass 1 adds.
// The tile of the next work item is fetched with cp.async into the second
// tile buffer while the current sub-chunk is computed.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc, int bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <int C>
__device__ __forceinline__ void fetch_tile_async(float2* __restrict__ tile, const float2* __restrict__ grd,
                                                 int64_t G, const BrickGeom3& geom, int brick, int cells,
                                                 int TS) {
  const BrickOrigin org = brick_origin(geom, brick);
  for (int t2 = threadIdx.x; t2 < C * cells; t2 += kT3) {
    const int c = t2 / cells;
    const int cl = t2 - c * cells;
    int64_t flat;
    const bool in = cell_flat_o(geom, org, cl, flat);
    const float2* src = in ? grd + static_cast<int64_t>(c) * G + flat : grd;
    cp_async8(tile + cl * C + c, src, in ? 8 : 0);  // cell-major; zero-fill outside the grid
  }
  cp_async_commit();
}

template <int C, bool OUTER>
__global__ void __launch_bounds__(kT3, 1) grog_degrid_v3_kernel(
    const float2* __restrict__ grid, int64_t G, float2* __restrict__ out, int64_t N,
    const float2* __restrict__ inner_h, int n_inner, const float2* __restrict__ outer_h, int n_outer,
    const int32_t* __restrict__ rep_src, const uint32_t* __restrict__ rep_meta,
    const float* __restrict__ rep_w, const int4* __restrict__ work, int n_work, BrickGeom3 geom,
    int accumulate) {
  constexpr int S = 32 / C;
  extern __shared__ float4 smem4[];
  float2* inner_s = reinterpret_cast<float2*>(smem4);
  const int cells = geom.bz * geom.by * geom.bx;
  const int TS = cells + 1;
  float2* tiles = inner_s + static_cast<int64_t>(n_inner) * C * C;  // (2, cells, C) cell-major
  float2* vs = tiles + 2 * C * TS;                                     // (kW3, 32)
  int* Msrc = reinterpret_cast<int*>(vs + kW3 * 32);
  uint32_t* Mmeta = reinterpret_cast<uint32_t*>(Msrc + 2 * kSC);
  float* Mw = reinterpret_cast<float*>(Mmeta + 2 * kSC);
  int* Moff = reinterpret_cast<int*>(Mw + 2 * kSC);
  const int n_out_eff = OUTER ? n_outer : 1;

  const int tid = threadIdx.x;
  const int b = blockIdx.y;
  const float2* grd = grid + static_cast<int64_t>(b) * C * G;
  float2* o = out + static_cast<int64_t>(b) * C * N;
  for (int64_t t = tid; t < static_cast<int64_t>(n_inner) * C * C; t += kT3) inner_s[t] = __ldg(inner_h + t);

  const int warp = tid >> 5, lane = tid & 31;
  const int slot = lane / C;
  const int ci = lane - slot * C;
  const unsigned smask = ((C == 32) ? 0xffffffffu : ((1u << C) - 1u)) << ((slot < S ? slot : 0) * C);
  float2* mysv = vs + warp * 32 + slot * C;

  Chunk c0 = chunk_at(work, n_work, blockIdx.x, -1);
  Chunk c1 = chunk_next(work, n_work, c0);
  int tb = 0;  // tile buffer of c0
  if (c0.it < n_work) {
    if (tid < kSC) {
      int a = -1, off = 0;
      uint32_t ck = 0;
      float ww = 0.f;
      if (tid < c0.e - c0.s)
        decode_meta(__ldg(rep_src + c0.s + tid), __ldg(rep_meta + c0.s + tid), __ldg(rep_w + c0.s + tid), N,
                    cells, n_inner, n_out_eff, C, a, ck, ww, off);
      Msrc[tid] = a;
      Mmeta[tid] = ck;
      Mw[tid] = ww;
      Moff[tid] = off;
    }
    fetch_tile_async<C>(tiles, grd, G, geom, c0.brick, cells, TS);
    cp_async_wait_all();
  }
  __syncthreads();

  for (int t = 0; c0.it < n_work; ++t) {
    const int bf = t & 1;
    const int n1 = c1.it < n_work ? c1.e - c1.s : 0;
    int mr_src = 0;
    uint32_t mr_meta = 0;
    float mr_w = 0.f;
    if (tid < n1) {
      mr_src = __ldg(rep_src + c1.s + tid);
      mr_meta = __ldg(rep_meta + c1.s + tid);
      mr_w = __ldg(rep_w + c1.s + tid);
    }
    const bool new_item = c1.it < n_work && c1.it != c0.it;
    if (new_item) fetch_tile_async<C>(tiles + (tb ^ 1) * C * TS, grd, G, geom, c1.brick, cells, TS);
    const float2* tile = tiles + tb * C * TS;

    if (slot < S) {
      const int n0 = c0.e - c0.s;
      const int gslot = warp * S + slot;
      const int nslots = kW3 * S;
      const int p0 = (n0 * gslot) / nslots;
      const int p1 = (n0 * (gslot + 1)) / nslots;
      const int* ms = Msrc + bf * kSC;
      const uint32_t* mm = Mmeta + bf * kSC;
      const float* mw = Mw + bf * kSC;
      const int* mo = Moff + bf * kSC;
      const float2* inner_lane = inner_s + ci * C;
      int cur_k = -1;
      float2 orow[C];
#pragma unroll
      for (int i = 0; i < C; ++i) orow[i] = make_float2(0.f, 0.f);
      for (int r = p0; r < p1; ++r) {
        const uint32_t ck = mm[r];
        const int src = ms[r];
        const float w = mw[r];
        const int cell = static_cast<int>(ck & 0xFFFFu);
        float2 gv[C];
        lds_row<C>(tile + cell * C, gv);  // cell-major tile: one broadcast vector
        if constexpr (OUTER) {
          const int k = static_cast<int>(ck >> 16);
          if (k != cur_k) {
            ldg_row<C>(outer_h + (static_cast<int64_t>(k) * C + ci) * C, orow);
            cur_k = k;
          }
          const float2 v = cdot<C>(orow, gv);
          __syncwarp(smask);
          mysv[ci] = v;
          __syncwarp(smask);
          lds_row<C>(mysv, gv);
        }
        float2 irow[C];
        lds_row<C>(inner_lane + mo[r], irow);
        const float2 y = cdot<C>(irow, gv);
        if (src >= 0) {
          float2* dst = o + static_cast<int64_t>(ci) * N + src;
          if (accumulate) {
            atomicAdd(&dst->x, w * y.x);
            atomicAdd(&dst->y, w * y.y);
          } else {
            *dst = make_float2(w * y.x, w * y.y);
          }
        }
      }
    }
    if (tid < kSC) {
      int a = -1, off = 0;
      uint32_t ck = 0;
      float ww = 0.f;
      if (tid < n1) decode_meta(mr_src, mr_meta, mr_w, N, cells, n_inner, n_out_eff, C, a, ck, ww, off);
      Msrc[(bf ^ 1) * kSC + tid] = a;
      Mmeta[(bf ^ 1) * kSC + tid] = ck;
      Mw[(bf ^ 1) * kSC + tid] = ww;
      Moff[(bf ^ 1) * kSC + tid] = off;
    }
    if (new_item) {
      cp_async_wait_all();
      tb ^= 1;
    }
    __syncthreads();
    c0 = c1;
    c1 = chunk_next(work, n_work, c1);
  }
}

#define PGB3_FOR_EACH_C(X) \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

static size_t v3_smem(int64_t C, int cells, int64_t n_inner, bool fwd) {
  // forward: table + tile + outer staging + 2 sample buffers; adjoint: table +
  // 2 tiles + staging
  size_t f2 = static_cast<size_t>(n_inner) * C * C + static_cast<size_t>(C) * (cells + 1) + kW3 * 32;
  f2 += fwd ? 2 * static_cast<size_t>(kSC) * C : static_cast<size_t>(C) * (cells + 1);
  return f2 * sizeof(float2) + 2 * kSC * (2 * sizeof(int) + sizeof(uint32_t) + sizeof(float));
}

static int v3_geom(const pgb_brick_plan* p, BrickGeom3& g, const char* who) {
  PGB_REQUIRE(p != nullptr, PGB_ERR_INVALID, "%s: null plan", who);
  auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
  PGB_REQUIRE(pow2(p->bz) && pow2(p->by) && pow2(p->bx) && p->gz >= 1 && p->gy >= 1 && p->gx >= 1,
              PGB_ERR_INVALID, "%s: brick extents must be powers of two", who);
  const int64_t cells = static_cast<int64_t>(p->bz) * p->by * p->bx;
  PGB_REQUIRE(cells <= 512, PGB_ERR_RANGE, "%s: brick of %lld cells exceeds 512", who, (long long)cells);
  PGB_REQUIRE(p->nbz == (p->gz + p->bz - 1) / p->bz && p->nby == (p->gy + p->by - 1) / p->by &&
                  p->nbx == (p->gx + p->bx - 1) / p->bx,
              PGB_ERR_INVALID, "%s: brick counts do not match the grid", who);
  PGB_REQUIRE(p->n_work >= 0, PGB_ERR_INVALID, "%s: negative work count", who);
  PGB_REQUIRE(p->n_work == 0 || (p->work && p->rep_src && p->rep_meta && p->rep_w), PGB_ERR_INVALID,
              "%s: null plan arrays", who);
  int lbx = 0, lby = 0;
  while ((1 << lbx) < p->bx) ++lbx;
  while ((1 << lby) < p->by) ++lby;
  g = BrickGeom3{p->gz, p->gy, p->gx, p->bz, p->by, p->bx, lbx, lby, p->nbz, p->nby, p->nbx};
  return PGB_OK;
}

// zero the bricks accumulated by several chunks (same as grog_fused.cu)
__global__ void zero_bricks_v3(float2* __restrict__ grid, int64_t G, int C, int B,
                               const int32_t* __restrict__ bricks, int n_bricks, BrickGeom3 geom) {
  const int cells = geom.bz * geom.by * geom.bx;
  const int64_t total = static_cast<int64_t>(n_bricks) * cells;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / cells);
    const int cl = static_cast<int>(t - static_cast<int64_t>(i) * cells);
    int64_t flat;
    if (!cell_flat3(geom, bricks[i], cl, flat)) continue;
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < C; ++c) grid[(static_cast<int64_t>(b) * C + c) * G + flat] = make_float2(0.f, 0.f);
  }
}

__global__ void zero_samples_v3(float2* __restrict__ out, int64_t N, int C, int B,
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

}  // namespace pgb

using namespace pgb;

extern "C" {

size_t pgb_grog_v3_smem_bytes(int64_t C, int64_t cells, int64_t n_inner, int forward) {
  return v3_smem(C, static_cast<int>(cells), n_inner, forward != 0);
}

int pgb_grog_grid_v3(const void* data, int64_t N, void* grid, int64_t G, const void* inner,
                     int64_t n_inner, const void* outer, int64_t n_outer, int64_t C, int64_t B,
                     const pgb_brick_plan* plan, void* stream) {
  clear_error();
  BrickGeom3 geom;
  int st = v3_geom(plan, geom, "grog_grid_v3");
  if (st) return st;
  PGB_REQUIRE(C >= 1 && C <= 16, PGB_ERR_UNSUPPORTED, "grog_grid_v3: ncoils must be 1..16, got %lld",
              (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 &&
                  n_inner <= 16384 && n_outer >= 1 && n_outer <= 128,
              PGB_ERR_RANGE, "grog_grid_v3: invalid N/B/table sizes");
  PGB_REQUIRE(n_outer == 1 || outer != nullptr, PGB_ERR_INVALID, "grog_grid_v3: null outer table");
  PGB_REQUIRE(G == static_cast<int64_t>(plan->gz) * plan->gy * plan->gx, PGB_ERR_INVALID,
              "grog_grid_v3: G does not match the plan grid");
  if (B == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(grid && inner && (data || N == 0), PGB_ERR_INVALID, "grog_grid_v3: null pointer");
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = v3_smem(C, cells, n_inner, true);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "grog_grid_v3: table + tile + staging need %zu B of shared memory", smem);
  cudaStream_t s = as_stream(stream);
  if (plan->n_split_bricks > 0) {
    PGB_REQUIRE(plan->split_bricks != nullptr, PGB_ERR_INVALID, "grog_grid_v3: null split list");
    const int64_t tot = static_cast<int64_t>(plan->n_split_bricks) * cells;
    zero_bricks_v3<<<grid_for(tot, 256, 148 * 16), 256, 0, s>>>(static_cast<float2*>(grid), G,
                                                               static_cast<int>(C), static_cast<int>(B),
                                                               plan->split_bricks, plan->n_split_bricks, geom);
    PGB_LAUNCH_CHECK("grog_grid_v3(zero split bricks)");
  }
  if (plan->n_work == 0) return PGB_OK;
  const int nblk = plan->n_work < kNumSMs ? plan->n_work : kNumSMs;
  dim3 grd(nblk, static_cast<unsigned>(B));
  const bool has_outer = n_outer > 1;
  switch (C) {
#define X(CC)                                                                                       \
  case CC: {                                                                                        \
    auto k = has_outer ? grog_grid_v3_kernel<CC, true> : grog_grid_v3_kernel<CC, false>;            \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                \
    k<<<grd, kT3, smem, s>>>(static_cast<const float2*>(data), N, static_cast<float2*>(grid), G,    \
                             static_cast<const float2*>(inner), static_cast<int>(n_inner),          \
                             static_cast<const float2*>(outer), static_cast<int>(n_outer),          \
                             plan->rep_src, plan->rep_meta, plan->rep_w,                            \
                             reinterpret_cast<const int4*>(plan->work), plan->n_work, geom);        \
  } break;
    PGB3_FOR_EACH_C(X)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK("grog_grid_v3");
  return PGB_OK;
}

int pgb_grog_degrid_v3(const void* grid, int64_t G, void* out, int64_t N, const void* inner_h,
                       int64_t n_inner, const void* outer_h, int64_t n_outer, int64_t C, int64_t B,
                       const pgb_brick_plan* primary, const pgb_brick_plan* secondary,
                       const int32_t* zero_src, int64_t n_zero, void* stream) {
  clear_error();
  BrickGeom3 geom;
  int st = v3_geom(primary, geom, "grog_degrid_v3");
  if (st) return st;
  if (secondary != nullptr) {
    BrickGeom3 g2;
    st = v3_geom(secondary, g2, "grog_degrid_v3(secondary)");
    if (st) return st;
  }
  PGB_REQUIRE(C >= 1 && C <= 16, PGB_ERR_UNSUPPORTED, "grog_degrid_v3: ncoils must be 1..16, got %lld",
              (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 &&
                  n_inner <= 16384 && n_outer >= 1 && n_outer <= 128 && n_zero >= 0,
              PGB_ERR_RANGE, "grog_degrid_v3: invalid N/B/table sizes");
  PGB_REQUIRE(n_outer == 1 || outer_h != nullptr, PGB_ERR_INVALID, "grog_degrid_v3: null outer table");
  PGB_REQUIRE(G == static_cast<int64_t>(primary->gz) * primary->gy * primary->gx, PGB_ERR_INVALID,
              "grog_degrid_v3: G does not match the plan grid");
  if (B == 0 || N == 0) return PGB_OK;
  PGB_REQUIRE(out && inner_h && (grid || G == 0), PGB_ERR_INVALID, "grog_degrid_v3: null pointer");
  const int cells = primary->bz * primary->by * primary->bx;
  const size_t smem = v3_smem(C, cells, n_inner, false);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "grog_degrid_v3: table + tile need %zu B of shared memory", smem);
  cudaStream_t s = as_stream(stream);
  if (n_zero > 0) {
    PGB_REQUIRE(zero_src != nullptr, PGB_ERR_INVALID, "grog_degrid_v3: null zero list");
    zero_samples_v3<<<grid_for(n_zero * C * B, 256, 148 * 8), 256, 0, s>>>(
        static_cast<float2*>(out), N, static_cast<int>(C), static_cast<int>(B), zero_src, n_zero);
    PGB_LAUNCH_CHECK("grog_degrid_v3(zero samples)");
  }
  const bool has_outer = n_outer > 1;
  for (int pass = 0; pass < 2; ++pass) {
    const pgb_brick_plan* p = pass == 0 ? primary : secondary;
    if (p == nullptr || p->n_work == 0) continue;
    const int nblk = p->n_work < kNumSMs ? p->n_work : kNumSMs;
    dim3 grd(nblk, static_cast<unsigned>(B));
    switch (C) {
#define X(CC)                                                                                       \
  case CC: {                                                                                        \
    auto k = has_outer ? grog_degrid_v3_kernel<CC, true> : grog_degrid_v3_kernel<CC, false>;        \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);                \
    k<<<grd, kT3, smem, s>>>(static_cast<const float2*>(grid), G, static_cast<float2*>(out), N,     \
                             static_cast<const float2*>(inner_h), static_cast<int>(n_inner),        \
                             static_cast<const float2*>(outer_h), static_cast<int>(n_outer),        \
                             p->rep_src, p->rep_meta, p->rep_w,                                     \
                             reinterpret_cast<const int4*>(p->work), p->n_work, geom, pass);        \
  } break;
      PGB3_FOR_EACH_C(X)
#undef X
      default:
        break;
    }
    PGB_LAUNCH_CHECK("grog_degrid_v3");
  }
  return PGB_OK;
}

}  // extern "C"
