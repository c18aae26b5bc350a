// grog_fused.cu -- fused GROG gridding (interpolate + weight + scatter), its
// adjoint (gather + conjugate-transposed GRAPPA shift), and the replica
// expansion behind GrogInterpolator.interpolate().
//
// Reference path replaced: calib/_grog.py:668-695 (_sparse_full_single:
// replicate, ext.grog_interpolate, copy back) and calib/_grog.py:736-902
// (_grid_kspace: pre_weights multiply, per-coil scatter_add).  The reference
// makes ~5 full passes over N*kw*C samples plus one scatter per coil; here
// one kernel reads each source sample once and writes each grid cell once.
//
// Layout (all complex64, coil-major exactly as the reference API):
//   data (B, C, N)   source samples        grid (B, C, G)   Cartesian grid
//   table (K, C, C)  GRAPPA shift operators, row = output coil.
// Work decomposition: the grid is tiled into bricks of (bz,by,bx) cells.
// Valid replicas are pre-sorted by (brick, cell) at plan time.  One CTA
// owns one brick (or one chunk of a hot brick): it accumulates the brick
// in shared memory as a (C, cells) tile and writes it out once, row by
// row, so every grid cell is written exactly once with coalesced stores.
// Lanes are grouped in "slots" of C lanes: lane co of a slot computes output
// coil co of one replica, reading row co of the shift operator with 16-byte
// loads.  Each slot walks a contiguous run of the sorted replicas and keeps
// a running sum while the target cell does not change, so hot cells (radial
// DC) cost one shared-memory atomic per run instead of one per replica.
#include "common.cuh"

namespace pgb {

struct BrickGeom {
  int gz, gy, gx;
  int bz, by, bx;
  int nbz, nby, nbx;
};

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ bool brick_cell_to_flat(const BrickGeom& g, int brick, int cl,
                                                   int64_t& flat) {
  const int bxy = g.nby * g.nbx;
  const int biz = brick / bxy;
  const int rem = brick - biz * bxy;
  const int biy = rem / g.nbx;
  const int bix = rem - biy * g.nbx;
  const int byx = g.by * g.bx;
  const int lz = cl / byx;
  const int r2 = cl - lz * byx;
  const int ly = r2 / g.bx;
  const int lx = r2 - ly * g.bx;
  const int z = biz * g.bz + lz, y = biy * g.by + ly, x = bix * g.bx + lx;
  if (z >= g.gz || y >= g.gy || x >= g.gx) return false;
  flat = (static_cast<int64_t>(z) * g.gy + y) * g.gx + x;
  return true;
}

// Load C complex values of one table row into registers (16-byte loads when
// the row is 16-byte aligned, i.e. C even).
template <int C>
__device__ __forceinline__ void load_row(const float2* __restrict__ row, float2 (&t)[C]) {
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

// ---------------------------------------------------------------------------
// Forward: grid[b, :, cell] = sum_r w_r * T[e_r] @ data[b, :, src_r]
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(kThreads) grog_grid_kernel(
    const float2* __restrict__ data, int64_t N, float2* __restrict__ grid, int64_t G,
    const float2* __restrict__ table, int64_t K, const int32_t* __restrict__ rep_src,
    const uint32_t* __restrict__ rep_meta, const float* __restrict__ rep_w,
    const int4* __restrict__ work, BrickGeom geom) {
  constexpr int S = 32 / C;  // slots per warp
  extern __shared__ float2 smem[];
  const int cells = geom.bz * geom.by * geom.bx;
  const int TS = cells + 1;  // padded tile row stride (bank spread)
  float2* tile = smem;                     // (C, TS)
  float2* sx = smem + C * TS;              // (kWarps, 32) staged source samples
  const int4 item = work[blockIdx.x];
  const int brick = item.x, begin = item.y, end = item.z, split = item.w;
  const int b = blockIdx.y;
  const float2* dat = data + static_cast<int64_t>(b) * C * N;
  float2* grd = grid + static_cast<int64_t>(b) * C * G;

  for (int t = threadIdx.x; t < C * TS; t += kThreads) tile[t] = make_float2(0.f, 0.f);
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / C;
  const int co = lane - slot * C;
  if (end > begin && slot < S) {
    const unsigned smask = ((C == 32) ? 0xffffffffu : ((1u << C) - 1u)) << (slot * C);
    const int gslot = warp * S + slot;
    const int nslots = kWarps * S;
    const int len = end - begin;
    const int p0 = begin + static_cast<int>((static_cast<int64_t>(len) * gslot) / nslots);
    const int p1 = begin + static_cast<int>((static_cast<int64_t>(len) * (gslot + 1)) / nslots);
    float2* mysx = sx + warp * 32 + slot * C;
    int cur = -1;
    float2 acc = make_float2(0.f, 0.f);
    for (int r = p0; r < p1; ++r) {
      const int src = __ldg(rep_src + r);
      const uint32_t meta = __ldg(rep_meta + r);
      const float w = __ldg(rep_w + r);
      const int e = static_cast<int>(meta & 0xFFFFFu);
      const int cell = static_cast<int>(meta >> 20);
      const bool ok = src >= 0 && src < N && e < K && cell < cells;
      float2 xo = make_float2(0.f, 0.f);
      if (ok) xo = __ldg(dat + static_cast<int64_t>(co) * N + src);
      __syncwarp(smask);
      mysx[co] = xo;
      __syncwarp(smask);
      if (!ok) continue;
      float2 trow[C];
      load_row<C>(table + (static_cast<int64_t>(e) * C + co) * C, trow);
      float2 y = make_float2(0.f, 0.f);
#pragma unroll
      for (int ci = 0; ci < C; ++ci) cfma(y, trow[ci], mysx[ci]);
      if (cell != cur) {
        if (cur >= 0) {
          atomicAdd(&tile[co * TS + cur].x, acc.x);
          atomicAdd(&tile[co * TS + cur].y, acc.y);
        }
        cur = cell;
        acc = make_float2(0.f, 0.f);
      }
      acc.x = fmaf(w, y.x, acc.x);
      acc.y = fmaf(w, y.y, acc.y);
    }
    if (cur >= 0) {
      atomicAdd(&tile[co * TS + cur].x, acc.x);
      atomicAdd(&tile[co * TS + cur].y, acc.y);
    }
  }
  __syncthreads();

  // Write the brick: row-major cells per coil, coalesced along x.
  for (int t = threadIdx.x; t < C * cells; t += kThreads) {
    const int c = t / cells;
    const int cl = t - c * cells;
    int64_t flat;
    if (!brick_cell_to_flat(geom, brick, cl, flat)) continue;
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
}

// Zero the bricks that are written by several chunks (accumulated atomically).
__global__ void zero_bricks_kernel(float2* __restrict__ grid, int64_t G, int C, int B,
                                   const int32_t* __restrict__ bricks, int n_bricks,
                                   BrickGeom geom) {
  const int cells = geom.bz * geom.by * geom.bx;
  const int64_t total = static_cast<int64_t>(n_bricks) * cells;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / cells);
    const int cl = static_cast<int>(t - static_cast<int64_t>(i) * cells);
    int64_t flat;
    if (!brick_cell_to_flat(geom, bricks[i], cl, flat)) continue;
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < C; ++c)
        grid[(static_cast<int64_t>(b) * C + c) * G + flat] = make_float2(0.f, 0.f);
  }
}

// ---------------------------------------------------------------------------
// Adjoint: out[b, :, src_r] (+)= w_r * T[e_r]^H @ grid[b, :, cell_r]
// table_h holds T^H so that lane ci reads a contiguous row.
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(kThreads) grog_degrid_kernel(
    const float2* __restrict__ grid, int64_t G, float2* __restrict__ out, int64_t N,
    const float2* __restrict__ table_h, int64_t K, const int32_t* __restrict__ rep_src,
    const uint32_t* __restrict__ rep_meta, const float* __restrict__ rep_w,
    const int4* __restrict__ work, BrickGeom geom, int accumulate) {
  constexpr int S = 32 / C;
  extern __shared__ float2 smem[];
  const int cells = geom.bz * geom.by * geom.bx;
  const int TS = cells + 1;
  float2* tile = smem;
  const int4 item = work[blockIdx.x];
  const int brick = item.x, begin = item.y, end = item.z;
  if (end <= begin) return;  // no replicas: nothing reads this brick
  const int b = blockIdx.y;
  const float2* grd = grid + static_cast<int64_t>(b) * C * G;
  float2* o = out + static_cast<int64_t>(b) * C * N;

  for (int t = threadIdx.x; t < C * cells; t += kThreads) {
    const int c = t / cells;
    const int cl = t - c * cells;
    int64_t flat;
    float2 v = make_float2(0.f, 0.f);
    if (brick_cell_to_flat(geom, brick, cl, flat)) v = grd[static_cast<int64_t>(c) * G + flat];
    tile[c * TS + cl] = v;
  }
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / C;
  const int ci = lane - slot * C;
  if (slot >= S) return;
  const int gslot = warp * S + slot;
  const int nslots = kWarps * S;
  const int len = end - begin;
  const int p0 = begin + static_cast<int>((static_cast<int64_t>(len) * gslot) / nslots);
  const int p1 = begin + static_cast<int>((static_cast<int64_t>(len) * (gslot + 1)) / nslots);
  for (int r = p0; r < p1; ++r) {
    const int src = __ldg(rep_src + r);
    const uint32_t meta = __ldg(rep_meta + r);
    const float w = __ldg(rep_w + r);
    const int e = static_cast<int>(meta & 0xFFFFFu);
    const int cell = static_cast<int>(meta >> 20);
    if (!(src >= 0 && src < N && e < K && cell < cells)) continue;
    float2 trow[C];
    load_row<C>(table_h + (static_cast<int64_t>(e) * C + ci) * C, trow);
    float2 y = make_float2(0.f, 0.f);
#pragma unroll
    for (int co = 0; co < C; ++co) cfma(y, trow[co], tile[co * TS + cell]);
    const float2 v = make_float2(w * y.x, w * y.y);
    float2* dst = o + static_cast<int64_t>(ci) * N + src;
    if (accumulate) {
      atomicAdd(&dst->x, v.x);
      atomicAdd(&dst->y, v.y);
    } else {
      *dst = v;
    }
  }
}

__global__ void zero_samples_kernel(float2* __restrict__ out, int64_t N, int C, int B,
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

// ---------------------------------------------------------------------------
// Replica expansion: out[b, co, n*kw + j] = T[idx[n*kw+j]] @ data[b, :, n]
// A slot handles one source sample and all of its kw replicas; results are
// staged in shared memory per block and written out coalesced per coil.
// ---------------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(kThreads) grog_expand_kernel(
    const float2* __restrict__ data, int64_t N, int kw, const int64_t* __restrict__ idx,
    const float2* __restrict__ table, int64_t K, float2* __restrict__ out) {
  constexpr int S = 32 / C;
  constexpr int SPB = kWarps * S;  // samples per block-iteration
  extern __shared__ float2 smem[];
  float2* stage = smem;                       // (C, SPB*kw)
  float2* sx = smem + static_cast<int64_t>(C) * SPB * kw;  // (kWarps, 32)
  const int b = blockIdx.y;
  const float2* dat = data + static_cast<int64_t>(b) * C * N;
  float2* o = out + static_cast<int64_t>(b) * C * N * kw;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = lane / C;
  const int co = lane - slot * C;
  const int RPB = SPB * kw;
  for (int64_t n0 = static_cast<int64_t>(blockIdx.x) * SPB; n0 < N;
       n0 += static_cast<int64_t>(gridDim.x) * SPB) {
    if (slot < S) {
      const unsigned smask = ((C == 32) ? 0xffffffffu : ((1u << C) - 1u)) << (slot * C);
      const int ls = warp * S + slot;
      const int64_t n = n0 + ls;
      float2* mysx = sx + warp * 32 + slot * C;
      float2 xo = make_float2(0.f, 0.f);
      if (n < N) xo = __ldg(dat + static_cast<int64_t>(co) * N + n);
      __syncwarp(smask);
      mysx[co] = xo;
      __syncwarp(smask);
      if (n < N) {
        for (int j = 0; j < kw; ++j) {
          const int64_t e = idx[n * kw + j];
          float2 y = make_float2(0.f, 0.f);
          if (e >= 0 && e < K) {
            float2 trow[C];
            load_row<C>(table + (e * C + co) * C, trow);
#pragma unroll
            for (int ci = 0; ci < C; ++ci) cfma(y, trow[ci], mysx[ci]);
          }
          stage[co * RPB + ls * kw + j] = y;
        }
      }
    }
    __syncthreads();
    const int64_t valid_s = (N - n0) < SPB ? (N - n0) : SPB;
    const int nrep = static_cast<int>(valid_s) * kw;
    for (int t = threadIdx.x; t < C * nrep; t += kThreads) {
      const int c = t / nrep;
      const int rr = t - c * nrep;
      o[static_cast<int64_t>(c) * N * kw + n0 * kw + rr] = stage[c * RPB + rr];
    }
    __syncthreads();
  }
}

#define PGB_FOR_EACH_C(X) \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) \
  X(17) X(18) X(19) X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32)

static int check_geom(const pgb_brick_plan* p, BrickGeom& g, const char* who) {
  PGB_REQUIRE(p != nullptr, PGB_ERR_INVALID, "%s: null plan", who);
  PGB_REQUIRE(p->bz >= 1 && p->by >= 1 && p->bx >= 1 && p->gz >= 1 && p->gy >= 1 && p->gx >= 1,
              PGB_ERR_INVALID, "%s: invalid brick geometry", who);
  const int64_t cells = static_cast<int64_t>(p->bz) * p->by * p->bx;
  PGB_REQUIRE(cells <= 4096, PGB_ERR_RANGE, "%s: brick of %lld cells exceeds 4096", who,
              (long long)cells);
  PGB_REQUIRE(p->nbz == (p->gz + p->bz - 1) / p->bz && p->nby == (p->gy + p->by - 1) / p->by &&
                  p->nbx == (p->gx + p->bx - 1) / p->bx,
              PGB_ERR_INVALID, "%s: brick counts do not match the grid", who);
  PGB_REQUIRE(p->n_work >= 0, PGB_ERR_INVALID, "%s: negative work count", who);
  PGB_REQUIRE(p->n_work == 0 || (p->work && p->rep_src && p->rep_meta && p->rep_w),
              PGB_ERR_INVALID, "%s: null plan arrays", who);
  g = BrickGeom{p->gz, p->gy, p->gx, p->bz, p->by, p->bx, p->nbz, p->nby, p->nbx};
  return PGB_OK;
}


}  // namespace pgb

using namespace pgb;

extern "C" {

int pgb_grog_grid(const void* data, int64_t N, void* grid, int64_t G, const void* table, int64_t K,
                  int64_t C, int64_t B, const pgb_brick_plan* plan, void* stream) {
  clear_error();
  BrickGeom geom;
  int st = check_geom(plan, geom, "grog_grid");
  if (st) return st;
  PGB_REQUIRE(C >= 1 && C <= 32, PGB_ERR_UNSUPPORTED, "grog_grid: ncoils must be 1..32, got %lld",
              (long long)C);
  PGB_REQUIRE(N >= 0 && B >= 0 && K >= 1 && K <= (1 << 20), PGB_ERR_RANGE,
              "grog_grid: invalid N/B/K (K must be <= 2^20)");
  PGB_REQUIRE(G == static_cast<int64_t>(plan->gz) * plan->gy * plan->gx, PGB_ERR_INVALID,
              "grog_grid: G does not match the plan grid");
  PGB_REQUIRE(N < (int64_t(1) << 31), PGB_ERR_RANGE, "grog_grid: N must be < 2^31");
  if (B == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(grid && table && (data || N == 0), PGB_ERR_INVALID, "grog_grid: null pointer");
  PGB_REQUIRE(B <= 65535, PGB_ERR_RANGE, "grog_grid: batch must be <= 65535");
  cudaStream_t s = as_stream(stream);
  if (plan->n_split_bricks > 0) {
    PGB_REQUIRE(plan->split_bricks != nullptr, PGB_ERR_INVALID, "grog_grid: null split list");
    const int64_t tot = static_cast<int64_t>(plan->n_split_bricks) * plan->bz * plan->by * plan->bx;
    zero_bricks_kernel<<<grid_for(tot, 256, 148 * 16), 256, 0, s>>>(
        static_cast<float2*>(grid), G, static_cast<int>(C), static_cast<int>(B),
        plan->split_bricks, plan->n_split_bricks, geom);
    PGB_LAUNCH_CHECK("grog_grid(zero split bricks)");
  }
  if (plan->n_work == 0) return PGB_OK;
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = (static_cast<size_t>(C) * (cells + 1) + kWarps * 32) * sizeof(float2);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED, "grog_grid: tile needs %zu B shared memory",
              smem);
  dim3 grd(plan->n_work, static_cast<unsigned>(B));
  switch (C) {
#define X(CC)                                                                              \
  case CC: {                                                                               \
    auto k = grog_grid_kernel<CC>;                                                         \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);       \
    k<<<grd, kThreads, smem, s>>>(static_cast<const float2*>(data), N,                     \
                                  static_cast<float2*>(grid), G,                           \
                                  static_cast<const float2*>(table), K, plan->rep_src,     \
                                  plan->rep_meta, plan->rep_w,                             \
                                  reinterpret_cast<const int4*>(plan->work), geom);        \
  } break;
    PGB_FOR_EACH_C(X)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK("grog_grid");
  return PGB_OK;
}

int pgb_grog_degrid(const void* grid, int64_t G, void* out, int64_t N, const void* table_h,
                    int64_t K, int64_t C, int64_t B, const pgb_brick_plan* plan, int accumulate,
                    const int32_t* zero_src, int64_t n_zero, void* stream) {
  clear_error();
  BrickGeom geom;
  int st = check_geom(plan, geom, "grog_degrid");
  if (st) return st;
  PGB_REQUIRE(C >= 1 && C <= 32, PGB_ERR_UNSUPPORTED,
              "grog_degrid: ncoils must be 1..32, got %lld", (long long)C);
  PGB_REQUIRE(N >= 0 && B >= 0 && K >= 1 && K <= (1 << 20) && n_zero >= 0, PGB_ERR_RANGE,
              "grog_degrid: invalid N/B/K");
  PGB_REQUIRE(G == static_cast<int64_t>(plan->gz) * plan->gy * plan->gx, PGB_ERR_INVALID,
              "grog_degrid: G does not match the plan grid");
  PGB_REQUIRE(N < (int64_t(1) << 31), PGB_ERR_RANGE, "grog_degrid: N must be < 2^31");
  if (B == 0 || N == 0) return PGB_OK;
  PGB_REQUIRE(out && table_h && (grid || G == 0), PGB_ERR_INVALID, "grog_degrid: null pointer");
  PGB_REQUIRE(B <= 65535, PGB_ERR_RANGE, "grog_degrid: batch must be <= 65535");
  cudaStream_t s = as_stream(stream);
  if (accumulate) {
    cudaError_t e = cudaMemsetAsync(out, 0, static_cast<size_t>(B * C * N) * sizeof(float2), s);
    PGB_REQUIRE(e == cudaSuccess, PGB_ERR_CUDA, "grog_degrid: memset failed: %s",
                cudaGetErrorString(e));
  } else if (n_zero > 0) {
    PGB_REQUIRE(zero_src != nullptr, PGB_ERR_INVALID, "grog_degrid: null zero list");
    zero_samples_kernel<<<grid_for(n_zero * C * B, 256, 148 * 8), 256, 0, s>>>(
        static_cast<float2*>(out), N, static_cast<int>(C), static_cast<int>(B), zero_src, n_zero);
    PGB_LAUNCH_CHECK("grog_degrid(zero samples)");
  }
  if (plan->n_work == 0) return PGB_OK;
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = static_cast<size_t>(C) * (cells + 1) * sizeof(float2);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "grog_degrid: tile needs %zu B shared memory", smem);
  dim3 grd(plan->n_work, static_cast<unsigned>(B));
  switch (C) {
#define X(CC)                                                                                 \
  case CC: {                                                                                  \
    auto k = grog_degrid_kernel<CC>;                                                          \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);          \
    k<<<grd, kThreads, smem, s>>>(static_cast<const float2*>(grid), G,                        \
                                  static_cast<float2*>(out), N,                               \
                                  static_cast<const float2*>(table_h), K, plan->rep_src,      \
                                  plan->rep_meta, plan->rep_w,                                \
                                  reinterpret_cast<const int4*>(plan->work), geom, accumulate); \
  } break;
    PGB_FOR_EACH_C(X)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK("grog_degrid");
  return PGB_OK;
}

int pgb_grog_expand(const void* data, int64_t N, int kw, const int64_t* interp_idx,
                    const void* table, int64_t K, int64_t C, int64_t B, void* out, void* stream) {
  clear_error();
  PGB_REQUIRE(C >= 1 && C <= 32, PGB_ERR_UNSUPPORTED,
              "grog_expand: ncoils must be 1..32, got %lld", (long long)C);
  PGB_REQUIRE(N >= 0 && B >= 0 && kw >= 1 && K >= 1, PGB_ERR_INVALID, "grog_expand: invalid sizes");
  if (N == 0 || B == 0) return PGB_OK;
  PGB_REQUIRE(data && interp_idx && table && out, PGB_ERR_INVALID, "grog_expand: null pointer");
  PGB_REQUIRE(B <= 65535, PGB_ERR_RANGE, "grog_expand: batch must be <= 65535");
  const int S = 32 / static_cast<int>(C);
  const int SPB = kWarps * S;
  const size_t smem = (static_cast<size_t>(C) * SPB * kw + kWarps * 32) * sizeof(float2);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "grog_expand: kw=%d too large for the staging tile", kw);
  const int64_t nblk = (N + SPB - 1) / SPB;
  dim3 grd(static_cast<unsigned>(nblk < 148 * 16 ? nblk : 148 * 16), static_cast<unsigned>(B));
  cudaStream_t s = as_stream(stream);
  switch (C) {
#define X(CC)                                                                             \
  case CC: {                                                                              \
    auto k = grog_expand_kernel<CC>;                                                      \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);      \
    k<<<grd, kThreads, smem, s>>>(static_cast<const float2*>(data), N, kw, interp_idx,    \
                                  static_cast<const float2*>(table), K,                   \
                                  static_cast<float2*>(out));                             \
  } break;
    PGB_FOR_EACH_C(X)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK("grog_expand");
  return PGB_OK;
}

}  // extern "C"
