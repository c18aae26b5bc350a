// grog_v5.cu -- fused GROG grid / degrid, one lane per replica.
//
// Each lane owns one replica: it loads its own C source coils (forward) or
// the C coils of its target cell from the shared-memory tile (adjoint) into
// registers and applies the whole C x C shift operator(s) itself.  Inside
// every brick the replicas are sorted by shift-table index, so the 32 lanes
// of a warp touch only a few distinct operators: the table rows they read
// from shared memory are (near) broadcasts.  Operators are stored with a
// 16-byte pad after every C x C matrix so that different operators start in
// different bank groups.  The factored table T[e] = outer[e % n] @ inner[e/n]
// keeps both factors in shared memory.
//
// Per-replica metadata as in grog_v3.cu: meta = cell | inner << 11 | outer << 25.
#include "common.cuh"

namespace pgb {

struct Geom5 {
  int gz, gy, gx;
  int bz, by, bx;
  int lbx, lby;
  int nbz, nby, nbx;
};

constexpr int kT5 = 256;
// threads per CTA: 16 warps where the per-lane register footprint allows it
template <int C>
struct Threads5 {
  static constexpr int value = C <= 12 ? 512 : 256;
};

template <int C>
struct Pad {
  static constexpr int kStride = C * C + 2;  // float2 per padded operator (16-byte pad)
};

__device__ __forceinline__ void origin5(const Geom5& g, int brick, int& z0, int& y0, int& x0) {
  const int bxy = g.nby * g.nbx;
  const int biz = brick / bxy;
  const int rem = brick - biz * bxy;
  const int biy = rem / g.nbx;
  z0 = biz * g.bz;
  y0 = biy * g.by;
  x0 = (rem - biy * g.nbx) * g.bx;
}

__device__ __forceinline__ bool flat5(const Geom5& g, int z0, int y0, int x0, int cl, int64_t& flat) {
  const int x = x0 + (cl & (g.bx - 1));
  const int y = y0 + ((cl >> g.lbx) & (g.by - 1));
  const int z = z0 + (cl >> (g.lbx + g.lby));
  if (z >= g.gz || y >= g.gy || x >= g.gx) return false;
  flat = (static_cast<int64_t>(z) * g.gy + y) * g.gx + x;
  return true;
}

// Copy (n, C, C) operators into the padded shared-memory layout.
template <int C>
__device__ __forceinline__ void stage_ops(float2* __restrict__ dst, const float2* __restrict__ src, int n) {
  const int per = C * C;
  for (int t = threadIdx.x; t < n * per; t += blockDim.x) {
    const int m = t / per;
    dst[m * Pad<C>::kStride + (t - m * per)] = __ldg(src + t);
  }
}

// y = M x for one C x C operator in shared memory (rows of M are contiguous).
template <int C>
__device__ __forceinline__ void apply_op(const float2* __restrict__ M, const float2 (&x)[C], float2 (&y)[C]) {
#pragma unroll
  for (int co = 0; co < C; ++co) {
    float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
    const float2* row = M + co * C;
    if constexpr ((C % 2) == 0) {
#pragma unroll
      for (int i = 0; i < C / 2; ++i) {
        const float4 v = reinterpret_cast<const float4*>(row)[i];
        cfma(a0, make_float2(v.x, v.y), x[2 * i]);
        cfma(a1, make_float2(v.z, v.w), x[2 * i + 1]);
      }
    } else {
#pragma unroll
      for (int i = 0; i < C; ++i) cfma((i & 1) ? a1 : a0, row[i], x[i]);
    }
    y[co] = make_float2(a0.x + a1.x, a0.y + a1.y);
  }
}

template <int C, bool OUTER>
__global__ void __launch_bounds__(Threads5<C>::value, 1) grog_grid_v5_kernel(
    const float2* __restrict__ data, int64_t N, float2* __restrict__ grid, int64_t G,
    const float2* __restrict__ inner, int n_inner, const float2* __restrict__ outer, int n_outer,
    const int32_t* __restrict__ rep_src, const uint32_t* __restrict__ rep_meta,
    const float* __restrict__ rep_w, const int4* __restrict__ work, int n_work, Geom5 geom) {
  extern __shared__ float4 smem4[];
  constexpr int PS = Pad<C>::kStride;
  float2* inner_s = reinterpret_cast<float2*>(smem4);
  float2* outer_s = inner_s + static_cast<int64_t>(n_inner) * PS;
  const int cells = geom.bz * geom.by * geom.bx;
  const int TS = cells + 1;
  float2* tile = outer_s + (OUTER ? static_cast<int64_t>(n_outer) * PS : 0);  // (C, TS)
  stage_ops<C>(inner_s, inner, n_inner);
  if (OUTER) stage_ops<C>(outer_s, outer, n_outer);
  const int b = blockIdx.y;
  const float2* dat = data + static_cast<int64_t>(b) * C * N;
  float2* grd = grid + static_cast<int64_t>(b) * C * G;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NT = Threads5<C>::value;
  constexpr int NW = NT / 32;

  for (int it = blockIdx.x; it < n_work; it += gridDim.x) {
    const int4 item = work[it];
    const int begin = item.y, end = item.z;
    for (int t = threadIdx.x; t < C * TS; t += NT) tile[t] = make_float2(0.f, 0.f);
    __syncthreads();
    // prefetch the first batch of this warp
    int r = begin + warp * 32 + lane;
    bool have = r < end;
    int src = 0, cell = 0, ii = 0, k = 0;
    float w = 0.f;
    float2 x[C];
    auto fetch = [&](int rr, bool h) {
      src = -1;
      cell = 0;
      ii = 0;
      k = 0;
      w = 0.f;
      if (h) {
        const int s_ = __ldg(rep_src + rr);
        const uint32_t m = __ldg(rep_meta + rr);
        const int c_ = static_cast<int>(m & 2047u);
        const int i_ = static_cast<int>((m >> 11) & 16383u);
        const int k_ = static_cast<int>(m >> 25);
        if (s_ >= 0 && s_ < N && c_ < cells && i_ < n_inner && (!OUTER || k_ < n_outer)) {
          src = s_;
          cell = c_;
          ii = i_;
          k = OUTER ? k_ : 0;
          w = __ldg(rep_w + rr);
        }
      }
#pragma unroll
      for (int c = 0; c < C; ++c)
        x[c] = src >= 0 ? __ldg(dat + static_cast<int64_t>(c) * N + src) : make_float2(0.f, 0.f);
    };
    fetch(r, have);
    while (true) {
      const bool active = r < end;
      if (!__any_sync(0xffffffffu, active)) break;
      const int cur_src = src, cur_cell = cell, cur_ii = ii, cur_k = k;
      const float cur_w = w;
      float2 xc[C];
#pragma unroll
      for (int c = 0; c < C; ++c) xc[c] = x[c];
      // prefetch the next batch while this one computes
      const int rn = r + NW * 32;
      fetch(rn, rn < end);
      float2 u[C];
      apply_op<C>(inner_s + static_cast<int64_t>(cur_ii) * PS, xc, u);
      if constexpr (OUTER) {
        float2 y[C];
        apply_op<C>(outer_s + static_cast<int64_t>(cur_k) * PS, u, y);
#pragma unroll
        for (int c = 0; c < C; ++c) u[c] = y[c];
      }
      if (active && cur_src >= 0) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
          atomicAdd(&tile[c * TS + cur_cell].x, cur_w * u[c].x);
          atomicAdd(&tile[c * TS + cur_cell].y, cur_w * u[c].y);
        }
      }
      r = rn;
    }
    __syncthreads();
    int z0, y0, x0;
    origin5(geom, item.x, z0, y0, x0);
    for (int t = threadIdx.x; t < C * cells; t += NT) {
      const int c = t / cells;
      const int cl = t - c * cells;
      int64_t flat;
      if (!flat5(geom, z0, y0, x0, cl, flat)) continue;
      const float2 v = tile[c * TS + cl];
      float2* dst = grd + static_cast<int64_t>(c) * G + flat;
      if (item.w) {
        if (v.x != 0.f || v.y != 0.f) {
          atomicAdd(&dst->x, v.x);
          atomicAdd(&dst->y, v.y);
        }
      } else {
        *dst = v;
      }
    }
    __syncthreads();
  }
}

template <int C, bool OUTER>
__global__ void __launch_bounds__(Threads5<C>::value, 1) grog_degrid_v5_kernel(
    const float2* __restrict__ grid, int64_t G, float2* __restrict__ out, int64_t N,
    const float2* __restrict__ inner_h, int n_inner, const float2* __restrict__ outer_h, int n_outer,
    const int32_t* __restrict__ rep_src, const uint32_t* __restrict__ rep_meta,
    const float* __restrict__ rep_w, const int4* __restrict__ work, int n_work, Geom5 geom,
    int accumulate) {
  extern __shared__ float4 smem4[];
  constexpr int PS = Pad<C>::kStride;
  float2* inner_s = reinterpret_cast<float2*>(smem4);
  float2* outer_s = inner_s + static_cast<int64_t>(n_inner) * PS;
  const int cells = geom.bz * geom.by * geom.bx;
  float2* tile = outer_s + (OUTER ? static_cast<int64_t>(n_outer) * PS : 0);  // (cells, C) cell-major
  stage_ops<C>(inner_s, inner_h, n_inner);
  if (OUTER) stage_ops<C>(outer_s, outer_h, n_outer);
  const int b = blockIdx.y;
  const float2* grd = grid + static_cast<int64_t>(b) * C * G;
  float2* o = out + static_cast<int64_t>(b) * C * N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NT = Threads5<C>::value;
  constexpr int NW = NT / 32;

  for (int it = blockIdx.x; it < n_work; it += gridDim.x) {
    const int4 item = work[it];
    const int begin = item.y, end = item.z;
    if (end <= begin) continue;  // block-uniform
    __syncthreads();             // previous item's readers are done with the tile
    int z0, y0, x0;
    origin5(geom, item.x, z0, y0, x0);
    for (int t = threadIdx.x; t < C * cells; t += NT) {
      const int c = t / cells;
      const int cl = t - c * cells;
      int64_t flat;
      float2 v = make_float2(0.f, 0.f);
      if (flat5(geom, z0, y0, x0, cl, flat)) v = __ldg(grd + static_cast<int64_t>(c) * G + flat);
      tile[cl * C + c] = v;
    }
    __syncthreads();
    for (int r = begin + warp * 32 + lane; __any_sync(0xffffffffu, r < end); r += NW * 32) {
      int src = -1, cell = 0, ii = 0, k = 0;
      float w = 0.f;
      if (r < end) {
        const int s_ = __ldg(rep_src + r);
        const uint32_t m = __ldg(rep_meta + r);
        const int c_ = static_cast<int>(m & 2047u);
        const int i_ = static_cast<int>((m >> 11) & 16383u);
        const int k_ = static_cast<int>(m >> 25);
        if (s_ >= 0 && s_ < N && c_ < cells && i_ < n_inner && (!OUTER || k_ < n_outer)) {
          src = s_;
          cell = c_;
          ii = i_;
          k = OUTER ? k_ : 0;
          w = __ldg(rep_w + r);
        }
      }
      float2 g[C];
      const float2* tc = tile + cell * C;
#pragma unroll
      for (int c = 0; c < C; ++c) g[c] = tc[c];
      float2 y[C];
      if constexpr (OUTER) {
        float2 v[C];
        apply_op<C>(outer_s + static_cast<int64_t>(k) * PS, g, v);
        apply_op<C>(inner_s + static_cast<int64_t>(ii) * PS, v, y);
      } else {
        apply_op<C>(inner_s + static_cast<int64_t>(ii) * PS, g, y);
      }
      if (src >= 0) {
#pragma unroll
        for (int c = 0; c < C; ++c) {
          float2* dst = o + static_cast<int64_t>(c) * N + src;
          if (accumulate) {
            atomicAdd(&dst->x, w * y[c].x);
            atomicAdd(&dst->y, w * y[c].y);
          } else {
            *dst = make_float2(w * y[c].x, w * y[c].y);
          }
        }
      }
    }
  }
}

#define PGB5_FOR_EACH_C(X) \
  X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

static size_t v5_smem(int64_t C, int cells, int64_t n_inner, int64_t n_outer) {
  const int64_t ps = C * C + 2;
  return static_cast<size_t>(n_inner * ps + (n_outer > 1 ? n_outer * ps : 0) + C * (cells + 1)) * sizeof(float2);
}

static int v5_geom(const pgb_brick_plan* p, Geom5& g, const char* who) {
  PGB_REQUIRE(p != nullptr, PGB_ERR_INVALID, "%s: null plan", who);
  auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
  PGB_REQUIRE(pow2(p->bz) && pow2(p->by) && pow2(p->bx) && p->gz >= 1 && p->gy >= 1 && p->gx >= 1,
              PGB_ERR_INVALID, "%s: brick extents must be powers of two", who);
  const int64_t cells = static_cast<int64_t>(p->bz) * p->by * p->bx;
  PGB_REQUIRE(cells <= 2048, PGB_ERR_RANGE, "%s: brick of %lld cells exceeds 2048", who, (long long)cells);
  PGB_REQUIRE(p->nbz == (p->gz + p->bz - 1) / p->bz && p->nby == (p->gy + p->by - 1) / p->by &&
                  p->nbx == (p->gx + p->bx - 1) / p->bx,
              PGB_ERR_INVALID, "%s: brick counts do not match the grid", who);
  PGB_REQUIRE(p->n_work >= 0, PGB_ERR_INVALID, "%s: negative work count", who);
  PGB_REQUIRE(p->n_work == 0 || (p->work && p->rep_src && p->rep_meta && p->rep_w), PGB_ERR_INVALID,
              "%s: null plan arrays", who);
  int lbx = 0, lby = 0;
  while ((1 << lbx) < p->bx) ++lbx;
  while ((1 << lby) < p->by) ++lby;
  g = Geom5{p->gz, p->gy, p->gx, p->bz, p->by, p->bx, lbx, lby, p->nbz, p->nby, p->nbx};
  return PGB_OK;
}

__global__ void zero_bricks_v5(float2* __restrict__ grid, int64_t G, int C, int B,
                               const int32_t* __restrict__ bricks, int n_bricks, Geom5 geom) {
  const int cells = geom.bz * geom.by * geom.bx;
  const int64_t total = static_cast<int64_t>(n_bricks) * cells;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / cells);
    const int cl = static_cast<int>(t - static_cast<int64_t>(i) * cells);
    int z0, y0, x0;
    origin5(geom, bricks[i], z0, y0, x0);
    int64_t flat;
    if (!flat5(geom, z0, y0, x0, cl, flat)) continue;
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < C; ++c) grid[(static_cast<int64_t>(b) * C + c) * G + flat] = make_float2(0.f, 0.f);
  }
}

__global__ void zero_samples_v5(float2* __restrict__ out, int64_t N, int C, int B,
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

size_t pgb_grog_v5_smem_bytes(int64_t C, int64_t cells, int64_t n_inner, int64_t n_outer) {
  return v5_smem(C, static_cast<int>(cells), n_inner, n_outer);
}

int pgb_grog_grid_v5(const void* data, int64_t N, void* grid, int64_t G, const void* inner,
                     int64_t n_inner, const void* outer, int64_t n_outer, int64_t C, int64_t B,
                     const pgb_brick_plan* plan, void* stream) {
  clear_error();
  Geom5 geom;
  int st = v5_geom(plan, geom, "grog_grid_v5");
  if (st) return st;
  PGB_REQUIRE(C >= 1 && C <= 16, PGB_ERR_UNSUPPORTED, "grog_grid_v5: ncoils must be 1..16, got %lld",
              (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 &&
                  n_inner <= 16384 && n_outer >= 1 && n_outer <= 128,
              PGB_ERR_RANGE, "grog_grid_v5: invalid N/B/table sizes");
  PGB_REQUIRE(n_outer == 1 || outer != nullptr, PGB_ERR_INVALID, "grog_grid_v5: null outer table");
  PGB_REQUIRE(G == static_cast<int64_t>(plan->gz) * plan->gy * plan->gx, PGB_ERR_INVALID,
              "grog_grid_v5: G does not match the plan grid");
  if (B == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(grid && inner && (data || N == 0), PGB_ERR_INVALID, "grog_grid_v5: null pointer");
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = v5_smem(C, cells, n_inner, n_outer);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "grog_grid_v5: tables + tile need %zu B of shared memory", smem);
  cudaStream_t s = as_stream(stream);
  if (plan->n_split_bricks > 0) {
    PGB_REQUIRE(plan->split_bricks != nullptr, PGB_ERR_INVALID, "grog_grid_v5: null split list");
    const int64_t tot = static_cast<int64_t>(plan->n_split_bricks) * cells;
    zero_bricks_v5<<<grid_for(tot, 256, 148 * 16), 256, 0, s>>>(static_cast<float2*>(grid), G,
                                                               static_cast<int>(C), static_cast<int>(B),
                                                               plan->split_bricks, plan->n_split_bricks, geom);
    PGB_LAUNCH_CHECK("grog_grid_v5(zero split bricks)");
  }
  if (plan->n_work == 0) return PGB_OK;
  const int nblk = plan->n_work < kNumSMs ? plan->n_work : kNumSMs;
  dim3 grd(nblk, static_cast<unsigned>(B));
  const bool has_outer = n_outer > 1;
  switch (C) {
#define X(CC)                                                                                    \
  case CC: {                                                                                     \
    auto k = has_outer ? grog_grid_v5_kernel<CC, true> : grog_grid_v5_kernel<CC, false>;         \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);             \
    k<<<grd, Threads5<CC>::value, smem, s>>>(static_cast<const float2*>(data), N, static_cast<float2*>(grid), G, \
                             static_cast<const float2*>(inner), static_cast<int>(n_inner),       \
                             static_cast<const float2*>(outer), static_cast<int>(n_outer),       \
                             plan->rep_src, plan->rep_meta, plan->rep_w,                         \
                             reinterpret_cast<const int4*>(plan->work), plan->n_work, geom);     \
  } break;
    PGB5_FOR_EACH_C(X)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK("grog_grid_v5");
  return PGB_OK;
}

int pgb_grog_degrid_v5(const void* grid, int64_t G, void* out, int64_t N, const void* inner_h,
                       int64_t n_inner, const void* outer_h, int64_t n_outer, int64_t C, int64_t B,
                       const pgb_brick_plan* primary, const pgb_brick_plan* secondary,
                       const int32_t* zero_src, int64_t n_zero, void* stream) {
  clear_error();
  Geom5 geom;
  int st = v5_geom(primary, geom, "grog_degrid_v5");
  if (st) return st;
  if (secondary != nullptr) {
    Geom5 g2;
    st = v5_geom(secondary, g2, "grog_degrid_v5(secondary)");
    if (st) return st;
  }
  PGB_REQUIRE(C >= 1 && C <= 16, PGB_ERR_UNSUPPORTED, "grog_degrid_v5: ncoils must be 1..16, got %lld",
              (long long)C);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535 && n_inner >= 1 &&
                  n_inner <= 16384 && n_outer >= 1 && n_outer <= 128 && n_zero >= 0,
              PGB_ERR_RANGE, "grog_degrid_v5: invalid N/B/table sizes");
  PGB_REQUIRE(n_outer == 1 || outer_h != nullptr, PGB_ERR_INVALID, "grog_degrid_v5: null outer table");
  PGB_REQUIRE(G == static_cast<int64_t>(primary->gz) * primary->gy * primary->gx, PGB_ERR_INVALID,
              "grog_degrid_v5: G does not match the plan grid");
  if (B == 0 || N == 0) return PGB_OK;
  PGB_REQUIRE(out && inner_h && (grid || G == 0), PGB_ERR_INVALID, "grog_degrid_v5: null pointer");
  const int cells = primary->bz * primary->by * primary->bx;
  const size_t smem = v5_smem(C, cells, n_inner, n_outer);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED,
              "grog_degrid_v5: tables + tile need %zu B of shared memory", smem);
  cudaStream_t s = as_stream(stream);
  if (n_zero > 0) {
    PGB_REQUIRE(zero_src != nullptr, PGB_ERR_INVALID, "grog_degrid_v5: null zero list");
    zero_samples_v5<<<grid_for(n_zero * C * B, 256, 148 * 8), 256, 0, s>>>(
        static_cast<float2*>(out), N, static_cast<int>(C), static_cast<int>(B), zero_src, n_zero);
    PGB_LAUNCH_CHECK("grog_degrid_v5(zero samples)");
  }
  const bool has_outer = n_outer > 1;
  for (int pass = 0; pass < 2; ++pass) {
    const pgb_brick_plan* p = pass == 0 ? primary : secondary;
    if (p == nullptr || p->n_work == 0) continue;
    const int nblk = p->n_work < kNumSMs ? p->n_work : kNumSMs;
    dim3 grd(nblk, static_cast<unsigned>(B));
    switch (C) {
#define X(CC)                                                                                    \
  case CC: {                                                                                     \
    auto k = has_outer ? grog_degrid_v5_kernel<CC, true> : grog_degrid_v5_kernel<CC, false>;     \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);             \
    k<<<grd, Threads5<CC>::value, smem, s>>>(static_cast<const float2*>(grid), G, static_cast<float2*>(out), N, \
                             static_cast<const float2*>(inner_h), static_cast<int>(n_inner),     \
                             static_cast<const float2*>(outer_h), static_cast<int>(n_outer),     \
                             p->rep_src, p->rep_meta, p->rep_w,                                  \
                             reinterpret_cast<const int4*>(p->work), p->n_work, geom, pass);     \
  } break;
      PGB5_FOR_EACH_C(X)
#undef X
      default:
        break;
    }
    PGB_LAUNCH_CHECK("grog_degrid_v5");
  }
  return PGB_OK;
}

}  // extern "C"
