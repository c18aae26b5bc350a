// grog_tc.cu -- fused GROG grid / degrid on the tensor cores (bf16x3 or bf16).
//
// The table factorises exactly.  The reference builds every per-axis
// fractional operator as G_a(d) = expm(d * L_a) with L_a = logm(G_a)
// (calib/_grappa.py:62-72, 184-208) and the table as the product
// T[i, j, k] = Gx(d_k) Gy(d_j) Gz(d_i) (calib/_grappa.py:130-181).  With the
// eigendecomposition L_a = V_a diag(l_a) V_a^-1 that is
//
//   T x = Vx Dx[k] Vx^-1 Vy Dy[j] Vy^-1 Vz Dz[i] Vz^-1 x,   D_a[s] = diag(exp(d_s l_a)),
//
// i.e. four dense C x C matrices W0 = Vz^-1, W1 = Vy^-1 Vz, W2 = Vx^-1 Vy,
// W3 = Vx shared by every replica, and three per-replica diagonals (two
// dense stages fewer in 2-D).  The dense stages are GEMMs over all replicas
// with no binning: each warp takes 16 replicas as the M rows of
// mma.m16n8k16 / m16n8k8 (bf16 in, fp32 accumulate), the complex C x C
// matrix realified with (re, im) interleaved so that an accumulator
// fragment of one stage is, register for register, the A fragment of the
// next, and the diagonal phases are lane-local complex products between
// stages.  The W fragments live in registers for the whole kernel; the
// diagonal tables (nsteps x C per axis) in shared memory.
//
// Precision: with terms == 3 every operand is split into a bf16 head and a
// bf16 tail (x = hi + lo) and each product is hi*hi + hi*lo + lo*hi with fp32
// accumulation (~2^-16 relative per stage); terms == 1 uses the heads only.
//
// Plans: the v6 brick plans (calib/_plan6.py) with the table index e split
// into its per-axis shift indices, meta.y = i | j << 8 | k << 16 in 3-D
// (e = (i nsteps + j) nsteps + k, nsteps <= 255) and i | k << 16 in 2-D
// (e = i nsteps + k).
// The forward plan orders each sub-chunk by (cell, sample) and marks cells
// whose run crosses an m-tile boundary (meta.x bit 30); the adjoint plans keep
// sample order (conflict-free result writes).
//
//   forward:  per sub-chunk, stage the samples' coils (cp.async, double
//             buffered), run the chain for 16 replicas per warp, sum each
//             cell's rows in registers (segmented scan over the m-tile) and
//             add the totals to the brick tile (plain read-modify-writes;
//             atomics only for runs crossing an m-tile); flush the tile once
//             per brick (global atomics only for bricks split over CTAs)
//   adjoint:  tile of the brick (cp.async, prefetched one brick ahead), the
//             adjoint chain W3^H conj(Dx) W2^H conj(Dy) W1^H conj(Dz) W0^H per
//             replica, w * y into a per-slot result buffer, flushed per
//             sub-chunk (atomic adds for the secondary replicas)
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "common.cuh"

namespace pgb {
namespace tc {

constexpr int kT = 256;  // threads per CTA: 8 warps x 2 m-tiles = 256 replicas per sub-chunk (128 above 16 coils)
constexpr int kFirst = 1, kLast = 2, kSplit = 4;
constexpr int kZeroPerFlush = 4;  // forward: clearing stores of empty bricks per brick item

// 16-byte groups of B-fragment words per n-tile (head or tail) for CP coils:
// ceil((2 * k16 chunks + k8 chunk) / 4), k16 = CP / 8, k8 = (CP / 4) % 2
__host__ __device__ constexpr int tc_wq(int CP) { return (2 * (CP / 8) + (CP / 4) % 2 + 3) / 4; }

template <int CP>
struct Shape {
  static constexpr int NT = CP / 4;                   // n-tiles of 8 real columns (4 complex coils)
  static constexpr int K16 = NT / 2;                  // k16 chunks of the next stage
  static constexpr int K8 = NT % 2;                   // trailing k8 chunk
  static constexpr int NFR = NT * (2 * K16 + K8);     // B-fragment words per lane per matrix
  static constexpr int FPN = 2 * K16 + K8;            // words per n-tile
  static constexpr int WQ = (FPN + 3) / 4;            // 16-byte groups per n-tile and head / tail
  static_assert(WQ == tc_wq(CP), "fragment group count");
  static constexpr int TS = CP + 1;                   // tile stride per cell (float2): conflict-free flush
  // m-tiles a warp runs side by side: two up to 16 coils (256-entry
  // sub-chunks), one above (128-entry sub-chunks: the registers of one tile)
  static constexpr int NTL = CP <= 16 ? 2 : 1;
};

template <int CP, int NS>
struct Regs {
  static constexpr int MINB = CP <= 12 ? 2 : 1;  // CTAs per SM the register budget (two m-tiles per warp) allows
};

struct Geom {
  int gz, gy, gx;
  int bz, by, bx;
  int lbx, lby;
  int nbz, nby, nbx;
};

__device__ __forceinline__ void origin(const Geom& g, int brick, int& z0, int& y0, int& x0) {
  const int bxy = g.nby * g.nbx;
  const int biz = brick / bxy;
  const int rem = brick - biz * bxy;
  const int biy = rem / g.nbx;
  z0 = biz * g.bz;
  y0 = biy * g.by;
  x0 = (rem - biy * g.nbx) * g.bx;
}

__device__ __forceinline__ bool flat_of(const Geom& g, int z0, int y0, int x0, int cl, int64_t& flat) {
  const int x = x0 + (cl & (g.bx - 1));
  const int y = y0 + ((cl >> g.lbx) & (g.by - 1));
  const int z = z0 + (cl >> (g.lbx + g.lby));
  if (z >= g.gz || y >= g.gy || x >= g.gx) return false;
  flat = (static_cast<int64_t>(z) * g.gy + y) * g.gx + x;
  return true;
}

__device__ __forceinline__ void cp8(void* smem_dst, const void* gsrc, int bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp16_cg(void* smem_dst, const void* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp4(void* smem_dst, const void* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void wait_groups() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---- TMA brick tiles ---------------------------------------------------------
// The grid (B, C, gz, gy, gx) complex64 is described to the tensor memory
// accelerator as a float32 tensor of dims {2 gx, gy, gz, B C}; one box
// {2 bx, by, bz, C} is one brick of all coils, laid out in shared memory as
// [coil][cell] (cell = (z by + y) bx + x).  Loads complete on an mbarrier,
// stores / reduce-adds are bulk groups.  No multicast.
__device__ int g_tc_timeouts;  // mbarrier waits that gave up (see pgb_grog_tc_timeouts)
constexpr long long kSpinLimit = 1ll << 26;
// Spin limit of the tile waits that gate compute (pgb_grog_tc_wait_limit sets
// it; the default is kSpinLimit).  The drain of copies still in flight after a
// wait gave up always uses kSpinLimit.
__device__ long long g_tc_wait_limit = kSpinLimit;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase `parity` of `bar`; false (and a recorded
// timeout) if it did not complete within the spin limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const long long limit = g_tc_wait_limit;
  for (long long i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (threadIdx.x == 0) atomicAdd(&g_tc_timeouts, 1);
  return false;
}
// Bounded wait used only on the way out after a timeout: lets a tensor copy
// that is still writing this CTA's shared memory finish before the CTA exits.
__device__ __forceinline__ void mbar_drain(uint64_t* bar, unsigned parity) {
  for (long long i = 0; i < kSpinLimit; ++i)
    if (mbar_try_wait(bar, parity)) return;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tma_load_tile(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_tile(const CUtensorMap* map, int x, int y, int z, int w, const void* src,
                                               bool add) {
  if (add) {
    asm volatile(
        "cp.reduce.async.bulk.tensor.4d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];\n" ::"l"(
            reinterpret_cast<uint64_t>(map)),
        "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(src))
        : "memory");
  } else {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];\n" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(src))
                 : "memory");
  }
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// d += A B, A 16x16 (4 bf16x2 words), B 16x8 (2 words), fp32 accumulate
__device__ __forceinline__ void mma16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                      uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}
// d += A B, A 16x8 (2 words), B 8x8 (1 word)
__device__ __forceinline__ void mma8(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b0) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(b0));
}

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 h) { return *reinterpret_cast<uint32_t*>(&h); }

// (re, im) -> bf16x2 head (re in the low half) and tail
__device__ __forceinline__ void split2(float2 v, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(v.x, v.y);
  const float2 hf = __bfloat1622float2(h);
  hi = bf2_bits(h);
  lo = bf2_bits(__floats2bfloat162_rn(v.x - hf.x, v.y - hf.y));
}

// v[T][r][m] = complex coil 4 m + t of row g + 8 r of the lane's m-tile T
// (g = lane / 4, t = lane % 4); a warp runs its two m-tiles side by side (two
// independent instruction streams).  One dense stage: v <- v W^T over the 16
// rows of each tile.  W's fragments come from shared memory, per n-tile one
// 16-byte word group of heads and one of tails per lane (lane-contiguous:
// conflict-free).
template <int CP, int TERMS>
__device__ __forceinline__ void mm_stage(float2 (&v)[Shape<CP>::NTL][2][Shape<CP>::NT], const uint4* __restrict__ wst, int lane) {
  constexpr int NT = Shape<CP>::NT, K16 = Shape<CP>::K16, K8 = Shape<CP>::K8;
  constexpr int NTL = Shape<CP>::NTL, WQ = Shape<CP>::WQ;
  uint32_t ah[NTL][2][NT], al[NTL][2][NT];
#pragma unroll
  for (int T = 0; T < NTL; ++T)
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int m = 0; m < NT; ++m) {
        if constexpr (TERMS == 3) {
          split2(v[T][r][m], ah[T][r][m], al[T][r][m]);
        } else {
          ah[T][r][m] = bf2_bits(__floats2bfloat162_rn(v[T][r][m].x, v[T][r][m].y));
          al[T][r][m] = 0u;
        }
      }
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
    uint32_t bh[4 * WQ], bl[4 * WQ];
#pragma unroll
    for (int q = 0; q < WQ; ++q) {
      const uint4 h4 = wst[((nt * 2) * WQ + q) * 32 + lane];
      const uint4 l4 = wst[((nt * 2 + 1) * WQ + q) * 32 + lane];
      bh[4 * q] = h4.x, bh[4 * q + 1] = h4.y, bh[4 * q + 2] = h4.z, bh[4 * q + 3] = h4.w;
      bl[4 * q] = l4.x, bl[4 * q + 1] = l4.y, bl[4 * q + 2] = l4.z, bl[4 * q + 3] = l4.w;
    }
    // products alternate between two accumulators per tile (tails first)
    float d[NTL][2][4];
#pragma unroll
    for (int T = 0; T < NTL; ++T)
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int e = 0; e < 4; ++e) d[T][a][e] = 0.f;
    int q = 0;
#pragma unroll
    for (int kc = 0; kc < K16; ++kc) {
      const int f = 2 * kc;
      if constexpr (TERMS == 3) {
#pragma unroll
        for (int T = 0; T < NTL; ++T)
          mma16(d[T][q & 1], al[T][0][2 * kc], al[T][1][2 * kc], al[T][0][2 * kc + 1], al[T][1][2 * kc + 1], bh[f],
                bh[f + 1]);
        ++q;
#pragma unroll
        for (int T = 0; T < NTL; ++T)
          mma16(d[T][q & 1], ah[T][0][2 * kc], ah[T][1][2 * kc], ah[T][0][2 * kc + 1], ah[T][1][2 * kc + 1], bl[f],
                bl[f + 1]);
        ++q;
      }
#pragma unroll
      for (int T = 0; T < NTL; ++T)
        mma16(d[T][q & 1], ah[T][0][2 * kc], ah[T][1][2 * kc], ah[T][0][2 * kc + 1], ah[T][1][2 * kc + 1], bh[f],
              bh[f + 1]);
      ++q;
    }
    if constexpr (K8) {
      const int f = 2 * K16;
      if constexpr (TERMS == 3) {
#pragma unroll
        for (int T = 0; T < NTL; ++T) mma8(d[T][q & 1], al[T][0][NT - 1], al[T][1][NT - 1], bh[f]);
        ++q;
#pragma unroll
        for (int T = 0; T < NTL; ++T) mma8(d[T][q & 1], ah[T][0][NT - 1], ah[T][1][NT - 1], bl[f]);
        ++q;
      }
#pragma unroll
      for (int T = 0; T < NTL; ++T) mma8(d[T][q & 1], ah[T][0][NT - 1], ah[T][1][NT - 1], bh[f]);
    }
#pragma unroll
    for (int T = 0; T < NTL; ++T) {
      v[T][0][nt] = make_float2(d[T][0][0] + d[T][1][0], d[T][0][1] + d[T][1][1]);
      v[T][1][nt] = make_float2(d[T][0][2] + d[T][1][2], d[T][0][3] + d[T][1][3]);
    }
  }
}

// W fragments of all NS + 1 stages into shared memory, layout (stage, n-tile,
// head/tail, lane, 4 words) from the global layout (stage, head/tail, word, lane).
template <int CP, int NS>
__device__ __forceinline__ void stage_w(uint32_t* __restrict__ wsm, const uint32_t* __restrict__ wfrag) {
  constexpr int NT = Shape<CP>::NT, NFR = Shape<CP>::NFR, FPN = Shape<CP>::FPN, WQ = Shape<CP>::WQ;
  constexpr int total = (NS + 1) * NT * 2 * WQ * 32 * 4;
  for (int i = threadIdx.x; i < total; i += kT) {  // layout (stage, nt, head / tail, q, lane, 4 words)
    const int w4 = i & 3;
    const int lane = (i >> 2) & 31;
    const int r = i >> 7;  // ((stage * NT + nt) * 2 + b) * WQ + q
    const int q = r % WQ;
    const int b = (r / WQ) & 1;
    const int snt = r / (WQ * 2);
    const int s = snt / NT;
    const int nt = snt - s * NT;
    const int w = 4 * q + w4;
    wsm[i] = w < FPN ? __ldg(wfrag + ((s * 2 + b) * NFR + nt * FPN + w) * 32 + lane) : 0u;
  }
}

// One replica row's decoded metadata.
struct Row {
  int cell, slot, ix0, ix1, ix2;
  float w;
  bool on, straddle;
};

template <int NS>
__device__ __forceinline__ Row decode(int2 m, float w, bool in_range, int cells, int nu, int nsteps) {
  Row r;
  r.cell = m.x & 0xFFFF;
  r.slot = (m.x >> 16) & 0x3FFF;
  r.straddle = (m.x >> 30) & 1;
  // axis indices packed by the plan: 3-D i | j << 8 | k << 16, 2-D i | k << 16
  const int a0 = NS == 3 ? (m.y & 0xFF) : (m.y & 0xFFFF);
  const int a1 = NS == 3 ? ((m.y >> 8) & 0xFF) : ((m.y >> 16) & 0xFFFF);
  const int a2 = NS == 3 ? ((m.y >> 16) & 0xFFFF) : 0;
  r.on = in_range && m.x >= 0 && r.cell < cells && r.slot < nu && a0 < nsteps && a1 < nsteps && a2 < nsteps;
  r.ix0 = r.on ? a0 : 0;
  r.ix1 = r.on ? a1 : 0;
  r.ix2 = r.on ? a2 : 0;
  r.cell = r.on ? r.cell : 0;
  r.slot = r.on ? r.slot : 0;
  r.w = r.on ? w : 0.f;
  return r;
}

template <int NS, bool ADJ>
__device__ __forceinline__ int diag_index(const Row& r, int s) {
  const int a = ADJ ? NS - 1 - s : s;
  return a == 0 ? r.ix0 : (a == 1 ? r.ix1 : r.ix2);
}

// The whole chain on a warp's two m-tiles: NS + 1 dense stages with the
// diagonal phases of table dt (NS, nsteps, row stride dstride) between them.
template <int CP, int NS, int TERMS, bool ADJ>
__device__ __forceinline__ void chain(float2 (&v)[Shape<CP>::NTL][2][Shape<CP>::NT], const uint4* __restrict__ wsm,
                                      const float2* __restrict__ dt, int nsteps, int dstride,
                                      const Row (&rw)[Shape<CP>::NTL][2], int lane) {
  constexpr int NT = Shape<CP>::NT, NTL = Shape<CP>::NTL, WQ = Shape<CP>::WQ;
  const int t = lane & 3;
#pragma unroll
  for (int s = 0; s <= NS; ++s) {
    mm_stage<CP, TERMS>(v, wsm + s * NT * 2 * WQ * 32, lane);
    if (s < NS) {
#pragma unroll
      for (int T = 0; T < NTL; ++T)
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const float2* drow = dt + (s * nsteps + diag_index<NS, ADJ>(rw[T][r], s)) * dstride + t;
#pragma unroll
          for (int m = 0; m < NT; ++m) v[T][r][m] = cmul(v[T][r][m], drow[4 * m]);
        }
    }
  }
}

// Per-CTA stream of sub-chunk descriptors: d loaded four ahead, the
// {brick, flags} words three ahead, so the L2 prefetch of sub-chunk p + 2
// and the staging of p + 1 never wait on a descriptor load.
struct Stream {
  const int4* sd;
  const int2* si;
  int p, p1;
  int4 d0, d1, d2, d3;
  int2 i0, i1, i2;
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
  }
  __device__ __forceinline__ void advance() {
    ++p;
    d0 = d1;
    d1 = d2;
    d2 = d3;
    i0 = i1;
    i1 = i2;
    d3 = ld_d(p + 3);
    i2 = ld_i(p + 2);
  }
};

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2::evict_last [%0];\n" ::"l"(p));
}

__device__ __forceinline__ int n_slots(int4 d, int cap) { return min(max(d.w - d.z, 0), cap); }
__device__ __forceinline__ int n_reps(int4 d, int cap) { return min(max(d.y - d.x, 0), cap); }

// Prefetch the replica metadata and weights of sub-chunk d into L2.
__device__ __forceinline__ void prefetch_meta(const int2* __restrict__ meta, const float* __restrict__ wts, int4 d,
                                              int cap) {
  const int nr = n_reps(d, cap);
  const int i = threadIdx.x * 16;  // one 128-byte line of int2 per 16 entries
  if (i < nr) {
    prefetch_l2(meta + d.x + i);
    if ((i & 31) == 0) prefetch_l2(wts + d.x + i);
  }
}

// Stage the replica metadata and weights of sub-chunk d (cp.async).
__device__ __forceinline__ void stage_meta(const int2* __restrict__ meta, const float* __restrict__ wts, int4 d,
                                           int cap, int2* __restrict__ ms, float* __restrict__ wsm) {
  const int nr = n_reps(d, cap);
  for (int i = threadIdx.x; i < nr; i += kT) {
    cp8(ms + i, meta + d.x + i, 8);
    cp4(wsm + i, wts + d.x + i);
  }
}

// Phase tables in shared memory: with 4 copies every step row is 16 float2
// (64 words, bank-aligned) and copy k starts 8 k words into the bank cycle,
// so the quarter-warps of rows g = 0..3 (copy g % 4) read disjoint banks
// whatever their shift indices; with 1 copy rows are CP float2.
struct Phases {
  int copies, stride, copy_sz;
  __host__ __device__ Phases(int CP, int NS, int nsteps) {
    const int sz4 = NS * nsteps * 16 + 4;
    if (CP <= 16 && 4 * sz4 * 8 <= 32 * 1024) {
      copies = 4;
      stride = 16;
      copy_sz = sz4;
    } else {
      copies = 1;
      stride = CP;
      copy_sz = NS * nsteps * CP;
    }
  }
};

// Shared-memory layout in float2 units: phase tables | tile(s) | staging (x or results)
struct Smem {
  int dt, wf, tile, tile_sz, xs, xs_sz, ms, wsm, bar, total;
  __host__ __device__ Smem(int CP, int NS, int nsteps, int cells, int cap, bool forward, bool tma = false) {
    dt = 0;
    const Phases ph(CP, NS, nsteps);
    wf = (ph.copies * ph.copy_sz + 1) & ~1;       // W fragments: (NS + 1) * (CP / 4) * 2 * WQ * 32 uint4
    tile = wf + (NS + 1) * (CP / 4) * 2 * tc_wq(CP) * 32 * 2;  // float2 units
    if (tma) {
      tile = (tile + 15) & ~15;  // 128-byte aligned TMA boxes, [coil][cell]
      tile_sz = (cells * CP + 15) & ~15;
    } else {
      tile_sz = (cells * (forward ? CP + 1 : CP) + 1) & ~1;  // forward: odd stride, conflict-free flush
    }
    xs = tile + (forward ? 1 : 2) * tile_sz;
    xs_sz = CP * (cap + 4);
    ms = xs + (forward ? 2 : 1) * xs_sz;  // 2 x cap replica metadata (int2)
    wsm = ms + 2 * cap;                   // 2 x cap replica weights (float)
    bar = wsm + cap;                      // 2 mbarriers (uint64)
    total = bar + 2;
  }
};

// Copy the (NS, nsteps, CP) phase table into its shared-memory copies.
__device__ __forceinline__ void stage_phases(float2* __restrict__ dt, const float2* __restrict__ dtab, int CP, int NS,
                                             int nsteps, const Phases& ph) {
  const int n = NS * nsteps * CP;
  for (int i = threadIdx.x; i < ph.copies * n; i += kT) {
    const int cp = i / n;
    const int e = i - cp * n;
    const int row = e / CP;
    dt[cp * ph.copy_sz + row * ph.stride + (e - row * CP)] = __ldg(dtab + e);
  }
}

// Sum the rows of one m-tile that belong to the same cell and add each cell's
// sum to the brick tile.  Rows hold sub-chunk positions p = 2 g + r in cell
// order (row g + 8 r of lane group g), so a cell is a run of consecutive
// positions: the pair of a lane is combined in registers, runs across lane
// groups by a segmented inclusive scan over g (shuffles by 4, 8, 16 lanes),
// and the last position of every run adds the total to tile[cell].  Runs
// that do not cross the m-tile (straddle bit clear) have no other writer in
// the sub-chunk and use plain read-modify-writes; the others add atomically.
template <int CP, bool FULLC, bool TMA>
__device__ __forceinline__ void reduce_rows_to_tile(float2 (&v)[2][Shape<CP>::NT], const Row (&rw)[2], int C,
                                                    float2* __restrict__ tile, int cells, int g, int t) {
  constexpr int NT = Shape<CP>::NT, TS = Shape<CP>::TS;
  constexpr unsigned FULL = 0xffffffffu;
  const int k0 = rw[0].on ? rw[0].cell : -1 - 2 * g;  // invalid rows: unique keys, never written
  const int k1 = rw[1].on ? rw[1].cell : -2 - 2 * g;
  int kprev = __shfl_up_sync(FULL, k1, 4);    // cell of position 2 g - 1
  int knext = __shfl_down_sync(FULL, k0, 4);  // cell of position 2 g + 2
  if (g == 0) kprev = -100;
  if (g == 7) knext = -101;
  const bool pair = k1 == k0;
  if (!__any_sync(FULL, pair || k0 == kprev)) {  // 16 distinct cells: no sums across rows
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      if (!rw[r].on) continue;
      float2* dst = tile + (TMA ? rw[r].cell : rw[r].cell * TS);
#pragma unroll
      for (int m = 0; m < NT; ++m) {
        const int c = 4 * m + t;
        if (!FULLC && c >= C) continue;
        if (rw[r].straddle) {
          atomicAdd(&dst[TMA ? c * cells : c].x, v[r][m].x);
          atomicAdd(&dst[TMA ? c * cells : c].y, v[r][m].y);
        } else {
          dst[TMA ? c * cells : c] = cadd(dst[TMA ? c * cells : c], v[r][m]);
        }
      }
    }
    return;
  }
  float2 a[NT];
#pragma unroll
  for (int m = 0; m < NT; ++m) a[m] = pair ? cadd(v[1][m], v[0][m]) : v[1][m];
  bool open = pair && k0 == kprev;  // position 2 g + 1's run continues into lane group g - 1
#pragma unroll
  for (int off = 1; off < 8; off <<= 1) {
    float2 ap[NT];
#pragma unroll
    for (int m = 0; m < NT; ++m) {
      ap[m].x = __shfl_up_sync(FULL, a[m].x, 4 * off);
      ap[m].y = __shfl_up_sync(FULL, a[m].y, 4 * off);
    }
    const bool op = __shfl_up_sync(FULL, open ? 1 : 0, 4 * off) != 0;
    if (g >= off && open) {
#pragma unroll
      for (int m = 0; m < NT; ++m) a[m] = cadd(a[m], ap[m]);
      open = op;
    }
  }
  float2 aprev[NT];  // scanned run total up to position 2 g - 1
#pragma unroll
  for (int m = 0; m < NT; ++m) {
    aprev[m].x = __shfl_up_sync(FULL, a[m].x, 4);
    aprev[m].y = __shfl_up_sync(FULL, a[m].y, 4);
  }
  // position 2 g ends a run when 2 g + 1 holds another cell
  if (!pair && rw[0].on) {
    const bool carry = k0 == kprev;
    float2* dst = tile + (TMA ? rw[0].cell : rw[0].cell * TS);
#pragma unroll
    for (int m = 0; m < NT; ++m) {
      const int c = 4 * m + t;
      if (!FULLC && c >= C) continue;
      const float2 val = carry ? cadd(v[0][m], aprev[m]) : v[0][m];
      if (rw[0].straddle) {
        atomicAdd(&dst[TMA ? c * cells : c].x, val.x);
        atomicAdd(&dst[TMA ? c * cells : c].y, val.y);
      } else {
        dst[TMA ? c * cells : c] = cadd(dst[TMA ? c * cells : c], val);
      }
    }
  }
  if (k1 != knext && rw[1].on) {
    float2* dst = tile + (TMA ? rw[1].cell : rw[1].cell * TS);
#pragma unroll
    for (int m = 0; m < NT; ++m) {
      const int c = 4 * m + t;
      if (!FULLC && c >= C) continue;
      if (rw[1].straddle) {
        atomicAdd(&dst[TMA ? c * cells : c].x, a[m].x);
        atomicAdd(&dst[TMA ? c * cells : c].y, a[m].y);
      } else {
        dst[TMA ? c * cells : c] = cadd(dst[TMA ? c * cells : c], a[m]);
      }
    }
  }
}

template <int CP, int NS, int TERMS, bool FULLC, bool TMA>
__global__ void __launch_bounds__(kT, Regs<CP, NS>::MINB) grog_grid_tc_kernel(
    const float2* __restrict__ data, int64_t N, float2* __restrict__ grid, int64_t G, int C,
    const uint32_t* __restrict__ wfrag, const float2* __restrict__ dtab, int nsteps, const int4* __restrict__ sd,
    const int2* __restrict__ si, const int32_t* __restrict__ cta_ptr, const int32_t* __restrict__ uniq,
    const int2* __restrict__ meta, const float* __restrict__ wts, int cap, Geom geom,
    const __grid_constant__ CUtensorMap tmap, const int32_t* __restrict__ zempty, int n_empty) {
  extern __shared__ __align__(128) float4 smem4[];
  constexpr int NT = Shape<CP>::NT, TS = Shape<CP>::TS;
  const int p0 = cta_ptr[blockIdx.x], p1 = cta_ptr[blockIdx.x + 1];
  if (p0 >= p1) return;  // block-uniform
  // bricks no sub-chunk touches (zempty, tensor-copy path only): this CTA
  // clears a share proportional to its sub-chunks by storing its tile while
  // the tile is clear (at the first sub-chunk of each brick item), at most
  // kZeroPerFlush per item and the rest when it is done, so that the
  // clearing writes overlap the chains.  Thread 0 keeps the position in the
  // list (z_next); every thread the count left (zleft).
  __shared__ int z_next;
  int zleft = 0;
  if (TMA && n_empty > 0) {
    const int64_t P = cta_ptr[gridDim.x];
    const int z0 = static_cast<int>(static_cast<int64_t>(n_empty) * p0 / P);
    zleft = static_cast<int>(static_cast<int64_t>(n_empty) * p1 / P) - z0;
    if (threadIdx.x == 0) z_next = z0;
  }
  const int cells = geom.bz * geom.by * geom.bx;
  const Smem lay(CP, NS, nsteps, cells, cap, true, TMA);
  const Phases ph(CP, NS, nsteps);
  const int XS = cap + 4;
  float2* base = reinterpret_cast<float2*>(smem4);
  float2* dt = base + lay.dt;
  float2* tile = base + lay.tile;
  float2* xs0 = base + lay.xs;
  int2* ms0 = reinterpret_cast<int2*>(base + lay.ms);
  float* ws0 = reinterpret_cast<float*>(base + lay.wsm);
  const int b = blockIdx.y;
  const float2* dat = data + static_cast<int64_t>(b) * C * N;
  float2* grd = grid + static_cast<int64_t>(b) * C * G;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const float2* dtl = dt + (ph.copies == 4 ? (g & 3) * ph.copy_sz : 0);  // this lane's phase copy

  auto ld_u = [&](int4 d, bool valid) -> int {
    return (valid && tid < n_slots(d, cap)) ? __ldg(uniq + d.z + tid) : -1;
  };
  // 16-byte copies need 16-byte aligned coil planes (even N, aligned base)
  const bool pairs_ok = (N & 1) == 0 && (XS & 1) == 0 && (reinterpret_cast<uintptr_t>(dat) & 15) == 0;
  auto stage_x = [&](int4 d, int u, float2* xs) {  // samples' coils of sub-chunk d, coil-major
    const int nu = n_slots(d, cap);
    // an even slot whose sample is even and whose odd neighbour holds the
    // next sample copies both with one 16-byte copy (L2 only); its neighbour
    // then copies nothing
    const int un = __shfl_down_sync(0xffffffffu, u, 1);
    const bool ok = tid < nu && u >= 0 && u < N;
    const bool lead = pairs_ok && ok && (tid & 1) == 0 && lane != 31 && tid + 1 < nu && un == u + 1 && (u & 1) == 0;
    const bool led = __shfl_up_sync(0xffffffffu, lead ? 1 : 0, 1) != 0 && (tid & 1) == 1;
    if (tid < nu && !led) {
      const float2* src = ok ? dat + u : dat;
#pragma unroll
      for (int c = 0; c < CP; ++c) {
        if (!(FULLC || c < C)) continue;
        if (lead)
          cp16_cg(xs + c * XS + tid, src + static_cast<int64_t>(c) * N);
        else
          cp8(xs + c * XS + tid, ok ? src + static_cast<int64_t>(c) * N : dat, ok ? 8 : 0);
      }
    }
  };

  auto prefetch_x = [&](int4 d, int u) {  // samples' coils of sub-chunk d into L2
    if (tid < n_slots(d, cap) && u >= 0 && u < N) {
      const float2* src = dat + u;
#pragma unroll
      for (int c = 0; c < CP; ++c)
        if (FULLC || c < C) prefetch_l2(src + static_cast<int64_t>(c) * N);
    }
  };

  Stream st;
  st.init(sd, si, p0, p1);
  stage_x(st.d0, ld_u(st.d0, true), xs0);
  stage_meta(meta, wts, st.d0, cap, ms0, ws0);
  commit();
  // staging slots of sub-chunks p + 1 (staged this iteration) and p + 2
  // (prefetched into L2 this iteration), loaded two and one iterations ahead
  int u1 = ld_u(st.d1, st.p + 1 < p1);
  int u2 = ld_u(st.d2, st.p + 2 < p1);
  uint4* wsm = reinterpret_cast<uint4*>(base + lay.wf);
  stage_w<CP, NS>(reinterpret_cast<uint32_t*>(wsm), wfrag);
  stage_phases(dt, dtab, CP, NS, nsteps, ph);
  for (int i = tid; i < lay.tile_sz; i += kT) tile[i] = make_float2(0.f, 0.f);
  if (TMA) fence_proxy_async();  // the cleared tile -> visible to tensor-copy stores

  int buf = 0;
  while (true) {
    const bool more = st.p + 1 < p1;
    if (more) {
      if (st.p + 2 < p1) {
        prefetch_x(st.d2, u2);
        prefetch_meta(meta, wts, st.d2, cap);
      }
      wait_groups<0>();  // sub-chunk p's copies (issued during iteration p - 1)
    } else {
      wait_groups<0>();
    }
    const int u3 = ld_u(st.d3, st.p + 3 < p1);
    __syncthreads();  // staging buffer `buf` complete; tile zeroed / flushed
    // block-uniform; an item's first sub-chunk follows a flush (or the start)
    const int zn = (TMA && (st.i0.y & kFirst)) ? min(kZeroPerFlush, zleft) : 0;
    if (TMA && zn > 0) {
      if (tid == 0) {
        const int z = z_next;
        for (int k = 0; k < zn; ++k) {
          int z0, y0, x0;
          origin(geom, __ldg(zempty + z + k), z0, y0, x0);
          tma_store_tile(&tmap, 2 * x0, y0, z0, b * C, tile, false);
        }
        z_next = z + zn;
      }
      zleft -= zn;
    }
    {
      const int nr = n_reps(st.d0, cap), nu = n_slots(st.d0, cap);
      const float2* xs = xs0 + buf * lay.xs_sz;
      const int2* msb = ms0 + buf * cap;
      const float* wsb = ws0 + buf * cap;
      constexpr int NTL = Shape<CP>::NTL;
      Row rw[NTL][2];
      float2 v[NTL][2][NT];
      const bool act = warp * 16 < nr;  // warp-uniform: m-tiles warp (and warp + 8 up to 16 coils)
      if (act) {
#pragma unroll
        for (int T = 0; T < NTL; ++T)
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            const int e = (warp + 8 * T) * 16 + 2 * g + r;  // cell-ordered rows: entry 2 g + r on row g + 8 r
            const bool in = e < nr;
            rw[T][r] = decode<NS>(in ? msb[e] : make_int2(-1, 0), in ? wsb[e] : 0.f, in, cells, nu, nsteps);
#pragma unroll
            for (int m = 0; m < NT; ++m) {
              const int c = 4 * m + t;
              v[T][r][m] = (rw[T][r].on && (FULLC || c < C)) ? xs[c * XS + rw[T][r].slot] : make_float2(0.f, 0.f);
            }
          }
        chain<CP, NS, TERMS, false>(v, wsm, dtl, nsteps, ph.stride, rw, lane);
      }
      // the next sub-chunk's copies go out between the chain and the row sums:
      // issued at the top of the iteration they competed with the chain's
      // shared-memory traffic for the load/store pipe (1.4% slower at 192^3)
      if (more) {
        stage_x(st.d1, u1, xs0 + (buf ^ 1) * lay.xs_sz);
        stage_meta(meta, wts, st.d1, cap, ms0 + (buf ^ 1) * cap, ws0 + (buf ^ 1) * cap);
        commit();
      }
      if (TMA && zn > 0) {  // the clearing stores have read the tile before it takes row sums
        if (tid == 0) bulk_wait_read_all();
        __syncthreads();
      }
      if (act) {
#pragma unroll
        for (int T = 0; T < NTL; ++T) {
          if ((warp + 8 * T) * 16 >= nr) break;  // warp-uniform
#pragma unroll
          for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int m = 0; m < NT; ++m) v[T][r][m] = cscale(v[T][r][m], rw[T][r].w);
          reduce_rows_to_tile<CP, FULLC, TMA>(v[T], rw[T], C, tile, cells, g, t);
          __syncwarp();
        }
      }
    }
    if (TMA) fence_proxy_async();  // this thread's tile writes -> visible to the tensor-copy store
    __syncthreads();  // tile complete for this sub-chunk; staging buffer `buf` free
    if (TMA && (st.i0.y & kLast)) {  // one tensor store (reduce-add for split bricks) per brick
      if (tid == 0) {
        int z0, y0, x0;
        origin(geom, st.i0.x, z0, y0, x0);
        tma_store_tile(&tmap, 2 * x0, y0, z0, b * C, tile, (st.i0.y & kSplit) != 0);
        bulk_wait_read_all();  // the tile has been read out: it can be cleared
      }
      __syncthreads();
      float4* t4 = reinterpret_cast<float4*>(tile);
      for (int i = tid; i < (C * cells) / 2; i += kT) t4[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (zleft > 0) fence_proxy_async();  // the cleared tile -> visible to the clearing stores
    } else if (st.i0.y & kLast) {
      int z0, y0, x0;
      origin(geom, st.i0.x, z0, y0, x0);
      const bool split = (st.i0.y & kSplit) != 0;
      for (int cl = tid; cl < cells; cl += kT) {  // one cell per thread, all coils
        int64_t flat;
        const bool in = flat_of(geom, z0, y0, x0, cl, flat);
        float2* trow = tile + cl * TS;
        float2* dst = grd + (in ? flat : 0);
#pragma unroll
        for (int c = 0; c < CP; ++c) {
          if (!FULLC && c >= C) break;
          const float2 v = trow[c];
          trow[c] = make_float2(0.f, 0.f);  // this thread re-zeroes what it flushed
          if (in) {
            if (split) {
              if (v.x != 0.f || v.y != 0.f) {
                atomicAdd(&dst->x, v.x);
                atomicAdd(&dst->y, v.y);
              }
            } else {
              *dst = v;
            }
          }
          dst += G;
        }
      }
    }
    if (!more) break;
    st.advance();
    u1 = u2;
    u2 = u3;
    buf ^= 1;
  }
  if (TMA && zleft > 0 && (st.i0.y & kLast)) {  // the last sub-chunk flushed its brick: the tile is clear
    __syncthreads();
    if (tid == 0)
      for (int k = z_next; k < z_next + zleft; ++k) {
        int z0, y0, x0;
        origin(geom, __ldg(zempty + k), z0, y0, x0);
        tma_store_tile(&tmap, 2 * x0, y0, z0, b * C, tile, false);
      }
  }
  if (TMA && tid == 0) bulk_wait_all();
}

template <int CP, int NS, int TERMS, bool ACC, bool FULLC, bool TMA>
__global__ void __launch_bounds__(kT, Regs<CP, NS>::MINB) grog_degrid_tc_kernel(
    const float2* __restrict__ grid, int64_t G, float2* __restrict__ out, int64_t N, int C,
    const uint32_t* __restrict__ wfrag, const float2* __restrict__ dtab, int nsteps, const int4* __restrict__ sd,
    const int2* __restrict__ si, const int32_t* __restrict__ cta_ptr, const int32_t* __restrict__ uniq,
    const int2* __restrict__ meta, const float* __restrict__ wts, int cap, Geom geom,
    const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) float4 smem4[];
  constexpr int NT = Shape<CP>::NT, TS = CP;  // tiles filled by cp.async: plain stride
  const int p0 = cta_ptr[blockIdx.x], p1 = cta_ptr[blockIdx.x + 1];
  if (p0 >= p1) return;
  const int cells = geom.bz * geom.by * geom.bx;
  const Smem lay(CP, NS, nsteps, cells, cap, false, TMA);
  uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<float2*>(smem4) + lay.bar);
  unsigned phase = 0;  // bit k: parity of the next completion of bars[k]
  unsigned pend = 0;   // bit k: a tensor copy into tile buffer k has been issued and not yet waited for
  __shared__ int s_ok;
  const int XS = cap + 4;
  float2* base = reinterpret_cast<float2*>(smem4);
  float2* dt = base + lay.dt;
  float2* tiles = base + lay.tile;  // 2 x (cells, TS)
  float2* res = base + lay.xs;      // (CP, XS) per-slot results
  int2* ms0 = reinterpret_cast<int2*>(base + lay.ms);
  float* ws0 = reinterpret_cast<float*>(base + lay.wsm);
  const Phases ph(CP, NS, nsteps);
  const int b = blockIdx.y;
  const float2* grd = grid + static_cast<int64_t>(b) * C * G;
  float2* o = out + static_cast<int64_t>(b) * C * N;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const float2* dtl = dt + (ph.copies == 4 ? (g & 3) * ph.copy_sz : 0);  // this lane's phase copy

  auto issue_tile = [&](int brick, float2* tl, int k) {  // brick tile of all coils into buffer k
    int z0, y0, x0;
    origin(geom, brick, z0, y0, x0);
    if (TMA) {  // one tensor copy, completion on bars[k]
      if (tid == 0) {
        fence_proxy_async();  // earlier reads of this buffer precede the copy
        mbar_expect_tx(bars + k, static_cast<unsigned>(C * cells * 8));
        tma_load_tile(tl, &tmap, 2 * x0, y0, z0, b * C, bars + k);
      }
      pend |= 1u << k;  // block-uniform bookkeeping
      return;
    }
    for (int cl = tid; cl < cells; cl += kT) {
      int64_t flat;
      const bool in = flat_of(geom, z0, y0, x0, cl, flat);
      const float2* src = grd + (in ? flat : 0);
#pragma unroll
      for (int c = 0; c < CP; ++c)
        if (FULLC || c < C) cp8(tl + cl * TS + c, in ? src + static_cast<int64_t>(c) * G : grd, in ? 8 : 0);
    }
  };
  auto ld_u = [&](int4 d, bool valid) -> int {
    return (valid && tid < n_slots(d, cap)) ? __ldg(uniq + d.z + tid) : -1;
  };
  auto prefetch_tile = [&](int brick) {  // brick tile into L2
    int z0, y0, x0;
    origin(geom, brick, z0, y0, x0);
    for (int cl = tid; cl < cells; cl += kT) {
      int64_t flat;
      if (!flat_of(geom, z0, y0, x0, cl, flat)) continue;
      if ((cl & (geom.bx - 1)) != 0 && ((flat & 15) != 0)) continue;  // one prefetch per 128-byte line
      const float2* src = grd + flat;
#pragma unroll
      for (int c = 0; c < CP; ++c)
        if (FULLC || c < C) prefetch_l2(src + static_cast<int64_t>(c) * G);
    }
  };

  if (TMA) {
    if (tid == 0) {
      mbar_init(bars, 1);
      mbar_init(bars + 1, 1);
      mbar_fence_init();
    }
    __syncthreads();
  }
  Stream st;
  st.init(sd, si, p0, p1);
  int par = 0, mb = 0;
  issue_tile(st.i0.x, tiles, 0);
  stage_meta(meta, wts, st.d0, cap, ms0, ws0);
  commit();
  uint4* wsm = reinterpret_cast<uint4*>(base + lay.wf);
  stage_w<CP, NS>(reinterpret_cast<uint32_t*>(wsm), wfrag);
  stage_phases(dt, dtab, CP, NS, nsteps, ph);
  for (int i = tid; i < lay.xs_sz; i += kT) res[i] = make_float2(0.f, 0.f);
  int u0 = ld_u(st.d0, true);

  while (true) {
    const bool more = st.p + 1 < p1;
    const bool last = (st.i0.y & kLast) != 0;
    if (more) {  // next sub-chunk's metadata (and next brick's tile) during this compute
      if (last) issue_tile(st.i1.x, tiles + (par ^ 1) * lay.tile_sz, par ^ 1);
      stage_meta(meta, wts, st.d1, cap, ms0 + (mb ^ 1) * cap, ws0 + (mb ^ 1) * cap);
      commit();
      if (st.p + 2 < p1) {  // sub-chunk p + 2 into L2: its metadata and, if it starts an item, its tile
        if (st.i2.y & kFirst) prefetch_tile(st.i2.x);
        prefetch_meta(meta, wts, st.d2, cap);
      }
      wait_groups<1>();
    } else {
      wait_groups<0>();
    }
    const int u1 = ld_u(st.d1, more);
    const bool wait_tile = TMA && (st.i0.y & kFirst);  // this item's tile: its tensor copy
    if (wait_tile && tid == 0) {
      s_ok = mbar_wait(bars + par, (phase >> par) & 1) ? 1 : 0;
      if (!s_ok) {  // give up on this CTA, but let every copy still in flight land first
        for (int k = 0; k < 2; ++k)
          if (pend & (1u << k)) mbar_drain(bars + k, (phase >> k) & 1);
      }
    }
    __syncthreads();  // tile of this brick complete; previous results flushed
    if (wait_tile) {
      if (!s_ok) {  // block-uniform: the copy did not complete in time (counted in g_tc_timeouts)
        wait_groups<0>();  // this thread's metadata copies, too
        return;
      }
      phase ^= 1u << par;
      pend &= ~(1u << par);
    }
    {
      const int nr = n_reps(st.d0, cap), nu = n_slots(st.d0, cap);
      const float2* tl = tiles + par * lay.tile_sz;
      const int2* msb = ms0 + mb * cap;
      const float* wsb = ws0 + mb * cap;
      if (warp * 16 < nr) {  // warp-uniform: m-tiles warp (and warp + 8 up to 16 coils)
        constexpr int NTL = Shape<CP>::NTL;
        Row rw[NTL][2];
        float2 v[NTL][2][NT];
#pragma unroll
        for (int T = 0; T < NTL; ++T)
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            const int e = (warp + 8 * T) * 16 + 8 * r + g;  // sample-ordered rows: entry 8 r + g on row g + 8 r
            const bool in = e < nr;
            rw[T][r] = decode<NS>(in ? msb[e] : make_int2(-1, 0), in ? wsb[e] : 0.f, in, cells, nu, nsteps);
#pragma unroll
            for (int m = 0; m < NT; ++m) {
              const int c = 4 * m + t;
              v[T][r][m] = (rw[T][r].on && (FULLC || c < C))
                               ? tl[TMA ? c * cells + rw[T][r].cell : rw[T][r].cell * TS + c]
                               : make_float2(0.f, 0.f);
            }
          }
        chain<CP, NS, TERMS, true>(v, wsm, dtl, nsteps, ph.stride, rw, lane);
#pragma unroll
        for (int T = 0; T < NTL; ++T)
#pragma unroll
          for (int r = 0; r < 2; ++r) {
            if (!rw[T][r].on) continue;
#pragma unroll
            for (int m = 0; m < NT; ++m) {
              const int c = 4 * m + t;
              if (FULLC || c < C) {
                float2* dst = res + c * XS + rw[T][r].slot;
                const float2 y = cscale(v[T][r][m], rw[T][r].w);
                if (ACC) {
                  atomicAdd(&dst->x, y.x);
                  atomicAdd(&dst->y, y.y);
                } else {
                  *dst = y;
                }
              }
            }
          }
      }
    }
    __syncthreads();  // results complete; this brick's tile no longer read
    if (tid < n_slots(st.d0, cap)) {
      const bool ok = u0 >= 0 && u0 < N;
      float2* dst = o + (ok ? u0 : 0);
#pragma unroll
      for (int c = 0; c < CP; ++c) {
        if (!FULLC && c >= C) break;
        float2* rv = res + c * XS + tid;
        const float2 v = *rv;
        if (ACC) *rv = make_float2(0.f, 0.f);  // this thread re-clears what it flushed
        if (ok) {
          if (ACC) {
            atomicAdd(&dst->x, v.x);
            atomicAdd(&dst->y, v.y);
          } else {
            *dst = v;
          }
        }
        dst += N;
      }
    }
    if (!more) break;
    if (last) par ^= 1;
    mb ^= 1;
    st.advance();
    u0 = u1;
  }
}

__global__ void zero_bricks_tc(float2* __restrict__ grid, int64_t G, int C, int B,
                               const int32_t* __restrict__ bricks, int n_bricks, Geom geom) {
  const int cells = geom.bz * geom.by * geom.bx;
  const int64_t total = static_cast<int64_t>(n_bricks) * cells;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int bi = static_cast<int>(i / cells);
    const int cl = static_cast<int>(i - static_cast<int64_t>(bi) * cells);
    int z0, y0, x0;
    origin(geom, bricks[bi], z0, y0, x0);
    int64_t flat;
    if (!flat_of(geom, z0, y0, x0, cl, flat)) continue;
    for (int b = 0; b < B; ++b)
      for (int c = 0; c < C; ++c) grid[(static_cast<int64_t>(b) * C + c) * G + flat] = make_float2(0.f, 0.f);
  }
}

__global__ void zero_samples_tc(float2* __restrict__ out, int64_t N, int C, int B, const int32_t* __restrict__ src,
                                int64_t n) {
  const int64_t total = n * C * B;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t k = i % n;
    const int64_t bc = i / n;
    const int64_t s = src[k];
    if (s >= 0 && s < N) out[bc * N + s] = make_float2(0.f, 0.f);
  }
}

// coil padding of the kernels: multiples of 4 up to 16, of 8 above (24, 32)
inline int padded(int64_t C) { return static_cast<int>(C <= 16 ? (C + 3) / 4 * 4 : (C + 7) / 8 * 8); }
// entries of one sub-chunk: 8 warps x 16 rows x the m-tiles a warp runs (Shape<CP>::NTL)
inline int tc_rows(int64_t C) { return padded(C) <= 16 ? 2 * 8 * 16 : 8 * 16; }

static int geom_of(const pgb_v6_plan* p, Geom& g, const char* who) {
  PGB_REQUIRE(p != nullptr, PGB_ERR_INVALID, "%s: null plan", who);
  auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
  PGB_REQUIRE(pow2(p->bz) && pow2(p->by) && pow2(p->bx) && p->gz >= 1 && p->gy >= 1 && p->gx >= 1,
              PGB_ERR_INVALID, "%s: brick extents must be powers of two", who);
  const int64_t cells = static_cast<int64_t>(p->bz) * p->by * p->bx;
  PGB_REQUIRE(cells <= 4096, PGB_ERR_RANGE, "%s: brick of %lld cells exceeds 4096", who, (long long)cells);
  PGB_REQUIRE(p->nbz == (p->gz + p->bz - 1) / p->bz && p->nby == (p->gy + p->by - 1) / p->by &&
                  p->nbx == (p->gx + p->bx - 1) / p->bx,
              PGB_ERR_INVALID, "%s: brick counts do not match the grid", who);
  PGB_REQUIRE(p->n_cta >= 0 && p->n_cta <= 65535 && p->sub_cap >= 1 && p->sub_cap <= kT, PGB_ERR_INVALID,
              "%s: invalid CTA count or sub-chunk capacity (1..%d)", who, kT);
  PGB_REQUIRE(p->n_cta == 0 || (p->cta_ptr && p->sd && p->si && p->uniq && p->meta && p->w), PGB_ERR_INVALID,
              "%s: null plan arrays", who);
  int lbx = 0, lby = 0;
  while ((1 << lbx) < p->bx) ++lbx;
  while ((1 << lby) < p->by) ++lby;
  g = Geom{p->gz, p->gy, p->gx, p->bz, p->by, p->bx, lbx, lby, p->nbz, p->nby, p->nbx};
  return PGB_OK;
}

static int check_common(const char* who, int64_t C, int64_t N, int64_t B, int64_t nsteps, int64_t ndim,
                        int64_t terms, const void* wfrag, const void* dtab) {
  PGB_REQUIRE(C >= 1 && C <= 32, PGB_ERR_UNSUPPORTED, "%s: ncoils must be 1..32, got %lld", who, (long long)C);
  PGB_REQUIRE(ndim == 2 || ndim == 3, PGB_ERR_INVALID, "%s: ndim must be 2 or 3", who);
  PGB_REQUIRE(terms == 1 || terms == 3, PGB_ERR_INVALID, "%s: terms must be 1 (bf16) or 3 (bf16x3)", who);
  PGB_REQUIRE(nsteps >= 1 && nsteps <= (ndim == 3 ? 255 : 65535), PGB_ERR_RANGE, "%s: invalid nsteps %lld", who,
              (long long)nsteps);
  PGB_REQUIRE(N >= 0 && N < (int64_t(1) << 31) && B >= 0 && B <= 65535, PGB_ERR_RANGE, "%s: invalid N/B", who);
  PGB_REQUIRE(wfrag != nullptr && dtab != nullptr, PGB_ERR_INVALID, "%s: null fragment or phase table", who);
  return PGB_OK;
}

}  // namespace tc
}  // namespace pgb

using namespace pgb;
using namespace pgb::tc;

namespace {

bool g_use_tma = true;

// Tensor map of the grid (B, C, gz, gy, gx) complex64 as float32 {2 gx, gy, gz, B C}
// with one brick of all coils per box.  False when the layout cannot be
// described (odd gx or brick width, unaligned base) or the driver entry point
// is missing; the kernels then stage tiles with per-element copies.
bool make_tile_map(CUtensorMap* map, const void* grid, const pgb_v6_plan* p, int64_t C, int64_t B) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static bool looked_up = false;
  if (!g_use_tma) return false;
  if (!looked_up) {
    looked_up = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    else
      cudaGetLastError();
  }
  if (encode == nullptr) return false;
  if ((p->gx & 1) || (p->bx & 1) || (reinterpret_cast<uintptr_t>(grid) & 15) != 0) return false;
  if (2 * p->bx > 256 || p->by > 256 || p->bz > 256 || C > 256 || B * C > (int64_t(1) << 31)) return false;
  const cuuint64_t gx = p->gx, gy = p->gy, gz = p->gz;
  cuuint64_t dims[4] = {2 * gx, gy, gz, static_cast<cuuint64_t>(B * C)};
  cuuint64_t strides[3] = {gx * 8, gx * gy * 8, gx * gy * gz * 8};
  cuuint32_t box[4] = {static_cast<cuuint32_t>(2 * p->bx), static_cast<cuuint32_t>(p->by),
                       static_cast<cuuint32_t>(p->bz), static_cast<cuuint32_t>(C)};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(grid), dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t tc_smem(int64_t C, int cells, int64_t nsteps, int64_t ndim, int cap, bool fwd, bool tma) {
  return static_cast<size_t>(Smem(padded(C), static_cast<int>(ndim), static_cast<int>(nsteps), cells, cap, fwd, tma)
                                 .total) *
         sizeof(float2);
}

}  // namespace

#define PGB_TC_DISPATCH(X) \
  X(4, 2) X(4, 3) X(8, 2) X(8, 3) X(12, 2) X(12, 3) X(16, 2) X(16, 3) X(24, 2) X(24, 3) X(32, 2) X(32, 3)

extern "C" {

size_t pgb_grog_tc_smem_bytes(int64_t C, int64_t cells, int64_t nsteps, int64_t ndim, int64_t sub_cap) {
  if (C < 1 || C > 32 || cells < 1 || cells > 4096 || nsteps < 1 || nsteps > 65535 || (ndim != 2 && ndim != 3) ||
      sub_cap < 1 || sub_cap > kT)
    return ~static_cast<size_t>(0);
  const int CP = padded(C), NS = static_cast<int>(ndim);
  size_t m = 0;
  for (int tma = 0; tma < 2; ++tma)
    for (int fwd = 0; fwd < 2; ++fwd) {
      const size_t v = Smem(CP, NS, static_cast<int>(nsteps), static_cast<int>(cells), static_cast<int>(sub_cap),
                            fwd != 0, tma != 0).total;
      m = v > m ? v : m;
    }
  return m * sizeof(float2);
}

int pgb_grog_tc_blocks_per_sm(int64_t C, int64_t ndim) {
  if (C < 1 || C > 32 || (ndim != 2 && ndim != 3)) return 0;
  switch (padded(C) * 10 + static_cast<int>(ndim)) {
#define X(CP, NS) \
  case CP * 10 + NS: \
    return Regs<CP, NS>::MINB;
    PGB_TC_DISPATCH(X)
#undef X
    default:
      return 0;
  }
}

int pgb_grog_grid_tc(const void* data, int64_t N, void* grid, int64_t G, const void* wfrag, const void* dtab,
                     int64_t nsteps, int64_t ndim, int64_t C, int64_t B, int64_t terms, const pgb_v6_plan* plan,
                     void* stream) {
  const char* who = "grog_grid_tc";
  clear_error();
  Geom geom;
  int st = geom_of(plan, geom, who);
  if (st) return st;
  st = check_common(who, C, N, B, nsteps, ndim, terms, wfrag, dtab);
  if (st) return st;
  PGB_REQUIRE(G == static_cast<int64_t>(plan->gz) * plan->gy * plan->gx, PGB_ERR_INVALID,
              "%s: G does not match the plan grid", who);
  PGB_REQUIRE(ndim == 3 || plan->gz == 1, PGB_ERR_INVALID, "%s: a 2-D table needs a 2-D plan", who);
  PGB_REQUIRE(plan->sub_cap <= tc_rows(C), PGB_ERR_INVALID, "%s: sub-chunks of %d coils hold at most %d entries",
              who, padded(C), tc_rows(C));
  if (B == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(grid && (data || N == 0), PGB_ERR_INVALID, "%s: null pointer", who);
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = pgb_grog_tc_smem_bytes(C, cells, nsteps, ndim, plan->sub_cap);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED, "%s: tile + staging need %zu B of shared memory", who, smem);
  PGB_REQUIRE(plan->n_zero_bricks >= 0 && plan->n_empty_tail >= 0 && plan->n_empty_tail <= plan->n_zero_bricks,
              PGB_ERR_INVALID, "%s: bad zero-brick counts", who);
  PGB_REQUIRE(plan->n_zero_bricks == 0 || plan->zero_bricks != nullptr, PGB_ERR_INVALID, "%s: null zero-brick list",
              who);
  cudaStream_t s = as_stream(stream);
  CUtensorMap tmap;
  memset(&tmap, 0, sizeof(tmap));
  const bool tma = plan->n_cta > 0 && C == padded(C) && make_tile_map(&tmap, grid, plan, C, B);
  // empty bricks at the end of the list are cleared by the gridding CTAs on
  // the tensor-copy path; the rest (split bricks, which take reduce-adds) first
  const int n_tail = tma ? plan->n_empty_tail : 0;
  const int n_pre = plan->n_zero_bricks - n_tail;
  if (n_pre > 0) {
    const int64_t tot = static_cast<int64_t>(n_pre) * cells;
    zero_bricks_tc<<<grid_for(tot, 256, 148 * 16), 256, 0, s>>>(static_cast<float2*>(grid), G, static_cast<int>(C),
                                                               static_cast<int>(B), plan->zero_bricks, n_pre, geom);
    PGB_LAUNCH_CHECK(who);
  }
  if (plan->n_cta == 0) return PGB_OK;
  dim3 grd(plan->n_cta, static_cast<unsigned>(B));
  const size_t smem_k = tc_smem(C, cells, nsteps, ndim, plan->sub_cap, true, tma);
  const int key = padded(C) * 10 + static_cast<int>(ndim);
  switch (key) {
#define X(CP, NS)                                                                                               \
  case CP * 10 + NS: {                                                                                          \
    const bool full = C == CP;                                                                                  \
    auto k = terms == 3 ? (tma ? grog_grid_tc_kernel<CP, NS, 3, true, true>                                     \
                               : (full ? grog_grid_tc_kernel<CP, NS, 3, true, false> : grog_grid_tc_kernel<CP, NS, 3, false, false>)) \
                        : (tma ? grog_grid_tc_kernel<CP, NS, 1, true, true>                                     \
                               : (full ? grog_grid_tc_kernel<CP, NS, 1, true, false> : grog_grid_tc_kernel<CP, NS, 1, false, false>)); \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_k);                          \
    k<<<grd, kT, smem_k, s>>>(static_cast<const float2*>(data), N, static_cast<float2*>(grid), G,               \
                              static_cast<int>(C), static_cast<const uint32_t*>(wfrag),                         \
                              static_cast<const float2*>(dtab), static_cast<int>(nsteps),                       \
                              reinterpret_cast<const int4*>(plan->sd), reinterpret_cast<const int2*>(plan->si),  \
                              plan->cta_ptr, plan->uniq, reinterpret_cast<const int2*>(plan->meta), plan->w,     \
                              plan->sub_cap, geom, tmap, plan->zero_bricks + n_pre, n_tail);                    \
  } break;
    PGB_TC_DISPATCH(X)
#undef X
    default:
      PGB_REQUIRE(false, PGB_ERR_UNSUPPORTED, "%s: no kernel for C=%lld ndim=%lld", who, (long long)C,
                  (long long)ndim);
  }
  PGB_LAUNCH_CHECK(who);
  return PGB_OK;
}

}  // extern "C"

namespace {

int degrid_tc_one(const char* who, const void* grid, int64_t G, void* out, int64_t N, const void* wfrag,
                  const void* dtab, int64_t nsteps, int64_t ndim, int64_t C, int64_t B, int64_t terms,
                  const pgb_v6_plan* plan, const Geom& geom, bool acc, cudaStream_t s) {
  if (plan->n_cta == 0) return PGB_OK;
  const int cells = plan->bz * plan->by * plan->bx;
  const size_t smem = pgb_grog_tc_smem_bytes(C, cells, nsteps, ndim, plan->sub_cap);
  PGB_REQUIRE(smem <= 227 * 1024, PGB_ERR_UNSUPPORTED, "%s: tiles + results need %zu B of shared memory", who, smem);
  dim3 grd(plan->n_cta, static_cast<unsigned>(B));
  CUtensorMap tmap;
  memset(&tmap, 0, sizeof(tmap));
  const bool tma = C == padded(C) && make_tile_map(&tmap, grid, plan, C, B);
  const size_t smem_k = tc_smem(C, cells, nsteps, ndim, plan->sub_cap, false, tma);
  const int key = padded(C) * 10 + static_cast<int>(ndim);
  switch (key) {
#define PGB_TC_DEG(P, Q, T3, A)                                                                                 \
  (tma ? grog_degrid_tc_kernel<P, Q, T3, A, true, true>                                                         \
       : (full ? grog_degrid_tc_kernel<P, Q, T3, A, true, false> : grog_degrid_tc_kernel<P, Q, T3, A, false, false>))
#define X(CP, NS)                                                                                               \
  case CP * 10 + NS: {                                                                                          \
    const bool full = C == CP;                                                                                  \
    auto k = terms == 3 ? (acc ? PGB_TC_DEG(CP, NS, 3, true) : PGB_TC_DEG(CP, NS, 3, false))                    \
                        : (acc ? PGB_TC_DEG(CP, NS, 1, true) : PGB_TC_DEG(CP, NS, 1, false));                   \
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_k);                          \
    k<<<grd, kT, smem_k, s>>>(static_cast<const float2*>(grid), G, static_cast<float2*>(out), N,                \
                              static_cast<int>(C), static_cast<const uint32_t*>(wfrag),                         \
                              static_cast<const float2*>(dtab), static_cast<int>(nsteps),                       \
                              reinterpret_cast<const int4*>(plan->sd), reinterpret_cast<const int2*>(plan->si),  \
                              plan->cta_ptr, plan->uniq, reinterpret_cast<const int2*>(plan->meta), plan->w,     \
                              plan->sub_cap, geom, tmap);                                                       \
  } break;
    PGB_TC_DISPATCH(X)
#undef X
#undef PGB_TC_DEG
    default:
      PGB_REQUIRE(false, PGB_ERR_UNSUPPORTED, "%s: no kernel for C=%lld ndim=%lld", who, (long long)C,
                  (long long)ndim);
  }
  PGB_LAUNCH_CHECK(who);
  return PGB_OK;
}

}  // namespace

extern "C" {

int pgb_grog_degrid_tc(const void* grid, int64_t G, void* out, int64_t N, const void* wfrag_h, const void* dtab_h,
                       int64_t nsteps, int64_t ndim, int64_t C, int64_t B, int64_t terms,
                       const pgb_v6_plan* primary, const pgb_v6_plan* secondary, const int32_t* zero_src,
                       int64_t n_zero, void* stream) {
  const char* who = "grog_degrid_tc";
  clear_error();
  Geom geom;
  int st = geom_of(primary, geom, who);
  if (st) return st;
  Geom g2;
  if (secondary != nullptr) {
    st = geom_of(secondary, g2, who);
    if (st) return st;
    PGB_REQUIRE(secondary->bz == primary->bz && secondary->by == primary->by && secondary->bx == primary->bx &&
                    secondary->gz == primary->gz && secondary->gy == primary->gy && secondary->gx == primary->gx,
                PGB_ERR_INVALID, "%s: primary and secondary plans differ in geometry", who);
  }
  st = check_common(who, C, N, B, nsteps, ndim, terms, wfrag_h, dtab_h);
  if (st) return st;
  PGB_REQUIRE(n_zero >= 0 && (n_zero == 0 || zero_src != nullptr), PGB_ERR_INVALID, "%s: bad zero-sample list",
              who);
  PGB_REQUIRE(primary->sub_cap <= tc_rows(C) && (secondary == nullptr || secondary->sub_cap <= tc_rows(C)),
              PGB_ERR_INVALID, "%s: sub-chunks of %d coils hold at most %d entries", who, padded(C), tc_rows(C));
  PGB_REQUIRE(G == static_cast<int64_t>(primary->gz) * primary->gy * primary->gx, PGB_ERR_INVALID,
              "%s: G does not match the plan grid", who);
  PGB_REQUIRE(ndim == 3 || primary->gz == 1, PGB_ERR_INVALID, "%s: a 2-D table needs a 2-D plan", who);
  if (B == 0 || N == 0) return PGB_OK;
  PGB_REQUIRE(out && grid, PGB_ERR_INVALID, "%s: null pointer", who);
  cudaStream_t s = as_stream(stream);
  st = degrid_tc_one(who, grid, G, out, N, wfrag_h, dtab_h, nsteps, ndim, C, B, terms, primary, geom, false, s);
  if (st) return st;
  if (secondary != nullptr) {
    st = degrid_tc_one(who, grid, G, out, N, wfrag_h, dtab_h, nsteps, ndim, C, B, terms, secondary, g2, true, s);
    if (st) return st;
  }
  if (n_zero > 0) {
    zero_samples_tc<<<grid_for(n_zero * C * B, 256), 256, 0, s>>>(static_cast<float2*>(out), N, static_cast<int>(C),
                                                                  static_cast<int>(B), zero_src, n_zero);
    PGB_LAUNCH_CHECK(who);
  }
  return PGB_OK;
}

}  // extern "C"

extern "C" {

int pgb_grog_tc_use_tma(int64_t enable) {
  const int prev = g_use_tma ? 1 : 0;
  if (enable >= 0) g_use_tma = enable != 0;
  return prev;
}

int pgb_grog_tc_wait_limit(int64_t limit, int64_t* previous) {
  clear_error();
  PGB_REQUIRE(limit >= -1, PGB_ERR_INVALID, "grog_tc_wait_limit: limit must be >= 0, or -1 for the default");
  long long prev = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&prev, g_tc_wait_limit, sizeof(prev));
  PGB_REQUIRE(e == cudaSuccess, PGB_ERR_CUDA, "grog_tc_wait_limit: %s", cudaGetErrorString(e));
  if (previous) *previous = prev;
  const long long v = limit < 0 ? kSpinLimit : static_cast<long long>(limit);
  e = cudaMemcpyToSymbol(g_tc_wait_limit, &v, sizeof(v));
  PGB_REQUIRE(e == cudaSuccess, PGB_ERR_CUDA, "grog_tc_wait_limit: %s", cudaGetErrorString(e));
  return PGB_OK;
}

int pgb_grog_tc_timeouts(int64_t* count, int64_t reset) {
  clear_error();
  PGB_REQUIRE(count != nullptr, PGB_ERR_INVALID, "grog_tc_timeouts: null output");
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_timeouts, sizeof(int));
  PGB_REQUIRE(e == cudaSuccess, PGB_ERR_CUDA, "grog_tc_timeouts: %s", cudaGetErrorString(e));
  *count = v;
  if (reset) {
    const int z = 0;
    e = cudaMemcpyToSymbol(g_tc_timeouts, &z, sizeof(int));
    PGB_REQUIRE(e == cudaSuccess, PGB_ERR_CUDA, "grog_tc_timeouts: %s", cudaGetErrorString(e));
  }
  return PGB_OK;
}

}  // extern "C"
