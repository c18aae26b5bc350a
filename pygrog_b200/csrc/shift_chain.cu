// shift_chain.cu -- the eigen-factored GROG shift chain on R replicas, in two
// tensor-core forms, for measuring which MMA flavour the chain should use.
//
// The reference builds every per-axis fractional operator as expm(d logm G)
// (calib/_grappa.py:62-72, 184-208), so the table product applied to one
// replica is exactly
//     y = W3 Dx[k] W2 Dy[j] W1 Dz[i] W0 x
// with four dense C x C matrices shared by all replicas and three diagonal
// phases picked by the replica's per-axis shift indices (i, j, k).  The
// gridders of grog_tc.cu run this chain with mma.sync; this file runs the
// chain alone, without staging, row sums or brick tiles, so that the two MMA
// flavours can be compared on the same work:
//
//   variant 0 (mma.sync): one warp per 16-replica m-tile, m16n8k16 / m16n8k8
//     bf16 MMAs, each stage's FP32 accumulators handed on in registers as the
//     next stage's A fragments (the dataflow of grog_tc.cu);
//   variant 1 (tcgen05): one CTA of 128 threads per 128-replica tile, one
//     thread per replica row; each stage is tcgen05.mma (M = 128, N = K = 2C
//     rounded up to 16, one elected thread issues it) with the accumulator in
//     tensor memory; the threads read it back (tcgen05.ld), apply the phase,
//     split it into bf16 heads and tails and write them to shared memory in
//     the canonical K-major layout as the next stage's A operand.
//
// Both compute bf16x3 products (hi*hi + hi*lo + lo*hi) with FP32 accumulation.
// Layouts: x and out (2C, R) float, realified (row 2c = Re of coil c, 2c + 1 =
// Im); idx int32 per replica, i | j << 8 | k << 16 (each < kSteps, larger bytes
// read step kSteps - 1); W (4, 2C,
// 2C) float, realified [stage][output][input]; ph (3, kSteps, C) float2.
// rep > 1 applies the chain rep times per loaded tile, so that the chain's
// time can be separated from the loads and stores.  Every mbarrier wait is
// bounded; a wait that runs out adds to *timeouts and the kernel completes
// without waiting again, and waits (bounded) for its own MMAs before it frees
// its tensor memory.
#include <cuda_bf16.h>

#include <algorithm>

#include "common.cuh"

namespace pgb {
namespace chain {

constexpr int kSteps = 11;                // shift steps per axis (precision 1)
constexpr long long kChainSpin = 1 << 20;  // try_wait rounds per mbarrier wait

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t bf2_bits(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}
// (a, b) -> packed bf16 heads, packed bf16 tails (a in the low half)
__device__ __forceinline__ void split_pair(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = bf2_bits(a - hf.x, b - hf.y);
}
// Shift step of stage s packed in byte s of a replica's index word, clamped to
// the table (a caller's out-of-range byte reads the last step, never past the
// shared-memory phase table).
__device__ __forceinline__ int step_of(int packed, int s) { return min((packed >> (8 * s)) & 0xFF, kSteps - 1); }
__device__ __forceinline__ void cmul_inplace(float& re, float& im, float2 p) {
  const float r = re * p.x - im * p.y;
  im = re * p.y + im * p.x;
  re = r;
}

// ---- tcgen05 ---------------------------------------------------------------------
// Shared-memory matrix descriptor, K-major without swizzle: start address >> 4
// in bits [0,14), leading byte offset (between the two 8-element K halves of a
// K = 16 step) >> 4 in [16,30), stride byte offset (between 8-row groups) >> 4
// in [32,46), descriptor version 1 in [46,48), layout 0 (no swizzle) in [61,64).
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: FP32 accumulator (bits [4,6) = 1), bf16
// A and B ([7,10) = 1, [10,13) = 1), both K-major, N >> 3 in [17,23), M >> 4 in
// [24,29).
__host__ __device__ constexpr uint32_t f16_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(N >> 3) << 17) |
         (static_cast<uint32_t>(M >> 4) << 24);
}
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kChainSpin; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void async_proxy_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// 16 consecutive tensor-memory columns of this warp's 32 lanes -> registers
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// Shared memory of the tcgen05 chain for C coils (bytes): W heads / tails of
// the four stages and the A heads / tails, both in the canonical K-major
// layout (8-row x 16-byte core matrices; a K = 16 step is two core-matrix
// columns LBO apart, 8-row groups SBO = 128 bytes apart), the phase tables
// (row stride C + 1 float2: the 11 rows of a stage start in distinct banks),
// two mbarriers and the tensor-memory address.
template <int C>
struct TcLayout {
  static constexpr int NC = 2 * C;                // realified width
  static constexpr int KP = (NC + 15) / 16 * 16;  // K = N, padded to the MMA's K step
  static constexpr int KS = KP / 16;              // K steps
  static constexpr int W_PART = KP * KP * 2;      // one stage, heads or tails
  static constexpr int A_PART = 128 * KP * 2;     // 128 rows, heads or tails
  static constexpr int PHS = C + 1;
  static constexpr int A_OFF = 8 * W_PART;
  static constexpr int PH_OFF = A_OFF + 2 * A_PART;
  static constexpr int BAR_OFF = (PH_OFF + 3 * kSteps * PHS * 8 + 15) / 16 * 16;
  static constexpr int SLOT_OFF = BAR_OFF + 16;
  static constexpr int BYTES = SLOT_OFF + 16;
  static constexpr uint32_t COLS = KP < 32 ? 32u : static_cast<uint32_t>(KP);  // power of two >= 32
  static_assert(KP == 32 || KP == 64, "tensor-memory allocation needs a power of two");
};

template <int C>
__global__ void __launch_bounds__(128) chain_tcgen05_kernel(const float* __restrict__ x, const int* __restrict__ idx,
                                                            const float* __restrict__ W,
                                                            const float2* __restrict__ ph, float* __restrict__ out,
                                                            long long R, int rep, int* __restrict__ timeouts) {
  using L = TcLayout<C>;
  constexpr int NC = L::NC, KP = L::KP, KS = L::KS;
  constexpr uint32_t kIdesc = f16_idesc(128, KP);
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* Wb = sm;
  uint8_t* Ab = sm + L::A_OFF;
  float2* phs = reinterpret_cast<float2*>(sm + L::PH_OFF);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + L::BAR_OFF);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + L::SLOT_OFF);
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(slot)),
                 "r"(L::COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  for (int i = tid; i < 4 * KP * KP; i += 128) {
    const int s = i / (KP * KP), n = (i / KP) % KP, k = i % KP;
    const float v = (n < NC && k < NC) ? W[(s * NC + n) * NC + k] : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    const int off = (((k >> 4) * 2 + ((k >> 3) & 1)) * (KP / 8) + (n >> 3)) * 128 + (n & 7) * 16 + (k & 7) * 2;
    *reinterpret_cast<__nv_bfloat16*>(Wb + (2 * s) * L::W_PART + off) = h;
    *reinterpret_cast<__nv_bfloat16*>(Wb + (2 * s + 1) * L::W_PART + off) = l;
  }
  for (int i = tid; i < 3 * kSteps * C; i += 128) phs[(i / C) * L::PHS + (i % C)] = ph[i];
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bars)) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(bars + 1)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  async_proxy_fence();  // the W tiles are read by the tensor cores
  tc_before_sync();
  __syncthreads();
  tc_after_sync();
  const uint32_t tmem = *slot;
  const uint32_t bar = smem_addr(bars), bar_end = smem_addr(bars + 1);
  const uint32_t a_base = smem_addr(Ab), w_base = smem_addr(Wb);
  const uint32_t t_row = tmem + (static_cast<uint32_t>(warp * 32) << 16);  // this warp's 32 lanes
  uint32_t parity = 0;
  bool ok = true;
  const long long ntiles = (R + 127) / 128;
  const int rg = tid >> 3, ri = tid & 7;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long r = tile * 128 + tid;
    const bool valid = r < R;
    float v[KP];
#pragma unroll
    for (int k = 0; k < KP; ++k) v[k] = (valid && k < NC) ? x[k * R + r] : 0.f;
    const int pi = valid ? idx[r] : 0;
    for (int it = 0; it < rep; ++it) {
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        // this thread's A row as bf16 heads and tails, 16 bytes per (K step, K half)
#pragma unroll
        for (int ks = 0; ks < KS; ++ks)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            uint32_t hh[4], ll[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              const int k = ks * 16 + h * 8 + 2 * e;
              split_pair(v[k], v[k + 1], hh[e], ll[e]);
            }
            const int off = ((ks * 2 + h) * 16 + rg) * 128 + ri * 16;
            *reinterpret_cast<uint4*>(Ab + off) = make_uint4(hh[0], hh[1], hh[2], hh[3]);
            *reinterpret_cast<uint4*>(Ab + L::A_PART + off) = make_uint4(ll[0], ll[1], ll[2], ll[3]);
          }
        async_proxy_fence();
        tc_before_sync();
        __syncthreads();
        if (tid == 0) {
          tc_after_sync();
#pragma unroll
          for (int ks = 0; ks < KS; ++ks) {
            const uint64_t ah = kmajor_desc(a_base + ks * 4096, 2048, 128);
            const uint64_t al = kmajor_desc(a_base + L::A_PART + ks * 4096, 2048, 128);
            const uint64_t bh = kmajor_desc(w_base + (2 * s) * L::W_PART + ks * KP * 32, KP * 16, 128);
            const uint64_t bl = kmajor_desc(w_base + (2 * s + 1) * L::W_PART + ks * KP * 32, KP * 16, 128);
            tc_mma(tmem, ah, bh, kIdesc, ks > 0 ? 1u : 0u);
            tc_mma(tmem, ah, bl, kIdesc, 1u);
            tc_mma(tmem, al, bh, kIdesc, 1u);
          }
          tc_commit(bar);
        }
        if (ok && !bar_wait(bar, parity)) ok = false;  // after one timeout, wait no more
        parity ^= 1u;
        tc_after_sync();
        uint32_t u[KP];
#pragma unroll
        for (int q = 0; q < KP / 16; ++q) tmem_ld16(t_row + 16 * q, u + 16 * q);
        tmem_wait_ld();
#pragma unroll
        for (int k = 0; k < KP; ++k) v[k] = __uint_as_float(u[k]);
        if (s < 3) {
          const float2* prow = phs + (s * kSteps + step_of(pi, s)) * L::PHS;
#pragma unroll
          for (int c = 0; c < C; ++c) cmul_inplace(v[2 * c], v[2 * c + 1], prow[c]);
        }
      }
    }
    if (valid) {
#pragma unroll
      for (int k = 0; k < NC; ++k) out[k * R + r] = v[k];
    }
  }
  // every MMA of this CTA complete before its tensor memory is freed
  tc_before_sync();
  const int bad = __syncthreads_or(ok ? 0 : 1);
  if (tid == 0) {
    tc_after_sync();
    tc_commit(bar_end);
    if (bad || !bar_wait(bar_end, 0)) atomicAdd(timeouts, 1);
  }
  __syncthreads();
  if (warp == 0) {
    tc_after_sync();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(L::COLS) : "memory");
  }
}

// ---- mma.sync --------------------------------------------------------------------
__device__ __forceinline__ void mma_k16(float (&d)[4], const uint32_t (&a)[4], uint2 b) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}
__device__ __forceinline__ void mma_k8(float (&d)[4], const uint32_t (&a)[2], uint32_t b) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(b));
}

// Shared memory of the mma.sync chain: B fragments of the four stages, heads
// and tails, lane-contiguous (K = 16 steps: uint2 {b0, b1}; a trailing K = 8
// step: uint32 b0), then the phase tables (row stride C + 1 float2).
template <int C>
struct MmaLayout {
  static constexpr int NC = 2 * C;
  static constexpr int NT = NC / 8;         // n-tiles
  static constexpr int K16 = NC / 16;       // full K = 16 steps
  static constexpr int K8 = (NC % 16) / 8;  // one K = 8 step when 2C is not a multiple of 16
  static constexpr int PHS = C + 1;
  static constexpr int F8_OFF = 4 * 2 * K16 * NT * 32 * 8;
  static constexpr int PH_OFF = F8_OFF + 4 * 2 * K8 * NT * 32 * 4;
  static constexpr int BYTES = PH_OFF + 3 * kSteps * PHS * 8;
  static_assert(NC % 8 == 0, "coils must be a multiple of 4");
};

template <int C>
__global__ void __launch_bounds__(256) chain_mma_kernel(const float* __restrict__ x, const int* __restrict__ idx,
                                                        const float* __restrict__ W, const float2* __restrict__ ph,
                                                        float* __restrict__ out, long long R, int rep) {
  using L = MmaLayout<C>;
  constexpr int NC = L::NC, NT = L::NT, K16 = L::K16, K8 = L::K8;
  extern __shared__ __align__(1024) uint8_t sm[];
  uint2* wf = reinterpret_cast<uint2*>(sm);
  uint32_t* wf8 = reinterpret_cast<uint32_t*>(sm + L::F8_OFF);
  float2* phs = reinterpret_cast<float2*>(sm + L::PH_OFF);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  // b0 = W[s][8j + g][k0 + 2t .. +1], b1 = W[s][8j + g][k0 + 2t + 8 .. +9]
  for (int i = tid; i < 4 * (K16 + K8) * NT * 32; i += 256) {
    const int L_ = i & 31, j = (i >> 5) % NT, ks = ((i >> 5) / NT) % (K16 + K8), s = ((i >> 5) / NT) / (K16 + K8);
    const int gg = L_ >> 2, tt = L_ & 3;
    const float* row = W + (s * NC + 8 * j + gg) * NC + 16 * ks + 2 * tt;
    uint32_t h0, l0;
    split_pair(row[0], row[1], h0, l0);
    if (ks < K16) {
      uint32_t h1, l1;
      split_pair(row[8], row[9], h1, l1);
      wf[(((s * 2 + 0) * K16 + ks) * NT + j) * 32 + L_] = make_uint2(h0, h1);
      wf[(((s * 2 + 1) * K16 + ks) * NT + j) * 32 + L_] = make_uint2(l0, l1);
    } else {
      wf8[((s * 2 + 0) * NT + j) * 32 + L_] = h0;
      wf8[((s * 2 + 1) * NT + j) * 32 + L_] = l0;
    }
  }
  for (int i = tid; i < 3 * kSteps * C; i += 256) phs[(i / C) * L::PHS + (i % C)] = ph[i];
  __syncthreads();
  const long long nmt = (R + 15) / 16;
  for (long long mt = static_cast<long long>(blockIdx.x) * 8 + warp; mt < nmt;
       mt += static_cast<long long>(gridDim.x) * 8) {
    const long long r0 = mt * 16 + g, r1 = r0 + 8;
    const bool v0 = r0 < R, v1 = r1 < R;
    float acc[NT][4];  // (c0, c1): row g, columns 2t, 2t + 1 of n-tile j; (c2, c3): row g + 8
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        acc[j][e] = v0 ? x[(8 * j + 2 * t + e) * R + r0] : 0.f;
        acc[j][2 + e] = v1 ? x[(8 * j + 2 * t + e) * R + r1] : 0.f;
      }
    const int p0 = v0 ? idx[r0] : 0, p1 = v1 ? idx[r1] : 0;
    for (int it = 0; it < rep; ++it) {
#pragma unroll 1
      for (int s = 0; s < 4; ++s) {
        float d[NT][4];
#pragma unroll
        for (int j = 0; j < NT; ++j) d[j][0] = d[j][1] = d[j][2] = d[j][3] = 0.f;
        // the accumulators of n-tiles 2 ks and 2 ks + 1 are the A fragment of K step ks
#pragma unroll
        for (int ks = 0; ks < K16; ++ks) {
          uint32_t ah[4], al[4];
          split_pair(acc[2 * ks][0], acc[2 * ks][1], ah[0], al[0]);
          split_pair(acc[2 * ks][2], acc[2 * ks][3], ah[1], al[1]);
          split_pair(acc[2 * ks + 1][0], acc[2 * ks + 1][1], ah[2], al[2]);
          split_pair(acc[2 * ks + 1][2], acc[2 * ks + 1][3], ah[3], al[3]);
#pragma unroll
          for (int j = 0; j < NT; ++j) {
            const uint2 bh = wf[(((s * 2 + 0) * K16 + ks) * NT + j) * 32 + lane];
            const uint2 bl = wf[(((s * 2 + 1) * K16 + ks) * NT + j) * 32 + lane];
            mma_k16(d[j], al, bh);
            mma_k16(d[j], ah, bl);
            mma_k16(d[j], ah, bh);
          }
        }
        if constexpr (K8 > 0) {
          uint32_t ah[2], al[2];
          split_pair(acc[2 * K16][0], acc[2 * K16][1], ah[0], al[0]);
          split_pair(acc[2 * K16][2], acc[2 * K16][3], ah[1], al[1]);
#pragma unroll
          for (int j = 0; j < NT; ++j) {
            const uint32_t bh = wf8[((s * 2 + 0) * NT + j) * 32 + lane];
            const uint32_t bl = wf8[((s * 2 + 1) * NT + j) * 32 + lane];
            mma_k8(d[j], al, bh);
            mma_k8(d[j], ah, bl);
            mma_k8(d[j], ah, bh);
          }
        }
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
          for (int e = 0; e < 4; ++e) acc[j][e] = d[j][e];
        if (s < 3) {
          const float2* q0 = phs + (s * kSteps + step_of(p0, s)) * L::PHS;
          const float2* q1 = phs + (s * kSteps + step_of(p1, s)) * L::PHS;
#pragma unroll
          for (int j = 0; j < NT; ++j) {  // columns 2t, 2t + 1 of n-tile j: coil 4 j + t
            cmul_inplace(acc[j][0], acc[j][1], q0[4 * j + t]);
            cmul_inplace(acc[j][2], acc[j][3], q1[4 * j + t]);
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        if (v0) out[(8 * j + 2 * t + e) * R + r0] = acc[j][e];
        if (v1) out[(8 * j + 2 * t + e) * R + r1] = acc[j][2 + e];
      }
  }
}

// Resident CTAs of `kernel` for the whole device (at most per_sm_cap per SM),
// from the SM's shared memory, registers and threads.  (The occupancy query
// reports one CTA per SM for the kernels that allocate tensor memory, although
// two of the 32-coil tcgen05 CTAs run side by side; the limits are taken here
// directly.)
template <typename K>
int launch_blocks(K kernel, int threads, int smem, long long need, int per_sm_cap) {
  int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 0, threads_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, kernel);
  const int warps = (threads + 31) / 32;
  const int regs_warp = ((fa.numRegs > 0 ? fa.numRegs : 255) * 32 + 255) / 256 * 256;  // 256-register granules
  int nb = per_sm_cap;
  nb = std::min(nb, smem_sm / (smem + reserved));
  nb = std::min(nb, regs_sm / (regs_warp * warps));
  nb = std::min(nb, threads_sm / threads);
  if (nb < 1) nb = 1;
  const long long cap = static_cast<long long>(nb) * kNumSMs;
  return static_cast<int>(need < cap ? (need < 1 ? 1 : need) : cap);
}

template <int C>
int run_chain(const float* x, const int* idx, const float* W, const float2* ph, float* out, long long R, int rep,
              int variant, int* timeouts, cudaStream_t s) {
  const char* who = "shift_chain";
  if (variant == 1) {
    using L = TcLayout<C>;
    auto k = chain_tcgen05_kernel<C>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES);
    PGB_REQUIRE(e == cudaSuccess, PGB_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
    // resident CTAs per SM share its 512 tensor-memory columns
    const int blocks = launch_blocks(k, 128, L::BYTES, (R + 127) / 128, static_cast<int>(512 / L::COLS));
    k<<<blocks, 128, L::BYTES, s>>>(x, idx, W, ph, out, R, rep, timeouts);
  } else {
    using L = MmaLayout<C>;
    auto k = chain_mma_kernel<C>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES);
    PGB_REQUIRE(e == cudaSuccess, PGB_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
    const int blocks = launch_blocks(k, 256, L::BYTES, ((R + 15) / 16 + 7) / 8, 8);
    k<<<blocks, 256, L::BYTES, s>>>(x, idx, W, ph, out, R, rep);
  }
  PGB_LAUNCH_CHECK(who);
  return PGB_OK;
}

}  // namespace chain
}  // namespace pgb

using namespace pgb;

extern "C" {

int pgb_shift_chain(const void* x, const void* idx, const void* W, const void* ph, void* out, int64_t R, int64_t C,
                    int64_t rep, int64_t variant, void* timeouts, void* stream) {
  const char* who = "shift_chain";
  clear_error();
  PGB_REQUIRE(C == 12 || C == 32, PGB_ERR_UNSUPPORTED, "%s: built for 12 and 32 coils, got %lld", who, (long long)C);
  PGB_REQUIRE(variant == 0 || variant == 1, PGB_ERR_INVALID, "%s: variant must be 0 (mma.sync) or 1 (tcgen05)", who);
  PGB_REQUIRE(R >= 0 && rep >= 1 && rep <= 1024, PGB_ERR_INVALID, "%s: need R >= 0 and 1 <= rep <= 1024", who);
  if (R == 0) return PGB_OK;
  PGB_REQUIRE(x && idx && W && ph && out, PGB_ERR_INVALID, "%s: null pointer", who);
  PGB_REQUIRE(variant == 0 || timeouts, PGB_ERR_INVALID, "%s: the tcgen05 variant needs a timeout counter", who);
  const auto* xf = static_cast<const float*>(x);
  const auto* ii = static_cast<const int*>(idx);
  const auto* wf = static_cast<const float*>(W);
  const auto* pf = static_cast<const float2*>(ph);
  auto* of = static_cast<float*>(out);
  auto* to = static_cast<int*>(timeouts);
  const int v = static_cast<int>(variant), rp = static_cast<int>(rep);
  if (C == 12) return chain::run_chain<12>(xf, ii, wf, pf, of, R, rp, v, to, as_stream(stream));
  return chain::run_chain<32>(xf, ii, wf, pf, of, R, rp, v, to, as_stream(stream));
}

}  // extern "C"
