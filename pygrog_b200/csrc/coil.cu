// coil.cu -- PCA coil compression, the step before the GROG path.
//
// The reference's utils/_coil_compress.py:23-57 (coil_compress) forwards to
// mrinufft's coil_compression: principal components of the multi-coil k-space
// (optionally only the samples near the k-space centre) give a (K, C)
// compression matrix, and the virtual coils are that matrix times the data.
// Here the covariance of the calibration samples is accumulated in FP64 on
// the device (pgb_coil_covariance), its eigendecomposition is a C x C host
// problem, and the compression itself (pgb_coil_compress) is one HBM-bound
// pass: every sample's C coils are read once, its K virtual coils written once.
#include <cuda_bf16.h>

#include "common.cuh"

namespace pgb {
namespace coil {

constexpr int kChunk = 64;   // samples per shared-memory chunk of the covariance
constexpr int kCovT = 256;   // threads of the covariance kernel

// cov[i * C + j] += sum_m D[i, m] conj(E[j, m]) over this block's sample chunks
// (D, E coil-major (C, M) complex64, accumulation in FP64; E == D for a
// covariance).
__global__ void __launch_bounds__(kCovT) coil_cov_kernel(const float2* __restrict__ D, const float2* __restrict__ E,
                                                         int64_t M, int C, double2* __restrict__ cov) {
  __shared__ float2 tile[32][kChunk + 1];
  __shared__ float2 tile_e[32][kChunk + 1];
  const int tid = threadIdx.x;
  const int pairs = C * C;
  double2 acc[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) acc[k] = make_double2(0.0, 0.0);
  for (int64_t m0 = static_cast<int64_t>(blockIdx.x) * kChunk; m0 < M;
       m0 += static_cast<int64_t>(gridDim.x) * kChunk) {
    for (int e = tid; e < C * kChunk; e += kCovT) {
      const int c = e / kChunk;
      const int s = e - c * kChunk;
      tile[c][s] = m0 + s < M ? D[static_cast<int64_t>(c) * M + m0 + s] : make_float2(0.f, 0.f);
      tile_e[c][s] = m0 + s < M ? E[static_cast<int64_t>(c) * M + m0 + s] : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int p = tid + k * kCovT;
      if (p < pairs) {
        const int i = p / C;
        const int j = p - i * C;
        double2 a = acc[k];
        for (int s = 0; s < kChunk; ++s) {
          const float2 u = tile[i][s], v = tile_e[j][s];
          a.x = fma(static_cast<double>(u.x), static_cast<double>(v.x), a.x);
          a.x = fma(static_cast<double>(u.y), static_cast<double>(v.y), a.x);
          a.y = fma(static_cast<double>(u.y), static_cast<double>(v.x), a.y);
          a.y = fma(-static_cast<double>(u.x), static_cast<double>(v.y), a.y);
        }
        acc[k] = a;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int p = tid + k * kCovT;
    if (p < pairs) {
      atomicAdd(&cov[p].x, acc[k].x);
      atomicAdd(&cov[p].y, acc[k].y);
    }
  }
}

__global__ void zero_f64(double2* __restrict__ p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = make_double2(0.0, 0.0);
}

// out[b, k, n] = sum_c mat[k, c] data[b, c, n]; one thread per sample, the
// sample's coils in registers, the matrix in shared memory (broadcast reads).
template <int CMAX>
__global__ void __launch_bounds__(256) coil_compress_kernel(const float2* __restrict__ data, int64_t N, int C, int K,
                                                            int B, const float2* __restrict__ mat,
                                                            float2* __restrict__ out) {
  extern __shared__ float2 ms[];
  for (int i = threadIdx.x; i < K * C; i += blockDim.x) ms[i] = mat[i];
  __syncthreads();
  const int64_t total = static_cast<int64_t>(B) * N;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t b = t / N;
    const int64_t n = t - b * N;
    const float2* src = data + b * C * N + n;
    float2 x[CMAX];
#pragma unroll
    for (int c = 0; c < CMAX; ++c) x[c] = c < C ? __ldg(src + static_cast<int64_t>(c) * N) : make_float2(0.f, 0.f);
    float2* dst = out + b * K * N + n;
    for (int k = 0; k < K; ++k) {
      const float2* row = ms + k * C;
      float2 a0 = make_float2(0.f, 0.f), a1 = make_float2(0.f, 0.f);
#pragma unroll
      for (int c = 0; c < CMAX; c += 2) {
        if (c < C) cfma(a0, row[c], x[c]);
        if (c + 1 < C) cfma(a1, row[c + 1], x[c + 1]);
      }
      dst[static_cast<int64_t>(k) * N] = make_float2(a0.x + a1.x, a0.y + a1.y);
    }
  }
}

// ---- tensor-core compression ---------------------------------------------------
// out = mat @ data, one 16-sample m-tile per warp and stage:
// D (16 samples x 8 NT) = A (16 samples x 2 CIP) B (2 CIP x 8 NT).  A holds the
// samples with (re, im) of every input coil interleaved along k, so each A word
// of a lane is one staged float2 sample (input coil 8 kc + t (+ 4), samples g
// and g + 8); B is the realified matrix with (re, im) of every output coil
// interleaved along n, held in registers, so the accumulator pairs (c0, c1) and
// (c2, c3) of a lane are the complex outputs of output coil 4 nt + t at samples
// g and g + 8.  12 output coils fill three n-tiles exactly.
// bf16x3: A = Ah + Al, B = Bh + Bl, D = Al Bh + Ah Bl + Ah Bh in FP32, with two
// accumulators per n-tile (even and odd k steps) so that the dependent MMA
// chains are half as long.
__device__ __forceinline__ void mma16c(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t bf2(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ void split_bf2(float x, float y, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(x, y);
  const float2 hf = __bfloat1622float2(h);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = bf2(x - hf.x, y - hf.y);
}

// Samples move in chunks of kCS per CTA stage (all input coils), staged in
// shared memory by 16-byte async copies kStages deep (in-flight bytes are what
// bound this HBM pass), coil stride kCS + 4 float2 so the four coils a lane
// quad reads fall in different banks.  Each warp computes one 16-sample m-tile
// per stage.
constexpr int kCS = 128;     // samples per chunk (8 warps x one 16-sample m-tile)
constexpr int kStages = 3;   // chunks in flight per CTA
constexpr int kXS = kCS + 4; // shared-memory coil stride (float2)

__device__ __forceinline__ void cpa16(void* dst, const void* src, int bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpa8(void* dst, const void* src, int bytes) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}

template <int CIP, int NT>  // CIP input coils (multiple of 8), NT n-tiles (4 output coils each)
__global__ void __launch_bounds__(256, 2) coil_compress_tc_kernel(const float2* __restrict__ data, int64_t N, int C,
                                                                  int K, int B, const float2* __restrict__ mat,
                                                                  float2* __restrict__ out) {
  constexpr int KC = CIP / 8;  // k16 steps (8 input coils each)
  extern __shared__ __align__(16) float2 xs_flat[];  // kStages buffers of CIP x kXS
  auto xs = [&](int k) { return xs_flat + k * (CIP * kXS); };
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  // B fragments of the realified matrix, heads and tails: b0 covers k rows 2t,
  // 2t + 1 (re, im of input coil 8 kc + t), b1 input coil 8 kc + t + 4; column
  // g is the real (even g) or imaginary (odd g) part of output coil 4 nt + g / 2
  uint32_t bh[NT][KC][2], bl[NT][KC][2];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int kc = 0; kc < KC; ++kc)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int ko = 4 * nt + (g >> 1);
        const int c = 8 * kc + t + 4 * h;
        float2 m = make_float2(0.f, 0.f);
        if (ko < K && c < C) m = __ldg(mat + ko * C + c);
        const float e0 = (g & 1) ? m.y : m.x;   // times x_re
        const float e1 = (g & 1) ? m.x : -m.y;  // times x_im
        split_bf2(e0, e1, bh[nt][kc][h], bl[nt][kc][h]);
      }
  const int64_t chunks_per_b = (N + kCS - 1) / kCS;
  const int64_t n_chunks = static_cast<int64_t>(B) * chunks_per_b;
  // 16-byte copies need even N and a 16-byte aligned base (pairs of samples)
  const bool wide = (N & 1) == 0 && (reinterpret_cast<uintptr_t>(data) & 15) == 0;
  // stage chunk q (all coils) into buffer k; q >= n_chunks commits an empty group
  auto stage = [&](int64_t q, int k) {
    if (q < n_chunks) {
      const int64_t b = q / chunks_per_b;
      const int64_t n0 = (q - b * chunks_per_b) * kCS;
      const float2* src = data + b * C * N;
      for (int i = tid; i < CIP * (kCS / 2); i += 256) {  // (coil, sample pair)
        const int c = i / (kCS / 2);
        const int pr = i - c * (kCS / 2);
        const int64_t n = n0 + 2 * pr;
        float2* dst = xs(k) + c * kXS + 2 * pr;
        const float2* sp = src + static_cast<int64_t>(c) * N + n;
        const bool c_ok = c < C;
        if (wide) {
          cpa16(dst, c_ok && n < N ? sp : data, c_ok && n < N ? 16 : 0);  // N even: pairs never straddle N
        } else {
          cpa8(dst, c_ok && n < N ? sp : data, c_ok && n < N ? 8 : 0);
          cpa8(dst + 1, c_ok && n + 1 < N ? sp + 1 : data, c_ok && n + 1 < N ? 8 : 0);
        }
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  const int64_t stride = gridDim.x;
  int64_t q = blockIdx.x;
  for (int j = 0; j < kStages - 1; ++j) stage(q + j * stride, j);
  for (int it = 0; q < n_chunks; ++it, q += stride) {
    const int k = it % kStages;
    asm volatile("cp.async.wait_group %0;\n" ::"n"(kStages - 2) : "memory");
    // chunk q complete in buffer k (every thread's copies), and every warp is
    // done with the previous chunk, whose buffer is staged next
    __syncthreads();
    stage(q + (kStages - 1) * stride, (it + kStages - 1) % kStages);
    const int64_t b = q / chunks_per_b;
    const int64_t n0 = (q - b * chunks_per_b) * kCS + 16 * warp;  // this warp's 16-sample m-tile
    if (n0 < N) {
      const float2* x = xs(k) + 16 * warp + g;  // sample g of the m-tile
      float d[NT][2][4];
#pragma unroll
      for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int j = 0; j < 2; ++j) d[nt][j][0] = d[nt][j][1] = d[nt][j][2] = d[nt][j][3] = 0.f;
#pragma unroll
      for (int kc = 0; kc < KC; ++kc) {
        // a0 / a1: input coil 8 kc + t at samples g / g + 8; a2 / a3: coil 8 kc + t + 4
        // (staged planes are zero beyond C and beyond N)
        uint32_t ah[4], al[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const float2 v = x[(8 * kc + t + 4 * (r >> 1)) * kXS + 8 * (r & 1)];
          split_bf2(v.x, v.y, ah[r], al[r]);
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          float(&acc)[4] = d[nt][kc & 1];
          mma16c(acc, al, bh[nt][kc][0], bh[nt][kc][1]);
          mma16c(acc, ah, bl[nt][kc][0], bl[nt][kc][1]);
          mma16c(acc, ah, bh[nt][kc][0], bh[nt][kc][1]);
        }
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int ko = 4 * nt + t;
        if (ko < K) {
          float2* dst = out + (b * K + ko) * N + n0 + g;
          const float* e = d[nt][0];
          const float* o = d[nt][1];
          if (n0 + g < N) dst[0] = make_float2(e[0] + o[0], e[1] + o[1]);
          if (n0 + g + 8 < N) dst[8] = make_float2(e[2] + o[2], e[3] + o[3]);
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

}  // namespace coil
}  // namespace pgb

using namespace pgb;
using namespace pgb::coil;

extern "C" {

int pgb_coil_cross_covariance(const void* data, const void* data2, int64_t M, int64_t C, void* cov, void* stream) {
  const char* who = "coil_cross_covariance";
  clear_error();
  PGB_REQUIRE(C >= 1 && C <= 32, PGB_ERR_UNSUPPORTED, "%s: 1..32 coils, got %lld", who, (long long)C);
  PGB_REQUIRE(M >= 0, PGB_ERR_INVALID, "%s: negative sample count", who);
  PGB_REQUIRE(cov != nullptr && ((data != nullptr && data2 != nullptr) || M == 0), PGB_ERR_INVALID,
              "%s: null pointer", who);
  cudaStream_t s = as_stream(stream);
  const int pairs = static_cast<int>(C * C);
  zero_f64<<<(pairs + 255) / 256, 256, 0, s>>>(static_cast<double2*>(cov), pairs);
  PGB_LAUNCH_CHECK(who);
  if (M == 0) return PGB_OK;
  const int blocks = grid_for((M + kChunk - 1) / kChunk, 1, 148 * 8);
  coil_cov_kernel<<<blocks, kCovT, 0, s>>>(static_cast<const float2*>(data), static_cast<const float2*>(data2), M,
                                          static_cast<int>(C), static_cast<double2*>(cov));
  PGB_LAUNCH_CHECK(who);
  return PGB_OK;
}

int pgb_coil_covariance(const void* data, int64_t M, int64_t C, void* cov, void* stream) {
  return pgb_coil_cross_covariance(data, data, M, C, cov, stream);
}

int pgb_coil_compress(const void* data, int64_t N, int64_t C, int64_t K, int64_t B, const void* mat, void* out,
                      void* stream) {
  const char* who = "coil_compress";
  clear_error();
  PGB_REQUIRE(C >= 1 && C <= 64, PGB_ERR_UNSUPPORTED, "%s: 1..64 coils, got %lld", who, (long long)C);
  PGB_REQUIRE(K >= 1 && K <= C, PGB_ERR_INVALID, "%s: need 1 <= K <= C, got K=%lld C=%lld", who, (long long)K,
              (long long)C);
  PGB_REQUIRE(N >= 0 && B >= 0, PGB_ERR_INVALID, "%s: negative size", who);
  if (N == 0 || B == 0) return PGB_OK;
  PGB_REQUIRE(data && mat && out, PGB_ERR_INVALID, "%s: null pointer", who);
  cudaStream_t s = as_stream(stream);
  const size_t smem = static_cast<size_t>(K * C) * sizeof(float2);
  const int blocks = grid_for(B * N, 256, 148 * 8);
  if (C <= 32) {
    coil_compress_kernel<32><<<blocks, 256, smem, s>>>(static_cast<const float2*>(data), N, static_cast<int>(C),
                                                       static_cast<int>(K), static_cast<int>(B),
                                                       static_cast<const float2*>(mat), static_cast<float2*>(out));
  } else {
    coil_compress_kernel<64><<<blocks, 256, smem, s>>>(static_cast<const float2*>(data), N, static_cast<int>(C),
                                                       static_cast<int>(K), static_cast<int>(B),
                                                       static_cast<const float2*>(mat), static_cast<float2*>(out));
  }
  PGB_LAUNCH_CHECK(who);
  return PGB_OK;
}

int pgb_coil_compress_tc(const void* data, int64_t N, int64_t C, int64_t K, int64_t B, const void* mat, void* out,
                         void* stream) {
  const char* who = "coil_compress_tc";
  clear_error();
  PGB_REQUIRE(C >= 1 && C <= 32, PGB_ERR_UNSUPPORTED, "%s: 1..32 coils, got %lld", who, (long long)C);
  PGB_REQUIRE(K >= 1 && K <= C && K <= 16, PGB_ERR_INVALID, "%s: need 1 <= K <= min(C, 16), got K=%lld", who,
              (long long)K);
  PGB_REQUIRE(N >= 0 && B >= 0, PGB_ERR_INVALID, "%s: negative size", who);
  if (N == 0 || B == 0) return PGB_OK;
  PGB_REQUIRE(data && mat && out, PGB_ERR_INVALID, "%s: null pointer", who);
  cudaStream_t s = as_stream(stream);
  const int64_t chunks = B * ((N + kCS - 1) / kCS);
  const int blocks = static_cast<int>(chunks < 148 * 2 ? chunks : 148 * 2);  // persistent: two CTAs per SM
  const int cip = static_cast<int>((C + 7) / 8 * 8);
  const int nt = static_cast<int>((K + 3) / 4);
  const float2* d = static_cast<const float2*>(data);
  const float2* m = static_cast<const float2*>(mat);
  float2* o = static_cast<float2*>(out);
  const int Ci = static_cast<int>(C), Ki = static_cast<int>(K), Bi = static_cast<int>(B);
  switch (cip * 10 + nt) {
#define X(CI, NTT)                                                                                  \
  case CI * 10 + NTT: {                                                                             \
    const int smem = kStages * CI * kXS * static_cast<int>(sizeof(float2));                         \
    cudaFuncSetAttribute(coil_compress_tc_kernel<CI, NTT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); \
    coil_compress_tc_kernel<CI, NTT><<<blocks, 256, smem, s>>>(d, N, Ci, Ki, Bi, m, o);              \
  } break;
    X(8, 1) X(8, 2) X(16, 1) X(16, 2) X(16, 3) X(16, 4) X(24, 1) X(24, 2) X(24, 3) X(24, 4)
    X(32, 1) X(32, 2) X(32, 3) X(32, 4)
#undef X
    default:
      PGB_REQUIRE(false, PGB_ERR_UNSUPPORTED, "%s: no kernel for C=%lld K=%lld", who, (long long)C, (long long)K);
  }
  PGB_LAUNCH_CHECK(who);
  return PGB_OK;
}

}  // extern "C"
