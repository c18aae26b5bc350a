// common.cuh -- shared helpers of the sm_100a GROG library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>

#include "../../include/pygrog_b200.h"

namespace pgb {

// ---- error reporting ------------------------------------------------------
void set_error(const char* fmt, ...);
void clear_error();

#define PGB_REQUIRE(cond, code, ...) \
  do {                               \
    if (!(cond)) {                   \
      ::pgb::set_error(__VA_ARGS__); \
      return (code);                 \
    }                                \
  } while (0)

// Launch check: returns PGB_ERR_CUDA from the enclosing function on failure.
#define PGB_LAUNCH_CHECK(name)                                                \
  do {                                                                        \
    cudaError_t e_ = cudaGetLastError();                                      \
    if (e_ != cudaSuccess) {                                                  \
      ::pgb::set_error("%s: launch failed: %s", name, cudaGetErrorString(e_)); \
      return PGB_ERR_CUDA;                                                    \
    }                                                                         \
  } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int kNumSMs = 148;  // B200

inline int grid_for(int64_t n, int block, int64_t max_blocks = 148 * 32) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return static_cast<int>(g);
}

// ---- complex arithmetic on float2 / double2 -------------------------------
template <typename R>
struct cplx;
template <>
struct cplx<float> {
  using T = float2;
};
template <>
struct cplx<double> {
  using T = double2;
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// acc += a * b
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
__device__ __forceinline__ void cfma_conj(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(-a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfma_conj(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}
template <typename V>
__device__ __forceinline__ V czero();
template <>
__device__ __forceinline__ float2 czero<float2>() {
  return make_float2(0.f, 0.f);
}
template <>
__device__ __forceinline__ double2 czero<double2>() {
  return make_double2(0.0, 0.0);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ void catomic_add(float2* p, float2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}
__device__ __forceinline__ void catomic_add(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

// Warp-aggregated complex atomic add: lanes holding the same key are summed
// in registers first, then one lane per distinct key issues the atomic.
// Keys must be valid (>= 0) for all lanes in `active`.
template <typename V>
__device__ __forceinline__ void warp_aggregated_add(V* base, int64_t key, V val,
                                                    unsigned active) {
  unsigned peers = __match_any_sync(active, (unsigned long long)key);
  int leader = __ffs(peers) - 1;
  unsigned m = peers;
  V acc = czero<V>();
  while (m) {
    int src = __ffs(m) - 1;
    m &= m - 1;
    V v;
    v.x = __shfl_sync(peers, val.x, src);
    v.y = __shfl_sync(peers, val.y, src);
    acc = cadd(acc, v);
  }
  if ((int)(threadIdx.x & 31) == leader) catomic_add(base + key, acc);
}

__device__ __forceinline__ void warp_aggregated_add_real(float* base, int64_t key, float val,
                                                         unsigned active) {
  unsigned peers = __match_any_sync(active, (unsigned long long)key);
  int leader = __ffs(peers) - 1;
  unsigned m = peers;
  float acc = 0.f;
  while (m) {
    int src = __ffs(m) - 1;
    m &= m - 1;
    acc += __shfl_sync(peers, val, src);
  }
  if ((int)(threadIdx.x & 31) == leader) atomicAdd(base + key, acc);
}
__device__ __forceinline__ void warp_aggregated_add_real(double* base, int64_t key, double val,
                                                         unsigned active) {
  unsigned peers = __match_any_sync(active, (unsigned long long)key);
  int leader = __ffs(peers) - 1;
  unsigned m = peers;
  double acc = 0.0;
  while (m) {
    int src = __ffs(m) - 1;
    m &= m - 1;
    acc += __shfl_sync(peers, val, src);
  }
  if ((int)(threadIdx.x & 31) == leader) atomicAdd(base + key, acc);
}

}  // namespace pgb
