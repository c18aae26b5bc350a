// lsmr.cu -- LSMR (Fong & Saunders) with the recurrence scalars in FP64 on
// the device.
//
// Reference: _solve/_solvers.py:145-262 (lsmr).  The reference computes the
// norms in the working precision (complex64 -> FP32) and calls .item() three
// times per iteration (two branch tests and the stopping test).  Here the
// norms accumulate in FP64, every scalar of the recurrence lives in a device
// block, and the branches and the stopping test are device flags, so one
// iteration is a fixed launch sequence (operator forward, u update + FP64
// norm, u scale, operator adjoint, v_full + FP64 norm, scalar recurrence,
// vector update) that can be captured in a CUDA graph and replayed.
//
// Scalar block (double[PGB_LSMR_SCALARS], device memory owned by the caller),
// slot names in include/pygrog_b200.h.  Vectors are complex64.  Once the
// stopping test has fired (STOP != 0), every later launch leaves the vectors
// and scalars unchanged.
#include "common.cuh"

namespace pgb {
namespace lsmr {

enum {
  ALPHA = 0, BETA = 1, ALPHABAR = 2, RHO = 3, RHOBAR = 4, CBAR = 5, SBAR = 6, ZETABAR = 7, ZETA = 8, NORMB = 9,
  STOP = 10, TOL = 11, DAMP = 12, C_HBAR = 13, C_X = 14, C_H = 15, BSQ = 16, ASQ = 17, RAN = 18, REL = 19,
  OKV = 20, ITER = 21
};
static_assert(PGB_LSMR_SCALARS >= 24, "scalar block");

constexpr int kThreads = 256;
constexpr int kBlocks = 296;  // 2 x SMs
constexpr int kScratchWords = kBlocks + 2;  // block partials + one counter word

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double warp_sums[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_sums[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (warp == 0) {
    s = lane < kThreads / 32 ? warp_sums[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;  // valid in thread 0
}

// Sum `acc` over the grid; the last block to finish writes scal[slot] and
// re-arms the counter.
__device__ __forceinline__ void grid_sum_to(double acc, double* __restrict__ scratch, double* __restrict__ scal,
                                            int slot) {
  const double s = block_sum(acc);
  __shared__ bool last;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kBlocks);
  if (threadIdx.x == 0) {
    scratch[blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += blockDim.x) t += scratch[i];
  t = block_sum(t);
  if (threadIdx.x == 0) {
    scal[slot] = t;
    *counter = 0u;
  }
}

__device__ __forceinline__ double norm2(float2 v) {
  return static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
}

// u <- Av - alpha u ;  BSQ <- ||u||^2 (FP64)
__global__ void __launch_bounds__(kThreads) u_update_kernel(float2* __restrict__ u, const float2* __restrict__ Av,
                                                            int64_t n, double* __restrict__ scal,
                                                            double* __restrict__ scratch) {
  if (scal[STOP] != 0.0) return;  // grid-uniform
  const float a = static_cast<float>(scal[ALPHA]);
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 w = Av[i], q = u[i];
    const float2 r = make_float2(w.x - a * q.x, w.y - a * q.y);
    u[i] = r;
    acc += norm2(r);
  }
  grid_sum_to(acc, scratch, scal, BSQ);
}

// u <- u / sqrt(BSQ) when BSQ > 0
__global__ void u_scale_kernel(float2* __restrict__ u, int64_t n, const double* __restrict__ scal) {
  if (scal[STOP] != 0.0 || !(scal[BSQ] > 0.0)) return;
  const float s = static_cast<float>(1.0 / sqrt(scal[BSQ]));
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 q = u[i];
    u[i] = make_float2(q.x * s, q.y * s);
  }
}

// vf <- Atu - beta v with beta = sqrt(BSQ) ;  ASQ <- ||vf||^2 (FP64); only when BSQ > 0
__global__ void __launch_bounds__(kThreads) v_full_kernel(float2* __restrict__ vf, const float2* __restrict__ Atu,
                                                          const float2* __restrict__ v, int64_t n,
                                                          double* __restrict__ scal, double* __restrict__ scratch) {
  if (scal[STOP] != 0.0 || !(scal[BSQ] > 0.0)) return;  // grid-uniform
  const float b = static_cast<float>(sqrt(scal[BSQ]));
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 w = Atu[i], q = v[i];
    const float2 r = make_float2(w.x - b * q.x, w.y - b * q.y);
    vf[i] = r;
    acc += norm2(r);
  }
  grid_sum_to(acc, scratch, scal, ASQ);
}

// The scalar part of one iteration (_solvers.py:212-255), one thread, FP64.
__global__ void scalar_kernel(double* __restrict__ s) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (s[STOP] != 0.0) {
    s[RAN] = 0.0;
    return;
  }
  s[RAN] = 1.0;
  const double beta = sqrt(s[BSQ] > 0.0 ? s[BSQ] : 0.0);
  s[BETA] = beta;
  s[OKV] = 0.0;
  if (beta > 0.0) {  // the v_full branch ran: alpha = ||v_full||, v = v_full / alpha when alpha > 0
    const double alpha = sqrt(s[ASQ] > 0.0 ? s[ASQ] : 0.0);
    s[ALPHA] = alpha;
    if (alpha > 0.0) s[OKV] = 1.0;
  }
  const double alpha = s[ALPHA], damp = s[DAMP];
  const double alphahat = sqrt(s[ALPHABAR] * s[ALPHABAR] + damp * damp);
  const double rhoold = s[RHO];
  const double rho = sqrt(alphahat * alphahat + beta * beta);
  const double c = alphahat / rho, sn = beta / rho;
  const double thetanew = sn * alpha;
  s[ALPHABAR] = c * alpha;
  const double rhobarold = s[RHOBAR];
  const double thetabar = s[SBAR] * rho;
  const double rhotemp = s[CBAR] * rho;
  const double rhobar = sqrt(rhotemp * rhotemp + thetanew * thetanew);
  const double cbar = rhotemp / rhobar, sbar = thetanew / rhobar;
  const double zeta = cbar * s[ZETABAR];
  const double zetabar = -sbar * s[ZETABAR];
  s[RHO] = rho;
  s[RHOBAR] = rhobar;
  s[CBAR] = cbar;
  s[SBAR] = sbar;
  s[ZETA] = zeta;
  s[ZETABAR] = zetabar;
  s[C_HBAR] = thetabar * rho / (rhoold * rhobarold);
  s[C_X] = zeta / (rho * rhobar);
  s[C_H] = thetanew / rho;
  const double rel = fabs(zetabar) / (s[NORMB] + 1e-30);
  s[REL] = rel;
  s[ITER] += 1.0;
  if (rel < s[TOL]) s[STOP] = 1.0;
}

// v <- vf / alpha (when OKV) ; hbar <- h - c1 hbar ; x <- x + c2 hbar ; h <- v - c3 h
__global__ void vec_update_kernel(float2* __restrict__ x, float2* __restrict__ h, float2* __restrict__ hbar,
                                  float2* __restrict__ v, const float2* __restrict__ vf, int64_t n,
                                  const double* __restrict__ s) {
  if (s[RAN] == 0.0) return;  // grid-uniform: the recurrence was frozen this iteration
  const bool okv = s[OKV] != 0.0;
  const float ia = okv ? static_cast<float>(1.0 / s[ALPHA]) : 1.f;
  const float c1 = static_cast<float>(s[C_HBAR]), c2 = static_cast<float>(s[C_X]), c3 = static_cast<float>(s[C_H]);
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    float2 vv = v[i];
    if (okv) {
      const float2 w = vf[i];
      vv = make_float2(w.x * ia, w.y * ia);
      v[i] = vv;
    }
    const float2 hh = h[i];
    float2 hb = hbar[i];
    hb = make_float2(hh.x - c1 * hb.x, hh.y - c1 * hb.y);
    hbar[i] = hb;
    const float2 xx = x[i];
    x[i] = make_float2(xx.x + c2 * hb.x, xx.y + c2 * hb.y);
    h[i] = make_float2(vv.x - c3 * hh.x, vv.y - c3 * hh.y);
  }
}

}  // namespace lsmr
}  // namespace pgb

using namespace pgb;

extern "C" {

size_t pgb_lsmr_scratch_bytes(void) { return static_cast<size_t>(lsmr::kScratchWords) * sizeof(double); }

int pgb_lsmr_u_update(void* u, const void* Av, int64_t n, void* scal, void* scratch, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0, PGB_ERR_INVALID, "lsmr_u_update: negative size");
  PGB_REQUIRE(scal && scratch && (n == 0 || (u && Av)), PGB_ERR_INVALID, "lsmr_u_update: null pointer");
  lsmr::u_update_kernel<<<grid_for(n, lsmr::kThreads, lsmr::kBlocks), lsmr::kThreads, 0, as_stream(stream)>>>(
      static_cast<float2*>(u), static_cast<const float2*>(Av), n, static_cast<double*>(scal),
      static_cast<double*>(scratch));
  PGB_LAUNCH_CHECK("lsmr_u_update");
  return PGB_OK;
}

int pgb_lsmr_u_scale(void* u, int64_t n, const void* scal, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0, PGB_ERR_INVALID, "lsmr_u_scale: negative size");
  PGB_REQUIRE(scal && (n == 0 || u), PGB_ERR_INVALID, "lsmr_u_scale: null pointer");
  lsmr::u_scale_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, as_stream(stream)>>>(static_cast<float2*>(u), n,
                                                                                 static_cast<const double*>(scal));
  PGB_LAUNCH_CHECK("lsmr_u_scale");
  return PGB_OK;
}

int pgb_lsmr_v_full(void* vf, const void* Atu, const void* v, int64_t n, void* scal, void* scratch, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0, PGB_ERR_INVALID, "lsmr_v_full: negative size");
  PGB_REQUIRE(scal && scratch && (n == 0 || (vf && Atu && v)), PGB_ERR_INVALID, "lsmr_v_full: null pointer");
  lsmr::v_full_kernel<<<grid_for(n, lsmr::kThreads, lsmr::kBlocks), lsmr::kThreads, 0, as_stream(stream)>>>(
      static_cast<float2*>(vf), static_cast<const float2*>(Atu), static_cast<const float2*>(v), n,
      static_cast<double*>(scal), static_cast<double*>(scratch));
  PGB_LAUNCH_CHECK("lsmr_v_full");
  return PGB_OK;
}

int pgb_lsmr_scalars(void* scal, void* stream) {
  clear_error();
  PGB_REQUIRE(scal != nullptr, PGB_ERR_INVALID, "lsmr_scalars: null pointer");
  lsmr::scalar_kernel<<<1, 32, 0, as_stream(stream)>>>(static_cast<double*>(scal));
  PGB_LAUNCH_CHECK("lsmr_scalars");
  return PGB_OK;
}

int pgb_lsmr_vec_update(void* x, void* h, void* hbar, void* v, const void* vf, int64_t n, const void* scal,
                        void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0, PGB_ERR_INVALID, "lsmr_vec_update: negative size");
  PGB_REQUIRE(scal && (n == 0 || (x && h && hbar && v && vf)), PGB_ERR_INVALID, "lsmr_vec_update: null pointer");
  lsmr::vec_update_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, as_stream(stream)>>>(
      static_cast<float2*>(x), static_cast<float2*>(h), static_cast<float2*>(hbar), static_cast<float2*>(v),
      static_cast<const float2*>(vf), n, static_cast<const double*>(scal));
  PGB_LAUNCH_CHECK("lsmr_vec_update");
  return PGB_OK;
}

}  // extern "C"
