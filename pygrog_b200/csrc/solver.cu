// solver.cu -- device-side conjugate-gradient scalars with FP64 reductions.
//
// Reference: _solve/_solvers.py:49-139 (cg).  The reference evaluates
// vdot / vector_norm in the working precision (complex64 -> FP32) and calls
// .item() every iteration.  Here every inner product and norm accumulates in
// FP64, the step scalars stay in device memory, and a device flag replaces
// the host-side `break`, so an iteration is a fixed launch sequence that can
// be captured in a CUDA graph and replayed.
//
// Scalar block (double[kScalars]), device memory owned by the caller:
//   [0] rz_old   [1] pAp   [2] rr (|r|^2)   [3] r0_norm   [4] rel   [5] done
//   [6] tol      [7] spare
#include <cuda.h>

#include <mutex>

#include "common.cuh"

namespace pgb {

enum { S_RZ = 0, S_PAP = 1, S_RR = 2, S_R0 = 3, S_REL = 4, S_DONE = 5, S_TOL = 6 };
constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 x SMs

// Block-partial FP64 sums of Re(conj(a) b) (b == nullptr: |a|^2); the last
// block to finish reduces the partials and writes *out (optionally also
// applying the scalar epilogue `mode`).  scratch holds kRedBlocks doubles
// followed by one unsigned counter, which the last block resets to 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double warp_sums[kRedThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_sums[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (warp == 0) {
    s = lane < kRedThreads / 32 ? warp_sums[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  }
  return s;  // valid in thread 0
}

// mode: 0 plain dot -> out;  1: out = rr and the CG residual check
// (rel = sqrt(rr) / r0, done |= rel < tol);  2: r0 initialisation
// (r0 = sqrt(rr) + 1e-30, rz_old = rr).
// Frame f = blockIdx.y works on a + f*n, b + f*n with its own scalar block
// scal + f*kScalars and scratch + f*kScratchWords (gridDim.y == 1: one frame).
constexpr int kScalars = 8;
constexpr int kScratchWords = kRedBlocks + 2;  // partials + two unsigned counters (one double)

__global__ void __launch_bounds__(kRedThreads) dot_f64_kernel(const float2* __restrict__ a,
                                                              const float2* __restrict__ b, int64_t n,
                                                              double* __restrict__ scratch,
                                                              double* __restrict__ scal, int out_slot,
                                                              int mode) {
  {
    const int64_t f = blockIdx.y;
    a += f * n;
    if (b) b += f * n;
    scratch += f * kScratchWords;
    scal += f * kScalars;
  }
  if (mode == 1 && scal[S_DONE] != 0.0) return;  // grid-uniform: converged, skip
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 x = a[i];
    if (b) {
      const float2 y = b[i];
      acc += static_cast<double>(x.x) * y.x + static_cast<double>(x.y) * y.y;
    } else {
      acc += static_cast<double>(x.x) * x.x + static_cast<double>(x.y) * x.y;
    }
  }
  const double s = block_sum(acc);
  __shared__ bool last;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kRedBlocks);
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
    if (mode == 0) {
      scal[out_slot] = t;
    } else if (mode == 1) {
      scal[S_RR] = t;
      const double rel = sqrt(t) / scal[S_R0];
      scal[S_REL] = rel;
      if (rel < scal[S_TOL]) scal[S_DONE] = 1.0;
    } else {
      scal[S_RR] = t;
      scal[S_RZ] = t;
      scal[S_R0] = sqrt(t) + 1e-30;
      scal[S_REL] = 1.0;
      scal[S_DONE] = 0.0;
    }
    *counter = 0u;
  }
}

// x += alpha p ; r -= alpha Ap   with alpha = rz_old / (pAp + 1e-30)
__global__ void cg_update_xr_kernel(float2* __restrict__ x, float2* __restrict__ r,
                                    const float2* __restrict__ p, const float2* __restrict__ Ap, int64_t n,
                                    const double* __restrict__ scal) {
  {
    const int64_t f = blockIdx.y;
    x += f * n;
    r += f * n;
    p += f * n;
    Ap += f * n;
    scal += f * kScalars;
  }
  if (scal[S_DONE] != 0.0) return;
  const float alpha = static_cast<float>(scal[S_RZ] / (scal[S_PAP] + 1e-30));
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 pv = p[i], av = Ap[i];
    float2 xv = x[i], rv = r[i];
    xv.x = fmaf(alpha, pv.x, xv.x);
    xv.y = fmaf(alpha, pv.y, xv.y);
    rv.x = fmaf(-alpha, av.x, rv.x);
    rv.y = fmaf(-alpha, av.y, rv.y);
    x[i] = xv;
    r[i] = rv;
  }
}

// x += alpha p ; r -= alpha Ap, and in the same pass rr = |r|^2 in FP64 with
// the residual check of dot_f64 mode 1 (rel = sqrt(rr) / r0, done |= rel < tol):
// one launch and one read of r fewer per iteration than update + dot.  At most
// kRedBlocks blocks (their partials go to scratch; the first counter).
__global__ void __launch_bounds__(kRedThreads) cg_update_xr_rr_kernel(float2* __restrict__ x,
                                                                      float2* __restrict__ r,
                                                                      const float2* __restrict__ p,
                                                                      const float2* __restrict__ Ap, int64_t n,
                                                                      double* __restrict__ scal,
                                                                      double* __restrict__ scratch) {
  {
    const int64_t f = blockIdx.y;
    x += f * n;
    r += f * n;
    p += f * n;
    Ap += f * n;
    scal += f * kScalars;
    scratch += f * kScratchWords;
  }
  if (scal[S_DONE] != 0.0) return;  // grid-uniform: converged, skip
  const float alpha = static_cast<float>(scal[S_RZ] / (scal[S_PAP] + 1e-30));
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 pv = p[i], av = Ap[i];
    float2 xv = x[i], rv = r[i];
    xv.x = fmaf(alpha, pv.x, xv.x);
    xv.y = fmaf(alpha, pv.y, xv.y);
    rv.x = fmaf(-alpha, av.x, rv.x);
    rv.y = fmaf(-alpha, av.y, rv.y);
    x[i] = xv;
    r[i] = rv;
    acc += static_cast<double>(rv.x) * rv.x + static_cast<double>(rv.y) * rv.y;
  }
  const double s = block_sum(acc);
  __shared__ bool last;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kRedBlocks);
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
    scal[S_RR] = t;
    const double rel = sqrt(t) / scal[S_R0];
    scal[S_REL] = rel;
    if (rel < scal[S_TOL]) scal[S_DONE] = 1.0;
    *counter = 0u;
  }
}

// p = r + beta p  with beta = rr / (rz_old + 1e-30); the last block then
// commits rz_old = rr for the next iteration (grid-wide ordering through a
// completion counter in scratch).
__global__ void cg_update_p_kernel(float2* __restrict__ p, const float2* __restrict__ r, int64_t n,
                                   double* __restrict__ scal, double* __restrict__ scratch) {
  {
    const int64_t f = blockIdx.y;
    p += f * n;
    r += f * n;
    scal += f * kScalars;
    scratch += f * kScratchWords;
  }
  if (scal[S_DONE] != 0.0) return;
  const double rr = scal[S_RR];
  const float beta = static_cast<float>(rr / (scal[S_RZ] + 1e-30));
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 rv = r[i];
    float2 pv = p[i];
    pv.x = fmaf(beta, pv.x, rv.x);
    pv.y = fmaf(beta, pv.y, rv.y);
    p[i] = pv;
  }
  __shared__ bool last;
  __syncthreads();
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kRedBlocks) + 1;
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    scal[S_RZ] = rr;
    *counter = 0u;
  }
}

// y = a * x + y (complex vectors, real a)
__global__ void axpy_kernel(float2* __restrict__ y, const float2* __restrict__ x, float a, int64_t n) {
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 xv = x[i];
    float2 yv = y[i];
    yv.x = fmaf(a, xv.x, yv.x);
    yv.y = fmaf(a, xv.y, yv.y);
    y[i] = yv;
  }
}

}  // namespace pgb

using namespace pgb;

extern "C" {

size_t pgb_reduce_scratch_bytes(void) { return kScratchWords * sizeof(double); }

int pgb_dot_f64(const void* a, const void* b, int64_t n, void* scratch, void* scalars, int out_slot, int mode,
                void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0 && out_slot >= 0 && out_slot < 8 && mode >= 0 && mode <= 2, PGB_ERR_INVALID,
              "dot_f64: invalid arguments");
  PGB_REQUIRE(a && scratch && scalars, PGB_ERR_INVALID, "dot_f64: null pointer");
  int blocks = grid_for(n, kRedThreads, kRedBlocks);
  dot_f64_kernel<<<blocks, kRedThreads, 0, as_stream(stream)>>>(
      static_cast<const float2*>(a), static_cast<const float2*>(b), n, static_cast<double*>(scratch),
      static_cast<double*>(scalars), out_slot, mode);
  PGB_LAUNCH_CHECK("dot_f64");
  return PGB_OK;
}

int pgb_cg_update_xr(void* x, void* r, const void* p, const void* Ap, int64_t n, const void* scalars,
                     void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0, PGB_ERR_INVALID, "cg_update_xr: negative size");
  if (n == 0) return PGB_OK;
  PGB_REQUIRE(x && r && p && Ap && scalars, PGB_ERR_INVALID, "cg_update_xr: null pointer");
  cg_update_xr_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, as_stream(stream)>>>(
      static_cast<float2*>(x), static_cast<float2*>(r), static_cast<const float2*>(p),
      static_cast<const float2*>(Ap), n, static_cast<const double*>(scalars));
  PGB_LAUNCH_CHECK("cg_update_xr");
  return PGB_OK;
}

int pgb_cg_update_xr_rr(void* x, void* r, const void* p, const void* Ap, int64_t n, void* scalars, void* scratch,
                        void* stream) {
  return pgb_cg_update_xr_rr_batched(x, r, p, Ap, n, 1, scalars, scratch, stream);
}

int pgb_cg_update_xr_rr_batched(void* x, void* r, const void* p, const void* Ap, int64_t n, int64_t frames,
                                void* scalars, void* scratch, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0 && frames >= 0 && frames <= 65535, PGB_ERR_INVALID, "cg_update_xr_rr: invalid sizes");
  if (n == 0 || frames == 0) return PGB_OK;
  PGB_REQUIRE(x && r && p && Ap && scalars && scratch, PGB_ERR_INVALID, "cg_update_xr_rr: null pointer");
  const dim3 grid(grid_for(n, kRedThreads, kRedBlocks), static_cast<unsigned>(frames));
  cg_update_xr_rr_kernel<<<grid, kRedThreads, 0, as_stream(stream)>>>(
      static_cast<float2*>(x), static_cast<float2*>(r), static_cast<const float2*>(p),
      static_cast<const float2*>(Ap), n, static_cast<double*>(scalars), static_cast<double*>(scratch));
  PGB_LAUNCH_CHECK("cg_update_xr_rr");
  return PGB_OK;
}

int pgb_cg_update_p(void* p, const void* r, int64_t n, void* scalars, void* scratch, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0, PGB_ERR_INVALID, "cg_update_p: negative size");
  if (n == 0) return PGB_OK;
  PGB_REQUIRE(p && r && scalars && scratch, PGB_ERR_INVALID, "cg_update_p: null pointer");
  cg_update_p_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, as_stream(stream)>>>(
      static_cast<float2*>(p), static_cast<const float2*>(r), n, static_cast<double*>(scalars),
      static_cast<double*>(scratch));
  PGB_LAUNCH_CHECK("cg_update_p");
  return PGB_OK;
}

int pgb_dot_f64_batched(const void* a, const void* b, int64_t n, int64_t frames, void* scratch, void* scalars,
                        int out_slot, int mode, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0 && frames >= 0 && frames <= 65535 && out_slot >= 0 && out_slot < kScalars && mode >= 0 &&
                  mode <= 2,
              PGB_ERR_INVALID, "dot_f64_batched: invalid arguments");
  if (frames == 0) return PGB_OK;
  PGB_REQUIRE(a && scratch && scalars, PGB_ERR_INVALID, "dot_f64_batched: null pointer");
  const dim3 grid(grid_for(n, kRedThreads, kRedBlocks), static_cast<unsigned>(frames));
  dot_f64_kernel<<<grid, kRedThreads, 0, as_stream(stream)>>>(
      static_cast<const float2*>(a), static_cast<const float2*>(b), n, static_cast<double*>(scratch),
      static_cast<double*>(scalars), out_slot, mode);
  PGB_LAUNCH_CHECK("dot_f64_batched");
  return PGB_OK;
}

int pgb_cg_update_xr_batched(void* x, void* r, const void* p, const void* Ap, int64_t n, int64_t frames,
                             const void* scalars, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0 && frames >= 0 && frames <= 65535, PGB_ERR_INVALID, "cg_update_xr_batched: invalid sizes");
  if (n == 0 || frames == 0) return PGB_OK;
  PGB_REQUIRE(x && r && p && Ap && scalars, PGB_ERR_INVALID, "cg_update_xr_batched: null pointer");
  const dim3 grid(grid_for(n, 256, 148 * 8), static_cast<unsigned>(frames));
  cg_update_xr_kernel<<<grid, 256, 0, as_stream(stream)>>>(
      static_cast<float2*>(x), static_cast<float2*>(r), static_cast<const float2*>(p),
      static_cast<const float2*>(Ap), n, static_cast<const double*>(scalars));
  PGB_LAUNCH_CHECK("cg_update_xr_batched");
  return PGB_OK;
}

int pgb_cg_update_p_batched(void* p, const void* r, int64_t n, int64_t frames, void* scalars, void* scratch,
                            void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0 && frames >= 0 && frames <= 65535, PGB_ERR_INVALID, "cg_update_p_batched: invalid sizes");
  if (n == 0 || frames == 0) return PGB_OK;
  PGB_REQUIRE(p && r && scalars && scratch, PGB_ERR_INVALID, "cg_update_p_batched: null pointer");
  const dim3 grid(grid_for(n, 256, 148 * 8), static_cast<unsigned>(frames));
  cg_update_p_kernel<<<grid, 256, 0, as_stream(stream)>>>(static_cast<float2*>(p), static_cast<const float2*>(r),
                                                          n, static_cast<double*>(scalars),
                                                          static_cast<double*>(scratch));
  PGB_LAUNCH_CHECK("cg_update_p_batched");
  return PGB_OK;
}

int pgb_axpy(void* y, const void* x, float a, int64_t n, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0, PGB_ERR_INVALID, "axpy: negative size");
  if (n == 0) return PGB_OK;
  PGB_REQUIRE(x && y, PGB_ERR_INVALID, "axpy: null pointer");
  axpy_kernel<<<grid_for(n, 256, 148 * 8), 256, 0, as_stream(stream)>>>(static_cast<float2*>(y),
                                                                      static_cast<const float2*>(x), a, n);
  PGB_LAUNCH_CHECK("axpy");
  return PGB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant of dot_f64: per-row FP64 inner products of
// `rows` contiguous vectors, with its block partials and completion counters
// in a fixed file-scope device array instead of caller-supplied scratch.
// ---------------------------------------------------------------------------
namespace pgb {

constexpr int kNoAllocMaxRows = 64;
constexpr int kNoAllocPartials = kNoAllocMaxRows * kRedBlocks;       // doubles
constexpr int kNoAllocCounterWords = kNoAllocMaxRows / 2;            // doubles holding the counters
constexpr int kNoAllocWords = kNoAllocPartials + kNoAllocCounterWords;  // 151,808 bytes

static_assert(kNoAllocCounterWords * sizeof(double) >= kNoAllocMaxRows * sizeof(unsigned),
              "counter words hold one unsigned per row");

// Partials: row r, block k at [r * kRedBlocks + k]; counters: unsigned[64]
// after the partials.  Only the counters must start at zero; every call
// clears the ones it uses on its stream before the kernel runs.
static __device__ __align__(256) double g_dot_rows_scratch[kNoAllocWords];

__global__ void __launch_bounds__(kRedThreads) dot_f64_rows_kernel(const float2* __restrict__ a,
                                                                   const float2* __restrict__ b, int64_t n,
                                                                   double* __restrict__ out,
                                                                   double* __restrict__ scratch) {
  const int row = blockIdx.y;
  const float2* ar = a + static_cast<int64_t>(row) * n;
  const float2* br = b ? b + static_cast<int64_t>(row) * n : nullptr;
  double acc = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float2 x = ar[i];
    if (br) {
      const float2 y = br[i];
      acc += static_cast<double>(x.x) * y.x + static_cast<double>(x.y) * y.y;
    } else {
      acc += static_cast<double>(x.x) * x.x + static_cast<double>(x.y) * x.y;
    }
  }
  const double s = block_sum(acc);
  double* part = scratch + static_cast<int64_t>(row) * kRedBlocks;
  unsigned* counter = reinterpret_cast<unsigned*>(scratch + kNoAllocPartials) + row;
  __shared__ bool last;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = s;
    __threadfence();
    last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int i = threadIdx.x; i < static_cast<int>(gridDim.x); i += blockDim.x) t += part[i];
  t = block_sum(t);
  if (threadIdx.x == 0) {
    out[row] = t;
    *counter = 0u;
  }
}

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};
void* g_noalloc_ctx[kNoAllocMaxDevices] = {};  // context the cached address belongs to

// The calling thread's current driver context (nullptr when none is current
// yet, or when the driver entry point is unavailable).
void* current_context() {
  using CtxGetCurrent = CUresult (*)(CUcontext*);
  static CtxGetCurrent get = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get = reinterpret_cast<CtxGetCurrent>(fn);
    else
      cudaGetLastError();
  }
  CUcontext c = nullptr;
  if (get == nullptr || get(&c) != CUDA_SUCCESS) return nullptr;
  return static_cast<void*>(c);
}

// Device address of g_dot_rows_scratch on the current device, looked up with
// that device current and cached per (device, context): after
// cudaDeviceReset the primary context, and with it the address, is new, so
// a changed context triggers a fresh lookup.
int noalloc_scratch(double** ptr) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error("dot_f64_noalloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
    return PGB_ERR_CUDA;
  }
  PGB_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, PGB_ERR_RANGE,
              "dot_f64_noalloc: device ordinal %d above the supported %d", dev, kNoAllocMaxDevices);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  void* ctx = current_context();
  if (!g_noalloc_ptr[dev] || ctx == nullptr || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_dot_rows_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("dot_f64_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                cudaGetErrorString(e));
      return PGB_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<double*>(p);
    g_noalloc_ctx[dev] = current_context();  // the lookup made the primary context current
  }
  *ptr = g_noalloc_ptr[dev];
  return PGB_OK;
}
}  // namespace

}  // namespace pgb

extern "C" {

int pgb_dot_f64_noalloc(const void* a, const void* b, int64_t n, int64_t rows, double* out, void* stream) {
  clear_error();
  PGB_REQUIRE(n >= 0 && rows >= 0, PGB_ERR_INVALID, "dot_f64_noalloc: negative size");
  PGB_REQUIRE(rows <= kNoAllocMaxRows, PGB_ERR_RANGE,
              "dot_f64_noalloc: rows=%lld exceeds the static scratch maximum of %d rows", (long long)rows,
              kNoAllocMaxRows);
  if (rows == 0) return PGB_OK;
  PGB_REQUIRE(out && (a || n == 0), PGB_ERR_INVALID, "dot_f64_noalloc: null pointer");
  double* scratch = nullptr;
  const int st = noalloc_scratch(&scratch);
  if (st != PGB_OK) return st;
  cudaStream_t s = as_stream(stream);
  cudaError_t e = cudaMemsetAsync(scratch + kNoAllocPartials, 0, static_cast<size_t>(rows) * sizeof(unsigned), s);
  if (e != cudaSuccess) {
    set_error("dot_f64_noalloc: clearing the counters failed: %s", cudaGetErrorString(e));
    return PGB_ERR_CUDA;
  }
  const dim3 grid(grid_for(n, kRedThreads, kRedBlocks), static_cast<unsigned>(rows));
  dot_f64_rows_kernel<<<grid, kRedThreads, 0, s>>>(static_cast<const float2*>(a),
                                                   static_cast<const float2*>(b), n, out, scratch);
  PGB_LAUNCH_CHECK("dot_f64_noalloc");
  return PGB_OK;
}

}  // extern "C"
