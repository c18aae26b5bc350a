// subspace.cu -- sparse <-> grid transfers of the low-rank subspace operator.
//
// Reference: gadgets/_subspace.py (SubspaceSparseFFT._adjoint_single 311-400,
// _forward_single 424-508) and _toep/_sub_toep.py (SubspaceToeplitzOp,
// PSF 120-208, apply 236-303).  The reference loops over coils and subspace
// components with one scatter / FFT per (c, k); here one pass reads every
// sample once for all K components:
//
//   scatter: u[b, k, c, cell_r] += w_r * B[k, t_r] * y[b, c, r]
//   gather:  y[b, c, r] = w_r * sum_k conj(B[k, t_r]) * U[b, k, c, cell_r]
//   psf:     V[b, k, c, g] = sum_k' P[g, k, k'] * U[b, k', c, g]   (in place)
//
// cell_r is the FFT-order grid position, t_r the sample's index along the
// encoding (time / contrast) axis; samples with cell or t out of range
// contribute nothing (gather writes 0).
#include "common.cuh"

namespace pgb {

constexpr int kMaxK = 32;

__global__ void __launch_bounds__(256) subspace_scatter_kernel(
    const float2* __restrict__ y, const int32_t* __restrict__ cellpos, const float* __restrict__ w,
    const int32_t* __restrict__ tidx, const float2* __restrict__ basis, float2* __restrict__ u, int B, int C,
    int K, int T, int64_t R, int64_t G) {
  const int64_t total = static_cast<int64_t>(B) * C * R;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x; base < total; base += stride) {
    const int64_t t = base + threadIdx.x;
    bool ok = false;
    int64_t b = 0, c = 0, cp = 0;
    int ti = 0;
    float2 val = make_float2(0.f, 0.f);
    if (t < total) {
      const int64_t r = t % R;
      const int64_t bc = t / R;
      b = bc / C;
      c = bc - b * C;
      cp = cellpos[r];
      ti = tidx[r];
      const float ww = w[r];
      ok = cp >= 0 && cp < G && ti >= 0 && ti < T && ww != 0.f;
      if (ok) val = cscale(y[t], ww);
    }
    for (int k = 0; k < K; ++k) {  // warp-uniform
      int64_t key = -1;
      float2 v = make_float2(0.f, 0.f);
      if (ok) {
        key = ((b * K + k) * C + c) * G + cp;
        v = cmul(__ldg(basis + static_cast<int64_t>(k) * T + ti), val);
      }
      const unsigned active = __ballot_sync(0xffffffffu, key >= 0);
      if (key >= 0) warp_aggregated_add(u, key, v, active);
    }
  }
}

__global__ void subspace_gather_kernel(const float2* __restrict__ U, const int32_t* __restrict__ cellpos,
                                       const float* __restrict__ w, const int32_t* __restrict__ tidx,
                                       const float2* __restrict__ basis, float2* __restrict__ out, int B, int C,
                                       int K, int T, int64_t R, int64_t G) {
  const int64_t total = static_cast<int64_t>(B) * C * R;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = t % R;
    const int64_t bc = t / R;
    const int64_t b = bc / C;
    const int64_t c = bc - b * C;
    const int64_t cp = cellpos[r];
    const int ti = tidx[r];
    float2 acc = make_float2(0.f, 0.f);
    if (cp >= 0 && cp < G && ti >= 0 && ti < T) {
      for (int k = 0; k < K; ++k)
        cfma_conj(acc, __ldg(basis + static_cast<int64_t>(k) * T + ti), U[((b * K + k) * C + c) * G + cp]);
      acc = cscale(acc, w[r]);
    }
    out[t] = acc;
  }
}

template <int KK>
__global__ void psf_apply_kk_kernel(float2* __restrict__ U, const float2* __restrict__ P, int B, int C,
                                    int64_t G) {
  const int64_t total = static_cast<int64_t>(B) * C * G;
  for (int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t g = t % G;
    const int64_t bc = t / G;
    const int64_t b = bc / C;
    const int64_t c = bc - b * C;
    float2 in[KK];
#pragma unroll
    for (int k = 0; k < KK; ++k) in[k] = U[((b * KK + k) * C + c) * G + g];
    const float2* Pg = P + g * KK * KK;
#pragma unroll
    for (int k = 0; k < KK; ++k) {
      float2 acc = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 0; j < KK; ++j) cfma(acc, __ldg(Pg + k * KK + j), in[j]);
      U[((b * KK + k) * C + c) * G + g] = acc;
    }
  }
}

}  // namespace pgb

using namespace pgb;

extern "C" {

int pgb_subspace_scatter(const void* y, const int32_t* cellpos, const float* w, const int32_t* tidx,
                         const void* basis, void* u, int64_t B, int64_t C, int64_t K, int64_t T, int64_t R,
                         int64_t G, void* stream) {
  clear_error();
  PGB_REQUIRE(B >= 0 && C >= 0 && R >= 0 && G >= 0 && T >= 1 && K >= 1 && K <= kMaxK, PGB_ERR_INVALID,
              "subspace_scatter: invalid sizes (K must be 1..%d)", kMaxK);
  if (B == 0 || C == 0 || R == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(B * C < (int64_t(1) << 31), PGB_ERR_RANGE, "subspace_scatter: too many frames");
  PGB_REQUIRE(y && cellpos && w && tidx && basis && u, PGB_ERR_INVALID, "subspace_scatter: null pointer");
  subspace_scatter_kernel<<<grid_for(B * C * R, 256, 148 * 16), 256, 0, as_stream(stream)>>>(
      static_cast<const float2*>(y), cellpos, w, tidx, static_cast<const float2*>(basis), static_cast<float2*>(u),
      static_cast<int>(B), static_cast<int>(C), static_cast<int>(K), static_cast<int>(T), R, G);
  PGB_LAUNCH_CHECK("subspace_scatter");
  return PGB_OK;
}

int pgb_subspace_gather(const void* U, const int32_t* cellpos, const float* w, const int32_t* tidx,
                        const void* basis, void* out, int64_t B, int64_t C, int64_t K, int64_t T, int64_t R,
                        int64_t G, void* stream) {
  clear_error();
  PGB_REQUIRE(B >= 0 && C >= 0 && R >= 0 && G >= 0 && T >= 1 && K >= 1 && K <= kMaxK, PGB_ERR_INVALID,
              "subspace_gather: invalid sizes (K must be 1..%d)", kMaxK);
  if (B == 0 || C == 0 || R == 0) return PGB_OK;
  PGB_REQUIRE(B * C < (int64_t(1) << 31), PGB_ERR_RANGE, "subspace_gather: too many frames");
  PGB_REQUIRE(U && cellpos && w && tidx && basis && out, PGB_ERR_INVALID, "subspace_gather: null pointer");
  subspace_gather_kernel<<<grid_for(B * C * R, 256, 148 * 32), 256, 0, as_stream(stream)>>>(
      static_cast<const float2*>(U), cellpos, w, tidx, static_cast<const float2*>(basis),
      static_cast<float2*>(out), static_cast<int>(B), static_cast<int>(C), static_cast<int>(K),
      static_cast<int>(T), R, G);
  PGB_LAUNCH_CHECK("subspace_gather");
  return PGB_OK;
}

int pgb_psf_apply_kk(void* U, const void* P, int64_t B, int64_t K, int64_t C, int64_t G, void* stream) {
  clear_error();
  PGB_REQUIRE(B >= 0 && C >= 0 && G >= 0 && K >= 1 && K <= 16, PGB_ERR_INVALID,
              "psf_apply_kk: invalid sizes (K must be 1..16)");
  if (B == 0 || C == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(B * C < (int64_t(1) << 31), PGB_ERR_RANGE, "psf_apply_kk: too many frames");
  PGB_REQUIRE(U && P, PGB_ERR_INVALID, "psf_apply_kk: null pointer");
  const int blocks = grid_for(B * C * G, 256, 148 * 32);
  cudaStream_t s = as_stream(stream);
  switch (K) {
#define X(KV)                                                                                            \
  case KV:                                                                                               \
    psf_apply_kk_kernel<KV><<<blocks, 256, 0, s>>>(static_cast<float2*>(U), static_cast<const float2*>(P), \
                                                   static_cast<int>(B), static_cast<int>(C), G);          \
    break;
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)
#undef X
    default:
      break;
  }
  PGB_LAUNCH_CHECK("psf_apply_kk");
  return PGB_OK;
}

}  // extern "C"
