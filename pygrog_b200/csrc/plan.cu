// plan.cu -- GROG plan geometry on the device, bit-exact against the
// reference's float32 host computation.
//
// Reference: calib/_grog.py:1125-1212 (_create_plan_single: nearest cell,
// target cells, distances, validity, EGROG Gaussian weights) and
// calib/_grog.py:406-417 (calc_interp_table shift quantisation).  Torch CPU
// evaluates each elementwise op separately in float32 with IEEE rounding and
// round-half-to-even; here every op is written with an explicit __f*_rn
// intrinsic and rintf so that nvcc cannot contract or reassociate them.
#include "common.cuh"

namespace pgb {

struct Axes3 {
  int64_t gshape[3];
  int64_t stride[3];
  float origin[3];
  float step[3];
};

__global__ void plan_geometry_kernel(const float* __restrict__ coords, int64_t npts, int ndim,
                                     const int32_t* __restrict__ offsets, int kw, Axes3 ax,
                                     int64_t* __restrict__ target, float* __restrict__ dist,
                                     float* __restrict__ gauss) {
  const int64_t R = npts * kw;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < R;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t n = r / kw;
    const int j = static_cast<int>(r - n * kw);
    bool valid = true;
    int64_t flat = 0;
    float dsq = 0.f;
    for (int d = 0; d < ndim; ++d) {
      const float c = coords[n * ndim + d];
      // frac_idx = (coords - origins) / grid_steps; nearest = round(frac_idx)
      const float frac = __fdiv_rn(__fsub_rn(c, ax.origin[d]), ax.step[d]);
      const int nearest = static_cast<int>(rintf(frac));
      const int t = nearest + offsets[j * ndim + d];
      // target_coords = origins + target_nd * grid_steps; distance = target - source
      const float tc = __fadd_rn(ax.origin[d], __fmul_rn(static_cast<float>(t), ax.step[d]));
      const float dd = __fsub_rn(tc, c);
      dist[r * ndim + d] = dd;
      valid = valid && (t >= 0) && (t < ax.gshape[d]) && (fabsf(dd) <= 0.5f);
      flat += static_cast<int64_t>(t) * ax.stride[d];
      const float dg = __fdiv_rn(dd, ax.step[d]);
      dsq = __fadd_rn(dsq, __fmul_rn(dg, dg));
    }
    target[r] = valid ? flat : -1;
    gauss[r] = valid ? expf(__fmul_rn(-0.5f, dsq)) : 0.f;
  }
}

__global__ void plan_gauss_sum_kernel(const int64_t* __restrict__ target,
                                      const float* __restrict__ gauss, int64_t R,
                                      double* __restrict__ gsum, int64_t G) {
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < R;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = target[r];
    if (t >= 0 && t < G) atomicAdd(gsum + t, static_cast<double>(gauss[r]));
  }
}

__global__ void plan_weights_kernel(const int64_t* __restrict__ target,
                                    const float* __restrict__ gauss,
                                    const double* __restrict__ gsum, int64_t R,
                                    float* __restrict__ w) {
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < R;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t t = target[r];
    float v = 0.f;
    if (t >= 0) {
      double s = gsum[t];
      if (s < 1e-12) s = 1e-12;
      v = __fdiv_rn(gauss[r], static_cast<float>(s));
    }
    w[r] = v;
  }
}

__global__ void plan_quantize_kernel(const float* __restrict__ dist, int64_t R, int ndim,
                                     float radius, float pfac, float stepsize, int nsteps,
                                     int64_t K, int64_t* __restrict__ out) {
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < R;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    int64_t acc = 0;
    float stride = 1.f;
    for (int d = 0; d < ndim; ++d) {
      const float dd = dist[r * ndim + d];
      const float a = rintf(__fmul_rn(dd, pfac));
      const float b = __fdiv_rn(a, pfac);
      const float c = __fadd_rn(radius, b);
      const float e = rintf(__fdiv_rn(c, stepsize));
      const float s = rintf(__fmul_rn(e, stride));
      acc += static_cast<int64_t>(static_cast<int32_t>(s));
      stride = __fmul_rn(stride, static_cast<float>(nsteps));
    }
    if (acc < 0) acc = 0;
    if (acc > K - 1) acc = K - 1;
    out[r] = acc;
  }
}

}  // namespace pgb

using namespace pgb;

extern "C" {

int pgb_plan_geometry(const float* coords_scaled, int64_t npts, int ndim, const int32_t* offsets,
                      int kw, const int64_t* grid_shape, const float* origins,
                      const float* grid_steps, int64_t* target_idx, float* distances, float* gauss,
                      void* stream) {
  clear_error();
  PGB_REQUIRE(ndim >= 1 && ndim <= 3, PGB_ERR_INVALID, "plan_geometry: ndim must be 1..3, got %d",
              ndim);
  PGB_REQUIRE(npts >= 0 && kw >= 1, PGB_ERR_INVALID, "plan_geometry: invalid sizes");
  if (npts == 0) return PGB_OK;
  PGB_REQUIRE(coords_scaled && offsets && grid_shape && origins && grid_steps && target_idx &&
                  distances && gauss,
              PGB_ERR_INVALID, "plan_geometry: null pointer");
  Axes3 ax{};
  int64_t st = 1;
  for (int d = ndim - 1; d >= 0; --d) {
    ax.gshape[d] = grid_shape[d];
    ax.stride[d] = st;
    st *= grid_shape[d];
    ax.origin[d] = origins[d];
    ax.step[d] = grid_steps[d];
  }
  const int64_t R = npts * kw;
  plan_geometry_kernel<<<grid_for(R, 256, 148 * 32), 256, 0, as_stream(stream)>>>(
      coords_scaled, npts, ndim, offsets, kw, ax, target_idx, distances, gauss);
  PGB_LAUNCH_CHECK("plan_geometry");
  return PGB_OK;
}

int pgb_plan_gauss_sum(const int64_t* target_idx, const float* gauss, int64_t R, double* gauss_sum,
                       int64_t G, void* stream) {
  clear_error();
  PGB_REQUIRE(R >= 0 && G >= 0, PGB_ERR_INVALID, "plan_gauss_sum: negative size");
  if (R == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(target_idx && gauss && gauss_sum, PGB_ERR_INVALID, "plan_gauss_sum: null pointer");
  plan_gauss_sum_kernel<<<grid_for(R, 256, 148 * 32), 256, 0, as_stream(stream)>>>(
      target_idx, gauss, R, gauss_sum, G);
  PGB_LAUNCH_CHECK("plan_gauss_sum");
  return PGB_OK;
}

int pgb_plan_weights(const int64_t* target_idx, const float* gauss, const double* gauss_sum,
                     int64_t R, float* weights, void* stream) {
  clear_error();
  PGB_REQUIRE(R >= 0, PGB_ERR_INVALID, "plan_weights: negative size");
  if (R == 0) return PGB_OK;
  PGB_REQUIRE(target_idx && gauss && gauss_sum && weights, PGB_ERR_INVALID,
              "plan_weights: null pointer");
  plan_weights_kernel<<<grid_for(R, 256, 148 * 32), 256, 0, as_stream(stream)>>>(
      target_idx, gauss, gauss_sum, R, weights);
  PGB_LAUNCH_CHECK("plan_weights");
  return PGB_OK;
}

int pgb_plan_quantize(const float* distances, int64_t R, int ndim, float radius, float pfac,
                      float stepsize, int nsteps, int64_t K, int64_t* interp_idx, void* stream) {
  clear_error();
  PGB_REQUIRE(ndim >= 1 && ndim <= 3 && R >= 0 && K >= 1 && nsteps >= 1, PGB_ERR_INVALID,
              "plan_quantize: invalid arguments");
  if (R == 0) return PGB_OK;
  PGB_REQUIRE(distances && interp_idx, PGB_ERR_INVALID, "plan_quantize: null pointer");
  plan_quantize_kernel<<<grid_for(R, 256, 148 * 32), 256, 0, as_stream(stream)>>>(
      distances, R, ndim, radius, pfac, stepsize, nsteps, K, interp_idx);
  PGB_LAUNCH_CHECK("plan_quantize");
  return PGB_OK;
}

}  // extern "C"
