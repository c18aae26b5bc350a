// fft_stage.cu -- pointwise stages around cuFFT for SparseFFT / MaskedFFT /
// the GROG Toeplitz normal operator.
//
// Reference: operator/_sparse_fft.py:574-621, 741-789, 1154-1177 (per-coil
// scatter -> centred IFFT -> crop -> conj-smaps accumulate, and smaps ->
// pad -> centred FFT -> gather -> unsort), operator/_masked_fft.py:
// 322-361, 408-430, _toep/_grog_toep.py:154-209, _base/_fftc.py:114-139.
//
// Centred transforms fftshift(fft(ifftshift(.))) are never materialised:
// the buffers handed to cuFFT are kept in "FFT order", where centred grid
// position p (per axis, extent g) sits at m = (p - g/2) mod g.  Padding,
// cropping, shifting, the coil-sensitivity multiply, the coil sum and the
// ortho scale all happen inside these kernels, so each stage is one pass
// over the coil grids instead of the reference's pad / shift / multiply /
// shift / crop / accumulate passes per coil.
#include "common.cuh"

namespace pgb {

struct Shape3 {
  int nd;        // 2 or 3 (2-D uses axis 0 = 1)
  int g[3];      // grid extent per axis (z, y, x)
  int n[3];      // image extent per axis
  int off[3];    // (g - n) / 2 : image origin inside the centred grid
};

// FFT-order index m -> centred index p (per axis)
__device__ __forceinline__ int m2p(int m, int g) {
  int p = m + g / 2;
  return p >= g ? p - g : p;
}
// centred index p -> FFT-order index m
__device__ __forceinline__ int p2m(int p, int g) {
  int m = p - g / 2;
  return m < 0 ? m + g : m;
}

// u[b, c, m] = scale * S[c, q] * x[b, q]   (or x[b, c, q] without smaps)
// for every FFT-order grid position m; zero outside the image.  One grid
// row (b, c, m0, m1) per block step: the row is decoded once and its
// threads run along x, so no element pays an integer division.
__global__ void fft_expand_kernel(const float2* __restrict__ x, const float2* __restrict__ smaps,
                                  float2* __restrict__ u, int B, int C, Shape3 s, float scale,
                                  int x_has_coils) {
  const int64_t I = static_cast<int64_t>(s.n[0]) * s.n[1] * s.n[2];
  const int g2 = s.g[2];
  const int64_t plane = static_cast<int64_t>(s.g[0]) * s.g[1];  // rows of one (b, c) grid
  const int64_t rows = static_cast<int64_t>(B) * C * plane;
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const int64_t bc = r / plane;
    const int rem = static_cast<int>(r - bc * plane);
    const int m0 = rem / s.g[1], m1 = rem - m0 * s.g[1];
    const int c = static_cast<int>(bc % C);
    const int64_t b = bc / C;
    const int q0 = m2p(m0, s.g[0]) - s.off[0];
    const int q1 = m2p(m1, s.g[1]) - s.off[1];
    float2* urow = u + r * g2;
    if (q0 < 0 || q0 >= s.n[0] || q1 < 0 || q1 >= s.n[1]) {  // block-uniform: a padding row
      for (int m2 = threadIdx.x; m2 < g2; m2 += blockDim.x) urow[m2] = make_float2(0.f, 0.f);
      continue;
    }
    const int64_t qrow = (static_cast<int64_t>(q0) * s.n[1] + q1) * s.n[2];
    const float2* xrow = x + (x_has_coils ? (b * C + c) * I : b * I) + qrow;
    const float2* srow = smaps ? smaps + static_cast<int64_t>(c) * I + qrow : nullptr;
    for (int m2 = threadIdx.x; m2 < g2; m2 += blockDim.x) {
      const int q2 = m2p(m2, g2) - s.off[2];
      float2 v = make_float2(0.f, 0.f);
      if (q2 >= 0 && q2 < s.n[2]) {
        v = xrow[q2];
        if (!x_has_coils && smaps) v = cmul(v, srow[q2]);
        v = cscale(v, scale);
      }
      urow[m2] = v;
    }
  }
}

// out[b, q] = scale * sum_c conj(S[c, q]) v[b, c, m(q)]   (smaps)
// out[b, c, q] = scale * v[b, c, m(q)]                      (no smaps)
// optionally + add_scale * add[b, (c,) q]  (damped normal equations).
// One output per thread: image row r = (b, (c,) q0, q1) from blockIdx.y
// (grid-stride) and threadIdx.y, q2 from blockIdx.x and threadIdx.x, so the
// only divisions are the row's.
__global__ void fft_combine_kernel(const float2* __restrict__ v, const float2* __restrict__ smaps,
                                   float2* __restrict__ out, int B, int C, Shape3 s, float scale,
                                   const float2* __restrict__ add, float add_scale) {
  const int64_t G = static_cast<int64_t>(s.g[0]) * s.g[1] * s.g[2];
  const int64_t I = static_cast<int64_t>(s.n[0]) * s.n[1] * s.n[2];
  const int n2 = s.n[2];
  const int q2 = blockIdx.x * blockDim.x + threadIdx.x;
  if (q2 >= n2) return;
  const int64_t plane = static_cast<int64_t>(s.n[0]) * s.n[1];  // image rows of one output plane
  const int64_t rows = static_cast<int64_t>(B) * (smaps ? 1 : C) * plane;
  for (int64_t r = static_cast<int64_t>(blockIdx.y) * blockDim.y + threadIdx.y; r < rows;
       r += static_cast<int64_t>(gridDim.y) * blockDim.y) {
    const int64_t bc = r / plane;  // frame (smaps) or frame * C + coil
    const int rem = static_cast<int>(r - bc * plane);
    const int q0 = rem / s.n[1], q1 = rem - q0 * s.n[1];
    const int64_t qrow = static_cast<int64_t>(rem) * n2;
    {
      const int64_t m = (static_cast<int64_t>(p2m(q0 + s.off[0], s.g[0])) * s.g[1] +
                         p2m(q1 + s.off[1], s.g[1])) * s.g[2] + p2m(q2 + s.off[2], s.g[2]);
      float2 acc = make_float2(0.f, 0.f);
      if (smaps) {
#pragma unroll 4  // loads of four coils in flight per thread
        for (int c = 0; c < C; ++c)
          cfma_conj(acc, smaps[static_cast<int64_t>(c) * I + qrow + q2], v[(bc * C + c) * G + m]);
      } else {
        acc = v[bc * G + m];
      }
      acc = cscale(acc, scale);
      const int64_t t = r * n2 + q2;
      if (add) {
        const float2 a = add[t];
        acc.x = fmaf(add_scale, a.x, acc.x);
        acc.y = fmaf(add_scale, a.y, acc.y);
      }
      out[t] = acc;
    }
  }
}

// u[b, c, cellpos[r]] += w[r] * data[b, c, r]  (warp-aggregated atomics; u zeroed by caller)
// plane bc = b * C + c in y (grid-stride), replicas r in x
__global__ void __launch_bounds__(256) sparse_scatter_kernel(const float2* __restrict__ data,
                                                             const int32_t* __restrict__ cellpos,
                                                             const float* __restrict__ w,
                                                             float2* __restrict__ u, int BC, int64_t R,
                                                             int64_t G) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int bc = blockIdx.y; bc < BC; bc += gridDim.y) {
    const float2* drow = data + static_cast<int64_t>(bc) * R;
    for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x; base < R; base += stride) {
      const int64_t r = base + threadIdx.x;
      int64_t key = -1;
      float2 val = make_float2(0.f, 0.f);
      if (r < R) {
        const int32_t cp = cellpos[r];
        const float ww = w[r];
        if (cp >= 0 && cp < G && ww != 0.f) {
          key = static_cast<int64_t>(bc) * G + cp;
          val = cscale(drow[r], ww);
        }
      }
      const unsigned active = __ballot_sync(0xffffffffu, key >= 0);
      if (key >= 0) warp_aggregated_add(u, key, val, active);
    }
  }
}

// out[b, c, r] = w[r] * U[b, c, cellpos[r]]   (plane bc in y, replicas r in x)
__global__ void sparse_gather_kernel(const float2* __restrict__ U, const int32_t* __restrict__ cellpos,
                                     const float* __restrict__ w, float2* __restrict__ out, int BC,
                                     int64_t R, int64_t G) {
  for (int bc = blockIdx.y; bc < BC; bc += gridDim.y) {
    const float2* Ub = U + static_cast<int64_t>(bc) * G;
    float2* ob = out + static_cast<int64_t>(bc) * R;
    for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < R;
         r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const int32_t cp = cellpos[r];
      float2 v = make_float2(0.f, 0.f);
      if (cp >= 0 && cp < G) v = cscale(Ub[cp], w[r]);
      ob[r] = v;
    }
  }
}

// U[bc, m] *= psf[m]  (real point-spread function in FFT order): a thread
// per position m reads psf[m] once and scales it in kPsfRows planes
// bc = blockIdx.y * kPsfRows + j (no per-element modulo).
constexpr int kPsfRows = 4;
__global__ void psf_apply_kernel(float2* __restrict__ U, const float* __restrict__ psf, int BC, int64_t G) {
  const int bc0 = blockIdx.y * kPsfRows;
  const int nb = min(kPsfRows, BC - bc0);
  for (int64_t m = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; m < G;
       m += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float w = psf[m];
    float2* col = U + static_cast<int64_t>(bc0) * G + m;
#pragma unroll
    for (int j = 0; j < kPsfRows; ++j)
      if (j < nb) col[j * G] = cscale(col[j * G], w);
  }
}

// dst[bc, m] = scale * mask[p(m)] * src[bc, p(m)]   (centred -> FFT order)
// dst[bc, p] = scale * mask[p] * src[bc, m(p)]      (FFT order -> centred), to_centred = 1
// Grid rows (bc, i0, i1): threadIdx.y picks one of blockDim.y rows per block
// step, decoded once; the x threads run along the last axis.
__global__ void fft_shift_kernel(const float2* __restrict__ src, const float* __restrict__ mask,
                                 float2* __restrict__ dst, int BC, Shape3 s, float scale, int to_centred) {
  const int64_t G = static_cast<int64_t>(s.g[0]) * s.g[1] * s.g[2];
  const int g2 = s.g[2];
  const int64_t plane = static_cast<int64_t>(s.g[0]) * s.g[1];
  const int64_t rows = static_cast<int64_t>(BC) * plane;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.y + threadIdx.y; r < rows;
       r += static_cast<int64_t>(gridDim.x) * blockDim.y) {
    const int64_t bc = r / plane;
    const int rem = static_cast<int>(r - bc * plane);
    const int a0 = rem / s.g[1], a1 = rem - a0 * s.g[1];
    const int64_t irow = static_cast<int64_t>(rem) * g2;  // this row within the plane
    const int64_t jrow = to_centred
                             ? (static_cast<int64_t>(p2m(a0, s.g[0])) * s.g[1] + p2m(a1, s.g[1])) * g2
                             : (static_cast<int64_t>(m2p(a0, s.g[0])) * s.g[1] + m2p(a1, s.g[1])) * g2;
    const float2* srow = src + bc * G + jrow;
    float2* drow = dst + r * g2;
    for (int a2 = threadIdx.x; a2 < g2; a2 += blockDim.x) {
      const int j2 = to_centred ? p2m(a2, g2) : m2p(a2, g2);
      const float mk = mask ? mask[to_centred ? irow + a2 : jrow + j2] : 1.f;
      drow[a2] = cscale(srow[j2], scale * mk);
    }
  }
}

static int make_shape(int nd, const int64_t* grid, const int64_t* image, Shape3& s, const char* who) {
  PGB_REQUIRE(nd == 2 || nd == 3, PGB_ERR_INVALID, "%s: ndim must be 2 or 3", who);
  PGB_REQUIRE(grid != nullptr, PGB_ERR_INVALID, "%s: null grid shape", who);
  s.nd = nd;
  const int o = 3 - nd;
  for (int d = 0; d < 3; ++d) {
    s.g[d] = 1;
    s.n[d] = 1;
    s.off[d] = 0;
  }
  for (int d = 0; d < nd; ++d) {
    s.g[o + d] = static_cast<int>(grid[d]);
    s.n[o + d] = image ? static_cast<int>(image[d]) : static_cast<int>(grid[d]);
    PGB_REQUIRE(s.g[o + d] >= 1 && s.n[o + d] >= 1 && s.n[o + d] <= s.g[o + d], PGB_ERR_INVALID,
                "%s: image extent must be within the grid extent", who);
    s.off[o + d] = (s.g[o + d] - s.n[o + d]) / 2;
  }
  return PGB_OK;
}

}  // namespace pgb

using namespace pgb;

extern "C" {

int pgb_fft_expand(const void* x, const void* smaps, void* u, int64_t B, int64_t C, int ndim,
                   const int64_t* grid_shape, const int64_t* image_shape, float scale, int x_has_coils,
                   void* stream) {
  clear_error();
  Shape3 s;
  int st = make_shape(ndim, grid_shape, image_shape, s, "fft_expand");
  if (st) return st;
  PGB_REQUIRE(B >= 0 && C >= 1, PGB_ERR_INVALID, "fft_expand: invalid B/C");
  if (B == 0) return PGB_OK;
  PGB_REQUIRE(x && u, PGB_ERR_INVALID, "fft_expand: null pointer");
  const int64_t G = static_cast<int64_t>(s.g[0]) * s.g[1] * s.g[2];
  const int64_t rows = B * C * G / s.g[2];
  fft_expand_kernel<<<static_cast<int>(rows < 148 * 64 ? rows : 148 * 64), 128, 0, as_stream(stream)>>>(
      static_cast<const float2*>(x), static_cast<const float2*>(smaps), static_cast<float2*>(u),
      static_cast<int>(B), static_cast<int>(C), s, scale, x_has_coils);
  PGB_LAUNCH_CHECK("fft_expand");
  return PGB_OK;
}

int pgb_fft_combine(const void* v, const void* smaps, void* out, int64_t B, int64_t C, int ndim,
                    const int64_t* grid_shape, const int64_t* image_shape, float scale, const void* add,
                    float add_scale, void* stream) {
  clear_error();
  Shape3 s;
  int st = make_shape(ndim, grid_shape, image_shape, s, "fft_combine");
  if (st) return st;
  PGB_REQUIRE(B >= 0 && C >= 1, PGB_ERR_INVALID, "fft_combine: invalid B/C");
  if (B == 0) return PGB_OK;
  PGB_REQUIRE(v && out, PGB_ERR_INVALID, "fft_combine: null pointer");
  const int64_t I = static_cast<int64_t>(s.n[0]) * s.n[1] * s.n[2];
  const int64_t rows = B * (smaps ? 1 : C) * I / s.n[2];
  const dim3 grd((s.n[2] + 31) / 32, static_cast<unsigned>(grid_for(rows, 8, 65535)));
  fft_combine_kernel<<<grd, dim3(32, 8), 0, as_stream(stream)>>>(
      static_cast<const float2*>(v), static_cast<const float2*>(smaps), static_cast<float2*>(out),
      static_cast<int>(B), static_cast<int>(C), s, scale, static_cast<const float2*>(add), add_scale);
  PGB_LAUNCH_CHECK("fft_combine");
  return PGB_OK;
}

int pgb_sparse_scatter(const void* data, const int32_t* cellpos, const float* w, void* u, int64_t BC,
                       int64_t R, int64_t G, void* stream) {
  clear_error();
  PGB_REQUIRE(BC >= 0 && R >= 0 && G >= 0, PGB_ERR_INVALID, "sparse_scatter: negative size");
  if (BC == 0 || R == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(data && cellpos && w && u, PGB_ERR_INVALID, "sparse_scatter: null pointer");
  const unsigned ys = static_cast<unsigned>(BC < 65535 ? BC : 65535);
  const int xs = grid_for(R, 256, (148 * 16 + ys - 1) / ys);
  sparse_scatter_kernel<<<dim3(xs, ys), 256, 0, as_stream(stream)>>>(
      static_cast<const float2*>(data), cellpos, w, static_cast<float2*>(u), static_cast<int>(BC), R, G);
  PGB_LAUNCH_CHECK("sparse_scatter");
  return PGB_OK;
}

int pgb_sparse_gather(const void* U, const int32_t* cellpos, const float* w, void* out, int64_t BC,
                      int64_t R, int64_t G, void* stream) {
  clear_error();
  PGB_REQUIRE(BC >= 0 && R >= 0 && G >= 0, PGB_ERR_INVALID, "sparse_gather: negative size");
  if (BC == 0 || R == 0) return PGB_OK;
  PGB_REQUIRE(U && cellpos && w && out, PGB_ERR_INVALID, "sparse_gather: null pointer");
  const unsigned ys = static_cast<unsigned>(BC < 65535 ? BC : 65535);
  const int xs = grid_for(R, 256, (148 * 32 + ys - 1) / ys);
  sparse_gather_kernel<<<dim3(xs, ys), 256, 0, as_stream(stream)>>>(
      static_cast<const float2*>(U), cellpos, w, static_cast<float2*>(out), static_cast<int>(BC), R, G);
  PGB_LAUNCH_CHECK("sparse_gather");
  return PGB_OK;
}

int pgb_psf_apply(void* U, const float* psf, int64_t BC, int64_t G, void* stream) {
  clear_error();
  PGB_REQUIRE(BC >= 0 && G >= 0, PGB_ERR_INVALID, "psf_apply: negative size");
  if (BC == 0 || G == 0) return PGB_OK;
  PGB_REQUIRE(U && psf, PGB_ERR_INVALID, "psf_apply: null pointer");
  PGB_REQUIRE(BC <= 65535 * static_cast<int64_t>(kPsfRows), PGB_ERR_RANGE, "psf_apply: too many planes");
  const dim3 grd(grid_for(G, 256, 148 * 32), static_cast<unsigned>((BC + kPsfRows - 1) / kPsfRows));
  psf_apply_kernel<<<grd, 256, 0, as_stream(stream)>>>(static_cast<float2*>(U), psf, static_cast<int>(BC), G);
  PGB_LAUNCH_CHECK("psf_apply");
  return PGB_OK;
}

int pgb_fft_shift(const void* src, const float* mask, void* dst, int64_t BC, int ndim,
                  const int64_t* grid_shape, float scale, int to_centred, void* stream) {
  clear_error();
  Shape3 s;
  int st = make_shape(ndim, grid_shape, nullptr, s, "fft_shift");
  if (st) return st;
  PGB_REQUIRE(BC >= 0, PGB_ERR_INVALID, "fft_shift: negative size");
  if (BC == 0) return PGB_OK;
  PGB_REQUIRE(src && dst && src != dst, PGB_ERR_INVALID, "fft_shift: null or aliased pointers");
  const int64_t G = static_cast<int64_t>(s.g[0]) * s.g[1] * s.g[2];
  fft_shift_kernel<<<grid_for(BC * G / s.g[2], 4, 148 * 64), dim3(64, 4), 0, as_stream(stream)>>>(
      static_cast<const float2*>(src), mask, static_cast<float2*>(dst), static_cast<int>(BC), s, scale,
      to_centred);
  PGB_LAUNCH_CHECK("fft_shift");
  return PGB_OK;
}

}  // extern "C"
