// snapi_psf.cu -- Gaussian instrumental broadening of Stokes spectra and node responses
// (convolve_spectra_with_gauss, cmlib/mathtools.cc:1350-1414; used by stokes_lm_fit at
// atmos_fit.cc:104-109 on the synthetic Stokes vector and on every node response).
//
// One CTA per vector of 4 x nlambda values (a pixel's Stokes spectra, or one node's responses):
//   1. the vector on the reference's uniform fine grid (lambda_1 - 10 w .. lambda_N + 10 w, step
//      ~w/2) by its monotone quadratic Bezier interpolation (interpol_1d, mathtools.cc:1057-1117;
//      constant outside the original range), FP64 arithmetic on FP32 data;
//   2. the Gaussian integral exp(-(dl/w)^2) / (sqrt(pi) w) with the end weights halved, truncated
//      where the kernel drops below 1e-31 of its peak (beyond FP32 resolution);
//   3. the same interpolation back to the original grid.
// Deliberate deviation: for the first interval of a grid interpol_1d reads h2 before setting it;
// this uses the interval's width.  The reference's output near the blue end is then undefined
// (values up to 1e44 were observed, spread by the kernel tails over ~12 w); beyond that it agrees.
#include <cmath>
#include <cstring>
#include <vector>

#include "snapi_internal.cuh"

namespace {

constexpr int kPsfThreads = 128;

struct PsfConst {
  int nl, nf, band;
  double lmin, step;
  const double *lam;  // [nl] the spectra's wavelength grid (air, as the observation gives it)
  const float *kt;    // [band + 1] kernel x weight step at |m - n| = d
};

__device__ __forceinline__ double comp(const float4 &v, int c) {
  return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}

// monotone quadratic Bezier interpolation of the 4 channels f[0..N) at xq (interpol_1d); X(i) gives
// the grid, i the interval with X(i) <= xq < X(i+1) (already found), 0 <= i <= N - 2
template <class GX>
__device__ float4 bezier_at(const float4 *f, GX X, int N, int i, double xq) {
  double out[4];
  const double xi = X(i), xi1 = X(i + 1);
  const double hi2 = xi1 - xi;
  const double hprev = i > 0 ? xi - X(i - 1) : 0.0;
  const double hnext = i + 1 < N - 1 ? X(i + 2) - xi1 : 0.0;
  const double u = (xq - xi) / hi2;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double fi = comp(f[i], c), fi1 = comp(f[i + 1], c);
    double fd1, h2, h1;
    if (i > 0) {
      h1 = hprev;
      h2 = hi2;
      const double d1 = (fi - comp(f[i - 1], c)) / h1, d2 = (fi1 - fi) / h2;
      const double al = (1.0 + h2 / (h1 + h2)) / 3.0;
      fd1 = d1 * d2 > 0.0 ? d1 * d2 / (al * d2 + (1.0 - al) * d1) : 0.0;
    } else {
      h2 = hi2;  // the reference leaves h2 unset on the first interval
      h1 = hi2;
      fd1 = (fi1 - fi) / hi2;
    }
    const double C0 = fi + h2 * 0.5 * fd1;
    double fd2;
    if (i + 1 < N - 1) {
      h1 = hi2;
      const double d1 = (fi1 - fi) / h1, d2 = (comp(f[i + 2], c) - fi1) / hnext;
      const double al = (1.0 + hnext / (h1 + hnext)) / 3.0;
      fd2 = d1 * d2 > 0.0 ? d1 * d2 / (al * d2 + (1.0 - al) * d1) : 0.0;
    } else {
      fd2 = (comp(f[N - 1], c) - comp(f[N - 2], c)) / (X(N - 1) - X(N - 2));
    }
    const double C1 = fi1 - h1 * 0.5 * fd2;
    const double Cm = 0.5 * (C0 + C1);
    out[c] = (1.0 - u) * (1.0 - u) * fi + u * u * fi1 + u * 2.0 * (1.0 - u) * Cm;
  }
  return make_float4((float)out[0], (float)out[1], (float)out[2], (float)out[3]);
}

__global__ void __launch_bounds__(kPsfThreads) k_broaden(float4 *data, int nvec, int vec_per_pix, const int *skip,
                                                         PsfConst C) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int v = blockIdx.x;
  if (skip && skip[v / vec_per_pix]) return;  // CTA-uniform
  float4 *in = reinterpret_cast<float4 *>(smem);
  float4 *fine = in + C.nl;
  float4 *conv = fine + C.nf;
  float4 *g = data + (size_t)v * C.nl;
  for (int l = threadIdx.x; l < C.nl; l += blockDim.x) in[l] = g[l];
  __syncthreads();
  const double *lam = C.lam;
  auto Xc = [lam](int i) { return lam[i]; };
  const double lmin = C.lmin, step = C.step;
  auto Xf = [lmin, step](int i) { return lmin + i * step; };
  // 1. onto the fine grid
  for (int m = threadIdx.x; m < C.nf; m += blockDim.x) {
    const double xq = Xf(m);
    float4 r;
    if (!(xq < lam[C.nl - 1] && xq > lam[0])) {
      r = xq >= lam[C.nl - 1] ? in[C.nl - 1] : in[0];
    } else {  // first i with xq < lam[i + 1]
      int lo = 0, hi = C.nl - 2;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (xq < lam[mid + 1]) hi = mid; else lo = mid + 1;
      }
      r = bezier_at(in, Xc, C.nl, lo, xq);
    }
    fine[m] = r;
  }
  __syncthreads();
  // 2. Gaussian integral (kernel x weights tabulated by |m - n|; half weights at both ends)
  for (int m = threadIdx.x; m < C.nf; m += blockDim.x) {
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    const int n0 = max(0, m - C.band), n1 = min(C.nf - 1, m + C.band);
    for (int n = n0; n <= n1; ++n) {
      float k = C.kt[abs(m - n)];
      if (n == 0 || n == C.nf - 1) k *= 0.5f;
      const float4 f = fine[n];
      a.x += k * f.x; a.y += k * f.y; a.z += k * f.z; a.w += k * f.w;
    }
    conv[m] = a;
  }
  __syncthreads();
  // 3. back onto the original grid
  for (int l = threadIdx.x; l < C.nl; l += blockDim.x) {
    const double xq = lam[l];
    float4 r;
    if (!(xq < Xf(C.nf - 1) && xq > Xf(0))) {
      r = xq >= Xf(C.nf - 1) ? conv[C.nf - 1] : conv[0];
    } else {
      int i = (int)floor((xq - lmin) / step);
      i = min(max(i, 0), C.nf - 2);
      while (i > 0 && !(xq >= Xf(i))) --i;          // exact strict-comparison search, as the
      while (i < C.nf - 2 && !(xq < Xf(i + 1))) ++i;  // reference's linear scan finds it
      r = bezier_at(conv, Xf, C.nf, i, xq);
    }
    g[l] = r;
  }
}

}  // namespace

namespace snapi {

// set-up of one broadening width on the context's wavelength grid (host)
int psf_prepare(snapi_ctx *ctx, double width) {
  if (!(width > 0.0)) return set_err(ctx, SNAPI_EINVAL, "spectral broadening width must be positive");
  if (ctx->psf_width == width && ctx->d_psf_kt) return SNAPI_OK;
  const std::vector<double> &lam = ctx->h_lamair;
  const double lmin = lam.front() - 10.0 * width, lmax = lam.back() + 10.0 * width;
  const int nf = int((lmax - lmin) / (0.5 * width)) + 1;
  const double step = (lmax - lmin) / (nf - 1);
  int band = (int)floor(8.5 * width / step);
  if (band > nf - 1) band = nf - 1;
  const size_t smem = sizeof(float4) * ((size_t)ctx->nl + 2 * (size_t)nf);
  if (smem > 200 * 1024)
    return set_err(ctx, SNAPI_EINVAL, "spectral broadening: %d fine-grid points exceed one CTA's shared memory", nf);
  std::vector<float> kt(band + 1);
  for (int d = 0; d <= band; ++d) {
    const double dl = d * step;
    kt[d] = (float)(0.56418958354 / width * exp(-dl * dl / width / width) * step);
  }
  SNAPI_CK(cudaSetDevice(ctx->device));
  SNAPI_CK(cudaStreamSynchronize(ctx->stream));
  cudaFree(ctx->d_psf_kt);
  ctx->d_psf_kt = nullptr;
  SNAPI_CK(cudaMalloc(&ctx->d_psf_kt, sizeof(float) * kt.size()));
  SNAPI_CK(cudaMemcpy(ctx->d_psf_kt, kt.data(), sizeof(float) * kt.size(), cudaMemcpyHostToDevice));
  SNAPI_CK(cudaFuncSetAttribute(k_broaden, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ctx->psf_width = width;
  ctx->psf_nf = nf;
  ctx->psf_band = band;
  ctx->psf_lmin = lmin;
  ctx->psf_step = step;
  return SNAPI_OK;
}

// broaden nvec device vectors [nvec][nl][4] in place; vectors of pixel p (vec_per_pix each) are
// skipped where skip[p] != 0 (skip may be null)
cudaError_t psf_launch(const snapi_ctx *ctx, float *data, int nvec, int vec_per_pix, const int *skip) {
  if (nvec <= 0) return cudaSuccess;
  PsfConst C;
  C.nl = ctx->nl; C.nf = ctx->psf_nf; C.band = ctx->psf_band; C.lmin = ctx->psf_lmin; C.step = ctx->psf_step;
  C.lam = ctx->d_lamair; C.kt = ctx->d_psf_kt;
  const size_t smem = sizeof(float4) * ((size_t)ctx->nl + 2 * (size_t)ctx->psf_nf);
  k_broaden<<<nvec, kPsfThreads, smem, ctx->stream>>>(reinterpret_cast<float4 *>(data), nvec, vec_per_pix, skip, C);
  return cudaGetLastError();
}

}  // namespace snapi

extern "C" {

int snapi_spectral_broaden(snapi_ctx *ctx, int nvec, float *spectra, double width, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (nvec < 0 || (nvec > 0 && !spectra) || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return snapi::set_err(ctx, SNAPI_EINVAL, "snapi_spectral_broaden: invalid arguments");
  int st = snapi::psf_prepare(ctx, width);
  if (st) return st;
  if (nvec == 0) return SNAPI_OK;
  const size_t n = (size_t)ctx->nl * 4;
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int v0 = 0; v0 < nvec; v0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, nvec - v0);
    float *d = spectra + (size_t)v0 * n;
    if (mem == SNAPI_MEM_HOST) {
      d = ctx->d_stokes;  // max_batch x nl x 4 floats of staging
      SNAPI_CK(cudaMemcpyAsync(d, spectra + (size_t)v0 * n, sizeof(float) * nb * n, cudaMemcpyHostToDevice,
                               ctx->stream));
    }
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    SNAPI_CK(snapi::psf_launch(ctx, d, nb, 1, nullptr));
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_launches += 1;
    if (mem == SNAPI_MEM_HOST)
      SNAPI_CK(cudaMemcpyAsync(spectra + (size_t)v0 * n, d, sizeof(float) * nb * n, cudaMemcpyDeviceToHost,
                               ctx->stream));
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return SNAPI_OK;
}

}  // extern "C"
