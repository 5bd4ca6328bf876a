// libsnapi_cuda -- sm_100a kernels and the C ABI of the SNAPI Stokes hot path.
//
// One CTA per pixel, one thread per wavelength (blockDim = nlambda rounded up to a warp).
// The pixel's column record is staged into shared memory with a TMA bulk copy
// (cp.async.bulk, completion on an mbarrier, bounded wait), the wavelength-independent
// per-depth constants are built once per CTA in shared memory, and every thread then runs
// the depth recursion of its wavelength in registers (snapi_sweep.cuh).  The adjoint kernel
// adds the reverse sweep; per-depth wavelength sums are reduced with warp shuffles and
// shared-memory atomics, chained to the record fields and contracted with the node tangents.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/snapi_cuda.h"
#include "snapi_sweep.cuh"

using namespace snapi;

namespace {

constexpr int kMaxThreads = SNAPI_MAX_LAMBDA;
constexpr long long kWaitLimit = 1LL << 26;  // mbarrier polls before a CTA gives up

// ------------------------------------------------------------------------------------------
// kernel parameters
struct KParams {
  int npix, nd, nl, nlines, nfield, npar, lpad, ncomp, nred;
  float lam_mid;
  double scale2;                // stokes_scale^2
  const float *rec;             // [npix][nd][nfield]
  const double *lamvac;         // [nl]
  const LineConst *lines;       // [nlines]
  const float *compS, *compD;   // [ncomp]
  const double *D;              // [nd-1]
  float *stokes;                // [npix][nl][4]
  const float *obs;             // [npix][nl][4]
  double ws[4];
  const float *mask;            // [npix][nl] or null
  const float *tangent;         // [npix][npar][nd][nfield] or null
  float4 *scratch;              // [npix][nd][4][lpad]
  double *rec_grad;             // [npix][nd][nfield] or null
  double *grad;                 // [npix][npar]
  double *chi2;                 // [npix] (or [npix][2 npar + 1] for fd)
  const double *fd_step;        // [npar]
  int *status;                  // device error word
};

struct SmemLayout {
  size_t rec, D, lines, compS, compD, dc, ld, acc, rb, mbar, wred, total;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

__host__ __device__ inline SmemLayout smem_layout(int nd, int nfield, int nlines, int ncomp, int nred, bool adj) {
  SmemLayout s;
  size_t o = 0;
  s.rec = o; o = align_up(o + sizeof(float) * nd * nfield, 16);
  s.D = o; o = align_up(o + sizeof(double) * (nd - 1), 16);
  s.lines = o; o = align_up(o + sizeof(LineConst) * (nlines > 0 ? nlines : 1), 16);
  s.compS = o; o = align_up(o + sizeof(float) * (ncomp > 0 ? ncomp : 1), 16);
  s.compD = o; o = align_up(o + sizeof(float) * (ncomp > 0 ? ncomp : 1), 16);
  s.dc = o; o = align_up(o + sizeof(DepthConst) * nd, 16);
  s.ld = o; o = align_up(o + sizeof(LineDepth) * nd * (nlines > 0 ? nlines : 1), 16);
  s.acc = o; if (adj) o = align_up(o + sizeof(float) * nd * nred, 16);
  s.rb = o; if (adj) o = align_up(o + sizeof(float) * nd * nfield, 16);
  s.mbar = o; o = align_up(o + 8, 16);
  s.wred = o; o = align_up(o + sizeof(double) * 32 * 16, 16);
  s.total = o;
  return s;
}

// ------------------------------------------------------------------------------------------
// TMA bulk copy global -> shared, completion tracked by an mbarrier (bounded wait)
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ bool tma_bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *mbar) {
  const uint32_t mb = smem_u32(mbar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mb));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(mb)
        : "memory");
  }
  uint32_t done = 0;
  for (long long it = 0; it < kWaitLimit && !done; ++it) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mb), "r"(0u)
        : "memory");
  }
  // every thread must take the same decision (the caller returns or syncs next)
  return __syncthreads_and(done != 0) != 0;
}

// ------------------------------------------------------------------------------------------
struct DevScratch {
  float4 *base;
  int lpad, l;
  __device__ void store(int z, const float *I, const float *kp, const float *S, float e, float tau) {
    float4 *p = base + (size_t)z * 4 * lpad + l;
    p[0] = make_float4(I[0], I[1], I[2], I[3]);
    p[lpad] = make_float4(kp[0], kp[1], kp[2], kp[3]);
    p[2 * lpad] = make_float4(kp[4], kp[5], e, tau);
    p[3 * lpad] = make_float4(S[0], S[1], S[2], S[3]);
  }
  __device__ void load(int z, float *I, float *kp, float *S, float &e, float &tau) const {
    const float4 *p = base + (size_t)z * 4 * lpad + l;
    float4 a = p[0], b = p[lpad], c = p[2 * lpad], d = p[3 * lpad];
    I[0] = a.x; I[1] = a.y; I[2] = a.z; I[3] = a.w;
    kp[0] = b.x; kp[1] = b.y; kp[2] = b.z; kp[3] = b.w;
    kp[4] = c.x; kp[5] = c.y; e = c.z; tau = c.w;
    S[0] = d.x; S[1] = d.y; S[2] = d.z; S[3] = d.w;
  }
};
struct NoScratch {
  __device__ void store(int, const float *, const float *, const float *, float, float) {}
};

struct DevReducer {
  float *acc;
  int nred;
  __device__ void add(int z, const float *red, int n) {
    const int lane = threadIdx.x & 31;
    for (int i = 0; i < n; ++i) {
      float v = red[i];
      v += __shfl_xor_sync(0xffffffffu, v, 16);
      v += __shfl_xor_sync(0xffffffffu, v, 8);
      v += __shfl_xor_sync(0xffffffffu, v, 4);
      v += __shfl_xor_sync(0xffffffffu, v, 2);
      v += __shfl_xor_sync(0xffffffffu, v, 1);
      if (lane == 0) atomicAdd(&acc[z * nred + i], v);
    }
  }
};

__device__ double block_sum(double v, double *wred) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) wred[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) s += wred[i];
  __syncthreads();
  return s;  // valid in thread 0
}

// Stage one pixel into shared memory and build the per-depth constants.  fd_pert: -1 none,
// otherwise the record is perturbed by sign * fd_step[p] * tangent_p (p = fd_pert).
__device__ bool stage_pixel(const KParams &P, int pix, unsigned char *smem, const SmemLayout &L, PixelView &pv,
                            int fd_pert, float fd_sign) {
  float *rec = reinterpret_cast<float *>(smem + L.rec);
  double *D = reinterpret_cast<double *>(smem + L.D);
  LineConst *lc = reinterpret_cast<LineConst *>(smem + L.lines);
  float *cS = reinterpret_cast<float *>(smem + L.compS);
  float *cD = reinterpret_cast<float *>(smem + L.compD);
  DepthConst *dc = reinterpret_cast<DepthConst *>(smem + L.dc);
  LineDepth *ld = reinterpret_cast<LineDepth *>(smem + L.ld);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + L.mbar);
  const int nrec = P.nd * P.nfield;
  const float *src = P.rec + (size_t)pix * nrec;
  const uint32_t bytes = (uint32_t)(sizeof(float) * nrec);
  bool ok = true;
  if ((bytes % 16u) == 0u && (reinterpret_cast<uintptr_t>(src) % 16u) == 0u) {
    ok = tma_bulk_load(rec, src, bytes, mbar);
  } else {
    for (int i = threadIdx.x; i < nrec; i += blockDim.x) rec[i] = src[i];
  }
  for (int i = threadIdx.x; i < P.nd - 1; i += blockDim.x) D[i] = P.D[i];
  for (int i = threadIdx.x; i < P.nlines; i += blockDim.x) lc[i] = P.lines[i];
  for (int i = threadIdx.x; i < P.ncomp; i += blockDim.x) { cS[i] = P.compS[i]; cD[i] = P.compD[i]; }
  __syncthreads();
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(P.status, SNAPI_ETIMEOUT);
    return false;
  }
  if (fd_pert >= 0) {
    const float *tp = P.tangent + ((size_t)pix * P.npar + fd_pert) * nrec;
    const float h = fd_sign * (float)P.fd_step[fd_pert];
    for (int i = threadIdx.x; i < nrec; i += blockDim.x) rec[i] += h * tp[i];
    __syncthreads();
  }
  for (int z = threadIdx.x; z < P.nd; z += blockDim.x)
    depth_precompute(rec + z * P.nfield, P.nlines, lc, P.lam_mid, dc[z], ld + z * P.nlines);
  __syncthreads();
  pv.nd = P.nd; pv.nlines = P.nlines; pv.nfield = P.nfield;
  pv.rec = rec; pv.dc = dc; pv.ld = ld; pv.lc = lc; pv.compS = cS; pv.compD = cD; pv.D = D;
  return true;
}

__device__ void thread_lambda(const KParams &P, const PixelView &pv, int l, LamConst &lam, float *delta) {
  const double lv = P.lamvac[l];
  lambda_precompute(lv, lam);
  for (int j = 0; j < P.nlines; ++j) delta[j] = (float)(pv.lc[j].lam0 - lv);
}

// ------------------------------------------------------------------------------------------
template <int MAXT>
__global__ void __launch_bounds__(MAXT) k_synth(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const int pix = blockIdx.x;
  PixelView pv;
  if (!stage_pixel(P, pix, smem, L, pv, -1, 0.f)) return;
  const int l = threadIdx.x;
  const int le = l < P.nl ? l : P.nl - 1;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, le, lam, delta);
  float out[4];
  NoScratch ns;
  forward_sweep<false>(pv, lam, delta, out, ns);
  if (l < P.nl) {
    float4 *o = reinterpret_cast<float4 *>(P.stokes + ((size_t)pix * P.nl + l) * 4);
    *o = make_float4(out[0], out[1], out[2], out[3]);
  }
}

template <int MAXT>
__global__ void __launch_bounds__(MAXT) k_adjoint(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, true);
  const int pix = blockIdx.x;
  PixelView pv;
  float *acc = reinterpret_cast<float *>(smem + L.acc);
  float *rb = reinterpret_cast<float *>(smem + L.rb);
  double *wred = reinterpret_cast<double *>(smem + L.wred);
  for (int i = threadIdx.x; i < P.nd * P.nred; i += blockDim.x) acc[i] = 0.f;
  for (int i = threadIdx.x; i < P.nd * P.nfield; i += blockDim.x) rb[i] = 0.f;
  if (!stage_pixel(P, pix, smem, L, pv, -1, 0.f)) return;
  const int l = threadIdx.x;
  const bool active = l < P.nl;
  const int le = active ? l : P.nl - 1;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, le, lam, delta);
  DevScratch sc;
  sc.base = P.scratch + (size_t)pix * P.nd * 4 * P.lpad;
  sc.lpad = P.lpad;
  sc.l = l;
  float out[4];
  forward_sweep<true>(pv, lam, delta, out, sc);
  // residual and seed (atmos_fit.cc:229-248)
  float seed[4] = {0.f, 0.f, 0.f, 0.f};
  double c2 = 0.0;
  if (active) {
    if (P.stokes) {
      float4 *o = reinterpret_cast<float4 *>(P.stokes + ((size_t)pix * P.nl + l) * 4);
      *o = make_float4(out[0], out[1], out[2], out[3]);
    }
    const float m = P.mask ? P.mask[(size_t)pix * P.nl + l] : 1.0f;
    const float *ob = P.obs + ((size_t)pix * P.nl + l) * 4;
    const double is2 = 1.0 / P.scale2;
    for (int s = 0; s < 4; ++s) {
      const double r = ((double)ob[s] - (double)out[s]) * P.ws[s] * m;
      c2 += r * r * is2;
      seed[s] = (float)(-2.0 * r * P.ws[s] * m * is2);
    }
  }
  const double c2tot = block_sum(c2, wred);
  if (threadIdx.x == 0) P.chi2[pix] = c2tot * P.scale2;
  // reverse sweep
  DevReducer rd;
  rd.acc = acc;
  rd.nred = P.nred;
  float red[kNumRed + kRedPerLine * kMaxLines];
  reverse_sweep(pv, lam, delta, seed, sc, rd, red, P.nred);
  __syncthreads();
  // chain to the record fields
  for (int z = threadIdx.x; z < P.nd; z += blockDim.x)
    depth_chain_adjoint(pv.rec + z * P.nfield, P.nlines, pv.lc, P.lam_mid, pv.dc[z], pv.ld + z * P.nlines,
                        acc + z * P.nred, rb + z * P.nfield);
  __syncthreads();
  const int nrec = P.nd * P.nfield;
  if (P.rec_grad)
    for (int i = threadIdx.x; i < nrec; i += blockDim.x)
      P.rec_grad[(size_t)pix * nrec + i] = (double)rb[i] * P.scale2;
  // contraction with the node tangents
  for (int p = 0; p < P.npar; ++p) {
    const float *tp = P.tangent + ((size_t)pix * P.npar + p) * nrec;
    double g = 0.0;
    for (int i = threadIdx.x; i < nrec; i += blockDim.x) g += (double)rb[i] * (double)tp[i];
    const double gt = block_sum(g, wred);
    if (threadIdx.x == 0) P.grad[(size_t)pix * P.npar + p] = gt * P.scale2;
  }
}

// finite differences: blockIdx.y = 0 base, 2p+1 plus, 2p+2 minus; chi2 [npix][2 npar + 1]
template <int MAXT>
__global__ void __launch_bounds__(MAXT) k_fd(KParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout L = smem_layout(P.nd, P.nfield, P.nlines, P.ncomp, P.nred, false);
  const int pix = blockIdx.x, v = blockIdx.y;
  double *wred = reinterpret_cast<double *>(smem + L.wred);
  PixelView pv;
  const int pert = v == 0 ? -1 : (v - 1) / 2;
  const float sign = v == 0 ? 0.f : (((v - 1) & 1) ? -1.f : 1.f);
  if (!stage_pixel(P, pix, smem, L, pv, pert, sign)) return;
  const int l = threadIdx.x;
  const bool active = l < P.nl;
  const int le = active ? l : P.nl - 1;
  LamConst lam;
  float delta[kMaxLines];
  thread_lambda(P, pv, le, lam, delta);
  float out[4];
  NoScratch ns;
  forward_sweep<false>(pv, lam, delta, out, ns);
  double c2 = 0.0;
  if (active) {
    const float m = P.mask ? P.mask[(size_t)pix * P.nl + l] : 1.0f;
    const float *ob = P.obs + ((size_t)pix * P.nl + l) * 4;
    for (int s = 0; s < 4; ++s) {
      const double r = ((double)ob[s] - (double)out[s]) * P.ws[s] * m;
      c2 += r * r;
    }
  }
  const double c2tot = block_sum(c2, wred);
  if (threadIdx.x == 0) P.chi2[(size_t)pix * gridDim.y + v] = c2tot;
}

__global__ void k_fd_combine(int npix, int npar, const double *chi2v, const double *step, double *chi2, double *grad) {
  const int pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= npix) return;
  const int nv = 2 * npar + 1;
  const double *c = chi2v + (size_t)pix * nv;
  chi2[pix] = c[0];
  for (int p = 0; p < npar; ++p) grad[(size_t)pix * npar + p] = (c[2 * p + 1] - c[2 * p + 2]) / (2.0 * step[p]);
}

}  // namespace

// =============================================================================================
// host side
struct snapi_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int nd = 0, nl = 0, nlines = 0, nfield = 0, ncomp = 0, nred = 0, lpad = 0, max_batch = 0;
  float lam_mid = 0.f;
  double scale2 = 1.0;
  double *d_lamvac = nullptr, *d_D = nullptr;
  LineConst *d_lines = nullptr;
  float *d_compS = nullptr, *d_compD = nullptr;
  int *d_status = nullptr;
  // work buffers (max_batch pixels)
  float *d_rec = nullptr, *d_stokes = nullptr, *d_obs = nullptr, *d_mask = nullptr, *d_tan = nullptr;
  float *d_dstokes = nullptr;
  double *d_recgrad = nullptr;
  double *d_grad = nullptr, *d_chi2 = nullptr, *d_chi2v = nullptr, *d_step = nullptr;
  float4 *d_scratch = nullptr;
  int cap_npar = 0;
  double last_ms = 0.0;
  int last_launches = 0;
  std::string err;
};

namespace {

int set_err(snapi_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return code;
}

#define CK(call)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return set_err(ctx, SNAPI_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

double airtovac_d(double lambda_air) {  // cmlib/mathtools.cc:1325-1330
  double s = 1E4 / (lambda_air * 1E8);
  double n = 1.0 + 0.00008336624212083 + 0.02408926869968 / (130.1065924522 - s * s) +
             0.0001599740894897 / (38.92568793293 - s * s);
  return lambda_air * n;
}

int ensure_npar(snapi_ctx *ctx, int npar) {
  if (npar <= ctx->cap_npar) return SNAPI_OK;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  cudaFree(ctx->d_tan); cudaFree(ctx->d_grad); cudaFree(ctx->d_chi2v); cudaFree(ctx->d_step);
  cudaFree(ctx->d_dstokes);
  ctx->d_tan = nullptr; ctx->d_grad = nullptr; ctx->d_chi2v = nullptr; ctx->d_step = nullptr; ctx->d_dstokes = nullptr;
  CK(cudaMalloc(&ctx->d_tan, sizeof(float) * ctx->max_batch * (size_t)npar * nrec));
  CK(cudaMalloc(&ctx->d_grad, sizeof(double) * ctx->max_batch * (size_t)npar));
  CK(cudaMalloc(&ctx->d_chi2v, sizeof(double) * ctx->max_batch * (size_t)(2 * npar + 1)));
  CK(cudaMalloc(&ctx->d_step, sizeof(double) * npar));
  CK(cudaMalloc(&ctx->d_dstokes, sizeof(float) * ctx->max_batch * (size_t)npar * ctx->nl * 4));
  ctx->cap_npar = npar;
  return SNAPI_OK;
}

KParams base_params(const snapi_ctx *ctx) {
  KParams P;
  memset(&P, 0, sizeof P);
  P.nd = ctx->nd; P.nl = ctx->nl; P.nlines = ctx->nlines; P.nfield = ctx->nfield; P.lpad = ctx->lpad;
  P.ncomp = ctx->ncomp; P.nred = ctx->nred; P.lam_mid = ctx->lam_mid; P.scale2 = ctx->scale2;
  P.lamvac = ctx->d_lamvac; P.lines = ctx->d_lines; P.compS = ctx->d_compS; P.compD = ctx->d_compD;
  P.D = ctx->d_D; P.status = ctx->d_status;
  return P;
}

int check_status(snapi_ctx *ctx) {
  int st = 0;
  CK(cudaMemcpyAsync(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (st != 0) {
    int zero = 0;
    cudaMemcpy(ctx->d_status, &zero, sizeof(int), cudaMemcpyHostToDevice);
    return set_err(ctx, st, "device status %d (a CTA gave up waiting for its TMA copy)", st);
  }
  return SNAPI_OK;
}

// copy helper: host<->device or device pointer passthrough
template <class T>
int stage_in(snapi_ctx *ctx, const T *src, T *dbuf, size_t n, int mem, const T **out) {
  if (!src) { *out = nullptr; return SNAPI_OK; }
  if (mem == SNAPI_MEM_DEVICE) { *out = src; return SNAPI_OK; }
  CK(cudaMemcpyAsync(dbuf, src, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream));
  *out = dbuf;
  return SNAPI_OK;
}

}  // namespace

extern "C" {

int snapi_zeeman_pattern(int ju2, int jl2, double gu, double gl, snapi_line *L) {
  if (!L) return SNAPI_EINVAL;
  for (int g = 0; g < 3; ++g) {
    L->ncomp[g] = 0;
    for (int i = 0; i < SNAPI_MAX_COMP; ++i) { L->S[g][i] = 0.0; L->D[g][i] = 0.0; }
  }
  L->split = ((ju2 - jl2 == 2) || (ju2 - jl2 == -2) || ((ju2 == jl2) && (ju2 != 0))) ? 1 : 0;
  if (!L->split) return SNAPI_OK;
  const int jmin2 = ju2 < jl2 ? ju2 : jl2;
  if (jmin2 + 1 > SNAPI_MAX_COMP || (ju2 + jl2) / 2 > SNAPI_MAX_COMP) return SNAPI_EINVAL;
  L->ncomp[0] = jmin2 + 1;
  L->ncomp[1] = L->ncomp[2] = (ju2 + jl2) / 2;
  const double ju = ju2 / 2.0, jmin = jmin2 / 2.0;
  double np = 0, nb = 0, nr = 0;
  if (ju2 == jl2) {  // delta J = 0
    for (int i = 0; i < L->ncomp[0]; ++i) {
      const double m = (double)i - ju;
      L->S[0][i] = m * m;
      L->D[0][i] = m * (gl - gu);
      np += L->S[0][i];
    }
    for (int i = 0; i < L->ncomp[0]; ++i) L->S[0][i] /= np;
    for (int i = 0; i < L->ncomp[1]; ++i) {
      double m = (double)i - ju + 1.0;
      L->S[1][i] = 0.5 * (ju + m) * (ju - m + 1.0);
      nb += L->S[1][i];
      L->D[1][i] = m * (gl - gu) - gl;
      m = (double)i - ju;
      L->S[2][i] = 0.5 * (ju - m) * (ju + m + 1);
      nr += L->S[2][i];
      L->D[2][i] = m * (gl - gu) + gl;
    }
    for (int i = 0; i < L->ncomp[1]; ++i) { L->S[1][i] /= nb; L->S[2][i] /= nr; }
  } else {  // delta J = +-1
    const double jl = jl2 / 2.0;
    const int offset = (jl2 > ju2) ? 1 : 0;
    for (int i = 0; i < L->ncomp[0]; ++i) {
      const double m = (double)i - jmin;
      if (jl < ju) {
        L->S[1][i] = 0.5 * (jmin + m + 1) * (jmin + m + 2);
        L->S[0][i] = (jmin + 1) * (jmin + 1) - m * m;
        L->S[2][i] = 0.5 * (jmin - m + 1) * (jmin - m + 2);
      } else {
        L->S[1][i] = 0.5 * (jmin - m + 1) * (jmin - m + 2);
        L->S[0][i] = (jmin + 1) * (jmin + 1) - m * m;
        L->S[2][i] = 0.5 * (jmin + m + 1) * (jmin + m + 2);
      }
      np += L->S[0][i]; nr += L->S[2][i]; nb += L->S[1][i];
      L->D[0][i] = m * (gl - gu);
      L->D[1][i] = (m - offset) * (gl - gu) - gu;
      L->D[2][i] = (m + offset) * (gl - gu) + gu;
    }
    for (int i = 0; i < L->ncomp[0]; ++i) { L->S[0][i] /= np; L->S[1][i] /= nb; L->S[2][i] /= nr; }
  }
  return SNAPI_OK;
}

void *snapi_host_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) return nullptr;
  return p;
}
void snapi_host_free(void *p) {
  if (p) cudaFreeHost(p);
}

const char *snapi_last_error(const snapi_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }
void *snapi_stream(snapi_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
double snapi_last_kernel_ms(const snapi_ctx *ctx) { return ctx ? ctx->last_ms : 0.0; }
int snapi_last_launches(const snapi_ctx *ctx) { return ctx ? ctx->last_launches : 0; }

void snapi_destroy(snapi_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  void *bufs[] = {ctx->d_lamvac, ctx->d_D, ctx->d_lines, ctx->d_compS, ctx->d_compD, ctx->d_status,
                  ctx->d_rec, ctx->d_stokes, ctx->d_obs, ctx->d_mask, ctx->d_tan, ctx->d_recgrad,
                  ctx->d_dstokes, ctx->d_grad, ctx->d_chi2, ctx->d_chi2v, ctx->d_step, ctx->d_scratch};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

snapi_ctx *snapi_create(const snapi_problem *prob, int device, int *status) {
  auto fail = [&](snapi_ctx *c, int code) -> snapi_ctx * {
    if (status) *status = code;
    if (c) {
      fprintf(stderr, "snapi_create: %s\n", c->err.c_str());
      snapi_destroy(c);
    }
    return nullptr;
  };
  if (!prob) return fail(nullptr, SNAPI_EINVAL);
  snapi_ctx *ctx = new snapi_ctx();
  ctx->device = device;
  if (prob->nd < 3 || prob->nlambda < 1 || prob->nlambda > SNAPI_MAX_LAMBDA || prob->nlines < 0 ||
      prob->nlines > SNAPI_MAX_LINES || !prob->lambda_air || !prob->tau500 || (prob->nlines && !prob->lines) ||
      !(prob->mu > 0.0 && prob->mu <= 1.0) || !(prob->stokes_scale > 0.0)) {
    set_err(ctx, SNAPI_EINVAL, "invalid problem (nd>=3, 1<=nlambda<=%d, 0<=nlines<=%d, 0<mu<=1, stokes_scale>0)",
            SNAPI_MAX_LAMBDA, SNAPI_MAX_LINES);
    return fail(ctx, SNAPI_EINVAL);
  }
  for (int i = 0; i + 1 < prob->nd; ++i)
    if (!(prob->tau500[i + 1] > prob->tau500[i])) {
      set_err(ctx, SNAPI_EINVAL, "tau500 must increase from the top down");
      return fail(ctx, SNAPI_EINVAL);
    }
  if (cudaSetDevice(device) != cudaSuccess) {
    set_err(ctx, SNAPI_ECUDA, "cudaSetDevice(%d) failed", device);
    return fail(ctx, SNAPI_ECUDA);
  }
  ctx->nd = prob->nd;
  ctx->nl = prob->nlambda;
  ctx->nlines = prob->nlines;
  ctx->nfield = SNAPI_NFIELD0 + 3 * prob->nlines;
  ctx->nred = kNumRed + kRedPerLine * prob->nlines;
  ctx->lpad = (prob->nlambda + 31) / 32 * 32;
  ctx->max_batch = prob->max_batch > 0 ? prob->max_batch : 4096;
  ctx->scale2 = prob->stokes_scale * prob->stokes_scale;
  // wavelengths
  std::vector<double> lv(ctx->nl);
  for (int l = 0; l < ctx->nl; ++l) lv[l] = airtovac_d(prob->lambda_air[l]);
  ctx->lam_mid = (float)(0.5 * (lv[ctx->nl - 1] + lv[0]));
  // path-length intervals
  std::vector<double> D(ctx->nd - 1);
  for (int i = 0; i + 1 < ctx->nd; ++i) D[i] = (prob->tau500[i + 1] - prob->tau500[i]) / prob->mu;
  // lines and components
  std::vector<LineConst> lc(ctx->nlines);
  std::vector<float> cS, cD;
  for (int j = 0; j < ctx->nlines; ++j) {
    const snapi_line &s = prob->lines[j];
    LineConst &L = lc[j];
    L.lam0 = s.lam0;
    L.sf = (float)s.sf;
    L.ar = (float)s.ar;
    L.two_k_over_m = (float)(2.0 * kK / s.mass);
    L.lam0_over_c = (float)(s.lam0 / kC);
    L.zee = (float)(4.67E-5 * s.lam0 * s.lam0);
    L.split = s.split ? 1 : 0;
    L.comp_off = (int)cS.size();
    for (int g = 0; g < 3; ++g) {
      L.ncomp[g] = s.split ? s.ncomp[g] : 0;
      if (L.ncomp[g] < 0 || L.ncomp[g] > SNAPI_MAX_COMP) {
        set_err(ctx, SNAPI_EINVAL, "line %d: bad component count", j);
        return fail(ctx, SNAPI_EINVAL);
      }
      for (int i = 0; i < L.ncomp[g]; ++i) { cS.push_back((float)s.S[g][i]); cD.push_back((float)s.D[g][i]); }
    }
  }
  ctx->ncomp = (int)cS.size();
  const SmemLayout Ls = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, true);
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if ((int)Ls.total > maxsm) {
    set_err(ctx, SNAPI_EINVAL, "problem needs %zu B of shared memory per CTA (> %d)", Ls.total, maxsm);
    return fail(ctx, SNAPI_EINVAL);
  }
#define CKC(call)                                                                        \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      set_err(ctx, e_ == cudaErrorMemoryAllocation ? SNAPI_ENOMEM : SNAPI_ECUDA, "%s: %s", #call, \
              cudaGetErrorString(e_));                                                   \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? SNAPI_ENOMEM : SNAPI_ECUDA);   \
    }                                                                                    \
  } while (0)
  CKC(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  CKC(cudaEventCreate(&ctx->ev0));
  CKC(cudaEventCreate(&ctx->ev1));
  CKC(cudaMalloc(&ctx->d_lamvac, sizeof(double) * ctx->nl));
  CKC(cudaMalloc(&ctx->d_D, sizeof(double) * (ctx->nd - 1)));
  CKC(cudaMalloc(&ctx->d_lines, sizeof(LineConst) * std::max(1, ctx->nlines)));
  CKC(cudaMalloc(&ctx->d_compS, sizeof(float) * std::max(1, ctx->ncomp)));
  CKC(cudaMalloc(&ctx->d_compD, sizeof(float) * std::max(1, ctx->ncomp)));
  CKC(cudaMalloc(&ctx->d_status, sizeof(int)));
  CKC(cudaMemset(ctx->d_status, 0, sizeof(int)));
  CKC(cudaMemcpy(ctx->d_lamvac, lv.data(), sizeof(double) * ctx->nl, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(ctx->d_D, D.data(), sizeof(double) * (ctx->nd - 1), cudaMemcpyHostToDevice));
  if (ctx->nlines) CKC(cudaMemcpy(ctx->d_lines, lc.data(), sizeof(LineConst) * ctx->nlines, cudaMemcpyHostToDevice));
  if (ctx->ncomp) {
    CKC(cudaMemcpy(ctx->d_compS, cS.data(), sizeof(float) * ctx->ncomp, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(ctx->d_compD, cD.data(), sizeof(float) * ctx->ncomp, cudaMemcpyHostToDevice));
  }
  const size_t B = ctx->max_batch, nrec = (size_t)ctx->nd * ctx->nfield;
  CKC(cudaMalloc(&ctx->d_rec, sizeof(float) * B * nrec));
  CKC(cudaMalloc(&ctx->d_stokes, sizeof(float) * B * ctx->nl * 4));
  CKC(cudaMalloc(&ctx->d_obs, sizeof(float) * B * ctx->nl * 4));
  CKC(cudaMalloc(&ctx->d_mask, sizeof(float) * B * ctx->nl));
  CKC(cudaMalloc(&ctx->d_recgrad, sizeof(double) * B * nrec));
  CKC(cudaMalloc(&ctx->d_chi2, sizeof(double) * B));
  CKC(cudaMalloc(&ctx->d_scratch, sizeof(float4) * B * ctx->nd * 4 * ctx->lpad));
  const SmemLayout Lsyn = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  CKC(cudaFuncSetAttribute(k_synth<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lsyn.total));
  CKC(cudaFuncSetAttribute(k_fd<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lsyn.total));
  CKC(cudaFuncSetAttribute(k_adjoint<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Ls.total));
  CKC(cudaFuncSetAttribute(k_synth<kMaxThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lsyn.total));
  CKC(cudaFuncSetAttribute(k_fd<kMaxThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lsyn.total));
  CKC(cudaFuncSetAttribute(k_adjoint<kMaxThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Ls.total));
#undef CKC
  if (status) *status = SNAPI_OK;
  return ctx;
}

int snapi_synth(snapi_ctx *ctx, int npix, const float *records, float *stokes, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || (npix > 0 && (!records || !stokes)) || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_synth: invalid arguments");
  CK(cudaSetDevice(ctx->device));
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < npix; p0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, npix - p0);
    KParams P = base_params(ctx);
    P.npix = nb;
    const float *rec;
    int st = stage_in(ctx, records + p0 * nrec, ctx->d_rec, nb * nrec, mem, &rec);
    if (st) return st;
    P.rec = rec;
    P.stokes = mem == SNAPI_MEM_DEVICE ? stokes + (size_t)p0 * ctx->nl * 4 : ctx->d_stokes;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (ctx->lpad <= 256) k_synth<256><<<nb, ctx->lpad, L.total, ctx->stream>>>(P);
    else k_synth<kMaxThreads><<<nb, ctx->lpad, L.total, ctx->stream>>>(P);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_launches += 1;
    if (mem == SNAPI_MEM_HOST)
      CK(cudaMemcpyAsync(stokes + (size_t)p0 * ctx->nl * 4, ctx->d_stokes, sizeof(float) * nb * ctx->nl * 4,
                         cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return check_status(ctx);
}

int snapi_adjoint(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                  const float *mask, int npar, const float *tangents, float *stokes, double *chi2, double *grad,
                  double *rec_grad, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || npar < 0 || (npix > 0 && (!records || !obs || !chi2)) || (npar > 0 && (!tangents || !grad)) ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_adjoint: invalid arguments");
  CK(cudaSetDevice(ctx->device));
  int st = ensure_npar(ctx, npar > 0 ? npar : 1);
  if (st) return st;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, true);
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < npix; p0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, npix - p0);
    KParams P = base_params(ctx);
    P.npix = nb;
    P.npar = npar;
    for (int s = 0; s < 4; ++s) P.ws[s] = w_stokes ? w_stokes[s] : 1.0;
    const float *rec, *ob, *mk, *tn;
    if ((st = stage_in(ctx, records + p0 * nrec, ctx->d_rec, nb * nrec, mem, &rec))) return st;
    if ((st = stage_in(ctx, obs + (size_t)p0 * ctx->nl * 4, ctx->d_obs, (size_t)nb * ctx->nl * 4, mem, &ob))) return st;
    if ((st = stage_in(ctx, mask ? mask + (size_t)p0 * ctx->nl : nullptr, ctx->d_mask, (size_t)nb * ctx->nl, mem, &mk)))
      return st;
    if ((st = stage_in(ctx, npar ? tangents + (size_t)p0 * npar * nrec : nullptr, ctx->d_tan, (size_t)nb * npar * nrec,
                       mem, &tn)))
      return st;
    P.rec = rec; P.obs = ob; P.mask = mk; P.tangent = tn;
    const bool dev = mem == SNAPI_MEM_DEVICE;
    P.stokes = stokes ? (dev ? stokes + (size_t)p0 * ctx->nl * 4 : ctx->d_stokes) : nullptr;
    P.chi2 = dev ? chi2 + p0 : ctx->d_chi2;
    P.grad = npar ? (dev ? grad + (size_t)p0 * npar : ctx->d_grad) : ctx->d_grad;
    P.rec_grad = rec_grad ? (dev ? rec_grad + (size_t)p0 * nrec : ctx->d_recgrad) : nullptr;
    P.scratch = ctx->d_scratch;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (ctx->lpad <= 256) k_adjoint<256><<<nb, ctx->lpad, L.total, ctx->stream>>>(P);
    else k_adjoint<kMaxThreads><<<nb, ctx->lpad, L.total, ctx->stream>>>(P);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_launches += 1;
    if (!dev) {
      if (stokes)
        CK(cudaMemcpyAsync(stokes + (size_t)p0 * ctx->nl * 4, ctx->d_stokes, sizeof(float) * nb * ctx->nl * 4,
                           cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(chi2 + p0, ctx->d_chi2, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream));
      if (npar)
        CK(cudaMemcpyAsync(grad + (size_t)p0 * npar, ctx->d_grad, sizeof(double) * nb * npar, cudaMemcpyDeviceToHost,
                           ctx->stream));
      if (rec_grad)
        CK(cudaMemcpyAsync(rec_grad + (size_t)p0 * nrec, ctx->d_recgrad, sizeof(double) * nb * nrec,
                           cudaMemcpyDeviceToHost, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return check_status(ctx);
}

int snapi_fd_grad(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                  const float *mask, int npar, const float *tangents, const double *step, double *chi2, double *grad,
                  int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (npix < 0 || npar < 1 || (npix > 0 && (!records || !obs || !chi2 || !grad || !tangents)) || !step ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_fd_grad: invalid arguments");
  CK(cudaSetDevice(ctx->device));
  int st = ensure_npar(ctx, npar);
  if (st) return st;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  const SmemLayout L = smem_layout(ctx->nd, ctx->nfield, ctx->nlines, ctx->ncomp, ctx->nred, false);
  CK(cudaMemcpyAsync(ctx->d_step, step, sizeof(double) * npar, cudaMemcpyHostToDevice, ctx->stream));
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < npix; p0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, npix - p0);
    KParams P = base_params(ctx);
    P.npix = nb;
    P.npar = npar;
    for (int s = 0; s < 4; ++s) P.ws[s] = w_stokes ? w_stokes[s] : 1.0;
    const float *rec, *ob, *mk, *tn;
    if ((st = stage_in(ctx, records + p0 * nrec, ctx->d_rec, nb * nrec, mem, &rec))) return st;
    if ((st = stage_in(ctx, obs + (size_t)p0 * ctx->nl * 4, ctx->d_obs, (size_t)nb * ctx->nl * 4, mem, &ob))) return st;
    if ((st = stage_in(ctx, mask ? mask + (size_t)p0 * ctx->nl : nullptr, ctx->d_mask, (size_t)nb * ctx->nl, mem, &mk)))
      return st;
    if ((st = stage_in(ctx, tangents + (size_t)p0 * npar * nrec, ctx->d_tan, (size_t)nb * npar * nrec, mem, &tn)))
      return st;
    P.rec = rec; P.obs = ob; P.mask = mk; P.tangent = tn; P.fd_step = ctx->d_step;
    P.chi2 = ctx->d_chi2v;
    const bool dev = mem == SNAPI_MEM_DEVICE;
    double *c_out = dev ? chi2 + p0 : ctx->d_chi2;
    double *g_out = dev ? grad + (size_t)p0 * npar : ctx->d_grad;
    CK(cudaEventRecord(ctx->ev0, ctx->stream));
    dim3 grid(nb, 2 * npar + 1);
    if (ctx->lpad <= 256) k_fd<256><<<grid, ctx->lpad, L.total, ctx->stream>>>(P);
    else k_fd<kMaxThreads><<<grid, ctx->lpad, L.total, ctx->stream>>>(P);
    CK(cudaGetLastError());
    k_fd_combine<<<(nb + 127) / 128, 128, 0, ctx->stream>>>(nb, npar, ctx->d_chi2v, ctx->d_step, c_out, g_out);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_launches += 2;
    if (!dev) {
      CK(cudaMemcpyAsync(chi2 + p0, ctx->d_chi2, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream));
      CK(cudaMemcpyAsync(grad + (size_t)p0 * npar, ctx->d_grad, sizeof(double) * nb * npar, cudaMemcpyDeviceToHost,
                         ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return check_status(ctx);
}

int snapi_responses(snapi_ctx *ctx, int npix, const float *records, int npar, const float *tangents, float *stokes,
                    float *dstokes, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  return set_err(ctx, SNAPI_EINVAL, "snapi_responses: not available in this build");
}

}  // extern "C"
