// snapi_internal.cuh -- device-side building blocks shared by the libsnapi_cuda kernels and the
// host-side context definition.
//
// Work decomposition: a CTA handles SNAPI_CHUNK consecutive wavelengths of one pixel (so one
// pixel spans ceil(nlambda / SNAPI_CHUNK) CTAs).  Wavelengths near the line cores cost several
// times more than continuum wavelengths (all four W4 regions are taken across a warp there), so
// small CTAs that retire independently let the block scheduler back-fill the SMs instead of
// holding a whole pixel's warps until its slowest warp finishes.  Wavelength sums that the
// adjoint needs per pixel are written per warp to a global partial buffer and summed in a fixed
// order by a per-pixel finish kernel (deterministic, no float atomics).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/snapi_cuda.h"
#include "snapi_sweep.cuh"

namespace snapi {

#ifndef SNAPI_CHUNK
#define SNAPI_CHUNK 64
#endif
constexpr int kChunk = SNAPI_CHUNK;           // wavelengths (threads) per sweep CTA
constexpr int kFinishThreads = 128;           // threads of the per-pixel finish kernels
constexpr long long kWaitLimit = 1LL << 26;   // mbarrier polls before a CTA gives up
// Opacity-adjoint sums per (pixel, group, depth): group 0 (continuum) fills R_COP..R_LT, group
// 1 + j (transition j) fills RL_OPN..RL_A then its share of R_ST2..R_S2.
constexpr int kOpSlots = kRedPerLine + 4;
constexpr int kOpThreads = 256;  // k_adj_opacity: threads per CTA at most
// Wavelength slices of the opacity adjoint: enough that nd x slices fills whole warps (80 depths
// -> 2 slices, 160 threads), at most kOpThreads threads.
__host__ __device__ inline int op_slices(int nd) {
#ifdef SNAPI_OP_NOSLICE
  return 1;
#endif
  int g = 32, a = nd;
  while (a % g) g >>= 1;  // gcd(nd, 32)
  int s = 32 / g;
  while (s > 1 && nd * s > kOpThreads) s >>= 1;
  return s;
}

// Launch shapes the autotuner (snapi_autotune) chooses between, per context and batch size; the
// defaults are the compiled constants.  All of them give bit-identical results: they change which
// thread or CTA handles a wavelength or pixel, never the order of a sum.
constexpr int kChunkCands[3] = {32, 64, 128};   // wavelengths per sweep CTA of the adjoint
constexpr int kOpTileCands[3] = {8, 16, 32};    // pixels per opacity-adjoint CTA tile
constexpr int kHeCands[3] = {32, 64, 128};      // threads per hydrostatic-march CTA
constexpr int kVarCands[3] = {64, 128, 256};    // threads per record-chemistry CTA
constexpr int kHeDefault = 64, kVarDefault = 64;  // the chemistry kernels' compiled CTA sizes
constexpr int kJvpDirs = 10;  // node directions (warps) per forward-mode responses CTA (two CTAs per SM)
struct AdjCfg {
  int chunk, optile;
  int rt128;  // the reverse DELO sweep at 128 registers per thread
};
struct BuildCfg {
  int he, var;
};

struct KParams {
  int npix, nd, nl, nlines, nfield, npar, lpad, ncomp, nred, nchunk, nwslot, nvar;
  int nslice;                   // wavelength slices of the opacity adjoint (threads = nd x nslice)
  int optile;                   // pixels per opacity-adjoint CTA tile
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
  const float *tangent;         // [npix][npar][nd][nfield], or packed [npix][ntcol][nd]; or null
  const int *tcol_off;          // packed tangents: node p's columns are [tcol_off[p], tcol_off[p+1])
  const int *tcol_field;        // packed tangents: record field of each column
  int ntcol;                    // packed tangents: columns per pixel (0: dense)
  float4 *scratch;              // [npix][nd][4][lpad]     forward state of the adjoint
  float4 *seed;                 // [npix][lpad]            adjoint of the emergent Stokes vector
  float4 *bars;                 // [npix][nl][3][nd]       (eta-bar, j-bar) per wavelength, depth
  float *opart;                 // [npix][1+nlines][nslice][nd][kOpSlots] wavelength sums of the opacity adjoint
  double *c2part;               // [npix][nvar][nwslot]      per-warp chi2 sums
  double *rec_grad;             // [npix][nd][nfield] or null
  double *grad;                 // [npix][npar]
  double *chi2;                 // [npix]
  float *dstokes;               // [npix][npar][nl][4] (responses)
  const double *fd_step;        // [npar]
  const int *skip;              // [npix] or null: pixels whose CTAs return at once (LM)
  int *status;                  // device error word
};

struct SmemLayout {
  size_t rec, D, lines, compS, compD, dc, ld, acc, rb, mbar, wred, total;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// acc / rb only for the per-pixel finish kernels
__host__ __device__ inline SmemLayout smem_layout(int nd, int nfield, int nlines, int ncomp, int nred, bool finish) {
  SmemLayout s;
  size_t o = 0;
  s.rec = o; o = align_up(o + sizeof(float) * nd * nfield, 16);
  s.D = o; o = align_up(o + sizeof(double) * (nd - 1), 16);
  s.lines = o; o = align_up(o + sizeof(LineConst) * (nlines > 0 ? nlines : 1), 16);
  s.compS = o; o = align_up(o + sizeof(float) * (ncomp > 0 ? ncomp : 1), 16);
  s.compD = o; o = align_up(o + sizeof(float) * (ncomp > 0 ? ncomp : 1), 16);
  s.dc = o; o = align_up(o + sizeof(DepthConst) * nd, 16);
  s.ld = o; o = align_up(o + sizeof(LineDepth) * nd * (nlines > 0 ? nlines : 1), 16);
  s.acc = o; if (finish) o = align_up(o + sizeof(float) * nd * nred, 16);
  s.rb = o; if (finish) o = align_up(o + sizeof(float) * nd * nfield, 16);
  s.mbar = o; o = align_up(o + 8, 16);
  s.wred = o; o = align_up(o + sizeof(double) * 32, 16);
  s.total = o;
  return s;
}

// ------------------------------------------------------------------------------------------
// TMA bulk copy global -> shared, completion tracked by an mbarrier; every wait is bounded and
// the decision to give up is taken uniformly by the whole CTA.
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ inline bool tma_bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *mbar) {
  const uint32_t mb = smem_u32(mbar);
  // the destination may hold this CTA's earlier generic-proxy writes (a record staged again)
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
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
  return __syncthreads_and(done != 0) != 0;
}

// ------------------------------------------------------------------------------------------
// forward state per (pixel, wavelength, depth): 4 float4 planes, coalesced across wavelengths
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
  __device__ void load_I(int z, float *I) const {
    const float4 a = base[(size_t)z * 4 * lpad + l];
    I[0] = a.x; I[1] = a.y; I[2] = a.z; I[3] = a.w;
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

// Reverse DELO sweep (phase R1): reads the forward state of wavelength l, writes the adjoint bars
// of each finished depth depth-contiguous ([l][plane][z]) for the per-depth opacity adjoint.
struct RtScratch {
  const float4 *state;
  float4 *bars;
  int lpad, l, nd;
  bool write;  // false for the padding lanes of the last wavelength chunk
  // the sweep asks for depth z+2 while it works on depth z, so the (DRAM-latency) loads of a
  // depth overlap the 4x4 algebra of the one before
  float4 pf[4];
  int pz = -1;
  __device__ void prefetch(int z) {
    if (z >= nd) return;
    const float4 *p = state + (size_t)z * 4 * lpad + l;
    pf[0] = p[0]; pf[1] = p[lpad]; pf[2] = p[2 * lpad]; pf[3] = p[3 * lpad];
    pz = z;
  }
  __device__ void load(int z, float *I, float *kp, float *S, float &e, float &tau) {
    float4 a, b, c, d;
    if (z == pz) {
      a = pf[0]; b = pf[1]; c = pf[2]; d = pf[3];
    } else {
      const float4 *p = state + (size_t)z * 4 * lpad + l;
      a = p[0]; b = p[lpad]; c = p[2 * lpad]; d = p[3 * lpad];
    }
    I[0] = a.x; I[1] = a.y; I[2] = a.z; I[3] = a.w;
    kp[0] = b.x; kp[1] = b.y; kp[2] = b.z; kp[3] = b.w;
    kp[4] = c.x; kp[5] = c.y; e = c.z; tau = c.w;
    S[0] = d.x; S[1] = d.y; S[2] = d.z; S[3] = d.w;
  }
  __device__ void store_bar(int z, const float *eb, const float *jb) {
    if (!write) return;
    float4 *p = bars + (size_t)l * 3 * nd + z;
    p[0] = make_float4(eb[0], eb[1], eb[2], eb[3]);
    p[nd] = make_float4(eb[4], eb[5], eb[6], jb[0]);
    p[2 * nd] = make_float4(jb[1], jb[2], jb[3], 0.f);
  }
};
struct NoScratch {
  __device__ void store(int, const float *, const float *, const float *, float, float) {}
};

__device__ __forceinline__ float warp_sum(float v) {
  v += __shfl_xor_sync(0xffffffffu, v, 16);
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sum over the CTA (valid in thread 0)
__device__ inline double block_sum(double v, double *wred) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) wred[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < nw; ++i) s += wred[i];
  __syncthreads();
  return s;
}

// Stage one pixel into shared memory and build its per-depth constants.  fd_pert: -1 none,
// otherwise the record is perturbed by sign * fd_step[p] * tangent_p (p = fd_pert).
__device__ inline bool stage_pixel(const KParams &P, int pix, unsigned char *smem, const SmemLayout &L,
                                   PixelView &pv, int fd_pert, float fd_sign) {
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

__device__ inline void thread_lambda(const KParams &P, const PixelView &pv, int l, LamConst &lam, float *delta) {
  const double lv = P.lamvac[l];
  lambda_precompute(lv, lam);
  for (int j = 0; j < P.nlines; ++j) delta[j] = (float)(pv.lc[j].lam0 - lv);
}

// residual, chi2 contribution (scaled) and adjoint seed of one wavelength (atmos_fit.cc:229-248)
__device__ inline double residual_seed(const KParams &P, int pix, int l, const float *out, float *seed) {
  const float m = P.mask ? P.mask[(size_t)pix * P.nl + l] : 1.0f;
  const float *ob = P.obs + ((size_t)pix * P.nl + l) * 4;
  const double is2 = 1.0 / P.scale2;
  double c2 = 0.0;
  for (int s = 0; s < 4; ++s) {
    const double r = ((double)ob[s] - (double)out[s]) * P.ws[s] * m;
    c2 += r * r * is2;
    seed[s] = (float)(-2.0 * r * P.ws[s] * m * is2);
  }
  return c2;
}

}  // namespace snapi

// =============================================================================================
// host-side context (shared by the .cu files of the library)
struct snapi_ctx {
  int device = 0;
  cudaStream_t stream = nullptr, copy_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  static constexpr int kStageChunks = 8;  // host-input chunks per round (adjoint_impl)
  cudaEvent_t ev_copy[kStageChunks] = {}, ev_free = nullptr;  // chunk uploaded / round's kernels done
  int nd = 0, nl = 0, nlines = 0, nfield = 0, ncomp = 0, nred = 0, lpad = 0, nchunk = 0, nwslot = 0, max_batch = 0;
  int lpad_max = 0;  // padded wavelengths of the widest sweep CTA the autotuner may pick (buffer sizes)
  int nbasis = 0;    // direction-independent W4 sums per (wavelength, depth) (jvp_basis_size)
  int jac_tangent = 0;  // node responses / LM Jacobian by forward-mode sweeps (snapi_jacobian_mode)
  // autotuner (snapi_autotune): off = the compiled launch shapes; per batch-size bucket the shapes
  // it measured fastest; an optional cache file shared across processes
  int tune = 0;
  std::string tune_cache;
  std::vector<std::pair<int, snapi::AdjCfg>> adj_tuned;
  std::vector<std::pair<int, snapi::BuildCfg>> build_tuned;
  float lam_mid = 0.f;
  double scale2 = 1.0;
  double *d_lamvac = nullptr, *d_D = nullptr;
  snapi::LineConst *d_lines = nullptr;
  float *d_compS = nullptr, *d_compD = nullptr;
  int *d_status = nullptr;
  int *d_tcol = nullptr;  // packed-tangent column tables: offsets [npar+1] then fields [ntcol]
  // Gaussian instrumental broadening (snapi_psf.cu): the observation's (air) grid and one width
  std::vector<double> h_lamair;
  double *d_lamair = nullptr;
  float *d_psf_kt = nullptr;
  double psf_width = 0.0, psf_lmin = 0.0, psf_step = 0.0;
  int psf_nf = 0, psf_band = 0;
  int cap_tcol = 0;
  // work buffers (max_batch pixels)
  float *d_rec = nullptr, *d_stokes = nullptr, *d_obs = nullptr, *d_mask = nullptr, *d_tan = nullptr;
  float *d_dstokes = nullptr, *d_opart = nullptr;
  float4 *d_seed = nullptr, *d_bars = nullptr;
  double *d_recgrad = nullptr, *d_grad = nullptr, *d_chi2 = nullptr, *d_c2part = nullptr, *d_step = nullptr;
  float4 *d_scratch = nullptr;
  int cap_npar = 0;
  double last_ms = 0.0;
  double phase_ms[2] = {0.0, 0.0};  // snapi_adjoint_nodes: node build, adjoint (device time)
  int last_launches = 0;
  std::string err;
  // LM work buffers (allocated on first use)
  void *lm = nullptr;
  // node model -> records (snapi_eos.cu): tables and work buffers, host copies it checks against
  void *eos = nullptr;
  std::vector<double> h_tau500, h_line_lam0, h_line_mass;
};

namespace snapi {
int set_err(snapi_ctx *c, int code, const char *fmt, ...);
int ensure_npar(snapi_ctx *ctx, int npar);
KParams base_params(const snapi_ctx *ctx);
int check_status(snapi_ctx *ctx);
// autotuner (snapi_cuda.cu): the batch-size bucket of npix, the tuned shapes of a bucket (false if
// none yet), their record in the context and the cache file
int tune_bucket(int npix);
bool tuned_adj(const snapi_ctx *ctx, int npix, AdjCfg *cfg);
bool tuned_build(const snapi_ctx *ctx, int npix, BuildCfg *cfg);
void tune_store_adj(snapi_ctx *ctx, int npix, const AdjCfg &cfg);
void tune_store_build(snapi_ctx *ctx, int npix, const BuildCfg &cfg);
// sweep launches for other translation units (P.npix pixels; P.nvar nodes for the responses)
cudaError_t launch_synth(const snapi_ctx *ctx, const KParams &P);
// the synthesis that also stores the forward state of every pixel in the context's scratch
// (P.npix <= max_batch), so that launch_responses with state_ready skips its own state pass
cudaError_t launch_synth_state(const snapi_ctx *ctx, const KParams &P);
cudaError_t launch_responses(const snapi_ctx *ctx, const KParams &P, bool state_ready = false);
void lm_free(snapi_ctx *ctx);  // LM work buffers (snapi_lm.cu)
void eos_free(snapi_ctx *ctx); // node-model tables and work buffers (snapi_eos.cu)
// the context has a node model with these npar node kinds (snapi_eos.cu)
bool eos_matches(const snapi_ctx *ctx, int npar, const int *node_kind);
// G[m] = M[m] M[m]^T for nmat matrices [16][K] (row-major) on the tensor cores (snapi_tc.cu)
cudaError_t launch_gram_tf32(const float *M, int nmat, int K, float *G, int *status, cudaStream_t st);
// Gaussian instrumental broadening (snapi_psf.cu): set-up for one width, in-place launch
int psf_prepare(snapi_ctx *ctx, double width);
cudaError_t psf_launch(const snapi_ctx *ctx, float *data, int nvec, int vec_per_pix, const int *skip);
}  // namespace snapi

#define SNAPI_CK(call)                                                                                  \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess) return snapi::set_err(ctx, SNAPI_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)
