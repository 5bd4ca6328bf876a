// snapi_lm.cu -- batched Levenberg-Marquardt node fit (stokes_lm_fit, atmos/atmos_fit.cc:18-227).
//
// One call of snapi_lm_step is one iteration of the reference's loop for every pixel still
// fitting.  The caller builds the records (and node tangents) of the node vectors the previous
// call requested; on the device:
//   k_synth          Stokes at the requested nodes (pixels that are done are skipped)
//   k_lm_eval        one CTA per pixel: chi2, accept / reject, damping, tracked chi2, stop rules
//   k_resp_sweep     Jacobian at the newly accepted nodes (central differences along tangents)
//   k_lm_rows        scaled Jacobian rows and residual of every pixel, 16 rows per pixel
//   k_gram_tf32      J^T J and J^T r of 8 pixels per CTA on the tcgen05 tensor cores, FP32
//                    accuracy by a three-product TF32 split (snapi_tc.cu); npar <= 15
//   k_lm_solve       one CTA per pixel: (J^T J and J^T r in FP64 when npar > 15), damped, symmetric
//                    eigen-decomposition (cyclic Jacobi) with the reference's 1e6 condition cut,
//                    bracketed trial nodes for the next call
#include <cmath>
#include <cstring>
#include <vector>

#include "snapi_internal.cuh"

using namespace snapi;

namespace {

constexpr int kLmThreads = 128;
constexpr int kMaxPar = SNAPI_LM_MAX_PAR;

enum LmPhase : int { PH_FIRST = 0, PH_TRIAL = 1, PH_DONE = 2 };

struct LmPix {
  double lm;          // damping parameter
  double chi2;        // chi2 of the current (accepted) nodes
  double tr_prev, tr_last;  // last two tracked chi2 values (atmos_fit.cc:168-176)
  int ntrack;         // number of tracked values
  int iter;           // iterations done
  int phase;          // LmPhase
  int brk;            // chi2 fell below stopping_chisq: end after the next trial
};

struct LmDev {
  int npix, npar, nl;
  double ws[4], scale2, delta, stopping, lm_floor;
  int max_iter;
  double scale[kMaxPar];  // J / correction scales per node (atmos_fit.cc:250-270)
  double lo[kMaxPar], hi[kMaxPar];  // node bounds (atmos_model.cc:12-19)
  const float *obs, *mask;   // [npix][nl][4], [npix][nl] or null
  const float *snew;         // [npix][nl][4] Stokes at the requested nodes
  float *scur;               // [npix][nl][4] Stokes at the current nodes
  const float *J;            // [npix][npar][nl][4] unscaled dS/dnode at the current nodes
  double *nodes, *req;       // [npix][npar]
  LmPix *pix;
  int *skip_syn, *skip_resp, *active;
  const float *G;            // [npix][16][16] tensor-core J^T J | J^T r, or null (FP64 sums here)
};

struct LmWork {
  int npix = 0, npar = 0, cap = 0, cap_par = 0;
  bool begun = false;
  LmDev D;
  double *d_nodes = nullptr, *d_req = nullptr, *d_step = nullptr;
  LmPix *d_pix = nullptr;
  float *d_obs = nullptr, *d_mask = nullptr, *d_scur = nullptr, *d_snew = nullptr, *d_J = nullptr;
  float *d_rec = nullptr, *d_tan = nullptr, *d_M = nullptr, *d_G = nullptr;
  int *d_skip_syn = nullptr, *d_skip_resp = nullptr, *d_active = nullptr;
  double *d_req_out = nullptr;  // snapi_lm_fit: the step's copies of request / active
  int *d_act_out = nullptr;
  std::vector<int> h_active, kind;
  double broaden = 0.0;  // Gaussian instrumental width [cm], 0: none
  // the last evaluation stored the forward state of its pixels (forward-mode Jacobian): the
  // Jacobian of the accepted pixels, evaluated at the same nodes, starts from it
  bool state_ready = false;
};

__device__ double block_sum_d(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sh[i];
  return s;
}

// chi2 of the requested nodes and the accept / reject decision (atmos_fit.cc:127-178)
__global__ void __launch_bounds__(kLmThreads) k_lm_eval(LmDev D) {
  __shared__ double sh[32];
  __shared__ int s_accept;
  const int p = blockIdx.x;
  LmPix st = D.pix[p];
  if (st.phase == PH_DONE) {
    if (threadIdx.x == 0) { D.skip_resp[p] = 1; D.skip_syn[p] = 1; D.active[p] = 0; }
    return;
  }
  const float *ob = D.obs + (size_t)p * D.nl * 4, *sn = D.snew + (size_t)p * D.nl * 4;
  double c = 0.0;
  for (int i = threadIdx.x; i < D.nl * 4; i += blockDim.x) {
    const double m = D.mask ? (double)D.mask[(size_t)p * D.nl + (i >> 2)] : 1.0;
    const double r = ((double)ob[i] - (double)sn[i]) * D.ws[i & 3] * m;
    c += r * r;
  }
  c = block_sum_d(c, sh) / D.scale2;
  if (threadIdx.x == 0) {
    int accept = 0;
    if (st.phase == PH_FIRST) {
      accept = 1;  // the starting model: Stokes and Jacobian at it
      st.chi2 = c;
      if (st.chi2 < D.stopping) st.brk = 1;
    } else {
      bool stop = st.brk != 0;
      if (c < st.chi2) {  // better: accept, damping / sqrt(10) (atmos_fit.cc:162-177)
        accept = 1;
        for (int i = 0; i < D.npar; ++i) D.nodes[(size_t)p * D.npar + i] = D.req[(size_t)p * D.npar + i];
        st.lm = fmax(st.lm / sqrt(10.0), D.lm_floor);
        st.tr_prev = st.tr_last;
        st.tr_last = st.chi2;  // the metric of the model the step started from
        st.ntrack += 1;
        if (st.ntrack >= 3 && fabs((st.tr_prev - st.tr_last) / st.tr_last) < D.delta) stop = true;
        st.chi2 = c;
      } else {  // worse: damping * sqrt(10)
        st.lm *= sqrt(10.0);
      }
      st.iter += 1;
      if (st.iter >= D.max_iter) stop = true;
      if (stop) {
        st.phase = PH_DONE;
      } else if (st.chi2 < D.stopping) {
        st.brk = 1;  // checked at the start of the next iteration; one more trial follows
      }
    }
    s_accept = accept;
    D.pix[p] = st;
    const bool done = st.phase == PH_DONE;
    D.skip_resp[p] = (accept && !done) ? 0 : 1;
    D.skip_syn[p] = done ? 1 : 0;
    D.active[p] = done ? 0 : 1;
  }
  __syncthreads();
  if (s_accept) {
    float *sc = D.scur + (size_t)p * D.nl * 4;
    for (int i = threadIdx.x; i < D.nl * 4; i += blockDim.x) sc[i] = sn[i];
  }
}

// Cyclic Jacobi eigen-decomposition of the symmetric n x n matrix A (row-major, destroyed):
// eigenvalues on A's diagonal, eigenvectors in the columns of V.
__device__ void jacobi_eigen(double *A, double *V, int n) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) V[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double off = 0.0, dia = 0.0;
    for (int i = 0; i < n; ++i) {
      dia += A[i * n + i] * A[i * n + i];
      for (int j = i + 1; j < n; ++j) off += A[i * n + j] * A[i * n + j];
    }
    if (off <= 1e-30 * dia || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p * n + q];
        if (apq == 0.0) continue;
        const double app = A[p * n + p], aqq = A[q * n + q];
        const double th = (aqq - app) / (2.0 * apq);
        const double t = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {  // A <- A R (columns p, q)
          const double akp = A[k * n + p], akq = A[k * n + q];
          A[k * n + p] = c * akp - s * akq;
          A[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {  // A <- R^T A (rows p, q)
          const double apk = A[p * n + k], aqk = A[q * n + k];
          A[p * n + k] = c * apk - s * aqk;
          A[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[k * n + p], vkq = V[k * n + q];
          V[k * n + p] = c * vkp - s * vkq;
          V[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
}

// Rows of the tensor-core Gram product: row i < npar = J_i * scale_i * w_s * mask / I_c, row npar =
// (obs - S) * w_s * mask / I_c, the rest zero (atmos_fit.cc:229-260); one CTA per (pixel, row).
__global__ void k_lm_rows(LmDev D, float *Mrows) {
  const int p = blockIdx.x / 16, i = blockIdx.x % 16, K = D.nl * 4;
  if (D.pix[p].phase == PH_DONE) return;  // CTA-uniform; the solve skips the pixel too
  float *out = Mrows + ((size_t)p * 16 + i) * K;
  const double ic = sqrt(D.scale2);
  const float *mk = D.mask ? D.mask + (size_t)p * D.nl : nullptr;
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    const double w = D.ws[k & 3] * (mk ? (double)mk[k >> 2] : 1.0) / ic;
    double v = 0.0;
    if (i < D.npar) v = (double)D.J[((size_t)p * D.npar + i) * K + k] * w * D.scale[i];
    else if (i == D.npar) v = ((double)D.obs[(size_t)p * K + k] - (double)D.scur[(size_t)p * K + k]) * w;
    out[k] = (float)v;
  }
}

// damped normal equations and the trial nodes (atmos_fit.cc:127-160, mathtools.cc:344-390)
__global__ void __launch_bounds__(kLmThreads) k_lm_solve(LmDev D) {
  __shared__ double A[kMaxPar * kMaxPar], V[kMaxPar * kMaxPar], rhs[kMaxPar];
  const int p = blockIdx.x, n = D.npar;
  const LmPix st = D.pix[p];
  double *req = D.req + (size_t)p * n;
  const double *nodes = D.nodes + (size_t)p * n;
  if (st.phase == PH_DONE) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) req[i] = nodes[i];
    return;
  }
  const int rows = D.nl * 4;
  const float *J = D.J + (size_t)p * n * rows;
  const float *ob = D.obs + (size_t)p * rows, *sc = D.scur + (size_t)p * rows;
  const float *mk = D.mask ? D.mask + (size_t)p * D.nl : nullptr;
  // one thread per entry of the upper triangle of J^T J, then one per entry of J^T r; J is
  // scaled by node scale x w_s x mask, r = (obs - S) w_s mask (atmos_fit.cc:229-260)
  const int npair = n * (n + 1) / 2;
  if (D.G) {  // tensor-core Gram matrix: [0, n) x [0, n) is J^T J, column n is J^T r
    const float *g = D.G + (size_t)p * 256;
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int i = e / n, j = e % n;
      A[e] = 0.5 * ((double)g[i * 16 + j] + (double)g[j * 16 + i]);
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x) rhs[i] = (double)g[i * 16 + n];
  }
  for (int e = threadIdx.x; e < (D.G ? 0 : npair + n); e += blockDim.x) {
    int i, j;
    if (e < npair) {
      i = 0;
      int rem = e;
      while (rem >= n - i) { rem -= n - i; ++i; }
      j = i + rem;
    } else {
      i = e - npair;
      j = -1;
    }
    const float *Ji = J + (size_t)i * rows;
    const float *Jj = j >= 0 ? J + (size_t)j * rows : nullptr;
    double acc = 0.0;
    for (int r = 0; r < rows; ++r) {
      const double w = D.ws[r & 3] * (mk ? (double)mk[r >> 2] : 1.0);
      const double a = (double)Ji[r] * w;
      const double b = Jj ? (double)Jj[r] * w : ((double)ob[r] - (double)sc[r]) * w;
      acc += a * b;
    }
    if (j >= 0) {
      const double v = acc * D.scale[i] * D.scale[j] / D.scale2;
      A[i * n + j] = v;
      A[j * n + i] = v;
    } else {
      rhs[i] = acc * D.scale[i] / D.scale2;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; ++i) A[i * n + i] *= (st.lm + 1.0);
    jacobi_eigen(A, V, n);
    double wmax = 0.0;
    for (int i = 0; i < n; ++i) wmax = fmax(wmax, fabs(A[i * n + i]));
    double corr[kMaxPar];
    for (int i = 0; i < n; ++i) corr[i] = 0.0;
    for (int k = 0; k < n; ++k) {
      const double w = fabs(A[k * n + k]);
      if (!(w > 0.0) || wmax / w > 1e6) continue;  // condition cut of solve_svd
      double t = 0.0;
      for (int i = 0; i < n; ++i) t += V[i * n + k] * rhs[i];
      t /= A[k * n + k];
      for (int i = 0; i < n; ++i) corr[i] += V[i * n + k] * t;
    }
    for (int i = 0; i < n; ++i) {
      double v = nodes[i] + corr[i] * D.scale[i];
      v = fmin(fmax(v, D.lo[i]), D.hi[i]);
      req[i] = v;
    }
    D.pix[p].phase = PH_TRIAL;
  }
}

void node_constants(int kind, double &scale, double &lo, double &hi) {
  // scales: cmlib/const.h:35-38; bounds: atmos/atmos_model.cc:12-19, 957-977 (angles unbounded)
  switch (kind) {
    case 1: scale = 5000.0; lo = 3400.0; hi = 12000.0; break;
    case 2: scale = 1e5; lo = 1e2; hi = 15e5; break;
    case 3: scale = 1e5; lo = -15e5; hi = 15e5; break;
    case 4: scale = 1000.0; lo = 1.0; hi = 1e4; break;
    default: scale = 1.0; lo = -HUGE_VAL; hi = HUGE_VAL; break;
  }
}

LmWork *work(snapi_ctx *ctx) { return static_cast<LmWork *>(ctx->lm); }

void free_bufs(LmWork *w) {
  void *b[] = {w->d_M, w->d_G, w->d_nodes, w->d_req, w->d_step, w->d_pix, w->d_obs, w->d_mask, w->d_scur, w->d_snew,
               w->d_J, w->d_rec, w->d_tan, w->d_skip_syn, w->d_skip_resp, w->d_active, w->d_req_out, w->d_act_out};
  for (void *x : b)
    if (x) cudaFree(x);
  w->d_req_out = nullptr;
  w->d_act_out = nullptr;
  w->d_nodes = w->d_req = w->d_step = nullptr;
  w->d_pix = nullptr;
  w->d_obs = w->d_mask = w->d_scur = w->d_snew = w->d_J = w->d_rec = w->d_tan = w->d_M = w->d_G = nullptr;
  w->d_skip_syn = w->d_skip_resp = w->d_active = nullptr;
  w->cap = w->cap_par = 0;
}

}  // namespace

namespace {

// one LM iteration in two phases (snapi_lm_step runs both; snapi_lm_fit builds the tangents between
// them for the pixels the first phase accepted):
// 1) synthesis at the requested nodes and the accept / reject decision; skip_resp[p] == 0 marks
//    the pixels whose Jacobian (and hence node tangents) the second phase needs
cudaError_t lm_eval_phase(snapi_ctx *ctx, LmWork *w, const float *rec) {
  KParams P = base_params(ctx);
  P.npix = w->npix;
  P.rec = rec;
  P.stokes = w->d_snew;
  P.skip = w->d_skip_syn;
  // forward-mode Jacobian: the synthesis at the requested nodes stores its sweep state, which the
  // Jacobian of the pixels it accepts reuses (their nodes are the requested ones)
  w->state_ready = ctx->jac_tangent && w->npix <= ctx->max_batch;
  cudaError_t e = w->state_ready ? launch_synth_state(ctx, P) : launch_synth(ctx, P);
  if (e != cudaSuccess) return e;
  if (w->broaden > 0.0 && (e = psf_launch(ctx, w->d_snew, w->npix, 1, w->d_skip_syn)) != cudaSuccess) return e;
  k_lm_eval<<<w->npix, kLmThreads, 0, ctx->stream>>>(w->D);
  return cudaGetLastError();
}

// 2) Jacobian at the accepted nodes along the tangents, normal equations, damped solve, next request
// the caller's Jacobian rows into J where the step renews them (skip[p] == 0)
__global__ void k_lm_copy_jac(const float *src, float *J, const int *skip, size_t row) {
  const int p = blockIdx.x;
  if (skip && skip[p]) return;
  const float *s = src + (size_t)p * row;
  float *d = J + (size_t)p * row;
  for (size_t i = threadIdx.x; i < row; i += blockDim.x) d[i] = s[i];
}

// jac (may be null): the caller's Jacobian dS/dnode [npix][npar][nl][4] (device), used instead of
// the responses along the record tangents
cudaError_t lm_solve_phase(snapi_ctx *ctx, LmWork *w, const float *rec, const float *tan, int &launches,
                           const float *jac = nullptr) {
  const int npix = w->npix, npar = w->npar;
  cudaError_t e = cudaSuccess;
  if (jac) {  // rows of pixels whose Jacobian is renewed this step (accepted or new); the others keep theirs
    const size_t row = (size_t)npar * ctx->nl * 4;
    k_lm_copy_jac<<<npix, 256, 0, ctx->stream>>>(jac, w->d_J, w->d_skip_resp, row);
    e = cudaGetLastError();
  } else {
    KParams R = base_params(ctx);
    R.npix = npix;
    R.npar = npar;
    R.nvar = npar;
    R.rec = rec;
    R.tangent = tan;
    R.fd_step = w->d_step;
    R.dstokes = w->d_J;
    R.skip = w->d_skip_resp;
    e = launch_responses(ctx, R, w->state_ready);
  }
  if (e != cudaSuccess) return e;
  if (w->broaden > 0.0 && (e = psf_launch(ctx, w->d_J, npix * npar, npar, w->d_skip_resp)) != cudaSuccess) return e;
  LmDev Ds = w->D;
  launches = 2;
  if (w->d_G && npar + 1 <= 16) {
    k_lm_rows<<<npix * 16, 256, 0, ctx->stream>>>(Ds, w->d_M);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_gram_tf32(w->d_M, npix, ctx->nl * 4, w->d_G, ctx->d_status, ctx->stream)) != cudaSuccess) return e;
    Ds.G = w->d_G;
    launches += 2;
  }
  k_lm_solve<<<npix, kLmThreads, 0, ctx->stream>>>(Ds);
  return cudaGetLastError();
}

// need[p] = 1 where the Jacobian is needed (skip_resp[p] == 0)
__global__ void k_lm_need(const int *skip_resp, int *need, int npix) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < npix) need[p] = skip_resp[p] ? 0 : 1;
}

}  // namespace

void snapi::lm_free(snapi_ctx *ctx) {
  if (!ctx || !ctx->lm) return;
  free_bufs(work(ctx));
  delete work(ctx);
  ctx->lm = nullptr;
}

extern "C" {

int snapi_lm_begin(snapi_ctx *ctx, int npix, const snapi_lm_opts *opts, const double *nodes0, const float *obs,
                   const double *w_stokes, const float *mask, double *request, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (!opts || npix < 1 || opts->npar < 1 || opts->npar > kMaxPar || !opts->node_kind || !opts->resp_step ||
      !nodes0 || !obs || !request || opts->max_iter < 1 || !(opts->lm_start >= 0.0) ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_lm_begin: invalid arguments");
  for (int i = 0; i < opts->npar; ++i) {
    if (opts->node_kind[i] < 1 || opts->node_kind[i] > 6)
      return set_err(ctx, SNAPI_EINVAL, "snapi_lm_begin: node_kind must be 1..6");
    if (!(opts->resp_step[i] > 0.0)) return set_err(ctx, SNAPI_EINVAL, "snapi_lm_begin: steps must be positive");
  }
  SNAPI_CK(cudaSetDevice(ctx->device));
  if (!ctx->lm) ctx->lm = new LmWork();
  LmWork *w = work(ctx);
  const int npar = opts->npar, nl = ctx->nl;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield;
  if (w->cap < npix || w->cap_par < npar) {
    free_bufs(w);
    SNAPI_CK(cudaMalloc(&w->d_nodes, sizeof(double) * npix * npar));
    SNAPI_CK(cudaMalloc(&w->d_req, sizeof(double) * npix * npar));
    SNAPI_CK(cudaMalloc(&w->d_step, sizeof(double) * npar));
    SNAPI_CK(cudaMalloc(&w->d_pix, sizeof(LmPix) * npix));
    SNAPI_CK(cudaMalloc(&w->d_obs, sizeof(float) * npix * nl * 4));
    SNAPI_CK(cudaMalloc(&w->d_mask, sizeof(float) * npix * nl));
    SNAPI_CK(cudaMalloc(&w->d_scur, sizeof(float) * npix * nl * 4));
    SNAPI_CK(cudaMalloc(&w->d_snew, sizeof(float) * npix * nl * 4));
    SNAPI_CK(cudaMalloc(&w->d_J, sizeof(float) * npix * npar * nl * 4));
    if (npar + 1 <= 16) {  // tensor-core normal equations
      SNAPI_CK(cudaMalloc(&w->d_M, sizeof(float) * npix * 16 * nl * 4));
      SNAPI_CK(cudaMalloc(&w->d_G, sizeof(float) * npix * 256));
    }
    SNAPI_CK(cudaMalloc(&w->d_rec, sizeof(float) * npix * nrec));
    // record tangents, or the staging of a caller's Jacobian (snapi_lm_step_jacobian)
    SNAPI_CK(cudaMalloc(&w->d_tan, sizeof(float) * npix * npar * std::max<size_t>(nrec, (size_t)nl * 4)));
    SNAPI_CK(cudaMalloc(&w->d_skip_syn, sizeof(int) * npix));
    SNAPI_CK(cudaMalloc(&w->d_skip_resp, sizeof(int) * npix));
    SNAPI_CK(cudaMalloc(&w->d_active, sizeof(int) * npix));
    w->cap = npix;
    w->cap_par = npar;
  }
  w->npix = npix;
  w->npar = npar;
  w->h_active.assign(npix, 1);
  w->kind.assign(opts->node_kind, opts->node_kind + npar);
  w->broaden = opts->spectral_broadening;
  if (w->broaden < 0.0) return set_err(ctx, SNAPI_EINVAL, "snapi_lm_begin: negative spectral broadening");
  if (w->broaden > 0.0) {
    const int st = psf_prepare(ctx, w->broaden);
    if (st) return st;
  }
  LmDev &D = w->D;
  memset(&D, 0, sizeof D);
  D.npix = npix; D.npar = npar; D.nl = nl;
  for (int s = 0; s < 4; ++s) D.ws[s] = w_stokes ? w_stokes[s] : 1.0;
  D.scale2 = ctx->scale2;
  D.delta = opts->delta;
  D.stopping = opts->stopping_chisq;
  D.lm_floor = 1e-5;
  D.max_iter = opts->max_iter;
  for (int i = 0; i < npar; ++i) node_constants(opts->node_kind[i], D.scale[i], D.lo[i], D.hi[i]);
  // bracketed starting nodes (atmos_fit.cc:91)
  std::vector<double> n0((size_t)npix * npar);
  if (mem == SNAPI_MEM_DEVICE)
    SNAPI_CK(cudaMemcpy(n0.data(), nodes0, sizeof(double) * n0.size(), cudaMemcpyDeviceToHost));
  else
    memcpy(n0.data(), nodes0, sizeof(double) * n0.size());
  for (int p = 0; p < npix; ++p)
    for (int i = 0; i < npar; ++i) {
      double &v = n0[(size_t)p * npar + i];
      v = std::fmin(std::fmax(v, D.lo[i]), D.hi[i]);
    }
  const cudaMemcpyKind in = mem == SNAPI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  SNAPI_CK(cudaMemcpyAsync(w->d_nodes, n0.data(), sizeof(double) * n0.size(), cudaMemcpyHostToDevice, ctx->stream));
  SNAPI_CK(cudaMemcpyAsync(w->d_req, n0.data(), sizeof(double) * n0.size(), cudaMemcpyHostToDevice, ctx->stream));
  SNAPI_CK(cudaMemcpyAsync(w->d_step, opts->resp_step, sizeof(double) * npar, cudaMemcpyHostToDevice, ctx->stream));
  SNAPI_CK(cudaMemcpyAsync(w->d_obs, obs, sizeof(float) * npix * nl * 4, in, ctx->stream));
  if (mask) SNAPI_CK(cudaMemcpyAsync(w->d_mask, mask, sizeof(float) * npix * nl, in, ctx->stream));
  std::vector<LmPix> st(npix);
  for (auto &x : st) {
    memset(&x, 0, sizeof x);
    x.lm = opts->lm_start;
    x.phase = PH_FIRST;
  }
  SNAPI_CK(cudaMemcpyAsync(w->d_pix, st.data(), sizeof(LmPix) * npix, cudaMemcpyHostToDevice, ctx->stream));
  SNAPI_CK(cudaMemsetAsync(w->d_skip_syn, 0, sizeof(int) * npix, ctx->stream));
  D.obs = w->d_obs;
  D.mask = mask ? w->d_mask : nullptr;
  D.snew = w->d_snew;
  D.scur = w->d_scur;
  D.J = w->d_J;
  D.nodes = w->d_nodes;
  D.req = w->d_req;
  D.pix = w->d_pix;
  D.skip_syn = w->d_skip_syn;
  D.skip_resp = w->d_skip_resp;
  D.active = w->d_active;
  if (mem == SNAPI_MEM_DEVICE)
    SNAPI_CK(cudaMemcpyAsync(request, w->d_req, sizeof(double) * n0.size(), cudaMemcpyDeviceToDevice, ctx->stream));
  else
    memcpy(request, n0.data(), sizeof(double) * n0.size());
  SNAPI_CK(cudaStreamSynchronize(ctx->stream));
  w->begun = true;
  return SNAPI_OK;
}

// snapi_lm_step (jac == false: `tangents` are record tangents) and snapi_lm_step_jacobian (jac:
// `tangents` is the caller's Jacobian dS/dnode [npix][npar][nl][4])
static int lm_step_impl(snapi_ctx *ctx, const float *records, const float *tangents, double *request, int *active,
                        int *n_active, int mem, bool jac) {
  if (!ctx) return SNAPI_EINVAL;
  LmWork *w = work(ctx);
  if (!w || !w->begun) return set_err(ctx, SNAPI_EINVAL, "snapi_lm_step: call snapi_lm_begin first");
  if (!records || !tangents || !request || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_lm_step: invalid arguments");
  SNAPI_CK(cudaSetDevice(ctx->device));
  const int npix = w->npix, npar = w->npar;
  const size_t nrec = (size_t)ctx->nd * ctx->nfield, nrow = jac ? (size_t)ctx->nl * 4 * npar : nrec * npar;
  const bool dev = mem == SNAPI_MEM_DEVICE;
  const float *rec = records, *tan = tangents;
  if (!dev) {
    // rows of inactive pixels are not needed: copy runs of active pixels only (a caller's Jacobian
    // is staged in the tangent buffer, which is larger, and copied into J after the evaluation)
    float *dst = w->d_tan;
    int p = 0;
    while (p < npix) {
      if (!w->h_active[p]) { ++p; continue; }
      int q = p;
      while (q < npix && w->h_active[q]) ++q;
      SNAPI_CK(cudaMemcpyAsync(w->d_rec + p * nrec, records + p * nrec, sizeof(float) * (q - p) * nrec,
                               cudaMemcpyHostToDevice, ctx->stream));
      SNAPI_CK(cudaMemcpyAsync(dst + (size_t)p * nrow, tangents + (size_t)p * nrow, sizeof(float) * (q - p) * nrow,
                               cudaMemcpyHostToDevice, ctx->stream));
      p = q;
    }
    rec = w->d_rec;
    tan = dst;
  }
  SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
  SNAPI_CK(lm_eval_phase(ctx, w, rec));
  int nl_solve = 0;
  SNAPI_CK(lm_solve_phase(ctx, w, rec, jac ? nullptr : tan, nl_solve, jac ? tan : nullptr));
  SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
  ctx->last_launches = 2 + nl_solve;
  SNAPI_CK(cudaMemcpyAsync(w->h_active.data(), w->d_active, sizeof(int) * npix, cudaMemcpyDeviceToHost, ctx->stream));
  if (dev) {
    SNAPI_CK(cudaMemcpyAsync(request, w->d_req, sizeof(double) * npix * npar, cudaMemcpyDeviceToDevice, ctx->stream));
    if (active)
      SNAPI_CK(cudaMemcpyAsync(active, w->d_active, sizeof(int) * npix, cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    SNAPI_CK(cudaMemcpyAsync(request, w->d_req, sizeof(double) * npix * npar, cudaMemcpyDeviceToHost, ctx->stream));
  }
  SNAPI_CK(cudaStreamSynchronize(ctx->stream));
  float ms = 0.f;
  SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
  ctx->last_ms = ms;
  int na = 0;
  for (int p = 0; p < npix; ++p) na += w->h_active[p] ? 1 : 0;
  if (!dev && active) memcpy(active, w->h_active.data(), sizeof(int) * npix);
  if (n_active) *n_active = na;
  return check_status(ctx);
}

int snapi_lm_step(snapi_ctx *ctx, const float *records, const float *tangents, double *request, int *active,
                  int *n_active, int mem) {
  return lm_step_impl(ctx, records, tangents, request, active, n_active, mem, false);
}

int snapi_lm_step_jacobian(snapi_ctx *ctx, const float *records, const float *jacobian, double *request,
                           int *active, int *n_active, int mem) {
  return lm_step_impl(ctx, records, jacobian, request, active, n_active, mem, true);
}

int snapi_lm_result(snapi_ctx *ctx, double *nodes, double *chi2, int *iters, float *stokes, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  LmWork *w = work(ctx);
  if (!w || !w->begun) return set_err(ctx, SNAPI_EINVAL, "snapi_lm_result: call snapi_lm_begin first");
  if (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE) return set_err(ctx, SNAPI_EINVAL, "snapi_lm_result: mem");
  SNAPI_CK(cudaSetDevice(ctx->device));
  const int npix = w->npix, npar = w->npar;
  std::vector<double> nd((size_t)npix * npar);
  std::vector<LmPix> st(npix);
  SNAPI_CK(cudaMemcpy(nd.data(), w->d_nodes, sizeof(double) * nd.size(), cudaMemcpyDeviceToHost));
  SNAPI_CK(cudaMemcpy(st.data(), w->d_pix, sizeof(LmPix) * npix, cudaMemcpyDeviceToHost));
  // polish_angles (atmos_model.cc:992-1002) on the returned nodes
  for (int p = 0; p < npix; ++p)
    for (int i = 0; i < npar; ++i) {
      double &v = nd[(size_t)p * npar + i];
      if (w->kind[i] == 5) v = std::acos(std::cos(v));
      if (w->kind[i] == 6) v = std::atan(std::tan(v));
    }
  const cudaMemcpyKind out = mem == SNAPI_MEM_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost;
  std::vector<double> c2(npix);
  std::vector<int> it(npix);
  for (int p = 0; p < npix; ++p) { c2[p] = st[p].chi2; it[p] = st[p].iter; }
  if (nodes) SNAPI_CK(cudaMemcpy(nodes, nd.data(), sizeof(double) * nd.size(), out));
  if (chi2) SNAPI_CK(cudaMemcpy(chi2, c2.data(), sizeof(double) * npix, out));
  if (iters) SNAPI_CK(cudaMemcpy(iters, it.data(), sizeof(int) * npix, out));
  if (stokes)
    SNAPI_CK(cudaMemcpy(stokes, w->d_scur, sizeof(float) * npix * ctx->nl * 4,
                        mem == SNAPI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost));
  return SNAPI_OK;
}

// The whole stokes_lm_fit (atmos_fit.cc:18-227) of a batch of pixels with the node -> record map
// on the device: every step builds the records and node tangents of the requested node vectors
// (snapi_build_records on the LM's own device buffers, active pixels only) and takes one LM
// iteration on them.  Nothing returns to the host between steps except the active count.
int snapi_lm_fit(snapi_ctx *ctx, int npix, const snapi_lm_opts *opts, const double *nodes0, const float *obs,
                 const double *w_stokes, const float *mask, double *nodes, double *chi2, int *iters, float *stokes,
                 int *n_steps, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (!opts || npix < 1 || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_lm_fit: invalid arguments");
  if (!eos_matches(ctx, opts->npar, opts->node_kind))
    return set_err(ctx, SNAPI_EINVAL, "snapi_lm_fit: no node model (snapi_eos_set) with these node kinds");
  std::vector<double> hreq;
  if (mem == SNAPI_MEM_HOST) hreq.resize((size_t)npix * opts->npar);
  SNAPI_CK(cudaSetDevice(ctx->device));
  double *req_dev = nullptr;
  if (mem == SNAPI_MEM_DEVICE) SNAPI_CK(cudaMalloc(&req_dev, sizeof(double) * (size_t)npix * opts->npar));
  int st = snapi_lm_begin(ctx, npix, opts, nodes0, obs, w_stokes, mask,
                          mem == SNAPI_MEM_HOST ? hreq.data() : req_dev, mem);
  if (req_dev) cudaFree(req_dev);
  if (st) return st;
  LmWork *w = work(ctx);
  if (!w->d_req_out) {
    SNAPI_CK(cudaMalloc(&w->d_req_out, sizeof(double) * (size_t)w->cap * w->cap_par));
    SNAPI_CK(cudaMalloc(&w->d_act_out, sizeof(int) * (size_t)w->cap));
  }
  SNAPI_CK(cudaMemcpyAsync(w->d_active, w->h_active.data(), sizeof(int) * npix, cudaMemcpyHostToDevice, ctx->stream));
  double ms = 0.0;
  int launches = 0, steps = 0;
  const int cap = 10 * opts->max_iter + 10;  // accepted + rejected steps of any pixel stay below this
  auto timed = [&](auto &&fn) -> int {  // device time of a stretch of launches on the context stream
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    SNAPI_CK(fn());
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    SNAPI_CK(cudaEventSynchronize(ctx->ev1));
    float t = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    ms += t;
    return SNAPI_OK;
  };
  // A build costs about a column's serial chain (~0.1 s on B200) plus a few us per column-variant
  // (9 per pixel with tangents).  Splitting a step (records of every active pixel; tangents only
  // where the trial step was accepted) saves the tangents of the rejected pixels but adds one
  // chain.  Measured on B200: 1024 pixels, 142 ms per step unsplit against 259 split; 16384 pixels,
  // 36.7 s per fit split throughout against 40.4 s when steps with fewer than 6144 active pixels
  // went unsplit.
  const int kSplitMin = 2048;
  int n_active = npix;
  for (;;) {
    if (n_active >= kSplitMin) {
      // records of the requested nodes of the active pixels; synthesis and accept / reject
      st = snapi_build_records(ctx, npix, w->d_req, w->d_active, w->d_rec, nullptr, nullptr, nullptr, nullptr,
                               SNAPI_MEM_DEVICE);
      if (st) return st;
      ms += ctx->last_ms;
      launches += ctx->last_launches;
      st = timed([&] {
        cudaError_t e = lm_eval_phase(ctx, w, w->d_rec);
        if (e != cudaSuccess) return e;
        k_lm_need<<<(npix + 255) / 256, 256, 0, ctx->stream>>>(w->d_skip_resp, w->d_act_out, npix);
        return cudaGetLastError();
      });
      if (st) return st;
      launches += 3 + (w->broaden > 0.0 ? 1 : 0);
      // node tangents only where the step was accepted (the Jacobian is taken there), as the
      // reference computes responses only at accepted models
      st = snapi_build_records(ctx, npix, w->d_req, w->d_act_out, w->d_rec, nullptr, w->d_tan, nullptr, nullptr,
                               SNAPI_MEM_DEVICE);
      if (st) return st;
      ms += ctx->last_ms;
      launches += ctx->last_launches;
    } else {
      // records and tangents of every active pixel in one build, then the step's evaluation
      st = snapi_build_records(ctx, npix, w->d_req, w->d_active, w->d_rec, nullptr, w->d_tan, nullptr, nullptr,
                               SNAPI_MEM_DEVICE);
      if (st) return st;
      ms += ctx->last_ms;
      launches += ctx->last_launches;
      st = timed([&] { return lm_eval_phase(ctx, w, w->d_rec); });
      if (st) return st;
      launches += 2 + (w->broaden > 0.0 ? 1 : 0);
    }
    int nls = 0;
    st = timed([&] { return lm_solve_phase(ctx, w, w->d_rec, w->d_tan, nls); });
    if (st) return st;
    launches += nls + (w->broaden > 0.0 ? 1 : 0);
    SNAPI_CK(cudaMemcpy(w->h_active.data(), w->d_active, sizeof(int) * npix, cudaMemcpyDeviceToHost));
    st = check_status(ctx);
    if (st) return st;
    int na = 0;
    for (int p = 0; p < npix; ++p) na += w->h_active[p] ? 1 : 0;
    n_active = na;
    ++steps;
    if (na == 0) break;
    if (steps >= cap) return set_err(ctx, SNAPI_ENONCONV, "snapi_lm_fit: %d pixels still active after %d steps", na, steps);
  }
  st = snapi_lm_result(ctx, nodes, chi2, iters, stokes, mem);
  ctx->last_ms = ms;
  ctx->last_launches = launches;
  if (n_steps) *n_steps = steps;
  return st;
}

}  // extern "C"
