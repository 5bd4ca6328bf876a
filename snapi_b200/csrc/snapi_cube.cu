// The master's inversion job (master/job.cc:304-379, 570-597) with every pixel fitted on the GPU
// and the cube streamed between .f0 files and HBM.
//
// Reference flow: read the whole observed cube (read_file 4-D, fileio.cc:54-87) and transpose it
// (mathtools.cc:603-613) into S[x][y][s][l]; scale it by synth_qs / obs_qs (observable::normalize,
// obs.cc:398-408); cut the subfield and wavelength window (observable::extract, obs.cc:360-390),
// writing it to cube_to_invert.f0; pack one task per pixel with its starting model (the job's
// model, or model_cube[x][y] of a model cube, job.cc:347-369) for the islaves, which run
// stokes_lm_fit; collect the fitted nodes and spectra and write inverted_nodes.f0 (write_file 3-D,
// fileio.cc:274-287), inverted_atmos.f0 (the 12 return_as_array rows of each fitted column) and
// inverted_spectra.f0 (write_file 4-D, fileio.cc:320-329).
//
// Here one batch ("chunk") of subfield pixels at a time travels as a contiguous run of file rows:
// the file stores each pixel's [4][nl] block contiguously (dims (nl, 4, ny, nx)), so a chunk of
// pixels of one x row is a single read.  A reader thread fetches chunk k+1 into pinned memory while
// the GPU fits chunk k (snapi_lm_fit, all of it device-resident), and a writer thread stores chunk
// k-1's spectra; the node cube (a few MB) is written at the end.  The scaling, window cut and
// Stokes transposition run in one kernel per chunk (k_cube_obs), the float64 spectra layout in
// another (k_cube_spectra).
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <fcntl.h>
#include <unistd.h>

#include "snapi_internal.cuh"
#include "snapi_f0_internal.h"

namespace {

constexpr int kThreads = 256;

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  const long long cap = 148 * 16;  // grid-stride beyond 16 CTAs per SM
  return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

// raw [npix][4][nl_full] (float32 or float64, native byte order) -> obs [npix][nl][4] float32 of
// the window l0 .. l0 + nl - 1, multiplied by scale in float64 as the reference does (fp_t S *=
// synth_qs / obs_qs); win [npix][4][nl] float64 of the same values (NULL: not needed).
__global__ void k_cube_obs(const void *raw, int is_f64, int npix, int nl_full, int l0, int nl, double scale,
                           float *__restrict__ obs, double *__restrict__ win) {
  const long long n = (long long)npix * nl * 4;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(o & 3);
    const long long t = o >> 2;
    const int l = (int)(t % nl);
    const long long p = t / nl;
    const long long src = (p * 4 + s) * nl_full + l0 + l;
    double v = is_f64 ? ((const double *)raw)[src] : (double)((const float *)raw)[src];
    v *= scale;
    obs[o] = (float)v;
    if (win) win[(p * 4 + s) * nl + l] = v;
  }
}

// stokes [npix][nl][4] float32 -> out [npix][4][nl] float64 (the reference's S[x][y][s][l])
__global__ void k_cube_spectra(const float *__restrict__ stokes, int npix, int nl, double *__restrict__ out) {
  const long long n = (long long)npix * nl * 4;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(o % nl);
    const long long t = o / nl;
    const int s = (int)(t & 3);
    const long long p = t >> 2;
    out[o] = (double)stokes[(p * nl + l) * 4 + s];
  }
}

// atm [npix][12][nd] -> out [12][npix][nd] (the chunk's part of inverted_atmos.f0's rows)
__global__ void k_cube_atm(const double *__restrict__ atm, int npix, int nd, double *__restrict__ out) {
  const long long n = (long long)npix * 12 * nd;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(o % nd);
    const long long t = o / nd;
    const int p = (int)(t % npix), k = (int)(t / npix);
    out[o] = atm[((size_t)p * 12 + k) * nd + z];
  }
}

// the window of the wavelength weights, repeated for every pixel of a chunk
__global__ void k_cube_mask(const float *__restrict__ m, int npix, int nl, float *__restrict__ out) {
  const long long n = (long long)npix * nl;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < n; o += (long long)gridDim.x * blockDim.x)
    out[o] = m[o % nl];
}

using Clock = std::chrono::steady_clock;
double secs(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double>(b - a).count(); }

// Two pinned buffers handed between the main thread and one worker thread.
struct Handoff {
  struct Slot {
    uint8_t *h = nullptr;
    bool full = false;
    long long p0 = 0;
    int n = 0;
  } slot[2];
  std::mutex mu;
  std::condition_variable cv;
  bool abort = false;
  std::string err;

  // waits until slot k % 2 is full (want_full) or empty; false on abort
  bool wait(int k, bool want_full, double *waited) {
    auto t0 = Clock::now();
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return abort || slot[k & 1].full == want_full; });
    if (waited) *waited += secs(t0, Clock::now());
    return !abort;
  }
  void set(int k, bool full) {
    { std::lock_guard<std::mutex> lk(mu); slot[k & 1].full = full; }
    cv.notify_all();
  }
  void fail(const std::string &e) {
    { std::lock_guard<std::mutex> lk(mu); if (err.empty()) err = e; abort = true; }
    cv.notify_all();
  }
};

struct Job {
  snapi_ctx *ctx = nullptr;
  // geometry (0-based subfield origin in the file)
  int nx_full = 0, ny_full = 0, nl_full = 0, x0 = 0, y0 = 0, nx = 0, ny = 0, l0 = 0, nl = 0, npar = 0;
  long long npix = 0;
  int chunk = 0, nchunk = 0;
  int fd = -1;
  snapi_f0_info info{};
  int esz = 0;
  double scale = 1.0;
  // device buffers (chunk pixels)
  void *d_raw = nullptr;
  float *d_obs = nullptr, *d_stokes = nullptr, *d_mask = nullptr, *d_maskwin = nullptr;
  double *d_win = nullptr, *d_spec = nullptr, *d_nodes0 = nullptr, *d_nodes = nullptr, *d_chi2 = nullptr;
  double *d_atm = nullptr, *d_atmT = nullptr;
  int *d_iters = nullptr;
  // pinned host buffers
  double *h_nodes0 = nullptr, *h_nodes = nullptr, *h_chi2 = nullptr;
  int *h_iters = nullptr;
  Handoff rd, wr;
  size_t raw_bytes = 0, spec_bytes = 0, atm_bytes = 0;
  int nd = 0;
  bool want_win = false;
  snapi_f0_file *f_spec = nullptr, *f_cube = nullptr, *f_atm = nullptr;
  std::vector<double> model;      // model cube, float64, file order
  long long mdim0 = 0, mdim1 = 0;
  std::vector<float> node_cube;   // [npar][ny][nx]
  long long bytes_read = 0, bytes_written = 0;

  ~Job() {
    if (fd >= 0) close(fd);
    for (void *p : {(void *)d_raw, (void *)d_obs, (void *)d_stokes, (void *)d_mask, (void *)d_maskwin, (void *)d_win,
                    (void *)d_spec, (void *)d_nodes0, (void *)d_nodes, (void *)d_chi2, (void *)d_iters,
                    (void *)d_atm, (void *)d_atmT})
      if (p) cudaFree(p);
    for (void *p : {(void *)h_nodes0, (void *)h_nodes, (void *)h_chi2, (void *)h_iters, (void *)rd.slot[0].h,
                    (void *)rd.slot[1].h, (void *)wr.slot[0].h, (void *)wr.slot[1].h})
      if (p) cudaFreeHost(p);
    if (f_spec) snapi_f0_close(f_spec);
    if (f_cube) snapi_f0_close(f_cube);
    if (f_atm) snapi_f0_close(f_atm);
  }

  int chunk_len(int k) const {
    long long a = (long long)k * chunk, b = a + chunk;
    return (int)((b > npix ? npix : b) - a);
  }

  // reader thread: the file rows of each chunk's pixels, in subfield order (x major)
  void reader() {
    std::vector<uint8_t> scratch;
    const long long pix_elems = 4LL * nl_full;
    for (int k = 0; k < nchunk; ++k) {
      if (!rd.wait(k, false, nullptr)) return;
      Handoff::Slot &s = rd.slot[k & 1];
      s.p0 = (long long)k * chunk;
      s.n = chunk_len(k);
      long long p = s.p0, end = s.p0 + s.n;
      uint8_t *dst = s.h;
      while (p < end) {
        const long long x = p / ny, y = p % ny;
        long long run = ny - y;
        if (run > end - p) run = end - p;
        const long long first = ((x0 + x) * ny_full + (y0 + y)) * pix_elems;
        if (snapi_f0::read_range(fd, info, first, run * pix_elems, dst, info.type, scratch)) {
          rd.fail(std::string("snapi_cube_invert: ") + snapi_f0_error());
          return;
        }
        dst += run * pix_elems * esz;
        p += run;
      }
      bytes_read += (long long)s.n * pix_elems * esz;
      rd.set(k, true);
    }
  }

  // writer thread: the chunk's float64 spectra (and window, and atmosphere rows) at its pixels'
  // place in the files
  void writer() {
    const long long pix_elems = 4LL * nl;
    for (int k = 0; k < nchunk; ++k) {
      if (!wr.wait(k, true, nullptr)) return;
      Handoff::Slot &s = wr.slot[k & 1];
      const double *spec = (const double *)s.h;
      const double *win = spec + (size_t)chunk * pix_elems;
      const double *atm = (const double *)(s.h + spec_bytes * (want_win ? 2 : 1));
      if (f_atm)  // row q of inverted_atmos.f0 holds [x][y][z]: this chunk's pixels are one run
        for (int q = 0; q < 12; ++q)
          if (snapi_f0_write_at(f_atm, ((long long)q * npix + s.p0) * nd, (long long)s.n * nd,
                                atm + (size_t)q * s.n * nd)) {
            wr.fail(std::string("snapi_cube_invert: ") + snapi_f0_error());
            return;
          }
      if (f_spec && snapi_f0_write_at(f_spec, s.p0 * pix_elems, s.n * pix_elems, spec)) {
        wr.fail(std::string("snapi_cube_invert: ") + snapi_f0_error());
        return;
      }
      if (f_cube && snapi_f0_write_at(f_cube, s.p0 * pix_elems, s.n * pix_elems, win)) {
        wr.fail(std::string("snapi_cube_invert: ") + snapi_f0_error());
        return;
      }
      bytes_written += (long long)s.n * pix_elems * 8 * ((f_spec ? 1 : 0) + (f_cube ? 1 : 0)) +
                       (f_atm ? (long long)s.n * 12 * nd * 8 : 0);
      wr.set(k, false);
    }
  }
};

}  // namespace

extern "C" int snapi_cube_invert(snapi_ctx *ctx, const snapi_lm_opts *opts, const snapi_cube_job *job,
                                 snapi_cube_stats *stats) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  if (!opts || !job || !job->obs_path) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: null argument");
  if (!job->nodes0 && !job->model_path)
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: neither nodes0 nor a model cube");
  if (!eos_matches(ctx, opts->npar, opts->node_kind))
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: no node model (snapi_eos_set) with these node kinds");
  const auto t_start = Clock::now();
  Job J;
  J.ctx = ctx;
  J.npar = opts->npar;
  J.fd = open(job->obs_path, O_RDONLY);
  if (J.fd < 0) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: cannot open %s", job->obs_path);
  if (snapi_f0::parse(J.fd, &J.info)) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %s", snapi_f0_error());
  const snapi_f0_info &I = J.info;
  if (I.ndim != 4) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: the cube has %d dimensions, not 4", I.ndim);
  if (I.type != SNAPI_F0_FLOAT32 && I.type != SNAPI_F0_FLOAT64)
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: data type of the cube is not floating point");
  if (I.compressed) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: compressed cube");
  if (I.dim[1] != 4) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %lld Stokes parameters, not 4", I.dim[1]);
  J.nl_full = (int)I.dim[0];
  J.ny_full = (int)I.dim[2];
  J.nx_full = (int)I.dim[3];
  J.esz = snapi_f0::type_size(I.type);
  const int xl = job->xl > 0 ? job->xl : 1, xh = job->xh > 0 ? job->xh : J.nx_full;
  const int yl = job->yl > 0 ? job->yl : 1, yh = job->yh > 0 ? job->yh : J.ny_full;
  const int ll = job->ll > 0 ? job->ll : 1, lh = job->lh > 0 ? job->lh : J.nl_full;
  if (xl > xh || xh > J.nx_full || yl > yh || yh > J.ny_full || ll > lh || lh > J.nl_full)
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: subfield / window outside the cube (%d x %d x %d)",
                   J.nx_full, J.ny_full, J.nl_full);
  J.x0 = xl - 1; J.y0 = yl - 1; J.l0 = ll - 1;
  J.nx = xh - xl + 1; J.ny = yh - yl + 1; J.nl = lh - ll + 1;
  if (J.nl != ctx->nl)
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: the window has %d wavelengths, the context %d", J.nl, ctx->nl);
  J.npix = (long long)J.nx * J.ny;
  // A fit's steps carry a fixed cost (the serial hydrostatic chain of the node build, ~0.1 s per
  // build) whatever the batch size, so few large chunks fit fastest: 16384 pixels of a 128 x 128
  // cube took 37 s as one chunk and 64 s as four.  65536 pixels hold < 10 GB of fit state.
  J.chunk = job->chunk > 0 ? job->chunk : 65536;
  if (J.chunk > J.npix) J.chunk = (int)J.npix;
  J.nchunk = (int)((J.npix + J.chunk - 1) / J.chunk);
  J.scale = (job->obs_qs != 0.0 || job->synth_qs != 0.0) ? job->synth_qs / job->obs_qs : 1.0;
  if (!std::isfinite(J.scale)) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: synth_qs / obs_qs is not finite");
  // starting nodes from a model cube (read_file 3-D: model_cube[x][y][p], file dims (nx, ny, npar))
  if (job->model_path) {
    snapi_f0_info mi;
    if (snapi_f0_stat(job->model_path, &mi))
      return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %s", snapi_f0_error());
    if (mi.ndim != 3 || mi.dim[0] < J.nx || mi.dim[1] < J.ny || mi.dim[2] != J.npar ||
        (mi.type != SNAPI_F0_FLOAT32 && mi.type != SNAPI_F0_FLOAT64))
      return set_err(ctx, SNAPI_EINVAL,
                     "snapi_cube_invert: the model cube must be floating point with dims (>= %d, >= %d, %d)", J.nx,
                     J.ny, J.npar);
    J.model.resize((size_t)mi.nelem);
    if (snapi_f0_read(job->model_path, 0, mi.nelem, J.model.data(), SNAPI_F0_FLOAT64))
      return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %s", snapi_f0_error());
    J.mdim0 = mi.dim[0]; J.mdim1 = mi.dim[1];
  }
  const int C = J.chunk, nl = J.nl, npar = J.npar;
  J.want_win = job->out_cube != nullptr;
  J.nd = ctx->nd;
  J.raw_bytes = (size_t)C * 4 * J.nl_full * J.esz;
  J.spec_bytes = (size_t)C * 4 * nl * sizeof(double);
  J.atm_bytes = job->out_atmos ? (size_t)C * 12 * J.nd * sizeof(double) : 0;
  SNAPI_CK(cudaSetDevice(ctx->device));
  SNAPI_CK(cudaMalloc(&J.d_raw, J.raw_bytes));
  SNAPI_CK(cudaMalloc(&J.d_obs, sizeof(float) * (size_t)C * nl * 4));
  SNAPI_CK(cudaMalloc(&J.d_stokes, sizeof(float) * (size_t)C * nl * 4));
  SNAPI_CK(cudaMalloc(&J.d_spec, J.spec_bytes));
  if (J.want_win) SNAPI_CK(cudaMalloc(&J.d_win, J.spec_bytes));
  SNAPI_CK(cudaMalloc(&J.d_nodes0, sizeof(double) * (size_t)C * npar));
  SNAPI_CK(cudaMalloc(&J.d_nodes, sizeof(double) * (size_t)C * npar));
  SNAPI_CK(cudaMalloc(&J.d_chi2, sizeof(double) * (size_t)C));
  SNAPI_CK(cudaMalloc(&J.d_iters, sizeof(int) * (size_t)C));
  if (J.atm_bytes) {
    SNAPI_CK(cudaMalloc(&J.d_atm, J.atm_bytes));
    SNAPI_CK(cudaMalloc(&J.d_atmT, J.atm_bytes));
  }
  SNAPI_CK(cudaHostAlloc((void **)&J.h_nodes0, sizeof(double) * (size_t)C * npar, cudaHostAllocDefault));
  SNAPI_CK(cudaHostAlloc((void **)&J.h_nodes, sizeof(double) * (size_t)C * npar, cudaHostAllocDefault));
  SNAPI_CK(cudaHostAlloc((void **)&J.h_chi2, sizeof(double) * (size_t)C, cudaHostAllocDefault));
  SNAPI_CK(cudaHostAlloc((void **)&J.h_iters, sizeof(int) * (size_t)C, cudaHostAllocDefault));
  for (int i = 0; i < 2; ++i) {
    SNAPI_CK(cudaHostAlloc((void **)&J.rd.slot[i].h, J.raw_bytes, cudaHostAllocDefault));
    SNAPI_CK(cudaHostAlloc((void **)&J.wr.slot[i].h, J.spec_bytes * (J.want_win ? 2 : 1) + J.atm_bytes,
                           cudaHostAllocDefault));
  }
  double ker_ms = 0.0;
  int launches = 0;
  if (job->mask) {
    SNAPI_CK(cudaMalloc(&J.d_maskwin, sizeof(float) * (size_t)nl));
    SNAPI_CK(cudaMalloc(&J.d_mask, sizeof(float) * (size_t)C * nl));
    SNAPI_CK(cudaMemcpyAsync(J.d_maskwin, job->mask + J.l0, sizeof(float) * nl, cudaMemcpyHostToDevice, ctx->stream));
    k_cube_mask<<<grid_for((long long)C * nl), kThreads, 0, ctx->stream>>>(J.d_maskwin, C, nl, J.d_mask);
    SNAPI_CK(cudaGetLastError());
    ++launches;
  }
  // output files: the spectra and the window are streamed, the node cube written at the end
  int st = SNAPI_OK;
  if (job->out_spectra) {
    const long long dims[4] = {nl, 4, J.ny, J.nx};
    J.f_spec = snapi_f0_create(job->out_spectra, SNAPI_F0_FLOAT64, 4, dims, nullptr, &st);
    if (!J.f_spec) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %s", snapi_f0_error());
  }
  if (job->out_cube) {
    const long long dims[4] = {nl, 4, J.ny, J.nx};
    J.f_cube = snapi_f0_create(job->out_cube, SNAPI_F0_FLOAT64, 4, dims, nullptr, &st);
    if (!J.f_cube) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %s", snapi_f0_error());
  }
  if (job->out_atmos) {
    const long long dims[4] = {J.nd, J.ny, J.nx, 12};
    J.f_atm = snapi_f0_create(job->out_atmos, SNAPI_F0_FLOAT64, 4, dims, nullptr, &st);
    if (!J.f_atm) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %s", snapi_f0_error());
  }
  if (job->out_nodes) J.node_cube.assign((size_t)npar * J.npix, 0.0f);

  double read_wait = 0.0, write_wait = 0.0, fit_s = 0.0;
  long long lm_steps = 0;
  std::thread t_rd([&] { J.reader(); }), t_wr([&] { J.writer(); });
  auto stop = [&](int code) {
    J.rd.fail(J.rd.err.empty() ? "stopped" : J.rd.err);
    J.wr.fail(J.wr.err.empty() ? "stopped" : J.wr.err);
    t_rd.join();
    t_wr.join();
    return code;
  };
#define CUBE_CK(call)                                                                                  \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess)                                                                             \
      return stop(set_err(ctx, SNAPI_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)));                  \
  } while (0)
  for (int k = 0; k < J.nchunk; ++k) {
    if (!J.rd.wait(k, true, &read_wait)) {
      std::string e = J.rd.err;
      return stop(set_err(ctx, SNAPI_EINVAL, "%s", e.c_str()));
    }
    const long long p0 = (long long)k * C;
    const int n = J.chunk_len(k);
    // starting nodes of the chunk's pixels
    for (int i = 0; i < n; ++i) {
      const long long p = p0 + i, x = p / J.ny, y = p % J.ny;
      for (int q = 0; q < npar; ++q)
        J.h_nodes0[(size_t)i * npar + q] =
            job->model_path ? J.model[(size_t)((q * J.mdim1 + y) * J.mdim0 + x)] : job->nodes0[q];
    }
    CUBE_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    CUBE_CK(cudaMemcpyAsync(J.d_raw, J.rd.slot[k & 1].h, (size_t)n * 4 * J.nl_full * J.esz, cudaMemcpyHostToDevice,
                            ctx->stream));
    CUBE_CK(cudaMemcpyAsync(J.d_nodes0, J.h_nodes0, sizeof(double) * (size_t)n * npar, cudaMemcpyHostToDevice,
                            ctx->stream));
    k_cube_obs<<<grid_for((long long)n * nl * 4), kThreads, 0, ctx->stream>>>(
        J.d_raw, I.type == SNAPI_F0_FLOAT64, n, J.nl_full, J.l0, nl, J.scale, J.d_obs, J.d_win);
    CUBE_CK(cudaGetLastError());
    CUBE_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CUBE_CK(cudaEventSynchronize(ctx->ev1));
    float t = 0.f;
    CUBE_CK(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    ker_ms += t;
    ++launches;
    J.rd.set(k, false);  // the reader may fill this slot with chunk k + 2
    const auto tf = Clock::now();
    int steps = 0;
    st = snapi_lm_fit(ctx, n, opts, J.d_nodes0, J.d_obs, job->w_stokes, job->mask ? J.d_mask : nullptr, J.d_nodes,
                      J.d_chi2, J.d_iters, J.d_stokes, &steps, SNAPI_MEM_DEVICE);
    fit_s += secs(tf, Clock::now());
    if (st) return stop(st);
    ker_ms += ctx->last_ms;
    launches += ctx->last_launches;
    lm_steps += steps;
    if (J.atm_bytes) {  // the fitted columns (job.cc:555-557)
      st = snapi_build_atmos(ctx, n, J.d_nodes, nullptr, job->x3, J.d_atm, nullptr, SNAPI_MEM_DEVICE);
      if (st) return stop(st);
      ker_ms += ctx->last_ms;
      launches += ctx->last_launches;
    }
    if (!J.wr.wait(k, false, &write_wait)) {
      std::string e = J.wr.err;
      return stop(set_err(ctx, SNAPI_EINVAL, "%s", e.c_str()));
    }
    Handoff::Slot &ws = J.wr.slot[k & 1];
    CUBE_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    k_cube_spectra<<<grid_for((long long)n * nl * 4), kThreads, 0, ctx->stream>>>(J.d_stokes, n, nl, J.d_spec);
    CUBE_CK(cudaGetLastError());
    ++launches;
    if (J.atm_bytes) {
      k_cube_atm<<<grid_for((long long)n * 12 * J.nd), kThreads, 0, ctx->stream>>>(J.d_atm, n, J.nd, J.d_atmT);
      CUBE_CK(cudaGetLastError());
      ++launches;
    }
    CUBE_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    CUBE_CK(cudaMemcpyAsync(ws.h, J.d_spec, sizeof(double) * (size_t)n * 4 * nl, cudaMemcpyDeviceToHost, ctx->stream));
    if (J.want_win)
      CUBE_CK(cudaMemcpyAsync(ws.h + J.spec_bytes, J.d_win, sizeof(double) * (size_t)n * 4 * nl,
                              cudaMemcpyDeviceToHost, ctx->stream));
    if (J.atm_bytes)
      CUBE_CK(cudaMemcpyAsync(ws.h + J.spec_bytes * (J.want_win ? 2 : 1), J.d_atmT,
                              sizeof(double) * (size_t)n * 12 * J.nd, cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CK(cudaMemcpyAsync(J.h_nodes, J.d_nodes, sizeof(double) * (size_t)n * npar, cudaMemcpyDeviceToHost,
                            ctx->stream));
    CUBE_CK(cudaMemcpyAsync(J.h_chi2, J.d_chi2, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CK(cudaMemcpyAsync(J.h_iters, J.d_iters, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CUBE_CK(cudaStreamSynchronize(ctx->stream));
    CUBE_CK(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    ker_ms += t;
    for (int i = 0; i < n; ++i) {
      const long long p = p0 + i, x = p / J.ny, y = p % J.ny;
      if (job->chi2) job->chi2[p] = J.h_chi2[i];
      if (job->iters) job->iters[p] = J.h_iters[i];
      if (job->out_nodes)  // write_file 3-D: element (x, y, q) at (q * ny + y) * nx + x
        for (int q = 0; q < npar; ++q)
          J.node_cube[(size_t)((q * J.ny + y) * J.nx + x)] = (float)J.h_nodes[(size_t)i * npar + q];
    }
    ws.p0 = p0;
    ws.n = n;
    J.wr.set(k, true);
  }
#undef CUBE_CK
  // drain the writer
  {
    const auto tw = Clock::now();
    std::unique_lock<std::mutex> lk(J.wr.mu);
    J.wr.cv.wait(lk, [&] { return J.wr.abort || (!J.wr.slot[0].full && !J.wr.slot[1].full); });
    write_wait += secs(tw, Clock::now());
  }
  t_rd.join();
  t_wr.join();
  if (!J.wr.err.empty()) return set_err(ctx, SNAPI_EINVAL, "%s", J.wr.err.c_str());
  if (!J.rd.err.empty()) return set_err(ctx, SNAPI_EINVAL, "%s", J.rd.err.c_str());
  if (J.f_spec) { snapi_f0_file *f = J.f_spec; J.f_spec = nullptr; if (snapi_f0_close(f)) st = SNAPI_EINVAL; }
  if (J.f_cube) { snapi_f0_file *f = J.f_cube; J.f_cube = nullptr; if (snapi_f0_close(f)) st = SNAPI_EINVAL; }
  if (J.f_atm) { snapi_f0_file *f = J.f_atm; J.f_atm = nullptr; if (snapi_f0_close(f)) st = SNAPI_EINVAL; }
  if (st) return set_err(ctx, st, "snapi_cube_invert: %s", snapi_f0_error());
  if (job->out_nodes) {
    const long long dims[3] = {J.nx, J.ny, npar};
    if (snapi_f0_write(job->out_nodes, J.node_cube.data(), SNAPI_F0_FLOAT32, 3, dims, nullptr))
      return set_err(ctx, SNAPI_EINVAL, "snapi_cube_invert: %s", snapi_f0_error());
    J.bytes_written += (long long)J.node_cube.size() * 4;
  }
  ctx->last_ms = ker_ms;
  ctx->last_launches = launches;
  if (stats) {
    stats->pixels = J.npix;
    stats->chunks = J.nchunk;
    stats->lm_steps = lm_steps;
    stats->wall_s = secs(t_start, Clock::now());
    stats->fit_s = fit_s;
    stats->read_wait_s = read_wait;
    stats->write_wait_s = write_wait;
    stats->bytes_read = J.bytes_read;
    stats->bytes_written = J.bytes_written;
    stats->kernel_ms = ker_ms;
    stats->launches = launches;
    stats->flagged = 0;
  }
  return SNAPI_OK;
}

// ---- the synthesis branch of the master's job (master/job.cc:384-409) ----------------------------------
// An atmosphere cube (the 12 return_as_array rows, dims (nd, ny, nx, 12), as atmosphere::read_spinor3d
// reads it, atmos_fio.cc:79-124) is streamed column chunk by column chunk: a reader thread fetches the
// next chunk's rows (12 reads per x row of the chunk), the GPU turns the columns into records
// (snapi_records_from_columns) and synthesises them (snapi_synth), and a writer thread stores the
// previous chunk's float64 spectra where write_file 4-D puts them (S[x][y][s][l], job.cc:595).
namespace {

// rows [12][cap][nd] (the chunk's file rows) -> cols [n][12][nd]
// T of columns [n][12][nd] floored at 3200 K in place (read_spinor3d's floor, which the records apply
// themselves, for the NLTE set-up that reads the columns as given)
__global__ void k_cube_floor_T(double *cols, int n, int nd) {
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < (long long)n * nd;
       o += (long long)gridDim.x * blockDim.x) {
    double *t = cols + (o / nd) * 12 * nd + 2 * nd + o % nd;
    if (!(*t > 3200.0)) *t = 3200.0;
  }
}

__global__ void k_cube_cols(const double *__restrict__ rows, int n, int cap, int nd, double *__restrict__ cols) {
  const long long m = (long long)n * 12 * nd;
  for (long long o = blockIdx.x * (long long)blockDim.x + threadIdx.x; o < m; o += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(o % nd);
    const long long t = o / nd;
    const int k = (int)(t % 12), p = (int)(t / 12);
    cols[o] = rows[((size_t)k * cap + p) * nd + z];
  }
}

struct SynthJob {
  int fd = -1;
  snapi_f0_info info{};
  int nx_full = 0, ny_full = 0, nd = 0, x0 = 0, y0 = 0, nx = 0, ny = 0, nl = 0, chunk = 0, nchunk = 0;
  long long npix = 0;
  double *d_rows = nullptr, *d_cols = nullptr, *d_spec = nullptr;
  float *d_rec = nullptr, *d_stokes = nullptr;
  int *d_st = nullptr;
  Handoff rd, wr;
  size_t rows_bytes = 0, spec_bytes = 0;
  snapi_f0_file *f_spec = nullptr;
  long long bytes_read = 0, bytes_written = 0;
  // an NLTE atom: the set-up's outputs (the iteration's columns), populations and statuses of a chunk
  double *d_ali = nullptr;
  snapi_ali_setup_out ali_out{};
  double *d_pops = nullptr;
  int *d_ast = nullptr;

  ~SynthJob() {
    if (fd >= 0) close(fd);
    for (void *p : {(void *)d_rows, (void *)d_cols, (void *)d_spec, (void *)d_rec, (void *)d_stokes, (void *)d_st,
                    (void *)d_ali, (void *)d_pops, (void *)d_ast})
      if (p) cudaFree(p);
    for (void *p : {(void *)rd.slot[0].h, (void *)rd.slot[1].h, (void *)wr.slot[0].h, (void *)wr.slot[1].h})
      if (p) cudaFreeHost(p);
    if (f_spec) snapi_f0_close(f_spec);
  }
  int chunk_len(int k) const {
    long long a = (long long)k * chunk, b = a + chunk;
    return (int)((b > npix ? npix : b) - a);
  }
  void reader() {
    std::vector<uint8_t> scratch;
    for (int k = 0; k < nchunk; ++k) {
      if (!rd.wait(k, false, nullptr)) return;
      Handoff::Slot &s = rd.slot[k & 1];
      s.p0 = (long long)k * chunk;
      s.n = chunk_len(k);
      double *dst = (double *)s.h;
      long long p = s.p0, end = s.p0 + s.n;
      while (p < end) {
        const long long x = p / ny, y = p % ny, i = p - s.p0;
        long long run = ny - y;
        if (run > end - p) run = end - p;
        for (int q = 0; q < 12; ++q) {  // element (q, x, y, z) at ((q * nx + x) * ny + y) * nd + z
          const long long first = ((q * (long long)nx_full + x0 + x) * ny_full + y0 + y) * nd;
          if (snapi_f0::read_range(fd, info, first, run * nd, dst + ((size_t)q * chunk + i) * nd, SNAPI_F0_FLOAT64,
                                   scratch)) {
            rd.fail(std::string("snapi_cube_synth: ") + snapi_f0_error());
            return;
          }
        }
        p += run;
      }
      bytes_read += (long long)s.n * 12 * nd * snapi_f0::type_size(info.type);
      rd.set(k, true);
    }
  }
  void writer() {
    const long long pix_elems = 4LL * nl;
    for (int k = 0; k < nchunk; ++k) {
      if (!wr.wait(k, true, nullptr)) return;
      Handoff::Slot &s = wr.slot[k & 1];
      if (f_spec && snapi_f0_write_at(f_spec, s.p0 * pix_elems, s.n * pix_elems, s.h)) {
        wr.fail(std::string("snapi_cube_synth: ") + snapi_f0_error());
        return;
      }
      if (f_spec) bytes_written += (long long)s.n * pix_elems * 8;
      wr.set(k, false);
    }
  }
};

}  // namespace

extern "C" int snapi_cube_synth(snapi_ctx *ctx, const snapi_cube_synth_job *job, snapi_cube_stats *stats) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  if (!job || !job->atmos_path) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: null argument");
  const auto t_start = Clock::now();
  SynthJob J;
  J.fd = open(job->atmos_path, O_RDONLY);
  if (J.fd < 0) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: cannot open %s", job->atmos_path);
  if (snapi_f0::parse(J.fd, &J.info)) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: %s", snapi_f0_error());
  const snapi_f0_info &I = J.info;
  if (I.ndim != 4 || I.dim[3] != 12)  // read_spinor3d: "does not have exactly 12 parameters"
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: the atmosphere cube must have dims (nd, ny, nx, 12)");
  if (I.type != SNAPI_F0_FLOAT32 && I.type != SNAPI_F0_FLOAT64)
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: data type of the cube is not floating point");
  if (I.compressed) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: compressed cube");
  J.nd = (int)I.dim[0];
  J.ny_full = (int)I.dim[1];
  J.nx_full = (int)I.dim[2];
  if (J.nd != ctx->nd)
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: the cube has %d depths, the context %d", J.nd, ctx->nd);
  const int xl = job->xl > 0 ? job->xl : 1, yl = job->yl > 0 ? job->yl : 1;
  // a range beyond the cube is cut to the cube, as the job reduces nx / ny to the model's (job.cc:391-398)
  const int xh = (job->xh > 0 && job->xh < J.nx_full) ? job->xh : J.nx_full;
  const int yh = (job->yh > 0 && job->yh < J.ny_full) ? job->yh : J.ny_full;
  if (xl > xh || yl > yh) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: empty subfield");
  J.x0 = xl - 1; J.y0 = yl - 1;
  J.nx = xh - xl + 1; J.ny = yh - yl + 1;
  J.nl = ctx->nl;
  J.npix = (long long)J.nx * J.ny;
  const bool nlte = job->ali != nullptr;
  if (nlte && (!job->ali_prob || !job->ali_tables || !job->line_level || job->ali_prob->nd != J.nd))
    return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: an NLTE atom needs its problem (the cube's depths), set-up "
                                      "tables and line levels");
  J.chunk = job->chunk > 0 ? job->chunk : (nlte ? 2048 : 16384);
  if (J.chunk > J.npix) J.chunk = (int)J.npix;
  J.nchunk = (int)((J.npix + J.chunk - 1) / J.chunk);
  const int C = J.chunk, nd = J.nd, nl = J.nl, nf = ctx->nfield;
  J.rows_bytes = (size_t)C * 12 * nd * sizeof(double);
  J.spec_bytes = (size_t)C * 4 * nl * sizeof(double);
  SNAPI_CK(cudaSetDevice(ctx->device));
  SNAPI_CK(cudaMalloc(&J.d_rows, J.rows_bytes));
  SNAPI_CK(cudaMalloc(&J.d_cols, J.rows_bytes));
  SNAPI_CK(cudaMalloc(&J.d_rec, sizeof(float) * (size_t)C * nd * nf));
  SNAPI_CK(cudaMalloc(&J.d_stokes, sizeof(float) * (size_t)C * nl * 4));
  SNAPI_CK(cudaMalloc(&J.d_spec, J.spec_bytes));
  SNAPI_CK(cudaMalloc(&J.d_st, sizeof(int) * (size_t)C));
  if (nlte) {  // the set-up's outputs in the layout of snapi_ali_columns, one block
    const snapi_ali_problem &P = *job->ali_prob;
    int nline = 0;
    for (int t = 0; t < P.ntrans; ++t) nline += P.cont_of[P.trans[2 * t]] != P.trans[2 * t + 1];
    const int nbf = P.ntrans - nline, nr = P.nray, nv = P.nlevel;
    const size_t sz[11] = {(size_t)nd, (size_t)nd, (size_t)nd, (size_t)nd, (size_t)nr * nd, (size_t)nline * nd,
                           (size_t)nline * nd, (size_t)nbf * nd, (size_t)nd * nv * nv, (size_t)nr * P.nlambda * nd,
                           (size_t)nr * P.nlambda * nd};
    size_t tot = 0;
    for (size_t v : sz) tot += v;
    SNAPI_CK(cudaMalloc(&J.d_ali, sizeof(double) * tot * C));
    double *q = J.d_ali;
    double **dst[11] = {&J.ali_out.T, &J.ali_out.ne, &J.ali_out.na, &J.ali_out.kappa, &J.ali_out.vray,
                        &J.ali_out.dld, &J.ali_out.adamp, &J.ali_out.bfratio, &J.ali_out.coll, &J.ali_out.bg_op,
                        &J.ali_out.bg_em};
    for (int i = 0; i < 11; ++i) {
      *dst[i] = q;
      q += sz[i] * C;
    }
    SNAPI_CK(cudaMalloc(&J.d_pops, sizeof(double) * (size_t)C * nd * nv));
    SNAPI_CK(cudaMalloc(&J.d_ast, sizeof(int) * (size_t)C));
  }
  for (int i = 0; i < 2; ++i) {
    SNAPI_CK(cudaHostAlloc((void **)&J.rd.slot[i].h, J.rows_bytes, cudaHostAllocDefault));
    SNAPI_CK(cudaHostAlloc((void **)&J.wr.slot[i].h, J.spec_bytes, cudaHostAllocDefault));
  }
  int st = SNAPI_OK;
  if (job->out_spectra) {
    const long long dims[4] = {nl, 4, J.ny, J.nx};
    J.f_spec = snapi_f0_create(job->out_spectra, SNAPI_F0_FLOAT64, 4, dims, nullptr, &st);
    if (!J.f_spec) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: %s", snapi_f0_error());
  }
  std::vector<int> hst(C);
  double read_wait = 0.0, write_wait = 0.0, ker_ms = 0.0, gpu_s = 0.0;
  long long flagged = 0;
  int launches = 0;
  std::thread t_rd([&] { J.reader(); }), t_wr([&] { J.writer(); });
  auto stop = [&](int code) {
    J.rd.fail(J.rd.err.empty() ? "stopped" : J.rd.err);
    J.wr.fail(J.wr.err.empty() ? "stopped" : J.wr.err);
    t_rd.join();
    t_wr.join();
    return code;
  };
#define SYN_CK(call)                                                                                   \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess)                                                                             \
      return stop(set_err(ctx, SNAPI_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)));                  \
  } while (0)
  for (int k = 0; k < J.nchunk; ++k) {
    if (!J.rd.wait(k, true, &read_wait)) {
      std::string e = J.rd.err;
      return stop(set_err(ctx, SNAPI_EINVAL, "%s", e.c_str()));
    }
    const long long p0 = (long long)k * C;
    const int n = J.chunk_len(k);
    const auto tg = Clock::now();
    SYN_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    SYN_CK(cudaMemcpyAsync(J.d_rows, J.rd.slot[k & 1].h, J.rows_bytes, cudaMemcpyHostToDevice, ctx->stream));
    k_cube_cols<<<grid_for((long long)n * 12 * nd), kThreads, 0, ctx->stream>>>(J.d_rows, n, C, nd, J.d_cols);
    SYN_CK(cudaGetLastError());
    SYN_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    SYN_CK(cudaEventSynchronize(ctx->ev1));
    float t = 0.f;
    SYN_CK(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    ker_ms += t;
    ++launches;
    J.rd.set(k, false);
    st = snapi_records_from_columns(ctx, n, J.d_cols, J.d_rec, J.d_st, SNAPI_MEM_DEVICE);
    if (st) return stop(st);
    ker_ms += ctx->last_ms;
    launches += ctx->last_launches;
    SYN_CK(cudaMemcpy(hst.data(), J.d_st, sizeof(int) * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i) {
      if (hst[i] & 8)
        return stop(set_err(ctx, SNAPI_EINVAL,
                            "snapi_cube_synth: the log tau row of pixel %lld is not the context's depth grid", p0 + i));
      if (hst[i]) ++flagged;
    }
    if (nlte) {  // nltepops of the chunk's columns, then the NLTE atom's line fields
      k_cube_floor_T<<<grid_for((long long)n * nd), kThreads, 0, ctx->stream>>>(J.d_cols, n, nd);
      SYN_CK(cudaGetLastError());
      ++launches;
      st = snapi_ali_setup(ctx, job->ali_prob, job->ali_tables, n, J.d_cols, &J.ali_out, J.d_pops, J.d_ast,
                           SNAPI_MEM_DEVICE);
      if (st) return stop(st);
      ker_ms += ctx->last_ms;
      launches += ctx->last_launches;
      std::vector<int> sst(n);  // the set-up's chemistry flags (cap, non-finite)
      SYN_CK(cudaMemcpy(sst.data(), J.d_ast, sizeof(int) * n, cudaMemcpyDeviceToHost));
      const snapi_ali_columns ac = {J.ali_out.T,    J.ali_out.ne,      J.ali_out.na,    J.ali_out.kappa,
                                    J.ali_out.vray, J.ali_out.dld,     J.ali_out.adamp, J.ali_out.bfratio,
                                    J.ali_out.coll, J.ali_out.bg_op,   J.ali_out.bg_em};
      st = snapi_ali_iter(job->ali, n, &ac, J.d_pops, job->ali_max_iter > 0 ? job->ali_max_iter : 100,
                          job->ali_tol > 0.0 ? job->ali_tol : 1e-2, nullptr, nullptr, J.d_ast, SNAPI_MEM_DEVICE);
      if (st) return stop(set_err(ctx, st, "snapi_cube_synth: %s", snapi_ali_last_error(job->ali)));
      ker_ms += snapi_ali_last_kernel_ms(job->ali);
      std::vector<int> ast(n);  // the iteration's: -1 populations that stayed negative
      SYN_CK(cudaMemcpy(ast.data(), J.d_ast, sizeof(int) * n, cudaMemcpyDeviceToHost));
      for (int i = 0; i < n; ++i)  // hst: the records' flags, counted above
        if (hst[i] == 0 && (sst[i] != 0 || ast[i] < 0)) ++flagged;
      st = snapi_records_set_populations(ctx, n, J.d_rec, J.d_pops, job->ali_prob->nlevel, job->line_level,
                                         SNAPI_MEM_DEVICE);
      if (st) return stop(st);
      launches += ctx->last_launches;
    }
    st = snapi_synth(ctx, n, J.d_rec, J.d_stokes, SNAPI_MEM_DEVICE);
    if (st) return stop(st);
    ker_ms += ctx->last_ms;
    launches += ctx->last_launches;
    if (job->stokes)
      SYN_CK(cudaMemcpy(job->stokes + (size_t)p0 * nl * 4, J.d_stokes, sizeof(float) * (size_t)n * nl * 4,
                        cudaMemcpyDeviceToHost));
    if (!J.wr.wait(k, false, &write_wait)) {
      std::string e = J.wr.err;
      return stop(set_err(ctx, SNAPI_EINVAL, "%s", e.c_str()));
    }
    Handoff::Slot &ws = J.wr.slot[k & 1];
    SYN_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    k_cube_spectra<<<grid_for((long long)n * nl * 4), kThreads, 0, ctx->stream>>>(J.d_stokes, n, nl, J.d_spec);
    SYN_CK(cudaGetLastError());
    SYN_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ++launches;
    SYN_CK(cudaMemcpyAsync(ws.h, J.d_spec, sizeof(double) * (size_t)n * 4 * nl, cudaMemcpyDeviceToHost, ctx->stream));
    SYN_CK(cudaStreamSynchronize(ctx->stream));
    SYN_CK(cudaEventElapsedTime(&t, ctx->ev0, ctx->ev1));
    ker_ms += t;
    gpu_s += secs(tg, Clock::now());
    ws.p0 = p0;
    ws.n = n;
    J.wr.set(k, true);
  }
#undef SYN_CK
  {
    const auto tw = Clock::now();
    std::unique_lock<std::mutex> lk(J.wr.mu);
    J.wr.cv.wait(lk, [&] { return J.wr.abort || (!J.wr.slot[0].full && !J.wr.slot[1].full); });
    write_wait += secs(tw, Clock::now());
  }
  t_rd.join();
  t_wr.join();
  if (!J.wr.err.empty()) return set_err(ctx, SNAPI_EINVAL, "%s", J.wr.err.c_str());
  if (!J.rd.err.empty()) return set_err(ctx, SNAPI_EINVAL, "%s", J.rd.err.c_str());
  if (J.f_spec) {
    snapi_f0_file *f = J.f_spec;
    J.f_spec = nullptr;
    if (snapi_f0_close(f)) return set_err(ctx, SNAPI_EINVAL, "snapi_cube_synth: %s", snapi_f0_error());
  }
  ctx->last_ms = ker_ms;
  ctx->last_launches = launches;
  if (stats) {
    stats->pixels = J.npix;
    stats->chunks = J.nchunk;
    stats->lm_steps = 0;
    stats->wall_s = secs(t_start, Clock::now());
    stats->fit_s = gpu_s;
    stats->read_wait_s = read_wait;
    stats->write_wait_s = write_wait;
    stats->bytes_read = J.bytes_read;
    stats->bytes_written = J.bytes_written;
    stats->kernel_ms = ker_ms;
    stats->launches = launches;
    stats->flagged = flagged;
  }
  return SNAPI_OK;
}
