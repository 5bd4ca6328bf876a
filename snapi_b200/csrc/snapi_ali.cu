// snapi_ali.cu -- NLTE level populations by accelerated lambda iteration for many 1-D columns
// (atmosphere::nltepops, atmos/atmos_pop.cc:67-240), one NLTE atom.
//
// Per iteration:
//   k_ali_formal  CTA = (column, ray, 64 wavelengths), thread = wavelength: background + active
//                 opacity / emissivity at every depth (W4 profiles of every bound-bound
//                 transition, bound-free with the LTE-ratio correction), scalar formal solution
//                 along the ray with the diagonal operator (atmos_ppbez_rts.cc:21-219); writes
//                 I, Lambda* and the total opacity per depth.  Profiles in FP32; opacity sums,
//                 optical depths and the recursion in FP64: the NLTE grid's background spans
//                 1e-13 .. 1e32 cm^-1 (1e45 after normalisation by kappa_500, beyond FP32) and
//                 the rates use J - Lambda* S, which cancels in optically thick line cores.
//   k_ali_rates   CTA = column, thread = depth: walks every (ray, wavelength) and sums the
//                 profile-weighted mean intensities and operators of every transition in FP64
//                 registers (atom::add, atom.cc:1865-1927), then the rate equations of its depth
//                 (atom::newpops, atom_pop.cc:27-145) in FP64 with the most populated level
//                 replaced by conservation, an LU solve, the relative change; negative
//                 populations anywhere in the column -> the same step without the operator; the
//                 column stops when the maximum relative change falls below tol.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "snapi_internal.cuh"

using namespace snapi;

namespace {

constexpr int kAliChunk = 64;
constexpr int kAliMaxLev = 16, kAliMaxLine = 32, kAliMaxBf = 16;
constexpr double kHc = kH * kC;
constexpr double kPi4 = 4.0 * kPi;
constexpr double kInvPi4 = 1.0 / kPi4, kInvHc = 1.0 / kHc;

struct AliDev {
  int ncol, nd, nl, nray, nlev, nline, nbf, nchunk;
  int nsl;  // k_ali_rates: wavelength slices per depth (adjacent lanes; a power of two <= 32)
  double tol;
  int max_iter;
  // problem
  const double *grid, *lambda, *lw, *ray_ct, *ray_w;
  const float *fudge;                           // [nl]
  const double *lam0, *Aul, *Blu, *Bul, *Eline; // [nline]
  const int *line_lo, *line_up;                 // [nline]
  const int *bf_lo, *bf_up;                     // [nbf]
  const float *sigma;                           // [nbf][nl]
  const double *A, *B;                          // [nlev][nlev]
  const int *stage, *cont_of, *tmap, *bf_of;    // [nlev], [nlev], [nlev][nlev], [nlev]
  // columns
  const double *T, *ne, *na, *kap, *vray, *dld, *adamp, *bfratio, *coll;
  const double *bgop, *bgem;
  double *pops;                                 // [ncol][nd][nlev]
  double *I, *L, *opp;                          // [ncol][nray][nl][nd]
  int *state, *iters;                           // [ncol]: state 0 running, 1 converged, 2 max_iter, -1 negative
  double *rel;                                  // [ncol]
};

struct FormalSmem {
  size_t kap, T, vr, idld, a, lop, lem, ni, ncr, total;
};
__host__ __device__ inline FormalSmem formal_smem(int nd, int nline, int nbf) {
  FormalSmem s;
  size_t o = 0;
  auto f = [&](size_t n) { const size_t r = o; o = align_up(o + sizeof(float) * n, 16); return r; };
  auto g = [&](size_t n) { const size_t r = o; o = align_up(o + sizeof(double) * n, 16); return r; };
  s.kap = f(nd); s.T = f(nd); s.vr = f(nd);
  s.idld = f((size_t)nline * nd); s.a = f((size_t)nline * nd); s.lop = f((size_t)nline * nd); s.lem = f((size_t)nline * nd);
  s.ni = g((size_t)nbf * nd); s.ncr = g((size_t)nbf * nd);
  s.total = o;
  return s;
}

__global__ void __launch_bounds__(kAliChunk) k_ali_formal(AliDev D) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int chunk = blockIdx.x % D.nchunk;
  const int ray = (blockIdx.x / D.nchunk) % D.nray;
  const int col = blockIdx.x / (D.nchunk * D.nray);
  if (D.state[col] != 0) return;  // CTA-uniform
  const FormalSmem S = formal_smem(D.nd, D.nline, D.nbf);
  float *kap = reinterpret_cast<float *>(smem + S.kap), *Tz = reinterpret_cast<float *>(smem + S.T);
  float *vr = reinterpret_cast<float *>(smem + S.vr);
  float *idld = reinterpret_cast<float *>(smem + S.idld), *ad = reinterpret_cast<float *>(smem + S.a);
  float *lop = reinterpret_cast<float *>(smem + S.lop), *lem = reinterpret_cast<float *>(smem + S.lem);
  double *ni = reinterpret_cast<double *>(smem + S.ni), *ncr = reinterpret_cast<double *>(smem + S.ncr);
  const int nd = D.nd;
  const double *pc = D.pops + (size_t)col * nd * D.nlev;
  for (int z = threadIdx.x; z < nd; z += blockDim.x) {
    kap[z] = (float)D.kap[(size_t)col * nd + z];
    Tz[z] = (float)D.T[(size_t)col * nd + z];
    vr[z] = (float)(D.vray[((size_t)col * D.nray + ray) * nd + z] / kC);
    const double *n = pc + (size_t)z * D.nlev;
    for (int k = 0; k < D.nline; ++k) {
      const double dl = D.dld[((size_t)col * D.nline + k) * nd + z];
      idld[k * nd + z] = (float)(1.0 / dl);
      ad[k * nd + z] = (float)D.adamp[((size_t)col * D.nline + k) * nd + z];
      lop[k * nd + z] = (float)(n[D.line_lo[k]] * D.Blu[k] - n[D.line_up[k]] * D.Bul[k]);
      lem[k * nd + z] = (float)(n[D.line_up[k]] * D.Aul[k]);
    }
    for (int b = 0; b < D.nbf; ++b) {
      ni[b * nd + z] = n[D.bf_lo[b]];
      ncr[b * nd + z] = n[D.bf_up[b]] * D.bfratio[((size_t)col * D.nbf + b) * nd + z];
    }
  }
  __syncthreads();
  const int l = chunk * kAliChunk + threadIdx.x;
  if (l >= D.nl) return;  // no barrier below
  const double lam = D.lambda[l];
  const float lamf = (float)lam;
  const double hc4pl = kHc / (kPi4 * lam), xpl = kHc / (lam * kK), pl5 = 2.0 * kHc * kC / (lam * lam * lam * lam * lam);
  float dl[kAliMaxLine];
  double sg[kAliMaxBf];
  for (int k = 0; k < D.nline; ++k) dl[k] = (float)(D.lam0[k] - lam);
  for (int b = 0; b < D.nbf; ++b) sg[b] = (double)D.sigma[(size_t)b * D.nl + l] * (double)D.fudge[l];
  const size_t row = (((size_t)col * D.nray + ray) * D.nl + l) * nd;
  const double *bo = D.bgop + row, *be = D.bgem + row;
  auto cell = [&](int z, double &oo, double &ee, double &op) {
    double o = bo[z], e = be[z];
    for (int k = 0; k < D.nline; ++k) {
      const float iv = idld[k * nd + z];
      float H, F;
      voigt((dl[k] - lamf * vr[z]) * iv, ad[k * nd + z], H, F);
      const double phi = (double)(H * iv) * hc4pl;
      o += phi * (double)lop[k * nd + z];
      e += phi * (double)lem[k * nd + z];
    }
    if (D.nbf) {
      const double x = xpl / (double)Tz[z];
      const double eb = exp(-x), pl = pl5 / (exp(x) - 1.0);
      for (int b = 0; b < D.nbf; ++b) {
        o += sg[b] * (ni[b * nd + z] - ncr[b * nd + z] * eb);
        e += sg[b] * ncr[b * nd + z] * (1.0 - eb) * pl;
      }
    }
    op = o;
    const double ik = 1.0 / (double)kap[z];
    oo = o * ik;
    ee = e * ik;
  };
  double *Io = D.I + row, *Lo = D.L + row, *Oo = D.opp + row;
  const double ct = D.ray_ct[ray];
  const int dz = ct > 0.0 ? 1 : -1, zl = ct > 0.0 ? 0 : nd - 1, zh = ct > 0.0 ? nd - 1 : 0;
  const double mct = -ct;
  // window: p (z - dz), c (z), n (z + dz)
  // each cell's source function and each interval's length once: the window carries them
  double oop, eep, opp_, ooc, eec, opc, oon = 0.0, een = 0.0, opn = 0.0;
  cell(zl, oop, eep, opp_);
  cell(zl + dz, ooc, eec, opc);
  double sp = eep / oop, sc = eec / ooc, sn = 0.0;
  double hz = (D.grid[zl + dz] - D.grid[zl]) / mct, hn = 0.0;
  double dprev = (ooc - oop) / hz;
  double I = ct > 0.0 ? 0.0 : sp;
  Io[zl] = I;
  Lo[zl] = ct > 0.0 ? 0.0 : 1.0;
  Oo[zl] = opp_;
  for (int z = zl + dz;; z += dz) {
    double dcur;
    if (z == zh) {
      dcur = (ooc - oop) / hz;
    } else {
      cell(z + dz, oon, een, opn);
      sn = een / oon;
      hn = (D.grid[z + dz] - D.grid[z]) / mct;
      dcur = opd_interior(oop, ooc, oon, hz, hn);
    }
    const double tb = bezier_dtau(oop, ooc, dprev, dcur, hz);
    // linear weights with the Taylor branch below 1e-2 (atmos_ppbez_rts.cc:1070-1096 scalar form)
    double w0, w1, etb;
    if (tb < 1e-2) {
      etb = 1.0 - tb + tb * tb * 0.5 - tb * tb * tb / 6.0;
      w0 = tb * (0.5 - tb * (1.0 / 3.0 - tb / 8.0));
      w1 = 0.5 * tb * (1.0 - tb / 3.0 * (1.0 - tb / 4.0));
    } else {
      etb = exp(-tb);
      const double itb = 1.0 / tb;
      w0 = itb - etb * (1.0 + itb);
      w1 = 1.0 - itb + etb * itb;
    }
    I = I * etb + w0 * sp + w1 * sc;
    Io[z] = I;
    Lo[z] = w1;
    Oo[z] = opc;
    if (z == zh) break;
    oop = ooc; opp_ = opc; sp = sc;
    ooc = oon; opc = opn; sc = sn;
    hz = hn;
    dprev = dcur;
  }
}

// radiative rate from level `from` to `to` of one stage (atom_rad.cc:1732-1756 / 1726-1729)
__device__ double rad_rate(const AliDev &D, int from, int to, double JJ, double LL, double nf, double nt, bool alo) {
  const double a = D.A[from * D.nlev + to], b = D.B[from * D.nlev + to];
  if (!alo) return a + b * JJ;
  if (to == from) return 0.0;
  int u, lo;
  double nu, nl;
  if (to > from) { u = to; lo = from; nu = nt; nl = nf; }
  else { u = from; lo = to; nu = nf; nl = nt; }
  const double sl = nu * D.A[u * D.nlev + lo] / (nl * D.B[lo * D.nlev + u] - nu * D.B[u * D.nlev + lo]);
  return a * (1.0 - LL) + b * (JJ - LL * sl);
}

// rate equations of one depth and their solution (atom_pop.cc:27-145); returns false if singular
__device__ bool solve_rates(const AliDev &D, const double *n, const double *coll, double Tz, double nez, double naz,
                            const double *Jl, const double *Ll, const double *nrm, const double *Jbu,
                            const double *Jbd, const double *bfr, bool alo, double *out) {
  const int m = D.nlev;
  double M[kAliMaxLev * kAliMaxLev], b[kAliMaxLev];
  for (int i = 0; i < m * m; ++i) M[i] = 0.0;
  for (int i = 0; i < m; ++i) b[i] = 0.0;
  for (int i = 0; i < m - 1; ++i) {
    for (int j = 0; j < m; ++j) {
      if (D.stage[j] != D.stage[i]) continue;
      const int k = D.tmap[i * m + j];
      const double JJ = k >= 0 ? Jl[k] / nrm[k] : -1.0;
      const double LL = k >= 0 ? Ll[k] / nrm[k] : 0.0;
      M[i * m + i] -= rad_rate(D, i, j, JJ, LL, n[i], n[j], alo) + coll[i * m + j];
      M[i * m + j] += rad_rate(D, j, i, JJ, LL, n[j], n[i], alo) + coll[j * m + i];
    }
    const int c = D.cont_of[i];
    if (c >= 0) {
      const int bb = D.bf_of[i];
      const double up = Jbu[bb] + coll[i * m + c];
      M[i * m + i] -= up;
      M[c * m + i] += up;
      const double down = Jbd[bb] * bfr[bb] + coll[c * m + i];  // every continuum has a bf transition
      M[i * m + c] += down;
      M[c * m + c] -= down;
    }
  }
  int rep = m - 1;
  double maxpop = n[rep];
  for (int i = 0; i < m - 1; ++i)
    if (n[i] > maxpop) { maxpop = n[i]; rep = i; }
  for (int j = 0; j < m; ++j) M[rep * m + j] = 1.0;
  b[rep] = naz;
  // LU without pivoting (Crout) and the two triangular solves
  for (int p = 0; p < m; ++p) {
    for (int i = p; i < m; ++i) {
      double s = M[i * m + p];
      for (int q = 0; q < p; ++q) s -= M[i * m + q] * M[q * m + p];
      M[i * m + p] = s;
    }
    if (M[p * m + p] == 0.0) return false;
    for (int j = p + 1; j < m; ++j) {
      double s = M[p * m + j];
      for (int q = 0; q < p; ++q) s -= M[p * m + q] * M[q * m + j];
      M[p * m + j] = s / M[p * m + p];
    }
  }
  for (int i = 0; i < m; ++i) {
    double s = b[i];
    for (int q = 0; q < i; ++q) s -= M[i * m + q] * out[q];
    out[i] = s / M[i * m + i];
  }
  for (int i = m - 1; i >= 0; --i) {
    double s = out[i];
    for (int q = i + 1; q < m; ++q) s -= M[i * m + q] * out[q];
    out[i] = s;
  }
  (void)Tz; (void)nez;
  return true;
}

__global__ void k_ali_rates(AliDev D) {
  __shared__ int s_neg;
  __shared__ double s_max;
  // thread = (depth, wavelength slice): the nsl lanes of a depth take every nsl-th wavelength and
  // their sums meet by shuffles, so a column's CTA keeps nsl times the warps in flight
  const int col = blockIdx.x, sl = threadIdx.x % D.nsl, z = threadIdx.x / D.nsl, nd = D.nd, m = D.nlev;
  const bool lead = sl == 0;
  if (D.state[col] != 0) return;  // CTA-uniform
  if (threadIdx.x == 0) { s_neg = 0; s_max = 0.0; }
  __syncthreads();
  const bool valid = z < nd;
  const int zz = valid ? z : nd - 1;
  double n[kAliMaxLev], nn[kAliMaxLev];
  double *pz = D.pops + ((size_t)col * nd + zz) * m;
  for (int i = 0; i < m; ++i) n[i] = pz[i];
  const double Tz = D.T[(size_t)col * nd + zz], nez = D.ne[(size_t)col * nd + zz], naz = D.na[(size_t)col * nd + zz];
  double Jl[kAliMaxLine], Ll[kAliMaxLine], nrm[kAliMaxLine], Jbu[kAliMaxBf], Jbd[kAliMaxBf], bfr[kAliMaxBf];
  double lfac[kAliMaxLine];
  float iv[kAliMaxLine], av[kAliMaxLine];
  for (int k = 0; k < D.nline; ++k) {
    Jl[k] = Ll[k] = nrm[k] = 0.0;
    iv[k] = (float)(1.0 / D.dld[((size_t)col * D.nline + k) * nd + zz]);
    av[k] = (float)D.adamp[((size_t)col * D.nline + k) * nd + zz];
    lfac[k] = (n[D.line_lo[k]] * D.Blu[k] - n[D.line_up[k]] * D.Bul[k]) * D.Eline[k] / kPi4;
  }
  for (int b = 0; b < D.nbf; ++b) {
    Jbu[b] = Jbd[b] = 0.0;
    bfr[b] = D.bfratio[((size_t)col * D.nbf + b) * nd + zz];
  }
  const double hckT = kHc / (kK * Tz);
  for (int r = 0; r < D.nray; ++r) {
    const float vrc = (float)(D.vray[((size_t)col * D.nray + r) * nd + zz] / kC);
    const double wr = D.ray_w[r];
    const size_t base = ((size_t)col * D.nray + r) * D.nl * nd + zz;
    // FP64 divisions hoisted: one reciprocal of the opacity and of lambda per (ray, wavelength), the
    // constant ones folded (the sums move by rounding only)
    for (int l = sl; l < D.nl; l += D.nsl) {
      const double I = D.I[base + (size_t)l * nd], Ls = D.L[base + (size_t)l * nd], op = D.opp[base + (size_t)l * nd];
      const double lam = D.lambda[l], w = D.lw[l] * wr, iop = 1.0 / op, wq = w * kInvPi4;
      const float lamf = (float)lam;
      for (int k = 0; k < D.nline; ++k) {
        float H, F;
        voigt(((float)(D.lam0[k] - lam) - lamf * vrc) * iv[k], av[k], H, F);
        const double phi = (double)(H * iv[k]);
        const double wp = wq * phi;
        const double lf = lfac[k] * phi * iop;
        nrm[k] += wp;
        Jl[k] += wp * I * lf;
        Ll[k] += wp * Ls * lf;
      }
      if (D.nbf) {
        const double il = 1.0 / lam, il2 = il * il;
        const double e = exp(-hckT * il);
        const double p5 = 2.0 * kHc * kC * (il2 * il2 * il);
        const double wl = w * lam * kInvHc;
        for (int b = 0; b < D.nbf; ++b) {
          const double s = wl * (double)D.sigma[(size_t)b * D.nl + l];
          Jbu[b] += s * I;
          Jbd[b] += s * (I + p5) * e;
        }
      }
    }
  }
  for (int off = 1; off < D.nsl; off <<= 1) {  // every lane of the depth ends with the totals
    for (int k = 0; k < D.nline; ++k) {
      Jl[k] += __shfl_xor_sync(0xffffffffu, Jl[k], off);
      Ll[k] += __shfl_xor_sync(0xffffffffu, Ll[k], off);
      nrm[k] += __shfl_xor_sync(0xffffffffu, nrm[k], off);
    }
    for (int b = 0; b < D.nbf; ++b) {
      Jbu[b] += __shfl_xor_sync(0xffffffffu, Jbu[b], off);
      Jbd[b] += __shfl_xor_sync(0xffffffffu, Jbd[b], off);
    }
  }
  const double *cz = D.coll + ((size_t)col * nd + zz) * m * m;
  // step with the local operator; negative populations anywhere -> without it (atmos_pop.cc:185-205)
  double rmax = 0.0;
  int neg = 0;
  bool ok = solve_rates(D, n, cz, Tz, nez, naz, Jl, Ll, nrm, Jbu, Jbd, bfr, true, nn);
  for (int i = 0; i < m; ++i) {
    const double rc = nn[i] / n[i] - 1.0;
    if (!(rc >= -1.0)) neg = 1;
    rmax = fmax(rmax, fabs(rc));
  }
  if (!ok) neg = 1;
  if (valid && lead && neg) atomicOr(&s_neg, 1);
  __syncthreads();
  int negative = s_neg;
  __syncthreads();
  if (negative) {
    if (threadIdx.x == 0) s_neg = 0;
    __syncthreads();
    ok = solve_rates(D, n, cz, Tz, nez, naz, Jl, Ll, nrm, Jbu, Jbd, bfr, false, nn);
    neg = ok ? 0 : 1;
    rmax = 0.0;
    for (int i = 0; i < m; ++i) {
      const double rc = nn[i] / n[i] - 1.0;
      if (!(rc >= -1.0)) neg = 1;
      rmax = fmax(rmax, fabs(rc));
    }
    if (valid && lead && neg) atomicOr(&s_neg, 1);
    __syncthreads();
    negative = s_neg;
  }
  if (negative) {  // stays negative: the column stops without updating (outcome -1)
    if (threadIdx.x == 0) { D.state[col] = -1; D.iters[col] += 1; }
    return;
  }
  if (valid && lead) {
    for (int i = 0; i < m; ++i) pz[i] = nn[i];
    // max of non-negative doubles through their bit patterns
    atomicMax(reinterpret_cast<unsigned long long *>(&s_max), __double_as_longlong(rmax));
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double r = s_max;
    D.rel[col] = r;
    D.iters[col] += 1;
    if (r < D.tol) D.state[col] = 1;
    else if (D.iters[col] >= D.max_iter) D.state[col] = 2;
  }
}

}  // namespace

struct snapi_ali_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int nd = 0, nl = 0, nray = 0, nlev = 0, ntr = 0, nline = 0, nbf = 0, nchunk = 0;
  std::vector<void *> bufs;  // problem constants
  AliDev D;
  // column work buffers (capacity cap columns)
  int cap = 0;
  double *d_T = nullptr, *d_ne = nullptr, *d_na = nullptr, *d_kap = nullptr, *d_vray = nullptr, *d_dld = nullptr,
         *d_adamp = nullptr, *d_bfr = nullptr, *d_coll = nullptr, *d_pops = nullptr, *d_rel = nullptr;
  double *d_bgop = nullptr, *d_bgem = nullptr, *d_I = nullptr, *d_L = nullptr, *d_opp = nullptr;
  int *d_state = nullptr, *d_iters = nullptr;
  double last_ms = 0.0;
  std::string err;
};

namespace {

int ali_err(snapi_ali_ctx *c, int code, const char *msg) {
  if (c) c->err = msg;
  return code;
}

template <class T>
T *upload(snapi_ali_ctx *c, const T *h, size_t n) {
  T *d = nullptr;
  if (cudaMalloc(&d, sizeof(T) * (n ? n : 1)) != cudaSuccess) return nullptr;
  c->bufs.push_back(d);
  if (n && cudaMemcpy(d, h, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
  return d;
}

void free_cols(snapi_ali_ctx *c) {
  void *b[] = {c->d_T, c->d_ne, c->d_na, c->d_kap, c->d_vray, c->d_dld, c->d_adamp, c->d_bfr, c->d_coll,
               c->d_pops, c->d_rel, c->d_bgop, c->d_bgem, c->d_I, c->d_L, c->d_opp, c->d_state, c->d_iters};
  for (void *x : b)
    if (x) cudaFree(x);
  c->d_T = c->d_ne = c->d_na = c->d_kap = c->d_vray = c->d_dld = c->d_adamp = c->d_bfr = c->d_coll = nullptr;
  c->d_pops = c->d_rel = nullptr;
  c->d_bgop = c->d_bgem = c->d_I = c->d_L = c->d_opp = nullptr;
  c->d_state = c->d_iters = nullptr;
  c->cap = 0;
}

}  // namespace

extern "C" {

snapi_ali_ctx *snapi_ali_create(const snapi_ali_problem *p, int device, int *status) {
  auto fail = [&](snapi_ali_ctx *c, int code) -> snapi_ali_ctx * {
    if (status) *status = code;
    if (c) { fprintf(stderr, "snapi_ali_create: %s\n", c->err.c_str()); snapi_ali_destroy(c); }
    return nullptr;
  };
  if (!p) return fail(nullptr, SNAPI_EINVAL);
  snapi_ali_ctx *c = new snapi_ali_ctx();
  c->device = device;
  if (p->nd < 3 || p->nlambda < 1 || p->nray < 1 || p->nlevel < 2 || p->nlevel > kAliMaxLev || p->ntrans < 1 ||
      !p->grid || !p->lambda || !p->lambda_w || !p->fudge || !p->ray_theta || !p->ray_w || !p->trans || !p->line_c ||
      !p->line_e || !p->A || !p->B || !p->stage || !p->cont_of || !p->sigma) {
    ali_err(c, SNAPI_EINVAL, "invalid ALI problem");
    return fail(c, SNAPI_EINVAL);
  }
  const int m = p->nlevel;
  std::vector<int> llo, lup, blo, bup, tmap(m * m, -1), bfof(m, -1), lineof(p->ntrans, -1), bfidx(p->ntrans, -1);
  std::vector<double> lam0, aul, blu, bul, eline;
  for (int t = 0; t < p->ntrans; ++t) {
    const int lo = p->trans[2 * t], up = p->trans[2 * t + 1];
    if (lo < 0 || lo >= m || up < 0 || up >= m || lo == up) {
      ali_err(c, SNAPI_EINVAL, "transition levels out of range");
      return fail(c, SNAPI_EINVAL);
    }
    if (p->cont_of[lo] == up) {
      bfof[lo] = (int)blo.size();
      bfidx[t] = (int)blo.size();
      blo.push_back(lo); bup.push_back(up);
    } else {
      const int k = (int)llo.size();
      tmap[lo * m + up] = tmap[up * m + lo] = k;
      lineof[t] = k;
      llo.push_back(lo); lup.push_back(up);
      lam0.push_back(p->line_c[4 * t]); aul.push_back(p->line_c[4 * t + 1]);
      blu.push_back(p->line_c[4 * t + 2]); bul.push_back(p->line_c[4 * t + 3]);
      eline.push_back(p->line_e[t]);
    }
  }
  for (int i = 0; i < m; ++i)
    if (p->cont_of[i] >= m || (p->cont_of[i] >= 0 && bfof[i] < 0)) {
      ali_err(c, SNAPI_EINVAL, "every level with a continuum needs its bound-free transition");
      return fail(c, SNAPI_EINVAL);
    }
  if ((int)llo.size() > kAliMaxLine || (int)blo.size() > kAliMaxBf) {
    ali_err(c, SNAPI_EINVAL, "too many transitions (lines <= 32, bound-free <= 16)");
    return fail(c, SNAPI_EINVAL);
  }
  c->nd = p->nd; c->nl = p->nlambda; c->nray = p->nray; c->nlev = m; c->ntr = p->ntrans;
  c->nline = (int)llo.size(); c->nbf = (int)blo.size();
  c->nchunk = (p->nlambda + kAliChunk - 1) / kAliChunk;
  const FormalSmem S = formal_smem(c->nd, c->nline, c->nbf);
  if (S.total > 200 * 1024) {
    ali_err(c, SNAPI_EINVAL, "too many depths x transitions for one CTA's shared memory");
    return fail(c, SNAPI_EINVAL);
  }
  if (p->nd > 1024) { ali_err(c, SNAPI_EINVAL, "nd > 1024"); return fail(c, SNAPI_EINVAL); }
  if (cudaSetDevice(device) != cudaSuccess) { ali_err(c, SNAPI_ECUDA, "cudaSetDevice failed"); return fail(c, SNAPI_ECUDA); }
  int maxsm = 0;
  std::vector<double> ct(p->nray);
  for (int r = 0; r < p->nray; ++r) ct[r] = cos(p->ray_theta[r]);
  std::vector<float> fud(p->fudge, p->fudge + p->nlambda), sig((size_t)c->nbf * p->nlambda);
  for (int t = 0; t < p->ntrans; ++t)
    if (bfidx[t] >= 0)
      for (int l = 0; l < p->nlambda; ++l) sig[(size_t)bfidx[t] * p->nlambda + l] = (float)p->sigma[(size_t)t * p->nlambda + l];
  AliDev &D = c->D;
  memset(&D, 0, sizeof D);
  D.nd = c->nd; D.nl = c->nl; D.nray = c->nray; D.nlev = m; D.nline = c->nline; D.nbf = c->nbf; D.nchunk = c->nchunk;
  D.nsl = c->nd <= 256 ? 4 : (c->nd <= 512 ? 2 : 1);  // nd * nsl <= 1024 threads per CTA
  bool ok = (D.grid = upload(c, p->grid, p->nd)) && (D.lambda = upload(c, p->lambda, p->nlambda)) &&
            (D.lw = upload(c, p->lambda_w, p->nlambda)) && (D.ray_ct = upload(c, ct.data(), ct.size())) &&
            (D.ray_w = upload(c, p->ray_w, p->nray)) && (D.fudge = upload(c, fud.data(), fud.size())) &&
            (D.lam0 = upload(c, lam0.data(), lam0.size())) && (D.Aul = upload(c, aul.data(), aul.size())) &&
            (D.Blu = upload(c, blu.data(), blu.size())) && (D.Bul = upload(c, bul.data(), bul.size())) &&
            (D.Eline = upload(c, eline.data(), eline.size())) && (D.line_lo = upload(c, llo.data(), llo.size())) &&
            (D.line_up = upload(c, lup.data(), lup.size())) && (D.bf_lo = upload(c, blo.data(), blo.size())) &&
            (D.bf_up = upload(c, bup.data(), bup.size())) && (D.sigma = upload(c, sig.data(), sig.size())) &&
            (D.A = upload(c, p->A, (size_t)m * m)) && (D.B = upload(c, p->B, (size_t)m * m)) &&
            (D.stage = upload(c, p->stage, m)) && (D.cont_of = upload(c, p->cont_of, m)) &&
            (D.tmap = upload(c, tmap.data(), tmap.size())) && (D.bf_of = upload(c, bfof.data(), bfof.size()));
  if (!ok) { ali_err(c, SNAPI_ENOMEM, "device allocation failed"); return fail(c, SNAPI_ENOMEM); }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      // the limit is per device and shared by every ALI context: the opt-in maximum, not this
      // problem's size, so a smaller context never lowers it under a larger one
      cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
      cudaFuncSetAttribute(k_ali_formal, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm) != cudaSuccess) {
    ali_err(c, SNAPI_ECUDA, "stream / event / attribute set-up failed");
    return fail(c, SNAPI_ECUDA);
  }
  if (status) *status = SNAPI_OK;
  return c;
}

void snapi_ali_destroy(snapi_ali_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_cols(c);
  for (void *b : c->bufs) cudaFree(b);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

const char *snapi_ali_last_error(const snapi_ali_ctx *c) { return c ? c->err.c_str() : "null context"; }
double snapi_ali_last_kernel_ms(const snapi_ali_ctx *c) { return c ? c->last_ms : 0.0; }

int snapi_ali_iter(snapi_ali_ctx *c, int ncol, const snapi_ali_columns *in, double *pops, int max_iter, double tol,
                   double *rel_change, int *iters, int *status, int mem) {
  if (!c) return SNAPI_EINVAL;
  if (ncol < 1 || !in || !pops || max_iter < 1 || !(tol > 0.0) || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE) ||
      !in->T || !in->ne || !in->na || !in->kappa || !in->vray || (c->nline && (!in->dld || !in->adamp)) ||
      (c->nbf && !in->bfratio) || !in->coll || !in->bg_op || !in->bg_em)
    return ali_err(c, SNAPI_EINVAL, "snapi_ali_iter: invalid arguments");
#define ACK(call)                                                                         \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) return ali_err(c, SNAPI_ECUDA, cudaGetErrorString(e_));         \
  } while (0)
  ACK(cudaSetDevice(c->device));
  const size_t nd = c->nd, nl = c->nl, nr = c->nray, m = c->nlev, C = ncol;
  if (c->cap < ncol) {
    free_cols(c);
    ACK(cudaMalloc(&c->d_T, sizeof(double) * C * nd));
    ACK(cudaMalloc(&c->d_ne, sizeof(double) * C * nd));
    ACK(cudaMalloc(&c->d_na, sizeof(double) * C * nd));
    ACK(cudaMalloc(&c->d_kap, sizeof(double) * C * nd));
    ACK(cudaMalloc(&c->d_vray, sizeof(double) * C * nr * nd));
    ACK(cudaMalloc(&c->d_dld, sizeof(double) * C * (c->nline ? c->nline : 1) * nd));
    ACK(cudaMalloc(&c->d_adamp, sizeof(double) * C * (c->nline ? c->nline : 1) * nd));
    ACK(cudaMalloc(&c->d_bfr, sizeof(double) * C * (c->nbf ? c->nbf : 1) * nd));
    ACK(cudaMalloc(&c->d_coll, sizeof(double) * C * nd * m * m));
    ACK(cudaMalloc(&c->d_pops, sizeof(double) * C * nd * m));
    ACK(cudaMalloc(&c->d_rel, sizeof(double) * C));
    ACK(cudaMalloc(&c->d_bgop, sizeof(double) * C * nr * nl * nd));
    ACK(cudaMalloc(&c->d_bgem, sizeof(double) * C * nr * nl * nd));
    ACK(cudaMalloc(&c->d_I, sizeof(double) * C * nr * nl * nd));
    ACK(cudaMalloc(&c->d_L, sizeof(double) * C * nr * nl * nd));
    ACK(cudaMalloc(&c->d_opp, sizeof(double) * C * nr * nl * nd));
    ACK(cudaMalloc(&c->d_state, sizeof(int) * C));
    ACK(cudaMalloc(&c->d_iters, sizeof(int) * C));
    c->cap = ncol;
  }
  const cudaMemcpyKind k = mem == SNAPI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaStream_t s = c->stream;
  ACK(cudaMemcpyAsync(c->d_T, in->T, sizeof(double) * C * nd, k, s));
  ACK(cudaMemcpyAsync(c->d_ne, in->ne, sizeof(double) * C * nd, k, s));
  ACK(cudaMemcpyAsync(c->d_na, in->na, sizeof(double) * C * nd, k, s));
  ACK(cudaMemcpyAsync(c->d_kap, in->kappa, sizeof(double) * C * nd, k, s));
  ACK(cudaMemcpyAsync(c->d_vray, in->vray, sizeof(double) * C * nr * nd, k, s));
  if (c->nline) {
    ACK(cudaMemcpyAsync(c->d_dld, in->dld, sizeof(double) * C * c->nline * nd, k, s));
    ACK(cudaMemcpyAsync(c->d_adamp, in->adamp, sizeof(double) * C * c->nline * nd, k, s));
  }
  if (c->nbf) ACK(cudaMemcpyAsync(c->d_bfr, in->bfratio, sizeof(double) * C * c->nbf * nd, k, s));
  ACK(cudaMemcpyAsync(c->d_coll, in->coll, sizeof(double) * C * nd * m * m, k, s));
  ACK(cudaMemcpyAsync(c->d_pops, pops, sizeof(double) * C * nd * m, k, s));
  ACK(cudaMemcpyAsync(c->d_bgop, in->bg_op, sizeof(double) * C * nr * nl * nd, k, s));
  ACK(cudaMemcpyAsync(c->d_bgem, in->bg_em, sizeof(double) * C * nr * nl * nd, k, s));
  ACK(cudaMemsetAsync(c->d_state, 0, sizeof(int) * C, s));
  ACK(cudaMemsetAsync(c->d_iters, 0, sizeof(int) * C, s));
  ACK(cudaMemsetAsync(c->d_rel, 0, sizeof(double) * C, s));
  AliDev D = c->D;
  D.ncol = ncol; D.tol = tol; D.max_iter = max_iter;
  D.T = c->d_T; D.ne = c->d_ne; D.na = c->d_na; D.kap = c->d_kap; D.vray = c->d_vray; D.dld = c->d_dld;
  D.adamp = c->d_adamp; D.bfratio = c->d_bfr; D.coll = c->d_coll; D.bgop = c->d_bgop; D.bgem = c->d_bgem;
  D.pops = c->d_pops; D.I = c->d_I; D.L = c->d_L; D.opp = c->d_opp; D.state = c->d_state; D.iters = c->d_iters;
  D.rel = c->d_rel;
  const FormalSmem S = formal_smem(c->nd, c->nline, c->nbf);
  const int nthr = (int)((nd * D.nsl + 31) / 32 * 32);
  std::vector<int> st(ncol);
  c->last_ms = 0.0;
  for (int it = 0; it < max_iter; ++it) {
    ACK(cudaEventRecord(c->ev0, s));
    k_ali_formal<<<(unsigned)(C * nr * c->nchunk), kAliChunk, S.total, s>>>(D);
    ACK(cudaGetLastError());
    k_ali_rates<<<ncol, nthr, 0, s>>>(D);
    ACK(cudaGetLastError());
    ACK(cudaEventRecord(c->ev1, s));
    ACK(cudaMemcpyAsync(st.data(), c->d_state, sizeof(int) * C, cudaMemcpyDeviceToHost, s));
    ACK(cudaStreamSynchronize(s));
    float ms = 0.f;
    ACK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms += ms;
    bool any = false;
    for (int i = 0; i < ncol; ++i) any = any || st[i] == 0;
    if (!any) break;
  }
  const cudaMemcpyKind o = mem == SNAPI_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  ACK(cudaMemcpyAsync(pops, c->d_pops, sizeof(double) * C * nd * m, o, s));
  if (rel_change) ACK(cudaMemcpyAsync(rel_change, c->d_rel, sizeof(double) * C, o, s));
  if (iters) ACK(cudaMemcpyAsync(iters, c->d_iters, sizeof(int) * C, o, s));
  ACK(cudaStreamSynchronize(s));
  if (status) {
    std::vector<int> out(ncol);
    for (int i = 0; i < ncol; ++i) out[i] = st[i] < 0 ? -1 : 0;
    ACK(cudaMemcpy(status, out.data(), sizeof(int) * C,
                   mem == SNAPI_MEM_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost));
  }
#undef ACK
  return SNAPI_OK;
}

}  // extern "C"
