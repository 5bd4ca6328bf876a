// CPU emulator of the CUDA kernels (test infrastructure).
//
// Compiles snapi_b200/csrc/snapi_core.cuh and snapi_sweep.cuh with the host compiler and runs
// the per-(pixel, wavelength) sweeps sequentially, with the same FP32 arithmetic, the same
// per-depth constants and the same reduction order per depth as the device code (up to the
// order of the wavelength sums).  Lets the tests check the kernel math against the oracle on a
// machine without a GPU.
#include <math.h>
#include <string.h>

#include <vector>

#include "../../snapi_b200/csrc/snapi_jvp.cuh"
#include "../../snapi_b200/csrc/snapi_sweep.cuh"

using namespace snapi;

namespace {

struct EmuLine {  // mirror of snapi_line (include/snapi_cuda.h)
  double lam0, sf, ar, mass;
  int split;
  int ncomp[3];
  double S[3][16];
  double D[3][16];
};

struct Problem {
  int nd, nl, nlines, nfield, nred;
  float lam_mid;
  std::vector<double> lamvac, D;
  std::vector<LineConst> lc;
  std::vector<float> cS, cD;
};

double airtovac_d(double la) {
  double s = 1E4 / (la * 1E8);
  double n = 1.0 + 0.00008336624212083 + 0.02408926869968 / (130.1065924522 - s * s) +
             0.0001599740894897 / (38.92568793293 - s * s);
  return la * n;
}

Problem make_problem(int nd, int nl, int nlines, const double *lam_air, const double *tau500, double mu,
                     const EmuLine *lines) {
  Problem P;
  P.nd = nd; P.nl = nl; P.nlines = nlines; P.nfield = F_LINE0 + 3 * nlines;
  P.nred = kNumRed + kRedPerLine * nlines;
  P.lamvac.resize(nl);
  for (int l = 0; l < nl; ++l) P.lamvac[l] = airtovac_d(lam_air[l]);
  P.lam_mid = (float)(0.5 * (P.lamvac[nl - 1] + P.lamvac[0]));
  P.D.resize(nd - 1);
  for (int i = 0; i + 1 < nd; ++i) P.D[i] = (tau500[i + 1] - tau500[i]) / mu;
  P.lc.resize(nlines);
  for (int j = 0; j < nlines; ++j) {
    const EmuLine &s = lines[j];
    LineConst &L = P.lc[j];
    L.lam0 = s.lam0; L.sf = (float)s.sf; L.ar = (float)s.ar;
    L.two_k_over_m = (float)(2.0 * kK / s.mass);
    L.lam0_over_c = (float)(s.lam0 / kC);
    L.zee = (float)(4.67E-5 * s.lam0 * s.lam0);
    L.split = s.split ? 1 : 0;
    L.comp_off = (int)P.cS.size();
    for (int g = 0; g < 3; ++g) {
      L.ncomp[g] = s.split ? s.ncomp[g] : 0;
      for (int i = 0; i < L.ncomp[g]; ++i) { P.cS.push_back((float)s.S[g][i]); P.cD.push_back((float)s.D[g][i]); }
    }
  }
  if (P.cS.empty()) { P.cS.push_back(0.f); P.cD.push_back(0.f); }
  return P;
}

struct PixelState {
  std::vector<float> rec;
  std::vector<DepthConst> dc;
  std::vector<LineDepth> ld;
  PixelView pv;
};

void stage(const Problem &P, const float *rec, PixelState &ps) {
  ps.rec.assign(rec, rec + P.nd * P.nfield);
  ps.dc.resize(P.nd);
  ps.ld.resize(P.nd * (P.nlines ? P.nlines : 1));
  for (int z = 0; z < P.nd; ++z)
    depth_precompute(&ps.rec[z * P.nfield], P.nlines, P.lc.data(), P.lam_mid, ps.dc[z], &ps.ld[z * P.nlines]);
  ps.pv.nd = P.nd; ps.pv.nlines = P.nlines; ps.pv.nfield = P.nfield;
  ps.pv.rec = ps.rec.data(); ps.pv.dc = ps.dc.data(); ps.pv.ld = ps.ld.data(); ps.pv.lc = P.lc.data();
  ps.pv.compS = P.cS.data(); ps.pv.compD = P.cD.data(); ps.pv.D = P.D.data();
}

void lambda_setup(const Problem &P, int l, LamConst &lam, float *delta) {
  lambda_precompute(P.lamvac[l], lam);
  for (int j = 0; j < P.nlines; ++j) delta[j] = (float)(P.lc[j].lam0 - P.lamvac[l]);
}

struct HostScratch {
  std::vector<float> buf;  // [nd][16]
  void store(int z, const float *I, const float *kp, const float *S, float e, float tau) {
    float *p = &buf[z * 16];
    for (int s = 0; s < 4; ++s) { p[s] = I[s]; p[12 + s] = S[s]; }
    for (int q = 0; q < 6; ++q) p[4 + q] = kp[q];
    p[10] = e; p[11] = tau;
  }
  void prefetch(int) {}
  void load(int z, float *I, float *kp, float *S, float &e, float &tau) const {
    const float *p = &buf[z * 16];
    for (int s = 0; s < 4; ++s) { I[s] = p[s]; S[s] = p[12 + s]; }
    for (int q = 0; q < 6; ++q) kp[q] = p[4 + q];
    e = p[10]; tau = p[11];
  }
  void store_bar(int z, const float *eb, const float *jb) {
    float *p = &buf[z * 16];
    for (int i = 0; i < 7; ++i) p[i] = eb[i];
    for (int i = 0; i < 4; ++i) p[7 + i] = jb[i];
  }
  void load_bar(int z, float *eb, float *jb) const {
    const float *p = &buf[z * 16];
    for (int i = 0; i < 7; ++i) eb[i] = p[i];
    for (int i = 0; i < 4; ++i) jb[i] = p[7 + i];
  }
};
struct NoStore {
  void store(int, const float *, const float *, const float *, float, float) {}
};
struct HostReducer {
  float *acc;
  int nred;
  void add(int z, const float *red, int n) {
    for (int i = 0; i < n; ++i) acc[z * nred + i] += red[i];
  }
};

}  // namespace

extern "C" {

int emu_synth(int nd, int nl, int nlines, const double *lam_air, const double *tau500, double mu, const void *lines,
              int npix, const float *records, float *stokes) {
  Problem P = make_problem(nd, nl, nlines, lam_air, tau500, mu, (const EmuLine *)lines);
  PixelState ps;
  for (int p = 0; p < npix; ++p) {
    stage(P, records + (size_t)p * nd * P.nfield, ps);
    for (int l = 0; l < nl; ++l) {
      LamConst lam;
      float delta[kMaxLines];
      lambda_setup(P, l, lam, delta);
      NoStore ns;
      forward_sweep<false>(ps.pv, lam, delta, stokes + ((size_t)p * nl + l) * 4, ns);
    }
  }
  return 0;
}

int emu_adjoint(int nd, int nl, int nlines, const double *lam_air, const double *tau500, double mu, const void *lines,
                double stokes_scale, int npix, const float *records, const float *obs, const double *ws,
                const float *mask, int npar, const float *tangents, float *stokes, double *chi2, double *grad,
                double *rec_grad) {
  Problem P = make_problem(nd, nl, nlines, lam_air, tau500, mu, (const EmuLine *)lines);
  const double scale2 = stokes_scale * stokes_scale;
  const int nrec = nd * P.nfield;
  PixelState ps;
  std::vector<float> acc(nd * P.nred), rb(nrec);
  HostScratch sc;
  sc.buf.resize(nd * 16);
  float red[kNumRed + kRedPerLine * kMaxLines];
  for (int p = 0; p < npix; ++p) {
    stage(P, records + (size_t)p * nrec, ps);
    std::fill(acc.begin(), acc.end(), 0.f);
    std::fill(rb.begin(), rb.end(), 0.f);
    double c2 = 0.0;
    for (int l = 0; l < nl; ++l) {
      LamConst lam;
      float delta[kMaxLines];
      lambda_setup(P, l, lam, delta);
      float out[4];
      forward_sweep<true>(ps.pv, lam, delta, out, sc);
      if (stokes)
        for (int s = 0; s < 4; ++s) stokes[((size_t)p * nl + l) * 4 + s] = out[s];
      const float m = mask ? mask[(size_t)p * nl + l] : 1.0f;
      float seed[4];
      for (int s = 0; s < 4; ++s) {
        const double r = ((double)obs[((size_t)p * nl + l) * 4 + s] - (double)out[s]) * ws[s] * m;
        c2 += r * r / scale2;
        seed[s] = (float)(-2.0 * r * ws[s] * m / scale2);
      }
      HostReducer rd{acc.data(), P.nred};
      reverse_sweep(ps.pv, lam, delta, seed, sc, rd, red, P.nred);
    }
    chi2[p] = c2 * scale2;
    for (int z = 0; z < nd; ++z)
      depth_chain_adjoint(&ps.rec[z * P.nfield], nlines, P.lc.data(), P.lam_mid, ps.dc[z], &ps.ld[z * nlines],
                          &acc[z * P.nred], &rb[z * P.nfield]);
    if (rec_grad)
      for (int i = 0; i < nrec; ++i) rec_grad[(size_t)p * nrec + i] = (double)rb[i] * scale2;
    for (int q = 0; q < npar; ++q) {
      const float *tp = tangents + ((size_t)p * npar + q) * nrec;
      double g = 0.0;
      for (int i = 0; i < nrec; ++i) g += (double)rb[i] * (double)tp[i];
      grad[(size_t)p * npar + q] = g * scale2;
    }
  }
  return 0;
}

// Node responses by the forward-mode (tangent) sweep, one direction at a time, each forming the
// direction-independent W4 sums of its cells itself (the kernel shares them among its directions):
// dstokes [npix][npar][nl][4].
int emu_jvp(int nd, int nl, int nlines, const double *lam_air, const double *tau500, double mu, const void *lines,
            int npix, const float *records, int npar, const float *tangents, float *dstokes) {
  Problem P = make_problem(nd, nl, nlines, lam_air, tau500, mu, (const EmuLine *)lines);
  const int nrec = nd * P.nfield, nb = jvp_basis_size(P.lc.data(), nlines), ntask = jvp_basis_tasks(P.lc.data(), nlines);
  PixelState ps;
  HostScratch sc;
  sc.buf.resize(nd * 16);
  std::vector<float> w(nb ? nb : 1);
  for (int p = 0; p < npix; ++p) {
    stage(P, records + (size_t)p * nrec, ps);
    for (int l = 0; l < nl; ++l) {
      LamConst lam;
      float delta[kMaxLines];
      lambda_setup(P, l, lam, delta);
      float out[4];
      forward_sweep<true>(ps.pv, lam, delta, out, sc);
      for (int q = 0; q < npar; ++q) {
        const float *tq = tangents + ((size_t)p * npar + q) * nrec;
        // tangents of K', S, eta_I at depth z
        auto depth_tan = [&](int z, float *dkp, float *dS, float &de) {
          DepthConst d;
          LineDepth ld[kMaxLines];
          DepthTan dd;
          LineTan dl[kMaxLines];
          depth_precompute_jvp(&ps.rec[z * P.nfield], tq + z * P.nfield, nlines, P.lc.data(), P.lam_mid, d, ld, dd,
                               dl);
          for (int k = 0; k < ntask; ++k)
            jvp_basis_task(d, ld, P.lc.data(), nlines, P.cS.data(), P.cD.data(), lam, delta, k, w.data());
          float deta[7], djj[4], I[4], kp[6], S[4], e, tau;
          cell_opacity_jvp(d, ld, P.lc.data(), nlines, lam, delta, w.data(), dd, dl, deta, djj);
          sc.load(z, I, kp, S, e, tau);
          depth_opacity_jvp(kp, S, e, deta, djj, dkp, dS, de);
        };
        float dkA[6], dSA[4], deA, dkB[6], dSB[4], deB, dkC[6], dSC[4], deC;
        depth_tan(nd - 1, dkA, dSA, deA);
        depth_tan(nd - 2, dkB, dSB, deB);
        float I[4], kA[6], SA[4], eA, tA, kB[6], SB[4], eB, tB, kC[6], SC[4], eC, tC;
        sc.load(nd - 1, I, kA, SA, eA, tA);
        sc.load(nd - 2, I, kB, SB, eB, tB);
        float dI[4] = {dSA[0], 0.f, 0.f, 0.f};
        double dopd_below = ((double)deB - (double)deA) / P.D[nd - 2];
        for (int z = nd - 2; z >= 1; --z) {
          depth_tan(z - 1, dkC, dSC, deC);
          float Id[4];
          sc.load(z - 1, Id, kC, SC, eC, tC);
          const double dopd_z = opd_interior_jvp(eA, eB, eC, P.D[z], P.D[z - 1], deA, deB, deC);
          const float dtau = (float)bezier_dtau_jvp(deA, deB, dopd_below, dopd_z, P.D[z]);
          float Ip[4], Ic[4], k_[6], S_[4], e_, tau;
          sc.load(z + 1, Ip, k_, S_, e_, tau);
          sc.load(z, Ic, k_, S_, e_, tau);
          float dIn[4];
          delo_step_jvp(Ip, kA, SA, kB, SB, tau, Ic, dI, dkA, dSA, dkB, dSB, dtau, dIn);
          for (int s = 0; s < 4; ++s) dI[s] = dIn[s];
          for (int k = 0; k < 6; ++k) { kA[k] = kB[k]; kB[k] = kC[k]; dkA[k] = dkB[k]; dkB[k] = dkC[k]; }
          for (int s = 0; s < 4; ++s) { SA[s] = SB[s]; SB[s] = SC[s]; dSA[s] = dSB[s]; dSB[s] = dSC[s]; }
          eA = eB; eB = eC; deA = deB; deB = deC;
          dopd_below = dopd_z;
        }
        float *o = dstokes + (((size_t)p * npar + q) * nl + l) * 4;
        for (int s = 0; s < 4; ++s) o[s] = dI[s];  // the top point copies the one below
      }
    }
  }
  return 0;
}

// W4 and its derivatives (for unit tests of the Voigt code)
void emu_voigt(float x, float a, float *out6) {
  float H, F, Hx, Fx, Ha, Fa;
  voigt_grad(x, a, H, F, Hx, Fx, Ha, Fa);
  out6[0] = H; out6[1] = F; out6[2] = Hx; out6[3] = Fx; out6[4] = Ha; out6[5] = Fa;
  float H2, F2;
  voigt(x, a, H2, F2);
  out6[0] = H2; out6[1] = F2;
}

}  // extern "C"

extern "C" int emu_opacity(int nd, int nl, int nlines, const double *lam_air, const double *tau500, double mu,
                           const void *lines, const float *record, int l, float *eta_out /*[nd][7]*/,
                           float *j_out /*[nd][4]*/) {
  Problem P = make_problem(nd, nl, nlines, lam_air, tau500, mu, (const EmuLine *)lines);
  PixelState ps;
  stage(P, record, ps);
  LamConst lam;
  float delta[kMaxLines];
  lambda_setup(P, l, lam, delta);
  for (int z = 0; z < nd; ++z)
    cell_opacity(ps.dc[z], &ps.ld[z * nlines], P.lc.data(), nlines, P.cS.data(), P.cD.data(), lam, delta,
                 eta_out + z * 7, j_out + z * 4);
  return 0;
}
