// snapi_jvp.cuh -- forward-mode (tangent) derivatives of the Stokes synthesis along record
// tangents: the node responses dS/dnode without finite differences.
//
// The reference carries the tangent of the opacity through its formal solver
// (atmos_ppbez::formal_with_responses_full, atmos/plpar/atmos_ppbez_rts.cc:1223-1704) with
// semi-analytic opacity derivatives (atom_rad_synthesis.cc:771-1026); here the tangent is the exact
// derivative of the FP32 forward model that the synthesis evaluates (the W4 region formulas, the
// Bezier optical depth with its monotone derivative, the linear-DELO weights and step), along the
// record tangent of one node, d(record)/d(node):
//
//   depth_precompute_jvp   the per-depth constants (DepthConst, LineDepth) and their tangents
//                          (depth_tangent_head + depth_tangent_line: one line per lane if wanted)
//   jvp_basis_task         direction-independent sums of each line's Zeeman components' W4 values
//                          and x / a derivatives (voigt_grad) at one (wavelength, depth)
//   cell_opacity_jvp       eta / j tangents at one (wavelength, depth) from those sums
//   opd_interior_jvp, bezier_dtau_jvp, delo_step_jvp   the optical depth and the DELO recursion
//
// Everything is __host__ __device__: the kernel (snapi_cuda.cu, k_resp_jvp) and the CPU emulator
// run the same arithmetic.
#pragma once
#include "snapi_core.cuh"

namespace snapi {

// tangents of DepthConst / LineDepth fields (same names)
struct DepthTan {
  float cop, cem, beta, st2, ctb, opc2, c2, s2, hb, hf, invT, lt;
};
struct LineTan {
  float inv_dld, a, bsh, opn, emn;
};

// the scalars of a depth row that every line's tangent uses
struct DepthTanHead {
  float T, vt, B, dT, dvt, dB, invk, dinvk;
};

// the scalars of a depth row that every line's tangent uses
SNAPI_HD void depth_tangent_scalars(const float *rec, const float *trec, DepthTanHead &h) {
  h.T = rec[F_T];
  h.vt = rec[F_VT];
  h.B = rec[F_B];
  h.dT = trec[F_T];
  h.dvt = trec[F_VT];
  h.dB = trec[F_B];
  h.invk = 1.0f / rec[F_KAP];
  h.dinvk = -trec[F_KAP] * h.invk * h.invk;
}

// the tangent of depth_precompute's depth constants along trec (the record row's tangent)
SNAPI_HD void depth_tangent_head(const float *rec, const float *trec, float lam_mid, DepthTan &dd, DepthTanHead &h) {
  depth_tangent_scalars(rec, trec, h);
  const float T = h.T, ne = rec[F_NE], B = h.B, dT = h.dT, dne = trec[F_NE], invk = h.invk, dinvk = h.dinvk;
  const float xpm = 1.4387769f / lam_mid;
  const float Em = fexp(xpm / T);
  const float plm = (float)(2.0 * 6.62606957 * 8.9875517E-7) / (lam_mid * lam_mid * lam_mid * lam_mid * lam_mid) / (Em - 1.0f);
  const float dEm = -Em * xpm / (T * T) * dT;
  const float dplm = -plm / (Em - 1.0f) * dEm;
  const float ope = ne * kSigmaT, dope = dne * kSigmaT;
  dd.cop = (dope + trec[F_BFOP]) * invk + (ope + rec[F_BFOP]) * dinvk;
  dd.cem = (dope * plm + ope * dplm + trec[F_BFEM]) * invk + (ope * plm + rec[F_BFEM]) * dinvk;
  dd.beta = trec[F_VLOS] * (float)(1.0 / kC);
  float th = rec[F_INC] * (float)(kPi / 180.0), ph = rec[F_AZI] * (float)(kPi / 180.0);
  float dth = trec[F_INC] * (float)(kPi / 180.0), dph = trec[F_AZI] * (float)(kPi / 180.0);
  if (B < 0.001f) th = ph = dth = dph = 0.0f;
  float sth, cth, s2p, c2p;
  fsincos(th, &sth, &cth);
  fsincos(2.0f * ph, &s2p, &c2p);
  dd.st2 = 2.0f * sth * cth * dth;
  dd.ctb = -sth * dth;
  dd.opc2 = -2.0f * cth * sth * dth;
  dd.c2 = -2.0f * s2p * dph;
  dd.s2 = 2.0f * c2p * dph;
  dd.hb = trec[F_HMBF] * invk + rec[F_HMBF] * dinvk;
  dd.hf = trec[F_HMFF] * invk + rec[F_HMFF] * dinvk;
  dd.invT = -dT / (T * T);
  dd.lt = -dT / (T * kLn10);
}

// the tangent of line j's depth constants (ld: the row's LineDepth of line j)
SNAPI_HD void depth_tangent_line(const float *rec, const float *trec, const LineConst &L, const LineDepth &ld, int j,
                                 const DepthTanHead &h, LineTan &t) {
  const float *rl = rec + F_LINE0 + 3 * j, *tl = trec + F_LINE0 + 3 * j;
  const float W = L.two_k_over_m * h.T + h.vt * h.vt;
  const float dW = L.two_k_over_m * h.dT + 2.0f * h.vt * h.dvt;
  const float idl = ld.inv_dld;
  // dld = sqrt(W) lam0/c:  d(1/dld) = -idl / (2 W) dW
  const float didl = -0.5f * idl * dW / W;
  t.inv_dld = didl;
  t.a = L.sf * (tl[2] * idl + (L.ar + rl[2]) * didl);
  t.bsh = L.zee * (h.dB * idl + h.B * didl);
  t.opn = tl[0] * h.invk * idl + rl[0] * (h.dinvk * idl + h.invk * didl);
  t.emn = tl[1] * h.invk * idl + rl[1] * (h.dinvk * idl + h.invk * didl);
}

// the tangent of depth_precompute along trec; ld: the row's LineDepth
SNAPI_HD void depth_tangent(const float *rec, const float *trec, int nlines, const LineConst *lc, float lam_mid,
                            const LineDepth *ld, DepthTan &dd, LineTan *dl) {
  DepthTanHead h;
  depth_tangent_head(rec, trec, lam_mid, dd, h);
  for (int j = 0; j < nlines; ++j) depth_tangent_line(rec, trec, lc[j], ld[j], j, h, dl[j]);
}

// depth_precompute and its tangent along trec
SNAPI_HD void depth_precompute_jvp(const float *rec, const float *trec, int nlines, const LineConst *lc,
                                   float lam_mid, DepthConst &d, LineDepth *ld, DepthTan &dd, LineTan *dl) {
  depth_precompute(rec, nlines, lc, lam_mid, d, ld);
  depth_tangent(rec, trec, nlines, lc, lam_mid, ld, dd, dl);
}

// The opacity tangent of a (wavelength, depth) cell is linear in a few scalars of the direction
// per line (dx0, d bsh, d a, d opn, d emn) and of the depth (DepthTan), so the Zeeman components'
// W4 values enter it only through sums that do not depend on the direction.  Per split line and
// group g (pi, sigma_b, sigma_r) 8 sums over the group's components c (strength S_c, shift D_c):
//   S H, S F, S Hx, S Fx, S Hx D, S Fx D, S Ha, S Fa
// (H, F the Voigt / Faraday values, x / a their derivatives, voigt_grad); per unsplit line 3:
// H, Hx, Ha.  The cell's basis holds them in line order; the W4 work of a cell is done once for
// all directions and each direction's tangent costs a few multiply-adds per line.
SNAPI_HD int jvp_basis_size(const LineConst *lc, int nlines) {
  int n = 3;  // + the H- factors exp(-xs / T), 10^f(log theta), exp(xp / T), one more task
  for (int j = 0; j < nlines; ++j) n += lc[j].split ? 24 : 3;
  return n;
}

// the basis is filled by tasks: one per (split line, group) and one per unsplit line
SNAPI_HD int jvp_basis_tasks(const LineConst *lc, int nlines) {
  int n = 1;
  for (int j = 0; j < nlines; ++j) n += lc[j].split ? 3 : 1;
  return n;
}

// task k of the cell at (lambda, depth): its components' W4 evaluations and their sums into B
SNAPI_HD void jvp_basis_task(const DepthConst &d, const LineDepth *ld, const LineConst *lc, int nlines,
                             const float *compS, const float *compD, const LamConst &lam, const float *delta, int k,
                             float *B) {
  int j = 0, off = 0;
  for (; j < nlines; ++j) {
    const int nt = lc[j].split ? 3 : 1;
    if (k < nt) break;
    k -= nt;
    off += lc[j].split ? 24 : 3;
  }
  if (j == nlines) {  // the H- bound-free / free-free factors of the cell
    B[off] = fexp(-lam.xs * d.invT);
    B[off + 1] = fexp(kLn10 * (lam.F0 + lam.f1 * d.lt + lam.f2 * d.lt * d.lt));
    B[off + 2] = fexp(lam.xp * d.invT);
    return;
  }
  const LineConst &L = lc[j];
  const LineDepth &q = ld[j];
  const float x0 = (delta[j] - lam.lam * d.beta) * q.inv_dld;
  float H, F, Hx, Fx, Ha, Fa;
  if (!L.split) {
    voigt_grad(x0, q.a, H, F, Hx, Fx, Ha, Fa);
    B[off] = H;
    B[off + 1] = Hx;
    B[off + 2] = Ha;
    return;
  }
  int c = L.comp_off;
  for (int g = 0; g < k; ++g) c += L.ncomp[g];
  float sH = 0.f, sF = 0.f, sHx = 0.f, sFx = 0.f, sHxD = 0.f, sFxD = 0.f, sHa = 0.f, sFa = 0.f;
  for (int i = 0; i < L.ncomp[k]; ++i, ++c) {
    const float D = compD[c], S = compS[c];
    voigt_grad(x0 + D * q.bsh, q.a, H, F, Hx, Fx, Ha, Fa);
    sH += H * S;
    sF += F * S;
    sHx += Hx * S;
    sFx += Fx * S;
    sHxD += Hx * D * S;
    sFxD += Fx * D * S;
    sHa += Ha * S;
    sFa += Fa * S;
  }
  float *b = B + off + 8 * k;
  b[0] = sH; b[1] = sF; b[2] = sHx; b[3] = sFx; b[4] = sHxD; b[5] = sFxD; b[6] = sHa; b[7] = sFa;
}

// Tangent of cell_opacity (eta[7], j[4]) along (dd, dl) from the cell's basis B (jvp_basis_task).
SNAPI_HD void cell_opacity_jvp(const DepthConst &d, const LineDepth *ld, const LineConst *lc, int nlines,
                               const LamConst &lam, const float *delta, const float *B, const DepthTan &dd,
                               const LineTan *dl, float *deta, float *djj) {
  deta[0] = dd.cop;
  deta[1] = deta[2] = deta[3] = deta[4] = deta[5] = deta[6] = 0.0f;
  djj[0] = dd.cem;
  djj[1] = djj[2] = djj[3] = 0.0f;
  int off = 0;
  for (int j = 0; j < nlines; ++j) {
    const LineConst &L = lc[j];
    const LineDepth &q = ld[j];
    const LineTan &t = dl[j];
    // x0 = (delta - lam beta) inv_dld; a component's x = x0 + D bsh
    const float xd = delta[j] - lam.lam * d.beta;
    const float dx0 = -lam.lam * dd.beta * q.inv_dld + xd * t.inv_dld;
    const float *b = B + off;
    if (!L.split) {
      const float dH = b[1] * dx0 + b[2] * t.a;
      deta[0] += t.opn * b[0] + q.opn * dH;
      djj[0] += t.emn * b[0] + q.emn * dH;
      off += 3;
    } else {
      float Hs[3], Fs[3], dHs[3], dFs[3];
#pragma unroll
      for (int g = 0; g < 3; ++g) {
        const float *bg = b + 8 * g;
        Hs[g] = bg[0];
        Fs[g] = bg[1];
        dHs[g] = bg[2] * dx0 + bg[4] * t.bsh + bg[6] * t.a;
        dFs[g] = bg[3] * dx0 + bg[5] * t.bsh + bg[7] * t.a;
      }
      off += 24;
      const float hrb = 0.5f * (Hs[2] + Hs[1]), dhrb = 0.5f * (dHs[2] + dHs[1]);
      const float frb = 0.5f * (Fs[2] + Fs[1]), dfrb = 0.5f * (dFs[2] + dFs[1]);
      const float hpm = Hs[0] - hrb, dhpm = dHs[0] - dhrb;
      const float fpm = Fs[0] - frb, dfpm = dFs[0] - dfrb;
      const float eI = 0.5f * (Hs[0] * d.st2 + hrb * d.opc2);
      const float deI = 0.5f * (dHs[0] * d.st2 + Hs[0] * dd.st2 + dhrb * d.opc2 + hrb * dd.opc2);
      const float sc = d.st2 * d.c2, ss = d.st2 * d.s2;
      const float dsc = dd.st2 * d.c2 + d.st2 * dd.c2, dss = dd.st2 * d.s2 + d.st2 * dd.s2;
      const float eQ = 0.5f * hpm * sc, deQ = 0.5f * (dhpm * sc + hpm * dsc);
      const float eU = 0.5f * hpm * ss, deU = 0.5f * (dhpm * ss + hpm * dss);
      const float eV = 0.5f * (Hs[2] - Hs[1]) * d.ctb, deV = 0.5f * ((dHs[2] - dHs[1]) * d.ctb + (Hs[2] - Hs[1]) * dd.ctb);
      const float rQ = 0.5f * fpm * sc, drQ = 0.5f * (dfpm * sc + fpm * dsc);
      const float rU = 0.5f * fpm * ss, drU = 0.5f * (dfpm * ss + fpm * dss);
      const float rV = 0.5f * (Fs[2] - Fs[1]) * d.ctb, drV = 0.5f * ((dFs[2] - dFs[1]) * d.ctb + (Fs[2] - Fs[1]) * dd.ctb);
      deta[0] += deI * q.opn + eI * t.opn;
      deta[1] += deQ * q.opn + eQ * t.opn;
      deta[2] += deU * q.opn + eU * t.opn;
      deta[3] += deV * q.opn + eV * t.opn;
      deta[4] += drQ * q.opn + rQ * t.opn;
      deta[5] += drU * q.opn + rU * t.opn;
      deta[6] += drV * q.opn + rV * t.opn;
      djj[0] += deI * q.emn + eI * t.emn;
      djj[1] += deQ * q.emn + eQ * t.emn;
      djj[2] += deU * q.emn + eU * t.emn;
      djj[3] += deV * q.emn + eV * t.emn;
    }
  }
  // H- bound-free + free-free and their LTE emissivity (the exponentials from the basis)
  const float e1 = B[off];
  const float de1 = -lam.xs * e1 * dd.invT;
  const float opbf = lam.afud * d.hb * (1.0f - e1);
  const float dopbf = lam.afud * (dd.hb * (1.0f - e1) - d.hb * de1);
  const float E10 = B[off + 1];
  const float dE10 = E10 * kLn10 * (lam.f1 + 2.0f * lam.f2 * d.lt) * dd.lt;
  const float opff = d.hf * E10, dopff = dd.hf * E10 + d.hf * dE10;
  const float oph = opbf + opff, doph = dopbf + dopff;
  const float Ep = B[off + 2];
  const float dEp = lam.xp * Ep * dd.invT;
  const float pl = lam.pp / (Ep - 1.0f), dpl = -pl / (Ep - 1.0f) * dEp;
  deta[0] += doph;
  djj[0] += doph * pl + oph * dpl;
}

// tangents of K' = eta_q / eta_I, S = j / eta_I and eta_I
SNAPI_HD void depth_opacity_jvp(const float *kp, const float *S, float e, const float *deta, const float *djj,
                                float *dkp, float *dS, float &de) {
  const float ie = 1.0f / e;
  de = deta[0];
#pragma unroll
  for (int q = 0; q < 6; ++q) dkp[q] = (deta[q + 1] - kp[q] * de) * ie;
#pragma unroll
  for (int s = 0; s < 4; ++s) dS[s] = (djj[s] - S[s] * de) * ie;
}

// tangent of opd_interior
// the interior optical-depth derivative's tangent is linear in the three opacities' tangents: its
// coefficients (direction-independent) and their use
SNAPI_HD void opd_interior_coef(double e_up, double e_c, double e_dn, double h1, double h2, double *g) {
  g[0] = g[1] = g[2] = 0.0;
  opd_interior_grad(e_up, e_c, e_dn, h1, h2, 1.0, g[0], g[1], g[2]);
}
SNAPI_HD double opd_interior_apply(const double *g, double de_up, double de_c, double de_dn) {
  return g[0] * de_up + g[1] * de_c + g[2] * de_dn;
}
SNAPI_HD double opd_interior_jvp(double e_up, double e_c, double e_dn, double h1, double h2, double de_up,
                                 double de_c, double de_dn) {
  double g[3];
  opd_interior_coef(e_up, e_c, e_dn, h1, h2, g);
  return opd_interior_apply(g, de_up, de_c, de_dn);
}

// tangent of bezier_dtau: dtau = dl/3 (e_b + e_a + (e_a + e_b)/2 + dl/4 (opd_b - opd_a))
SNAPI_HD double bezier_dtau_jvp(double de_below, double de_above, double dopd_below, double dopd_above, double dl) {
  return dl / 3.0 * (1.5 * (de_below + de_above) + 0.25 * dl * (dopd_below - dopd_above));
}

// tangent of delo_step: A Ic = B with A = 1 + w1 K'_c, B = -w0 K'_p I_p + w0 S_p + w1 S_c + etb I_p,
// so dIc = A^-1 (dB - dA Ic).  Ic: the forward result.  The weights are functions of tau_b, so
//   dB - dA Ic = dtb [gw0 (S_p - K'_p I_p) + gw1 (S_c - K'_c Ic) + getb I_p]
//                - w0 (dK'_p I_p + K'_p dI_p) + w0 dS_p + w1 dS_c + etb dI_p - w1 dK'_c Ic
// (gw0, gw1, getb the weights' derivatives).  The direction-independent part of a step -- the
// weights, the bracket multiplying dtb and the LU of A -- is delo_jvp_prep; delo_jvp_apply adds a
// direction's tangent to it.
struct DeloPrep {
  float w0, w1, etb, g[4], LU[16];
};
constexpr int kDeloPrepFloats = 23;
static_assert(sizeof(DeloPrep) == sizeof(float) * kDeloPrepFloats, "DeloPrep is copied as a float array");

SNAPI_HD void delo_jvp_prep(const float *Ip, const float *kpp, const float *Sp, const float *kpc, const float *Sc,
                            float tb, const float *Ic, DeloPrep &p) {
  float gw0, gw1, getb, A[16], t1[4], t3[4];
  delo_weights(tb, p.w0, p.w1, p.etb);
  delo_weights_grad(tb, gw0, gw1, getb);
  kp_mul(kpc, Ic, t1);  // K'_c Ic
  kp_mul(kpp, Ip, t3);  // K'_p Ip
#pragma unroll
  for (int s = 0; s < 4; ++s) p.g[s] = gw0 * (Sp[s] - t3[s]) + gw1 * (Sc[s] - t1[s]) + getb * Ip[s];
  build_A(kpc, p.w1, false, A);
  crout4(A, p.LU);
}

SNAPI_HD void delo_jvp_apply(const DeloPrep &p, const float *Ip, const float *kpp, const float *Ic, const float *dIp,
                             const float *dkpp, const float *dSp, const float *dkpc, const float *dSc, float dtb,
                             float *dIc) {
  float r[4], t2[4], t4[4], t5[4];
  kp_mul(dkpc, Ic, t2);  // dK'_c Ic
  kp_mul(dkpp, Ip, t4);  // dK'_p Ip
  kp_mul(kpp, dIp, t5);  // K'_p dIp
#pragma unroll
  for (int s = 0; s < 4; ++s)
    r[s] = dtb * p.g[s] - p.w0 * (t4[s] + t5[s]) + p.w0 * dSp[s] + p.w1 * dSc[s] + p.etb * dIp[s] - p.w1 * t2[s];
  solve_crout4(p.LU, r, dIc);
}

SNAPI_HD void delo_step_jvp(const float *Ip, const float *kpp, const float *Sp, const float *kpc, const float *Sc,
                            float tb, const float *Ic, const float *dIp, const float *dkpp, const float *dSp,
                            const float *dkpc, const float *dSc, float dtb, float *dIc) {
  DeloPrep p;
  delo_jvp_prep(Ip, kpp, Sp, kpc, Sc, tb, Ic, p);
  delo_jvp_apply(p, Ip, kpp, Ic, dIp, dkpp, dSp, dkpc, dSc, dtb, dIc);
}

}  // namespace snapi
