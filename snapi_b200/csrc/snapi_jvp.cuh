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
//   cell_opacity_jvp       eta / j tangents at one (wavelength, depth), from each Zeeman component's
//                          W4 value and x / a derivatives (voigt_grad), which a caller may share
//                          among directions
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

// the tangent of depth_precompute along trec (the record row's tangent); ld: the row's LineDepth
SNAPI_HD void depth_tangent(const float *rec, const float *trec, int nlines, const LineConst *lc, float lam_mid,
                            const LineDepth *ld, DepthTan &dd, LineTan *dl) {
  const float T = rec[F_T], vt = rec[F_VT], ne = rec[F_NE], B = rec[F_B];
  const float dT = trec[F_T], dvt = trec[F_VT], dne = trec[F_NE], dB = trec[F_B];
  const float invk = 1.0f / rec[F_KAP];
  const float dinvk = -trec[F_KAP] * invk * invk;
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
  for (int j = 0; j < nlines; ++j) {
    const LineConst &L = lc[j];
    const float *rl = rec + F_LINE0 + 3 * j, *tl = trec + F_LINE0 + 3 * j;
    const float W = L.two_k_over_m * T + vt * vt;
    const float dW = L.two_k_over_m * dT + 2.0f * vt * dvt;
    const float idl = ld[j].inv_dld;
    // dld = sqrt(W) lam0/c:  d(1/dld) = -idl / (2 W) dW
    const float didl = -0.5f * idl * dW / W;
    dl[j].inv_dld = didl;
    dl[j].a = L.sf * (tl[2] * idl + (L.ar + rl[2]) * didl);
    dl[j].bsh = L.zee * (dB * idl + B * didl);
    dl[j].opn = tl[0] * invk * idl + rl[0] * (dinvk * idl + invk * didl);
    dl[j].emn = tl[1] * invk * idl + rl[1] * (dinvk * idl + invk * didl);
  }
}

// depth_precompute and its tangent along trec
SNAPI_HD void depth_precompute_jvp(const float *rec, const float *trec, int nlines, const LineConst *lc,
                                   float lam_mid, DepthConst &d, LineDepth *ld, DepthTan &dd, LineTan *dl) {
  depth_precompute(rec, nlines, lc, lam_mid, d, ld);
  depth_tangent(rec, trec, nlines, lc, lam_mid, ld, dd, dl);
}

// Number of W4 evaluations of one (wavelength, depth): one per Zeeman component of split lines,
// one per unsplit line.  Component c of the enumeration (lines in order, groups pi, sigma_b,
// sigma_r) has offset x = x0_j + D_c bsh_j.
SNAPI_HD int w4_count(const LineConst *lc, int nlines) {
  int n = 0;
  for (int j = 0; j < nlines; ++j) n += lc[j].split ? lc[j].ncomp[0] + lc[j].ncomp[1] + lc[j].ncomp[2] : 1;
  return n;
}

// W4 values and derivatives of evaluation c at (lambda, depth): w6 = {H, F, Hx, Fx, Ha, Fa}
SNAPI_HD void w4_eval(const DepthConst &d, const LineDepth *ld, const LineConst *lc, int nlines, const float *compD,
                      const LamConst &lam, const float *delta, int c, float *w6) {
  int j = 0, k = c;
  while (j < nlines) {
    const int n = lc[j].split ? lc[j].ncomp[0] + lc[j].ncomp[1] + lc[j].ncomp[2] : 1;
    if (k < n) break;
    k -= n;
    ++j;
  }
  const LineConst &L = lc[j];
  const LineDepth &q = ld[j];
  float x = (delta[j] - lam.lam * d.beta) * q.inv_dld;
  if (L.split) x += compD[L.comp_off + k] * q.bsh;
  voigt_grad(x, q.a, w6[0], w6[1], w6[2], w6[3], w6[4], w6[5]);
}

// Tangent of cell_opacity (eta[7], j[4]) along (dd, dl), given the W4 evaluations of this
// (lambda, depth) in the w4_count enumeration: w[c * wstride + k], k = H, F, Hx, Fx, Ha, Fa.
SNAPI_HD void cell_opacity_jvp(const DepthConst &d, const LineDepth *ld, const LineConst *lc, int nlines,
                               const float *compS, const float *compD, const LamConst &lam, const float *delta,
                               const float *w, int wstride, const DepthTan &dd, const LineTan *dl, float *deta,
                               float *djj) {
  deta[0] = dd.cop;
  deta[1] = deta[2] = deta[3] = deta[4] = deta[5] = deta[6] = 0.0f;
  djj[0] = dd.cem;
  djj[1] = djj[2] = djj[3] = 0.0f;
  int c = 0;
  for (int j = 0; j < nlines; ++j) {
    const LineConst &L = lc[j];
    const LineDepth &q = ld[j];
    const LineTan &t = dl[j];
    // x0 = (delta - lam beta) inv_dld
    const float xd = delta[j] - lam.lam * d.beta;
    const float dx0 = -lam.lam * dd.beta * q.inv_dld + xd * t.inv_dld;
    if (!L.split) {
      const float *v = w + (size_t)c * wstride;
      const float dH = v[2] * dx0 + v[4] * t.a;
      deta[0] += t.opn * v[0] + q.opn * dH;
      djj[0] += t.emn * v[0] + q.emn * dH;
      ++c;
    } else {
      float Hs[3] = {0.f, 0.f, 0.f}, Fs[3] = {0.f, 0.f, 0.f}, dHs[3] = {0.f, 0.f, 0.f}, dFs[3] = {0.f, 0.f, 0.f};
      int off = L.comp_off;
      for (int g = 0; g < 3; ++g) {
        for (int i = 0; i < L.ncomp[g]; ++i, ++off, ++c) {
          const float *v = w + (size_t)c * wstride;
          const float dx = dx0 + compD[off] * t.bsh;
          const float S = compS[off];
          Hs[g] += v[0] * S;
          Fs[g] += v[1] * S;
          dHs[g] += (v[2] * dx + v[4] * t.a) * S;
          dFs[g] += (v[3] * dx + v[5] * t.a) * S;
        }
      }
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
  // H- bound-free + free-free and their LTE emissivity
  const float e1 = fexp(-lam.xs * d.invT);
  const float de1 = -lam.xs * e1 * dd.invT;
  const float opbf = lam.afud * d.hb * (1.0f - e1);
  const float dopbf = lam.afud * (dd.hb * (1.0f - e1) - d.hb * de1);
  const float E10 = fexp(kLn10 * (lam.F0 + lam.f1 * d.lt + lam.f2 * d.lt * d.lt));
  const float dE10 = E10 * kLn10 * (lam.f1 + 2.0f * lam.f2 * d.lt) * dd.lt;
  const float opff = d.hf * E10, dopff = dd.hf * E10 + d.hf * dE10;
  const float oph = opbf + opff, doph = dopbf + dopff;
  const float Ep = fexp(lam.xp * d.invT);
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
SNAPI_HD double opd_interior_jvp(double e_up, double e_c, double e_dn, double h1, double h2, double de_up,
                                 double de_c, double de_dn) {
  double gup = 0.0, gc = 0.0, gdn = 0.0;
  opd_interior_grad(e_up, e_c, e_dn, h1, h2, 1.0, gup, gc, gdn);
  return gup * de_up + gc * de_c + gdn * de_dn;
}

// tangent of bezier_dtau: dtau = dl/3 (e_b + e_a + (e_a + e_b)/2 + dl/4 (opd_b - opd_a))
SNAPI_HD double bezier_dtau_jvp(double de_below, double de_above, double dopd_below, double dopd_above, double dl) {
  return dl / 3.0 * (1.5 * (de_below + de_above) + 0.25 * dl * (dopd_below - dopd_above));
}

// tangent of delo_step: A Ic = B with A = 1 + w1 K'_c, B = -w0 K'_p I_p + w0 S_p + w1 S_c + etb I_p,
// so dIc = A^-1 (dB - dA Ic).  Ic: the forward result.
SNAPI_HD void delo_step_jvp(const float *Ip, const float *kpp, const float *Sp, const float *kpc, const float *Sc,
                            float tb, const float *Ic, const float *dIp, const float *dkpp, const float *dSp,
                            const float *dkpc, const float *dSc, float dtb, float *dIc) {
  float w0, w1, etb, gw0, gw1, getb;
  delo_weights(tb, w0, w1, etb);
  delo_weights_grad(tb, gw0, gw1, getb);
  const float dw0 = gw0 * dtb, dw1 = gw1 * dtb, detb = getb * dtb;
  float A[16], LU[16], r[4], t1[4], t2[4], t3[4], t4[4], t5[4];
  kp_mul(kpc, Ic, t1);    // K'_c Ic
  kp_mul(dkpc, Ic, t2);   // dK'_c Ic
  kp_mul(kpp, Ip, t3);    // K'_p Ip
  kp_mul(dkpp, Ip, t4);   // dK'_p Ip
  kp_mul(kpp, dIp, t5);   // K'_p dIp
#pragma unroll
  for (int s = 0; s < 4; ++s)
    r[s] = -dw0 * t3[s] - w0 * (t4[s] + t5[s]) + dw0 * Sp[s] + w0 * dSp[s] + dw1 * Sc[s] + w1 * dSc[s] +
           detb * Ip[s] + etb * dIp[s] - (dw1 * t1[s] + w1 * t2[s]);
  build_A(kpc, w1, false, A);
  crout4(A, LU);
  solve_crout4(LU, r, dIc);
}

}  // namespace snapi
