// snapi_core.cuh -- per-cell math of the B200 Stokes synthesis / adjoint path.
//
// Everything here is __host__ __device__ so that the CUDA kernels (snapi_cuda.cu) and the
// CPU emulator used by the tests run the same FP32 arithmetic.
//
// Physics follows the reference:
//   W4 Voigt-Faraday                  cmlib/profiles.cc:7-37
//   Zeeman pi / sigma assembly        atmos/atmol/atom/atom_rad_synthesis.cc:416-499
//   Thomson, bound-free, H-           atmos/atmos_rad_synthesis.cc:31-50,
//                                     atmos/atmol/atom/atom_rad_synthesis.cc:226-262,
//                                     atmos/atmol/mol/mol.cc:379-412, :516-632
//   normalisation by kappa_500        atmos/atmos_rad.cc:175-185
//   polarized linear-DELO step        atmos/plpar/atmos_ppbez_rts.cc:1055-1197 (w2 = 0 branch:
//                                     bezier_delimiter = 1e10 is never exceeded, :13, :1073)
//   Bezier optical depth              atmos/plpar/atmos_ppbez_rts.cc:962-988
// The adjoint functions are hand-written reverse-mode derivatives of exactly these forms
// (including the W4 region formulas, not the Faddeeva identity), so the gradient is the
// gradient of the forward model that is actually evaluated.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define SNAPI_HD __host__ __device__ __forceinline__
#else
#define SNAPI_HD inline
#endif
// The Voigt evaluations are the largest code blocks.  Each adjoint phase is its own kernel, so
// inlining them (one copy per call site) costs little instruction footprint and saves the call
// ABI's register traffic: 13 % on the synthesis, 10 % on the adjoint (measured on B200).  Set
// SNAPI_VOIGT_NOINLINE=1 to keep them out of line.
#ifndef SNAPI_VOIGT_NOINLINE
#define SNAPI_VOIGT_NOINLINE 0
#endif
#if defined(__CUDACC__) && SNAPI_VOIGT_NOINLINE
#define SNAPI_VOIGT_FN __host__ __device__ __noinline__
#elif defined(__CUDACC__)
#define SNAPI_VOIGT_FN __host__ __device__ __forceinline__
#else
#define SNAPI_VOIGT_FN inline
#endif

namespace snapi {

// ---------------------------------------------------------------------------------------------
// Column record layout (per pixel, depth-major [nd][nfield], nfield = 12 + 3*nlines)
enum RecField : int {
  F_T = 0, F_VT = 1, F_NE = 2, F_VLOS = 3, F_B = 4, F_INC = 5, F_AZI = 6, F_KAP = 7,
  F_HMBF = 8, F_HMFF = 9, F_BFOP = 10, F_BFEM = 11, F_LINE0 = 12
};
constexpr int kMaxLines = 16;
constexpr int kMaxComp = 16;      // per Zeeman group
constexpr int kNumRed = 10;       // depth-level adjoint sums that are not per line
constexpr int kRedPerLine = 6;    // per-line depth-level adjoint sums

// reduced adjoint vector per depth: [kNumRed + kRedPerLine*nlines]
enum RedIdx : int {
  R_COP = 0, R_CEM = 1, R_HB = 2, R_HF = 3, R_INVT = 4, R_LT = 5,
  R_ST2 = 6, R_CTB = 7, R_C2 = 8, R_S2 = 9
};
enum RedLine : int { RL_OPN = 0, RL_EMN = 1, RL_XL = 2, RL_XD = 3, RL_B = 4, RL_A = 5 };

// physical constants as the reference defines them (cmlib/const.h)
constexpr double kC = 2.99792458E10;
constexpr double kH = 6.6260687652E-27;
constexpr double kK = 1.3806503E-16;
constexpr double kPi = 3.141592653589793238462643383279502884197169399375105;
constexpr float kSqrtPiInv = 1.0f / 1.77245386399759f;
constexpr float kSigmaT = 6.65E-25f;
constexpr float kLn10 = 2.302585092994046f;

// per-line constants (identical for every pixel)
struct LineConst {
  double lam0;         // vacuum line centre [cm]
  float sf;            // lam0^2 / (4 pi c)
  float ar;            // radiative damping
  float two_k_over_m;  // 2 k / mass
  float lam0_over_c;
  float zee;           // 4.67e-5 * lam0^2 (Zeeman splitting per Gauss)
  int split;
  int ncomp[3];
  int comp_off;        // offset of this line's components in the component table
};

// per-wavelength constants of one thread
struct LamConst {
  float lam;           // vacuum wavelength [cm]
  float afud;          // H- bound-free alpha(lambda) * fudge
  float F0, f1, f2;    // H- free-free exponent coefficients (F0 includes log10(fudge))
  float xs;            // h c / (lambda k)  (stimulated emission)
  float xp;            // 1.4387769 / lambda (Planck)
  float pp;            // 2 h c^2 / lambda^5 (Planck prefactor, reference's constants)
};

// per-depth, per-pixel constants (wavelength independent), built from the record
struct DepthConst {
  float cop, cem;      // normalised flat continuum opacity / emissivity
  float beta;          // v_los / c
  float st2, ctb, opc2, c2, s2;  // sin^2 theta_B, cos theta_B, 1+cos^2, cos 2phi, sin 2phi
  float hb, hf;        // H- bound-free / free-free depth factors (normalised)
  float invT, lt;      // 1/T, log10(5040/T)
};
struct LineDepth {
  float inv_dld, a, bsh, opn, emn;
};

// ---------------------------------------------------------------------------------------------
// small complex helpers (the reference's own formulation of * and /, cmlib/types.h:28-55)
struct cf { float re, im; };
SNAPI_HD cf cmk(float r, float i) { cf z; z.re = r; z.im = i; return z; }
SNAPI_HD cf cadd(cf a, cf b) { return cmk(a.re + b.re, a.im + b.im); }
SNAPI_HD cf csub(cf a, cf b) { return cmk(a.re - b.re, a.im - b.im); }
SNAPI_HD cf cmul(cf a, cf b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
SNAPI_HD float frcp(float x);
SNAPI_HD cf cdiv(cf a, cf b) {
  const float r = frcp(b.re * b.re + b.im * b.im);
  return cmk((a.re * b.re + a.im * b.im) * r, (a.im * b.re - a.re * b.im) * r);
}
SNAPI_HD cf caddr(float a, cf b) { return cmk(b.re + a, b.im); }
SNAPI_HD cf csubr(float a, cf b) { return cmk(a - b.re, -b.im); }
SNAPI_HD cf cscl(cf a, float s) { return cmk(a.re * s, a.im * s); }
struct cd { double re, im; };
SNAPI_HD cd dmk(double r, double i) { cd z; z.re = r; z.im = i; return z; }
SNAPI_HD cd dadd(cd a, cd b) { return dmk(a.re + b.re, a.im + b.im); }
SNAPI_HD cd dsub(cd a, cd b) { return dmk(a.re - b.re, a.im - b.im); }
SNAPI_HD cd dmul(cd a, cd b) { return dmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
SNAPI_HD cd ddiv(cd a, cd b) {
  double f = b.re * b.re + b.im * b.im;
  return dmk((a.re * b.re + a.im * b.im) / f, (a.im * b.re - a.re * b.im) / f);
}
SNAPI_HD cd daddr(double a, cd b) { return dmk(b.re + a, b.im); }
SNAPI_HD cd dsubr(double a, cd b) { return dmk(a - b.re, -b.im); }
SNAPI_HD cd dscl(cd a, double s) { return dmk(a.re * s, a.im * s); }

// Transcendentals of the per-cell math.  On the device the SFU forms are used: their error
// (about 2 ulp for exp; for sin / cos an absolute error ~1e-6 |x| / pi, with |x| < 10 in W4 region 4
// where the factor e^{a^2 - v^2} multiplying them is < 2e-4 whenever |x| > 2) stays far below
// the FP32 rounding of the sums they feed.  frcp (the reciprocal of |d|^2 in the complex divisions) is
// the SFU reciprocal (__fdividef, within 2 ulp for |x| < 2^126; |d|^2 < 1e22 in W4): replacing the
// correctly rounded one made the adjoint call 6 % faster and the synthesis 15 %, with the parity
// tests unchanged.  The library is built with -prec-div=false -prec-sqrt=false, so the other FP32
// divisions and square roots (DELO weights, source functions, the 4x4 solves) take the SFU forms
// too (another 7 %).
#ifdef __CUDA_ARCH__
SNAPI_HD float fexp(float x) { return __expf(x); }
SNAPI_HD void fsincos(float x, float *s, float *c) { __sincosf(x, s, c); }
SNAPI_HD float frcp(float x) { return __fdividef(1.0f, x); }
#else
SNAPI_HD float fexp(float x) { return expf(x); }
SNAPI_HD void fsincos(float x, float *s, float *c) { *s = sinf(x); *c = cosf(x); }
SNAPI_HD float frcp(float x) { return 1.0f / x; }
#endif

// Humlicek W4 (published region split and coefficients); H, F divided by sqrt(pi).
SNAPI_VOIGT_FN void voigt(float x, float a, float &H, float &F) {
  const float v = x;
  const float s = fabsf(v) + a;
  const cf t = cmk(a, -v);
  const cf u = cmk(a * a - v * v, -2.0f * a * v);
  cf w4;
  if (s >= 15.0f) {
    w4 = cdiv(cscl(t, 0.5641896f), caddr(0.5f, u));
  } else if (s > 5.5f) {
    w4 = cdiv(cmul(t, caddr(1.410474f, cscl(u, 0.5641896f))), caddr(0.75f, cmul(u, caddr(3.0f, u))));
  } else if (a > (0.195f * fabsf(v) - 0.176f)) {
    cf n = caddr(3.778987f, cscl(t, 0.5642236f));
    n = caddr(11.96482f, cmul(t, n));
    n = caddr(20.20933f, cmul(t, n));
    n = caddr(16.4955f, cmul(t, n));
    cf d = caddr(6.699398f, t);
    d = caddr(21.69274f, cmul(t, d));
    d = caddr(39.27121f, cmul(t, d));
    d = caddr(38.82363f, cmul(t, d));
    d = caddr(16.4955f, cmul(t, d));
    w4 = cdiv(n, d);
  } else {
    cf p = csubr(1.320522f, cscl(u, 0.56419f));
    p = csubr(35.76683f, cmul(u, p));
    p = csubr(219.0313f, cmul(u, p));
    p = csubr(1540.787f, cmul(u, p));
    p = csubr(3321.9905f, cmul(u, p));
    p = csubr(36183.31f, cmul(u, p));
    cf q = csubr(1.841439f, u);
    q = csubr(61.57037f, cmul(u, q));
    q = csubr(364.2191f, cmul(u, q));
    q = csubr(2186.181f, cmul(u, q));
    q = csubr(9022.228f, cmul(u, q));
    q = csubr(24322.84f, cmul(u, q));
    q = csubr(32066.6f, cmul(u, q));
    float su, cu;
    fsincos(u.im, &su, &cu);
    const float eu = fexp(u.re);
    w4 = csub(cmk(eu * sqrtf(1.0f - su * su), eu * su), cdiv(cmul(t, p), q));
  }
  H = w4.re * kSqrtPiInv;
  F = w4.im * kSqrtPiInv;
}

// Region 4 of W4 with its exact derivatives.  With R = t p(u)/q(u) the derivative is written as
// r = p/q, r' = (p' - r q')/q, dR/dt = r + 2u r', which keeps every intermediate within FP32
// range (|q| < 3e10 in this region; forming q^2 and dividing by it would overflow).
SNAPI_VOIGT_FN void voigt_grad_core(float a, float v, cf &w4, cf &dwa, cf &dwv) {
  const cf t = cmk(a, -v);
  const cf u = cmk(a * a - v * v, -2.0f * a * v);
  cf p = csubr(1.320522f, cscl(u, 0.56419f));
  p = csubr(35.76683f, cmul(u, p));
  p = csubr(219.0313f, cmul(u, p));
  p = csubr(1540.787f, cmul(u, p));
  p = csubr(3321.9905f, cmul(u, p));
  p = csubr(36183.31f, cmul(u, p));
  // p(u) = c0 - c1 u + c2 u^2 - c3 u^3 + c4 u^4 - c5 u^5 + c6 u^6
  // p'(u) = -c1 + 2 c2 u - 3 c3 u^2 + 4 c4 u^3 - 5 c5 u^4 + 6 c6 u^5
  cf pp = cmk(6.0f * 0.56419f, 0.0f);
  pp = caddr(-5.0f * 1.320522f, cmul(u, pp));
  pp = caddr(4.0f * 35.76683f, cmul(u, pp));
  pp = caddr(-3.0f * 219.0313f, cmul(u, pp));
  pp = caddr(2.0f * 1540.787f, cmul(u, pp));
  pp = caddr(-3321.9905f, cmul(u, pp));
  cf q = csubr(1.841439f, u);
  q = csubr(61.57037f, cmul(u, q));
  q = csubr(364.2191f, cmul(u, q));
  q = csubr(2186.181f, cmul(u, q));
  q = csubr(9022.228f, cmul(u, q));
  q = csubr(24322.84f, cmul(u, q));
  q = csubr(32066.6f, cmul(u, q));
  // q(u) = d0 - d1 u + d2 u^2 - d3 u^3 + d4 u^4 - d5 u^5 + d6 u^6 - u^7
  cf qp = cmk(-7.0f, 0.0f);
  qp = caddr(6.0f * 1.841439f, cmul(u, qp));
  qp = caddr(-5.0f * 61.57037f, cmul(u, qp));
  qp = caddr(4.0f * 364.2191f, cmul(u, qp));
  qp = caddr(-3.0f * 2186.181f, cmul(u, qp));
  qp = caddr(2.0f * 9022.228f, cmul(u, qp));
  qp = caddr(-24322.84f, cmul(u, qp));
  float su, cu;
  fsincos(u.im, &su, &cu);
  const float eu = fexp(u.re);
  const float ca = sqrtf(1.0f - su * su);
  const cf r = cdiv(p, q);
  const cf rp = cdiv(csub(pp, cmul(r, qp)), q);
  const cf R = cmul(t, r);
  const cf E = cmk(eu * ca, eu * su);
  w4 = csub(E, R);
  const cf Rp = cadd(r, cmul(cscl(u, 2.0f), rp));
  // E = e^{ur} (|cos ui|, sin ui): dE/dur = E, dE/dui = e^{ur} (-sgn(cos ui) sin ui, cos ui)
  const float sg = (cu > 0.0f) ? 1.0f : ((cu < 0.0f) ? -1.0f : 0.0f);
  const cf Eui = cmk(-eu * sg * su, eu * cu);
  // ur = a^2 - v^2, ui = -2 a v, dt/da = 1, dt/dv = -i
  dwa = csub(cadd(cscl(E, 2.0f * a), cscl(Eui, -2.0f * v)), Rp);
  const cf Rv = cmk(Rp.im, -Rp.re);
  dwv = csub(cadd(cscl(E, -2.0f * v), cscl(Eui, -2.0f * a)), Rv);
}

// W4 with its exact partial derivatives with respect to x (= v) and a.
SNAPI_VOIGT_FN void voigt_grad(float x, float a, float &H, float &F, float &Hx, float &Fx, float &Ha, float &Fa) {
  const float v = x;
  const float s = fabsf(v) + a;
  const cf t = cmk(a, -v);
  const cf u = cmk(a * a - v * v, -2.0f * a * v);
  cf w4, dwa, dwv;  // dw/da, dw/dv
  if (s >= 15.0f || s > 5.5f || a > (0.195f * fabsf(v) - 0.176f)) {
    cf n, np, d, dp;  // numerator / denominator as functions of t, and d/dt
    if (s >= 15.0f) {
      n = cscl(t, 0.5641896f);
      np = cmk(0.5641896f, 0.0f);
      d = caddr(0.5f, u);
      dp = cscl(t, 2.0f);
    } else if (s > 5.5f) {
      n = cmul(t, caddr(1.410474f, cscl(u, 0.5641896f)));
      np = caddr(1.410474f, cscl(u, 3.0f * 0.5641896f));
      d = caddr(0.75f, cmul(u, caddr(3.0f, u)));
      dp = cmul(t, caddr(6.0f, cscl(u, 4.0f)));
    } else {
      n = caddr(3.778987f, cscl(t, 0.5642236f));
      n = caddr(11.96482f, cmul(t, n));
      n = caddr(20.20933f, cmul(t, n));
      n = caddr(16.4955f, cmul(t, n));
      np = caddr(3.0f * 3.778987f, cscl(t, 4.0f * 0.5642236f));
      np = caddr(2.0f * 11.96482f, cmul(t, np));
      np = caddr(20.20933f, cmul(t, np));
      d = caddr(6.699398f, t);
      d = caddr(21.69274f, cmul(t, d));
      d = caddr(39.27121f, cmul(t, d));
      d = caddr(38.82363f, cmul(t, d));
      d = caddr(16.4955f, cmul(t, d));
      dp = caddr(4.0f * 6.699398f, cscl(t, 5.0f));
      dp = caddr(3.0f * 21.69274f, cmul(t, dp));
      dp = caddr(2.0f * 39.27121f, cmul(t, dp));
      dp = caddr(38.82363f, cmul(t, dp));
    }
    w4 = cdiv(n, d);
    // w' = (n' d - n d') / d^2 = (n' - w d') / d
    cf wp = cdiv(csub(np, cmul(w4, dp)), d);
    dwa = wp;                        // dt/da = 1
    dwv = cmk(wp.im, -wp.re);        // dt/dv = -i
  } else {
    voigt_grad_core(a, v, w4, dwa, dwv);
  }
  H = w4.re * kSqrtPiInv;
  F = w4.im * kSqrtPiInv;
  Hx = dwv.re * kSqrtPiInv;
  Fx = dwv.im * kSqrtPiInv;
  Ha = dwa.re * kSqrtPiInv;
  Fa = dwa.im * kSqrtPiInv;
}

// ---------------------------------------------------------------------------------------------
// Planck function with the reference's constants (cmlib/mathtools.cc:1150-1152), lambda in cm
SNAPI_HD double planck_d(double lam, double T) {
  return 2.0 * 6.62606957 * 8.9875517E-7 / lam / lam / lam / lam / lam / (exp(1.4387769 / lam / T) - 1.0);
}

// per-depth precompute from the record row rec[nfield]; lam_mid: mid vacuum wavelength
SNAPI_HD void depth_precompute(const float *rec, int nlines, const LineConst *lc, float lam_mid,
                               DepthConst &d, LineDepth *ld) {
  const float T = rec[F_T], vt = rec[F_VT], ne = rec[F_NE], B = rec[F_B];
  const float invk = 1.0f / rec[F_KAP];
  const float xpm = 1.4387769f / lam_mid;
  const float Em = fexp(xpm / T);
  const float plm = (float)(2.0 * 6.62606957 * 8.9875517E-7) / (lam_mid * lam_mid * lam_mid * lam_mid * lam_mid) / (Em - 1.0f);
  const float ope = ne * kSigmaT;
  d.cop = (ope + rec[F_BFOP]) * invk;
  d.cem = (ope * plm + rec[F_BFEM]) * invk;
  d.beta = rec[F_VLOS] * (float)(1.0 / kC);
  float th = rec[F_INC] * (float)(kPi / 180.0), ph = rec[F_AZI] * (float)(kPi / 180.0);
  if (B < 0.001f) th = ph = 0.0f;
  float sth, cth, s2p, c2p;
  fsincos(th, &sth, &cth);
  fsincos(2.0f * ph, &s2p, &c2p);
  d.st2 = sth * sth;
  d.ctb = cth;
  d.opc2 = 1.0f + cth * cth;
  d.c2 = c2p;
  d.s2 = s2p;
  d.hb = rec[F_HMBF] * invk;
  d.hf = rec[F_HMFF] * invk;
  d.invT = 1.0f / T;
  d.lt = log10f(5040.0f / T);
  for (int j = 0; j < nlines; ++j) {
    const LineConst &L = lc[j];
    const float *rl = rec + F_LINE0 + 3 * j;
    const float W = L.two_k_over_m * T + vt * vt;
    const float dld = sqrtf(W) * L.lam0_over_c;
    const float idl = 1.0f / dld;
    ld[j].inv_dld = idl;
    ld[j].a = L.sf * (L.ar + rl[2]) * idl;
    ld[j].bsh = L.zee * B * idl;
    ld[j].opn = rl[0] * invk * idl;
    ld[j].emn = rl[1] * invk * idl;
  }
}

// per-wavelength constants; lam_vac in cm (double)
SNAPI_HD void lambda_precompute(double lam, LamConst &c) {
  static const double ca[7] = {1.99654, -1.18267E-5, 2.64243E-6, -4.40524E-10, 3.23992E-14,
                               -1.39568E-18, 2.78701E-23};
  double lA = lam * 1E8, alpha = 0.0, pw = 1.0;
  for (int i = 0; i < 7; ++i) { alpha += ca[i] * pw; pw *= lA; }
  double lb = 2.1177 * exp(-(lA - 2087.7) * (lA - 2087.7) / 2.421E6) + 0.68738;
  if (lA > 4500.0) lb = 0.0;
  double fud = 1.0 + 0.666667 * lb;
  double l = log10(lA);
  double f0 = -2.2763 - 1.6850 * l + 0.76661 * l * l - 0.053346 * l * l * l;
  double f1 = 15.2827 - 9.2846 * l + 1.99381 * l * l - 0.142631 * l * l * l;
  double f2 = -197.789 + 190.266 * l - 67.9775 * l * l + 10.6913 * l * l * l - 0.625151 * l * l * l * l;
  c.lam = (float)lam;
  c.afud = (float)(alpha * fud);
  c.F0 = (float)(f0 + log10(fud));
  c.f1 = (float)f1;
  c.f2 = (float)f2;
  c.xs = (float)(kH * kC / lam / kK);
  c.xp = (float)(1.4387769 / lam);
  c.pp = (float)(2.0 * 6.62606957 * 8.9875517E-7 / lam / lam / lam / lam / lam);
}

// ---------------------------------------------------------------------------------------------
// Opacity (eta_I, eta_Q, eta_U, eta_V, rho_Q, rho_U, rho_V) and emissivity (j_I..j_V), both
// normalised by kappa_500, at one (lambda, depth).  delta[j] = lam0_j - lambda (FP64 -> FP32).
SNAPI_HD void cell_opacity(const DepthConst &d, const LineDepth *ld, const LineConst *lc, int nlines,
                           const float *compS, const float *compD, const LamConst &lc_l,
                           const float *delta, float *eta, float *jj) {
  eta[0] = d.cop;
  eta[1] = eta[2] = eta[3] = eta[4] = eta[5] = eta[6] = 0.0f;
  jj[0] = d.cem;
  jj[1] = jj[2] = jj[3] = 0.0f;
  for (int j = 0; j < nlines; ++j) {
    const LineConst &L = lc[j];
    const LineDepth &q = ld[j];
    const float x0 = (delta[j] - lc_l.lam * d.beta) * q.inv_dld;
    if (!L.split) {
      float H, F;
      voigt(x0, q.a, H, F);
      eta[0] += q.opn * H;
      jj[0] += q.emn * H;
    } else {
      float Hs[3] = {0.f, 0.f, 0.f}, Fs[3] = {0.f, 0.f, 0.f};
      int off = L.comp_off;
      for (int g = 0; g < 3; ++g) {
        for (int i = 0; i < L.ncomp[g]; ++i, ++off) {
          float H, F;
          voigt(x0 + compD[off] * q.bsh, q.a, H, F);
          Hs[g] += H * compS[off];
          Fs[g] += F * compS[off];
        }
      }
      const float hpm = Hs[0] - 0.5f * (Hs[2] + Hs[1]);
      const float fpm = Fs[0] - 0.5f * (Fs[2] + Fs[1]);
      const float eI = 0.5f * (Hs[0] * d.st2 + 0.5f * (Hs[2] + Hs[1]) * d.opc2);
      const float eQ = 0.5f * hpm * d.st2 * d.c2;
      const float eU = 0.5f * hpm * d.st2 * d.s2;
      const float eV = 0.5f * (Hs[2] - Hs[1]) * d.ctb;
      const float rQ = 0.5f * fpm * d.st2 * d.c2;
      const float rU = 0.5f * fpm * d.st2 * d.s2;
      const float rV = 0.5f * (Fs[2] - Fs[1]) * d.ctb;
      eta[0] += eI * q.opn; eta[1] += eQ * q.opn; eta[2] += eU * q.opn; eta[3] += eV * q.opn;
      eta[4] += rQ * q.opn; eta[5] += rU * q.opn; eta[6] += rV * q.opn;
      jj[0] += eI * q.emn; jj[1] += eQ * q.emn; jj[2] += eU * q.emn; jj[3] += eV * q.emn;
    }
  }
  // H- bound-free + free-free, LTE emissivity
  const float e1 = fexp(-lc_l.xs * d.invT);
  const float opbf = lc_l.afud * d.hb * (1.0f - e1);
  const float E10 = fexp(kLn10 * (lc_l.F0 + lc_l.f1 * d.lt + lc_l.f2 * d.lt * d.lt));
  const float opff = d.hf * E10;
  const float oph = opbf + opff;
  const float Ep = fexp(lc_l.xp * d.invT);
  const float pl = lc_l.pp / (Ep - 1.0f);
  eta[0] += oph;
  jj[0] += oph * pl;
}

// Reverse of cell_opacity: given eta_bar[7], j_bar[4] accumulate the depth-level adjoint sums
// red[kNumRed + kRedPerLine*nlines] (wavelength-summed later).
// Opacity adjoint of transition j at one (lambda, depth): adds the six per-line sums rl[RL_*] and
// the four angle sums ang[] (st2, ctb, c2, s2).  lam = (float) vacuum wavelength, delta_j =
// lam0_j - lambda (FP64 -> FP32).
SNAPI_HD void line_opacity_adjoint(const DepthConst &d, const LineDepth &q, const LineConst &L, const float *compS,
                                   const float *compD, float lam, float delta_j, const float *etab, const float *jb,
                                   float *rl, float *ang) {
  const float xd = delta_j - lam * d.beta;
  const float x0 = xd * q.inv_dld;
  float x0b = 0.f, bb = 0.f, ab = 0.f;
  if (!L.split) {
    float H, F, Hx, Fx, Ha, Fa;
    voigt_grad(x0, q.a, H, F, Hx, Fx, Ha, Fa);
    rl[RL_OPN] += etab[0] * H;
    rl[RL_EMN] += jb[0] * H;
    const float Hb_ = q.opn * etab[0] + q.emn * jb[0];
    x0b += Hb_ * Hx;
    ab += Hb_ * Ha;
  } else {
    // adjoints of the component sums depend only on (eta-bar, j-bar) and the angles, so one
    // pass of voigt_grad per component gives both the sums and the x / a adjoints
    float Pb[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) Pb[k] = q.opn * etab[k] + (k < 4 ? q.emn * jb[k] : 0.0f);
    const float hpmb = 0.5f * d.st2 * (d.c2 * Pb[1] + d.s2 * Pb[2]);
    const float fpmb = 0.5f * d.st2 * (d.c2 * Pb[4] + d.s2 * Pb[5]);
    float Hsb[3], Fsb[3];
    Hsb[0] = 0.5f * d.st2 * Pb[0] + hpmb;
    Hsb[1] = 0.25f * d.opc2 * Pb[0] - 0.5f * hpmb - 0.5f * d.ctb * Pb[3];
    Hsb[2] = 0.25f * d.opc2 * Pb[0] - 0.5f * hpmb + 0.5f * d.ctb * Pb[3];
    Fsb[0] = fpmb;
    Fsb[1] = -0.5f * fpmb - 0.5f * d.ctb * Pb[6];
    Fsb[2] = -0.5f * fpmb + 0.5f * d.ctb * Pb[6];
    float Hs[3] = {0.f, 0.f, 0.f}, Fs[3] = {0.f, 0.f, 0.f};
    int off = L.comp_off;
#pragma unroll
    for (int g = 0; g < 3; ++g)
      for (int i = 0; i < L.ncomp[g]; ++i, ++off) {
        float H, F, Hx, Fx, Ha, Fa;
        voigt_grad(x0 + compD[off] * q.bsh, q.a, H, F, Hx, Fx, Ha, Fa);
        const float S = compS[off];
        Hs[g] += H * S;
        Fs[g] += F * S;
        const float hb_ = Hsb[g] * S, fb_ = Fsb[g] * S;
        const float xb = hb_ * Hx + fb_ * Fx;
        x0b += xb;
        bb += xb * compD[off];
        ab += hb_ * Ha + fb_ * Fa;
      }
    const float hpm = Hs[0] - 0.5f * (Hs[2] + Hs[1]);
    const float fpm = Fs[0] - 0.5f * (Fs[2] + Fs[1]);
    const float P[7] = {0.5f * (Hs[0] * d.st2 + 0.5f * (Hs[2] + Hs[1]) * d.opc2),
                        0.5f * hpm * d.st2 * d.c2,
                        0.5f * hpm * d.st2 * d.s2,
                        0.5f * (Hs[2] - Hs[1]) * d.ctb,
                        0.5f * fpm * d.st2 * d.c2,
                        0.5f * fpm * d.st2 * d.s2,
                        0.5f * (Fs[2] - Fs[1]) * d.ctb};
    float gop = 0.f, gem = 0.f;
#pragma unroll
    for (int k = 0; k < 7; ++k) gop += etab[k] * P[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) gem += jb[k] * P[k];
    rl[RL_OPN] += gop;
    rl[RL_EMN] += gem;
    ang[0] += 0.5f * Hs[0] * Pb[0] + 0.5f * hpm * (d.c2 * Pb[1] + d.s2 * Pb[2]) +
              0.5f * fpm * (d.c2 * Pb[4] + d.s2 * Pb[5]);
    ang[1] += 2.0f * d.ctb * (0.25f * (Hs[2] + Hs[1]) * Pb[0]) + 0.5f * (Hs[2] - Hs[1]) * Pb[3] +
              0.5f * (Fs[2] - Fs[1]) * Pb[6];
    ang[2] += 0.5f * d.st2 * (hpm * Pb[1] + fpm * Pb[4]);
    ang[3] += 0.5f * d.st2 * (hpm * Pb[2] + fpm * Pb[5]);
  }
  rl[RL_XL] += x0b * lam;
  rl[RL_XD] += x0b * xd;
  rl[RL_B] += bb;
  rl[RL_A] += ab;
}

// Continuum part of the opacity adjoint (Thomson + bound-free totals, H-): adds red[R_COP..R_LT].
SNAPI_HD void continuum_opacity_adjoint(const DepthConst &d, const LamConst &lc_l, float etab0, float jb0,
                                        float *red) {
  red[R_COP] += etab0;
  red[R_CEM] += jb0;
  const float e1 = fexp(-lc_l.xs * d.invT);
  const float E10 = fexp(kLn10 * (lc_l.F0 + lc_l.f1 * d.lt + lc_l.f2 * d.lt * d.lt));
  const float oph = lc_l.afud * d.hb * (1.0f - e1) + d.hf * E10;
  const float Ep = fexp(lc_l.xp * d.invT);
  const float pl = lc_l.pp / (Ep - 1.0f);
  const float ophb = etab0 + jb0 * pl;
  const float plb = jb0 * oph;
  red[R_HB] += ophb * lc_l.afud * (1.0f - e1);
  red[R_HF] += ophb * E10;
  red[R_INVT] += ophb * lc_l.afud * d.hb * lc_l.xs * e1 - plb * pl * lc_l.xp * Ep / (Ep - 1.0f);
  red[R_LT] += ophb * d.hf * E10 * kLn10 * (lc_l.f1 + 2.0f * lc_l.f2 * d.lt);
}

// Adjoint of cell_opacity at one (lambda, depth): adds every depth sum of red[] (continuum, angle
// and per-line terms).
SNAPI_HD void cell_opacity_adjoint(const DepthConst &d, const LineDepth *ld, const LineConst *lc, int nlines,
                                   const float *compS, const float *compD, const LamConst &lc_l,
                                   const float *delta, const float *etab, const float *jb, float *red) {
  for (int j = 0; j < nlines; ++j)
    line_opacity_adjoint(d, ld[j], lc[j], compS, compD, lc_l.lam, delta[j], etab, jb, red + kNumRed + kRedPerLine * j,
                         red + R_ST2);
  continuum_opacity_adjoint(d, lc_l, etab[0], jb[0], red);
}

// Chain the wavelength-summed depth adjoint sums red[] to the record fields (adds into rb[nfield]).
SNAPI_HD void depth_chain_adjoint(const float *rec, int nlines, const LineConst *lc, float lam_mid,
                                  const DepthConst &d, const LineDepth *ld, const float *red, float *rb) {
  const float T = rec[F_T], vt = rec[F_VT], ne = rec[F_NE], B = rec[F_B];
  const float invk = 1.0f / rec[F_KAP];
  const float xpm = 1.4387769f / lam_mid;
  const float Em = fexp(xpm / T);
  const float plm = (float)(2.0 * 6.62606957 * 8.9875517E-7) / (lam_mid * lam_mid * lam_mid * lam_mid * lam_mid) / (Em - 1.0f);
  const float dplm_dT = plm * xpm * Em / (Em - 1.0f) / (T * T);
  float Tb = 0.f, vtb = 0.f, kapb = 0.f, Bb = 0.f, betab = 0.f;
  // continuum
  rb[F_NE] += red[R_COP] * kSigmaT * invk + red[R_CEM] * kSigmaT * plm * invk;
  rb[F_BFOP] += red[R_COP] * invk;
  rb[F_BFEM] += red[R_CEM] * invk;
  kapb -= (red[R_COP] * d.cop + red[R_CEM] * d.cem) * invk;
  Tb += red[R_CEM] * ne * kSigmaT * dplm_dT * invk;
  // H-
  rb[F_HMBF] += red[R_HB] * invk;
  rb[F_HMFF] += red[R_HF] * invk;
  kapb -= (red[R_HB] * d.hb + red[R_HF] * d.hf) * invk;
  Tb += -red[R_INVT] * d.invT * d.invT - red[R_LT] / (T * kLn10);
  // angles
  if (!(B < 0.001f)) {
    const float th = rec[F_INC] * (float)(kPi / 180.0), ph = rec[F_AZI] * (float)(kPi / 180.0);
    float sth, cth, s2p, c2p;
    fsincos(th, &sth, &cth);
    fsincos(2.0f * ph, &s2p, &c2p);
    const float dr = (float)(kPi / 180.0);
    rb[F_INC] += (red[R_ST2] * 2.0f * sth * cth - red[R_CTB] * sth) * dr;
    rb[F_AZI] += (-red[R_C2] * 2.0f * s2p + red[R_S2] * 2.0f * c2p) * dr;
  }
  // lines
  for (int j = 0; j < nlines; ++j) {
    const LineConst &L = lc[j];
    const LineDepth &q = ld[j];
    const float *rl = red + kNumRed + kRedPerLine * j;
    const float *rec_l = rec + F_LINE0 + 3 * j;
    const float opnb = rl[RL_OPN], emnb = rl[RL_EMN], ab = rl[RL_A], bshb = rl[RL_B];
    betab += -q.inv_dld * rl[RL_XL];
    float idlb = rl[RL_XD];
    idlb += ab * L.sf * (L.ar + rec_l[2]);
    idlb += bshb * L.zee * B;
    idlb += opnb * rec_l[0] * invk + emnb * rec_l[1] * invk;
    const float W = L.two_k_over_m * T + vt * vt;
    // inv_dld = 1/(sqrt(W) lam0/c): d/dW = -0.5 inv_dld / W
    const float dW = -0.5f * q.inv_dld / W * idlb;
    Tb += dW * L.two_k_over_m;
    vtb += dW * 2.0f * vt;
    Bb += bshb * L.zee * q.inv_dld;
    float *rbl = rb + F_LINE0 + 3 * j;
    rbl[0] += opnb * invk * q.inv_dld;
    rbl[1] += emnb * invk * q.inv_dld;
    rbl[2] += ab * L.sf * q.inv_dld;
    kapb -= (opnb * q.opn + emnb * q.emn) * invk;
  }
  rb[F_T] += Tb;
  rb[F_VT] += vtb;
  rb[F_KAP] += kapb;
  rb[F_B] += Bb;
  rb[F_VLOS] += betab * (float)(1.0 / kC);
}

// ---------------------------------------------------------------------------------------------
// Reduced absorption matrix K' = K/eta_I - 1 from the 7 opacities: kp = (q,u,v,rq,ru,rv)
//   K' = [[0, q, u, v], [q, 0, rv, -ru], [u, -rv, 0, rq], [v, ru, -rq, 0]]
SNAPI_HD void kprime_full(const float *kp, float *M) {
  M[0] = 0.f;   M[1] = kp[0];  M[2] = kp[1];  M[3] = kp[2];
  M[4] = kp[0]; M[5] = 0.f;    M[6] = kp[5];  M[7] = -kp[4];
  M[8] = kp[1]; M[9] = -kp[5]; M[10] = 0.f;  M[11] = kp[3];
  M[12] = kp[2]; M[13] = kp[4]; M[14] = -kp[3]; M[15] = 0.f;
}
// adjoint of kprime_full: accumulate d<Mb, K'>/dkp
SNAPI_HD void kprime_proj(const float *Mb, float *kpb) {
  kpb[0] += Mb[1] + Mb[4];
  kpb[1] += Mb[2] + Mb[8];
  kpb[2] += Mb[3] + Mb[12];
  kpb[3] += Mb[11] - Mb[14];
  kpb[4] += Mb[13] - Mb[7];
  kpb[5] += Mb[6] - Mb[9];
}

// Crout LU without pivoting, unit upper diagonal (cmlib/mathtools.cc:487-514)
SNAPI_HD void crout4(const float *S, float *D) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
#pragma unroll
    for (int i = k; i < 4; ++i) {
      float sum = 0.f;
#pragma unroll
      for (int p = 0; p < k; ++p) sum += D[i * 4 + p] * D[p * 4 + k];
      D[i * 4 + k] = S[i * 4 + k] - sum;
    }
#pragma unroll
    for (int j = k + 1; j < 4; ++j) {
      float sum = 0.f;
#pragma unroll
      for (int p = 0; p < k; ++p) sum += D[k * 4 + p] * D[p * 4 + j];
      D[k * 4 + j] = (S[k * 4 + j] - sum) * frcp(D[k * 4 + k]);
    }
  }
}
SNAPI_HD void solve_crout4(const float *LU, const float *b, float *x) {
  float y[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float sum = 0.f;
#pragma unroll
    for (int k = 0; k < i; ++k) sum += LU[i * 4 + k] * y[k];
    y[i] = (b[i] - sum) * frcp(LU[i * 4 + i]);
  }
#pragma unroll
  for (int i = 3; i >= 0; --i) {
    float sum = 0.f;
#pragma unroll
    for (int k = i + 1; k < 4; ++k) sum += LU[i * 4 + k] * x[k];
    x[i] = (y[i] - sum);
  }
}

// linear DELO weights (atmos_ppbez_rts.cc:1070, :1085-1096).  Below tb = 1e-2 the reference's own
// three-term expansion.  Above it the closed forms 1/tb - e^-tb (1 + 1/tb) and 1 - 1/tb + e^-tb/tb
// cancel to ~tb/2 from terms of size 1/tb, so up to tb = 0.5 they are evaluated by their exact
// power series (w0 = sum_k (-1)^(k+1) k/(k+1)! tb^k, w1 = sum_k (-1)^(k+1) tb^k/(k+1)!, truncated
// after the tb^11 term: < 1e-11 relative), above that by the closed forms (cancellation <= 16x).
SNAPI_HD void delo_weights(float tb, float &w0, float &w1, float &etb) {
  if (tb < 1E-2f) {
    etb = 1.0f - tb + tb * tb * 0.5f - tb * tb * tb / 6.0f;
    w0 = tb * (0.5f - tb * (1.0f / 3.0f - tb / 8.0f));
    w1 = 0.5f * tb * (1.0f - tb / 3.0f * (1.0f - tb / 4.0f));
  } else if (tb < 0.5f) {
    etb = fexp(-tb);
    // coefficients of tb^k, k = 11 .. 1
    float a = -11.0f / 479001600.0f, b = -1.0f / 479001600.0f;
    a = a * tb + 10.0f / 39916800.0f;  b = b * tb + 1.0f / 39916800.0f;
    a = a * tb - 9.0f / 3628800.0f;    b = b * tb - 1.0f / 3628800.0f;
    a = a * tb + 8.0f / 362880.0f;     b = b * tb + 1.0f / 362880.0f;
    a = a * tb - 7.0f / 40320.0f;      b = b * tb - 1.0f / 40320.0f;
    a = a * tb + 6.0f / 5040.0f;       b = b * tb + 1.0f / 5040.0f;
    a = a * tb - 5.0f / 720.0f;        b = b * tb - 1.0f / 720.0f;
    a = a * tb + 4.0f / 120.0f;        b = b * tb + 1.0f / 120.0f;
    a = a * tb - 3.0f / 24.0f;         b = b * tb - 1.0f / 24.0f;
    a = a * tb + 2.0f / 6.0f;          b = b * tb + 1.0f / 6.0f;
    a = a * tb - 0.5f;                 b = b * tb - 0.5f;
    w0 = -a * tb;
    w1 = -b * tb;
  } else {
    etb = fexp(-tb);
    const float it = frcp(tb);
    w0 = it - etb * (1.0f + it);
    w1 = 1.0f - it + etb * it;
  }
}
SNAPI_HD void delo_weights_grad(float tb, float &dw0, float &dw1, float &detb) {
  if (tb < 1E-2f) {
    detb = -1.0f + tb - 0.5f * tb * tb;
    dw0 = 0.5f - tb * (2.0f / 3.0f - 3.0f * tb / 8.0f);
    dw1 = 0.5f - tb / 3.0f + tb * tb / 8.0f;
  } else if (tb < 0.5f) {
    detb = -fexp(-tb);
    // d/dtb of the series above: sum_k (-1)^(k+1) k^2/(k+1)! tb^(k-1), sum_k (-1)^(k+1) k/(k+1)! tb^(k-1)
    float a = -121.0f / 479001600.0f, b = -11.0f / 479001600.0f;
    a = a * tb + 100.0f / 39916800.0f; b = b * tb + 10.0f / 39916800.0f;
    a = a * tb - 81.0f / 3628800.0f;   b = b * tb - 9.0f / 3628800.0f;
    a = a * tb + 64.0f / 362880.0f;    b = b * tb + 8.0f / 362880.0f;
    a = a * tb - 49.0f / 40320.0f;     b = b * tb - 7.0f / 40320.0f;
    a = a * tb + 36.0f / 5040.0f;      b = b * tb + 6.0f / 5040.0f;
    a = a * tb - 25.0f / 720.0f;       b = b * tb - 5.0f / 720.0f;
    a = a * tb + 16.0f / 120.0f;       b = b * tb + 4.0f / 120.0f;
    a = a * tb - 9.0f / 24.0f;         b = b * tb - 3.0f / 24.0f;
    a = a * tb + 4.0f / 6.0f;          b = b * tb + 2.0f / 6.0f;
    dw0 = -(a * tb - 0.5f);
    dw1 = -(b * tb - 0.5f);
  } else {
    const float e = fexp(-tb);
    const float it = frcp(tb);
    detb = -e;
    dw0 = -it * it + e * (1.0f + it) + e * it * it;
    dw1 = it * it - e * it - e * it * it;
  }
}

// y = K' x and y = K'^T x for K' given by kp = (q,u,v,rq,ru,rv)
SNAPI_HD void kp_mul(const float *kp, const float *x, float *y) {
  y[0] = kp[0] * x[1] + kp[1] * x[2] + kp[2] * x[3];
  y[1] = kp[0] * x[0] + kp[5] * x[2] - kp[4] * x[3];
  y[2] = kp[1] * x[0] - kp[5] * x[1] + kp[3] * x[3];
  y[3] = kp[2] * x[0] + kp[4] * x[1] - kp[3] * x[2];
}
SNAPI_HD void kp_mul_t(const float *kp, const float *x, float *y) {
  y[0] = kp[0] * x[1] + kp[1] * x[2] + kp[2] * x[3];
  y[1] = kp[0] * x[0] - kp[5] * x[2] + kp[4] * x[3];
  y[2] = kp[1] * x[0] + kp[5] * x[1] - kp[3] * x[3];
  y[3] = kp[2] * x[0] - kp[4] * x[1] + kp[3] * x[2];
}
// adjoint of y = K'(kp) x w.r.t. kp for the outer product yb x^T: d<yb, K'x>/dkp
SNAPI_HD void kp_outer_proj(const float *yb, const float *x, float scale, float *kpb) {
  kpb[0] += scale * (yb[0] * x[1] + yb[1] * x[0]);
  kpb[1] += scale * (yb[0] * x[2] + yb[2] * x[0]);
  kpb[2] += scale * (yb[0] * x[3] + yb[3] * x[0]);
  kpb[3] += scale * (yb[2] * x[3] - yb[3] * x[2]);
  kpb[4] += scale * (yb[3] * x[1] - yb[1] * x[3]);
  kpb[5] += scale * (yb[1] * x[2] - yb[2] * x[1]);
}
// A = 1 + w1 K' (transpose: flip the sign of the rho terms)
SNAPI_HD void build_A(const float *kp, float w1, bool transpose, float *A) {
  const float r = transpose ? -w1 : w1;
  A[0] = 1.0f;        A[1] = w1 * kp[0]; A[2] = w1 * kp[1]; A[3] = w1 * kp[2];
  A[4] = w1 * kp[0];  A[5] = 1.0f;       A[6] = r * kp[5];  A[7] = -r * kp[4];
  A[8] = w1 * kp[1];  A[9] = -r * kp[5]; A[10] = 1.0f;      A[11] = r * kp[3];
  A[12] = w1 * kp[2]; A[13] = r * kp[4]; A[14] = -r * kp[3]; A[15] = 1.0f;
}

// One linear-DELO step: I_c = (1 + w1 K'_c)^-1 [ -w0 K'_p I_p + w0 S_p + w1 S_c + etb I_p ]
SNAPI_HD void delo_step(const float *Ip, const float *kpp, const float *Sp, const float *kpc, const float *Sc,
                        float tb, float *Ic) {
  float w0, w1, etb;
  delo_weights(tb, w0, w1, etb);
  float A[16], LU[16], B[4], tv[4];
  kp_mul(kpp, Ip, tv);
  build_A(kpc, w1, false, A);
#pragma unroll
  for (int s = 0; s < 4; ++s) B[s] = -w0 * tv[s] + w0 * Sp[s] + w1 * Sc[s] + Ip[s] * etb;
  crout4(A, LU);
  solve_crout4(LU, B, Ic);
}

// Reverse of delo_step.  Inputs: forward values and Icb (adjoint of I_c).  Accumulates into
// Ipb, kppb, Spb, kpcb, Scb and returns the adjoint of tb.
SNAPI_HD float delo_step_adjoint(const float *Ip, const float *kpp, const float *Sp, const float *kpc,
                                 const float *Sc, float tb, const float *Ic, const float *Icb, float *Ipb,
                                 float *kppb, float *Spb, float *kpcb, float *Scb) {
  float w0, w1, etb, dw0, dw1, detb;
  delo_weights(tb, w0, w1, etb);
  delo_weights_grad(tb, dw0, dw1, detb);
  float AT[16], LU[16], Bb[4], tv[4];
  // A^T Bb = Icb
  build_A(kpc, w1, true, AT);
  crout4(AT, LU);
  solve_crout4(LU, Icb, Bb);
  // A-bar = -Bb Ic^T ;  A = 1 + w1 K'_c  ->  kpc-bar += -w1 proj(Bb Ic^T), w1-bar += -Bb^T K'_c Ic
  kp_outer_proj(Bb, Ic, -w1, kpcb);
  kp_mul(kpc, Ic, tv);
  float w1b = -(Bb[0] * tv[0] + Bb[1] * tv[1] + Bb[2] * tv[2] + Bb[3] * tv[3]);
  // B = -w0 K'_p I_p + w0 S_p + w1 S_c + etb I_p
  kp_mul(kpp, Ip, tv);
  float w0b = 0.f, etbb = 0.f;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    w0b += Bb[s] * (Sp[s] - tv[s]);
    w1b += Bb[s] * Sc[s];
    etbb += Bb[s] * Ip[s];
    Spb[s] += w0 * Bb[s];
    Scb[s] += w1 * Bb[s];
  }
  // Ip-bar = etb Bb - w0 K'_p^T Bb ; kpp-bar += -w0 proj(Bb Ip^T)
  kp_mul_t(kpp, Bb, tv);
#pragma unroll
  for (int s = 0; s < 4; ++s) Ipb[s] += etb * Bb[s] - w0 * tv[s];
  kp_outer_proj(Bb, Ip, -w0, kppb);
  return w0b * dw0 + w1b * dw1 + etbb * detb;
}

// ---------------------------------------------------------------------------------------------
// Optical depth (FP64): monotone derivative of eta_I at an interior point and the Bezier
// increment over one interval (atmos_ppbez_rts.cc:966-988), written on the path-length
// intervals D[i] = (tau500[i+1] - tau500[i]) / mu between depths i (above) and i+1 (below).
//
// interior point z (1..nd-2):  h1 = D[z] (upwind side, below), h2 = D[z-1] (downwind, above)
SNAPI_HD double opd_interior(double e_up, double e_c, double e_dn, double h1, double h2) {
  // e_up = eta[z+1] (below), e_c = eta[z], e_dn = eta[z-1] (above)
  const double d1 = (e_c - e_up) / h1;
  const double d2 = (e_dn - e_c) / h2;
  if (d1 * d2 > 0) {
    const double alpha = (1.0 + h1 / (h1 + h2)) / 3.0;
    return d1 * d2 / (alpha * d1 + (1.0 - alpha) * d2);
  }
  return 0.0;
}
// gradient of opd_interior w.r.t. (e_up, e_c, e_dn)
SNAPI_HD void opd_interior_grad(double e_up, double e_c, double e_dn, double h1, double h2, double g,
                                double &gup, double &gc, double &gdn) {
  const double d1 = (e_c - e_up) / h1;
  const double d2 = (e_dn - e_c) / h2;
  if (d1 * d2 > 0) {
    const double alpha = (1.0 + h1 / (h1 + h2)) / 3.0;
    const double den = alpha * d1 + (1.0 - alpha) * d2;
    const double dd1 = (1.0 - alpha) * d2 * d2 / (den * den);
    const double dd2 = alpha * d1 * d1 / (den * den);
    gup += -g * dd1 / h1;
    gc += g * dd1 / h1 - g * dd2 / h2;
    gdn += g * dd2 / h2;
  }
}
// Bezier optical depth over the interval between depth z (above) and z+1 (below):
//   dl = D[z];  C0 = e_z - dl/2 opd_z ;  C1 = e_{z+1} + dl/2 opd_{z+1} ;  dtau = dl/3 (e_{z+1} + e_z + (C0+C1)/2)
SNAPI_HD double bezier_dtau(double e_below, double e_above, double opd_below, double opd_above, double dl) {
  const double C0 = e_above - dl / 2.0 * opd_above;
  const double C1 = e_below + dl / 2.0 * opd_below;
  const double C = 0.5 * (C0 + C1);
  return dl / 3.0 * (e_below + e_above + C);
}

}  // namespace snapi
