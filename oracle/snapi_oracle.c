/*
 * snapi_oracle.c -- FP64 CPU restatement of the SNAPI Stokes synthesis hot path.
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA path); see snapi_oracle.h for the map of
 * every function to the reference file:line it follows.
 */
#include "snapi_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* CGS constants as the reference defines them (cmlib/const.h:5-18) */
#define SNO_PI 3.141592653589793238462643383279502884197169399375105
#define SNO_C 2.99792458E10
#define SNO_H 6.6260687652E-27
#define SNO_K 1.3806503E-16
#define SNO_SQRTPI 1.77245386399759

/* complex arithmetic in the reference's own formulation (cmlib/types.h:28-55) */
typedef struct { double re, im; } cx;
static cx cmk(double r, double i) { cx z = {r, i}; return z; }
static cx cadd(cx a, cx b) { return cmk(a.re + b.re, a.im + b.im); }
static cx csub(cx a, cx b) { return cmk(a.re - b.re, a.im - b.im); }
static cx cmul(cx a, cx b) { return cmk(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static cx cdiv(cx a, cx b) {
  double f = b.re * b.re + b.im * b.im;
  return cmk((a.re * b.re + a.im * b.im) / f, (a.im * b.re - a.re * b.im) / f);
}
static cx caddr(double a, cx b) { return cmk(b.re + a, b.im); }
static cx csubr(double a, cx b) { return cmk(a - b.re, -b.im); }
static cx cscl(cx a, double s) { return cmk(a.re * s, a.im * s); }

/* Humlicek (1982) W4 as evaluated by cmlib/profiles.cc:7-37 (region tests and coefficients
 * of the published method; cos(Im u) taken as +sqrt(1 - sin^2), as the reference does). */
void sno_voigt(double x, double a, double *H, double *F) {
  double v = x;
  double s = fabs(v) + a;
  cx t = cmk(a, -v);
  cx u = cmk(a * a - v * v, -2.0 * a * v);
  cx w4;
  if (s >= 15.0) {
    w4 = cdiv(cscl(t, 0.5641896), caddr(0.5, u));
  } else if (s > 5.5) {
    w4 = cdiv(cmul(t, caddr(1.410474, cscl(u, 0.5641896))), caddr(0.75, cmul(u, caddr(3.0, u))));
  } else if (a > (0.195 * fabs(v) - 0.176)) {
    cx num = caddr(16.4955, cmul(t, caddr(20.20933, cmul(t, caddr(11.96482, cmul(t, caddr(3.778987, cscl(t, 0.5642236))))))));
    cx den = caddr(16.4955, cmul(t, caddr(38.82363, cmul(t, caddr(39.27121, cmul(t, caddr(21.69274, cmul(t, caddr(6.699398, t)))))))));
    w4 = cdiv(num, den);
  } else {
    cx p = csubr(1.320522, cscl(u, 0.56419));
    p = csubr(35.76683, cmul(u, p));
    p = csubr(219.0313, cmul(u, p));
    p = csubr(1540.787, cmul(u, p));
    p = csubr(3321.9905, cmul(u, p));
    p = csubr(36183.31, cmul(u, p));
    cx w = cmul(t, p);
    cx q = csubr(1.841439, u);
    q = csubr(61.57037, cmul(u, q));
    q = csubr(364.2191, cmul(u, q));
    q = csubr(2186.181, cmul(u, q));
    q = csubr(9022.228, cmul(u, q));
    q = csubr(24322.84, cmul(u, q));
    q = csubr(32066.6, cmul(u, q));
    double su = sin(u.im);
    double eu = exp(u.re);
    w4 = csub(cmk(eu * sqrt(1.0 - su * su), eu * su), cdiv(w, q));
  }
  *H = w4.re / SNO_SQRTPI;
  *F = w4.im / SNO_SQRTPI;
}

/* atom::zeeman_setup (atmos/atmol/atom/atom.cc:1636-1757); J given as 2J. */
int sno_zeeman_pattern(int ju2, int jl2, double gu, double gl, sno_line *L) {
  int i, g;
  for (g = 0; g < 3; ++g) {
    L->ncomp[g] = 0;
    for (i = 0; i < SNO_MAXCOMP; ++i) { L->S[g][i] = 0.0; L->D[g][i] = 0.0; }
  }
  L->split = 0;
  if ((ju2 - jl2 == 2) || (ju2 - jl2 == -2) || ((ju2 == jl2) && (ju2 != 0))) L->split = 1;
  if (!L->split) return 0;
  int jmin2 = ju2 < jl2 ? ju2 : jl2;
  L->ncomp[0] = jmin2 + 1;
  L->ncomp[1] = L->ncomp[2] = (ju2 + jl2) / 2;
  double ju = ju2 / 2.0, jmin = jmin2 / 2.0;
  double np = 0, nb = 0, nr = 0;
  if (ju2 == jl2) {
    for (i = 0; i < L->ncomp[0]; ++i) {
      double mi = (double)i - ju;
      L->S[0][i] = mi * mi;
      L->D[0][i] = mi * (gl - gu);
      np += L->S[0][i];
    }
    for (i = 0; i < L->ncomp[0]; ++i) L->S[0][i] /= np;
    for (i = 0; i < L->ncomp[1]; ++i) {
      double mi = (double)i - ju + 1.0;
      L->S[1][i] = 0.5 * (ju + mi) * (ju - mi + 1.0);
      nb += L->S[1][i];
      L->D[1][i] = mi * (gl - gu) - gl;
      mi = (double)i - ju;
      L->S[2][i] = 0.5 * (ju - mi) * (ju + mi + 1);
      nr += L->S[2][i];
      L->D[2][i] = mi * (gl - gu) + gl;
    }
    for (i = 0; i < L->ncomp[1]; ++i) { L->S[1][i] /= nb; L->S[2][i] /= nr; }
  } else {
    double jl = jl2 / 2.0;
    int offset = (jl2 > ju2) ? 1 : 0;
    for (i = 0; i < L->ncomp[0]; ++i) {
      double mi = (double)i - jmin;
      if (jl < ju) {
        L->S[1][i] = 0.5 * (jmin + mi + 1) * (jmin + mi + 2);
        L->S[0][i] = (jmin + 1) * (jmin + 1) - mi * mi;
        L->S[2][i] = 0.5 * (jmin - mi + 1) * (jmin - mi + 2);
      } else {
        L->S[1][i] = 0.5 * (jmin - mi + 1) * (jmin - mi + 2);
        L->S[0][i] = (jmin + 1) * (jmin + 1) - mi * mi;
        L->S[2][i] = 0.5 * (jmin + mi + 1) * (jmin + mi + 2);
      }
      np += L->S[0][i]; nr += L->S[2][i]; nb += L->S[1][i];
      L->D[0][i] = mi * (gl - gu);
      L->D[1][i] = (mi - offset) * (gl - gu) - gu;
      L->D[2][i] = (mi + offset) * (gl - gu) + gu;
    }
    for (i = 0; i < L->ncomp[0]; ++i) { L->S[0][i] /= np; L->S[1][i] /= nb; L->S[2][i] /= nr; }
  }
  return 1;
}

/* cmlib/mathtools.cc:1325-1330 */
double sno_airtovac(double lambda_air) {
  double s = 1E4 / (lambda_air * 1E8);
  double n = 1.0 + 0.00008336624212083 + 0.02408926869968 / (130.1065924522 - s * s) +
             0.0001599740894897 / (38.92568793293 - s * s);
  return lambda_air * n;
}

/* cmlib/mathtools.cc:1150-1152 (lambda in cm) */
double sno_planck(double lambda, double T) {
  return 2.0 * 6.62606957 * 8.9875517E-7 / lambda / lambda / lambda / lambda / lambda /
         (exp(1.4387769 / lambda / T) - 1.0);
}

/* atmosphere::get_opacity_fudge without a fudge table (atmos/atmos_rad.cc:657-675) */
static double sno_fudge(double lambda_cm) {
  double l = lambda_cm * 1E8;
  double lb = 2.1177 * exp(-(l - 2087.7) * (l - 2087.7) / 2.421E6) + 0.68738;
  if (l > 4500.0) lb = 0.0;
  return 1.0 * (1.0 + 0.666667 * lb);
}

void sno_opacity(const double *rec, int nlines, const sno_line *lines, double lam, double lam_mid,
                 double *op, double *em) {
  int s, j, g, i;
  const double T = rec[0], vt = rec[1], ne = rec[2], vlos = rec[3], Bmag = rec[4];
  for (i = 0; i < 16; ++i) op[i] = 0.0;
  for (s = 0; s < 4; ++s) em[s] = 0.0;
  /* Thomson (atmos_rad_synthesis.cc:41-50) */
  double ope = ne * 6.65E-25;
  op[0] = ope;
  em[0] = ope * sno_planck(lam_mid, T);
  /* bound-free of all atoms, flat in the window */
  op[0] += rec[10];
  em[0] += rec[11];
  /* bound-bound (atom_rad_synthesis.cc:400-499) */
  double theta_B = rec[5] * SNO_PI / 180.0, phi_B = rec[6] * SNO_PI / 180.0;
  if (Bmag < 0.001) theta_B = phi_B = 0.0;
  double sp = sin(2.0 * phi_B), cp = cos(2.0 * phi_B);
  double st = sin(theta_B), ctb = cos(theta_B);
  for (j = 0; j < nlines; ++j) {
    const sno_line *L = &lines[j];
    double lam0 = L->lam0;
    double lambda_B = 4.67E-5 * lam0 * lam0 * Bmag;
    double dld = sqrt(2.0 * SNO_K * T / L->mass + vt * vt) * lam0 / SNO_C;
    double gc = rec[12 + 3 * j + 2];
    double a = L->sf * (L->ar + gc * 1.0) / dld;
    double op_loc = rec[12 + 3 * j + 0], em_loc = rec[12 + 3 * j + 1];
    double lshift = lam * (1.0 + vlos / SNO_C);
    if (!L->split) {
      double H, F;
      double x = (lam0 - lshift) / dld;
      sno_voigt(x, a, &H, &F);
      double prof = H / dld;
      op[0] += op_loc * prof;
      em[0] += em_loc * prof;
    } else {
      double Hs[3] = {0, 0, 0}, Fs[3] = {0, 0, 0};
      for (g = 0; g < 3; ++g)
        for (i = 0; i < L->ncomp[g]; ++i) {
          double H, F;
          double x = (lam0 + L->D[g][i] * lambda_B - lshift) / dld;
          sno_voigt(x, a, &H, &F);
          Hs[g] += H * L->S[g][i];
          Fs[g] += F * L->S[g][i];
        }
      double Hp = Hs[0] / dld, Hb = Hs[1] / dld, Hr = Hs[2] / dld;
      double Fp = Fs[0] / dld, Fb = Fs[1] / dld, Fr = Fs[2] / dld;
      double eI = 0.5 * (Hp * st * st + 0.5 * (Hr + Hb) * (1.0 + ctb * ctb));
      double eQ = 0.5 * (Hp - 0.5 * (Hr + Hb)) * st * st * cp;
      double eU = 0.5 * (Hp - 0.5 * (Hr + Hb)) * st * st * sp;
      double eV = 0.5 * (Hr - Hb) * ctb;
      double rQ = 0.5 * (Fp - 0.5 * (Fr + Fb)) * st * st * cp;
      double rU = 0.5 * (Fp - 0.5 * (Fr + Fb)) * st * st * sp;
      double rV = 0.5 * (Fr - Fb) * ctb;
      op[0] += eI * op_loc;
      op[1] += eQ * op_loc;
      op[2] += eU * op_loc;
      op[3] += eV * op_loc;
      op[2 * 4 + 3] += rQ * op_loc; /* [3][4] */
      op[3 * 4 + 1] += rU * op_loc; /* [4][2] */
      op[1 * 4 + 2] += rV * op_loc; /* [2][3] */
      em[0] += eI * em_loc;
      em[1] += eQ * em_loc;
      em[2] += eU * em_loc;
      em[3] += eV * em_loc;
    }
  }
  /* H- bound-free and free-free (mol.cc:609-632, :516-545), emissivity in LTE (:393-397) */
  {
    static const double ca[7] = {1.99654, -1.18267E-5, 2.64243E-6, -4.40524E-10, 3.23992E-14,
                                 -1.39568E-18, 2.78701E-23};
    double lA = lam * 1E8;
    double alpha = 0.0;
    for (i = 0; i < 7; ++i) alpha += ca[i] * pow(lA, i);
    double fud = sno_fudge(lam);
    double op_bf = alpha * rec[8] * (1.0 - exp(-SNO_H * SNO_C / lam / SNO_K / T)) * fud;
    double l = log10(lA);
    double f0 = -2.2763 - 1.6850 * l + 0.76661 * l * l - 0.053346 * l * l * l;
    double f1 = 15.2827 - 9.2846 * l + 1.99381 * l * l - 0.142631 * l * l * l;
    double f2 = -197.789 + 190.266 * l - 67.9775 * l * l + 10.6913 * l * l * l - 0.625151 * l * l * l * l;
    double lt = log10(5040. / T);
    double op_ff = rec[9] * pow(10.0, f0 + f1 * lt + f2 * lt * lt) * fud;
    double oph = op_bf + op_ff;
    op[0] += oph;
    em[0] += oph * sno_planck(lam, T);
  }
  /* fill (atmos_rad_synthesis.cc:57-68) */
  op[5] = op[10] = op[15] = op[0];
  op[4] = op[1];
  op[8] = op[2];
  op[12] = op[3];
  op[9] = -op[6];   /* [3][2] = -[2][3] */
  op[7] = -op[13];  /* [2][4] = -[4][2] */
  op[14] = -op[11]; /* [4][3] = -[3][4] */
  /* normalise to kappa_500 (atmos_rad.cc:175-185) */
  {
    double kap = rec[7];
    for (s = 0; s < 4; ++s) {
      em[s] /= kap;
      for (i = 0; i < 4; ++i) op[s * 4 + i] /= kap;
    }
  }
}

/* Crout without pivoting, unit upper diagonal (cmlib/mathtools.cc:487-514) */
static void crout4(const double *S, double *D) {
  int k, i, j, p;
  for (k = 0; k < 4; ++k) {
    for (i = k; i < 4; ++i) {
      double sum = 0.;
      for (p = 0; p < k; ++p) sum += D[i * 4 + p] * D[p * 4 + k];
      D[i * 4 + k] = S[i * 4 + k] - sum;
    }
    for (j = k + 1; j < 4; ++j) {
      double sum = 0.;
      for (p = 0; p < k; ++p) sum += D[k * 4 + p] * D[p * 4 + j];
      D[k * 4 + j] = (S[k * 4 + j] - sum) / D[k * 4 + k];
    }
  }
}
static void solvecrout4(const double *LU, const double *b, double *x) {
  double y[4];
  int i, k;
  for (i = 0; i < 4; ++i) {
    double sum = 0.;
    for (k = 0; k < i; ++k) sum += LU[i * 4 + k] * y[k];
    y[i] = (b[i] - sum) / LU[i * 4 + i];
  }
  for (i = 3; i >= 0; --i) {
    double sum = 0.;
    for (k = i + 1; k < 4; ++k) sum += LU[i * 4 + k] * x[k];
    x[i] = (y[i] - sum);
  }
}

#define EXPANSION_DELIMITER 1E-2

/* atmos_ppbez::formal, polarized (atmos/plpar/atmos_ppbez_rts.cc:918-1218).
 * Index k = 0 (top) .. nd-1 (bottom); the spatial grid is the reference's tau_referent = -tau500. */
void sno_formal(int nd, const double *tau500, const double *oo, const double *ee, double ct, double *I) {
  int z, s, sp, q;
  const int dz = (ct > 0) ? 1 : -1;
  const int zl = (ct > 0) ? 0 : nd - 1;
  const int zh = (ct > 0) ? nd - 1 : 0;
#define GRID(kk) (-tau500[kk])
#define OO(kk, a, b) oo[(kk) * 16 + (a) * 4 + (b)]
#define EE(kk, a) ee[(kk) * 4 + (a)]
  double *dtau = (double *)calloc(nd, sizeof(double));
  double *opd = (double *)calloc(nd, sizeof(double));
  double *src = (double *)calloc(nd * 4, sizeof(double));
  double *sd = (double *)calloc(nd * 4, sizeof(double));
  double *K = (double *)calloc(nd * 16, sizeof(double));
  double *Kd = (double *)calloc(nd * 16, sizeof(double));

  I[zl * 4 + 0] = (ct > 0) ? 0.0 : EE(zl, 0) / OO(zl, 0, 0);
  I[zl * 4 + 1] = I[zl * 4 + 2] = I[zl * 4 + 3] = 0.0;

  /* monotone derivative of eta_I along the ray (:966-979) */
  opd[zl] = (OO(zl + dz, 0, 0) - OO(zl, 0, 0)) / (GRID(zl + dz) - GRID(zl)) * (-ct);
  opd[zh] = (OO(zh, 0, 0) - OO(zh - dz, 0, 0)) / (GRID(zh) - GRID(zh - dz)) * (-ct);
  for (z = zl + dz; (z - zh) * dz < 0; z += dz) {
    opd[z] = 0.0;
    double h2 = (GRID(z + dz) - GRID(z)) / (-ct);
    double h1 = (GRID(z) - GRID(z - dz)) / (-ct);
    double d2 = (OO(z + dz, 0, 0) - OO(z, 0, 0)) / h2;
    double d1 = (OO(z, 0, 0) - OO(z - dz, 0, 0)) / h1;
    if (d1 * d2 > 0) {
      double alpha = (1.0 + h1 / (h1 + h2)) / 3.0;
      opd[z] = d1 * d2 / (alpha * d1 + (1.0 - alpha) * d2);
    }
  }
  /* Bezier optical depth increments (:981-988) */
  dtau[zl] = 0.0;
  for (z = zl + dz; (z - zh - dz) * dz < 0; z += dz) {
    double dl = (GRID(z) - GRID(z - dz)) / (-ct);
    double C0 = OO(z, 0, 0) - dl / 2.0 * opd[z];
    double C1 = OO(z - dz, 0, 0) + dl / 2.0 * opd[z - dz];
    double C = 0.5 * (C0 + C1);
    dtau[z] = dl / 3.0 * (OO(z - dz, 0, 0) + OO(z, 0, 0) + C);
  }
  /* source function and its monotone derivative (:993-1013) */
  for (s = 0; s < 4; ++s) {
    sd[zl * 4 + s] = (EE(zl + dz, s) / OO(zl + dz, 0, 0) - EE(zl, s) / OO(zl, 0, 0)) / dtau[zl + dz];
    sd[zh * 4 + s] = (EE(zh, s) / OO(zh, 0, 0) - EE(zh - dz, s) / OO(zh - dz, 0, 0)) / dtau[zh];
  }
  for (z = zl + dz; (z - zh) * dz < 0; z += dz)
    for (s = 0; s < 4; ++s) {
      sd[z * 4 + s] = 0.0;
      double h2 = dtau[z + dz], h1 = dtau[z];
      double d2 = (EE(z + dz, s) / OO(z + dz, 0, 0) - EE(z, s) / OO(z, 0, 0)) / h2;
      double d1 = (EE(z, s) / OO(z, 0, 0) - EE(z - dz, s) / OO(z - dz, 0, 0)) / h1;
      if (d1 * d2 > 0) {
        double alpha = (1.0 + h1 / (h1 + h2)) / 3.0;
        sd[z * 4 + s] = d1 * d2 / (alpha * d1 + (1.0 - alpha) * d2);
      }
    }
  for (z = 0; z < nd; ++z)
    for (s = 0; s < 4; ++s) src[z * 4 + s] = EE(z, s) / OO(z, 0, 0);
  /* reduced absorption matrix K' = K/eta_I - 1 and its derivative (:1018-1049) */
  for (z = 0; z < nd; ++z)
    for (s = 0; s < 4; ++s) {
      for (sp = 0; sp < 4; ++sp) K[z * 16 + s * 4 + sp] = OO(z, s, sp) / OO(z, 0, 0);
      K[z * 16 + s * 4 + s] -= 1.0;
    }
  for (s = 0; s < 4; ++s)
    for (sp = 0; sp < 4; ++sp) {
      Kd[zl * 16 + s * 4 + sp] = (K[(zl + dz) * 16 + s * 4 + sp] - K[zl * 16 + s * 4 + sp]) / dtau[zl + dz];
      Kd[zh * 16 + s * 4 + sp] = (K[zh * 16 + s * 4 + sp] - K[(zh - dz) * 16 + s * 4 + sp]) / dtau[zh];
    }
  for (z = zl + dz; (z - zh) * dz < 0; z += dz)
    for (s = 0; s < 4; ++s)
      for (sp = 0; sp < 4; ++sp) {
        Kd[z * 16 + s * 4 + sp] = 0.0;
        double h2 = dtau[z + dz], h1 = dtau[z];
        double d2 = (K[(z + dz) * 16 + s * 4 + sp] - K[z * 16 + s * 4 + sp]) / h2;
        double d1 = (K[z * 16 + s * 4 + sp] - K[(z - dz) * 16 + s * 4 + sp]) / h1;
        if (d1 * d2 > 0) {
          double alpha = (1.0 + h1 / (h1 + h2)) / 3.0;
          Kd[z * 16 + s * 4 + sp] = d1 * d2 / (alpha * d1 + (1.0 - alpha) * d2);
        }
      }
  /* depth recursion (:1055-1197): linear DELO (w2 = 0 since the Bezier branch is never taken) */
  for (z = zl + dz; (z - zh) * dz < 0; z += dz) {
    double tb = dtau[z];
    double etb = (tb < EXPANSION_DELIMITER) ? (1.0 - tb + tb * tb * 0.5 - tb * tb * tb / 6.0) : exp(-tb);
    double w0, w1, w2 = 0.0;
    if (tb < EXPANSION_DELIMITER) {
      w0 = tb * (0.5 - tb * (1.0 / 3.0 - tb / 8.0));
      w1 = 0.5 * tb * (1.0 - tb / 3.0 * (1.0 - tb / 4.0));
    } else {
      w0 = 1.0 / tb - etb * (1.0 + 1.0 / tb);
      w1 = 1.0 - 1.0 / tb + etb / tb;
    }
    const double *Kp = &K[(z - dz) * 16], *Kc = &K[z * 16];
    const double *Kdp = &Kd[(z - dz) * 16], *Kdc = &Kd[z * 16];
    const double *Ip = &I[(z - dz) * 4];
    double A[16], B[4], LU[16], tmp[16], tv[4], C1k[4], C0k[4], c0k[16];
    /* C1k (:1108-1126) */
    for (s = 0; s < 4; ++s)
      for (sp = 0; sp < 4; ++sp) {
        double m = 0.0;
        for (q = 0; q < 4; ++q) m += Kp[s * 4 + q] * Kp[q * 4 + sp];
        m += Kp[s * 4 + sp] + Kdp[s * 4 + sp];
        m *= tb / 2.0;
        m += Kp[s * 4 + sp];
        tmp[s * 4 + sp] = m;
      }
    for (s = 0; s < 4; ++s) { tv[s] = 0.0; for (q = 0; q < 4; ++q) tv[s] += tmp[s * 4 + q] * Ip[q]; }
    for (s = 0; s < 4; ++s) {
      for (sp = 0; sp < 4; ++sp) tmp[s * 4 + sp] = tb / 2.0 * Kp[s * 4 + sp];
      tmp[s * 4 + s] += 1.0;
    }
    for (s = 0; s < 4; ++s) {
      C1k[s] = 0.0;
      for (q = 0; q < 4; ++q) C1k[s] += tmp[s * 4 + q] * src[(z - dz) * 4 + q];
      C1k[s] += tb / 2.0 * sd[(z - dz) * 4 + s] - tv[s];
    }
    /* C0k, c0k (:1133-1155) */
    for (s = 0; s < 4; ++s) {
      for (sp = 0; sp < 4; ++sp) tmp[s * 4 + sp] = -tb / 2.0 * Kc[s * 4 + sp];
      tmp[s * 4 + s] += 1.0;
    }
    for (s = 0; s < 4; ++s) {
      C0k[s] = 0.0;
      for (q = 0; q < 4; ++q) C0k[s] += tmp[s * 4 + q] * src[z * 4 + q];
      C0k[s] -= tb / 2.0 * sd[z * 4 + s];
    }
    for (s = 0; s < 4; ++s)
      for (sp = 0; sp < 4; ++sp) {
        double m = 0.0;
        for (q = 0; q < 4; ++q) m += Kc[s * 4 + q] * Kc[q * 4 + sp];
        m += Kc[s * 4 + sp] + Kdc[s * 4 + sp];
        m *= tb / 2.0;
        m -= Kc[s * 4 + sp];
        c0k[s * 4 + sp] = m;
      }
    /* A, B (:1158-1168) */
    for (s = 0; s < 4; ++s) {
      for (sp = 0; sp < 4; ++sp) A[s * 4 + sp] = w1 * Kc[s * 4 + sp] - w2 / 2.0 * c0k[s * 4 + sp];
      A[s * 4 + s] += 1.0;
    }
    for (s = 0; s < 4; ++s) { tv[s] = 0.0; for (q = 0; q < 4; ++q) tv[s] += Kp[s * 4 + q] * Ip[q]; }
    for (s = 0; s < 4; ++s)
      B[s] = -w0 * tv[s] + w0 * src[(z - dz) * 4 + s] + w1 * src[z * 4 + s] + Ip[s] * etb +
             w2 / 2.0 * (C1k[s] + C0k[s]);
    crout4(A, LU);
    solvecrout4(LU, B, &I[z * 4]);
  }
  if (zl != zh)
    for (s = 0; s < 4; ++s) I[zh * 4 + s] = I[(zh - dz) * 4 + s];
  free(dtau); free(opd); free(src); free(sd); free(K); free(Kd);
#undef GRID
#undef OO
#undef EE
}

void sno_synth_pixel(int nd, int nl, const double *lam_air, const double *tau500, const double *rec,
                     int nlines, const sno_line *lines, double ct, double *stokes) {
  int nf = 12 + 3 * nlines;
  double *op = (double *)malloc(sizeof(double) * nd * 16);
  double *em = (double *)malloc(sizeof(double) * nd * 4);
  double *I = (double *)malloc(sizeof(double) * nd * 4);
  double lam_mid = 0.5 * (sno_airtovac(lam_air[nl - 1]) + sno_airtovac(lam_air[0]));
  int l, k, s;
  for (l = 0; l < nl; ++l) {
    double lv = sno_airtovac(lam_air[l]);
    for (k = 0; k < nd; ++k) sno_opacity(rec + k * nf, nlines, lines, lv, lam_mid, op + k * 16, em + k * 4);
    sno_formal(nd, tau500, op, em, ct, I);
    for (s = 0; s < 4; ++s) stokes[l * 4 + s] = I[0 * 4 + s];
  }
  free(op); free(em); free(I);
}

void sno_synth_batch(int npix, int nd, int nl, const double *lam_air, const double *tau500,
                     const double *rec, int nlines, const sno_line *lines, double ct, double *stokes) {
  int nf = 12 + 3 * nlines, p;
  for (p = 0; p < npix; ++p)
    sno_synth_pixel(nd, nl, lam_air, tau500, rec + (size_t)p * nd * nf, nlines, lines, ct,
                    stokes + (size_t)p * nl * 4);
}

double sno_chi2(int nl, const double *S, const double *obs, const double *ws, const double *mask) {
  double chi = 0.0;
  int l, s;
  for (l = 0; l < nl; ++l)
    for (s = 0; s < 4; ++s) {
      double r = (obs[l * 4 + s] - S[l * 4 + s]) * ws[s] * mask[l];
      chi += r * r;
    }
  return chi;
}

void sno_chi2_grad_fd(int nd, int nl, const double *lam_air, const double *tau500, const double *rec,
                      int nlines, const sno_line *lines, double ct, const double *obs, const double *ws,
                      const double *mask, int npar, const double *tangent, double step, double *chi2,
                      double *grad) {
  int nf = 12 + 3 * nlines, n = nd * nf, p, i;
  double *S = (double *)malloc(sizeof(double) * nl * 4);
  double *r = (double *)malloc(sizeof(double) * n);
  sno_synth_pixel(nd, nl, lam_air, tau500, rec, nlines, lines, ct, S);
  *chi2 = sno_chi2(nl, S, obs, ws, mask);
  for (p = 0; p < npar; ++p) {
    const double *t = tangent + (size_t)p * n;
    for (i = 0; i < n; ++i) r[i] = rec[i] + step * t[i];
    sno_synth_pixel(nd, nl, lam_air, tau500, r, nlines, lines, ct, S);
    double cp = sno_chi2(nl, S, obs, ws, mask);
    for (i = 0; i < n; ++i) r[i] = rec[i] - step * t[i];
    sno_synth_pixel(nd, nl, lam_air, tau500, r, nlines, lines, ct, S);
    double cm = sno_chi2(nl, S, obs, ws, mask);
    grad[p] = (cp - cm) / (2.0 * step);
  }
  free(S); free(r);
}

void sno_stokes_jvp_fd(int nd, int nl, const double *lam_air, const double *tau500, const double *rec,
                       int nlines, const sno_line *lines, double ct, int npar, const double *tangent,
                       double step, double *dS) {
  int nf = 12 + 3 * nlines, n = nd * nf, p, i;
  double *Sp = (double *)malloc(sizeof(double) * nl * 4);
  double *Sm = (double *)malloc(sizeof(double) * nl * 4);
  double *r = (double *)malloc(sizeof(double) * n);
  for (p = 0; p < npar; ++p) {
    const double *t = tangent + (size_t)p * n;
    for (i = 0; i < n; ++i) r[i] = rec[i] + step * t[i];
    sno_synth_pixel(nd, nl, lam_air, tau500, r, nlines, lines, ct, Sp);
    for (i = 0; i < n; ++i) r[i] = rec[i] - step * t[i];
    sno_synth_pixel(nd, nl, lam_air, tau500, r, nlines, lines, ct, Sm);
    for (i = 0; i < nl * 4; ++i) dS[(size_t)p * nl * 4 + i] = (Sp[i] - Sm[i]) / (2.0 * step);
  }
  free(Sp); free(Sm); free(r);
}
