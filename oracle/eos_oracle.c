/*
 * eos_oracle -- FP64 CPU restatement of the node -> column-record build of the reference.
 *
 * TEST INFRASTRUCTURE ONLY.  The checker of snapi_build_records (the CUDA path); only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.  The product never calls it.
 *
 * Restates, in the reference's order of operations and on the tables of snapi_eos_model
 * (include/snapi_cuda.h):
 *   partition functions trav::U, trav::dU, qas_f, dqas_f, irwin::U, cpf / pf   partf.cc:217-283, 345-358
 *   ionisation fractions atom::ionfrc                                          atom.cc:892-925
 *   equilibrium constants eqc_poly::K, eqc_hmin::K, eqc_cnst                   moleqc.cc:108-114, 150-163
 *   chemical equilibrium atmosphere::chemeq                                    atmos_chm.cc:14-18, 28-330
 *   Saha-Boltzmann atom::lte                                                   atom.cc:779-787
 *   continuum opacity atmosphere::opacity_continuum, atom::opacity_continuum,
 *     h_minus_mol::opacity_continuum                                           atmos_rad.cc:286-294,
 *                                                                              atom_rad.cc:151-187, mol.cc:669-694
 *   node interpolation atmospheric_interpolation (+ interpol_1d)               mathtools.cc:1057-1117, 1208-1315
 *   hydrostatic equilibrium atmos_pp::build_from_nodes                         atmos_pp.cc:58-248
 *   record set-up: compute_op_referent, project, transform, bound-free window,
 *     line factors, atom::damp_col                                             atmos_ppbez_rts.cc:268-281,
 *                                                                              atmos_rad.cc:14-48,
 *                                                                              atom_rad_synthesis.cc:226-262,
 *                                                                              atom.cc:938-959
 *   tangents by central differences (thermal nodes: full build; others: re-interpolation)
 *                                                                              atmos_fit.cc:1225-1307
 * Deviations (also those of the CUDA path): Gaussian elimination with partial pivoting instead of
 * the SVD in chemeq; interpol_1d's unset h2 in its first interval replaced by that interval's width.
 */
#include <math.h>
#include <stddef.h>
#include <string.h>

#include "../include/snapi_cuda.h"

/* reference constants (cmlib/const.h, CGS) */
#define C_PI 3.141592653589793238462643383279502884197169399375105
#define C_C 2.99792458E10
#define C_H 6.6260687652E-27
#define C_K 1.3806503E-16
#define C_ME 9.1093818872E-28
#define C_E 4.8032042510E-10
#define C_RYD 1.097373156853955E5
#define C_E0 7.957747154594775607E-02
#define C_SAHA 2.0706615382E-16

#define MS SNAPI_EOS_MAX_STAGES
#define ML SNAPI_EOS_MAX_LEVELS
#define MA SNAPI_EOS_MAX_ATOMS
#define MM SNAPI_EOS_MAX_MOLS

/* ---- partition functions (partf.cc) ---------------------------------------------------------- */
static double qas_f(double l, double p, double Dz) {
  if (p > l) {
    double llm = l - 1.0;
    return ((1.3333333 * p + 0.5) * p + 0.16666667 + 1.33333333 * Dz) * p - 0.4 * Dz * Dz / p -
           ((0.33333333 * llm - 0.5) * llm - 0.16666667 - Dz) * llm + 0.5 * Dz * Dz / l;
  }
  double axl2 = Dz / (l * l);
  return (1.0 + axl2 * (0.33333333 + 0.1 * axl2)) * p * p * p * p / l;
}

static double dqas_f(double l, double p, double Dz) {
  if (p > l) return ((3.0 * 1.3333333 * p + 1.0) * p + 0.16666667 + 1.33333333 * Dz) + 0.4 * Dz * Dz / (p * p);
  double axl2 = Dz / (l * l);
  return 4.0 * (1.0 + axl2 * (0.33333333 + 0.1 * axl2)) * p * p * p / l;
}

static double trav_f(void) {
  double er = C_E * C_RYD * C_RYD;
  return 1.405169521381833474E+05 * ((4.0 * C_PI * C_E0) / (er * er));
}

static double pf_U(const snapi_partition *P, double T, double ne) {
  switch (P->type) {
    case SNAPI_PF_CONST: return P->value;
    case SNAPI_PF_TRAV: {
      double x = 5040.0 / T, f = trav_f();
      double p = P->zeff * f / pow(ne, 1.0 / 6.0);
      double alpha = 31.321 * P->zeff * P->zeff * x;
      double sum = P->g0;
      for (int i = 0; i < P->nterm; ++i) {
        for (int l = 0; l < P->m[i]; ++l) sum += P->a[i][l] * exp(-2.302585 * P->gam[i][l] * x);
        sum += P->g2[i] * exp(-2.302585 * P->ee[i] * x) * qas_f(P->ll[i], p, alpha);
      }
      return sum;
    }
    case SNAPI_PF_IRWIN: {
      double lnT = log(T), sum = 0.0;
      for (int i = 0; i < P->ncoef; ++i) sum += P->coef[i] * pow(lnT, i);
      return exp(sum);
    }
    default: return 1.0;
  }
}

/* trav::dU assigns (does not accumulate) per term: only the last term survives (partf.cc:247-248) */
static double pf_dU(const snapi_partition *P, double T, double ne) {
  if (P->type != SNAPI_PF_TRAV) return 0.0;
  double x = 5040.0 / T, f = trav_f();
  double p = P->zeff * f / pow(ne, 1.0 / 6.0);
  double alpha = 31.321 * P->zeff * P->zeff * x;
  double dsum = 0.0;
  for (int i = 0; i < P->nterm; ++i)
    dsum = -P->g2[i] * exp(-2.302585 * P->ee[i] * x) * dqas_f(P->ll[i], p, alpha) * P->zeff * f /
           (6.0 * pow(ne, 7.0 / 6.0));
  return dsum;
}

/* ---- atom::ionfrc ------------------------------------------------------------------------------ */
static void ionfrc(const snapi_eos_atom *A, double T, double ne, double *fk, double *df) {
  int Z = A->nstage - 1;
  double fct = 2.0 * pow((2.0 * C_PI * C_ME * C_K * T) / (C_H * C_H), 1.5);
  double Up = pf_U(&A->pf[0], T, ne);
  double dUp = pf_dU(&A->pf[0], T, ne) / Up;
  double fsum = (fk[0] = 1.0);
  double dfsum = (df[0] = 0.0);
  for (int z = 0; z < Z; ++z) {
    double Un = pf_U(&A->pf[z + 1], T, ne);
    double dUn = pf_dU(&A->pf[z + 1], T, ne) / Un;
    double f = fct * (Un / Up) * exp(-A->ip[z] / (C_K * T)) / ne;
    double fd = f * ((dUn) - (dUp * ne + 1.0) / ne);
    fsum += (fk[z + 1] = fk[z] * f);
    dfsum += (df[z + 1] = (df[z] * f + fk[z] * fd));
    Up = Un;
    dUp = dUn;
  }
  for (int z = 0; z <= Z; ++z) {
    df[z] = (df[z] - dfsum * fk[z] / fsum) / fsum;
    fk[z] /= fsum;
  }
}

/* ---- molecules (moleqc.cc) --------------------------------------------------------------------- */
static double mol_K(const snapi_eos_molecule *M, double T) {
  double x = 5040.0 / T;
  if (M->eqc == SNAPI_EQC_POLY) {
    double sum = M->coef[M->ncoef - 1];
    for (int i = M->ncoef - 2; i >= 0; --i) sum = M->coef[i] + x * sum;
    return exp(2.302585093 * sum);
  }
  if (M->eqc == SNAPI_EQC_HMIN) {
    double sum = 0.1249 + (2.5 * log(T) / 2.302585) - 0.747 * x;
    return exp(2.302585093 * sum);
  }
  if (M->eqc == SNAPI_EQC_CONST) return M->coef[0];
  return 0.0;
}

/* ---- linear solve (replaces the SVD of atmos_chm.cc:262-292) ----------------------------------- */
/* Gaussian elimination with partial pivoting.  On return A holds the factors in elimination order:
 * U on and above the diagonal, the multiplier of row r at step c in A[r][c] (rows are swapped from
 * column c on, so a multiplier stays where it was computed), and piv[c] the row swapped with row c
 * at step c -- lu_apply solves another right-hand side with them. */
static void gauss_solve(int n, double *A /*[n][n], factored*/, double *b /*rhs in, solution out*/, int *piv) {
  for (int c = 0; c < n; ++c) {
    int p = c;
    double best = fabs(A[c * n + c]);
    for (int r = c + 1; r < n; ++r)
      if (fabs(A[r * n + c]) > best) { best = fabs(A[r * n + c]); p = r; }
    piv[c] = p;
    if (p != c) {
      for (int j = c; j < n; ++j) { double t = A[c * n + j]; A[c * n + j] = A[p * n + j]; A[p * n + j] = t; }
      double t = b[c]; b[c] = b[p]; b[p] = t;
    }
    double d = A[c * n + c];
    for (int r = c + 1; r < n; ++r) {
      double f = A[r * n + c] / d;
      A[r * n + c] = f;
      if (f == 0.0) continue;
      for (int j = c + 1; j < n; ++j) A[r * n + j] -= f * A[c * n + j];
      b[r] -= f * b[c];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    double s = b[r];
    for (int j = r + 1; j < n; ++j) s -= A[r * n + j] * b[j];
    b[r] = s / A[r * n + r];
  }
}

/* the solve of gauss_solve for another right-hand side, from its factors */
static void lu_apply(int n, const double *LU, const int *piv, double *b) {
  for (int c = 0; c < n; ++c) {
    if (piv[c] != c) { double t = b[c]; b[c] = b[piv[c]]; b[piv[c]] = t; }
    for (int r = c + 1; r < n; ++r) b[r] -= LU[r * n + c] * b[c];
  }
  for (int r = n - 1; r >= 0; --r) {
    double s = b[r];
    for (int j = r + 1; j < n; ++j) s -= LU[r * n + j] * b[j];
    b[r] = s / LU[r * n + r];
  }
}

/* ---- atmosphere::chemeq ------------------------------------------------------------------------
 * T, Nt in; Ne in/out; out: Natom[a] (free particles of atom a), fk[a][z] (ionisation fractions of
 * the last Newton pass), and the number of Newton passes (negative: stopped at the cap). */
typedef struct {
  double Ne;
  double Natom[MA];
  double fk[MA][MS];
  int passes;
  int have;        /* Ne / Natom hold an earlier solution of this column, at particle density Nt_prev */
  double Nt_prev;
  /* the continued start's predictors: the factors of the last Newton pass's Jacobian (at
     temperature lu_T; lu_n = 0: none), and log(N / Nt) of the last solutions at the two latest
     temperatures T1 (the most recent) and T2 (nhist of them held) */
  double LU[(MA + 1) * (MA + 1)];
  int piv[MA + 1], lu_n, nhist;
  double lu_T, lx1[MA + 1], lx2[MA + 1], T1, T2;
} chem_state;

static void chem_reset(chem_state *c) {
  c->Ne = 1.0;
  c->have = 0;
  c->lu_n = 0;
  c->nhist = 0;
}

/* How chemeq starts in the hydrostatic march (SNAPI_CHEM_START_*, the device's
 * snapi_eos_chem_start): COLD, the reference's start at every solve (the default here); CONTINUE,
 * the CUDA path's default -- Newton from the previous solution of the same column scaled by the
 * particle-density ratio, at most 8 passes, else the cold start.  The record solves start cold in
 * either mode.  Restated here so that the device's continued start has an exact-path checker; the
 * reference itself always starts cold. */
static int g_chem_start = SNAPI_CHEM_START_COLD;

/* The continued start's first iterate (1: N set; 0: none applies, scale the last solution by the
 * particle-density ratio).  At the temperature of the last Jacobian (the next hydrostatic iterate
 * of the same depth) a first-order step along dN/dNt = J^-1 e_1 (the defect of row 1 is
 * sum N - Nt); at a new temperature (the next depth) log(N / Nt) extrapolated linearly in T from
 * the last two temperatures' solutions (the ratio clipped to [0, 2]; 1 when they share T).  An
 * iterate with a density below the Newton pass's floor (1e-2) or not finite is not used. */
static int predict_start(const chem_state *c, int na, double T, double Nt, double *N) {
  const int n = na + 1;
  if (c->lu_n == n && T == c->lu_T) {
    double x[MA + 1];
    for (int i = 0; i < n; ++i) x[i] = 0.0;
    x[1] = 1.0;
    lu_apply(n, c->LU, c->piv, x);
    const double dNt = Nt - c->Nt_prev;
    N[0] = c->Ne + x[0] * dNt;
    for (int a = 1; a <= na; ++a) N[a] = c->Natom[a - 1] + x[a] * dNt;
  } else if (c->nhist == 2 && T != c->T1) {
    double r = c->T1 != c->T2 ? (T - c->T1) / (c->T1 - c->T2) : 1.0;
    r = fmin(fmax(r, 0.0), 2.0);
    for (int a = 0; a <= na; ++a) N[a] = Nt * exp(c->lx1[a] + (c->lx1[a] - c->lx2[a]) * r);
  } else {
    return 0;
  }
  for (int a = 0; a <= na; ++a)
    if (!(N[a] >= 1E-2) || !isfinite(N[a])) return 0;
  return 1;
}

static void chemeq(const snapi_eos_model *m, double T, double Nt, chem_state *out) {
  const int na = m->natom, nm = m->nmol;
  double abund[MA + 1];
  for (int a = 1; a <= na; ++a) abund[a] = m->atoms[a - 1].abundance;
  int cmpidx[MM][SNAPI_MOL_MAX_COMP], cmpion[MM][SNAPI_MOL_MAX_COMP];
  int molmul[MM][MA + 1];
  double K[MM], q[MM], nmd[MM], dm[MM][MA + 1];
  memset(molmul, 0, sizeof molmul);
  for (int mm = 0; mm < nm; ++mm) {
    const snapi_eos_molecule *M = &m->mols[mm];
    q[mm] = 0.0;
    for (int i = 0; i < M->ncomp; ++i) {
      int idx = M->comp_atom[i] + 1;            /* 0: electron */
      molmul[mm][idx] += 1;
      cmpidx[mm][i] = idx;
      cmpion[mm][i] = M->comp_charge[i] > 0 ? M->comp_charge[i] : 0;
      q[mm] += (double)M->comp_charge[i];
    }
    K[mm] = mol_K(M, T);
  }
  double N[MA + 1];
  double Np = Nt - (N[0] = out->Ne);
  for (int a = 1; a <= na; ++a) N[a] = Np * abund[a];
  double fk[MA + 1][MS], df[MA + 1][MS];
  int nk[MA + 1];
  fk[0][0] = 1.0;
  df[0][0] = 0.0;
  nk[0] = 1;
  for (int a = 1; a <= na; ++a) nk[a] = m->atoms[a - 1].nstage;
  /* starting values: ionisation only, no molecules (atmos_chm.cc:129-171) */
  double F1 = 0.0, S1 = 0.0;
  for (int a = 1; a <= na; ++a) {
    ionfrc(&m->atoms[a - 1], T, 1.0, fk[a], df[a]);
    double sum = 0.0;
    for (int i = 0; i < nk[a]; ++i) sum += i * fk[a][i];
    F1 += abund[a] * sum;
    S1 += abund[a];
  }
  double F3 = 0.0, S3 = 0.0;
  for (int a = 1; a <= na; ++a) {
    ionfrc(&m->atoms[a - 1], T, Nt, fk[a], df[a]);
    double sum = 0.0;
    for (int i = 0; i < nk[a]; ++i) sum += i * fk[a][i];
    F3 += abund[a] * sum;
    S3 += abund[a];
  }
  double aa = F3 / (S3 * Nt);
  double bb = F1 / S1 - aa;
  double cc = -bb * Nt;
  bb += 1.0 - aa * Nt;
  /* the continued start (g_chem_start): Newton from the previous solution, the cold start if
     that has not converged after 8 passes or left non-finite values */
  int warm = g_chem_start == SNAPI_CHEM_START_CONTINUE && out->have;
  int maxpass = 50;
  if (warm) {
    if (!predict_start(out, na, T, Nt, N)) {
      const double sc = Nt / out->Nt_prev;
      N[0] = out->Ne * sc;
      for (int a = 1; a <= na; ++a) N[a] = out->Natom[a - 1] * sc;
    }
    maxpass = 8;
    goto newton;
  }
cold:
  warm = 0;
  maxpass = 50;
  N[0] = fmax((-bb + sqrt(bb * bb - 4.0 * aa * cc)) / (2.0 * aa), 1.0);
  double esum;
  do {
    esum = 0.0;
    for (int a = 1; a <= na; ++a) {
      ionfrc(&m->atoms[a - 1], T, N[0], fk[a], df[a]);
      N[a] = (Nt - N[0]) * abund[a] / S3;
      for (int i = 0; i < nk[a]; ++i) esum += fk[a][i] * N[a] * (double)i;
    }
    N[0] = 0.5 * (N[0] + esum);
  } while ((1E-2 * (N[0] + esum)) < fabs(N[0] - esum));
  /* Newton-Raphson (atmos_chm.cc:176-305) */
newton:;
  const int n = na + 1;
  double d[MA + 1], A[(MA + 1) * (MA + 1)];
  int piv[MA + 1];
  int iter = 0, conv;
  do {
    for (int a = 1; a <= na; ++a) ionfrc(&m->atoms[a - 1], T, N[0], fk[a], df[a]);
    for (int mm = 0; mm < nm; ++mm) {
      nmd[mm] = 1.0 / (K[mm] * C_K * T);
      for (int a = 0; a <= na; ++a) dm[mm][a] = 0.0;
      for (int i = 0; i < m->mols[mm].ncomp; ++i) {
        int a = cmpidx[mm][i], z = cmpion[mm][i];
        nmd[mm] *= fk[a][z] * N[a] * C_K * T;
        dm[mm][a] += 1.0 / N[a];
        dm[mm][0] += df[a][z] / fk[a][z];
      }
      for (int a = 0; a <= na; ++a) dm[mm][a] *= nmd[mm];
    }
    d[0] = -N[0];
    for (int a = 1; a <= na; ++a)
      for (int i = 0; i < nk[a]; ++i) d[0] += N[a] * fk[a][i] * (double)i;
    for (int mm = 0; mm < nm; ++mm) d[0] += q[mm] * nmd[mm];
    d[1] = N[0] - Nt;
    for (int a = 1; a <= na; ++a) d[1] += N[a];
    for (int mm = 0; mm < nm; ++mm) d[1] += nmd[mm];
    double Nr = N[1];
    for (int mm = 0; mm < nm; ++mm) Nr += nmd[mm] * (double)(molmul[mm][1]);
    for (int a = 2; a <= na; ++a) {
      double Nc = N[a];
      for (int mm = 0; mm < nm; ++mm) Nc += nmd[mm] * (double)(molmul[mm][a]);
      d[a] = abund[a] * Nr - abund[1] * Nc;
    }
    /* Jacobian, row-major A[row][col] */
    A[0] = -1.0;
    for (int a = 1; a <= na; ++a)
      for (int i = 1; i < nk[a]; ++i) A[0] += N[a] * df[a][i] * (double)i;
    for (int mm = 0; mm < nm; ++mm) A[0] += q[mm] * dm[mm][0];
    A[1 * n + 0] = 1.0;
    for (int mm = 0; mm < nm; ++mm) A[1 * n + 0] += dm[mm][0];
    double dNr = 0.0;
    for (int mm = 0; mm < nm; ++mm) dNr += dm[mm][0] * (double)(molmul[mm][1]);
    for (int a = 2; a <= na; ++a) {
      double dNc = 0.0;
      for (int mm = 0; mm < nm; ++mm) dNc += dm[mm][0] * (double)(molmul[mm][a]);
      A[a * n + 0] = abund[a] * dNr - abund[1] * dNc;
    }
    for (int b = 1; b <= na; ++b) {
      A[0 * n + b] = 0.0;
      for (int i = 0; i < nk[b]; ++i) A[0 * n + b] += fk[b][i] * (double)i;
      for (int mm = 0; mm < nm; ++mm) A[0 * n + b] += q[mm] * dm[mm][b];
      A[1 * n + b] = 1.0;
      for (int mm = 0; mm < nm; ++mm) A[1 * n + b] += dm[mm][b];
      dNr = 0.0;
      for (int mm = 0; mm < nm; ++mm) dNr += dm[mm][b] * (double)(molmul[mm][1]);
      if (b == 1) dNr += 1.0;
      for (int a = 2; a <= na; ++a) {
        double dNc = 0.0;
        for (int mm = 0; mm < nm; ++mm) dNc += dm[mm][b] * (double)(molmul[mm][a]);
        if (b == a) dNc += 1.0;
        A[a * n + b] = abund[a] * dNr - abund[1] * dNc;
      }
    }
    double v[MA + 1];
    for (int i = 0; i < n; ++i) v[i] = d[i];
    gauss_solve(n, A, v, piv);
    int finite = 1;
    for (int a = 0; a <= na; ++a) {
      N[a] -= v[a];
      if (N[a] < 1E-2) N[a] = 1E-2;
      finite &= isfinite(N[a]) != 0;
    }
    if (!finite && warm) goto cold;
    iter += 2;   /* ++iter in the message and iter++ after it (atmos_chm.cc:294, 300) */
    if (iter > 2 * maxpass) {
      if (warm) goto cold;
      break;
    }
    conv = 1;
    for (int i = 0; i <= na; ++i) if (fabs(d[i] / N[i]) > 1E-4) conv = 0;
  } while (!conv);
  if (g_chem_start == SNAPI_CHEM_START_CONTINUE) {  /* keep what the next start predicts from */
    memcpy(out->LU, A, sizeof(double) * n * n);
    memcpy(out->piv, piv, sizeof(int) * n);
    out->lu_n = n;
    out->lu_T = T;
    if (out->nhist == 0 || T != out->T1) {
      memcpy(out->lx2, out->lx1, sizeof(double) * n);
      out->T2 = out->T1;
      if (out->nhist < 2) out->nhist++;
    }
    for (int a = 0; a <= na; ++a) out->lx1[a] = log(N[a] / Nt);
    out->T1 = T;
  }
  out->Ne = N[0];
  out->have = 1;
  out->Nt_prev = Nt;
  out->passes = iter > 2 * maxpass ? -iter / 2 : iter / 2;
  for (int a = 1; a <= na; ++a) {
    out->Natom[a - 1] = N[a];
    for (int z = 0; z < nk[a]; ++z) out->fk[a - 1][z] = fk[a][z];
  }
}

/* ---- atom::pupdate + atom::lte: stage totals and level populations ------------------------------ */
typedef struct {
  double Nst[MA][MS];
  double n[MA][MS][ML];
} pops;

static void lte_pops(const snapi_eos_model *m, double T, const chem_state *c, pops *P) {
  for (int a = 0; a < m->natom; ++a) {
    const snapi_eos_atom *A = &m->atoms[a];
    for (int z = 0; z < A->nstage; ++z) {
      P->Nst[a][z] = c->Natom[a] * c->fk[a][z];
      double U = pf_U(&A->pf[z], T, c->Ne);
      for (int l = 0; l < A->nlevel[z]; ++l) {
        double g = A->level[z][l].g;
        P->n[a][z][l] = P->Nst[a][z] * ((g) ? g * exp(-A->level[z][l].ee / (C_K * T)) / U : 1.0);
      }
    }
  }
}

/* bound-free departure-corrected population term of atom_rad.cc:169-174 (without sigma) */
static double bf_popmod(const snapi_eos_atom *A, const double (*n)[ML], int z, int l, double T, double Ne) {
  return n[z + 1][0] * Ne * C_SAHA * pow(T, -1.5) * A->level[z][l].g / A->level[z + 1][0].g *
         exp((A->ip[z] - A->level[z][l].ee) / C_K / T);
}

/* atmosphere::opacity_continuum at lambda (which = 0: the HE wavelength and sigma_he, 1: kappa) */
static double opacity_continuum(const snapi_eos_model *m, double T, double Ne, const pops *P, int which) {
  double lambda = which ? m->lambda_kappa : m->lambda_he;
  double op_cont = 6.65E-25 * Ne;
  for (int a = 0; a < m->natom; ++a) {
    const snapi_eos_atom *A = &m->atoms[a];
    if (A->nlte) continue;
    double op = 0.0;
    for (int z = 0; z < A->nstage - 1; ++z)
      for (int l = 0; l < A->nlevel[z]; ++l) {
        double sigma = which ? A->level[z][l].sigma_kappa : A->level[z][l].sigma_he;
        if (sigma) {
          double pop_mod = bf_popmod(A, P->n[a], z, l, T, Ne);
          op += sigma * (P->n[a][z][l] - pop_mod * exp(-C_H * C_C / lambda / C_K / T));
        }
      }
    op_cont += op;
  }
  for (int mm = 0; mm < m->nmol; ++mm) {
    if (m->mols[mm].eqc != SNAPI_EQC_HMIN) continue;
    static const double ca[7] = {1.99654, -1.18267E-5, 2.64243E-6, -4.40524E-10, 3.23992E-14, -1.39568E-18,
                                 2.78701E-23};
    double alpha = 0.0;
    for (int i = 0; i < 7; ++i) alpha += ca[i] * pow(lambda * 1E8, i);
    double nH0 = P->Nst[0][0];
    double T_P = 5040. / T;
    double op_bf = 4.158E-28 * alpha * Ne * C_K * T * pow(T_P, 2.5) * pow(10.0, 0.754 * T_P) * nH0 *
                   (1.0 - exp(-C_H * C_C / lambda / C_K / T));
    double l = log10(lambda * 1E8);
    double f_0 = -2.2763 - 1.6850 * l + 0.76661 * l * l - 0.053346 * l * l * l;
    double f_1 = 15.2827 - 9.2846 * l + 1.99381 * l * l - 0.142631 * l * l * l;
    double f_2 = -197.789 + 190.266 * l - 67.9775 * l * l + 10.6913 * l * l * l - 0.625151 * l * l * l * l;
    T_P = 5040. / T;
    double op_ff = 1E-26 * Ne * C_K * T * pow(10.0, f_0 + f_1 * log10(T_P) + f_2 * log10(T_P) * log10(T_P)) * nH0;
    op_cont += op_bf + op_ff;
  }
  return op_cont;
}

/* one (T, Nt) point: chemistry, populations, kappa (which as above) */
static double chem_point(const snapi_eos_model *m, double T, double Nt, chem_state *c, pops *P, int which) {
  chemeq(m, T, Nt, c);
  lte_pops(m, T, c, P);
  return opacity_continuum(m, T, c->Ne, P, which);
}

/* ---- interpolation (mathtools.cc) --------------------------------------------------------------- */
static double interpol_1d(const double *f, const double *x, int N, double xq) {
  if (xq < x[N - 1] && xq > x[0]) {
    int i;
    for (i = 0; i <= N - 2; ++i)
      if (xq < x[i + 1]) break;
    double h1 = 0.0, h2 = 0.0, d1, d2, fd1, fd2;
    if (i > 0) {
      h1 = x[i] - x[i - 1];
      h2 = x[i + 1] - x[i];
      d1 = (f[i] - f[i - 1]) / h1;
      d2 = (f[i + 1] - f[i]) / h2;
      double alpha = 1.0 / 3.0 * (1.0 + h2 / (h1 + h2));
      fd1 = (d1 * d2 > 0) ? d1 * d2 / (alpha * d2 + (1.0 - alpha) * d1) : 0.0;
    } else {
      fd1 = (f[1] - f[0]) / (x[1] - x[0]);
      h2 = x[1] - x[0];   /* unset in the reference */
      h1 = x[1] - x[0];
    }
    double C0 = f[i] + h2 * 0.5 * fd1;
    if (i + 1 < N - 1) {
      h1 = x[i + 1] - x[i];
      h2 = x[i + 2] - x[i + 1];
      d1 = (f[i + 1] - f[i]) / h1;
      d2 = (f[i + 2] - f[i + 1]) / h2;
      double alpha = 1.0 / 3.0 * (1.0 + h2 / (h1 + h2));
      fd2 = (d1 * d2 > 0) ? d1 * d2 / (alpha * d2 + (1.0 - alpha) * d1) : 0.0;
    } else
      fd2 = (f[N - 1] - f[N - 2]) / (x[N - 1] - x[N - 2]);
    double C1 = f[i + 1] - h1 * 0.5 * fd2;
    double C = (C0 + C1) * 0.5;
    double u = (xq - x[i]) / (x[i + 1] - x[i]);
    return (1.0 - u) * (1.0 - u) * f[i] + u * u * f[i + 1] + u * 2.0 * (1.0 - u) * C;
  } else if (xq >= x[N - 1])
    return f[N - 1];
  return f[0];
}

/* atmospheric_interpolation of N nodes (tau, val) onto the grid lt[nd] */
static void atm_interp(const double *tau, const double *val, int N, const double *lt, int nd, double *q, int is_temp) {
  if (N > 1) {
    double der[SNAPI_EOS_MAX_PAR];
    der[0] = 0.0;
    if (!is_temp) der[N - 1] = 0.0;
    else {
      static const double d_T_falc[11] = {1694.91525424, 2164.5021645, 2342.50815695, 2289.18827635, 2155.92183045,
                                          2094.90240415, 2080.69183003, 2066.44925898, 1960.27182436, 1826.11342193,
                                          1729.74468968};
      static const double tau_falc[11] = {-0.01232, 0.08798, 0.2002, 0.32704, 0.46667, 0.61462, 0.7674,
                                          0.92221, 1.07711, 1.22829, 1.37282};
      if (tau[N - 1] < tau_falc[0]) der[N - 1] = d_T_falc[0];
      else if (tau[N - 1] > tau_falc[10]) der[N - 1] = d_T_falc[10];
      else der[N - 1] = interpol_1d(d_T_falc, tau_falc, 11, tau[N - 1]);
    }
    for (int i = 1; i <= N - 2; ++i) {
      double h1 = tau[i] - tau[i - 1], h2 = tau[i + 1] - tau[i];
      double d1 = (val[i] - val[i - 1]) / h1, d2 = (val[i + 1] - val[i]) / h2;
      der[i] = 0.0;
      if (d1 * d2 > 0) {
        double alpha = 0.3333333 * (1.0 + h2 / (h1 + h2));
        der[i] = d1 * d2 / (alpha * d2 + (1.0 - alpha) * d1);
      }
    }
    for (int x = 0; x < nd; ++x) {
      if (lt[x] < tau[0]) q[x] = val[0] + der[0] * (lt[x] - tau[0]);
      else if (lt[x] > tau[N - 1]) q[x] = val[N - 1] + der[N - 1] * (lt[x] - tau[N - 1]);
      else {
        int ii;
        for (ii = 0; ii < N - 1; ++ii)
          if (lt[x] <= tau[ii + 1]) break;
        double E = val[ii] + (tau[ii + 1] - tau[ii]) / 3.0 * der[ii];
        double F = val[ii + 1] - (tau[ii + 1] - tau[ii]) / 3.0 * der[ii + 1];
        double u = (lt[x] - tau[ii]) / (tau[ii + 1] - tau[ii]);
        q[x] = (1.0 - u) * (1.0 - u) * (1.0 - u) * val[ii] + u * u * u * val[ii + 1] + 3.0 * u * (1.0 - u) * (1.0 - u) * E +
               3.0 * u * u * (1.0 - u) * F;
      }
    }
    if (is_temp)
      for (int x = 0; x < nd; ++x) {
        if (q[x] < 3400.0) q[x] = 3400.0;
        if (q[x] > 20000.0) q[x] = 20000.0;
      }
  } else if (N == 1) {
    for (int x = 0; x < nd; ++x) q[x] = val[0];
  } else {
    for (int x = 0; x < nd; ++x) q[x] = 0.0;
  }
}

/* ---- the column ---------------------------------------------------------------------------------- */
#define MAXD 1024
typedef struct {
  double lt[MAXD], T[MAXD], vt[MAXD], vz[MAXD], B[MAXD], th[MAXD], ph[MAXD], Nt[MAXD];
  int status;
} column;

static void kind_nodes(const snapi_eos_model *m, const double *nodes, int kind, double *tau, double *val, int *N) {
  *N = 0;
  for (int p = 0; p < m->npar; ++p)
    if (m->node_kind[p] == kind) { tau[*N] = m->node_tau[p]; val[*N] = nodes[p]; ++*N; }
}

/* node interpolation of every quantity; build = 1: build_from_nodes' defaults (B, theta, phi TINY =
 * 1e-3 when nodeless, theta floored at TINY), 0: interpolate_from_nodes' (B 0) */
static void interp_all(const snapi_eos_model *m, int nd, const double *nodes, column *c, int build) {
  double tau[SNAPI_EOS_MAX_PAR], val[SNAPI_EOS_MAX_PAR];
  int N;
  for (int x = 0; x < nd; ++x) c->lt[x] = m->tau_min + (m->tau_max - m->tau_min) / (nd - 1) * x;
  kind_nodes(m, nodes, 1, tau, val, &N); atm_interp(tau, val, N, c->lt, nd, c->T, 1);
  kind_nodes(m, nodes, 2, tau, val, &N); atm_interp(tau, val, N, c->lt, nd, c->vt, 0);
  kind_nodes(m, nodes, 3, tau, val, &N); atm_interp(tau, val, N, c->lt, nd, c->vz, 0);
  kind_nodes(m, nodes, 4, tau, val, &N);
  if (N) atm_interp(tau, val, N, c->lt, nd, c->B, 0);
  else for (int x = 0; x < nd; ++x) c->B[x] = build ? 1E-3 : 0.0;
  kind_nodes(m, nodes, 5, tau, val, &N);
  if (N) atm_interp(tau, val, N, c->lt, nd, c->th, 0);
  else for (int x = 0; x < nd; ++x) c->th[x] = 1E-3;
  if (build)
    for (int x = 0; x < nd; ++x) if (fabs(c->th[x]) < 1E-3) c->th[x] = 1E-3;
  kind_nodes(m, nodes, 6, tau, val, &N);
  if (N) atm_interp(tau, val, N, c->lt, nd, c->ph, 0);
  else for (int x = 0; x < nd; ++x) c->ph[x] = 1E-3;
}

/* hydrostatic equilibrium (atmos_pp.cc:184-238) -> Nt */
static void hydrostatic(const snapi_eos_model *m, int nd, column *c) {
  chem_state cs;
  pops P;
  const int MAX_ITER = 20;
  const double break_me = 1E-2;
  double op[MAXD], rho[MAXD];
  chem_reset(&cs);
  c->Nt[0] = 0.3 / C_K / c->T[0];
  for (int iter = 0; iter < MAX_ITER; ++iter) {
    op[0] = chem_point(m, c->T[0], c->Nt[0], &cs, &P, 0);
    if (cs.passes < 0) c->status |= 1;
    rho[0] = cs.Natom[0] * 1.4 * 1.67E-24;
    double dN = (pow(10.0, c->lt[0]) * rho[0] * m->grav / op[0]) / C_K / c->T[0] - c->Nt[0];
    c->Nt[0] += dN;
    if (fabs(dN / c->Nt[0]) < break_me) break;
    if (iter == MAX_ITER - 1) c->status |= 2;
  }
  for (int x = 1; x < nd; ++x) {
    double delta_tau = (pow(10, c->lt[x]) - pow(10, c->lt[x - 1]));
    double delta_p = rho[x - 1] * m->grav / op[x - 1] * delta_tau;
    c->Nt[x] = (c->Nt[x - 1] * C_K * c->T[x - 1] + delta_p) / C_K / c->T[x];
    for (int iter = 0; iter < MAX_ITER; ++iter) {
      op[x] = chem_point(m, c->T[x], c->Nt[x], &cs, &P, 0);
      if (cs.passes < 0) c->status |= 1;
      rho[x] = cs.Natom[0] * 1.4 * 1.67E-24;
      double kappa_mean = sqrt(op[x] * op[x - 1] / rho[x] / rho[x - 1]);
      delta_p = m->grav / kappa_mean * delta_tau;
      double dN = (c->Nt[x - 1] * C_K * c->T[x - 1] + delta_p) / C_K / c->T[x] - c->Nt[x];
      c->Nt[x] += dN;
      if (fabs(dN / c->Nt[0]) < break_me) break;
      if (iter == MAX_ITER - 1) c->status |= 2;
    }
  }
}

static double planck_f(double lambda, double T) {
  return 2.0 * 6.62606957 * 8.9875517E-7 / lambda / lambda / lambda / lambda / lambda / (exp(1.4387769 / lambda / T) - 1.0);
}

/* the record fields of one depth from (T, Nt) and the interpolated kinematics / field */
static void record_depth(const snapi_eos_model *m, int nlines, const double *lam0, const double *mass, const column *c,
                         int x, double *r, int *status) {
  chem_state cs;
  pops P;
  const double T = c->T[x];
  chem_reset(&cs);  /* record solves start cold in either mode (their fields follow the solve's path) */
  double kap = chem_point(m, T, c->Nt[x], &cs, &P, 1);
  if (cs.passes < 0) *status |= 1;
  const double Ne = cs.Ne;
  /* project / transform (atmos_rad.cc:14-48) with V_x = V_y = 0 */
  double w3 = cos(C_PI - m->theta);
  double vlos = sin(m->phi) * sin(C_PI - m->theta) * 0.0 + cos(m->phi) * sin(C_PI - m->theta) * 0.0 + w3 * c->vz[x];
  double Bx = c->B[x] * sin(c->th[x]) * cos(c->ph[x]);
  double By = c->B[x] * sin(c->th[x]) * sin(c->ph[x]);
  double Bz = c->B[x] * cos(c->th[x]);
  double cp = cos(m->phi), sp = sin(m->phi), ct = cos(C_PI - m->theta), st = sin(C_PI - m->theta);
  double mg = sqrt(Bx * Bx + By * By + Bz * Bz);
  double nBx = ct * cp * Bx + sp * By - st * cp * Bz;
  double nBy = -ct * sp * Bx + cp * By + st * sp * Bz;
  double nBz = st * Bx + ct * Bz;
  r[0] = T;
  r[1] = c->vt[x];
  r[2] = Ne;
  r[3] = vlos;
  r[4] = mg;
  r[5] = acos(nBz / mg) * 180.0 / C_PI;
  r[6] = atan(nBy / nBx) * 180.0 / C_PI;
  r[7] = kap;
  double nH0 = P.Nst[0][0], tp = 5040.0 / T;
  int hm = 0;
  for (int mm = 0; mm < m->nmol; ++mm) if (m->mols[mm].eqc == SNAPI_EQC_HMIN) hm = 1;
  r[8] = hm ? 4.158E-28 * Ne * C_K * T * pow(tp, 2.5) * pow(10.0, 0.754 * tp) * nH0 : 0.0;
  r[9] = hm ? 1E-26 * Ne * C_K * T * nH0 : 0.0;
  /* bound-free totals of the window (atom::boundfree_op_em_vector), all atoms */
  double bop = 0.0, bem = 0.0;
  for (int a = 0; a < m->natom; ++a) {
    const snapi_eos_atom *A = &m->atoms[a];
    for (int z = 0; z < A->nstage - 1; ++z)
      for (int l = 0; l < A->nlevel[z]; ++l) {
        double lw = A->level[z][l].lambda_win;
        if (!(lw > 0.0)) continue;
        double sigma = A->level[z][l].sigma_win;
        double pop_mod = bf_popmod(A, P.n[a], z, l, T, Ne);
        double op_loc = sigma * (P.n[a][z][l] - pop_mod * exp(-C_H * C_C / lw / C_K / T));
        double em_loc = sigma * pop_mod * (1.0 - exp(-C_H * C_C / lw / C_K / T)) * planck_f(lw, T);
        bop += op_loc;
        bem += em_loc;
      }
  }
  r[10] = bop;
  r[11] = bem;
  for (int j = 0; j < nlines; ++j) {
    const snapi_eos_line *L = &m->lines[j];
    const double *nn = P.n[L->atom][L->stage];
    r[SNAPI_NFIELD0 + 3 * j + 0] = (nn[L->lower] * L->Blu - nn[L->upper] * L->Bul) * C_H * C_C / lam0[j] / 4.0 / C_PI;
    r[SNAPI_NFIELD0 + 3 * j + 1] = nn[L->upper] * L->A * C_H * C_C / lam0[j] / 4.0 / C_PI;
    double red_mass = 1.66E-24 / (1.0 / 1.008 + 1.66E-24 / mass[j]);
    double vmean = sqrt(8.0 * C_K * T / C_PI / red_mass);
    r[SNAPI_NFIELD0 + 3 * j + 2] = nH0 * vmean * pow(vmean / 1E6, -L->alpha_col) * L->sigma_col;
  }
}

/* ---- exported ------------------------------------------------------------------------------------ */

/* The chemistry start of the following calls (SNAPI_CHEM_START_COLD or _CONTINUE); returns the old. */
int sne_set_chem_start(int mode) {
  const int old = g_chem_start;
  g_chem_start = mode;
  return old;
}

/* Chemistry of one (T, Nt) point: Ne, stage totals [natom][MS], level populations [natom][MS][ML],
 * kappa at lambda_he and lambda_kappa.  Returns the Newton passes (negative: cap reached). */
int sne_chem(const snapi_eos_model *m, double T, double Nt, double *Ne, double *Nst, double *npop, double *kap_he,
             double *kap) {
  chem_state cs;
  pops P;
  chem_reset(&cs);
  *kap_he = chem_point(m, T, Nt, &cs, &P, 0);
  *kap = opacity_continuum(m, T, cs.Ne, &P, 1);
  *Ne = cs.Ne;
  for (int a = 0; a < m->natom; ++a)
    for (int z = 0; z < MS; ++z) {
      Nst[a * MS + z] = z < m->atoms[a].nstage ? P.Nst[a][z] : 0.0;
      for (int l = 0; l < ML; ++l)
        npop[(a * MS + z) * ML + l] = (z < m->atoms[a].nstage && l < m->atoms[a].nlevel[z]) ? P.n[a][z][l] : 0.0;
    }
  return cs.passes;
}

/* One column: T [nd], Nt [nd] (HE) and the record [nd][nfield] of the node vector; returns the
 * status bits (1 chemistry cap, 2 HE cap). */
int sne_build(const snapi_eos_model *m, int nd, int nlines, const double *lam0, const double *mass,
              const double *nodes, double *T, double *Nt, double *rec) {
  static column c;
  if (nd > MAXD || nd < 2) return -1;
  c.status = 0;
  interp_all(m, nd, nodes, &c, 1);
  hydrostatic(m, nd, &c);
  const int nf = SNAPI_NFIELD0 + 3 * nlines;
  for (int x = 0; x < nd; ++x) {
    if (T) T[x] = c.T[x];
    if (Nt) Nt[x] = c.Nt[x];
    if (rec) record_depth(m, nlines, lam0, mass, &c, x, rec + (size_t)x * nf, &c.status);
  }
  return c.status;
}

/* The 12 rows of atmosphere::return_as_array (atmos.cc:547-569) of the node vector's column after
 * build_from_nodes and compute_op_referent (atmos_ppbez_rts.cc:268-281): out [12][nd]; x3 [nd]
 * the heights (NULL: 0).  Returns the status bits as sne_build. */
int sne_atmos(const snapi_eos_model *m, int nd, const double *nodes, const double *x3, double *out) {
  static column c;
  if (nd > MAXD || nd < 2) return -1;
  c.status = 0;
  interp_all(m, nd, nodes, &c, 1);
  hydrostatic(m, nd, &c);
  const double bx0 = c.B[0] * sin(c.th[0]) * cos(c.ph[0]);
  for (int x = 0; x < nd; ++x) {
    chem_state cs;
    pops P;
    chem_reset(&cs);
    const double kap = chem_point(m, c.T[x], c.Nt[x], &cs, &P, 1);
    if (cs.passes < 0) c.status |= 1;
    const double Bx = c.B[x] * sin(c.th[x]) * cos(c.ph[x]);
    const double By = c.B[x] * sin(c.th[x]) * sin(c.ph[x]);
    const double Bz = c.B[x] * cos(c.th[x]);
    const double mg = sqrt(Bx * Bx + By * By + Bz * Bz);
    const double tau = -pow(10.0, c.lt[x]);
    double r[12] = {log10(-tau), x3 ? x3[x] : 0.0, c.T[x], c.Nt[x] * C_K * c.T[x], cs.Ne * C_K * c.T[x], 0.0, kap,
                    mg, c.vt[x], c.vz[x], acos(Bz / mg), atan(By / bx0)};
    for (int k = 0; k < 12; ++k) out[(size_t)k * nd + x] = r[k];
  }
  return c.status;
}

/* The record [nd][nfield] of a given column in the 12-row layout of sne_atmos, as
 * atmosphere::read_spinor3d reads it (atmos_fio.cc:100-121: T floored at 3200 K, Nt = Pg / (k T))
 * and obs_stokes' set-up completes it.  Returns the status bits as sne_build. */
int sne_columns(const snapi_eos_model *m, int nd, int nlines, const double *lam0, const double *mass,
                const double *cols, double *rec) {
  static column c;
  if (nd > MAXD || nd < 2) return -1;
  c.status = 0;
  for (int x = 0; x < nd; ++x) {
    const double T = cols[2 * nd + x] > 3200.0 ? cols[2 * nd + x] : 3200.0;
    c.lt[x] = cols[x];
    c.T[x] = T;
    c.Nt[x] = cols[3 * nd + x] / (C_K * T);
    c.B[x] = cols[7 * nd + x];
    c.vt[x] = cols[8 * nd + x];
    c.vz[x] = cols[9 * nd + x];
    c.th[x] = cols[10 * nd + x];
    c.ph[x] = cols[11 * nd + x];
  }
  const int nf = SNAPI_NFIELD0 + 3 * nlines;
  for (int x = 0; x < nd; ++x) record_depth(m, nlines, lam0, mass, &c, x, rec + (size_t)x * nf, &c.status);
  return c.status;
}

/* Node tangents [npar][nd][nfield] by central differences (steps [npar]; NULL: the reference's). */
int sne_tangents(const snapi_eos_model *m, int nd, int nlines, const double *lam0, const double *mass,
                 const double *nodes, const double *step, double *tan) {
  static column cp, cm;
  static double rp[MAXD * (SNAPI_NFIELD0 + 3 * SNAPI_MAX_LINES)], rm[MAXD * (SNAPI_NFIELD0 + 3 * SNAPI_MAX_LINES)];
  const int nf = SNAPI_NFIELD0 + 3 * nlines;
  double nv[SNAPI_EOS_MAX_PAR];
  int status = 0;
  for (int p = 0; p < m->npar; ++p) {
    static const double ref_step[7] = {0.0, 5.0, 20.0, 20.0, 0.01, 0.001, 0.001};
    int kind = m->node_kind[p];
    double st = step ? step[p] : ref_step[kind];
    for (int side = 0; side < 2; ++side) {
      column *c = side ? &cm : &cp;
      double *r = side ? rm : rp;
      memcpy(nv, nodes, sizeof(double) * m->npar);
      c->status = 0;
      if (kind == 1) {
        nv[p] += side ? -0.5 * st : 0.5 * st;
        interp_all(m, nd, nv, c, 1);
        hydrostatic(m, nd, c);
      } else {
        interp_all(m, nd, nv, c, 1);
        hydrostatic(m, nd, c);
        nv[p] += side ? -0.5 * st : 0.5 * st;
        column tmp = *c;
        interp_all(m, nd, nv, &tmp, 0);
        memcpy(c->vt, tmp.vt, sizeof tmp.vt); memcpy(c->vz, tmp.vz, sizeof tmp.vz);
        memcpy(c->B, tmp.B, sizeof tmp.B); memcpy(c->th, tmp.th, sizeof tmp.th); memcpy(c->ph, tmp.ph, sizeof tmp.ph);
        memcpy(c->T, tmp.T, sizeof tmp.T);
      }
      for (int x = 0; x < nd; ++x) record_depth(m, nlines, lam0, mass, c, x, r + (size_t)x * nf, &c->status);
      status |= c->status;
    }
    for (int i = 0; i < nd * nf; ++i) {
      /* a kinematic / field node moves only its own fields (v_turb 1, v_los 3, the field 4-6); the
         others are unchanged (their difference is 0, or NaN - NaN where B = 0 without B nodes) */
      const int f = i % nf;
      const int kin = (f == 1 || (f >= 3 && f <= 6));
      const int own = kind == 2 ? f == 1 : (kind == 3 ? f == 3 : (f >= 4 && f <= 6));
      tan[(size_t)p * nd * nf + i] = (kind != 1 && kin && !own) ? 0.0 : (rp[i] - rm[i]) / st;
    }
  }
  return status;
}
