// snapi_eos.cu -- node model -> column records on the device (snapi_eos_set, snapi_build_records).
//
// The reference builds each pixel's atmosphere from its nodes on the host before every synthesis
// (atmos_pp::build_from_nodes, atmos/plpar/atmos_pp.cc:58-248): node interpolation, hydrostatic
// equilibrium with the chemistry, LTE populations and the continuum opacity at every step, and,
// for the fit, two more builds per temperature node for the record tangents (atmos_fit.cc:
// 1225-1307).  Here that whole map runs on the GPU in FP64 (the chemistry spans 40 decades and
// its Newton system is badly scaled, so FP32 is not an option; the B200's FP64 rate is half its
// FP32 rate):
//
//   k_eos_he   one thread per (pixel, variant): the column's temperature from its nodes and the
//              hydrostatic particle densities, depth by depth (inherently serial in depth).
//              Variant 0 is the node vector itself, variants 2i+1 / 2i+2 move temperature node i
//              by +- step / 2.  Threads are ordered pixel-fastest, so a warp holds 32 pixels of the
//              same variant at the same depth: similar (T, Nt), similar iteration counts.
//   k_eos_var  one thread per (pixel, variant, depth): the chemistry at the final (T, Nt) and the
//              thermal record fields, FP64 (a tangent is a 5 K difference of them).
//   k_eos_rec  one thread per (depth, pixel): the records, and the tangent rows (thermal nodes from
//              the variants, kinematic / field nodes by re-interpolation).
//
// The chemistry (atmosphere::chemeq, atmos/atmos_chm.cc:28-330) is evaluated per call in the
// reference's steps, with what depends on T alone hoisted out of the ~20 ionisation sweeps of a
// call: the Traving partition sums over tabulated levels (partf.cc:224-228), the asymptotic-term
// weights g2 exp(-2.302585 ee x), the Boltzmann factors of the ionisation energies and the
// molecular equilibrium constants.  A sweep then costs per stage one Fischel-Sparks polynomial
// per asymptotic term and one division.  The 10 x 10 Newton system is solved by Gaussian
// elimination with partial pivoting (the reference: SVD, same solution).  Loops the reference
// leaves unbounded (the halving of its starting electron density) are capped at 400 passes and
// flag the pixel.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "snapi_internal.cuh"

namespace snapi {
namespace {

constexpr int kEA = SNAPI_EOS_MAX_ATOMS;  // atoms
constexpr int kES = 64;                   // ionisation stages over all atoms
constexpr int kET = 96;                   // Traving asymptotic terms over all stages
constexpr int kEC = 512;                  // Traving / Irwin coefficients over all terms
constexpr int kEM = SNAPI_EOS_MAX_MOLS;   // molecules
constexpr int kER = 32;                   // stages whose ionisation fraction is kept per sweep
constexpr int kEL = 64;                   // levels whose population enters a record
constexpr int kEB = 32;                   // bound-free levels
constexpr int kEP = SNAPI_EOS_MAX_PAR;    // nodes
constexpr int kEBm = 8;                    // bound-free edges of the march's opacity (compact path)
constexpr int kELm = 16;                   // their levels
constexpr int kRecThreads = 64;
constexpr int kPolishCap = 400;

// the reference's constants (cmlib/const.h, CGS)
constexpr double cPI = 3.141592653589793238462643383279502884197169399375105;
constexpr double cC = 2.99792458E10, cH = 6.6260687652E-27, cK = 1.3806503E-16, cME = 9.1093818872E-28;
constexpr double cE = 4.8032042510E-10, cRYD = 1.097373156853955E5, cE0 = 7.957747154594775607E-02;
constexpr double cSAHA = 2.0706615382E-16;

// per-stage and per-term constants packed for two 16-byte loads each in the ionisation sweep
struct __align__(16) StageTab {
  double zf, izf;  // Traving: z f and its inverse
  double zz;       // Traving: 31.321 z^2 (the asymptotic term's D_z is zz x, x = 5040 / T)
  int t0, t1;      // Traving asymptotic terms [t0, t1) (empty for the other types)
  int ref, pad;    // kept-fraction slot (-1 none)
};
struct __align__(16) TermTab {
  double l, il, A, g2;  // l, 1/l, ((1/3 (l-1) - 1/2)(l-1) - 1/6)(l-1), g2
};

struct EosDev {
  int natom, nmol, nst, nlev, nbf, nlines, npar, nd, nref, hm, href;
  double lambda_he, lambda_kappa, grav, tau_min, tau_max, theta, phi, ftrav;
  double abund[kEA];
  int s0[kEA], ns[kEA];
  int zkeep[kEA];  // 1 + the highest stage of the atom with a kept fraction (0: none)
  // the Newton system reduced to the electrons, hydrogen and the atoms in molecules: nr unknowns,
  // rfull[i] the full index (0 electrons, a + 1 atom a) of reduced unknown i, rmap the inverse
  // (-1: an atom in no molecule, eliminated); simple[0..nsimple) those atoms' full indices
  int nr, nsimple;
  int rfull[kEA + 1], rmap[kEA + 1], simple[kEA];
  int nmref, mrefs[kER];  // the kept-fraction slots that molecule components read
  // the hydrostatic march's opacity (continuum at lambda_he): its LTE bound-free edges and the
  // levels they read, compact (mfast = 0: more than the compact lists hold, the general path)
  int mfast, nbf_m, nlev_m;
  int bf_m[kEBm], bfl_m[kEBm], bfn_m[kEBm];  // bound-free index, its level and next-stage ground in lev_m
  int lev_m[kELm];                           // level slots
  // stages
  int pft[kES];
  double pfv[kES];   // CONST: value; TRAV: g0; NONE: 1
  double zeff[kES];
  double eion[kES];  // ionisation energy to the next stage [erg]
  int t0[kES], t1[kES];  // TRAV: asymptotic terms [t0, t1); IRWIN: coefficients [t0, t1) of cA
  int ref[kES];      // kept-fraction slot, -1 none
  int satom[kES];    // atom of each stage
  // Traving asymptotic terms and level sums
  double g2[kET], tee[kET], tll[kET], til[kET], tA[kET];  // til = 1/l, tA = ((1/3 (l-1) - 1/2)(l-1) - 1/6)(l-1)
  double zf[kES], izf[kES];  // Traving: z * f (Fischel-Sparks cut constant) and its inverse
  StageTab stab[kES];
  TermTab ttab[kET];
  int c0[kET], c1[kET];
  double cA[kEC], cG[kEC];
  // molecules (components: 1-based atom, 0 the electron)
  int mnc[kEM];
  int matom[kEM][SNAPI_MOL_MAX_COMP], mref[kEM][SNAPI_MOL_MAX_COMP];
  int mdup[kEM][SNAPI_MOL_MAX_COMP];  // 1: the component's atom is also an earlier component's
  int mmul[kEM][kEA + 1];
  double mq[kEM];
  int meqc[kEM], mncoef[kEM];
  double mcoef[kEM][SNAPI_PF_MAX_COEF];
  // levels entering a record: stage, statistical weight, energy
  int lst[kEL];
  double lg[kEL], lee[kEL];
  // bound-free levels: level, next stage's ground level, LTE flag, cross-sections, window
  int bfl[kEB], bfn[kEB], bflte[kEB];
  double bfg[kEB], bfgn[kEB], bfip[kEB], sig_he[kEB], sig_k[kEB], sig_w[kEB], lam_w[kEB];
  // lines: lower / upper level slots
  int llo[SNAPI_MAX_LINES], lup[SNAPI_MAX_LINES];
  double lBlu[SNAPI_MAX_LINES], lBul[SNAPI_MAX_LINES], lA[SNAPI_MAX_LINES], lalpha[SNAPI_MAX_LINES],
      lsig[SNAPI_MAX_LINES], llam0[SNAPI_MAX_LINES], lmass[SNAPI_MAX_LINES];
  // nodes (kinds contiguous and non-decreasing)
  double ntau[kEP];
  int nkind[kEP];
  int kfirst[7], kcount[7];
};

// ---- the chemistry of one (T, Nt) point, one thread -----------------------------------------------------
// Ionisation sweep (atom::ionfrc, atom.cc:892-925) in division-free form.  The reference chains
// f_z = fct (U_{z+1} / U_z) exp(-chi_z / kT) / ne and fk_{z+1} = fk_z f_z, then normalises; the chain
// telescopes to fk_z = (U_z / U_0) prod_{z'<z} c_{z'} / ne with c = fct exp(-chi / kT) (T only), and
// U_0 cancels in the normalisation, so a stage costs U_z (its Fischel-Sparks terms, whose T-only parts
// are hoisted) and two products.  Likewise the Ne derivative recursion of the reference,
// df_{z+1} = df_z f_z + fk_z f_z (dlnU_{z+1} - dlnU_z - 1/ne), sums to df_z = fk_z (dlnU_z - dlnU_0 - z/ne).
// Traving U (partf.cc:217-238): U = Ut + sum_t w2_t qas_f(l_t, p, Dz) with p = zf / ne^(1/6) and
// qas_f (Fischel-Sparks eq. 26 / 27, partf.cc:256-270) written as
//   p > l:  ((4/3 p + 1/2) p + 1/6 + 4/3 Dz) p - 0.4 Dz^2 / p - (A_l - Dz (l - 1)) + 0.5 Dz^2 / l
//   p <= l: (1 + a (1/3 + a / 10)) p^4 / l,  a = Dz / l^2
// with A_l = ((1/3 (l-1) - 1/2)(l-1) - 1/6)(l-1) and the reference's decimal constants; dU keeps only
// the last term, as trav::dU does (partf.cc:247-248).
//
// One thread per column: a warp holding one column per lane (and sharing its stage loops) issues 32
// columns per instruction.  A warp per column (stages in lanes, butterfly sums) shortens a column's
// chain but measured 14x slower at 4096 columns x 9 variants, where the GPU is full either way.
// R: the kept-fraction capacity (the build kernels: kER; the NLTE set-up keeps every stage)
template <int R>
struct ChemT {
  const EosDev &E;
  double T, kT;
  double x5040;  // 5040 / T
  // per stage, one 16-byte load in the sweep: the thread-local state of a column is what the
  // march's L1 has to hold for every resident column
  struct __align__(16) SLoc {
    double Ut;  // T-only part of U (whole U for CONST / IRWIN / NONE)
    double cz;  // fct exp(-chi / kT): the T-only factor of the stage ratio
  } sl[kES];
  double w2[kET];   // g2 exp(-2.302585 ee x)
  double iKkT[kEM];  // 1 / (K_m k T) of each molecule at this T
  // the march's opacity factors at this T (set_march): stimulated emission, each edge's
  // saha T^-1.5 g / g_next exp(chi / kT), each level's g exp(-E / kT), the H- bf + ff factor
  double mstim, mhm, mcb[kEBm], mlf[kELm];
  double Ea[kEA + 1], Da[kEA + 1];  // sum_i i f_i, sum_i i df_i / dNe per atom (1-based)
  double fr[R], dr[R];              // kept ionisation fractions and their Ne derivatives
  double N[kEA + 1];
  double A[(kEA + 1) * (kEA + 1)], d[kEA + 1];
  int capped;
  int have;        // N holds the solution of an earlier solve of this column, at particle density Nt_prev
  double Nt_prev;
  // the continued start's predictors: after a solve A holds the factors of its last Newton pass's
  // reduced Jacobian in elimination order (piv: the row swapped with row c at step c; with gr the
  // eliminated atoms follow), valid at temperature lu_T when lu_ok; lx1 / lx2: log(N / Nt) of the last solutions at the two latest temperatures
  // T1 (the most recent) and T2, nhist of them held
  int piv[kEA + 1];
  double gr[kEA + 1];  // d(sum_m nmv_m mul_mH) / d x over the reduced unknowns (the last pass's)
  int lu_ok, nhist;
  double lu_T, T1, T2;
  double lx1[kEA + 1], lx2[kEA + 1];

  __device__ explicit ChemT(const EosDev &e) : E(e), T(-1.0), have(0), Nt_prev(0.0), lu_ok(0), nhist(0) {}

  // The whole state as 8-byte words (kStateWords of them), word k of a thread at s[k * stride]: a
  // march split into depth segments carries it from one launch to the next (the layout keeps a
  // warp's accesses coalesced).  Integers travel as doubles (exact).
  static constexpr int kStateWords = 3 + 2 * kES + kET + kEM + 2 + kEBm + kELm + 2 * (kEA + 1) + 2 * R +
                                     (kEA + 1) + (kEA + 1) * (kEA + 1) + (kEA + 1) + 3 + (kEA + 1) + (kEA + 1) +
                                     2 + 3 + 2 * (kEA + 1);
  template <bool kSave, class V>
  __device__ __forceinline__ void state_words(V *s, size_t stride) {
    size_t k = 0;
    auto w = [&](double &v) {
      if (kSave) s[k * stride] = v; else v = s[k * stride];
      ++k;
    };
    auto wi = [&](int &v) {
      double t = (double)v;
      w(t);
      v = (int)t;
    };
    w(T); w(kT); w(x5040);
    for (int i = 0; i < kES; ++i) { w(sl[i].Ut); w(sl[i].cz); }
    for (int i = 0; i < kET; ++i) w(w2[i]);
    for (int i = 0; i < kEM; ++i) w(iKkT[i]);
    w(mstim); w(mhm);
    for (int i = 0; i < kEBm; ++i) w(mcb[i]);
    for (int i = 0; i < kELm; ++i) w(mlf[i]);
    for (int i = 0; i <= kEA; ++i) { w(Ea[i]); w(Da[i]); }
    for (int i = 0; i < R; ++i) { w(fr[i]); w(dr[i]); }
    for (int i = 0; i <= kEA; ++i) w(N[i]);
    for (int i = 0; i < (kEA + 1) * (kEA + 1); ++i) w(A[i]);
    for (int i = 0; i <= kEA; ++i) w(d[i]);
    wi(capped); wi(have); w(Nt_prev);
    for (int i = 0; i <= kEA; ++i) wi(piv[i]);
    for (int i = 0; i <= kEA; ++i) w(gr[i]);
    wi(lu_ok); wi(nhist);
    w(lu_T); w(T1); w(T2);
    for (int i = 0; i <= kEA; ++i) { w(lx1[i]); w(lx2[i]); }
  }
  __device__ void save_state(double *s, size_t stride) { state_words<true>(s, stride); }
  __device__ void load_state(const double *s, size_t stride) { state_words<false>(const_cast<double *>(s), stride); }

  __device__ void set_T(double Tin) {
    T = Tin;
    kT = cK * T;
    const double x = 5040.0 / T;
    x5040 = x;
    const double fct = 2.0 * pow((2.0 * cPI * cME * cK * T) / (cH * cH), 1.5);
    for (int s = 0; s < E.nst; ++s) {
      const int ty = E.pft[s];
      double u = E.pfv[s];
      if (ty == SNAPI_PF_TRAV) {
        for (int t = E.t0[s]; t < E.t1[s]; ++t) {
          for (int c = E.c0[t]; c < E.c1[t]; ++c) u += E.cA[c] * exp(-2.302585 * E.cG[c] * x);
          w2[t] = E.g2[t] * exp(-2.302585 * E.tee[t] * x);
        }
      } else if (ty == SNAPI_PF_IRWIN) {
        const double lnT = log(T);
        double sum = 0.0;
        for (int c = E.t0[s]; c < E.t1[s]; ++c) sum += E.cA[c] * pow(lnT, (double)(c - E.t0[s]));
        u = exp(sum);
      }
      sl[s].Ut = u;
      sl[s].cz = fct * exp(-E.eion[s] / kT);
    }
    for (int m = 0; m < E.nmol; ++m) {
      double k = 0.0;
      if (E.meqc[m] == SNAPI_EQC_POLY) {
        const int n = E.mncoef[m];
        double sum = E.mcoef[m][n - 1];
        for (int i = n - 2; i >= 0; --i) sum = E.mcoef[m][i] + x * sum;
        k = exp(2.302585093 * sum);
      } else if (E.meqc[m] == SNAPI_EQC_HMIN) {
        k = exp(2.302585093 * (0.1249 + (2.5 * log(T) / 2.302585) - 0.747 * x));
      } else if (E.meqc[m] == SNAPI_EQC_CONST) {
        k = E.mcoef[m][0];
      }
      iKkT[m] = 1.0 / (k * kT);
    }
  }

  // the T-only factors of the march's opacity (continuum at lambda_he, atmos_rad.cc:286-294 and
  // mol.cc's H- bound-free / free-free) for the compact path of chem_point
  __device__ void set_march() {
    const double lambda = E.lambda_he;
    mstim = exp(-cH * cC / lambda / cK / T);
    for (int k = 0; k < E.nbf_m; ++k) {
      const int b = E.bf_m[k];
      mcb[k] = cSAHA * pow(T, -1.5) * E.bfg[b] / E.bfgn[b] * exp(E.bfip[b] / cK / T);
    }
    for (int k = 0; k < E.nlev_m; ++k) {
      const int l = E.lev_m[k];
      mlf[k] = E.lg[l] != 0.0 ? E.lg[l] * exp(-E.lee[l] / (cK * T)) : 0.0;
    }
    mhm = 0.0;
    if (E.hm) {
      const double ca[7] = {1.99654, -1.18267E-5, 2.64243E-6, -4.40524E-10, 3.23992E-14, -1.39568E-18, 2.78701E-23};
      double alpha = 0.0;
      for (int i = 0; i < 7; ++i) alpha += ca[i] * pow(lambda * 1E8, (double)i);
      const double T_P = 5040. / T;
      const double l = log10(lambda * 1E8);
      const double f_0 = -2.2763 - 1.6850 * l + 0.76661 * l * l - 0.053346 * l * l * l;
      const double f_1 = 15.2827 - 9.2846 * l + 1.99381 * l * l - 0.142631 * l * l * l;
      const double f_2 = -197.789 + 190.266 * l - 67.9775 * l * l + 10.6913 * l * l * l - 0.625151 * l * l * l * l;
      const double lt = log10(T_P);
      mhm = 4.158E-28 * alpha * cK * T * pow(T_P, 2.5) * pow(10.0, 0.754 * T_P) * (1.0 - mstim) +
            1E-26 * cK * T * pow(10.0, f_0 + f_1 * lt + f_2 * lt * lt);
    }
  }

  // U of a stage and (kDeriv) dU / dNe from its packed constants; ine = 1/ne, pne = ne^(1/6), ipne = 1/pne
  template <bool kDeriv>
  __device__ __forceinline__ void stage_u(const StageTab &S, const SLoc &L, double ine, double pne, double ipne,
                                          double &U, double &dU) const {
    U = L.Ut;
    dU = 0.0;
    if (S.t1 <= S.t0) return;
    const double zf = S.zf, p = zf * ipne, ip = pne * S.izf, dz = S.zz * x5040;
    double dq = 0.0, wl = 0.0;
    for (int t = S.t0; t < S.t1; ++t) {
      const TermTab Tt = E.ttab[t];
      const double l = Tt.l, il = Tt.il;
      double q;
      if (p > l) {
        q = ((1.3333333 * p + 0.5) * p + 0.16666667 + 1.33333333 * dz) * p - 0.4 * dz * dz * ip -
            (Tt.A - dz * (l - 1.0)) + 0.5 * dz * dz * il;
        if (kDeriv) dq = ((3.0 * 1.3333333 * p + 1.0) * p + 0.16666667 + 1.33333333 * dz) + 0.4 * dz * dz * ip * ip;
      } else {
        const double axl2 = dz * il * il, k4 = (1.0 + axl2 * (0.33333333 + 0.1 * axl2)) * il;
        q = k4 * p * p * p * p;
        if (kDeriv) dq = 4.0 * k4 * p * p * p;
      }
      wl = w2[t];
      U += wl * q;
    }
    if (kDeriv) dU = -wl * dq * zf * ine * ipne * (1.0 / 6.0);
  }

  template <bool kDeriv>
  __device__ __forceinline__ void stage_u(int s, double ine, double pne, double ipne, double &U, double &dU) const {
    const StageTab S = E.stab[s];
    const SLoc L = sl[s];
    stage_u<kDeriv>(S, L, ine, pne, ipne, U, dU);
  }

  // atom a (0-based): Ea, and with kDeriv Da and the kept fractions
  template <bool kDeriv>
  __device__ __forceinline__ void sweep_atom(int a, double ine, double pne, double ipne) {
    const int s0 = E.s0[a], ns = E.ns[a], zk = E.zkeep[a];
    int zend = ns;
    double h = 1.0, fsum = 0.0, S1 = 0.0, dfsum = 0.0, S2 = 0.0, dl0 = 0.0;
    for (int z = 0; z < ns; ++z) {
      const StageTab S = E.stab[s0 + z];
      const SLoc L = sl[s0 + z];
      double U, dU;
      stage_u<kDeriv>(S, L, ine, pne, ipne, U, dU);
      const double f = U * h;
      fsum += f;
      S1 += (double)z * f;
      double df = 0.0;
      if (kDeriv) {
        if (z == 0) dl0 = dU / U;
        else df = h * dU - f * (dl0 + (double)z * ine);
        dfsum += df;
        S2 += (double)z * df;
        if (S.ref >= 0) { fr[S.ref] = f; dr[S.ref] = df; }
      }
      h *= L.cz * ine;
      // Past the stages with kept fractions, stop once the next stage's weight is below 1e-30 of
      // the sum: the ionisation energies rise with z, so every further ratio c_z / n_e is smaller
      // than the ones that brought h this low, and the remaining terms (< 1e-26 of each sum with
      // U <= 1e4) cannot change an FP64 sum.
      if (z + 1 >= zk && h < 1e-30 * fsum) {
        zend = z + 1;
        break;
      }
    }
    const double inv = 1.0 / fsum;
    Ea[a + 1] = S1 * inv;
    if (kDeriv) {
      Da[a + 1] = (S2 - dfsum * S1 * inv) * inv;
      for (int z = 0; z < zend; ++z) {
        const int r = E.stab[s0 + z].ref;
        if (r >= 0) { dr[r] = (dr[r] - dfsum * fr[r] * inv) * inv; fr[r] *= inv; }
      }
    }
  }

  template <bool kDeriv>
  __device__ void sweep(double ne) {
    const double ine = 1.0 / ne, pne = cbrt(sqrt(ne)), ipne = 1.0 / pne;
    for (int a = 0; a < E.natom; ++a) sweep_atom<kDeriv>(a, ine, pne, ipne);
  }

  // U of stage s at the final Ne (atom::lte uses the partition function at T, Ne)
  __device__ double stage_U(int s, double ne) const {
    const double pne = cbrt(sqrt(ne));
    double U, dU;
    stage_u<false>(s, 1.0 / ne, pne, 1.0 / pne, U, dU);
    return U;
  }

  // atmosphere::chemeq (atmos_chm.cc:28-330): N[0] = Ne, N[1..na] free atoms; the kept fractions
  // fr are those of the last Newton sweep (before the last update), as pupdate uses them.
  //
  // Two starts.  Cold (warm = false, or no earlier solution): the reference's, at every call --
  // the ionisation-only quadratic for n_e and the halving loop to 1e-2 (atmos_chm.cc:129-171),
  // ~18 of the ~20 ionisation sweeps of a solve.  Continued (warm = true, the hydrostatic march
  // only): Newton from a predicted iterate (predict: a step along dN/dNt at the same depth,
  // ~1.2 passes; a temperature extrapolation at a new depth, ~2.2 passes) or else the previous
  // solution of the same column scaled by the particle-density ratio; if that Newton has not met
  // the stop rule after kWarmPasses passes, or left non-finite values, the cold start runs.  Both
  // stop on the reference's rule (all relative defects below 1e-4 before the last update), so the
  // march's opacities differ by up to that last update's size and its particle densities by
  // ~4e-8 relative (up to ~1e-6 on a model with a temperature node at every depth); the records'
  // own solves always start cold (their stage fractions are those of the last sweep before the
  // final update, i.e. they follow the path).
  static constexpr int kWarmPasses = 8;

  __device__ void solve(double Nt, bool warm) {
    capped = 0;
    if (warm && have) {
      if (!predict(Nt)) {
        const double sc = Nt / Nt_prev;
        for (int a = 0; a <= E.natom; ++a) N[a] *= sc;
      }
      if (newton(Nt, kWarmPasses, true) == 1) {
        finish(Nt, warm);
        return;
      }
    }
    cold_start(Nt);
    if (newton(Nt, 50, false) != 1) capped = 1;
    finish(Nt, warm);
  }

  __device__ void finish(double Nt, bool warm) {
    have = 1;
    Nt_prev = Nt;
    if (!warm) return;
    lu_ok = 1;
    lu_T = T;
    const int na = E.natom;
    if (nhist == 0 || T != T1) {
      for (int a = 0; a <= na; ++a) lx2[a] = lx1[a];
      T2 = T1;
      if (nhist < 2) ++nhist;
    }
    for (int a = 0; a <= na; ++a) lx1[a] = log(N[a] / Nt);
    T1 = T;
  }

  // The continued start's first iterate into N (true), or false: none applies, and the caller
  // scales the last solution by the particle-density ratio.  At the temperature of the last
  // Jacobian (the next hydrostatic iterate of the same depth) a first-order step along
  // dN/dNt = J^-1 e_1 (the defect of row 1 is sum N - Nt), solved with the kept factors; at a new
  // temperature (the next depth) log(N / Nt) extrapolated linearly in T from the last two
  // temperatures' solutions (the ratio clipped to [0, 2]; 1 when they share T).  An iterate with a
  // density below the Newton pass's floor (1e-2) or not finite is not used.
  // the full update from the reduced one: v_b = w for the reduced unknowns, the eliminated atoms
  // from u = w_1 + gr . w (rhs: their defects d_a, or null for zero)
  __device__ void expand(const double *w, const double *rhs, double *v) const {
    const int nr = E.nr;
    double u = w[1];
    for (int k = 0; k < nr; ++k) {
      v[E.rfull[k]] = w[k];
      u += gr[k] * w[k];
    }
    const double iabH = 1.0 / E.abund[0];
    for (int k = 0; k < E.nsimple; ++k) {
      const int sa = E.simple[k];
      v[sa] = (E.abund[sa - 1] * u - (rhs ? rhs[sa] : 0.0)) * iabH;
    }
  }

  __device__ bool predict(double Nt) {
    const int na = E.natom, nr = E.nr;
    double x[kEA + 1];
    if (lu_ok && T == lu_T) {
      // J x = e_1 (the defect of row 1 is sum N - Nt): reduced right-hand side (c0 e0 = 0, 1, 0, ...)
      double w[kEA + 1];
      for (int i = 0; i < nr; ++i) w[i] = 0.0;
      w[1] = 1.0;
      for (int c = 0; c < nr; ++c) {
        const int p = piv[c];
        if (p != c) { const double t = w[c]; w[c] = w[p]; w[p] = t; }
        for (int r = c + 1; r < nr; ++r) w[r] -= A[r * nr + c] * w[c];
      }
      for (int r = nr - 1; r >= 0; --r) {
        double sum = w[r];
        for (int j = r + 1; j < nr; ++j) sum -= A[r * nr + j] * w[j];
        w[r] = sum / A[r * nr + r];
      }
      expand(w, nullptr, x);
      const double dNt = Nt - Nt_prev;
      for (int a = 0; a <= na; ++a) x[a] = N[a] + x[a] * dNt;
    } else if (nhist == 2 && T != T1) {
      double r = T1 != T2 ? (T - T1) / (T1 - T2) : 1.0;
      r = fmin(fmax(r, 0.0), 2.0);
      for (int a = 0; a <= na; ++a) x[a] = Nt * exp(lx1[a] + (lx1[a] - lx2[a]) * r);
    } else {
      return false;
    }
    for (int a = 0; a <= na; ++a)
      if (!(x[a] >= 1E-2) || !isfinite(x[a])) return false;
    for (int a = 0; a <= na; ++a) N[a] = x[a];
    return true;
  }

  // the reference's starting values: ionisation-only quadratic and the halving loop
  __device__ void cold_start(double Nt) {
    const int na = E.natom;
    double F1 = 0.0, S1 = 0.0;
    sweep<false>(1.0);
    for (int a = 0; a < na; ++a) { F1 += E.abund[a] * Ea[a + 1]; S1 += E.abund[a]; }
    double F3 = 0.0, S3 = 0.0;
    sweep<false>(Nt);
    for (int a = 0; a < na; ++a) { F3 += E.abund[a] * Ea[a + 1]; S3 += E.abund[a]; }
    const double aa = F3 / (S3 * Nt);
    double bb = F1 / S1 - aa;
    const double cc = -bb * Nt;
    bb += 1.0 - aa * Nt;
    N[0] = fmax((-bb + sqrt(bb * bb - 4.0 * aa * cc)) / (2.0 * aa), 1.0);
    double esum;
    int pass = 0;
    do {
      esum = 0.0;
      sweep<false>(N[0]);
      for (int a = 1; a <= na; ++a) {
        N[a] = (Nt - N[0]) * E.abund[a - 1] / S3;
        esum += Ea[a] * N[a];
      }
      N[0] = 0.5 * (N[0] + esum);
      if (++pass >= kPolishCap) { capped = 1; break; }
    } while ((1E-2 * (N[0] + esum)) < fabs(N[0] - esum));
  }

  // Newton passes (atmos_chm.cc:176-305) from N, at most maxpass: 1 converged, 0 the pass cap was
  // reached (the reference stops there: iter > 100 counting two per pass), -1 a non-finite state
  // (only with bail: the continued start then falls back to the cold one; the cold path iterates
  // on as the reference does)
  __device__ int newton(double Nt, int maxpass, bool bail) {
    const int na = E.natom, nm = E.nmol;
    int iter = 0;
    bool conv;
    do {
      sweep<true>(N[0]);
      // defects (atmos_chm.cc:200-216) and Jacobian (:220-259); molecules enter as rank-one
      // updates: dm[m][b] = nm count_b / N[b], dm[m][0] = nm (count_e / N0 + sum df / f)
      // Rows 0 (charge) and 1 (particles) and the abundance rows a >= 2: d_a = abund_a Nr -
      // abund_H Nc_a with Nr = N_H + sum_m nmv_m mul_mH, Nc_a = N_a + sum_m nmv_m mul_ma, so row a
      // of the Jacobian is abund_a (e_1 + gr) - abund_H (e_a + sum_{m contains a} mul_ma grad nmv_m),
      // gr = sum_m mul_mH grad nmv_m (nonzero only at the electrons and the atoms in molecules).
      // The row of an atom in no molecule is abund_a (e_1 + gr) - abund_H e_a: its unknown is
      // v_a = (abund_a u - d_a) / abund_H with u = v_1 + gr . v, and rows 0 / 1 take it through
      // c0 = sum Ea_a abund_a / abund_H, c1 = sum abund_a / abund_H (and the defects through e0 /
      // e1).  What remains is the system of the electrons, hydrogen and the atoms in molecules
      // (nr unknowns), solved by Gaussian elimination with partial pivoting: the same solution as
      // the full system's, in about (nr / n)^3 of the work.
      const int nr = E.nr;
      const double abH = E.abund[0], iabH = 1.0 / abH;
      for (int k = 0; k < nr * nr; ++k) A[k] = 0.0;
      double d0 = -N[0], d1 = N[0] - Nt, a00 = -1.0, a10 = 1.0;
      for (int a = 1; a <= na; ++a) {
        d0 += N[a] * Ea[a];
        d1 += N[a];
        a00 += N[a] * Da[a];
        const int ra = E.rmap[a];
        if (ra >= 0) {
          A[ra] = Ea[a];    // row 0
          A[nr + ra] = 1.0; // row 1
        }
      }
      for (int k = 2; k < nr; ++k) A[k * nr + k] = -abH;
      for (int k = 0; k < nr; ++k) gr[k] = 0.0;
      double Nr = N[1];
      double Nc[kEA + 1], iN[kEA + 1];
      for (int a = 2; a <= na; ++a) Nc[a] = N[a];
      double dlf[R];  // dr / fr of the kept fractions the molecules use
      for (int k = 0; k < nr; ++k) iN[E.rfull[k]] = 1.0 / N[E.rfull[k]];
      for (int k = 0; k < E.nmref; ++k) dlf[E.mrefs[k]] = dr[E.mrefs[k]] / fr[E.mrefs[k]];
      double gr0 = 0.0;
      for (int m = 0; m < nm; ++m) {
        double nmv = iKkT[m], dm0 = 0.0;
        const int nc = E.mnc[m];
        for (int i = 0; i < nc; ++i) {
          const int a = E.matom[m][i];
          if (a == 0) {
            nmv *= N[0] * kT;
            dm0 += iN[0];
          } else {
            const int r = E.mref[m][i];
            nmv *= fr[r] * N[a] * kT;
            dm0 += dlf[r];
          }
        }
        dm0 *= nmv;
        const double q = E.mq[m], hm = (double)E.mmul[m][1];
        d0 += q * nmv;
        d1 += nmv;
        Nr += nmv * hm;
        a00 += q * dm0;
        a10 += dm0;
        gr0 += hm * dm0;
        for (int i = 0; i < nc; ++i) {
          const int b = E.matom[m][i];
          if (b == 0 || E.mdup[m][i]) continue;  // each distinct component atom once
          const int rb = E.rmap[b];
          const double mb = (double)E.mmul[m][b];
          const double dmb = nmv * mb * iN[b];
          A[rb] += q * dmb;
          A[nr + rb] += dmb;
          gr[rb] += hm * dmb;
          if (b >= 2) {
            Nc[b] += nmv * mb;
            A[rb * nr] -= abH * mb * dm0;
          }
          for (int j = 0; j < nc; ++j) {
            const int a = E.matom[m][j];
            if (a < 2 || E.mdup[m][j]) continue;
            A[E.rmap[a] * nr + rb] -= abH * (double)E.mmul[m][a] * dmb;
          }
        }
      }
      d[0] = d0;
      d[1] = d1;
      A[0] = a00;
      A[nr] = a10;
      gr[0] = gr0;
      for (int a = 2; a <= na; ++a) d[a] = E.abund[a - 1] * Nr - abH * Nc[a];
      for (int k = 2; k < nr; ++k) {
        const double ab = E.abund[E.rfull[k] - 1];
        for (int b = 0; b < nr; ++b) A[k * nr + b] += ab * gr[b];
        A[k * nr + 1] += ab;
      }
      double c0 = 0.0, c1 = 0.0, e0 = 0.0, e1 = 0.0;
      for (int k = 0; k < E.nsimple; ++k) {
        const int sa = E.simple[k];
        const double as = E.abund[sa - 1] * iabH;
        c0 += Ea[sa] * as;
        c1 += as;
        e0 += Ea[sa] * d[sa] * iabH;
        e1 += d[sa] * iabH;
      }
      for (int b = 0; b < nr; ++b) {
        A[b] += c0 * gr[b];
        A[nr + b] += c1 * gr[b];
      }
      A[1] += c0;
      A[nr + 1] += c1;
      // Gaussian elimination with partial pivoting on the reduced system; the factors stay in A
      // (multipliers where they were computed: rows are swapped from column c on) for the
      // continued start's predictor
      double w[kEA + 1], v[kEA + 1];
      w[0] = d[0] + e0;
      w[1] = d[1] + e1;
      for (int k = 2; k < nr; ++k) w[k] = d[E.rfull[k]];
      for (int c = 0; c < nr; ++c) {
        int p = c;
        double best = fabs(A[c * nr + c]);
        for (int r = c + 1; r < nr; ++r) {
          const double t = fabs(A[r * nr + c]);
          if (t > best) { best = t; p = r; }
        }
        piv[c] = p;
        if (p != c) {
          for (int j = c; j < nr; ++j) { const double t = A[c * nr + j]; A[c * nr + j] = A[p * nr + j]; A[p * nr + j] = t; }
          const double t = w[c]; w[c] = w[p]; w[p] = t;
        }
        const double ipv = 1.0 / A[c * nr + c];
        for (int r = c + 1; r < nr; ++r) {
          const double f = A[r * nr + c] * ipv;
          A[r * nr + c] = f;
          if (f == 0.0) continue;
          for (int j = c + 1; j < nr; ++j) A[r * nr + j] -= f * A[c * nr + j];
          w[r] -= f * w[c];
        }
      }
      for (int r = nr - 1; r >= 0; --r) {
        double sum = w[r];
        for (int j = r + 1; j < nr; ++j) sum -= A[r * nr + j] * w[j];
        w[r] = sum / A[r * nr + r];
      }
      expand(w, d, v);
      bool finite = true;
      for (int a = 0; a <= na; ++a) {
        N[a] -= v[a];
        if (N[a] < 1E-2) N[a] = 1E-2;
        finite &= isfinite(N[a]);
      }
      if (bail && !finite) return -1;
      iter += 2;  // the reference counts two per pass (atmos_chm.cc:294, 300)
      if (iter > 2 * maxpass) return 0;
      conv = true;
      for (int i = 0; i <= na; ++i) if (fabs(d[i] / N[i]) > 1E-4) conv = false;
    } while (!conv);
    return 1;
  }

  // stage total of stage s (with a kept fraction) after solve
  __device__ __forceinline__ double stage_total(int s, int a) const { return N[a + 1] * fr[E.ref[s]]; }

  // LTE population of level slot l (atom::lte, atom.cc:779-787), U = partition function at the final Ne
  __device__ double level_pop(int l, double U) const {
    const int s = E.lst[l];
    const double g = E.lg[l];
    return stage_total(s, E.satom[s]) * ((g != 0.0) ? g * exp(-E.lee[l] / (cK * T)) / U : 1.0);
  }
};
using Chem = ChemT<kER>;

// ---- node interpolation (atmospheric_interpolation, mathtools.cc:1208-1315) -------------------------------
__device__ double interpol_1d_falc(double xq) {
  const double f[11] = {1694.91525424, 2164.5021645, 2342.50815695, 2289.18827635, 2155.92183045,
                        2094.90240415, 2080.69183003, 2066.44925898, 1960.27182436, 1826.11342193, 1729.74468968};
  const double x[11] = {-0.01232, 0.08798, 0.2002, 0.32704, 0.46667, 0.61462, 0.7674,
                        0.92221, 1.07711, 1.22829, 1.37282};
  const int N = 11;
  if (xq < x[0]) return f[0];
  if (xq > x[10]) return f[10];
  if (!(xq < x[N - 1] && xq > x[0])) return xq >= x[N - 1] ? f[N - 1] : f[0];
  int i;
  for (i = 0; i <= N - 2; ++i)
    if (xq < x[i + 1]) break;
  double h1, h2, d1, d2, fd1, fd2;
  if (i > 0) {
    h1 = x[i] - x[i - 1];
    h2 = x[i + 1] - x[i];
    d1 = (f[i] - f[i - 1]) / h1;
    d2 = (f[i + 1] - f[i]) / h2;
    const double alpha = 1.0 / 3.0 * (1.0 + h2 / (h1 + h2));
    fd1 = (d1 * d2 > 0) ? d1 * d2 / (alpha * d2 + (1.0 - alpha) * d1) : 0.0;
  } else {
    fd1 = (f[1] - f[0]) / (x[1] - x[0]);
    h1 = h2 = x[1] - x[0];  // the reference reads an unset h2 here
  }
  const double C0 = f[i] + h2 * 0.5 * fd1;
  if (i + 1 < N - 1) {
    h1 = x[i + 1] - x[i];
    h2 = x[i + 2] - x[i + 1];
    d1 = (f[i + 1] - f[i]) / h1;
    d2 = (f[i + 2] - f[i + 1]) / h2;
    const double alpha = 1.0 / 3.0 * (1.0 + h2 / (h1 + h2));
    fd2 = (d1 * d2 > 0) ? d1 * d2 / (alpha * d2 + (1.0 - alpha) * d1) : 0.0;
  } else {
    fd2 = (f[N - 1] - f[N - 2]) / (x[N - 1] - x[N - 2]);
  }
  const double C1 = f[i + 1] - h1 * 0.5 * fd2;
  const double C = (C0 + C1) * 0.5;
  const double u = (xq - x[i]) / (x[i + 1] - x[i]);
  return (1.0 - u) * (1.0 - u) * f[i] + u * u * f[i + 1] + u * 2.0 * (1.0 - u) * C;
}

// Node values of one kind with an optional perturbation of node `pidx` (global index) by `pert`.
struct NodeView {
  const double *v;  // the pixel's node vector
  int pidx;
  double pert;
  __device__ double operator()(int g) const { return g == pidx ? v[g] + pert : v[g]; }
};

// value of kind `kind` at depth x; build: build_from_nodes' defaults, else interpolate_from_nodes'
__device__ double interp_kind(const EosDev &E, const NodeView &nv, int kind, int x, bool build) {
  const int N = E.kcount[kind], f0 = E.kfirst[kind];
  const bool is_temp = (kind == 1);
  const double lt = E.tau_min + (E.tau_max - E.tau_min) / (E.nd - 1) * x;
  double q;
  if (N > 1) {
    auto der = [&](int i) -> double {
      if (i == 0) return 0.0;
      if (i == N - 1) return is_temp ? interpol_1d_falc(E.ntau[f0 + N - 1]) : 0.0;
      const double h1 = E.ntau[f0 + i] - E.ntau[f0 + i - 1], h2 = E.ntau[f0 + i + 1] - E.ntau[f0 + i];
      const double d1 = (nv(f0 + i) - nv(f0 + i - 1)) / h1, d2 = (nv(f0 + i + 1) - nv(f0 + i)) / h2;
      if (d1 * d2 > 0) {
        const double alpha = 0.3333333 * (1.0 + h2 / (h1 + h2));
        return d1 * d2 / (alpha * d2 + (1.0 - alpha) * d1);
      }
      return 0.0;
    };
    if (lt < E.ntau[f0]) q = nv(f0) + der(0) * (lt - E.ntau[f0]);
    else if (lt > E.ntau[f0 + N - 1]) q = nv(f0 + N - 1) + der(N - 1) * (lt - E.ntau[f0 + N - 1]);
    else {
      int ii;
      for (ii = 0; ii < N - 1; ++ii)
        if (lt <= E.ntau[f0 + ii + 1]) break;
      const double ta = E.ntau[f0 + ii], tb = E.ntau[f0 + ii + 1];
      const double va = nv(f0 + ii), vb = nv(f0 + ii + 1);
      const double Ec = va + (tb - ta) / 3.0 * der(ii);
      const double Fc = vb - (tb - ta) / 3.0 * der(ii + 1);
      const double u = (lt - ta) / (tb - ta);
      q = (1.0 - u) * (1.0 - u) * (1.0 - u) * va + u * u * u * vb + 3.0 * u * (1.0 - u) * (1.0 - u) * Ec +
          3.0 * u * u * (1.0 - u) * Fc;
    }
    if (is_temp) q = fmin(fmax(q, 3400.0), 20000.0);
  } else if (N == 1) {
    q = nv(f0);
  } else {
    q = (kind == 4) ? (build ? 1E-3 : 0.0) : (kind >= 5 ? 1E-3 : 0.0);
  }
  if (build && kind == 5 && fabs(q) < 1E-3) q = 1E-3;
  return q;
}

__device__ __forceinline__ double logtau(const EosDev &E, int x) {
  return E.tau_min + (E.tau_max - E.tau_min) / (E.nd - 1) * x;
}

// atmosphere::opacity_continuum (atmos_rad.cc:286-294) from a solved Chem; which: 0 = lambda_he
// with sigma_he, 1 = lambda_kappa with sigma_kappa.  lev[]: populations of the level slots.
template <class CH>
__device__ double continuum(const EosDev &E, const CH &c, const double *lev, double nH0, int which) {
  const double T = c.T, Ne = c.N[0], lambda = which ? E.lambda_kappa : E.lambda_he;
  double op = 6.65E-25 * Ne;
  const double stim = exp(-cH * cC / lambda / cK / T);
  for (int b = 0; b < E.nbf; ++b) {
    if (!E.bflte[b]) continue;
    const double sigma = which ? E.sig_k[b] : E.sig_he[b];
    if (sigma == 0.0) continue;
    const double pop_mod = lev[E.bfn[b]] * Ne * cSAHA * pow(T, -1.5) * E.bfg[b] / E.bfgn[b] * exp(E.bfip[b] / cK / T);
    op += sigma * (lev[E.bfl[b]] - pop_mod * stim);
  }
  if (E.hm) {
    const double ca[7] = {1.99654, -1.18267E-5, 2.64243E-6, -4.40524E-10, 3.23992E-14, -1.39568E-18, 2.78701E-23};
    double alpha = 0.0;
    for (int i = 0; i < 7; ++i) alpha += ca[i] * pow(lambda * 1E8, (double)i);
    const double T_P = 5040. / T;
    const double op_bf =
        4.158E-28 * alpha * Ne * cK * T * pow(T_P, 2.5) * pow(10.0, 0.754 * T_P) * nH0 * (1.0 - stim);
    const double l = log10(lambda * 1E8);
    const double f_0 = -2.2763 - 1.6850 * l + 0.76661 * l * l - 0.053346 * l * l * l;
    const double f_1 = 15.2827 - 9.2846 * l + 1.99381 * l * l - 0.142631 * l * l * l;
    const double f_2 = -197.789 + 190.266 * l - 67.9775 * l * l + 10.6913 * l * l * l - 0.625151 * l * l * l * l;
    const double lt = log10(T_P);
    op += op_bf + 1E-26 * Ne * cK * T * pow(10.0, f_0 + f_1 * lt + f_2 * lt * lt) * nH0;
  }
  return op;
}

// chemistry + populations + kappa (which as in continuum); returns kappa, fills lev and nH0.  The
// T-only tables are rebuilt only when T changes (the hydrostatic iterations of one depth share T).
template <class CH>
__device__ double chem_point(const EosDev &E, CH &c, double T, double Nt, double *lev, double &nH0, int which,
                             bool warm = false) {
  const bool fast = which == 0 && E.mfast;
  if (T != c.T) {
    c.set_T(T);
    if (fast) c.set_march();
  }
  c.solve(Nt, warm);
  if (fast) {  // the march: the levels of the LTE bound-free edges at lambda_he only
    const double ne = c.N[0], pne = cbrt(sqrt(ne)), ine = 1.0 / ne, ipne = 1.0 / pne;
    double lm[kELm];
    for (int k = 0; k < E.nlev_m; ++k) {
      const int l = E.lev_m[k], st = E.lst[l];
      double U, dU;
      c.template stage_u<false>(st, ine, pne, ipne, U, dU);
      const double tot = c.stage_total(st, E.satom[st]);
      lm[k] = E.lg[l] != 0.0 ? tot * (c.mlf[k] / U) : tot;
    }
    nH0 = c.stage_total(E.s0[0], 0);
    double op = 6.65E-25 * ne;
    for (int k = 0; k < E.nbf_m; ++k)
      op += E.sig_he[E.bf_m[k]] * (lm[E.bfl_m[k]] - lm[E.bfn_m[k]] * ne * c.mcb[k] * c.mstim);
    return op + c.mhm * ne * nH0;
  }
  for (int l = 0; l < E.nlev; ++l) lev[l] = c.level_pop(l, c.stage_U(E.lst[l], c.N[0]));
  nH0 = c.stage_total(E.s0[0], 0);
  return continuum(E, c, lev, nH0, which);
}

// ---- k_eos_he: hydrostatic equilibrium per (pixel, variant) ---------------------------------------------
struct EosArgs {
  const EosDev *tab;
  int npix, nvar, nd, npar, nf;
  const double *nodes;    // [npix][npar]
  const int *active;      // [npix] or null
  const double *step;     // [npar]
  double *T, *Nt;         // [npix][nvar][nd]
  float *rec;             // [npix][nd][nf]
  float *tan;             // [npix][npar][nd][nf] or null
  double *Nt_out;         // [npix][nd] or null
  double *F;              // [npix][nvar][nd][nf]: thermal fields of every variant (FP64)
  int *status;            // [npix]
  int warm;               // continued chemistry starts in the hydrostatic march (Chem::solve)
  // k_eos_he: the depths [x0, x1) of the march; hs_in / hs_out (x0 > 0 / x1 < nd): the march's state
  // at the segment's start / end, [kHeStateWords][npix * nvar] each (two buffers: a variant starting
  // in this segment reads variant 0's start state while variant 0 writes its end state)
  int x0, x1;
  const double *hs_in;
  double *hs_out;
  // [npix][nvar]: each variant's first depth whose temperature differs from variant 0's (above it
  // the variant's march, records and fields are variant 0's, bit for bit); written by the march's
  // first launch
  int *xf;
  // k_eos_var: the depths [vx0, vx1)
  int vx0, vx1;
};
// the state a march carries between depth segments: the chemistry's and six march scalars
constexpr int kHeStateWords = Chem::kStateWords + 6;
// depth segments of the march with tangents: boundaries at these fractions of the depth count (the
// record chemistry grows with depth: the temperature-node variants differ from the node vector only
// below their nodes' first segment)
constexpr int kHeMaxSeg = 5;
constexpr double kHeSegFrac[kHeMaxSeg - 1] = {0.28, 0.5, 0.7, 0.85};

__device__ __forceinline__ void variant_pert(const EosDev &E, const EosArgs &A, int v, int &pidx, double &pert) {
  pidx = -1;
  pert = 0.0;
  if (v > 0) {
    pidx = E.kfirst[1] + (v - 1) / 2;
    pert = ((v - 1) % 2 == 0 ? 0.5 : -0.5) * A.step[pidx];
  }
}

// each temperature-node variant's first depth whose temperature differs from the node vector's
// (interpolation only, before the march), thread = (pixel, variant > 0)
__global__ void __launch_bounds__(kRecThreads) k_eos_xf(EosArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.npix * (A.nvar - 1)) return;
  const int p = i % A.npix, v = 1 + i / A.npix;
  if (A.active && !A.active[p]) return;
  const EosDev &E = *A.tab;
  NodeView nv{A.nodes + (size_t)p * A.npar, -1, 0.0};
  variant_pert(E, A, v, nv.pidx, nv.pert);
  const NodeView n0{A.nodes + (size_t)p * A.npar, -1, 0.0};
  int xf = 0;
  while (xf < A.nd && interp_kind(E, nv, 1, xf, true) == interp_kind(E, n0, 1, xf, true)) ++xf;
  A.xf[(size_t)p * A.nvar + v] = xf;
}

// kSeg: a depth segment of the march with tangents (variants start where they first differ, the state
// carried between launches); without: the whole march of every (pixel, variant) in one launch
template <bool kSeg>
__global__ void __launch_bounds__(128, 4) k_eos_he(EosArgs A) {  // launched with kHeCands threads; <= 128 registers
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nth = A.npix * A.nvar;
  if (i >= nth) return;
  const int p = i % A.npix, v = i / A.npix;
  if (A.active && !A.active[p]) return;
  const EosDev &E = *A.tab;
  NodeView nv{A.nodes + (size_t)p * A.npar, -1, 0.0};
  variant_pert(E, A, v, nv.pidx, nv.pert);
  double *Tc = A.T + ((size_t)p * A.nvar + v) * A.nd;
  double *Nc = A.Nt + ((size_t)p * A.nvar + v) * A.nd;
  // A temperature-node variant is variant 0 above the first depth whose temperature it moves: it
  // runs no segment that ends above that depth, and starts in its first segment from variant 0's
  // state at the segment's top (the same bits its own march would have reached there).
  int xf = 0;  // k_eos_xf
  if (kSeg && v > 0) {
    xf = A.xf[(size_t)p * A.nvar + v];
    if (xf >= A.x1) return;
  }
  const bool from_v0 = kSeg && v > 0 && A.x0 > 0 && xf >= A.x0;
  Chem c(E);
  double lev[kEL];
  double nH0;
  int st = 0;
  const bool warm = A.warm != 0;
  double Ntop, op_prev, rho_prev, Tprev, Nprev;
  if (!kSeg || A.x0 == 0) {
    // top: fixed point from 0.3 / k T (atmos_pp.cc:184-202)
    double T0 = interp_kind(E, nv, 1, 0, true);
    Tc[0] = T0;
    double Nt = 0.3 / cK / T0;
    op_prev = rho_prev = 0.0;
    for (int iter = 0; iter < 20; ++iter) {
      const double op = chem_point(E, c, T0, Nt, lev, nH0, 0, warm);
      st |= c.capped;
      const double rho = c.N[1] * 1.4 * 1.67E-24;
      const double dN = (pow(10.0, logtau(E, 0)) * rho * E.grav / op) / cK / T0 - Nt;
      Nt += dN;
      op_prev = op;
      rho_prev = rho;
      if (fabs(dN / Nt) < 1E-2) break;
      if (iter == 19) st |= 2;
    }
    Nc[0] = Nt;
    Ntop = Nt;
    Tprev = T0;
    Nprev = Nt;
  } else {  // the state the previous segment left (variant 0's for a variant starting here)
    const double *hs = A.hs_in + (from_v0 ? p : i);
    c.load_state(hs, (size_t)nth);
    const double *m = hs + (size_t)Chem::kStateWords * nth;
    Ntop = m[0];
    op_prev = m[(size_t)nth];
    rho_prev = m[2 * (size_t)nth];
    Tprev = m[3 * (size_t)nth];
    Nprev = m[4 * (size_t)nth];
  }
  const int xb = kSeg ? A.x0 : 0, xe = kSeg ? A.x1 : A.nd;
  for (int x = xb > 1 ? xb : 1; x < xe; ++x) {
    const double Tx = interp_kind(E, nv, 1, x, true);
    Tc[x] = Tx;
    const double delta_tau = pow(10.0, logtau(E, x)) - pow(10.0, logtau(E, x - 1));
    double delta_p = rho_prev * E.grav / op_prev * delta_tau;
    double N = (Nprev * cK * Tprev + delta_p) / cK / Tx;
    double op = 0.0, rho = 0.0;
    for (int iter = 0; iter < 20; ++iter) {
      op = chem_point(E, c, Tx, N, lev, nH0, 0, warm);
      st |= c.capped;
      rho = c.N[1] * 1.4 * 1.67E-24;
      const double kappa_mean = sqrt(op * op_prev / rho / rho_prev);
      delta_p = E.grav / kappa_mean * delta_tau;
      const double dN = (Nprev * cK * Tprev + delta_p) / cK / Tx - N;
      N += dN;
      if (fabs(dN / Ntop) < 1E-2) break;  // relative to the TOP density, as atmos_pp.cc:235
      if (iter == 19) st |= 2;
    }
    Nc[x] = N;
    op_prev = op;
    rho_prev = rho;
    Tprev = Tx;
    Nprev = N;
  }
  if (kSeg && A.x1 < A.nd) {
    double *hs = A.hs_out + i;
    c.save_state(hs, (size_t)nth);
    double *m = hs + (size_t)Chem::kStateWords * nth;
    m[0] = Ntop;
    m[(size_t)nth] = op_prev;
    m[2 * (size_t)nth] = rho_prev;
    m[3 * (size_t)nth] = Tprev;
    m[4 * (size_t)nth] = Nprev;
  }
  if (st) atomicOr(A.status + p, st);
}

// ---- k_eos_rec: records and tangents per (depth, pixel) ------------------------------------------------
// thermal fields of a record (those that move with (T, Nt)); the others are kinematic / field
__device__ void thermal_fields(const EosDev &E, Chem &c, double T, double Nt, double *f, int &st) {
  double lev[kEL], nH0;
  const double kap = chem_point(E, c, T, Nt, lev, nH0, 1);
  st |= c.capped;
  const double Ne = c.N[0], tp = 5040.0 / T;
  f[0] = T;
  f[2] = Ne;
  f[7] = kap;
  f[8] = E.hm ? 4.158E-28 * Ne * cK * T * pow(tp, 2.5) * pow(10.0, 0.754 * tp) * nH0 : 0.0;
  f[9] = E.hm ? 1E-26 * Ne * cK * T * nH0 : 0.0;
  double bop = 0.0, bem = 0.0;
  for (int b = 0; b < E.nbf; ++b) {
    const double lw = E.lam_w[b];
    if (!(lw > 0.0)) continue;
    const double pop_mod = lev[E.bfn[b]] * Ne * cSAHA * pow(T, -1.5) * E.bfg[b] / E.bfgn[b] * exp(E.bfip[b] / cK / T);
    const double stim = exp(-cH * cC / lw / cK / T);
    bop += E.sig_w[b] * (lev[E.bfl[b]] - pop_mod * stim);
    const double planck = 2.0 * 6.62606957 * 8.9875517E-7 / lw / lw / lw / lw / lw / (exp(1.4387769 / lw / T) - 1.0);
    bem += E.sig_w[b] * pop_mod * (1.0 - stim) * planck;
  }
  f[10] = bop;
  f[11] = bem;
  for (int j = 0; j < E.nlines; ++j) {
    const double nl = lev[E.llo[j]], nu = lev[E.lup[j]];
    f[SNAPI_NFIELD0 + 3 * j + 0] = (nl * E.lBlu[j] - nu * E.lBul[j]) * cH * cC / E.llam0[j] / 4.0 / cPI;
    f[SNAPI_NFIELD0 + 3 * j + 1] = nu * E.lA[j] * cH * cC / E.llam0[j] / 4.0 / cPI;
    const double red_mass = 1.66E-24 / (1.0 / 1.008 + 1.66E-24 / E.lmass[j]);
    const double vmean = sqrt(8.0 * cK * T / cPI / red_mass);
    f[SNAPI_NFIELD0 + 3 * j + 2] = nH0 * vmean * pow(vmean / 1E6, -E.lalpha[j]) * E.lsig[j];
  }
}

// kinematic / field fields 1, 3, 4, 5, 6 of given v_turb, v_z, |B|, inclination, azimuth (project and
// transform, atmos_rad.cc:14-48; V_x = V_y = 0)
__device__ void project_fields(const EosDev &E, double vt, double vz, double B, double th, double ph, double *f) {
  const double sp = sin(E.phi), cp = cos(E.phi), ct = cos(cPI - E.theta), st = sin(cPI - E.theta);
  f[1] = vt;
  f[3] = sp * st * 0.0 + cp * st * 0.0 + ct * vz;
  const double Bx = B * sin(th) * cos(ph), By = B * sin(th) * sin(ph), Bz = B * cos(th);
  const double mg = sqrt(Bx * Bx + By * By + Bz * Bz);
  const double nBx = ct * cp * Bx + sp * By - st * cp * Bz;
  const double nBy = -ct * sp * Bx + cp * By + st * sp * Bz;
  const double nBz = st * Bx + ct * Bz;
  f[4] = mg;
  f[5] = acos(nBz / mg) * 180.0 / cPI;
  f[6] = atan(nBy / nBx) * 180.0 / cPI;
}

// the same fields of the node model at depth x
__device__ void field_fields(const EosDev &E, const NodeView &nv, int x, bool build, double *f) {
  project_fields(E, interp_kind(E, nv, 2, x, build), interp_kind(E, nv, 3, x, build), interp_kind(E, nv, 4, x, build),
                 interp_kind(E, nv, 5, x, build), interp_kind(E, nv, 6, x, build), f);
}

// thermal fields of every (pixel, variant, depth), one thread each (pixel fastest: a warp holds 32
// pixels of one variant at one depth), FP64 into F [npix][nvar][nd][nf]
__global__ void __launch_bounds__(256) k_eos_var(EosArgs A) {  // launched with kVarCands threads
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)A.npix * A.nvar * (A.vx1 - A.vx0)) return;
  const int p = (int)(i % A.npix);
  const long long r = i / A.npix;
  const int v = (int)(r % A.nvar), x = A.vx0 + (int)(r / A.nvar);
  if (A.active && !A.active[p]) return;
  const size_t cv = ((size_t)p * A.nvar + v) * A.nd + x;
  // A temperature-node variant leaves T, and so the march, bit-identical to variant 0 above the
  // first depth whose interpolation segment uses that node: its fields there are variant 0's
  // (k_eos_rec reads those), and the tangent's difference is exactly 0, as the reference's is.
  if (v > 0 && x < A.xf[(size_t)p * A.nvar + v]) return;
  const EosDev &E = *A.tab;
  Chem c(E);
  int st = 0;
  double f[SNAPI_NFIELD0 + 3 * SNAPI_MAX_LINES];
  // the reference's start, whatever the march used: the record fields take the stage fractions of
  // the last Newton sweep before its final update, so they follow the solve's path to ~1e-4
  thermal_fields(E, c, A.T[cv], A.Nt[cv], f, st);
  double *o = A.F + cv * A.nf;
  for (int k = 0; k < A.nf; ++k) o[k] = (k == 1 || (k >= 3 && k <= 6)) ? 0.0 : f[k];
  if (st) atomicOr(A.status + p, st);
}

// records and tangent rows per (depth, pixel): thermal fields from F, kinematic / field fields by
// (re-)interpolation
__global__ void __launch_bounds__(kRecThreads) k_eos_rec(EosArgs A) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.npix * A.nd) return;
  const int p = i % A.npix, x = i / A.npix;
  if (A.active && !A.active[p]) return;
  const EosDev &E = *A.tab;
  const int nf = A.nf;
  const double *nodes = A.nodes + (size_t)p * A.npar;
  int st = 0;
  double r0[SNAPI_NFIELD0 + 3 * SNAPI_MAX_LINES];
  const double *F0 = A.F + ((size_t)p * A.nvar * A.nd + x) * nf;  // variant 0
  for (int f = 0; f < nf; ++f) r0[f] = F0[f];
  NodeView nv0{nodes, -1, 0.0};
  field_fields(E, nv0, x, true, r0);
  float *rp = A.rec + ((size_t)p * A.nd + x) * nf;
  bool finite = true;
  for (int f = 0; f < nf; ++f) {
    rp[f] = (float)r0[f];
    finite &= isfinite(r0[f]);
  }
  if (A.Nt_out) A.Nt_out[(size_t)p * A.nd + x] = A.Nt[(size_t)p * A.nvar * A.nd + x];
  if (A.tan) {
    double fp[SNAPI_NFIELD0 + 3 * SNAPI_MAX_LINES], fm[SNAPI_NFIELD0 + 3 * SNAPI_MAX_LINES];
    for (int q = 0; q < A.npar; ++q) {
      float *tq = A.tan + (((size_t)p * A.npar + q) * A.nd + x) * nf;
      const double stp = A.step[q];
      if (q >= E.kfirst[1] && q < E.kfirst[1] + E.kcount[1]) {
        const int v = 1 + 2 * (q - E.kfirst[1]);
        // a variant identical to variant 0 at this depth has variant 0's fields (k_eos_var skips it)
        auto fields = [&](int w) {
          const size_t cw = ((size_t)p * A.nvar + w) * A.nd + x, cb = (size_t)p * A.nvar * A.nd + x;
          return A.F + (x < A.xf[(size_t)p * A.nvar + w] ? cb : cw) * nf;
        };
        const double *Fp = fields(v);
        const double *Fm = fields(v + 1);
        for (int f = 0; f < nf; ++f) {
          const bool th = !(f == 1 || (f >= 3 && f <= 6));
          tq[f] = th ? (float)((Fp[f] - Fm[f]) / stp) : 0.f;
        }
      } else {
        NodeView np{nodes, q, 0.5 * stp}, nm{nodes, q, -0.5 * stp};
        field_fields(E, np, x, false, fp);
        field_fields(E, nm, x, false, fm);
        // a kinematic / field node moves only its own fields (v_turb 1, v_los 3, the field 4-6);
        // the reference's differences of the others are 0, or NaN - NaN where B = 0 without B nodes
        const int kind = E.nkind[q];
        for (int f = 0; f < nf; ++f) {
          const bool own = kind == 2 ? f == 1 : (kind == 3 ? f == 3 : (f >= 4 && f <= 6));
          tq[f] = own ? (float)((fp[f] - fm[f]) / stp) : 0.f;
        }
      }
    }
  }
  if (!finite) st |= 4;
  if (st) atomicOr(A.status + p, st);
}

// atmosphere::return_as_array (atmos.cc:547-569) of the variant-0 columns, as the master collects
// them after stokes_lm_fit's final build_from_nodes and compute_op_referent: one thread per
// (depth, pixel); atm [npix][12][nd]
__global__ void __launch_bounds__(kRecThreads) k_eos_atm(EosArgs A, const double *x3, double *atm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.npix * A.nd) return;
  const int p = i % A.npix, x = i / A.npix;
  if (A.active && !A.active[p]) return;
  const EosDev &E = *A.tab;
  const double *F0 = A.F + ((size_t)p * A.nvar * A.nd + x) * A.nf;  // variant 0
  const double T = F0[0], Ne = F0[2], kap = F0[7], Nt = A.Nt[(size_t)p * A.nvar * A.nd + x];
  NodeView nv{A.nodes + (size_t)p * A.npar, -1, 0.0};
  // build_from_nodes' magnetic vector (atmos_pp.cc:169-173); the azimuth row divides by the top
  // depth's Bx (atmos.cc:566)
  auto bvec = [&](int xx, double &bx, double &by, double &bz) {
    const double B = interp_kind(E, nv, 4, xx, true), th = interp_kind(E, nv, 5, xx, true);
    const double ph = interp_kind(E, nv, 6, xx, true);
    bx = B * sin(th) * cos(ph);
    by = B * sin(th) * sin(ph);
    bz = B * cos(th);
  };
  double bx, by, bz, bx0, by0, bz0;
  bvec(x, bx, by, bz);
  bvec(0, bx0, by0, bz0);
  const double mg = sqrt(bx * bx + by * by + bz * bz);
  const double tau = -pow(10.0, logtau(E, x));  // tau_referent as build_from_nodes stores it
  double r[12];
  r[0] = log10(-tau);
  r[1] = x3 ? x3[x] : 0.0;
  r[2] = T;
  r[3] = Nt * cK * T;
  r[4] = Ne * cK * T;
  r[5] = 0.0;
  r[6] = kap;
  r[7] = mg;
  r[8] = interp_kind(E, nv, 2, x, true);
  r[9] = interp_kind(E, nv, 3, x, true);
  r[10] = acos(bz / mg);
  r[11] = atan(by / bx0);
  double *o = atm + (size_t)p * 12 * A.nd + x;
  for (int k = 0; k < 12; ++k) o[(size_t)k * A.nd] = r[k];
}

// Records of given columns in the 12-row layout of k_eos_atm, as atmosphere::read_spinor3d reads a
// cube (atmos_fio.cc:100-121: T floored at 3200 K, Nt from the gas pressure, the field from |B|,
// inclination and azimuth, V_z, V_t) and obs_stokes' set-up completes it (the chemistry, n_e and the
// opacity at airtovac(lambda_referent)).  One thread per (depth, pixel); status bit 8: the column's
// log tau row is not the context's grid (beyond 1e-6).
__global__ void __launch_bounds__(kRecThreads) k_eos_col(const EosDev *tab, int npix, int nd, int nf,
                                                        const double *cols, float *rec, int *status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix * nd) return;
  const int p = i % npix, x = i / npix;
  const EosDev &E = *tab;
  const double *c = cols + (size_t)p * 12 * nd + x;
  auto row = [&](int k) { return c[(size_t)k * nd]; };
  const double T = row(2) > 3200.0 ? row(2) : 3200.0;
  const double Nt = row(3) / (cK * T);
  Chem ch(E);
  int st = 0;
  double f[SNAPI_NFIELD0 + 3 * SNAPI_MAX_LINES];
  thermal_fields(E, ch, T, Nt, f, st);
  project_fields(E, row(8), row(9), row(7), row(10), row(11), f);
  // the grid to float32 rounding (a float32 cube holds log tau to ~2.4e-7); the synthesis runs on
  // the context's grid
  if (!(fabs(row(0) - logtau(E, x)) <= 1e-6)) st |= 8;
  float *r = rec + ((size_t)p * nd + x) * nf;
  bool finite = true;
  for (int k = 0; k < nf; ++k) {
    r[k] = (float)f[k];
    finite &= isfinite(f[k]);
  }
  if (!finite) st |= 4;
  if (st) atomicOr(status + p, st);
}

// ---- host side ---------------------------------------------------------------------------------------------
// The autotuner's pick among three CTA sizes for one launch: each is run once and timed by CUDA
// events on the context's stream; the default when no timing succeeds.
template <class F>
int tune_launch(snapi_ctx *ctx, const int (&cands)[3], F launch, int fallback) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return fallback;
  if (cudaEventCreate(&e1) != cudaSuccess) { cudaEventDestroy(e0); return fallback; }
  int best = fallback;
  float best_ms = -1.f;
  for (int t : cands) {
    cudaEventRecord(e0, ctx->stream);
    launch(t);
    cudaEventRecord(e1, ctx->stream);
    float ms = -1.f;
    if (cudaGetLastError() == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess)
      cudaEventElapsedTime(&ms, e0, e1);
    if (ms > 0.f && (best_ms < 0.f || ms < best_ms)) { best_ms = ms; best = t; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}
struct EosCtx {
  EosDev *d_tab = nullptr;
  int npar = 0, ntherm = 0;
  std::vector<int> kind;
  std::vector<double> ref_step;
  // work buffers for cap pixels
  int cap = 0, cap_var = 0;
  double *d_T = nullptr, *d_Nt = nullptr, *d_nodes = nullptr, *d_step = nullptr, *d_Ntout = nullptr;
  double *d_F = nullptr;
  int *d_active = nullptr, *d_status = nullptr;
  int chem_start = SNAPI_CHEM_START_CONTINUE;
  int segmented = 1;  // with tangents: the march in depth segments, each followed by its record chemistry
  // snapi_adjoint_nodes with host arrays: a chunk's node vectors and build status (max_batch pixels)
  double *d_nn = nullptr;
  int *d_nst = nullptr;
  float *d_rec = nullptr, *d_tan = nullptr;
  // return_as_array rows of snapi_build_atmos (cap_atm pixels) and the caller's heights
  double *d_atm = nullptr, *d_x3 = nullptr;
  int cap_atm = 0;
  // snapi_records_from_columns: staged columns, records and status (cap_col pixels)
  double *d_cols = nullptr;
  float *d_crec = nullptr;
  int *d_cst = nullptr;
  int cap_col = 0;
  // the NLTE set-up (snapi_ali_setup): the host copy of the tables and the model's atoms it derives
  // its own tables from, its device tables and work buffers (cap_su columns: bgf, staged inputs /
  // outputs for host arrays)
  std::vector<EosDev> h_tab;
  std::vector<snapi_eos_atom> atoms;
  void *d_su = nullptr;
  size_t cap_su = 0;
  // the march in depth segments: its state between segments (two buffers of cap_hs words), each
  // variant's first moved depth (cap_xf entries)
  double *d_hs = nullptr;
  size_t cap_hs = 0;
  int *d_xf = nullptr;
  size_t cap_xf = 0;
};

void eos_free_bufs(EosCtx *e) {
  void *b[] = {e->d_T, e->d_Nt, e->d_nodes, e->d_step, e->d_Ntout, e->d_active, e->d_status, e->d_rec, e->d_tan,
               e->d_F};
  for (void *p : b) cudaFree(p);
  e->d_T = e->d_Nt = e->d_nodes = e->d_step = e->d_Ntout = e->d_F = nullptr;
  e->d_active = e->d_status = nullptr;
  e->d_rec = e->d_tan = nullptr;
  e->cap = e->cap_var = 0;
  cudaFree(e->d_atm);
  cudaFree(e->d_x3);
  e->d_atm = e->d_x3 = nullptr;
  e->cap_atm = 0;
  cudaFree(e->d_cols);
  cudaFree(e->d_crec);
  cudaFree(e->d_cst);
  e->d_cols = nullptr;
  e->d_crec = nullptr;
  e->d_cst = nullptr;
  e->cap_col = 0;
  cudaFree(e->d_su);
  e->d_su = nullptr;
  e->cap_su = 0;
  cudaFree(e->d_hs);
  e->d_hs = nullptr;
  e->cap_hs = 0;
  cudaFree(e->d_xf);
  e->d_xf = nullptr;
  e->cap_xf = 0;
}

}  // namespace

bool eos_matches(const snapi_ctx *ctx, int npar, const int *node_kind) {
  const EosCtx *e = static_cast<const EosCtx *>(ctx->eos);
  if (!e || !node_kind || npar != e->npar) return false;
  for (int q = 0; q < npar; ++q)
    if (node_kind[q] != e->kind[q]) return false;
  return true;
}

void eos_free(snapi_ctx *ctx) {
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (!e) return;
  eos_free_bufs(e);
  cudaFree(e->d_nn);
  cudaFree(e->d_nst);
  cudaFree(e->d_tab);
  delete e;
  ctx->eos = nullptr;
}

}  // namespace snapi

using snapi::set_err;

extern "C" {

int snapi_eos_set(snapi_ctx *ctx, const snapi_eos_model *m) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  if (!m || m->natom < 1 || m->natom > SNAPI_EOS_MAX_ATOMS || !m->atoms || m->nmol < 0 ||
      m->nmol > SNAPI_EOS_MAX_MOLS || (m->nmol && !m->mols) || (ctx->nlines && !m->lines) || m->npar < 1 ||
      m->npar > SNAPI_EOS_MAX_PAR || !m->node_kind || !m->node_tau)
    return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: invalid model");
  if (!(m->lambda_he > 0.0) || !(m->lambda_kappa > 0.0) || !(m->grav > 0.0) || !(m->tau_max > m->tau_min))
    return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: invalid constants");
  // the context's depth grid must be the model's
  for (int x = 0; x < ctx->nd; ++x) {
    const double t = pow(10.0, m->tau_min + (m->tau_max - m->tau_min) / (ctx->nd - 1) * x);
    if (fabs(t - ctx->h_tau500[x]) > 1e-12 * t)
      return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: the problem's tau500 is not the model's log tau grid");
  }
  std::vector<EosDev> hv(1);
  EosDev &H = hv[0];
  memset(&H, 0, sizeof(EosDev));
  H.natom = m->natom;
  H.nmol = m->nmol;
  H.nlines = ctx->nlines;
  H.npar = m->npar;
  H.nd = ctx->nd;
  H.lambda_he = m->lambda_he;
  H.lambda_kappa = m->lambda_kappa;
  H.grav = m->grav;
  H.tau_min = m->tau_min;
  H.tau_max = m->tau_max;
  H.theta = m->theta;
  H.phi = m->phi;
  {
    const double er = cE * cRYD * cRYD;
    H.ftrav = 1.405169521381833474E+05 * ((4.0 * cPI * cE0) / (er * er));
  }
  int ns = 0, nt = 0, nc = 0;
  for (int a = 0; a < m->natom; ++a) {
    const snapi_eos_atom &At = m->atoms[a];
    if (At.nstage < 1 || At.nstage > SNAPI_EOS_MAX_STAGES || ns + At.nstage > kES)
      return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: atom %d: too many ionisation stages", a);
    H.abund[a] = At.abundance;
    H.s0[a] = ns;
    for (int z = 0; z < At.nstage; ++z) H.satom[ns + z] = a;
    H.ns[a] = At.nstage;
    for (int z = 0; z < At.nstage; ++z, ++ns) {
      const snapi_partition &P = At.pf[z];
      H.pft[ns] = P.type;
      H.pfv[ns] = P.type == SNAPI_PF_CONST ? P.value : (P.type == SNAPI_PF_TRAV ? P.g0 : 1.0);
      H.zeff[ns] = P.zeff;
      H.zf[ns] = P.zeff * H.ftrav;
      H.izf[ns] = P.zeff != 0.0 ? 1.0 / H.zf[ns] : 0.0;
      H.eion[ns] = z + 1 < At.nstage ? At.ip[z] : 0.0;
      if (z + 1 < At.nstage && !std::isfinite(At.ip[z]))
        return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: atom %d stage %d: no ionisation energy", a, z);
      H.ref[ns] = -1;
      if (P.type == SNAPI_PF_TRAV) {
        if (P.nterm < 0 || P.nterm > SNAPI_PF_MAX_TERMS || nt + P.nterm > kET)
          return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many partition-function terms");
        H.t0[ns] = nt;
        for (int t = 0; t < P.nterm; ++t, ++nt) {
          if (!(P.ll[t] > 0.0))
            return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: atom %d stage %d: Traving term with l <= 0", a, z);
          H.g2[nt] = P.g2[t];
          H.tee[nt] = P.ee[t];
          H.tll[nt] = P.ll[t];
          H.til[nt] = 1.0 / P.ll[t];
          {
            const double llm = P.ll[t] - 1.0;
            H.tA[nt] = ((0.33333333 * llm - 0.5) * llm - 0.16666667) * llm;
          }
          if (P.m[t] < 0 || P.m[t] > SNAPI_PF_MAX_COEF || nc + P.m[t] > kEC)
            return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many partition-function coefficients");
          H.c0[nt] = nc;
          for (int k = 0; k < P.m[t]; ++k, ++nc) { H.cA[nc] = P.a[t][k]; H.cG[nc] = P.gam[t][k]; }
          H.c1[nt] = nc;
        }
        H.t1[ns] = nt;
      } else if (P.type == SNAPI_PF_IRWIN) {
        if (P.ncoef < 0 || P.ncoef > SNAPI_PF_MAX_COEF || nc + P.ncoef > kEC)
          return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many Irwin coefficients");
        H.t0[ns] = nc;
        for (int k = 0; k < P.ncoef; ++k, ++nc) H.cA[nc] = P.coef[k];
        H.t1[ns] = nc;
      } else if (P.type != SNAPI_PF_CONST && P.type != SNAPI_PF_NONE) {
        return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: unknown partition function type %d", P.type);
      }
    }
  }
  H.nst = ns;
  // kept fractions: molecule components, then the stages of record levels
  int nref = 0;
  auto keep = [&](int s) -> int {
    if (H.ref[s] < 0) {
      if (nref >= kER) return -1;
      H.ref[s] = nref++;
    }
    return H.ref[s];
  };
  for (int mm = 0; mm < m->nmol; ++mm) {
    const snapi_eos_molecule &M = m->mols[mm];
    if (M.ncomp < 1 || M.ncomp > SNAPI_MOL_MAX_COMP)
      return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: molecule %d: bad component count", mm);
    if (M.eqc != SNAPI_EQC_POLY && M.eqc != SNAPI_EQC_HMIN && M.eqc != SNAPI_EQC_CONST)
      return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: molecule %d: unknown equilibrium constant", mm);
    if (M.eqc == SNAPI_EQC_POLY && (M.ncoef < 1 || M.ncoef > SNAPI_PF_MAX_COEF))
      return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: molecule %d: bad coefficients", mm);
    H.mnc[mm] = M.ncomp;
    H.meqc[mm] = M.eqc;
    H.mncoef[mm] = M.ncoef;
    for (int k = 0; k < SNAPI_PF_MAX_COEF; ++k) H.mcoef[mm][k] = M.coef[k];
    if (M.eqc == SNAPI_EQC_HMIN) H.hm = 1;
    double q = 0.0;
    for (int i = 0; i < M.ncomp; ++i) {
      const int a = M.comp_atom[i];
      if (a < -1 || a >= m->natom) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: molecule %d: bad atom", mm);
      const int idx = a + 1;
      H.matom[mm][i] = idx;
      H.mmul[mm][idx] += 1;
      H.mdup[mm][i] = 0;
      for (int j = 0; j < i; ++j)
        if (H.matom[mm][j] == idx) H.mdup[mm][i] = 1;
      q += (double)M.comp_charge[i];
      if (a >= 0) {
        const int z = M.comp_charge[i] > 0 ? M.comp_charge[i] : 0;
        if (z >= m->atoms[a].nstage)
          return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: molecule %d: bad component charge", mm);
        const int r = keep(H.s0[a] + z);
        if (r < 0) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many kept ionisation fractions");
        H.mref[mm][i] = r;
      } else {
        H.mref[mm][i] = -1;
      }
    }
    H.mq[mm] = q;
  }
  // level slots: hydrogen's neutral stage is always kept (H-, damping, rho uses the free total)
  if (keep(H.s0[0]) < 0) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many kept ionisation fractions");
  int nlev = 0;
  std::vector<int> slot(m->natom * SNAPI_EOS_MAX_STAGES * SNAPI_EOS_MAX_LEVELS, -1);
  auto level_slot = [&](int a, int z, int l) -> int {
    int &sl = slot[(a * SNAPI_EOS_MAX_STAGES + z) * SNAPI_EOS_MAX_LEVELS + l];
    if (sl < 0) {
      if (nlev >= kEL) return -1;
      const int s = H.s0[a] + z;
      if (keep(s) < 0) return -1;
      H.lst[nlev] = s;
      H.lg[nlev] = m->atoms[a].level[z][l].g;
      H.lee[nlev] = m->atoms[a].level[z][l].ee;
      sl = nlev++;
    }
    return sl;
  };
  int nbf = 0;
  for (int a = 0; a < m->natom; ++a) {
    const snapi_eos_atom &At = m->atoms[a];
    for (int z = 0; z + 1 < At.nstage; ++z) {
      if (At.nlevel[z] < 0 || At.nlevel[z] > SNAPI_EOS_MAX_LEVELS)
        return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: atom %d stage %d: bad level count", a, z);
      for (int l = 0; l < At.nlevel[z]; ++l) {
        const snapi_eos_level &L = At.level[z][l];
        if (L.sigma_he == 0.0 && L.sigma_kappa == 0.0 && !(L.lambda_win > 0.0)) continue;
        if (At.nlevel[z + 1] < 1)
          return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: atom %d: bound-free level without a next stage", a);
        if (nbf >= kEB) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many bound-free levels");
        const int sl = level_slot(a, z, l), sn = level_slot(a, z + 1, 0);
        if (sl < 0 || sn < 0) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many levels");
        H.bfl[nbf] = sl;
        H.bfn[nbf] = sn;
        H.bflte[nbf] = At.nlte ? 0 : 1;
        H.bfg[nbf] = L.g;
        H.bfgn[nbf] = At.level[z + 1][0].g;
        H.bfip[nbf] = At.ip[z] - L.ee;
        H.sig_he[nbf] = L.sigma_he;
        H.sig_k[nbf] = L.sigma_kappa;
        H.sig_w[nbf] = L.sigma_win;
        H.lam_w[nbf] = L.lambda_win;
        ++nbf;
      }
    }
  }
  H.nbf = nbf;
  {  // the march's compact opacity lists
    H.mfast = 1;
    H.nbf_m = H.nlev_m = 0;
    auto mslot = [&](int l) -> int {
      for (int k = 0; k < H.nlev_m; ++k)
        if (H.lev_m[k] == l) return k;
      if (H.nlev_m >= kELm) return -1;
      H.lev_m[H.nlev_m] = l;
      return H.nlev_m++;
    };
    for (int b = 0; b < nbf && H.mfast; ++b) {
      if (!H.bflte[b] || H.sig_he[b] == 0.0) continue;
      const int kl = mslot(H.bfl[b]), kn = mslot(H.bfn[b]);
      if (kl < 0 || kn < 0 || H.nbf_m >= kEBm) {
        H.mfast = 0;
        break;
      }
      H.bf_m[H.nbf_m] = b;
      H.bfl_m[H.nbf_m] = kl;
      H.bfn_m[H.nbf_m] = kn;
      ++H.nbf_m;
    }
  }
  for (int j = 0; j < ctx->nlines; ++j) {
    const snapi_eos_line &L = m->lines[j];
    if (L.atom < 0 || L.atom >= m->natom || L.stage < 0 || L.stage >= m->atoms[L.atom].nstage || L.lower < 0 ||
        L.upper < 0 || L.lower >= m->atoms[L.atom].nlevel[L.stage] || L.upper >= m->atoms[L.atom].nlevel[L.stage])
      return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: line %d: bad level reference", j);
    const int lo = level_slot(L.atom, L.stage, L.lower), up = level_slot(L.atom, L.stage, L.upper);
    if (lo < 0 || up < 0) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: too many levels");
    H.llo[j] = lo;
    H.lup[j] = up;
    H.lBlu[j] = L.Blu;
    H.lBul[j] = L.Bul;
    H.lA[j] = L.A;
    H.lalpha[j] = L.alpha_col;
    H.lsig[j] = L.sigma_col;
    H.llam0[j] = ctx->h_line_lam0[j];
    H.lmass[j] = ctx->h_line_mass[j];
  }
  H.nlev = nlev;
  H.nref = nref;
  H.href = H.ref[H.s0[0]];
  {
    bool inmol[kEA + 1] = {};
    inmol[0] = inmol[1] = true;
    for (int mm = 0; mm < m->nmol; ++mm)
      for (int i = 0; i < H.mnc[mm]; ++i) inmol[H.matom[mm][i]] = true;
    H.nmref = 0;
    bool seen[kER] = {};
    for (int mm = 0; mm < m->nmol; ++mm)
      for (int i = 0; i < H.mnc[mm]; ++i)
        if (H.matom[mm][i] > 0 && !seen[H.mref[mm][i]]) {
          seen[H.mref[mm][i]] = true;
          H.mrefs[H.nmref++] = H.mref[mm][i];
        }
    H.nr = H.nsimple = 0;
    for (int b = 0; b <= m->natom; ++b) {
      if (inmol[b]) {
        H.rmap[b] = H.nr;
        H.rfull[H.nr++] = b;
      } else {
        H.rmap[b] = -1;
        H.simple[H.nsimple++] = b;
      }
    }
  }
  for (int a = 0; a < m->natom; ++a) {
    H.zkeep[a] = 0;
    for (int z = 0; z < H.ns[a]; ++z)
      if (H.ref[H.s0[a] + z] >= 0) H.zkeep[a] = z + 1;
  }
  for (int q = 0; q < H.nst; ++q) {
    StageTab &S = H.stab[q];
    S.zf = H.zf[q];
    S.izf = H.izf[q];
    S.zz = 31.321 * H.zeff[q] * H.zeff[q];
    S.t0 = H.pft[q] == SNAPI_PF_TRAV ? H.t0[q] : 0;
    S.t1 = H.pft[q] == SNAPI_PF_TRAV ? H.t1[q] : 0;
    S.ref = H.ref[q];
    S.pad = 0;
  }
  for (int q = 0; q < nt; ++q) {
    TermTab &Tt = H.ttab[q];
    Tt.l = H.tll[q];
    Tt.il = H.til[q];
    Tt.A = H.tA[q];
    Tt.g2 = H.g2[q];
  }
  // nodes: kinds 1..6, contiguous, non-decreasing
  for (int k = 0; k < 7; ++k) { H.kfirst[k] = 0; H.kcount[k] = 0; }
  int prev = 0;
  for (int q = 0; q < m->npar; ++q) {
    const int k = m->node_kind[q];
    if (k < 1 || k > 6 || k < prev) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: node kinds must be 1..6, non-decreasing");
    if (k != prev) H.kfirst[k] = q;
    H.kcount[k] += 1;
    prev = k;
    H.ntau[q] = m->node_tau[q];
    H.nkind[q] = k;
  }
  for (int k = 1; k <= 6; ++k)
    for (int i = 1; i < H.kcount[k]; ++i)
      if (!(H.ntau[H.kfirst[k] + i] > H.ntau[H.kfirst[k] + i - 1]))
        return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: node log tau must increase within a kind");
  if (H.kcount[1] < 1) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_set: at least one temperature node");

  SNAPI_CK(cudaSetDevice(ctx->device));
  SNAPI_CK(cudaStreamSynchronize(ctx->stream));
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (!e) {
    e = new EosCtx();
    ctx->eos = e;
  }
  if (!e->d_tab) SNAPI_CK(cudaMalloc(&e->d_tab, sizeof(EosDev)));
  SNAPI_CK(cudaMemcpy(e->d_tab, &H, sizeof(EosDev), cudaMemcpyHostToDevice));
  e->h_tab.assign(1, H);
  e->atoms.assign(m->atoms, m->atoms + m->natom);
  e->npar = m->npar;
  e->chem_start = SNAPI_CHEM_START_CONTINUE;
  e->ntherm = H.kcount[1];
  e->kind.assign(m->node_kind, m->node_kind + m->npar);
  e->ref_step.assign(m->npar, 0.0);
  static const double ref_step[7] = {0.0, 5.0, 20.0, 20.0, 0.01, 0.001, 0.001};  // const.h:27-32
  for (int q = 0; q < m->npar; ++q) e->ref_step[q] = ref_step[m->node_kind[q]];
  return SNAPI_OK;
}

int snapi_eos_chem_start(snapi_ctx *ctx, int mode) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (!e) return set_err(ctx, SNAPI_EINVAL, "snapi_eos_chem_start: no node model (snapi_eos_set)");
  if (mode != SNAPI_CHEM_START_CONTINUE && mode != SNAPI_CHEM_START_COLD)
    return set_err(ctx, SNAPI_EINVAL, "snapi_eos_chem_start: unknown mode %d", mode);
  e->chem_start = mode;
  return SNAPI_OK;
}

// snapi_build_records (records != NULL) and snapi_build_atmos (atmos != NULL; x3 a host array)
static int build_impl(snapi_ctx *ctx, int npix, const double *nodes, const int *active, float *records, double *Nt,
                      float *tangents, const double *step, int *pix_status, int mem, const double *x3,
                      double *atmos) {
  using namespace snapi;
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (npix == 0) return SNAPI_OK;
  const int npar = e->npar, nd = ctx->nd, nf = ctx->nfield;
  const int nvar = tangents ? 1 + 2 * e->ntherm : 1;
  std::vector<double> hstep = e->ref_step;
  if (step)
    for (int q = 0; q < npar; ++q) {
      if (!(step[q] > 0.0)) return set_err(ctx, SNAPI_EINVAL, "snapi_build_records: steps must be positive");
      hstep[q] = step[q];
    }
  SNAPI_CK(cudaSetDevice(ctx->device));
  // the build is latency-bound per column: launch as many columns as the scratch allows (the FP64
  // (T, Nt) scratch of 16384 columns with 9 variants is 190 MB)
  const int B = std::min(npix, std::max(ctx->max_batch, 16384));
  if (B > e->cap || nvar > e->cap_var) {
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    eos_free_bufs(e);
    const size_t Bz = (size_t)B;
    SNAPI_CK(cudaMalloc(&e->d_T, sizeof(double) * Bz * nvar * nd));
    SNAPI_CK(cudaMalloc(&e->d_F, sizeof(double) * Bz * nvar * nd * nf));
    SNAPI_CK(cudaMalloc(&e->d_Nt, sizeof(double) * Bz * nvar * nd));
    SNAPI_CK(cudaMalloc(&e->d_nodes, sizeof(double) * Bz * npar));
    SNAPI_CK(cudaMalloc(&e->d_step, sizeof(double) * SNAPI_EOS_MAX_PAR));
    SNAPI_CK(cudaMalloc(&e->d_Ntout, sizeof(double) * Bz * nd));
    SNAPI_CK(cudaMalloc(&e->d_active, sizeof(int) * Bz));
    SNAPI_CK(cudaMalloc(&e->d_status, sizeof(int) * Bz));
    SNAPI_CK(cudaMalloc(&e->d_rec, sizeof(float) * Bz * nd * nf));
    if (nvar > 1) SNAPI_CK(cudaMalloc(&e->d_tan, sizeof(float) * Bz * npar * nd * nf));
    e->cap = B;
    e->cap_var = nvar;
  }
  if (atmos && B > e->cap_atm) {
    cudaFree(e->d_atm);
    e->d_atm = nullptr;
    e->cap_atm = 0;
    SNAPI_CK(cudaMalloc(&e->d_atm, sizeof(double) * (size_t)B * 12 * nd));
    e->cap_atm = B;
  }
  if (atmos && x3) {
    if (!e->d_x3) SNAPI_CK(cudaMalloc(&e->d_x3, sizeof(double) * nd));
    SNAPI_CK(cudaMemcpyAsync(e->d_x3, x3, sizeof(double) * nd, cudaMemcpyHostToDevice, ctx->stream));
  }
  SNAPI_CK(cudaMemcpyAsync(e->d_step, hstep.data(), sizeof(double) * npar, cudaMemcpyHostToDevice, ctx->stream));
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  const bool host = (mem == SNAPI_MEM_HOST);
  for (int p0 = 0; p0 < npix; p0 += B) {
    const int nb = std::min(B, npix - p0);
    EosArgs A;
    A.tab = e->d_tab;
    A.npix = nb;
    A.nvar = nvar;
    A.nd = nd;
    A.npar = npar;
    A.nf = nf;
    A.step = e->d_step;
    A.T = e->d_T;
    A.Nt = e->d_Nt;
    A.F = e->d_F;
    A.status = e->d_status;
    A.warm = e->chem_start == SNAPI_CHEM_START_CONTINUE;
    A.x0 = 0;
    A.x1 = nd;
    A.hs_in = nullptr;
    A.hs_out = nullptr;
    A.vx0 = 0;
    A.vx1 = nd;
    if ((size_t)nb * nvar > e->cap_xf) {
      SNAPI_CK(cudaStreamSynchronize(ctx->stream));
      cudaFree(e->d_xf);
      e->d_xf = nullptr;
      e->cap_xf = 0;
      SNAPI_CK(cudaMalloc(&e->d_xf, sizeof(int) * (size_t)B * nvar));
      e->cap_xf = (size_t)B * nvar;
    }
    A.xf = e->d_xf;
    if (host) {
      SNAPI_CK(cudaMemcpyAsync(e->d_nodes, nodes + (size_t)p0 * npar, sizeof(double) * nb * npar,
                               cudaMemcpyHostToDevice, ctx->stream));
      if (active)
        SNAPI_CK(cudaMemcpyAsync(e->d_active, active + p0, sizeof(int) * nb, cudaMemcpyHostToDevice, ctx->stream));
      A.nodes = e->d_nodes;
      A.active = active ? e->d_active : nullptr;
      A.rec = records ? e->d_rec : nullptr;
      A.tan = tangents ? e->d_tan : nullptr;
      A.Nt_out = Nt ? e->d_Ntout : nullptr;
      if (active) {  // rows of inactive pixels are left untouched: start from the caller's
        if (records)
          SNAPI_CK(cudaMemcpyAsync(e->d_rec, records + (size_t)p0 * nd * nf, sizeof(float) * nb * nd * nf,
                                   cudaMemcpyHostToDevice, ctx->stream));
        if (atmos)
          SNAPI_CK(cudaMemcpyAsync(e->d_atm, atmos + (size_t)p0 * 12 * nd, sizeof(double) * nb * 12 * nd,
                                   cudaMemcpyHostToDevice, ctx->stream));
        if (tangents)
          SNAPI_CK(cudaMemcpyAsync(e->d_tan, tangents + (size_t)p0 * npar * nd * nf,
                                   sizeof(float) * nb * npar * nd * nf, cudaMemcpyHostToDevice, ctx->stream));
        if (Nt)
          SNAPI_CK(cudaMemcpyAsync(e->d_Ntout, Nt + (size_t)p0 * nd, sizeof(double) * nb * nd,
                                   cudaMemcpyHostToDevice, ctx->stream));
      }
    } else {
      A.nodes = nodes + (size_t)p0 * npar;
      A.active = active ? active + p0 : nullptr;
      A.rec = records ? records + (size_t)p0 * nd * nf : nullptr;
      A.tan = tangents ? tangents + (size_t)p0 * npar * nd * nf : nullptr;
      A.Nt_out = Nt ? Nt + (size_t)p0 * nd : nullptr;
    }
    SNAPI_CK(cudaMemsetAsync(e->d_status, 0, sizeof(int) * nb, ctx->stream));
    if (nvar > 1) {  // the variants' first moved depths, read by the march, the record chemistry, the records
      const int nx = nb * (nvar - 1);
      k_eos_xf<<<(nx + kRecThreads - 1) / kRecThreads, kRecThreads, 0, ctx->stream>>>(A);
      SNAPI_CK(cudaGetLastError());
    }
    const int nhe = nb * nvar;
    const long long nvx = (long long)nb * nvar * nd;
    auto launch_he = [&](int t) { k_eos_he<false><<<(nhe + t - 1) / t, t, 0, ctx->stream>>>(A); };
    auto launch_var = [&](int t) {
      k_eos_var<<<(unsigned)((nvx + t - 1) / t), t, 0, ctx->stream>>>(A);
    };
    (void)nvx;
    BuildCfg cfg{kHeDefault, kVarDefault};
    if (ctx->tune && !tuned_build(ctx, npix, &cfg) && p0 == 0) {
      // the autotuner: each CTA size once on this chunk (same results; timed by CUDA events)
      cfg.he = tune_launch(ctx, kHeCands, launch_he, kHeDefault);
      cfg.var = tune_launch(ctx, kVarCands, launch_var, kVarDefault);
      tune_store_build(ctx, npix, cfg);
      SNAPI_CK(cudaMemsetAsync(e->d_status, 0, sizeof(int) * nb, ctx->stream));
    }
    // With tangents the march runs in depth segments, its state carried from one launch to the next,
    // each followed by the record chemistry of its depths: measured 53 ms against 55 ms for one march
    // launch and one record launch at 4096 columns x 9 variants (same arithmetic, same results).
    // Running the record chemistry of finished segments concurrently on a second stream measured 90
    // ms: its CTAs' local memory evicts the march's per-column state from L1 and every chain slows.
    int bounds[kHeMaxSeg + 1] = {0, nd};
    int nseg = 1;
    if (nvar > 1 && nd >= 4 * kHeMaxSeg && e->segmented) {
      nseg = kHeMaxSeg;
      for (int k = 1; k < nseg; ++k) bounds[k] = (int)(kHeSegFrac[k - 1] * nd);
      bounds[nseg] = nd;
      const size_t need = (size_t)kHeStateWords * nhe;
      if (need > e->cap_hs) {
        SNAPI_CK(cudaStreamSynchronize(ctx->stream));
        cudaFree(e->d_hs);
        e->d_hs = nullptr;
        e->cap_hs = 0;
        SNAPI_CK(cudaMalloc(&e->d_hs, 2 * sizeof(double) * need));
        e->cap_hs = need;
      }
    }
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    if (nseg == 1) {
      launch_he(cfg.he);
      SNAPI_CK(cudaGetLastError());
      launch_var(cfg.var);
      SNAPI_CK(cudaGetLastError());
      ctx->last_launches += 2;
    } else {
      for (int k = 0; k < nseg; ++k) {
        A.x0 = A.vx0 = bounds[k];
        A.x1 = A.vx1 = bounds[k + 1];
        A.hs_in = e->d_hs + (size_t)(k & 1) * e->cap_hs;
        A.hs_out = e->d_hs + (size_t)((k + 1) & 1) * e->cap_hs;
        k_eos_he<true><<<(nhe + cfg.he - 1) / cfg.he, cfg.he, 0, ctx->stream>>>(A);
        SNAPI_CK(cudaGetLastError());
        const long long nv_k = (long long)nb * nvar * (A.vx1 - A.vx0);
        k_eos_var<<<(unsigned)((nv_k + cfg.var - 1) / cfg.var), cfg.var, 0, ctx->stream>>>(A);
        SNAPI_CK(cudaGetLastError());
      }
      A.x0 = A.vx0 = 0;
      A.x1 = A.vx1 = nd;
      ctx->last_launches += 2 * nseg;
    }
    const int nrec = nb * nd;
    if (records) {
      k_eos_rec<<<(nrec + kRecThreads - 1) / kRecThreads, kRecThreads, 0, ctx->stream>>>(A);
      SNAPI_CK(cudaGetLastError());
      ++ctx->last_launches;
    }
    if (atmos) {
      double *atm_out = host ? e->d_atm : atmos + (size_t)p0 * 12 * nd;
      k_eos_atm<<<(nrec + kRecThreads - 1) / kRecThreads, kRecThreads, 0, ctx->stream>>>(A, x3 ? e->d_x3 : nullptr,
                                                                                        atm_out);
      SNAPI_CK(cudaGetLastError());
      ++ctx->last_launches;
    }
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    if (host && atmos)
      SNAPI_CK(cudaMemcpyAsync(atmos + (size_t)p0 * 12 * nd, e->d_atm, sizeof(double) * nb * 12 * nd,
                               cudaMemcpyDeviceToHost, ctx->stream));
    if (host) {
      if (records)
        SNAPI_CK(cudaMemcpyAsync(records + (size_t)p0 * nd * nf, e->d_rec, sizeof(float) * nb * nd * nf,
                                 cudaMemcpyDeviceToHost, ctx->stream));
      if (tangents)
        SNAPI_CK(cudaMemcpyAsync(tangents + (size_t)p0 * npar * nd * nf, e->d_tan, sizeof(float) * nb * npar * nd * nf,
                                 cudaMemcpyDeviceToHost, ctx->stream));
      if (Nt)
        SNAPI_CK(cudaMemcpyAsync(Nt + (size_t)p0 * nd, e->d_Ntout, sizeof(double) * nb * nd, cudaMemcpyDeviceToHost,
                                 ctx->stream));
    }
    if (pix_status)
      SNAPI_CK(cudaMemcpyAsync(pix_status + p0, e->d_status, sizeof(int) * nb,
                               host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return SNAPI_OK;
}

int snapi_build_records(snapi_ctx *ctx, int npix, const double *nodes, const int *active, float *records, double *Nt,
                        float *tangents, const double *step, int *pix_status, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (!ctx->eos) return snapi::set_err(ctx, SNAPI_EINVAL, "snapi_build_records: no node model (snapi_eos_set)");
  if (npix < 0 || (npix > 0 && (!nodes || !records)) || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return snapi::set_err(ctx, SNAPI_EINVAL, "snapi_build_records: invalid arguments");
  return build_impl(ctx, npix, nodes, active, records, Nt, tangents, step, pix_status, mem, nullptr, nullptr);
}

int snapi_records_from_columns(snapi_ctx *ctx, int npix, const double *columns, float *records, int *pix_status,
                               int mem) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (!e) return set_err(ctx, SNAPI_EINVAL, "snapi_records_from_columns: no atom tables (snapi_eos_set)");
  if (npix < 0 || (npix > 0 && (!columns || !records)) || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_records_from_columns: invalid arguments");
  if (npix == 0) return SNAPI_OK;
  const int nd = ctx->nd, nf = ctx->nfield;
  const bool host = mem == SNAPI_MEM_HOST;
  SNAPI_CK(cudaSetDevice(ctx->device));
  const int B = std::min(npix, std::max(ctx->max_batch, 16384));
  if (B > e->cap_col) {
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(e->d_cols);
    cudaFree(e->d_crec);
    cudaFree(e->d_cst);
    e->d_cols = nullptr;
    e->d_crec = nullptr;
    e->d_cst = nullptr;
    e->cap_col = 0;
    if (host) {
      SNAPI_CK(cudaMalloc(&e->d_cols, sizeof(double) * (size_t)B * 12 * nd));
      SNAPI_CK(cudaMalloc(&e->d_crec, sizeof(float) * (size_t)B * nd * nf));
    }
    SNAPI_CK(cudaMalloc(&e->d_cst, sizeof(int) * (size_t)B));
    e->cap_col = B;
  } else if (host && !e->d_cols) {
    SNAPI_CK(cudaMalloc(&e->d_cols, sizeof(double) * (size_t)e->cap_col * 12 * nd));
    SNAPI_CK(cudaMalloc(&e->d_crec, sizeof(float) * (size_t)e->cap_col * nd * nf));
  }
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < npix; p0 += B) {
    const int nb = std::min(B, npix - p0);
    const double *cols = columns + (size_t)p0 * 12 * nd;
    float *rec = records + (size_t)p0 * nd * nf;
    if (host) {
      SNAPI_CK(cudaMemcpyAsync(e->d_cols, cols, sizeof(double) * nb * 12 * nd, cudaMemcpyHostToDevice, ctx->stream));
      cols = e->d_cols;
    }
    SNAPI_CK(cudaMemsetAsync(e->d_cst, 0, sizeof(int) * nb, ctx->stream));
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    const int n = nb * nd;
    k_eos_col<<<(n + kRecThreads - 1) / kRecThreads, kRecThreads, 0, ctx->stream>>>(e->d_tab, nb, nd, nf, cols,
                                                                                    host ? e->d_crec : rec, e->d_cst);
    SNAPI_CK(cudaGetLastError());
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ++ctx->last_launches;
    if (host)
      SNAPI_CK(cudaMemcpyAsync(rec, e->d_crec, sizeof(float) * nb * nd * nf, cudaMemcpyDeviceToHost, ctx->stream));
    if (pix_status)
      SNAPI_CK(cudaMemcpyAsync(pix_status + p0, e->d_cst, sizeof(int) * nb,
                               host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, ctx->stream));
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return SNAPI_OK;
}

int snapi_adjoint_nodes(snapi_ctx *ctx, int npix, const double *nodes, const float *obs, const double *w_stokes,
                        const float *mask, float *stokes, double *chi2, double *grad, int *pix_status, int mem) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (!e) return set_err(ctx, SNAPI_EINVAL, "snapi_adjoint_nodes: no node model (snapi_eos_set)");
  if (npix < 0 || (npix > 0 && (!nodes || !obs || !chi2 || !grad)) ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_adjoint_nodes: invalid arguments");
  if (npix == 0) return SNAPI_OK;
  SNAPI_CK(cudaSetDevice(ctx->device));
  const int npar = e->npar, nl = ctx->nl;
  int st = ensure_npar(ctx, npar);
  if (st) return st;
  const bool host = mem == SNAPI_MEM_HOST;
  if (host && !e->d_nn) {
    SNAPI_CK(cudaMalloc(&e->d_nn, sizeof(double) * (size_t)ctx->max_batch * npar));
    SNAPI_CK(cudaMalloc(&e->d_nst, sizeof(int) * (size_t)ctx->max_batch));
  }
  double total_ms = 0.0, phase[2] = {0.0, 0.0};
  int launches = 0;
  for (int p0 = 0; p0 < npix; p0 += ctx->max_batch) {
    const int nb = std::min(ctx->max_batch, npix - p0);
    const double *dn = nodes + (size_t)p0 * npar;
    const float *dobs = obs + (size_t)p0 * nl * 4;
    const float *dmask = mask ? mask + (size_t)p0 * nl : nullptr;
    float *dst = stokes ? stokes + (size_t)p0 * nl * 4 : nullptr;
    double *dchi = chi2 + p0, *dgrad = grad + (size_t)p0 * npar;
    int *dps = pix_status ? pix_status + p0 : nullptr;
    if (host) {  // stage the chunk's inputs; results land in the context's buffers
      SNAPI_CK(cudaMemcpyAsync(e->d_nn, dn, sizeof(double) * nb * npar, cudaMemcpyHostToDevice, ctx->stream));
      SNAPI_CK(cudaMemcpyAsync(ctx->d_obs, dobs, sizeof(float) * nb * nl * 4, cudaMemcpyHostToDevice, ctx->stream));
      if (mask)
        SNAPI_CK(cudaMemcpyAsync(ctx->d_mask, dmask, sizeof(float) * nb * nl, cudaMemcpyHostToDevice, ctx->stream));
      dn = e->d_nn;
      dobs = ctx->d_obs;
      dmask = mask ? ctx->d_mask : nullptr;
      dst = stokes ? ctx->d_stokes : nullptr;
      dchi = ctx->d_chi2;
      dgrad = ctx->d_grad;
      dps = pix_status ? e->d_nst : nullptr;
    }
    // records and node tangents (the reference's steps) of the chunk, kept on the device
    st = build_impl(ctx, nb, dn, nullptr, ctx->d_rec, nullptr, ctx->d_tan, nullptr, dps, SNAPI_MEM_DEVICE, nullptr,
                    nullptr);
    if (st) return st;
    total_ms += ctx->last_ms;
    phase[0] += ctx->last_ms;
    launches += ctx->last_launches;
    st = snapi_adjoint(ctx, nb, ctx->d_rec, dobs, w_stokes, dmask, npar, ctx->d_tan, dst, dchi, dgrad, nullptr,
                       SNAPI_MEM_DEVICE);
    total_ms += ctx->last_ms;
    phase[1] += ctx->last_ms;
    launches += ctx->last_launches;
    if (st) return st;
    if (host) {
      if (stokes)
        SNAPI_CK(cudaMemcpyAsync(stokes + (size_t)p0 * nl * 4, ctx->d_stokes, sizeof(float) * nb * nl * 4,
                                 cudaMemcpyDeviceToHost, ctx->stream));
      SNAPI_CK(cudaMemcpyAsync(chi2 + p0, ctx->d_chi2, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream));
      SNAPI_CK(cudaMemcpyAsync(grad + (size_t)p0 * npar, ctx->d_grad, sizeof(double) * nb * npar,
                               cudaMemcpyDeviceToHost, ctx->stream));
      if (pix_status)
        SNAPI_CK(cudaMemcpyAsync(pix_status + p0, e->d_nst, sizeof(int) * nb, cudaMemcpyDeviceToHost, ctx->stream));
      SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    }
  }
  ctx->last_ms = total_ms;
  ctx->phase_ms[0] = phase[0];
  ctx->phase_ms[1] = phase[1];
  ctx->last_launches = launches;
  return SNAPI_OK;
}

int snapi_build_atmos(snapi_ctx *ctx, int npix, const double *nodes, const int *active, const double *x3,
                      double *atmos, int *pix_status, int mem) {
  if (!ctx) return SNAPI_EINVAL;
  if (!ctx->eos) return snapi::set_err(ctx, SNAPI_EINVAL, "snapi_build_atmos: no node model (snapi_eos_set)");
  if (npix < 0 || (npix > 0 && (!nodes || !atmos)) || (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return snapi::set_err(ctx, SNAPI_EINVAL, "snapi_build_atmos: invalid arguments");
  return build_impl(ctx, npix, nodes, active, nullptr, nullptr, nullptr, nullptr, pix_status, mem, x3, atmos);
}

}  // extern "C"

// ==== NLTE set-up on the device (snapi_ali_setup) ==========================================================
// The population-independent inputs of the level-population iteration (atmosphere::nltepops,
// atmos/atmos_pop.cc:70-130), per column, in FP64:
//   k_alis_depth  thread = (column, depth): the chemistry at (T, Nt) with the reference's cold start and
//                 every ionisation stage's fraction kept (ChemT<kES>), LTE populations, kappa_500, the
//                 NLTE atom's total and start populations, projected velocities, line widths and damping,
//                 bound-free LTE ratios, collisional rates, and the depth's background factors: the
//                 free-free coefficient, the Rayleigh density, the H- factors, each LTE bound-free
//                 level's population and LTE ratio, each LTE level pair's width, damping and opacity
//                 factor (bgf [column][field][depth]).
//   k_alis_bg     thread = (column, ray, wavelength, depth), depth fastest: the LTE background opacity
//                 and emissivity from those factors and the per-wavelength table (cross-sections, the
//                 fudge factor, H- polynomials, Rayleigh cross-section); bound-bound profiles by W4 in
//                 FP64.
namespace snapi {
namespace {

constexpr int kSuLev = 16, kSuLine = 32, kSuBft = 16, kSuRay = 32, kSuBf = 32, kSuBb = 64, kSuAtomLev = 96;
constexpr int kSuRayAtom = 8, kSuLt = 8, kSuThreads = 128;

struct AlisDev {
  int nd, nray, nlam, nlev, nline, nbft, nbf, nbb, nray_atom, nal, nst, nf;
  double gcont;                 // Seaton's factor of the NLTE atom
  double ct[kSuRay];            // cos(pi - theta) of each ray (atmosphere::project with V_x = V_y = 0)
  // every level of the NLTE atom (its total, compute_active_population): stage, g, E
  int al_st[kSuAtomLev];
  double al_g[kSuAtomLev], al_e[kSuAtomLev];
  // the problem's levels: stage, offset to the continuum level (0: none), g, E, the stage's ionisation
  // energy, the next stage's ground g, the edge cross-section
  int lv_st[kSuLev], lv_dl[kSuLev];
  double lv_g[kSuLev], lv_e[kSuLev], lv_ip[kSuLev], lv_gn[kSuLev], lv_se[kSuLev];
  int cn[kSuLev * kSuLev];      // collisional table points (0: no rate: the diagonal, other stages)
  double ctab[kSuLev * kSuLev * 8], cval[kSuLev * kSuLev * 8];
  // lines of the problem: lambda0, damping constants, mass, radiative damping
  double ln_l0[kSuLine], ln_al[kSuLine], ln_sg[kSuLine], ln_ms[kSuLine], ln_ar[kSuLine];
  int bft_lev[kSuBft];          // lower level of each bound-free transition
  // background bound-free levels: stage, g, E, next stage ground g / E, ionisation energy
  int bf_st[kSuBf];
  double bf_g[kSuBf], bf_e[kSuBf], bf_gn[kSuBf], bf_en[kSuBf], bf_ip[kSuBf];
  // background level pairs
  int bb_st[kSuBb];
  double bb_glo[kSuBb], bb_elo[kSuBb], bb_gup[kSuBb], bb_eup[kSuBb], bb_l0[kSuBb], bb_blu[kSuBb], bb_bul[kSuBb],
      bb_ar[kSuBb], bb_al[kSuBb], bb_sg[kSuBb], bb_ms[kSuBb];
  double zz[kES];               // z^2 of every stage (free-free)
  int ray_st[kSuRayAtom];       // neutral stage of each Rayleigh atom
};

// n of a level (atom::lte, atom.cc:763-789) from the solved chemistry: stage total x Boltzmann / U
template <class CH>
__device__ __forceinline__ double su_level(const EosDev &E, const CH &c, int s, double g, double ee) {
  const double tot = c.stage_total(s, E.satom[s]);
  return g != 0.0 ? tot * (g * exp(-ee / (cK * c.T)) / c.stage_U(s, c.N[0])) : tot;
}

// collisional damping of a line (atom::damp_col, atom.cc:939-959)
__device__ __forceinline__ double su_damp_col(double T, double nH0, double alpha, double sig, double mass) {
  const double red_mass = 1.66E-24 / (1.0 / 1.008 + 1.66E-24 / mass);
  const double vmean = sqrt(8.0 * cK * T / cPI / red_mass);
  return nH0 * vmean * pow(vmean / 1E6, -alpha) * sig;
}

// tabulated rate (tbcr::interpol, colr.cc:111-115)
__device__ __forceinline__ double su_tab(const double *t, const double *v, int n, double T) {
  for (int i = 1; i < n; ++i)
    if (t[i] > T) return (v[i] * (T - t[i - 1]) + v[i - 1] * (t[i] - T)) / (t[i] - t[i - 1]);
  return v[n - 1];
}

__global__ void __launch_bounds__(kSuThreads) k_alis_depth(const EosDev *tab, const AlisDev *ad, int ncol,
                                                          const double *cols, double *oT, double *one, double *ona,
                                                          double *okap, double *ovray, double *odld, double *oad,
                                                          double *obfr, double *ocoll, double *opop, double *bgf,
                                                          int *status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const AlisDev &A = *ad;
  const int nd = A.nd;
  if (i >= ncol * nd) return;
  const int p = i / nd, x = i % nd;
  const EosDev &E = *tab;
  const double *cc = cols + (size_t)p * 12 * nd + x;
  const double T = cc[2 * nd], Nt = cc[3 * nd] / (cK * cc[2 * nd]), vt = cc[8 * nd], vz = cc[9 * nd];
  ChemT<kES> c(E);
  double lev[kEL], nH0;
  const double kap = chem_point(E, c, T, Nt, lev, nH0, 1);
  int st = c.capped;
  const double ne = c.N[0], kT = cK * T;
  const size_t pd = (size_t)p * nd + x;
  oT[pd] = T;
  one[pd] = ne;
  okap[pd] = kap;
  double na = 0.0;
  for (int k = 0; k < A.nal; ++k) na += su_level(E, c, A.al_st[k], A.al_g[k], A.al_e[k]);
  ona[pd] = na;
  bool fin = isfinite(ne) && isfinite(kap) && isfinite(na);
  double *pp = opop + pd * A.nlev;
  for (int k = 0; k < A.nlev; ++k) pp[k] = su_level(E, c, A.lv_st[k], A.lv_g[k], A.lv_e[k]);
  for (int r = 0; r < A.nray; ++r) ovray[((size_t)p * A.nray + r) * nd + x] = A.ct[r] * vz;
  for (int q = 0; q < A.nline; ++q) {
    const double l0 = A.ln_l0[q];
    const double dld = sqrt(2.0 * cK * T / A.ln_ms[q] + vt * vt) * l0 / cC;
    const double gc = su_damp_col(T, nH0, A.ln_al[q], A.ln_sg[q], A.ln_ms[q]);
    odld[((size_t)p * A.nline + q) * nd + x] = dld;
    oad[((size_t)p * A.nline + q) * nd + x] = l0 * l0 / (4.0 * cPI * cC) * (A.ln_ar[q] + gc) / dld;
  }
  for (int q = 0; q < A.nbft; ++q) {
    const int k = A.bft_lev[q];
    obfr[((size_t)p * A.nbft + q) * nd + x] =
        ne * cSAHA * pow(T, -1.5) * A.lv_g[k] / A.lv_gn[k] * exp((A.lv_ip[k] - A.lv_e[k]) / kT);
  }
  // the rate matrix's collisional rates (atom_pop.cc:27-145, atom_rad.cc:1769-1901)
  {
    const int nl = A.nlev;
    double *C = ocoll + pd * nl * nl;
    for (int k = 0; k < nl * nl; ++k) C[k] = 0.0;
    for (int a = 0; a + 1 < nl; ++a) {
      for (int b = 0; b < nl; ++b) {
        const int n = A.cn[a * nl + b];
        if (!n) continue;
        double rate = su_tab(A.ctab + (size_t)(a * nl + b) * 8, A.cval + (size_t)(a * nl + b) * 8, n, T) * ne;
        if (a < b) {  // excitation: detailed balance of the tabulated de-excitation
          const double u0 = fabs(A.lv_e[b] - A.lv_e[a]) / kT;
          rate *= exp(-u0) * A.lv_g[b] / A.lv_g[a];
        }
        C[a * nl + b] = rate;
      }
      const int dl = A.lv_dl[a];
      if (dl) {
        const double dE = A.lv_ip[a] - A.lv_e[a], u0 = dE / kT;
        const double ci = 1.55E13 / sqrt(T) * A.gcont * A.lv_se[a] * exp(-u0) / u0 * ne;
        C[a * nl + a + dl] = ci;
        C[(a + dl) * nl + a] = ci * A.lv_g[a] / A.lv_gn[a] * exp(dE / kT) * pow(T, -1.5) * ne * cSAHA;
      }
    }
  }
  // background factors of this depth
  const size_t fs = (size_t)nd, f0 = (size_t)p * A.nf * nd + x;
  double zs = 0.0;
  for (int s = 0; s < A.nst; ++s)
    if (A.zz[s] != 0.0) zs += A.zz[s] * c.stage_total(s, E.satom[s]);
  const double fct = (cE * cE * cC * cH * cH * cRYD) / (6.0 * cPI * cPI * cPI * cE0 * cME * cC) *
                     sqrt((2.0 * cPI) / (3.0 * cK * cME * cME * cME));
  double nray0 = 0.0;
  for (int k = 0; k < A.nray_atom; ++k) nray0 += c.stage_total(A.ray_st[k], E.satom[A.ray_st[k]]);
  const double tp = 5040.0 / T;
  bgf[f0] = T;
  bgf[f0 + fs] = fct * 1.1 * ne / (sqrt(T) * cC * cC * cC) * zs;
  bgf[f0 + 2 * fs] = nray0;
  bgf[f0 + 3 * fs] = E.hm ? 4.158E-28 * ne * kT * pow(tp, 2.5) * pow(10.0, 0.754 * tp) * nH0 : 0.0;
  bgf[f0 + 4 * fs] = E.hm ? 1E-26 * ne * kT * nH0 : 0.0;
  bgf[f0 + 5 * fs] = log10(tp);
  for (int b = 0; b < A.nbf; ++b) {
    const int s = A.bf_st[b];
    const double nl_ = su_level(E, c, s, A.bf_g[b], A.bf_e[b]);
    const double nn = su_level(E, c, s + 1, A.bf_gn[b], A.bf_en[b]);
    bgf[f0 + (6 + 2 * b) * fs] = nl_;
    bgf[f0 + (7 + 2 * b) * fs] = nn * ne * cSAHA * pow(T, -1.5) * A.bf_g[b] / A.bf_gn[b] * exp((A.bf_ip[b] - A.bf_e[b]) / kT);
  }
  const int fb = 6 + 2 * A.nbf;
  for (int q = 0; q < A.nbb; ++q) {
    const int s = A.bb_st[q];
    const double nlo = su_level(E, c, s, A.bb_glo[q], A.bb_elo[q]);
    const double nup = su_level(E, c, s, A.bb_gup[q], A.bb_eup[q]);
    const double l0 = A.bb_l0[q];
    const double dld = sqrt(2.0 * cK * T / A.bb_ms[q] + vt * vt) * l0 / cC;
    const double gc = su_damp_col(T, nH0, A.bb_al[q], A.bb_sg[q], A.bb_ms[q]);
    bgf[f0 + (fb + 3 * q) * fs] = dld;
    bgf[f0 + (fb + 3 * q + 1) * fs] = l0 * l0 / (4.0 * cPI * cC) * (A.bb_ar[q] + gc) / dld;
    bgf[f0 + (fb + 3 * q + 2) * fs] = nlo * A.bb_blu[q] * (1.0 - nup / nlo * A.bb_bul[q] / A.bb_blu[q]);
  }
  if (!fin) st |= 4;
  if (st) atomicOr(status + p, st);
}

// Humlicek W4 real part / sqrt(pi) in FP64 (cmlib/profiles.cc:7-37: the published region split and
// coefficients, cos taken as sqrt(1 - sin^2) in region 4 as there)
struct Cd {
  double re, im;
};
__device__ __forceinline__ Cd cd_mul(Cd a, Cd b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ Cd cd_div(Cd a, Cd b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
__device__ __forceinline__ Cd cd_add(double s, Cd a) { return {s + a.re, a.im}; }
__device__ __forceinline__ Cd cd_rsub(double s, Cd a) { return {s - a.re, -a.im}; }
__device__ __forceinline__ Cd cd_scl(Cd a, double s) { return {a.re * s, a.im * s}; }

__device__ double w4_re(double v, double a) {
  const double s = fabs(v) + a;
  const Cd t = {a, -v}, u = {a * a - v * v, -2.0 * a * v};
  Cd w;
  if (s >= 15.0) {
    w = cd_div(cd_scl(t, 0.5641896), cd_add(0.5, u));
  } else if (s > 5.5) {
    w = cd_div(cd_mul(t, cd_add(1.410474, cd_scl(u, 0.5641896))), cd_add(0.75, cd_mul(u, cd_add(3.0, u))));
  } else if (a > (0.195 * fabs(v) - 0.176)) {
    Cd n = cd_add(3.778987, cd_scl(t, 0.5642236));
    n = cd_add(11.96482, cd_mul(t, n));
    n = cd_add(20.20933, cd_mul(t, n));
    n = cd_add(16.4955, cd_mul(t, n));
    Cd d = cd_add(6.699398, t);
    d = cd_add(21.69274, cd_mul(t, d));
    d = cd_add(39.27121, cd_mul(t, d));
    d = cd_add(38.82363, cd_mul(t, d));
    d = cd_add(16.4955, cd_mul(t, d));
    w = cd_div(n, d);
  } else {
    Cd pn = cd_rsub(1.320522, cd_scl(u, 0.56419));
    pn = cd_rsub(35.76683, cd_mul(u, pn));
    pn = cd_rsub(219.0313, cd_mul(u, pn));
    pn = cd_rsub(1540.787, cd_mul(u, pn));
    pn = cd_rsub(3321.9905, cd_mul(u, pn));
    pn = cd_rsub(36183.31, cd_mul(u, pn));
    Cd q = cd_rsub(1.841439, u);
    q = cd_rsub(61.57037, cd_mul(u, q));
    q = cd_rsub(364.2191, cd_mul(u, q));
    q = cd_rsub(2186.181, cd_mul(u, q));
    q = cd_rsub(9022.228, cd_mul(u, q));
    q = cd_rsub(24322.84, cd_mul(u, q));
    q = cd_rsub(32066.6, cd_mul(u, q));
    const double su = sin(u.im), eu = exp(u.re);
    const Cd r = cd_div(cd_mul(t, pn), q);
    w = {eu * sqrt(1.0 - su * su) - r.re, eu * su - r.im};
  }
  return w.re / 1.77245386399759;
}

// per-wavelength table: lambda, fudge, h c / lambda, H- bound-free polynomial, H- free-free f0 f1 f2,
// Rayleigh cross-section (kSuLt doubles per wavelength)
__global__ void __launch_bounds__(kSuThreads) k_alis_bg(const AlisDev *ad, int ncol, const double *lt,
                                                       const double *sig, const double *bgf, const double *vray,
                                                       double *bgop, double *bgem) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const AlisDev &A = *ad;
  const int nd = A.nd, nl = A.nlam, nr = A.nray;
  if (i >= (long long)ncol * nr * nl * nd) return;
  const int x = (int)(i % nd);
  const long long q1 = i / nd;
  const int l = (int)(q1 % nl);
  const long long q2 = q1 / nl;
  const int r = (int)(q2 % nr), p = (int)(q2 / nr);
  const double *L = lt + (size_t)l * kSuLt;
  const double lam = L[0], fudge = L[1], hcl = L[2];
  const size_t fs = (size_t)nd;
  const double *F = bgf + (size_t)p * A.nf * nd + x;
  const double T = F[0], kT = cK * T;
  const double v = vray[((size_t)p * nr + r) * nd + x];
  const double lv = lam * (1.0 + v / cC);
  double op = F[fs] * lv * lv * lv * (1.0 - exp(-(cH * cC) / kT / lv)) * fudge;
  op += L[7] * F[2 * fs];
  const double stim = exp(-hcl / kT);
  for (int b = 0; b < A.nbf; ++b) {
    const double s = sig[(size_t)b * nl + l];
    if (s != 0.0) op += s * (F[(6 + 2 * b) * fs] - F[(7 + 2 * b) * fs] * stim) * fudge;
  }
  const int fb = 6 + 2 * A.nbf;
  for (int q = 0; q < A.nbb; ++q) {
    const double dld = F[(fb + 3 * q) * fs];
    const double xv = (A.bb_l0[q] - lv) / dld;
    op += w4_re(xv, F[(fb + 3 * q + 1) * fs]) / dld * F[(fb + 3 * q + 2) * fs] * cH * cC / lam / 4.0 / cPI;
  }
  const double lt_ = F[5 * fs];
  op += L[3] * F[3 * fs] * (1.0 - stim) * fudge;
  op += pow(10.0, L[4] + L[5] * lt_ + L[6] * lt_ * lt_) * F[4 * fs] * fudge;
  const size_t o = (((size_t)p * nr + r) * nl + l) * nd + x;
  bgop[o] = op;
  bgem[o] = op * (2.0 * 6.62606957 * 8.9875517E-7 / lam / lam / lam / lam / lam / (exp(1.4387769 / lam / T) - 1.0));
}

}  // namespace
}  // namespace snapi

namespace snapi {
namespace {

// the set-up's device tables from the ALI problem, the caller's set-up tables and the model's atoms;
// returns an error text, or nullptr
const char *alis_tables(const EosCtx *e, const snapi_ali_problem *P, const snapi_ali_setup_tables *T, AlisDev &A,
                        std::vector<double> &lt, std::vector<double> &sig) {
  const EosDev &H = e->h_tab[0];
  const auto &At = e->atoms;
  const int natom = (int)At.size();
  memset(&A, 0, sizeof(AlisDev));
  A.nd = P->nd;
  A.nray = P->nray;
  A.nlam = P->nlambda;
  A.nlev = P->nlevel;
  A.nst = H.nst;
  if (P->nray > kSuRay) return "too many rays (<= 32)";
  if (P->nlevel > kSuLev) return "too many levels (<= 16)";
  if (T->atom < 0 || T->atom >= natom) return "bad NLTE atom";
  if (T->nbf < 0 || T->nbf > kSuBf || (T->nbf && (!T->bf_level || !T->bf_sigma))) return "bad bound-free list (<= 32)";
  if (T->nbb < 0 || T->nbb > kSuBb || (T->nbb && !T->bb)) return "bad bound-bound list (<= 64)";
  if (T->nray_atom < 0 || T->nray_atom > kSuRayAtom - 1 || (T->nray_atom && !T->ray_atom)) return "bad Rayleigh atoms";
  if (!T->level || !T->sigma_edge || !T->coll_n || !T->coll_t || !T->coll_v || !T->line_damp)
    return "missing set-up tables";
  A.gcont = T->atom_Z == 1 ? 0.1 : (T->atom_Z == 2 ? 0.2 : 0.3);
  for (int r = 0; r < P->nray; ++r) A.ct[r] = cos(cPI - P->ray_theta[r]);
  const snapi_eos_atom &Na = At[T->atom];
  const int s0 = H.s0[T->atom];
  for (int z = 0; z < Na.nstage; ++z)
    for (int l = 0; l < Na.nlevel[z]; ++l) {
      if (A.nal >= kSuAtomLev) return "NLTE atom: too many levels";
      A.al_st[A.nal] = s0 + z;
      A.al_g[A.nal] = Na.level[z][l].g;
      A.al_e[A.nal] = Na.level[z][l].ee;
      ++A.nal;
    }
  const int nlev = P->nlevel;
  for (int k = 0; k < nlev; ++k) {
    const int z = T->level[2 * k], l = T->level[2 * k + 1];
    if (z < 0 || z >= Na.nstage || l < 0 || l >= Na.nlevel[z]) return "bad level map";
    // the rate-matrix loop of the reference walks the levels of a stage as consecutive indices
    if (k > 0 && T->level[2 * k - 2] == z && T->level[2 * k - 1] != l - 1) return "levels of a stage not consecutive";
    if (l > 0 && (k == 0 || T->level[2 * k - 2] != z)) return "levels of a stage not consecutive";
    A.lv_st[k] = s0 + z;
    A.lv_g[k] = Na.level[z][l].g;
    A.lv_e[k] = Na.level[z][l].ee;
    A.lv_se[k] = T->sigma_edge[k];
    if (z + 1 < Na.nstage) {
      A.lv_ip[k] = Na.ip[z];
      A.lv_gn[k] = Na.level[z + 1][0].g;
    }
  }
  for (int k = 0; k + 1 < nlev; ++k) {
    const int z = T->level[2 * k], l = T->level[2 * k + 1];
    for (int ll = 0; ll < Na.nlevel[z]; ++ll) {
      const int j = k + (ll - l);
      if (j < 0 || j >= nlev) return "rate-matrix level outside the problem's levels";
      if (ll == l) continue;
      const int n = T->coll_n[k * nlev + j];
      if (n < 1 || n > 8) return "a collisional rate without a table (only tabulated rates on the device)";
      A.cn[k * nlev + j] = n;
      for (int q = 0; q < n; ++q) {
        A.ctab[(k * nlev + j) * 8 + q] = T->coll_t[(k * nlev + j) * 8 + q];
        A.cval[(k * nlev + j) * 8 + q] = T->coll_v[(k * nlev + j) * 8 + q];
      }
    }
    const int dl = Na.nlevel[z] - l;
    if (k + dl >= nlev) return "continuum level outside the problem's levels";
    A.lv_dl[k] = dl;
  }
  for (int t = 0; t < P->ntrans; ++t) {
    const int lo = P->trans[2 * t], up = P->trans[2 * t + 1];
    if (P->cont_of[lo] == up) {
      if (A.nbft >= kSuBft) return "too many bound-free transitions";
      A.bft_lev[A.nbft++] = lo;
    } else {
      if (A.nline >= kSuLine) return "too many lines";
      const int q = A.nline++;
      A.ln_l0[q] = P->line_c[4 * t];
      A.ln_al[q] = T->line_damp[4 * q];
      A.ln_sg[q] = T->line_damp[4 * q + 1];
      A.ln_ms[q] = T->line_damp[4 * q + 2];
      A.ln_ar[q] = T->line_damp[4 * q + 3];
    }
  }
  A.nbf = T->nbf;
  for (int b = 0; b < T->nbf; ++b) {
    const int a = T->bf_level[3 * b], z = T->bf_level[3 * b + 1], l = T->bf_level[3 * b + 2];
    if (a < 0 || a >= natom || z < 0 || z + 1 >= At[a].nstage || l < 0 || l >= At[a].nlevel[z] ||
        At[a].nlevel[z + 1] < 1)
      return "bad bound-free level";
    A.bf_st[b] = H.s0[a] + z;
    A.bf_g[b] = At[a].level[z][l].g;
    A.bf_e[b] = At[a].level[z][l].ee;
    A.bf_gn[b] = At[a].level[z + 1][0].g;
    A.bf_en[b] = At[a].level[z + 1][0].ee;
    A.bf_ip[b] = At[a].ip[z];
  }
  A.nbb = T->nbb;
  for (int q = 0; q < T->nbb; ++q) {
    const snapi_ali_bb &B = T->bb[q];
    if (B.atom < 0 || B.atom >= natom || B.stage < 0 || B.stage >= At[B.atom].nstage || B.lower < 0 ||
        B.upper < 0 || B.lower >= At[B.atom].nlevel[B.stage] || B.upper >= At[B.atom].nlevel[B.stage] ||
        !(B.mass > 0.0))
      return "bad bound-bound pair";
    A.bb_st[q] = H.s0[B.atom] + B.stage;
    A.bb_glo[q] = At[B.atom].level[B.stage][B.lower].g;
    A.bb_elo[q] = At[B.atom].level[B.stage][B.lower].ee;
    A.bb_gup[q] = At[B.atom].level[B.stage][B.upper].g;
    A.bb_eup[q] = At[B.atom].level[B.stage][B.upper].ee;
    A.bb_l0[q] = B.lambda0;
    A.bb_blu[q] = B.Blu;
    A.bb_bul[q] = B.Bul;
    A.bb_ar[q] = B.a_rad;
    A.bb_al[q] = B.alpha_col;
    A.bb_sg[q] = B.sigma_col;
    A.bb_ms[q] = B.mass;
  }
  // Rayleigh: the listed atoms, and the NLTE atom itself when its Z is 1 (its free-free and Rayleigh
  // opacity enter the background as the LTE atoms' do)
  for (int k = 0; k < T->nray_atom; ++k) {
    if (T->ray_atom[k] < 0 || T->ray_atom[k] >= natom) return "bad Rayleigh atom";
    A.ray_st[A.nray_atom++] = H.s0[T->ray_atom[k]];
  }
  if (T->atom_Z == 1) A.ray_st[A.nray_atom++] = s0;
  for (int a = 0; a < natom; ++a)
    for (int z = 0; z < At[a].nstage; ++z) A.zz[H.s0[a] + z] = (double)z * (double)z;
  A.nf = 6 + 2 * A.nbf + 3 * A.nbb;
  // per-wavelength table (kSuLt): lambda, fudge, h c / lambda, H- bound-free polynomial (mol.cc:
  // 609-632), H- free-free f0 f1 f2 (mol.cc:516-545), Rayleigh cross-section (atom_rad.cc:268-298)
  lt.assign((size_t)P->nlambda * kSuLt, 0.0);
  for (int l = 0; l < P->nlambda; ++l) {
    const double lam = P->lambda[l];
    double *L = &lt[(size_t)l * kSuLt];
    L[0] = lam;
    L[1] = P->fudge[l];
    L[2] = cH * cC / lam;
    const double ca[7] = {1.99654, -1.18267E-5, 2.64243E-6, -4.40524E-10, 3.23992E-14, -1.39568E-18, 2.78701E-23};
    double alpha = 0.0;
    for (int i = 0; i < 7; ++i) alpha += ca[i] * pow(lam * 1E8, (double)i);
    L[3] = alpha;
    const double lg = log10(lam * 1E8);
    L[4] = -2.2763 - 1.6850 * lg + 0.76661 * lg * lg - 0.053346 * lg * lg * lg;
    L[5] = 15.2827 - 9.2846 * lg + 1.99381 * lg * lg - 0.142631 * lg * lg * lg;
    L[6] = -197.789 + 190.266 * lg - 67.9775 * lg * lg + 10.6913 * lg * lg * lg - 0.625151 * lg * lg * lg * lg;
    // the reference's coefficient loop reads its first coefficient for every power and then squares
    // the cross-section; kept as it stands
    const double l0 = 1215.67E-8;
    double cs = 0.0;
    for (int ii = 0; ii <= 5; ++ii) cs += 1.26563 * pow(l0 / lam, 2 * ii);
    cs *= pow(l0 / lam, 4);
    L[7] = cs * cs * 6.65E-25;
  }
  sig.assign(T->bf_sigma, T->bf_sigma + (size_t)T->nbf * P->nlambda);
  return nullptr;
}

}  // namespace
}  // namespace snapi

extern "C" {

int snapi_ali_setup(snapi_ctx *ctx, const snapi_ali_problem *prob, const snapi_ali_setup_tables *tab, int ncol,
                    const double *columns, const snapi_ali_setup_out *out, double *pops0, int *status, int mem) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (!e || e->h_tab.empty()) return set_err(ctx, SNAPI_EINVAL, "snapi_ali_setup: no atom tables (snapi_eos_set)");
  if (!prob || !tab || !out || ncol < 0 || (ncol > 0 && (!columns || !pops0)) ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_ali_setup: invalid arguments");
  if (prob->nd < 3 || prob->nlambda < 1 || prob->nray < 1 || prob->nlevel < 2 || prob->ntrans < 1 || !prob->lambda ||
      !prob->fudge || !prob->ray_theta || !prob->trans || !prob->line_c || !prob->cont_of)
    return set_err(ctx, SNAPI_EINVAL, "snapi_ali_setup: invalid ALI problem");
  for (int t = 0; t < prob->ntrans; ++t)
    if (prob->trans[2 * t] < 0 || prob->trans[2 * t] >= prob->nlevel || prob->trans[2 * t + 1] < 0 ||
        prob->trans[2 * t + 1] >= prob->nlevel)
      return set_err(ctx, SNAPI_EINVAL, "snapi_ali_setup: transition levels out of range");
  std::vector<AlisDev> hv(1);
  AlisDev &A = hv[0];
  std::vector<double> lt, sig;
  if (const char *msg = alis_tables(e, prob, tab, A, lt, sig)) return set_err(ctx, SNAPI_EINVAL, "snapi_ali_setup: %s", msg);
  if (!out->T || !out->ne || !out->na || !out->kappa || !out->vray || (A.nline && (!out->dld || !out->adamp)) ||
      (A.nbft && !out->bfratio) || !out->coll || !out->bg_op || !out->bg_em)
    return set_err(ctx, SNAPI_EINVAL, "snapi_ali_setup: missing output arrays");
  if (ncol == 0) return SNAPI_OK;
  // the set-up's chemistry table: the node model's, every ionisation stage's fraction kept
  std::vector<EosDev> ev(1, e->h_tab[0]);
  {
    EosDev &S = ev[0];
    int nref = S.nref;
    for (int s = 0; s < S.nst; ++s)
      if (S.ref[s] < 0) S.ref[s] = nref++;
    S.nref = nref;
    for (int a = 0; a < S.natom; ++a) S.zkeep[a] = S.ns[a];
    for (int q = 0; q < S.nst; ++q) S.stab[q].ref = S.ref[q];
  }
  const int nd = A.nd, nr = A.nray, nl = A.nlam, nv = A.nlev, nli = A.nline, nbt = A.nbft;
  const bool host = mem == SNAPI_MEM_HOST;
  // work arena: tables, per-wavelength table, cross-sections, status, background factors; host arrays
  // also stage the columns and every output.  Chunks of up to 4096 columns, host staging within ~2 GB.
  const size_t per_col_out = (size_t)nd * (4 + nr + 2 * nli + nbt + nv * nv + nv) + 2 * (size_t)nr * nl * nd;
  int B = std::min(ncol, 4096);
  if (host) B = (int)std::max<size_t>(1, std::min<size_t>(B, ((size_t)2 << 30) / (sizeof(double) * per_col_out)));
  size_t off = 0;
  auto take = [&](size_t bytes) { const size_t o = off; off += (bytes + 255) & ~(size_t)255; return o; };
  const size_t o_tab = take(sizeof(EosDev)), o_ad = take(sizeof(AlisDev)), o_lt = take(sizeof(double) * lt.size()),
               o_sig = take(sizeof(double) * std::max<size_t>(sig.size(), 1)), o_st = take(sizeof(int) * B),
               o_bgf = take(sizeof(double) * (size_t)B * A.nf * nd);
  const size_t o_cols = host ? take(sizeof(double) * (size_t)B * 12 * nd) : 0;
  const size_t o_out = host ? take(sizeof(double) * (size_t)B * per_col_out) : 0;
  SNAPI_CK(cudaSetDevice(ctx->device));
  if (off > e->cap_su) {
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(e->d_su);
    e->d_su = nullptr;
    e->cap_su = 0;
    SNAPI_CK(cudaMalloc(&e->d_su, off));
    e->cap_su = off;
  }
  char *base = static_cast<char *>(e->d_su);
  EosDev *d_tab = reinterpret_cast<EosDev *>(base + o_tab);
  AlisDev *d_ad = reinterpret_cast<AlisDev *>(base + o_ad);
  double *d_lt = reinterpret_cast<double *>(base + o_lt), *d_sig = reinterpret_cast<double *>(base + o_sig);
  int *d_st = reinterpret_cast<int *>(base + o_st);
  double *d_bgf = reinterpret_cast<double *>(base + o_bgf);
  SNAPI_CK(cudaMemcpyAsync(d_tab, ev.data(), sizeof(EosDev), cudaMemcpyHostToDevice, ctx->stream));
  SNAPI_CK(cudaMemcpyAsync(d_ad, hv.data(), sizeof(AlisDev), cudaMemcpyHostToDevice, ctx->stream));
  SNAPI_CK(cudaMemcpyAsync(d_lt, lt.data(), sizeof(double) * lt.size(), cudaMemcpyHostToDevice, ctx->stream));
  if (!sig.empty())
    SNAPI_CK(cudaMemcpyAsync(d_sig, sig.data(), sizeof(double) * sig.size(), cudaMemcpyHostToDevice, ctx->stream));
  ctx->last_ms = 0.0;
  ctx->last_launches = 0;
  for (int p0 = 0; p0 < ncol; p0 += B) {
    const int nb = std::min(B, ncol - p0);
    // this chunk's arrays: the caller's (device) or the staging area (host)
    const double *cols = columns + (size_t)p0 * 12 * nd;
    double *aT, *ane, *ana, *akap, *avr, *adld, *aad, *abfr, *acoll, *aop, *aem, *apop;
    if (host) {
      SNAPI_CK(cudaMemcpyAsync(base + o_cols, cols, sizeof(double) * nb * 12 * nd, cudaMemcpyHostToDevice, ctx->stream));
      cols = reinterpret_cast<const double *>(base + o_cols);
      double *q = reinterpret_cast<double *>(base + o_out);
      aT = q; q += (size_t)B * nd;
      ane = q; q += (size_t)B * nd;
      ana = q; q += (size_t)B * nd;
      akap = q; q += (size_t)B * nd;
      avr = q; q += (size_t)B * nr * nd;
      adld = q; q += (size_t)B * nli * nd;
      aad = q; q += (size_t)B * nli * nd;
      abfr = q; q += (size_t)B * nbt * nd;
      acoll = q; q += (size_t)B * nd * nv * nv;
      apop = q; q += (size_t)B * nd * nv;
      aop = q; q += (size_t)B * nr * nl * nd;
      aem = q;
    } else {
      aT = out->T + (size_t)p0 * nd;
      ane = out->ne + (size_t)p0 * nd;
      ana = out->na + (size_t)p0 * nd;
      akap = out->kappa + (size_t)p0 * nd;
      avr = out->vray + (size_t)p0 * nr * nd;
      adld = nli ? out->dld + (size_t)p0 * nli * nd : nullptr;
      aad = nli ? out->adamp + (size_t)p0 * nli * nd : nullptr;
      abfr = nbt ? out->bfratio + (size_t)p0 * nbt * nd : nullptr;
      acoll = out->coll + (size_t)p0 * nd * nv * nv;
      apop = pops0 + (size_t)p0 * nd * nv;
      aop = out->bg_op + (size_t)p0 * nr * nl * nd;
      aem = out->bg_em + (size_t)p0 * nr * nl * nd;
    }
    SNAPI_CK(cudaMemsetAsync(d_st, 0, sizeof(int) * nb, ctx->stream));
    SNAPI_CK(cudaEventRecord(ctx->ev0, ctx->stream));
    const int n1 = nb * nd;
    k_alis_depth<<<(n1 + kSuThreads - 1) / kSuThreads, kSuThreads, 0, ctx->stream>>>(
        d_tab, d_ad, nb, cols, aT, ane, ana, akap, avr, adld, aad, abfr, acoll, apop, d_bgf, d_st);
    SNAPI_CK(cudaGetLastError());
    const long long n2 = (long long)nb * nr * nl * nd;
    k_alis_bg<<<(unsigned)((n2 + kSuThreads - 1) / kSuThreads), kSuThreads, 0, ctx->stream>>>(d_ad, nb, d_lt, d_sig,
                                                                                              d_bgf, avr, aop, aem);
    SNAPI_CK(cudaGetLastError());
    SNAPI_CK(cudaEventRecord(ctx->ev1, ctx->stream));
    ctx->last_launches += 2;
    if (host) {
      auto back = [&](double *dst, const double *src, size_t per_col) -> cudaError_t {
        return cudaMemcpyAsync(dst + (size_t)p0 * per_col, src, sizeof(double) * nb * per_col, cudaMemcpyDeviceToHost,
                               ctx->stream);
      };
      SNAPI_CK(back(out->T, aT, nd));
      SNAPI_CK(back(out->ne, ane, nd));
      SNAPI_CK(back(out->na, ana, nd));
      SNAPI_CK(back(out->kappa, akap, nd));
      SNAPI_CK(back(out->vray, avr, (size_t)nr * nd));
      if (nli) SNAPI_CK(back(out->dld, adld, (size_t)nli * nd));
      if (nli) SNAPI_CK(back(out->adamp, aad, (size_t)nli * nd));
      if (nbt) SNAPI_CK(back(out->bfratio, abfr, (size_t)nbt * nd));
      SNAPI_CK(back(out->coll, acoll, (size_t)nd * nv * nv));
      SNAPI_CK(back(pops0, apop, (size_t)nd * nv));
      SNAPI_CK(back(out->bg_op, aop, (size_t)nr * nl * nd));
      SNAPI_CK(back(out->bg_em, aem, (size_t)nr * nl * nd));
    }
    if (status)
      SNAPI_CK(cudaMemcpyAsync(status + p0, d_st, sizeof(int) * nb, host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                               ctx->stream));
    SNAPI_CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0.f;
    SNAPI_CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_ms += ms;
  }
  return SNAPI_OK;
}

}  // extern "C"

// ==== records of an NLTE atom's lines from level populations (snapi_records_set_populations) =============
namespace snapi {
namespace {

struct PopLines {
  int n;                                    // lines whose fields are set
  int line[SNAPI_MAX_LINES], lo[SNAPI_MAX_LINES], up[SNAPI_MAX_LINES];
  double Blu[SNAPI_MAX_LINES], Bul[SNAPI_MAX_LINES], A[SNAPI_MAX_LINES], lam0[SNAPI_MAX_LINES];
};

// thread = (pixel, depth): the opacity and emissivity fields of each listed line
__global__ void __launch_bounds__(kRecThreads) k_rec_pops(PopLines L, int npix, int nd, int nf, int nlev,
                                                         const double *pops, float *rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix * nd) return;
  const double *n = pops + (size_t)i * nlev;
  float *r = rec + (size_t)i * nf;
  for (int k = 0; k < L.n; ++k) {
    const double nl = n[L.lo[k]], nu = n[L.up[k]];
    const int j = L.line[k];
    // the record's line fields as the node build forms them from LTE populations (thermal_fields)
    r[SNAPI_NFIELD0 + 3 * j] = (float)((nl * L.Blu[k] - nu * L.Bul[k]) * cH * cC / L.lam0[k] / 4.0 / cPI);
    r[SNAPI_NFIELD0 + 3 * j + 1] = (float)(nu * L.A[k] * cH * cC / L.lam0[k] / 4.0 / cPI);
  }
}

}  // namespace
}  // namespace snapi

extern "C" {

int snapi_records_set_populations(snapi_ctx *ctx, int npix, float *records, const double *pops, int nlevel,
                                  const int *line_level, int mem) {
  using namespace snapi;
  if (!ctx) return SNAPI_EINVAL;
  EosCtx *e = static_cast<EosCtx *>(ctx->eos);
  if (!e || e->h_tab.empty())
    return set_err(ctx, SNAPI_EINVAL, "snapi_records_set_populations: no atom tables (snapi_eos_set)");
  if (npix < 0 || (npix > 0 && (!records || !pops)) || nlevel < 1 || !line_level ||
      (mem != SNAPI_MEM_HOST && mem != SNAPI_MEM_DEVICE))
    return set_err(ctx, SNAPI_EINVAL, "snapi_records_set_populations: invalid arguments");
  const EosDev &H = e->h_tab[0];
  PopLines L;
  memset(&L, 0, sizeof(L));
  for (int j = 0; j < ctx->nlines; ++j) {
    const int lo = line_level[2 * j], up = line_level[2 * j + 1];
    if (lo < 0 && up < 0) continue;
    if (lo < 0 || up < 0 || lo >= nlevel || up >= nlevel)
      return set_err(ctx, SNAPI_EINVAL, "snapi_records_set_populations: line %d: bad level indices", j);
    const int k = L.n++;
    L.line[k] = j;
    L.lo[k] = lo;
    L.up[k] = up;
    // atom_rad_synthesis.cc:405-435 with the node model's Einstein coefficients
    L.Blu[k] = H.lBlu[j];
    L.Bul[k] = H.lBul[j];
    L.A[k] = H.lA[j];
    L.lam0[k] = H.llam0[j];
  }
  if (npix == 0 || L.n == 0) return SNAPI_OK;
  const int nd = ctx->nd, nf = ctx->nfield;
  SNAPI_CK(cudaSetDevice(ctx->device));
  float *d_rec = records;
  const double *d_pops = pops;
  void *stage = nullptr;
  const size_t brec = sizeof(float) * (size_t)npix * nd * nf, bpop = sizeof(double) * (size_t)npix * nd * nlevel;
  if (mem == SNAPI_MEM_HOST) {
    SNAPI_CK(cudaMalloc(&stage, brec + bpop));
    d_rec = static_cast<float *>(stage);
    d_pops = reinterpret_cast<const double *>(static_cast<char *>(stage) + brec);
    SNAPI_CK(cudaMemcpyAsync(d_rec, records, brec, cudaMemcpyHostToDevice, ctx->stream));
    SNAPI_CK(cudaMemcpyAsync(const_cast<double *>(d_pops), pops, bpop, cudaMemcpyHostToDevice, ctx->stream));
  }
  const int n = npix * nd;
  k_rec_pops<<<(n + kRecThreads - 1) / kRecThreads, kRecThreads, 0, ctx->stream>>>(L, npix, nd, nf, nlevel, d_pops,
                                                                                  d_rec);
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess && mem == SNAPI_MEM_HOST)
    err = cudaMemcpyAsync(records, d_rec, brec, cudaMemcpyDeviceToHost, ctx->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
  if (stage) cudaFree(stage);
  if (err != cudaSuccess) return set_err(ctx, SNAPI_ECUDA, "snapi_records_set_populations: %s", cudaGetErrorString(err));
  ctx->last_launches = 1;
  return SNAPI_OK;
}

}  // extern "C"
