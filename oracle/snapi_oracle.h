/*
 * snapi_oracle -- FP64 CPU restatement of SNAPI's Stokes synthesis hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.  The product
 * (snapi_b200, libsnapi_cuda) never calls it.
 *
 * It restates, in plain C and in the reference's order of operations:
 *   - fvoigt (Humlicek W4 region split)          cmlib/profiles.cc:7-37, :91-115
 *   - Zeeman component pattern                   atmos/atmol/atom/atom.cc:1620-1773
 *   - opacity / emissivity assembly per (lambda, depth) from a column record:
 *       Thomson at lambda_mid                    atmos/atmos_rad_synthesis.cc:31-50
 *       bound-free (flat below the edge)         atmos/atmol/atom/atom_rad_synthesis.cc:226-262
 *       bound-bound Zeeman Voigt-Faraday         atmos/atmol/atom/atom_rad_synthesis.cc:396-505
 *       H- bound-free + free-free per lambda     atmos/atmol/mol/mol.cc:379-412, :516-632
 *       symmetric / antisymmetric fill           atmos/atmos_rad_synthesis.cc:57-68
 *       division by kappa_500                    atmos/atmos_rad.cc:175-185
 *   - polarized DELO-"Bezier" formal solution     atmos/plpar/atmos_ppbez_rts.cc:918-1218
 *     (monotone Bezier optical depth, linear DELO weights, 4x4 Crout, top point copied)
 *   - airtovac, Planck_f                         cmlib/mathtools.cc:1325-1338, :1150-1152
 *
 * Pinned against the compiled reference (oracle/_ref/snapi_ref_dump) by tests/test_oracle.py.
 *
 * Column record layout (per pixel, depth-major [nd][nfield], nfield = 12 + 3*nlines):
 *   0 T [K]   1 v_turb [cm/s]   2 n_e [cm^-3]   3 v_los projected on the ray [cm/s]
 *   4 |B| [G] 5 inclination [deg, ray frame]    6 azimuth [deg, ray frame]
 *   7 kappa_500 [cm^-1]   8 H- bound-free factor   9 H- free-free factor
 *   10 bound-free opacity (all atoms)   11 bound-free emissivity (all atoms)
 *   12+3j line j: opacity factor (n_l B_lu - n_u B_ul) h c / (4 pi lambda0),
 *   13+3j line j: emissivity factor n_u A_ul h c / (4 pi lambda0),  14+3j collisional damping
 */
#ifndef SNAPI_ORACLE_H
#define SNAPI_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define SNO_MAXCOMP 16

typedef struct {
  double lam0;   /* line centre, vacuum [cm] */
  double sf;     /* lam0^2 / (4 pi c) */
  double ar;     /* radiative damping rate [s^-1] */
  double mass;   /* atomic mass [g] */
  int split;     /* 1: Zeeman split, 0: single Voigt */
  int ncomp[3];  /* pi, sigma_b, sigma_r component counts */
  double S[3][SNO_MAXCOMP];   /* strengths, normalised per group */
  double D[3][SNO_MAXCOMP];   /* shifts in units of lambda_B */
} sno_line;

/* Humlicek W4: H(x,a), F(x,a) (both already divided by sqrt(pi)) */
void sno_voigt(double x, double a, double *H, double *F);

/* Zeeman pattern for 2J values ju2, jl2 and Lande factors gu, gl; returns split flag */
int sno_zeeman_pattern(int ju2, int jl2, double gu, double gl, sno_line *L);

double sno_airtovac(double lambda_air_cm);
double sno_planck(double lambda_cm, double T);

/* Normalised opacity (16, row-major) and emissivity (4) at one depth and one vacuum wavelength.
 * lam_mid: mid wavelength of the vacuum grid (Thomson emissivity).  rec: nfield values. */
void sno_opacity(const double *rec, int nlines, const sno_line *lines, double lam_vac,
                 double lam_mid, double *op16, double *em4);

/* Polarised formal solution.  tau500[nd] positive, top->bottom.  op[nd][16], em[nd][4]
 * normalised.  ct = cos(theta) of the ray (theta = pi for mu = 1).  I[nd][4] out;
 * the emergent Stokes vector is I[0]. */
void sno_formal(int nd, const double *tau500, const double *op, const double *em, double ct,
                double *I);

/* Full synthesis of one pixel: stokes[nl][4] from its record [nd][nfield]. */
void sno_synth_pixel(int nd, int nl, const double *lam_air, const double *tau500, const double *rec,
                     int nlines, const sno_line *lines, double ct, double *stokes);

/* Batch synthesis over npix pixels (records contiguous). */
void sno_synth_batch(int npix, int nd, int nl, const double *lam_air, const double *tau500,
                     const double *rec, int nlines, const sno_line *lines, double ct, double *stokes);

/* chi2 = sum_l,s ((obs - S) * ws[s] * mask[l])^2 for one pixel */
double sno_chi2(int nl, const double *stokes, const double *obs, const double *ws, const double *mask);

/* Directional derivative of chi2 by central differences of the record along tangent
 * directions: grad[p] = (chi2(rec + h tan_p) - chi2(rec - h tan_p)) / 2h, with h = step. */
void sno_chi2_grad_fd(int nd, int nl, const double *lam_air, const double *tau500, const double *rec,
                      int nlines, const sno_line *lines, double ct, const double *obs, const double *ws,
                      const double *mask, int npar, const double *tangent, double step, double *chi2,
                      double *grad);

/* Stokes tangent (JVP) by central differences: dS[p][nl][4]. */
void sno_stokes_jvp_fd(int nd, int nl, const double *lam_air, const double *tau500, const double *rec,
                       int nlines, const sno_line *lines, double ct, int npar, const double *tangent,
                       double step, double *dS);

#ifdef __cplusplus
}
#endif
#endif
