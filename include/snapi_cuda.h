/*
 * libsnapi_cuda -- B200 (sm_100a) drop-in for SNAPI's per-pixel Stokes hot path.
 *
 * Plain C ABI: plain pointers and sizes, no C++ or torch types.  One context per host thread;
 * calls on one context are serialised on the context's CUDA stream and return when done.
 *
 * Interfaces replaced (paths within the reference project):
 *   atmosphere::obs_stokes                     atmos/atmos.h:275, atmos/atmos_obs.cc:16-87
 *       -> snapi_synth
 *   atmosphere::obs_stokes_responses_to_nodes  atmos/atmos.h:269, atmos/atmos_fit.cc:1205-1352,
 *   (+ obs_stokes_responses, formal_pert_numerical)  atmos/atmos_rad_synthesis.cc:166-399,
 *                                              atmos/plpar/atmos_ppbez_rts.cc:1780-1857
 *       -> snapi_responses (forward mode), snapi_adjoint (reverse mode, chi2 gradient)
 *   atmosphere::stokes_lm_fit                  atmos/atmos.h:300, atmos/atmos_fit.cc:18-227
 *       -> snapi_lm_begin / snapi_lm_step (one reference iteration) / snapi_lm_result
 *   atmosphere::nltepops                       atmos/atmos.h, atmos/atmos_pop.cc:67-240
 *       -> snapi_ali_create / snapi_ali_iter
 *   atom::zeeman_setup                         atmos/atmol/atom/atom.cc:1620-1773
 *       -> snapi_zeeman_pattern
 *
 * Data model.  The caller (the reference's islave, after build_from_nodes / chemistry) marshals
 * each pixel's column into a "record": depth-major float32 [nd][nfield] with
 * nfield = SNAPI_NFIELD0 + 3 * nlines:
 *   0 T [K]   1 v_turb [cm/s]   2 n_e [cm^-3]   3 v_los projected on the ray [cm/s]
 *   4 |B| [G] 5 inclination [deg, ray frame]   6 azimuth [deg, ray frame]   7 kappa_500 [cm^-1]
 *   8 H- bound-free factor 4.158e-28 n_e k T theta^2.5 10^(0.754 theta) n_H0
 *   9 H- free-free factor 1e-26 n_e k T n_H0            (theta = 5040/T)
 *   10 bound-free opacity of all atoms   11 bound-free emissivity of all atoms
 *   12+3j  line j opacity factor  (n_l B_lu - n_u B_ul) h c / (4 pi lambda0)
 *   13+3j  line j emissivity factor n_u A_ul h c / (4 pi lambda0)
 *   14+3j  line j collisional damping rate (atom::damp_col)
 * Records of npix pixels are contiguous.  Depth index 0 is the top of the atmosphere.
 *
 * Node tangents for the gradient / responses: float32 [npix][npar][nd][nfield], the derivative
 * of each record field with respect to each node (the reference builds the same map with
 * central differences of build_from_nodes / interpolate_from_nodes, atmos_fit.cc:1225-1307).
 *
 * Memory: every array argument lives either in host memory (mem = SNAPI_MEM_HOST; the call
 * copies in and out, pinned memory from snapi_host_alloc is fastest) or in device memory of the
 * context's GPU (mem = SNAPI_MEM_DEVICE; no copies).
 */
#ifndef SNAPI_CUDA_H
#define SNAPI_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define SNAPI_OK 0
#define SNAPI_EINVAL (-1)
#define SNAPI_ECUDA (-2)
#define SNAPI_ETIMEOUT (-3)
#define SNAPI_ENONCONV (-4)
#define SNAPI_ENOMEM (-5)

#define SNAPI_MEM_HOST 0
#define SNAPI_MEM_DEVICE 1

#define SNAPI_NFIELD0 12
#define SNAPI_MAX_LINES 16
#define SNAPI_MAX_COMP 16
#define SNAPI_MAX_LAMBDA 8192

typedef struct snapi_ctx snapi_ctx;

/* One spectral line (bound-bound transition with A > 1, atom_rad_synthesis.cc:403). */
typedef struct {
  double lam0;           /* vacuum line centre [cm] = h c / (E_u - E_l) */
  double sf;             /* lam0^2 / (4 pi c) */
  double ar;             /* radiative damping rate, atom::damp_rad [s^-1] */
  double mass;           /* atomic mass [g] */
  int split;             /* 1: Zeeman split (pattern below), 0: single Voigt profile */
  int ncomp[3];          /* number of pi, sigma_b, sigma_r components */
  double S[3][SNAPI_MAX_COMP];  /* component strengths, normalised per group */
  double D[3][SNAPI_MAX_COMP];  /* component shifts in units of lambda_B = 4.67e-5 lam0^2 B */
} snapi_line;

typedef struct {
  int nd;                    /* depth points (>= 3) */
  int nlambda;               /* wavelengths (1..SNAPI_MAX_LAMBDA) */
  int nlines;                /* lines (0..SNAPI_MAX_LINES) */
  const double *lambda_air;  /* [nlambda] air wavelengths [cm]; converted with airtovac */
  const double *tau500;      /* [nd] tau_500 of the depth grid, increasing top -> bottom */
  double mu;                 /* cosine of the ray to the outward normal (reference: -cos(EL)), (0,1] */
  const snapi_line *lines;   /* [nlines] */
  double stokes_scale;       /* chi2 is computed internally in units of stokes_scale^2 (> 0) */
  int max_batch;             /* pixels per device batch (sizes the work buffers); 0 = 4096 */
} snapi_problem;

/* Create a context on CUDA device `device`.  Returns NULL on error (status set). */
snapi_ctx *snapi_create(const snapi_problem *prob, int device, int *status);
void snapi_destroy(snapi_ctx *ctx);
/* Last error message of the context (never NULL). */
const char *snapi_last_error(const snapi_ctx *ctx);

/* Stokes synthesis: stokes [npix][nlambda][4] (I, Q, U, V), from records [npix][nd][nfield]. */
int snapi_synth(snapi_ctx *ctx, int npix, const float *records, float *stokes, int mem);

/* Synthesis + chi2 + its gradient w.r.t. npar nodes in one forward and one reverse (adjoint)
 * sweep.  obs [npix][nlambda][4]; w_stokes [4]; mask [npix][nlambda] (NULL = all ones);
 * tangents [npix][npar][nd][nfield] (NULL when npar == 0).
 * chi2 = sum_{l,s} ((obs - S) w_s mask_l)^2 (atmos_fit.cc:239-248).
 * Outputs: stokes (may be NULL), chi2 [npix], grad [npix][npar] (d chi2 / d node),
 * rec_grad [npix][nd][nfield] (d chi2 / d record field; may be NULL). */
int snapi_adjoint(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                  const float *mask, int npar, const float *tangents, float *stokes, double *chi2,
                  double *grad, double *rec_grad, int mem);

/* The adjoint with node tangents in packed form.  Node p touches only the record fields whose bits
 * are set in field_mask[p] (bit f = field f; nfield <= 64): packed_tangents [npix][ntcol][nd] holds,
 * node by node and within a node field by field in increasing order, the depth profile
 * d record[z][f] / d node_p; ntcol = sum of the masks' bit counts.  Same result as snapi_adjoint
 * with the dense tangents (the omitted entries are zeros).  The reference's node tangents are
 * sparse this way: a temperature node moves T, n_e and the opacity fields (22 of 27 for Fe I 6300),
 * v_turb one field, v_los one, B / inclination / azimuth the three field fields, so the packed
 * form is 100 of 270 columns -- 2.7x less host-to-device traffic. */
int snapi_adjoint_packed(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                         const float *mask, int npar, const unsigned long long *field_mask,
                         const float *packed_tangents, float *stokes, double *chi2, double *grad, int mem);

/* Node responses dstokes [npix][npar][nlambda][4] = d Stokes / d node, the quantity
 * obs_stokes_responses_to_nodes returns (atmos_fit.cc:1205-1352), by central differences of the
 * record along each node tangent: (S(rec + h_p t_p) - S(rec - h_p t_p)) / 2 h_p, step [npar] in
 * node units (2 npar forward solves; FP32, ~1e-3 relative with steps ~1e-3 of the node scale).
 * stokes (the unperturbed synthesis) may be NULL. */
int snapi_responses(snapi_ctx *ctx, int npix, const float *records, int npar, const float *tangents,
                    const double *step, float *stokes, float *dstokes, int mem);

/* How snapi_responses and the LM (snapi_lm_step, snapi_lm_fit) form dS/dnode.
 *   SNAPI_JACOBIAN_FD (default): central differences of the record along each node tangent, steps
 *     in node units (2 npar forward solves).
 *   SNAPI_JACOBIAN_TANGENT: forward mode -- the exact derivative of the FP32 synthesis along each
 *     node tangent, carried through the opacity (W4 with its x / a derivatives), the Bezier
 *     optical depth and the DELO recursion, as the reference carries its semi-analytic
 *     derivatives through formal_with_responses_full (atmos_ppbez_rts.cc:1223-1704); steps are not
 *     used.  One forward pass storing the state, then one sweep per node in which the W4
 *     evaluations are shared among the nodes.
 * The setting lasts for the context. */
#define SNAPI_JACOBIAN_FD 0
#define SNAPI_JACOBIAN_TANGENT 1
int snapi_jacobian_mode(snapi_ctx *ctx, int mode);

/* Plain finite-difference gradient (the baseline the adjoint replaces): for each node p the
 * records are perturbed by +-step[p] * tangent_p and synthesised again (2 npar + 1 solves).
 * step [npar] in node units. */
int snapi_fd_grad(snapi_ctx *ctx, int npix, const float *records, const float *obs, const double *w_stokes,
                  const float *mask, int npar, const float *tangents, const double *step, double *chi2,
                  double *grad, int mem);

/* Zeeman pattern of a transition, 2J values ju2 / jl2 and Lande factors (atom::zeeman_setup). */
/* ---------------------------------------------------------------------------------------------
 * Batched Levenberg-Marquardt node fit: stokes_lm_fit (atmos/atmos_fit.cc:18-227) for many pixels
 * at once, each with its own damping, iteration count, mask and stop decision.  The node ->
 * record map (build_from_nodes: interpolation, hydrostatic equilibrium, chemistry) stays with
 * the caller; every step hands back the node vectors whose records and tangents the next step
 * needs, so one step per reference iteration:
 *   snapi_lm_begin(ctx, npix, &opts, nodes0, obs, w_stokes, mask, request, mem);
 *   do { build records + tangents at request[p] for pixels with active[p];
 *        snapi_lm_step(ctx, records, tangents, request, active, &n_active, mem); } while (n_active);
 *   snapi_lm_result(ctx, nodes, chi2, iters, stokes, mem);
 * Per pixel and step (atmos_fit.cc:93-205): synthesis at the trial nodes; chi2; accept (damping
 * / sqrt(10), floor 1e-5, chi2 tracked, stop when the relative change of the last two tracked
 * values is below delta) or reject (damping * sqrt(10)); on acceptance the Jacobian at the new
 * nodes (snapi_responses on the given tangents); J scaled by T 5000 K, velocities 1e5 cm/s,
 * B 1000 G, angles 1 (atmos_fit.cc:250-260), J^T J and J^T r in FP64, diagonal * (1 + damping),
 * solution by the symmetric eigen-decomposition with singular values below max / 1e6 dropped
 * (solve_svd, cmlib/mathtools.cc:344-390), correction added and bracketed to the node bounds
 * (T 3400..12000 K, v_turb 1e2..1.5e6, v_los -1.5e6..1.5e6 cm/s, B 1..1e4 G,
 * atmos_model.cc:12-19,957-977).  Angles are polished (acos cos, atan tan) in snapi_lm_result.
 * chi2 here is sum(((obs - S) w_s mask)^2) / stokes_scale^2. */
#define SNAPI_LM_MAX_PAR 32
typedef struct {
  int npar;                 /* nodes per pixel (<= SNAPI_LM_MAX_PAR) */
  const int *node_kind;     /* [npar]: 1 T, 2 v_turb, 3 v_los, 4 B, 5 inclination, 6 azimuth */
  double lm_start;          /* initial damping (observable start_lambda) */
  int max_iter;             /* iterations (observable no_iterations) */
  double delta;             /* relative chi2 change that ends the fit (atmos_fit.cc:16, 1e-3) */
  double stopping_chisq;    /* chi2 below which the fit ends after one more step */
  const double *resp_step;  /* [npar] central-difference steps of the Jacobian, node units */
  double spectral_broadening; /* Gaussian instrumental width [cm] (cfg SPECTRAL_BROADENING mA x 1e-11
                                 / 2.35), applied to the Stokes vectors and the Jacobian as
                                 stokes_lm_fit does (atmos_fit.cc:104-109); 0: none */
} snapi_lm_opts;

/* nodes0, request: double [npix][npar]; obs float [npix][nlambda][4]; mask float [npix][nlambda]
 * or NULL; w_stokes double [4] or NULL.  request receives the bracketed initial nodes. */
int snapi_lm_begin(snapi_ctx *ctx, int npix, const snapi_lm_opts *opts, const double *nodes0, const float *obs,
                   const double *w_stokes, const float *mask, double *request, int mem);
/* records / tangents of the node vectors in request (rows of inactive pixels are ignored);
 * request, active [npix] and *n_active are updated. */
int snapi_lm_step(snapi_ctx *ctx, const float *records, const float *tangents, double *request, int *active,
                  int *n_active, int mem);
/* snapi_lm_step with the caller's Jacobian instead of record tangents: jacobian [npix][npar][nlambda]
 * [4] (float, unscaled dS/dnode at the requested nodes, in the node order and units of
 * snapi_responses) -- e.g. the reference's own semi-analytic responses (obs_stokes_responses_to_nodes,
 * atmos_fit.cc:1205-1352), as its stokes_lm_fit uses them (atmos_fit.cc:100-133).  Rows of pixels
 * whose step is rejected keep the previous Jacobian, as the reference's do. */
int snapi_lm_step_jacobian(snapi_ctx *ctx, const float *records, const float *jacobian, double *request,
                           int *active, int *n_active, int mem);
/* fitted nodes [npix][npar], chi2 [npix], iterations [npix] and Stokes [npix][nlambda][4]
 * (any may be NULL). */
int snapi_lm_result(snapi_ctx *ctx, double *nodes, double *chi2, int *iters, float *stokes, int mem);

/* ---------------------------------------------------------------------------------------------
 * NLTE level populations: the accelerated lambda iteration of atmosphere::nltepops
 * (atmos/atmos_pop.cc:67-240) for one NLTE atom in many 1-D columns.  Per iteration and column:
 * for every ray and wavelength of the NLTE grid the scalar formal solution with its diagonal
 * operator (atmos_ppbez::formal, atmos/plpar/atmos_ppbez_rts.cc:21-219: Bezier optical depth with
 * monotone derivatives, linear short characteristics, Taylor branch below 1e-2) of background +
 * active opacity; the profile-weighted mean intensities and operators of every transition
 * (atom::add, atmos/atmol/atom/atom.cc:1865-1927); per depth the rate equations with the local
 * operator (atom::newpops, atom_pop.cc:27-145; R_ij_local_ALO, R_i_cont, R_cont_i, atom_rad.cc:
 * 1732-1901), the most populated level replaced by particle conservation, an LU solve in FP64;
 * the maximum relative change; negative populations -> the same step without the operator, and
 * the column stops with status -1 if they stay negative (atmos_pop.cc:185-210).
 * Everything that does not depend on the NLTE populations comes from the caller (the reference's
 * own set-up in islave): the wavelength grid (atom::getlambda) and weights, the rays
 * (anglesetup), the LTE background opacity / emissivity per ray and wavelength, the collisional
 * rates per depth, Doppler widths and damping per line, the bound-free cross sections. */
typedef struct {
  int nd, nlambda, nray, nlevel, ntrans;
  const double *grid;       /* [nd] coordinate of the formal solution (-tau500, top first) */
  const double *lambda;     /* [nlambda] NLTE wavelength grid [cm] */
  const double *lambda_w;   /* [nlambda] wavelength integration weights */
  const double *fudge;      /* [nlambda] bound-free opacity fudge factor */
  const double *ray_theta;  /* [nray] ray angles [rad] (theta > pi/2: outgoing) */
  const double *ray_w;      /* [nray] angular weights */
  const int *trans;         /* [ntrans][2]: lower, upper level; a transition whose upper level is
                               a continuum (cont_of[lower] == upper) is bound-free */
  const double *line_c;     /* [ntrans][4] for lines: lambda0 [cm], A_ul, B_lu, B_ul */
  const double *line_e;     /* [ntrans] E_upper - E_lower [erg] (lines) */
  const double *A, *B;      /* [nlevel][nlevel] Einstein coefficients from -> to (same stage) */
  const int *stage;         /* [nlevel] ionisation stage of each level */
  const int *cont_of;       /* [nlevel] level index of the continuum of each level, -1 if none */
  const double *sigma;      /* [ntrans][nlambda] bound-free cross sections (rows of bf transitions) */
} snapi_ali_problem;

typedef struct {            /* per column; lines / bf transitions in transition order */
  const double *T, *ne, *na, *kappa;  /* [ncol][nd]: temperature, electrons, atom total, kappa_500 */
  const double *vray;                 /* [ncol][nray][nd] velocity projected on each ray [cm/s] */
  const double *dld, *adamp;          /* [ncol][nline][nd] Doppler width [cm], damping parameter */
  const double *bfratio;              /* [ncol][nbf][nd] n_e saha T^-1.5 g_i/g_c exp((ip-E_i)/kT) */
  const double *coll;                 /* [ncol][nd][nlevel][nlevel] collisional rate from -> to */
  const double *bg_op, *bg_em;        /* [ncol][nray][nlambda][nd] LTE background */
} snapi_ali_columns;

typedef struct snapi_ali_ctx snapi_ali_ctx;
snapi_ali_ctx *snapi_ali_create(const snapi_ali_problem *prob, int device, int *status);
void snapi_ali_destroy(snapi_ali_ctx *ctx);
const char *snapi_ali_last_error(const snapi_ali_ctx *ctx);
/* Iterates every column (pops [ncol][nd][nlevel] in: starting populations, out: result) until
 * its maximum relative change falls below tol or max_iter iterations; rel_change [ncol], iters
 * [ncol], status [ncol] (0 converged or stopped at max_iter, -1 negative populations) may be
 * NULL.  Host arrays (SNAPI_MEM_HOST) or device arrays (SNAPI_MEM_DEVICE). */
int snapi_ali_iter(snapi_ali_ctx *ctx, int ncol, const snapi_ali_columns *cols, double *pops, int max_iter,
                   double tol, double *rel_change, int *iters, int *status, int mem);
double snapi_ali_last_kernel_ms(const snapi_ali_ctx *ctx);

/* ---------------------------------------------------------------------------------------------
 * The population-independent set-up of nltepops on the device: what the reference computes once
 * per column before its iterations (atmos/atmos_pop.cc:70-130) and what snapi_ali_iter otherwise
 * takes from the caller.  From a column (the 12 rows of snapi_build_atmos: T, the gas pressure
 * Nt k T, v_turb and v_z are read) and the node model's atom tables (snapi_eos_set on ctx):
 *   - the chemistry and LTE populations at (T, Nt) (ltepops, atmos_pop.cc:31-46; chemeq with the
 *     reference's cold start, atom::lte), kappa_500 (compute_op_referent), the NLTE atom's total
 *     over all its levels (compute_active_population, atom.cc:793-810) and its LTE populations
 *     (pops0 [ncol][nd][nlevel], the iteration's start);
 *   - per ray the projected velocity (atmosphere::project, atmos_rad.cc:15-30);
 *   - the LTE background per ray, NLTE wavelength and depth (opacity_lte / emissivity_lte,
 *     atmos_rad.cc:225-246, whose Thomson term is zeroed): every LTE atom's free-free (atom_rad.cc:
 *     203-236), Rayleigh (atom_rad.cc:268-298, atoms with atom::Z == 1, the reference's coefficient
 *     loop as it stands), bound-free (atom_rad.cc:312-340) and bound-bound opacity (atom_rad.cc:
 *     502-535: every level pair, FP64 W4 profile), H- bound-free and free-free (mol.cc:516-632), plus
 *     the NLTE atom's own free-free; the emissivity is the opacity times the Planck function;
 *   - per line of the NLTE atom the Doppler width and damping (atom_rad.cc:879-883, atom.cc:926-959),
 *     per bound-free transition the LTE ratio factor (atom_rad.cc:327-335), and the collisional
 *     rates of the rate matrix (atom_rad.cc:1769-1901: tabulated de-excitation rates linear in T
 *     times n_e, excitation by detailed balance; Seaton's continuum rate and its inverse).
 * All FP64.  The caller fills the tables from its atom objects (the reference: atom::bf, B, A,
 * alpha_col_dam, col_dam_cross_section, mass, cr, rmap): */
typedef struct {
  int atom, stage, lower, upper;  /* LTE atom (index in the node model's tables) and level pair */
  double lambda0;                 /* h c / (E_upper - E_lower) [cm] */
  double Blu, Bul;                /* atom::B[z][lower][upper], B[z][upper][lower] */
  double a_rad;                   /* atom::damp_rad(A[z], lower, upper) */
  double alpha_col, sigma_col;    /* alpha_col_dam[z][upper][lower], col_dam_cross_section[z][upper][lower] */
  double mass;                    /* atom mass [g] */
} snapi_ali_bb;

typedef struct {
  int nbf;                  /* bound-free levels of the LTE atoms (atom::bf[z][l] set, z < Z) */
  const int *bf_level;      /* [nbf][3]: atom, stage, level */
  const double *bf_sigma;   /* [nbf][nlambda]: bf[z][l]->U at the problem's NLTE wavelengths [cm^2] */
  int nbb;                  /* bound-bound level pairs of the LTE atoms (every pair of every stage) */
  const snapi_ali_bb *bb;   /* [nbb] */
  int nray_atom;            /* atoms with Rayleigh scattering (atom::Z == 1) */
  const int *ray_atom;      /* [nray_atom] */
  int atom;                 /* the NLTE atom (index in the node model's tables) */
  int atom_Z;               /* its atom::Z (Seaton's factor: 0.1 for Z = 1, 0.2 for Z = 2, else 0.3) */
  const int *level;         /* [nlevel][2]: stage and level of each of the problem's levels; the
                               levels of a stage consecutive and in order (atom::rmap) */
  const double *line_damp;  /* [nline][4] per line transition (problem order): alpha_col, sigma_col,
                               mass [g], a_rad */
  const double *sigma_edge; /* [nlevel] bf[z][l]->U(h c / (ip_z - E_l)) (-1 where the reference has
                               no cross-section; 0 for the top stage) */
  const int *coll_n;        /* [nlevel][nlevel] points of the tabulated rate between two levels of a
                               stage (atom::cr[z][upper][lower], stored for both orders; <= 8) */
  const double *coll_t;     /* [nlevel][nlevel][8] temperatures [K] */
  const double *coll_v;     /* [nlevel][nlevel][8] de-excitation rate coefficients [cm^3 s^-1] */
} snapi_ali_setup_tables;

typedef struct {            /* output arrays, the layout of snapi_ali_columns */
  double *T, *ne, *na, *kappa, *vray, *dld, *adamp, *bfratio, *coll, *bg_op, *bg_em;
} snapi_ali_setup_out;

/* The set-up of ncol columns [ncol][12][nd] (nd = prob->nd; the rows of snapi_build_atmos) for the
 * NLTE problem prob (the same problem as the snapi_ali_ctx that iterates them) with ctx's atom
 * tables: out (every array set), pops0 [ncol][nd][nlevel], status [ncol] (may be NULL: 0, or a sum
 * of 1 -- a chemistry solve hit its iteration cap -- and 4 -- non-finite values).  The arrays of
 * out, passed on as a snapi_ali_columns, and pops0 are the inputs of snapi_ali_iter.  mem: all
 * arrays on the host (SNAPI_MEM_HOST) or on ctx's GPU (SNAPI_MEM_DEVICE).  Returns SNAPI_EINVAL
 * for a pair of the NLTE atom's levels without a tabulated collisional rate (the reference's
 * van Regemorter fallback is not on the device). */
int snapi_ali_setup(snapi_ctx *ctx, const snapi_ali_problem *prob, const snapi_ali_setup_tables *tab, int ncol,
                    const double *columns, const snapi_ali_setup_out *out, double *pops0, int *status, int mem);

/* The records of an NLTE atom's lines from its level populations -- the synthesis after nltepops
 * (obs_stokes, atmos_obs.cc:16-87: op_em_vector reads the populations nltepops left,
 * atom_rad_synthesis.cc:405-435).  For each of the context's lines j with line_level[j] = {lower,
 * upper} (indices into the levels of pops [npix][nd][nlevel], e.g. snapi_ali_iter's), the opacity
 * and emissivity fields of records [npix][nd][nfield] become (n_l B_lu - n_u B_ul) h c / (4 pi
 * lambda0) and n_u A h c / (4 pi lambda0) with the node model's Einstein coefficients (snapi_eos_set);
 * lines with {-1, -1} keep their fields.  The other fields do not depend on the NLTE atom's
 * populations (its continuum is not in kappa_500, nltepops leaves n_e as it is).  mem: records and
 * pops on the host or on the device; line_level [nlines][2] is always a host array. */
int snapi_records_set_populations(snapi_ctx *ctx, int npix, float *records, const double *pops, int nlevel,
                                  const int *line_level, int mem);

/* Batched small Gram matrices on the tensor cores: G[m] = M[m] M[m]^T for nmat matrices M[m]
 * [16][K] (row-major, float32, device memory), G [nmat][16][16] float32 (device).  tcgen05 MMA with a
 * three-product TF32 split (hi hi^T + hi lo^T + lo hi^T), FP32 accumulation: ~1e-6 relative.  This
 * is how snapi_lm_step forms J^T J and J^T r (atmos_fit.cc:135-137) for up to 15 nodes; exported for
 * callers with their own small normal equations.  stream: a cudaStream_t or NULL.  The call
 * allocates nothing (its status word is a static device word, shared by calls that overlap on a
 * GPU) and waits for its stream once. */
int snapi_batched_gram(int nmat, int K, const float *M, float *G, void *stream);

/* Gaussian instrumental broadening in place: spectra [nvec][nlambda][4] on the context's wavelength
 * grid (convolve_spectra_with_gauss, cmlib/mathtools.cc:1350-1414; observable::spectral_convolve).
 * width [cm] as the reference holds it (cfg SPECTRAL_BROADENING in mA x 1e-11 / 2.35).  Where the
 * reference reads an unset interval width (the first interval of its interpolation grid,
 * mathtools.cc:1073-1093) this uses that interval's width; the reference's output there is undefined
 * (values up to 1e44, which its kernel tails spread over ~12 widths from the blue end). */
int snapi_spectral_broaden(snapi_ctx *ctx, int nvec, float *spectra, double width, int mem);

int snapi_zeeman_pattern(int ju2, int jl2, double g_upper, double g_lower, snapi_line *line);

/* ---------------------------------------------------------------------------------------------
 * Node model -> column records on the device: atmos_pp::build_from_nodes (atmos/plpar/atmos_pp.cc:
 * 58-248) followed by the set-up obs_stokes performs before its wavelength loop, i.e. what the
 * caller otherwise marshals into records:
 *   - log tau_500 grid tau_min + (tau_max - tau_min) / (nd - 1) * x, and every quantity from its
 *     nodes by atmospheric_interpolation (cmlib/mathtools.cc:1208-1315: monotone cubic Bezier, flat
 *     ends except the temperature's bottom slope from the FAL-C table, T bracketed to 3400..20000 K);
 *     B, inclination, azimuth -> B_x, B_y, B_z (atmos_pp.cc:169-173) -> the ray frame (transform,
 *     atmos_rad.cc:24-48); v_z projected on the ray (project, atmos_rad.cc:14-22);
 *   - hydrostatic equilibrium: the top particle density by fixed point from 0.3 / k T (at most 20
 *     steps, stop at 1e-2 relative change), then downward p_i = p_{i-1} + g dtau / kappa_mean with
 *     kappa_mean the geometric mean of kappa / rho (at most 20 steps per depth, stop when the change
 *     is below 1e-2 of the TOP density, as the reference writes it: atmos_pp.cc:209-236), each
 *     step with the chemistry, the LTE populations, kappa at lambda_referent
 *     (opacity_continuum) and rho = 1.4 * 1.67e-24 * (free hydrogen nuclei);
 *   - chemistry per depth (atmosphere::chemeq, atmos/atmos_chm.cc:28-371): the starting electron
 *     density from the ionisation balance (quadratic guess + halving), then Newton on charge and
 *     particle conservation and the abundance ratios, molecules through their equilibrium
 *     constants (moleqc.cc: polynomial in 5040 / T, the H- form), at most 51 iterations, converged
 *     when every defect is below 1e-4 of its density; ionisation fractions (atom::ionfrc,
 *     atom.cc:892-925) from the partition functions (Traving with Fischel-Sparks asymptotic terms,
 *     Irwin, constant; partf.cc:217-283, 345-358); Saha-Boltzmann level populations (atom::lte,
 *     atom.cc:779-787);
 *   - the record of each depth: T, v_turb, n_e, projected v_los, |B|, inclination, azimuth,
 *     kappa_500 at airtovac(lambda_referent) (compute_op_referent, atmos_ppbez_rts.cc:268-281:
 *     Thomson + bound-free of the LTE atoms with stimulated emission + H- bound-free and free-free,
 *     atmos_rad.cc:286-294, atom_rad.cc:151-187, mol.cc:669-694), the H- factors, the bound-free
 *     totals of the wavelength window (atom_rad_synthesis.cc:226-262), per line the opacity and
 *     emissivity factors and atom::damp_col (atom.cc:938-959);
 *   - with tangents: d(record)/d(node) by central differences with the reference's steps (or the
 *     caller's): a temperature node by two full builds (HE + chemistry), the other nodes by
 *     re-interpolation only (atmos_fit.cc:1225-1307).
 * Deliberate deviations: the 10 x 10 (atoms + 1) Newton system of chemeq is solved by Gaussian
 * elimination with partial pivoting instead of an SVD (same solution for the non-singular
 * system; the reference exits on a singular one); where the FAL-C slope table's interpolation
 * reads an unset interval width (bottom temperature node in -0.0123..0.088, mathtools.cc:1073,
 * 1093) this uses that interval's width.
 *
 * The caller fills the tables from its atom / molecule objects (the reference: atom::abund, ip,
 * partf, nl, g, ee, bf; mol components and K; the model's nodes): */
#define SNAPI_EOS_MAX_ATOMS 16
#define SNAPI_EOS_MAX_STAGES 12      /* ionisation stages per atom (Z + 1) */
#define SNAPI_EOS_MAX_LEVELS 16      /* levels per stage (atom::nl[z]) */
#define SNAPI_EOS_MAX_MOLS 32
#define SNAPI_MOL_MAX_COMP 4
#define SNAPI_EOS_MAX_PAR 128         /* nodes of the model (one per depth is common for T) */
#define SNAPI_PF_MAX_TERMS 8
#define SNAPI_PF_MAX_COEF 8
#define SNAPI_PF_NONE 0               /* U = 1 */
#define SNAPI_PF_CONST 1
#define SNAPI_PF_TRAV 2
#define SNAPI_PF_IRWIN 3
#define SNAPI_EQC_CONST 1
#define SNAPI_EQC_POLY 2
#define SNAPI_EQC_HMIN 3              /* marks the H- molecule (h_minus_mol): its continuum opacity */

typedef struct {                      /* one stage's partition function (class pf and derived) */
  int type;                           /* SNAPI_PF_* */
  int nterm;                          /* TRAV: terms */
  int ncoef;                          /* IRWIN: coefficients of ln U in powers of ln T */
  int m[SNAPI_PF_MAX_TERMS];          /* TRAV: coefficients per term */
  double value;                       /* CONST */
  double zeff;                        /* TRAV: stage charge + 1 (trav::z) */
  double g0;                          /* TRAV: ground statistical weight */
  double g2[SNAPI_PF_MAX_TERMS], ee[SNAPI_PF_MAX_TERMS], ll[SNAPI_PF_MAX_TERMS];
  double gam[SNAPI_PF_MAX_TERMS][SNAPI_PF_MAX_COEF];  /* trav::g: excitation energies [eV] */
  double a[SNAPI_PF_MAX_TERMS][SNAPI_PF_MAX_COEF];    /* trav::a: weights */
  double coef[SNAPI_PF_MAX_COEF];     /* IRWIN */
} snapi_partition;

typedef struct {                      /* one level of one stage */
  double g;                           /* statistical weight (atom::g; 0: population = stage total) */
  double ee;                          /* energy [erg] (atom::ee) */
  /* bound-free cross-section bf[z][l]->U(lambda) [cm^2] evaluated by the caller at: */
  double sigma_he;                    /* lambda_he */
  double sigma_kappa;                 /* lambda_kappa */
  double sigma_win;                   /* lambda_win */
  double lambda_win;                  /* vacuum window wavelength of atom::boundfree_op_em_vector: the
                                         last of the problem's wavelengths at or blueward of the
                                         edge [cm]; 0 when the edge lies blueward of all of them */
} snapi_eos_level;

typedef struct {
  double abundance;                   /* atom::abund, relative to the first atom */
  int nstage;                         /* Z + 1 */
  int nlte;                           /* 1: left out of the continuum opacity (check_if_nlte) */
  double ip[SNAPI_EOS_MAX_STAGES];    /* ionisation energy of stage z [erg], z < nstage - 1 */
  int nlevel[SNAPI_EOS_MAX_STAGES];
  snapi_partition pf[SNAPI_EOS_MAX_STAGES];
  snapi_eos_level level[SNAPI_EOS_MAX_STAGES][SNAPI_EOS_MAX_LEVELS];
} snapi_eos_atom;

typedef struct {
  int ncomp;
  int comp_atom[SNAPI_MOL_MAX_COMP];  /* atom index, -1 for the electron */
  int comp_charge[SNAPI_MOL_MAX_COMP];/* component charge (struct ion z; -1 for the electron) */
  int eqc;                            /* SNAPI_EQC_* */
  int ncoef;
  double coef[SNAPI_PF_MAX_COEF];     /* POLY: log10 K = sum coef[i] (5040 / T)^i; CONST: coef[0] = K */
} snapi_eos_molecule;

typedef struct {                      /* the level pair of each of the problem's lines */
  int atom, stage, lower, upper;
  double Blu, Bul, A;                 /* Einstein coefficients (atom::B[z][lo][up], B[z][up][lo], A) */
  double alpha_col, sigma_col;        /* atom::alpha_col_dam[z][up][lo], col_dam_cross_section[z][up][lo] */
} snapi_eos_line;

typedef struct {
  int natom;                          /* atoms in the reference's order; atoms[0] is hydrogen: its
                                         neutral stage feeds H- and the collisional damping, its
                                         free total the mass density */
  const snapi_eos_atom *atoms;
  int nmol;
  const snapi_eos_molecule *mols;
  const snapi_eos_line *lines;        /* [problem nlines] */
  double lambda_he;                   /* lambda_referent [cm] (opacity of the HE iteration) */
  double lambda_kappa;                /* airtovac(lambda_referent) [cm] (the record's kappa_500) */
  double grav;                        /* surface gravity [cm s^-2] (grav_acc) */
  double tau_min, tau_max;            /* log tau_500 at the first and last depth */
  double theta, phi;                  /* ray direction [rad] (observable EL, AZ) */
  int npar;                           /* nodes (<= SNAPI_EOS_MAX_PAR), kinds non-decreasing */
  const int *node_kind;               /* [npar] 1 T, 2 v_turb, 3 v_los, 4 B, 5 inclination, 6 azimuth */
  const double *node_tau;             /* [npar] log tau_500 of each node */
} snapi_eos_model;

/* Attach a node model to the context (tables copied to the device).  The problem's tau500 grid
 * must be 10^(log tau grid) of the model. */
int snapi_eos_set(snapi_ctx *ctx, const snapi_eos_model *model);

/* How the chemistry (atmosphere::chemeq, atmos_chm.cc:28-330) of the hydrostatic march of
 * snapi_build_records / snapi_build_atmos / snapi_adjoint_nodes / snapi_lm_fit starts each solve.
 * The reference starts every solve cold: an ionisation-only quadratic for n_e and a halving loop to
 * 1e-2 (atmos_chm.cc:129-171), then Newton to relative defects below 1e-4 -- about 20 ionisation
 * sweeps per solve, ~18 of them in the start; the march does ~215 solves per column.
 *   SNAPI_CHEM_START_CONTINUE (default): in the march, Newton from the previous solution of the
 *     same column (the next hydrostatic iterate or depth, scaled by the particle-density ratio),
 *     cold if that has not converged after 8 passes.  Same stop rule; ~2 sweeps per solve.  The
 *     march's particle densities agree with the cold start's to ~3e-8 relative (the size of the
 *     last Newton update); the record solves at the final (T, Nt) start cold as the reference's do,
 *     so records agree to ~4e-8 relative and node tangents to ~4e-5 of each field's scale (the noise
 *     the 1e-4 stop leaves in the reference's own 5 K differences).
 *   SNAPI_CHEM_START_COLD: the reference's start at every solve (its iterates, to rounding).
 * Needs a node model (snapi_eos_set); the setting lasts until changed or the next snapi_eos_set. */
#define SNAPI_CHEM_START_CONTINUE 0
#define SNAPI_CHEM_START_COLD 1
int snapi_eos_chem_start(snapi_ctx *ctx, int mode);
/* Records [npix][nd][nfield] (float) of the node vectors nodes [npix][npar] (double), the particle
 * density Nt [npix][nd] (double, may be NULL) and, if tangents != NULL, the node tangents
 * [npix][npar][nd][nfield] with central-difference steps step [npar] (NULL: the reference's 5 K,
 * 20 cm/s, 20 cm/s, 0.01 G, 1e-3 rad, 1e-3 rad; const.h:27-32).  active [npix] (may be NULL):
 * rows of pixels with active[p] == 0 are left untouched.  pix_status [npix] (may be NULL): 0, or
 * a sum of 1 (a chemistry solve hit its iteration cap, as the reference then continues with the
 * last iterate), 2 (a hydrostatic step hit its cap), 4 (non-finite values). */
int snapi_build_records(snapi_ctx *ctx, int npix, const double *nodes, const int *active, float *records,
                        double *Nt, float *tangents, const double *step, int *pix_status, int mem);

/* Stokes synthesis, chi2 and its gradient with respect to the nodes, from node vectors: the work of
 * the reference's build_from_nodes + obs_stokes + obs_stokes_responses_to_nodes (atmos_pp.cc:58-248,
 * atmos_obs.cc:16-87, atmos_fit.cc:1205-1352) contracted with the weighted residual as
 * stokes_lm_fit forms J^T r (atmos_fit.cc:125-137), i.e. d chi2 / d node without the responses.
 * Per chunk of max_batch pixels: snapi_build_records of nodes [npix][npar] with tangents (the
 * reference's steps) into the context's device buffers, then snapi_adjoint on them.  obs, mask,
 * w_stokes, stokes, chi2 as snapi_adjoint; grad [npix][npar] (double) in the model's node order;
 * pix_status [npix] (may be NULL) the build's status bits.  Needs a node model (snapi_eos_set).
 * snapi_last_kernel_ms: the build's and the adjoint's device time together. */
int snapi_adjoint_nodes(snapi_ctx *ctx, int npix, const double *nodes, const float *obs, const double *w_stokes,
                        const float *mask, float *stokes, double *chi2, double *grad, int *pix_status, int mem);

/* The columns of the node vectors as the master collects them after a fit: the 12 rows of
 * atmosphere::return_as_array (atmos.cc:547-569) after build_from_nodes and compute_op_referent,
 * atmos [npix][12][nd] float64: log10 tau_500, height (x3 [nd], a host array, the caller's depth
 * grid; NULL: 0), T, gas pressure Nt k T, electron pressure n_e k T, 0, kappa at
 * airtovac(lambda_referent), |B|, v_turb, v_z, acos(B_z / |B|), atan(B_y / B_x of the TOP depth)
 * (the reference divides by the top depth's B_x).  active / pix_status as snapi_build_records. */
int snapi_build_atmos(snapi_ctx *ctx, int npix, const double *nodes, const int *active, const double *x3,
                      double *atmos, int *pix_status, int mem);

/* Records of given atmosphere columns -- the synthesis branch of the master's job, which reads an
 * atmosphere cube with atmosphere::read_spinor3d (atmos_fio.cc:79-124) and synthesises each column
 * (master/job.cc:384-409).  columns [npix][12][nd] float64 in the row layout of snapi_build_atmos:
 * T is floored at 3200 K and Nt = gas pressure / (k T) as read_spinor3d does; |B|, inclination,
 * azimuth, v_turb and v_z are taken as given; n_e, the populations and kappa are recomputed by the
 * chemistry as obs_stokes' set-up does (the pressure, n_e and kappa rows of the file are not used).
 * Needs the context's atom tables (snapi_eos_set).  pix_status [npix] (may be NULL): 0, or a sum of
 * 1 (chemistry iteration cap), 4 (non-finite values), 8 (the column's log tau row differs from the
 * context's depth grid by more than 1e-6, i.e. beyond the float32 rounding of a float32 cube; the
 * records are for the context's grid). */
int snapi_records_from_columns(snapi_ctx *ctx, int npix, const double *columns, float *records, int *pix_status,
                               int mem);

/* The whole atmosphere::stokes_lm_fit (atmos_fit.cc:18-227) of npix pixels with the node -> record
 * map on the device: the loop snapi_lm_begin; { snapi_build_records of the requested node vectors of
 * the active pixels (with the reference's tangent steps); snapi_lm_step } ...; snapi_lm_result, all
 * buffers resident on the GPU.  The context needs a node model (snapi_eos_set) whose node kinds are
 * opts->node_kind.  Outputs as snapi_lm_result; n_steps (may be NULL): LM steps taken. */
int snapi_lm_fit(snapi_ctx *ctx, int npix, const snapi_lm_opts *opts, const double *nodes0, const float *obs,
                 const double *w_stokes, const float *mask, double *nodes, double *chi2, int *iters, float *stokes,
                 int *n_steps, int mem);

/* Pinned host memory for SNAPI_MEM_HOST arguments. */
void *snapi_host_alloc(size_t bytes);
void snapi_host_free(void *p);

/* The context's CUDA stream (a cudaStream_t) and the device time of the kernels of the last
 * call, measured with CUDA events on that stream [ms]. */
void *snapi_stream(snapi_ctx *ctx);
double snapi_last_kernel_ms(const snapi_ctx *ctx);
/* Device time [ms] of one phase of the last snapi_adjoint_nodes call: 0 the node build (records and
 * tangents), 1 the adjoint (synthesis, chi2, reverse sweep, chain rule); 0 for other calls' phases. */
double snapi_last_phase_ms(const snapi_ctx *ctx, int phase);
/* Number of kernel launches of the last call. */
int snapi_last_launches(const snapi_ctx *ctx);

/* The autotuner: launch shapes picked per context and batch size by timing them.  No counterpart in
 * the reference (its loops have no launch shapes).  The shapes it chooses between compute the same
 * bits (they change which thread or CTA handles a wavelength or a pixel, never the order of a sum):
 *   the adjoint: 32, 64 or 128 wavelengths per sweep CTA (the padding of the wavelength grid to the
 *     CTA width, e.g. 201 -> 224 / 256 / 256, against the CTA's staging cost), 8, 16 or 32 pixels
 *     per opacity-adjoint tile (L2 reuse of a tile's adjoint bars across its transitions), and the
 *     reverse DELO sweep's register budget (unbounded, or 128 for more resident warps);
 *   the node build: 32, 64 or 128 threads per hydrostatic-march CTA, 64, 128 or 256 per
 *     record-chemistry CTA.
 * mode 1: the first snapi_adjoint / snapi_adjoint_nodes call with device buffers (SNAPI_MEM_DEVICE;
 * calls on host buffers use tuned shapes but do not tune) and the first node build of each
 * batch-size bucket (the next power of two >= npix) runs every candidate once on its own inputs,
 * timed by CUDA events, keeps the fastest and then computes the call with it; later calls of the
 * bucket reuse it.  cache_path (may be NULL): a text file of earlier choices, read now (entries for
 * this device and problem shape) and appended to after each tuning, so that other processes skip
 * the trials.  mode 0 (the default): the compiled shapes (64 wavelengths, 16-pixel tiles, 64 and 64
 * threads).  Switching the mode forgets earlier choices. */
int snapi_autotune(snapi_ctx *ctx, int mode, const char *cache_path);
/* The shapes in use for a batch of npix pixels: cfg[5] = {wavelengths per sweep CTA, pixels per
 * opacity tile, march CTA threads, record-chemistry CTA threads, reverse sweep at 128 registers}.  Returns a bit set: 1 the adjoint
 * shapes were tuned, 2 the build's were (0: the compiled defaults). */
int snapi_tuned_config(const snapi_ctx *ctx, int npix, int *cfg);

/* The measured fused multiply-add peak of GPU `device` in TFLOP/s (fp64 = 0: FP32, 1: FP64): a
 * kernel of independent FMA chains filling every SM, timed by CUDA events (best of three launches
 * after a warm-up).  The denominator of the benchmark's compute rooflines; no counterpart in the
 * reference. */
int snapi_fma_peak(int device, int fp64, double *tflops);

/* snapi_adjoint for callers that cannot allocate device memory: applications whose GPU memory
 * is owned by another allocator (a framework pool with a fixed budget) and loops that must not
 * take the device-wide synchronisation and latency of cudaMalloc / cudaFree.  It has no
 * counterpart in the reference (whose per-pixel CPU loops have no device memory at all).
 *
 * No context and no allocation: every work buffer lives in one static device array of
 * SNAPI_STATIC_SCRATCH_BYTES (64 MiB) that each GPU loading this library holds until the process
 * exits.  All array arguments are device pointers on `device`; w_stokes is a host array [4];
 * `stream` is a cudaStream_t created on `device` (NULL = default stream; a stream of another
 * device is rejected with SNAPI_EINVAL).  Every call waits for its stream (cudaStreamSynchronize)
 * and returns when the results are in place.  Pixels are processed in batches that fit the static
 * array; a problem whose single pixel does not fit (at nd = 80 and 201 wavelengths one pixel needs
 * ~1.4 MB) is rejected with SNAPI_EINVAL.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress).  Every call synchronizes its stream, so none can be captured
 * into a CUDA graph.  Calls share the array and the kernels' shared-memory limits: calls that
 * overlap on the GPU race.
 * On error, snapi_noalloc_last_error() (per host thread) describes it. */
#define SNAPI_STATIC_SCRATCH_BYTES (64u << 20)
int snapi_adjoint_noalloc(const snapi_problem *prob, int device, void *stream, int npix, const float *records,
                          const float *obs, const double *w_stokes, const float *mask, int npar,
                          const float *tangents, float *stokes, double *chi2, double *grad);
const char *snapi_noalloc_last_error(void);

/* ---- ANA ".f0" files: the observed Stokes cubes, model cubes and results ------------------------
 * Replaces ana_fzread (cmlib/ana_read.cc:74-178), ana_fzwrite (cmlib/ana_write.cc:129-175) and the
 * streaming ana_file (cmlib/ana_write.cc:177-239).  Elements are stored with dim[0] varying
 * fastest: a cube the reference writes from an array a[x1][x2][x3][x4] has dim = {n4, n3, n2, n1}.
 * Uncompressed files only (compressed ones hold integer images, never a cube of this path).
 * Errors return SNAPI_EINVAL; snapi_f0_error() (per host thread) says why. */
#define SNAPI_F0_INT8 0
#define SNAPI_F0_INT16 1
#define SNAPI_F0_INT32 2
#define SNAPI_F0_FLOAT32 3
#define SNAPI_F0_FLOAT64 4
#define SNAPI_F0_INT64 5
#define SNAPI_F0_MAX_DIM 16

typedef struct {
  int type;                      /* SNAPI_F0_* of the stored elements */
  int ndim;
  long long dim[SNAPI_F0_MAX_DIM];  /* dim[0] varies fastest */
  long long nelem;
  long long data_offset;         /* bytes before the first element (512 per header block) */
  int nhb;                       /* header blocks */
  int swap;                      /* 1: elements stored in the other byte order (swapped on read) */
  int compressed;                /* 1: anacrunch-compressed (not readable here) */
  int reversed_synch;            /* 1: byte-reversed synch pattern (the reference warns, flips swap) */
  char header[15 * 256 + 1];     /* text of all header blocks, concatenated */
} snapi_f0_info;

int snapi_f0_stat(const char *path, snapi_f0_info *info);
/* Elements [first, first + count) into out, converted to out_type (the file's own type,
 * SNAPI_F0_FLOAT32 or SNAPI_F0_FLOAT64), native byte order. */
int snapi_f0_read(const char *path, long long first, long long count, void *out, int out_type);
/* The file ana_fzwrite writes: header (NULL: none; up to 15 blocks of 255 characters) and data. */
int snapi_f0_write(const char *path, const void *data, int type, int ndim, const long long *dim, const char *header);
/* Streaming writer: the same header, then element ranges in any order from any thread;
 * snapi_f0_close reports a file whose elements were not all written (as ana_file does). */
typedef struct snapi_f0_file snapi_f0_file;
snapi_f0_file *snapi_f0_create(const char *path, int type, int ndim, const long long *dim, const char *header,
                               int *status);
int snapi_f0_write_at(snapi_f0_file *f, long long first, long long count, const void *data);
int snapi_f0_close(snapi_f0_file *f);
const char *snapi_f0_error(void);

/* ---- Cube inversion: the master's invert job with every pixel fitted on the GPU ----------------
 * Replaces the inversion branch of job_class (master/job.cc:304-379: read the cube, scale it by
 * synth_qs / obs_qs, cut the subfield and wavelength window, one islave stokes_lm_fit per pixel)
 * and its result collection (master/job.cc:570-597).  The cube is streamed: a reader thread fetches
 * the next batch of pixels from the file while the GPU fits the current one (snapi_lm_fit) and a
 * writer thread stores the previous one.
 *   observed cube  dims (nl, 4, ny, nx), float32 or float64 (read_file 4-D + transpose, job.cc:308)
 *   model cube     dims (>= nx_sub, >= ny_sub, npar): node values of each pixel (job.cc:347-369),
 *                  read as float32 / float64
 *   out_nodes      inverted_nodes.f0: float32, dims (nx_sub, ny_sub, npar)        (job.cc:579)
 *   out_spectra    inverted_spectra.f0: float64, dims (nl_win, 4, ny_sub, nx_sub), the fitted
 *                  Stokes vectors (job.cc:597)
 *   out_cube       cube_to_invert.f0: float64, the scaled window of the observation (job.cc:334)
 *   out_atmos      inverted_atmos.f0: float64, dims (nd, ny_sub, nx_sub, 12), the columns of the
 *                  fitted nodes as snapi_build_atmos gives them (job.cc:555-585), built from the
 *                  returned nodes (angles polished as the reference's model is: the same columns
 *                  for one inclination and one azimuth node)
 * The context's wavelength grid is the window ll..lh of the cube's grid. */
typedef struct {
  const char *obs_path;
  int xl, xh, yl, yh, ll, lh;    /* 1-based inclusive subfield and window; xh = 0 etc.: to the end */
  double obs_qs, synth_qs;       /* the observation is multiplied by synth_qs / obs_qs (0, 0: 1) */
  const double *nodes0;          /* [npar] starting nodes of every pixel (the job's model), or NULL */
  const char *model_path;        /* or a model cube of starting nodes (NULL: nodes0) */
  const float *mask;             /* [nl of the cube] wavelength weights (observable mask), or NULL */
  const double *w_stokes;        /* [4] Stokes weights, or NULL */
  const char *out_nodes, *out_spectra, *out_cube;  /* NULL: not written */
  double *chi2;                  /* [nx_sub * ny_sub] final chi2 per pixel (x major), or NULL */
  int *iters;                    /* [nx_sub * ny_sub] iterations per pixel, or NULL */
  int chunk;                     /* pixels per GPU batch (0: 65536) */
  const char *out_atmos;         /* NULL: not written */
  const double *x3;              /* [nd] heights of the job's atmosphere for out_atmos, or NULL */
} snapi_cube_job;

typedef struct {
  long long pixels, chunks, lm_steps;
  double wall_s;                 /* the whole call */
  double fit_s;                  /* inside snapi_lm_fit (snapi_cube_synth: the GPU work of the chunks) */
  double read_wait_s;            /* waiting for the reader (reads not hidden behind the fits) */
  double write_wait_s;           /* waiting for the writer */
  long long bytes_read, bytes_written;
  double kernel_ms;              /* device time of all kernels */
  int launches;
  long long flagged;             /* snapi_cube_synth: pixels with a non-zero record status */
} snapi_cube_stats;

int snapi_cube_invert(snapi_ctx *ctx, const snapi_lm_opts *opts, const snapi_cube_job *job,
                      snapi_cube_stats *stats);

/* ---- Cube synthesis: the synthesis branch of the master's job -----------------------------------
 * Replaces master/job.cc:384-409 with an atmosphere cube read by atmosphere::read_spinor3d
 * (atmos_fio.cc:79-124): every column of the subfield synthesised (obs_stokes) and the spectra
 * written as write_file 4-D does (job.cc:595).  The cube is streamed in chunks: a reader thread
 * fetches the next chunk's rows while the GPU builds records (snapi_records_from_columns) and
 * synthesises (snapi_synth), and a writer thread stores the previous chunk's spectra.
 *   atmos cube   dims (nd, ny, nx, 12), float32 or float64: the 12 rows of snapi_build_atmos (what
 *                snapi_cube_invert writes to inverted_atmos.f0); the log tau row must be the
 *                context's depth grid and nd the context's
 *   out_spectra  float64, dims (nlambda, 4, ny_sub, nx_sub) on the context's wavelength grid
 * A subfield reaching beyond the cube is cut to it, as the job cuts nx / ny to the model's. */
typedef struct {
  const char *atmos_path;
  int xl, xh, yl, yh;            /* 1-based inclusive subfield; 0 = the cube's extent */
  const char *out_spectra;       /* NULL: not written */
  float *stokes;                 /* [nx_sub * ny_sub][nlambda][4] host copy (x major), or NULL */
  int chunk;                     /* pixels per GPU batch (0: 16384; 2048 with an NLTE atom) */
  /* An NLTE atom (all NULL: LTE populations).  As obs_stokes runs nltepops for an NLTE atom
   * (atmos_obs.cc:16-87, atmos_pop.cc:67-240), each chunk's columns get the population-independent
   * set-up (snapi_ali_setup with ctx's atom tables, T floored at 3200 K as read_spinor3d floors it),
   * the level-population iteration (snapi_ali_iter on ali, from the LTE populations, up to
   * ali_max_iter iterations to ali_tol) and the NLTE atom's line fields from those populations
   * (snapi_records_set_populations with line_level) before the synthesis.  A column whose set-up
   * chemistry was flagged (snapi_ali_setup's status) or whose populations stayed negative is
   * counted in stats->flagged and synthesised with the last populations. */
  snapi_ali_ctx *ali;
  const snapi_ali_problem *ali_prob;       /* the problem ali was created with */
  const snapi_ali_setup_tables *ali_tables;
  const int *line_level;                   /* [nlines][2], host */
  int ali_max_iter;                        /* 0: 100 */
  double ali_tol;                          /* 0: 1e-2, the reference's stop */
} snapi_cube_synth_job;

int snapi_cube_synth(snapi_ctx *ctx, const snapi_cube_synth_job *job, snapi_cube_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
