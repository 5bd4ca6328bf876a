"""CPU restatement of one iteration of the reference's Levenberg-Marquardt loop (test infrastructure:
the checker of the device LM step, never the product path).

atmosphere::stokes_lm_fit (atmos/atmos_fit.cc:92-178) for one pixel, given the Stokes vector S and the
node responses dS/dnode the iteration takes at the current model:

  scale_rf            J[4 l + s][i] = dS_{s,l}/dnode_i * scale(kind_i) * ws_s * mask_l   (:250-259)
  calc_residual       r[4 l + s] = (S_fit - S)_{s,l} * ws_s * mask_l                      (:229-237)
  normal equations    J^T J, J^T r; the diagonal times (lm + 1)                           (:128-140)
  solve_svd           singular values below 1e-6 of the largest dropped; the matrix is
                      symmetric positive semi-definite, so its eigen-decomposition gives the same
                      solution (singular values = |eigenvalues|)                          (:143)
  scale_corrections   correction_i * scale(kind_i)                                        (:262-269)
  correct + bracket   nodes + correction, T / v_turb / v_los / B clipped to the model's
                      limits (atmos_model.cc:12-19, 901-977); angles unbounded
  accept              chi2(trial) < chi2(current): lm / sqrt(10) (floor 1e-5), else lm * sqrt(10)
                      (:41, 162-177)

The reference forms S (and J) with obs_stokes_responses_to_nodes and judges the trial with
forward_evaluate (the obs_stokes synthesis); the two syntheses differ by up to ~1e-3 I_c on the
config-4 pixels, so a restatement fed the obs_stokes spectrum takes steps up to ~3e-3 of their size
away from the reference's.
"""
import numpy as np

# scale, lower, upper per node kind (1 T, 2 v_turb, 3 v_los, 4 B, 5 inclination, 6 azimuth):
# cmlib/const.h:35-38, atmos/atmos_model.cc:12-19
NODE_LIMITS = {1: (5000.0, 3400.0, 12000.0), 2: (1e5, 1e2, 15e5), 3: (1e5, -15e5, 15e5),
               4: (1000.0, 1.0, 1e4), 5: (1.0, -np.inf, np.inf), 6: (1.0, -np.inf, np.inf)}
LM_MULT = np.sqrt(10.0)
LM_FLOOR = 1e-5


def _consts(kinds):
    c = np.array([NODE_LIMITS[int(k)] for k in kinds])
    return c[:, 0], c[:, 1], c[:, 2]


def bracket(nodes, kinds):
    _, lo, hi = _consts(kinds)
    return np.clip(nodes, lo, hi)


def chi2(target, S, mask, ws=(1.0, 1.0, 1.0, 1.0)):
    """calc_chisq (atmos_fit.cc:239-247): target, S [nlambda, 4]; mask [nlambda]."""
    r = (np.asarray(target, np.float64) - S) * np.asarray(ws)[None, :] * np.asarray(mask, np.float64)[:, None]
    return float((r * r).sum())


def trial(nodes, resp, S, target, mask, kinds, lm, ws=(1.0, 1.0, 1.0, 1.0), cut=1e6):
    """The bracketed trial node vector of one iteration.  nodes [npar]; resp [npar, nlambda, 4];
    S, target [nlambda, 4]; mask [nlambda]."""
    scale, _, _ = _consts(kinds)
    w = np.asarray(ws, np.float64)[None, :] * np.asarray(mask, np.float64)[:, None]  # [nlambda, 4]
    J = (np.asarray(resp, np.float64) * scale[:, None, None] * w[None]).reshape(len(kinds), -1).T
    r = ((np.asarray(target, np.float64) - np.asarray(S, np.float64)) * w).ravel()
    A = J.T @ J
    b = J.T @ r
    A[np.diag_indices_from(A)] *= lm + 1.0
    ev, V = np.linalg.eigh(A)
    wmax = np.abs(ev).max()
    keep = (np.abs(ev) > 0.0) & (wmax / np.maximum(np.abs(ev), 1e-300) <= cut)
    corr = V @ np.where(keep, (V.T @ b) / np.where(keep, ev, 1.0), 0.0)
    return bracket(np.asarray(nodes, np.float64) + corr * scale, kinds)


def update_lm(lm, accepted):
    return max(lm / LM_MULT, LM_FLOOR) if accepted else lm * LM_MULT
