"""Shared helpers of the tests (no GPU needed)."""
import ctypes

import numpy as np

# the reference's LM scales of the node parameters (atmos_fit.cc:250-260, cmlib/const.h:35-38)
NODE_SCALE = {1: 5000.0, 2: 1e5, 3: 1e5, 4: 1000.0, 5: 1.0, 6: 1.0}
# FD steps of the oracle gradient check, per node kind (T, v_turb, v_los, B, theta, phi)
FD_STEP = {1: 0.5, 2: 10.0, 3: 10.0, 4: 0.1, 5: 1e-4, 6: 1e-4}


def node_scales(node_kind):
    return np.array([NODE_SCALE[int(k)] for k in node_kind])


def node_steps(node_kind):
    return np.array([FD_STEP[int(k)] for k in node_kind])


def oracle_grad(so, fx, p, obs, mask=None):
    lines = so.lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])
    nl = fx["lambda_air"].shape[0]
    tan = fx["tangent"][p].astype(np.float64)
    steps = node_steps(fx["node_kind"])
    g = np.zeros(tan.shape[0])
    chi = 0.0
    m = np.ones(nl) if mask is None else mask
    for q in range(tan.shape[0]):
        chi, gq = so.chi2_grad_fd(fx["lambda_air"], fx["tau500"], fx["record"][p], lines, obs, np.ones(4), m,
                                  tan[q:q + 1], steps[q])
        g[q] = gq[0]
    return chi, g


def scaled_rel_err(g, gref, node_kind):
    s = node_scales(node_kind)
    return float(np.linalg.norm((g - gref) * s) / np.linalg.norm(gref * s))


def emu_lines(so, fx):
    return so.lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])


def P(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)
