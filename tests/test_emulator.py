"""The kernels' FP32 math, run on the CPU by the emulator (tests/emu/snapi_emu.cc compiles the
same snapi_core.cuh / snapi_sweep.cuh), against the FP64 oracle."""
import ctypes

import numpy as np
import pytest

from helpers import P, emu_lines, oracle_grad, scaled_rel_err


def _emu_synth(E, so, fx, rec):
    lines = emu_lines(so, fx)
    rec = np.ascontiguousarray(rec, np.float32)
    npix, nd, _ = rec.shape
    nl = fx["lambda_air"].shape[0]
    out = np.zeros((npix, nl, 4), np.float32)
    E.emu_synth(nd, nl, len(lines), P(fx["lambda_air"]), P(fx["tau500"]), 1.0, ctypes.addressof(lines), npix, P(rec),
                P(out))
    return out


def _emu_adjoint(E, so, fx, rec, obs, tan, scale, mask=None):
    lines = emu_lines(so, fx)
    rec = np.ascontiguousarray(rec, np.float32)
    npix, nd, nf = rec.shape
    nl = fx["lambda_air"].shape[0]
    npar = tan.shape[1]
    obs32 = np.ascontiguousarray(obs, np.float32)
    tan32 = np.ascontiguousarray(tan, np.float32)
    m32 = None if mask is None else np.ascontiguousarray(mask, np.float32)
    st = np.zeros((npix, nl, 4), np.float32)
    chi = np.zeros(npix)
    g = np.zeros((npix, npar))
    rg = np.zeros((npix, nd, nf))
    E.emu_adjoint(nd, nl, len(lines), P(fx["lambda_air"]), P(fx["tau500"]), 1.0, ctypes.addressof(lines), scale, npix,
                  P(rec), P(obs32), P(np.ones(4)), P(m32), npar, P(tan32), P(st), P(chi), P(g), P(rg))
    return st, chi, g, rg


@pytest.mark.parametrize("cfg", ["config1", "config2", "config3"])
def test_emulated_synthesis_within_1e5_ic(emu, oracle_lib, cfg, request):
    fx = request.getfixturevalue(cfg)
    out = _emu_synth(emu, oracle_lib, fx, fx["record"])
    ic = fx["stokes"][:, :, 0].max(axis=1)[:, None, None]
    err = np.abs(out - fx["stokes"]) / ic
    assert err.max() < 1e-5, err.max()
    assert np.median(err[..., 0]) < 1e-6


def test_voigt_derivatives(emu, oracle_lib):
    rng = np.random.default_rng(0)
    so = oracle_lib

    def region(x, a):
        s = abs(x) + a
        return 1 if s >= 15 else 2 if s > 5.5 else 3 if a > 0.195 * abs(x) - 0.176 else 4

    worst = 0.0
    for _ in range(3000):
        x, a = rng.uniform(-30, 30), 10 ** rng.uniform(-3, 0)
        h, ha = 1e-6, 1e-7 * a
        r = region(x, a)
        if any(region(*q) != r for q in ((x + h, a), (x - h, a), (x, a + ha), (x, a - ha))):
            continue
        out = np.zeros(6, np.float32)
        emu.emu_voigt(x, a, out.ctypes.data)
        fd = np.array([(so.voigt(x + h, a)[0] - so.voigt(x - h, a)[0]) / (2 * h),
                       (so.voigt(x + h, a)[1] - so.voigt(x - h, a)[1]) / (2 * h),
                       (so.voigt(x, a + ha)[0] - so.voigt(x, a - ha)[0]) / (2 * ha),
                       (so.voigt(x, a + ha)[1] - so.voigt(x, a - ha)[1]) / (2 * ha)])
        worst = max(worst, float(np.max(np.abs(out[2:] - fd) / (np.abs(fd).max() + 1e-12))))
    assert worst < 1e-4, worst


def test_emulated_adjoint_coherent_residual(emu, oracle_lib, config3):
    """Residuals of one sign (obs = 0.97 S): the adjoint matches FP64 central differences."""
    fx = config3
    obs = fx["stokes"][:3] * 0.97
    ic = float(fx["stokes"][:, :, 0].max())
    _, chi, g, _ = _emu_adjoint(emu, oracle_lib, fx, fx["record"][:3], obs, fx["tangent"][:3], ic)
    for p in range(3):
        c_ref, g_ref = oracle_grad(oracle_lib, fx, p, obs[p])
        assert abs(chi[p] - c_ref) < 1e-4 * c_ref
        assert scaled_rel_err(g[p], g_ref, fx["node_kind"]) < 1e-4


def test_emulated_adjoint_noisy_target(emu, oracle_lib, config3):
    """Config 3: chi2 against a noisy target near the truth.  There the gradient is J^T r with
    residuals r of random sign, so it amplifies the ~1e-6 Ic FP32 forward error (r changes by
    ~1e-3 of itself).  Two checks: (a) the adjoint is the exact gradient of the FP32 model -- the
    oracle given the same residuals agrees within 1e-3 (LM-scaled norm); (b) against the FP64
    model with the same target, within 2e-2."""
    so, fx = oracle_lib, config3
    ic = float(fx["stokes"][:, :, 0].max())
    st, chi, g, _ = _emu_adjoint(emu, so, fx, fx["record"][:3], fx["target"][:3], fx["tangent"][:3], ic)
    lines = emu_lines(so, fx)
    s64 = so.synth(fx["lambda_air"], fx["tau500"], fx["record"][:3], lines)
    for p in range(3):
        _, g_same = oracle_grad(so, fx, p, fx["target"][p] + (s64[p] - st[p]))
        assert scaled_rel_err(g[p], g_same, fx["node_kind"]) < 1e-3
        c_ref, g_ref = oracle_grad(so, fx, p, fx["target"][p])
        assert abs(chi[p] - c_ref) < 1e-4 * c_ref
        assert scaled_rel_err(g[p], g_ref, fx["node_kind"]) < 2e-2


def test_emulated_record_gradient(emu, oracle_lib, config3):
    """d chi2 / d record field at a few depths against FP64 finite differences."""
    so, fx = oracle_lib, config3
    obs = fx["stokes"][:1] * 0.97
    ic = float(fx["stokes"][:, :, 0].max())
    _, _, _, rg = _emu_adjoint(emu, so, fx, fx["record"][:1], obs, fx["tangent"][:1], ic)
    lines = emu_lines(so, fx)
    rec = fx["record"][0]
    nd, nf = rec.shape
    nl = fx["lambda_air"].shape[0]
    # fields with a non-negligible influence at these depths
    for k in (40, 55, 62):
        for f in (0, 1, 3, 4, 7, 8, 9, 21, 23, 24, 26):
            h = 1e-4 * abs(rec[k, f]) if rec[k, f] != 0 else 1e-3
            t = np.zeros((1, nd, nf))
            t[0, k, f] = 1.0
            _, gq = so.chi2_grad_fd(fx["lambda_air"], fx["tau500"], rec, lines, obs[0], np.ones(4), np.ones(nl), t, h)
            assert abs(rg[0, k, f] - gq[0]) <= 1e-3 * abs(gq[0]) + 1e-30, (k, f, rg[0, k, f], gq[0])


def emu_jvp(emu, oracle_lib, fx, rec, tan):
    lines = emu_lines(oracle_lib, fx)
    rec = np.ascontiguousarray(rec, np.float32)
    tan = np.ascontiguousarray(tan, np.float32)
    npix, npar = tan.shape[0], tan.shape[1]
    nd, nl = fx["tau500"].shape[0], fx["lambda_air"].shape[0]
    out = np.zeros((npix, npar, nl, 4), np.float32)
    emu.emu_jvp(nd, nl, len(lines), P(fx["lambda_air"]), P(fx["tau500"]), 1.0, ctypes.addressof(lines), npix, P(rec),
                npar, P(tan), P(out))
    return out


# central-difference steps of the FP64 check, per node kind (small: the model is smooth there)
JVP_FD_STEP = {1: 1e-2, 2: 1.0, 3: 1.0, 4: 1e-3, 5: 1e-6, 6: 1e-6}


def test_emulated_tangent_responses_vs_fp64_differences(emu, oracle_lib, config3):
    """Forward-mode responses (the tangent of the FP32 synthesis along each node tangent,
    snapi_jvp.cuh) against FP64 central differences of the oracle with small steps.  Where the
    model has a kink (a branch of the monotone optical-depth derivative or of the W4 regions
    switching inside the step) a central difference is not a derivative: those points, flagged by
    differences at two steps that disagree, are left out -- fewer than 1 % of them."""
    fx = config3
    n = 3
    out = emu_jvp(emu, oracle_lib, fx, fx["record"][:n], fx["tangent"][:n])
    lines = oracle_lib.lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])
    kinds = fx["node_kind"].astype(int)
    kinks = total = 0
    for p in range(n):
        rec = fx["record"][p].astype(np.float32).astype(np.float64)
        for q in range(kinds.size):
            t = fx["tangent"][p, q:q + 1].astype(np.float32).astype(np.float64)
            h = JVP_FD_STEP[kinds[q]]
            d1 = np.asarray(oracle_lib.stokes_jvp_fd(fx["lambda_air"], fx["tau500"], rec, lines, t, h)).reshape(-1, 4)
            d2 = np.asarray(oracle_lib.stokes_jvp_fd(fx["lambda_air"], fx["tau500"], rec, lines, t, h / 10))
            d2 = d2.reshape(-1, 4)
            sc = np.abs(d1).max()
            smooth = np.abs(d1 - d2) < 1e-5 * sc
            kinks += int((~smooth).sum())
            total += smooth.size
            err = np.abs(out[p, q] - d1)[smooth].max() / sc
            assert err < 1e-4, (p, q, err)
    assert kinks < 0.01 * total, (kinks, total)
