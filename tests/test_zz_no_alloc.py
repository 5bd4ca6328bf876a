"""snapi_adjoint_noalloc: the adjoint for callers that cannot allocate device memory.

Such callers own their GPU memory through another allocator (a framework pool with a fixed
budget) or run loops that must not take the device-wide synchronisation and latency of
cudaMalloc / cudaFree.  The entry point takes only caller-owned device buffers and keeps its work
memory in one static device array.  These tests call it through the C ABI and check its results
against snapi_adjoint (the context entry point, same kernels), identical up to the tolerance the
parity tests use: two calls in a row on different pixel sets (the first larger than one
static-array chunk, the second smaller, so stale contents of the shared array would show), and a
call after a context of a smaller problem was created on the same device (the kernels'
shared-memory limit is a per-device setting both paths share).

Kept in its own file, collected last (test_zz_*), so that a failure here comes after every other
test has run; it passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(sb, fx):
    lines, n = sb.lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])
    lam = np.ascontiguousarray(fx["lambda_air"], dtype=np.float64)
    tau = np.ascontiguousarray(fx["tau500"], dtype=np.float64)
    prob = sb.api.SnapiProblem()
    prob.nd, prob.nlambda, prob.nlines = tau.shape[0], lam.shape[0], n
    prob.lambda_air = lam.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    prob.tau500 = tau.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    prob.mu = 1.0
    prob.lines = ctypes.cast(lines, ctypes.POINTER(sb.SnapiLine))
    prob.stokes_scale = float(fx["stokes"][:, :, 0].max())
    prob.max_batch = 0
    return prob, (lines, lam, tau)  # keep the arrays alive


def _lib(sb):
    lib = sb.lib()
    vp = ctypes.c_void_p
    lib.snapi_adjoint_noalloc.restype = ctypes.c_int
    lib.snapi_adjoint_noalloc.argtypes = [ctypes.POINTER(sb.api.SnapiProblem), ctypes.c_int, vp, ctypes.c_int, vp,
                                          vp, vp, vp, ctypes.c_int, vp, vp, vp, vp]
    lib.snapi_noalloc_last_error.restype = ctypes.c_char_p
    return lib


def _inputs(fx, idx):
    rec = np.ascontiguousarray(fx["record"][idx], np.float32)
    obs = np.ascontiguousarray(fx["target"][idx], np.float32)
    tan = np.ascontiguousarray(fx["tangent"][idx], np.float32)
    return rec, obs, tan


def _context_adjoint(sb, fx, rec, obs, tan):
    ctx = sb.Context.from_fixture(fx, stokes_scale=float(fx["stokes"][:, :, 0].max()))
    ref = ctx.adjoint(rec, obs, tan)
    ctx.close()
    return ref


def _noalloc(lib, prob, rec, obs, tan, nl):
    import torch

    dev = torch.device("cuda:0")
    npix, npar = rec.shape[0], tan.shape[1]
    ws = np.array([1.0, 1.0, 1.0, 1.0])
    d_rec = torch.from_numpy(rec).to(dev)
    d_obs = torch.from_numpy(obs).to(dev)
    d_tan = torch.from_numpy(tan).to(dev)
    d_st = torch.full((npix, nl, 4), float("nan"), dtype=torch.float32, device=dev)
    d_chi2 = torch.full((npix,), float("nan"), dtype=torch.float64, device=dev)
    d_grad = torch.full((npix, npar), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = lib.snapi_adjoint_noalloc(ctypes.byref(prob), 0, None, npix, d_rec.data_ptr(), d_obs.data_ptr(),
                                   ws.ctypes.data, None, npar, d_tan.data_ptr(), d_st.data_ptr(),
                                   d_chi2.data_ptr(), d_grad.data_ptr())
    assert rc == 0, lib.snapi_noalloc_last_error().decode()
    torch.cuda.synchronize()
    return {"stokes": d_st.cpu().numpy(), "chi2": d_chi2.cpu().numpy(), "grad": d_grad.cpu().numpy()}


def _check(fx, got, ref):
    ic = float(fx["stokes"][:, :, 0].max())
    assert np.abs(got["stokes"] - ref["stokes"]).max() / ic < 1e-6
    np.testing.assert_allclose(got["chi2"], ref["chi2"], rtol=1e-9)
    np.testing.assert_allclose(got["grad"], ref["grad"], rtol=1e-5, atol=1e-6 * np.abs(ref["grad"]).max())


def test_noalloc_adjoint_matches_context_adjoint(config3):
    import snapi_b200 as sb
    from snapi_b200 import build as b

    b.build_cuda()
    lib = _lib(sb)
    fx = config3
    nl = fx["lambda_air"].shape[0]
    prob, keep = _problem(sb, fx)
    npx = fx["record"].shape[0]
    # first call: 100 pixels, more than one chunk of the 64 MiB static array at nd = 80, 201
    # wavelengths; second call: 37 other pixels (a different order), fewer than one chunk
    for idx in (np.arange(100) % npx, (np.arange(37) * 5 + 3) % npx):
        rec, obs, tan = _inputs(fx, idx)
        ref = _context_adjoint(sb, fx, rec, obs, tan)
        _check(fx, _noalloc(lib, prob, rec, obs, tan, nl), ref)
    del keep


def test_noalloc_after_smaller_context(config3):
    """A context of a smaller problem (40 depths) created between two calls must not lower the
    shared-memory limit the 80-depth call needs."""
    import snapi_b200 as sb

    lib = _lib(sb)
    fx = config3
    nl = fx["lambda_air"].shape[0]
    prob, keep = _problem(sb, fx)
    rec, obs, tan = _inputs(fx, np.arange(fx["record"].shape[0]))
    ref = _context_adjoint(sb, fx, rec, obs, tan)
    _check(fx, _noalloc(lib, prob, rec, obs, tan, nl), ref)
    small = dict(fx)
    small["tau500"] = fx["tau500"][:40]
    ctx = sb.Context.from_fixture(small, stokes_scale=float(fx["stokes"][:, :, 0].max()))
    _check(fx, _noalloc(lib, prob, rec, obs, tan, nl), ref)
    ctx.close()
    del keep


def test_noalloc_rejects_oversized_problem(config3):
    """A problem whose single pixel does not fit the static array is refused with SNAPI_EINVAL."""
    import torch

    import snapi_b200 as sb

    lib = _lib(sb)
    fx = dict(config3)
    nl = 8000  # 8000 wavelengths x 400 depths: ~205 MB of forward state for one pixel
    fx["lambda_air"] = np.linspace(6.3010e-5, 6.3034e-5, nl)
    fx["tau500"] = np.logspace(-6, 1, 400)
    prob, keep = _problem(sb, fx)
    # real (small) device buffers; the size check rejects the call before any of them is used
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    rc = lib.snapi_adjoint_noalloc(ctypes.byref(prob), 0, None, 1, buf.data_ptr(), buf.data_ptr(), None, None, 0,
                                   None, None, buf.data_ptr(), None)
    assert rc == -1
    assert b"static array" in lib.snapi_noalloc_last_error()
    del keep
