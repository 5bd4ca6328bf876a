"""GPU parity: libsnapi_cuda (through its C ABI) against the FP64 oracle and the emulator."""
import ctypes

import numpy as np
import pytest

from helpers import P, emu_lines, node_scales, oracle_grad, scaled_rel_err

pytestmark = pytest.mark.gpu

IC_TOL = 1e-5  # Stokes tolerance, in units of the continuum intensity


@pytest.fixture(scope="module")
def sb():
    import snapi_b200
    from snapi_b200 import build as b
    b.build_cuda()
    return snapi_b200


def _ic(fx):
    return float(fx["stokes"][:, :, 0].max())


def _ctx(sb, fx, **kw):
    kw.setdefault("stokes_scale", _ic(fx))
    return sb.Context.from_fixture(fx, **kw)


@pytest.mark.parametrize("cfg", ["config1", "config2", "config2_720", "config3", "config5", "config5_spec"])
def test_synth_matches_oracle(sb, oracle_lib, cfg):
    import os
    from conftest import GOLDEN, load_fixture
    if not os.path.exists(os.path.join(GOLDEN, cfg + ".npz")):
        pytest.skip("fixture %s.npz not generated" % cfg)
    fx = load_fixture(cfg)
    ctx = _ctx(sb, fx)
    st = ctx.synth(fx["record"])
    assert ctx.last_launches >= 1 and ctx.last_kernel_ms > 0.0
    ctx.close()
    ic = fx["stokes"][:, :, 0].max(axis=1)[:, None, None]
    err = np.abs(st - fx["stokes"]) / ic
    assert np.all(np.isfinite(st))
    assert err.max() < IC_TOL, err.max()


def test_synth_matches_emulator(sb, emu, oracle_lib, config2):
    fx = config2
    ctx = _ctx(sb, fx)
    st = ctx.synth(fx["record"])
    ctx.close()
    lines = emu_lines(oracle_lib, fx)
    rec = np.ascontiguousarray(fx["record"], np.float32)
    npix, nd, _ = rec.shape
    nl = fx["lambda_air"].shape[0]
    out = np.zeros((npix, nl, 4), np.float32)
    emu.emu_synth(nd, nl, len(lines), P(fx["lambda_air"]), P(fx["tau500"]), 1.0, ctypes.addressof(lines), npix, P(rec),
                  P(out))
    # the device uses SFU exp/sin/cos and rounded reciprocals, the emulator libm and IEEE division
    assert np.abs(st - out).max() / _ic(fx) < 5e-6


def test_adjoint_gradient(sb, oracle_lib, config3):
    fx = config3
    n = fx["record"].shape[0]  # every pixel of the fixture
    ctx = _ctx(sb, fx)
    out = ctx.adjoint(fx["record"][:n], fx["target"][:n], fx["tangent"][:n], want_rec_grad=True)
    ctx.close()
    assert np.all(np.isfinite(out["grad"])) and np.all(np.isfinite(out["rec_grad"]))
    lines = emu_lines(oracle_lib, fx)
    s64 = oracle_lib.synth(fx["lambda_air"], fx["tau500"], fx["record"][:n], lines)
    ic = _ic(fx)
    assert np.abs(out["stokes"] - s64).max() / ic < IC_TOL
    for p in range(n):
        # (a) the adjoint is the gradient of the FP32 model: the FP64 oracle given the same
        # residuals agrees within 1e-3 (LM-scaled norm)
        _, g_same = oracle_grad(oracle_lib, fx, p, fx["target"][p] + (s64[p] - out["stokes"][p]))
        assert scaled_rel_err(out["grad"][p], g_same, fx["node_kind"]) < 1e-3
        # (b) against the FP64 model with the same noisy target: near the minimum the gradient is a
        # sum of random-sign terms that amplifies the ~1e-6 Ic FP32 forward error
        c_ref, g_ref = oracle_grad(oracle_lib, fx, p, fx["target"][p])
        assert abs(out["chi2"][p] - c_ref) < 1e-4 * c_ref
        assert scaled_rel_err(out["grad"][p], g_ref, fx["node_kind"]) < 2e-2


def test_adjoint_coherent_residual(sb, oracle_lib, config3):
    fx = config3
    obs = fx["stokes"][:2] * 0.97
    ctx = _ctx(sb, fx)
    out = ctx.adjoint(fx["record"][:2], obs, fx["tangent"][:2])
    ctx.close()
    for p in range(2):
        _, g_ref = oracle_grad(oracle_lib, fx, p, obs[p])
        assert scaled_rel_err(out["grad"][p], g_ref, fx["node_kind"]) < 1e-4


def test_adjoint_coherent_residual_pool(sb, oracle_lib):
    """The 32 reference-built columns of the benchmark pool (records and node tangents from the
    reference's build_from_nodes): adjoint gradient against FP64 central differences of the
    oracle, coherent residual (target = 0.97 x the reference's Stokes), every column."""
    from conftest import load_fixture
    fx = load_fixture("bench_pool")
    obs = (fx["stokes"] * 0.97).astype(np.float32)
    ctx = _ctx(sb, fx)
    out = ctx.adjoint(fx["record"], obs, fx["tangent"])
    ctx.close()
    worst = 0.0
    for p in range(fx["record"].shape[0]):
        _, g_ref = oracle_grad(oracle_lib, fx, p, obs[p].astype(np.float64))
        worst = max(worst, scaled_rel_err(out["grad"][p], g_ref, fx["node_kind"]))
    print("pool: worst scaled gradient error %.2e" % worst)
    assert worst < 1e-4


def test_fd_gradient_agrees_with_adjoint(sb, config3):
    """The plain FD baseline (2 npar + 1 FP32 solves) agrees with the adjoint to its own accuracy."""
    fx = config3
    obs = fx["stokes"][:4] * 0.97
    steps = np.array([5.0, 5.0, 5.0, 5.0, 2e3, 2e3, 2e3, 5.0, 5e-3, 5e-3])
    ctx = _ctx(sb, fx)
    a = ctx.adjoint(fx["record"][:4], obs, fx["tangent"][:4])
    f = ctx.fd_grad(fx["record"][:4], obs, fx["tangent"][:4], steps)
    ctx.close()
    np.testing.assert_allclose(f["chi2"], a["chi2"], rtol=1e-5)
    for p in range(4):
        assert scaled_rel_err(f["grad"][p], a["grad"][p], fx["node_kind"]) < 2e-2


def test_mask_and_stokes_weights(sb, oracle_lib, config3):
    fx = config3
    nl = fx["lambda_air"].shape[0]
    rng = np.random.default_rng(7)
    mask = (rng.uniform(size=(1, nl)) > 0.3).astype(np.float32)
    mask[0, :40] = 0.0
    ws = (1.0, 0.5, 0.5, 2.0)
    ctx = _ctx(sb, fx)
    out = ctx.adjoint(fx["record"][:1], fx["target"][:1], fx["tangent"][:1], w_stokes=ws, mask=mask)
    ctx.close()
    r = (fx["target"][0] - out["stokes"][0]) * np.array(ws)[None, :] * mask[0][:, None]
    assert abs(out["chi2"][0] - np.sum(r.astype(np.float64) ** 2)) < 1e-6 * out["chi2"][0]


def test_batches_larger_than_device_batch(sb, config2):
    fx = config2
    ctx1 = _ctx(sb, fx, max_batch=5)
    ctx2 = _ctx(sb, fx)
    a = ctx1.synth(fx["record"])
    b = ctx2.synth(fx["record"])
    ctx1.close()
    ctx2.close()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("nl", [1, 37, 64, 201])
def test_ragged_wavelength_counts(sb, oracle_lib, config1, nl):
    """Wavelength counts that are not multiples of the warp size (inactive lanes) and one
    wavelength only."""
    fx = dict(config1)
    idx = np.linspace(0, 200, nl).astype(int) if nl > 1 else np.array([116])
    fx["lambda_air"] = np.ascontiguousarray(fx["lambda_air"][idx])
    ctx = _ctx(sb, fx)
    st = ctx.synth(fx["record"])
    ctx.close()
    lines = emu_lines(oracle_lib, fx)
    ref = oracle_lib.synth(fx["lambda_air"], fx["tau500"], fx["record"], lines)
    assert np.abs(st - ref).max() / _ic(config1) < IC_TOL


def test_weak_field_branch(sb, oracle_lib, config3):
    """|B| < 0.001 G: the reference zeroes both field angles (atom_rad_synthesis.cc:419-420)."""
    fx = config3
    rec = fx["record"][:1].copy()
    rec[0, :, 4] = 0.0
    ctx = _ctx(sb, fx)
    st = ctx.synth(rec)
    out = ctx.adjoint(rec, fx["target"][:1], fx["tangent"][:1])
    ctx.close()
    lines = emu_lines(oracle_lib, fx)
    ref = oracle_lib.synth(fx["lambda_air"], fx["tau500"], rec, lines)
    assert np.abs(st - ref).max() / _ic(fx) < IC_TOL
    assert np.all(np.isfinite(out["grad"]))
    assert np.abs(st[0, :, 1:]).max() < 1e-6 * _ic(fx)


def test_empty_batch_and_invalid_arguments(sb, config3):
    fx = config3
    ctx = _ctx(sb, fx)
    st = ctx.synth(np.zeros((0, fx["record"].shape[1], fx["record"].shape[2]), np.float32))
    assert st.shape[0] == 0
    with pytest.raises(ValueError):
        ctx.synth(fx["record"][:, :10])
    lib = sb.lib()
    rc = lib.snapi_synth(ctypes.c_void_p(ctx._ctx), -1, None, None, 0)
    assert rc == -1
    rc = lib.snapi_adjoint(ctypes.c_void_p(ctx._ctx), 1, None, None, None, None, 0, None, None, None, None, None, 0)
    assert rc == -1
    ctx.close()
    bad = dict(fx)
    bad["tau500"] = fx["tau500"][::-1].copy()
    with pytest.raises(sb.SnapiError):
        sb.Context.from_fixture(bad, stokes_scale=1.0)
    with pytest.raises(sb.SnapiError):
        sb.Context.from_fixture(fx, stokes_scale=1.0, mu=0.0)


def test_device_pointer_api(sb, config3):
    import torch
    fx = config3
    n = 3
    ctx = _ctx(sb, fx)
    ref = ctx.adjoint(fx["record"][:n], fx["target"][:n], fx["tangent"][:n])
    dev = torch.device("cuda:0")
    rec = torch.tensor(fx["record"][:n], dtype=torch.float32, device=dev)
    obs = torch.tensor(fx["target"][:n], dtype=torch.float32, device=dev)
    tan = torch.tensor(fx["tangent"][:n], dtype=torch.float32, device=dev)
    chi2 = torch.zeros(n, dtype=torch.float64, device=dev)
    grad = torch.zeros(n, 10, dtype=torch.float64, device=dev)
    st = torch.zeros(n, fx["lambda_air"].shape[0], 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    ctx.adjoint_device(n, rec.data_ptr(), obs.data_ptr(), 10, tan.data_ptr(), chi2.data_ptr(), grad.data_ptr(),
                       stokes_ptr=st.data_ptr())
    ctx.close()
    np.testing.assert_allclose(chi2.cpu().numpy(), ref["chi2"], rtol=1e-12)
    # equal up to the order of the shared-memory float atomics of the reduction
    np.testing.assert_allclose(grad.cpu().numpy(), ref["grad"], rtol=1e-5, atol=1e-6 * np.abs(ref["grad"]).max())
    assert np.array_equal(st.cpu().numpy(), ref["stokes"])


def test_size_independent_properties_at_scale(sb, config3):
    """Full-size batch (64x64 pixels built from the fixture columns): finite outputs, identical
    results for identical pixels, and linearity of the gradient in the tangents."""
    fx = config3
    npix = 4096
    idx = np.arange(npix) % fx["record"].shape[0]
    rec = fx["record"][idx]
    obs = fx["target"][idx]
    tan = fx["tangent"][idx]
    ctx = _ctx(sb, fx)
    out = ctx.adjoint(rec, obs, tan)
    out2 = ctx.adjoint(rec[:8], obs[:8], 2.0 * tan[:8])
    ctx.close()
    assert np.all(np.isfinite(out["grad"])) and np.all(np.isfinite(out["stokes"]))
    k = fx["record"].shape[0]
    gmax = np.abs(out["grad"]).max(axis=0)
    for p in range(k):
        # identical pixels: equal up to the order of the shared-memory float atomics
        same = out["grad"][idx == p]
        assert np.all(np.abs(same - same[0]) <= 1e-5 * gmax)
        st = out["stokes"][idx == p]
        assert np.all(st == st[0])
    np.testing.assert_allclose(out2["grad"], 2.0 * out["grad"][:8], rtol=1e-6,
                               atol=1e-6 * np.abs(out["grad"][:8]).max())


def test_responses_match_oracle_and_reference(sb, oracle_lib, config3):
    """dStokes/dnode: the device central differences against the FP64 oracle's central differences
    with the same steps, and against the reference's own responses_to_nodes output."""
    fx = config3
    n = 3
    kinds = fx["node_kind"]
    steps = 1e-2 * node_scales(kinds)
    ctx = _ctx(sb, fx)
    st, ds = ctx.responses(fx["record"][:n], fx["tangent"][:n], steps)
    ctx.close()
    lines = emu_lines(oracle_lib, fx)
    ic = _ic(fx)
    assert np.abs(st - fx["stokes"][:n]).max() / ic < IC_TOL
    for p in range(n):
        tan = fx["tangent"][p].astype(np.float64) * steps[:, None, None]
        ref = oracle_lib.stokes_jvp_fd(fx["lambda_air"], fx["tau500"], fx["record"][p], lines, tan, 1.0)
        ref /= steps[:, None, None]
        for q in range(ref.shape[0]):
            scale = np.abs(ref[q]).max()
            # FP32 solves differenced over a 1e-2 node step: a few ulp of I / (2 h |dS/dnode|)
            assert np.abs(ds[p, q] - ref[q]).max() < 5e-3 * scale, (p, q)
            # the reference's semi-analytic responses differ from central differences by up to ~5 %
            # (inclination nodes; 0.1-1 % elsewhere)
            rr = fx["responses"][p, q]
            assert np.abs(ds[p, q] - rr).max() < 8e-2 * np.abs(rr).max(), (p, q)


def test_packed_tangents_match_dense(sb, config3):
    """snapi_adjoint_packed (only the record fields each node touches) gives the dense result."""
    fx = config3
    obs = fx["target"]
    tan = fx["tangent"]
    fm = sb.tangent_field_mask(tan)
    assert sum(bin(int(m)).count("1") for m in fm) < tan.shape[1] * tan.shape[3]
    ptan = sb.pack_tangents(tan, fm)
    ctx = _ctx(sb, fx, max_batch=5)  # several rounds and chunks of the pipelined host path
    dense = ctx.adjoint(fx["record"], obs, tan)
    packed = ctx.adjoint_packed(fx["record"], obs, fm, ptan)
    ctx.close()
    np.testing.assert_allclose(packed["chi2"], dense["chi2"], rtol=1e-12)
    np.testing.assert_allclose(packed["grad"], dense["grad"], rtol=1e-6, atol=1e-9 * np.abs(dense["grad"]).max())
    assert np.array_equal(packed["stokes"], dense["stokes"])


@pytest.mark.parametrize("fwhm", [45, 150])
def test_spectral_broadening_matches_reference(sb, config3, fwhm):
    """snapi_spectral_broaden against the reference's convolve_spectra_with_gauss (Stokes spectra and
    node responses), away from the blue end where the reference's output is undefined."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "psf.npz"))
    lam = z["lambda_air"]
    w = float(z["width_%d" % fwhm][0])
    ctx = _ctx(sb, config3)
    out = ctx.broaden(z["spectra"], w)
    ctx.close()
    ref = z["conv_%d" % fwhm]
    inner = lam > lam[1] + 12 * w  # the reference's blue-end values (up to 1e44) leak ~11 w
    scale = np.abs(ref[:, inner]).max(axis=(1, 2))
    err = np.abs(out[:, inner] - ref[:, inner]).max(axis=(1, 2)) / scale
    assert np.all(np.isfinite(out)) and err.max() < 1e-6, err.max()


def test_tangent_responses(sb, emu, oracle_lib, config3):
    """Forward-mode responses (snapi_jacobian_mode TANGENT: k_resp_state + k_resp_jvp, the
    direction-independent W4 sums shared among the nodes' warps) against the CPU emulator of the
    same tangent sweep (checked there against FP64 differences), against the device's central
    differences, and against the reference's own semi-analytic responses; also across direction
    groups (32 nodes made of the 10 repeated: the CTAs carry at most 10 directions, so 32 nodes
    take four groups, and each node's result is bit-identical to its 10-node run)."""
    from test_emulator import emu_jvp
    fx = config3
    n = 4
    kinds = fx["node_kind"]
    rec, tan = fx["record"][:n], fx["tangent"][:n]
    ctx = _ctx(sb, fx)
    st_fd, ds_fd = ctx.responses(rec, tan, 1e-2 * node_scales(kinds))
    ctx.jacobian_mode(sb.api.JACOBIAN_TANGENT)
    st, ds = ctx.responses(rec, tan, np.ones(kinds.size))
    tan32 = np.concatenate([tan, tan, tan, tan[:, :2]], axis=1)  # 32 directions: two groups of 16
    ds32 = ctx.responses(rec, tan32, np.ones(32), want_stokes=False)
    ctx.close()
    assert np.abs(st - st_fd).max() < 1e-6 * _ic(fx)  # the state pass synthesises as k_synth does
    em = emu_jvp(emu, oracle_lib, fx, rec, tan)
    for p in range(n):
        for q in range(kinds.size):
            sc = np.abs(em[p, q]).max()
            assert np.abs(ds[p, q] - em[p, q]).max() < 1e-4 * sc, (p, q)
            # central differences with steps of 1e-2 of the node scale (50 K on a temperature
            # node) carry their truncation error: the FP64 oracle's own differences at that step
            # and at 1e-4 of the scale differ by up to 5.4e-3 (pixel 3, temperature node 1)
            assert np.abs(ds[p, q] - ds_fd[p, q]).max() < 1e-2 * sc, (p, q)
            rr = fx["responses"][p, q]
            assert np.abs(ds[p, q] - rr).max() < 8e-2 * np.abs(rr).max(), (p, q)
            for k in (q, q + 10, q + 20):
                np.testing.assert_array_equal(ds32[p, k], ds[p, q])
