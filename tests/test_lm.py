"""Batched Levenberg-Marquardt fit (snapi_lm_begin / snapi_lm_step / snapi_lm_result) against the
reference's stokes_lm_fit (config-4 pixels: uneven wavelength masks, 10 nodes, noisy targets)."""
import os

import numpy as np
import pytest

from helpers import emu_lines, node_scales
from ref_builder import LinearBuilder, RefBuilder, ref_builder_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import snapi_b200
    from snapi_b200 import build as b
    b.build_cuda()
    return snapi_b200


def _ic(fx):
    return float(np.abs(fx["target"][:, :, 0]).max())


def _delta(fx):
    """The relative chi2 stop rule the fixture's reference fits used (the configuration's 1e-4 from
    the patched reference build; 1e-3, the compiled DELTA, for fixtures without the key)."""
    return float(fx["delta"][0]) if "delta" in fx else 1e-3


def test_lm_linear_nodes_recovers_truth(sb, oracle_lib, config3):
    """Fit v_turb, v_los x2, B, inclination, azimuth (records exactly linear in them) from offset
    starting values; the fit reaches the noise level and the FP64 oracle agrees on its chi2."""
    fx = config3
    sel = np.arange(4, 10)
    truth = fx["nodes"][:, sel]
    kinds = fx["node_kind"][sel]
    offs = np.array([3e4, 3e4, 3e4, 200.0, 0.1, 0.1])
    n0 = truth + offs
    tan = fx["tangent"][:, sel]
    build = LinearBuilder(fx["record"], tan, truth)
    ic = _ic(fx)
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    out = ctx.lm_fit(n0, fx["target"], build, kinds, 1e-2 * node_scales(kinds), lm_start=1e3, max_iter=30,
                     delta=1e-3)
    ctx.close()
    npix, nl = fx["target"].shape[:2]
    noise = (1e-3 * fx["stokes"][:, :, 0].max(axis=1) / ic) ** 2 * 4 * nl
    assert np.all(out["chi2"] < 1.5 * noise), out["chi2"] / noise
    assert np.all(np.abs(out["nodes"][:, 3] - truth[:, 3]) < 20.0)  # B [G]
    # the FP64 oracle at the fitted nodes gives the same chi2
    lines = emu_lines(oracle_lib, fx)
    rec, _ = build(out["nodes"], np.ones(npix, bool))
    s64 = oracle_lib.synth(fx["lambda_air"], fx["tau500"], rec.astype(np.float64), lines)
    c64 = (((fx["target"] - s64) / ic) ** 2).sum(axis=(1, 2))
    np.testing.assert_allclose(out["chi2"], c64, rtol=2e-3)


@pytest.mark.skipif(not ref_builder_available(), reason="reference builder (oracle/_ref) not built")
def test_lm_matches_reference_fit(sb, config4):
    """Same starting nodes, targets and masks as the reference's stokes_lm_fit run (the fixture's
    stop rule: the configuration's DELTA 1e-4 from the patched reference build; start damping 1e3,
    30 iterations).  The device fit reaches a chi2 at least as low as the
    reference's (measured 3-13 % lower: the reference stops on DELTA while its semi-analytic
    responses, 0.1-5 % off the exact derivative, still slow its steps) and the same nodes within a
    fraction of their noise-limited spread."""
    fx = config4
    ic = _ic(fx)
    kinds = fx["node_kind"]
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    out = ctx.lm_fit(fx["nodes0"], fx["target"], RefBuilder(), kinds, 1e-2 * node_scales(kinds),
                     mask=fx["mask"], lm_start=1e3, max_iter=int(fx["iters"][0]), delta=_delta(fx))
    ctx.close()
    ours = out["chi2"] * ic * ic
    ref = fx["fit_chi2"]
    print("chi2 ours / reference:", ours / ref, "iterations", out["iters"], "steps", out["steps"])
    print("node differences:", np.round(out["nodes"] - fx["fit_nodes"], 3))
    assert np.all(ours / ref < 1.01) and np.all(ours / ref > 0.8)
    d = out["nodes"] - fx["fit_nodes"]
    d[:, 9] = (d[:, 9] + np.pi / 2) % np.pi - np.pi / 2  # azimuth is defined modulo pi
    assert np.all(np.abs(d[:, :4]) < 80.0)           # T nodes [K]
    assert np.all(np.abs(d[:, 4:7]) < 5e3)           # velocities [cm/s]
    assert np.all(np.abs(d[:, 7]) < 10.0)            # B [G]
    assert np.all(np.abs(d[:, 8:10]) < 0.02)         # angles [rad]


@pytest.mark.skipif(not ref_builder_available(), reason="reference builder (oracle/_ref) not built")
def test_lm_trajectory_with_reference_jacobian(sb, config4):
    """The LM iteration itself: with the reference's own responses as the Jacobian
    (snapi_lm_step_jacobian, responses from obs_stokes_responses_to_nodes at every requested node
    vector) the device's first three trial node vectors are the restated iteration's
    (oracle/lm_oracle.py, pinned to the reference's printed trial models by
    tests/test_lm_oracle.py) fed the same Jacobian and the obs_stokes spectrum, to 1e-4 of each
    step: the same residual, J^T J, damping, 1e6 condition cut (eigen-decomposition here, SVD
    there), bracketing and accept / reject.  The remaining difference is the FP32 synthesis and the
    TF32-split Gram product.  The reference itself forms its residual from the responses call's
    spectrum, which differs from obs_stokes by up to ~1e-3 I_c; its trial models are therefore
    within ~3e-3 of a step of the device's."""
    import lm_oracle as lo
    fx = config4
    sel = np.arange(4)
    ic = _ic(fx)
    kinds = fx["node_kind"]
    scale = node_scales(kinds)
    tgt, mask = fx["target"][sel], fx["mask"][sel]
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    trace = []
    rb = RefBuilder(responses=True, history=True)
    ctx.lm_fit(fx["nodes0"][sel], tgt, rb, kinds, 1e-2 * scale, jacobian=True, trace=trace, mask=mask,
               lm_start=1e3, max_iter=4, delta=_delta(fx))
    ctx.close()
    h = rb.history
    cur = trace[0].copy()
    resp, S = h[0]["responses"].copy(), h[0]["stokes"].copy()
    chi = np.array([lo.chi2(tgt[p], S[p], mask[p]) for p in sel])
    lm = np.full(sel.size, 1e3)
    for k in range(1, 4):
        exp = np.array([lo.trial(cur[p], resp[p], S[p], tgt[p], mask[p], kinds, lm[p]) for p in sel])
        step = np.linalg.norm((exp - cur) / scale, axis=1)
        rel = np.linalg.norm((trace[k] - exp) / scale, axis=1) / step
        ref_rel = np.linalg.norm((fx["trace_trial"][sel, k - 1] - trace[k]) / scale, axis=1) / step
        print("iteration", k, "device - restated trial / step:", rel, "  reference's trial:", ref_rel)
        assert np.all(rel < 1e-4), (k, rel)
        # accept / reject on the trial's obs_stokes spectrum, as the device and the reference judge
        St = h[k]["stokes"]
        for p in sel:
            c = lo.chi2(tgt[p], St[p], mask[p])
            acc = c < chi[p]
            lm[p] = lo.update_lm(lm[p], acc)
            if acc:
                cur[p], resp[p], S[p], chi[p] = trace[k][p], h[k]["responses"][p], St[p], c


@pytest.mark.skipif(not ref_builder_available(), reason="reference builder (oracle/_ref) not built")
def test_lm_with_spectral_broadening_matches_reference(sb, config4_psf):
    """LM with the 45 mA Gaussian instrumental profile (synthesis and responses broadened as
    stokes_lm_fit does) against the reference's fit of the same pixels.  Only pixels 0 and 1: the
    reference's broadening is undefined near the blue end (its interpolation reads an unset
    interval width), which wrecks its fits of pixels 2 and 3 whose masks reach that region."""
    fx = config4_psf
    sel = np.array([0, 1])
    w = float(fx["broadening"][0])
    mask = fx["mask"][sel]
    target = np.where(mask[:, :, None] > 0, fx["target"][sel], 0.0)  # masked samples do not count
    ic = float(np.abs(target[:, :, 0]).max())
    kinds = fx["node_kind"]
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    out = ctx.lm_fit(fx["nodes0"][sel], target, RefBuilder(), kinds, 1e-2 * node_scales(kinds), mask=mask,
                     lm_start=1e3, max_iter=int(fx["iters"][0]), delta=_delta(fx), spectral_broadening=w)
    ctx.close()
    ours = out["chi2"] * ic * ic
    ref = fx["fit_chi2"][sel]
    print("broadened fit: chi2 ours / reference", ours / ref, "iterations", out["iters"])
    assert np.all(ours / ref < 1.01) and np.all(ours / ref > 0.8)
    d = out["nodes"] - fx["fit_nodes"][sel]
    d[:, 9] = (d[:, 9] + np.pi / 2) % np.pi - np.pi / 2
    assert np.all(np.abs(d[:, :4]) < 80.0) and np.all(np.abs(d[:, 7]) < 10.0) and np.all(np.abs(d[:, 8:10]) < 0.02)


def _eos_tables():
    from conftest import load_fixture
    from snapi_b200.eos_tables import EosTables
    return EosTables(load_fixture("eos_c3"))


@pytest.mark.parametrize("jacobian", ["fd", "tangent"])
def test_lm_device_build_matches_reference_fit(sb, config4, jacobian):
    """The whole stokes_lm_fit on the GPU (snapi_lm_fit: node -> record build + LM steps, nothing
    back on the host between steps) against the reference's fit of the same config-4 pixels, with
    the tolerances of the host-builder test above; the Jacobian by central differences or by the
    forward-mode sweeps."""
    fx = config4
    ic = _ic(fx)
    kinds = fx["node_kind"]
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    ctx.eos_set(_eos_tables())
    if jacobian == "tangent":
        ctx.jacobian_mode(sb.api.JACOBIAN_TANGENT)
    out = ctx.lm_fit_device(fx["nodes0"], fx["target"], kinds, 1e-2 * node_scales(kinds), mask=fx["mask"],
                            lm_start=1e3, max_iter=int(fx["iters"][0]), delta=_delta(fx))
    ctx.close()
    ours = out["chi2"] * ic * ic
    ref = fx["fit_chi2"]
    print("device-built fit: chi2 ours / reference:", ours / ref, "iterations", out["iters"], "steps", out["steps"])
    assert np.all(ours / ref < 1.01) and np.all(ours / ref > 0.8)
    d = out["nodes"] - fx["fit_nodes"]
    d[:, 9] = (d[:, 9] + np.pi / 2) % np.pi - np.pi / 2
    assert np.all(np.abs(d[:, :4]) < 80.0)
    assert np.all(np.abs(d[:, 4:7]) < 5e3)
    assert np.all(np.abs(d[:, 7]) < 10.0)
    assert np.all(np.abs(d[:, 8:10]) < 0.02)


def test_lm_device_build_with_spectral_broadening(sb, config4_psf):
    """snapi_lm_fit with the 45 mA instrumental profile against the reference's broadened fit
    (pixels 0 and 1, as the host-builder test)."""
    fx = config4_psf
    sel = np.array([0, 1])
    w = float(fx["broadening"][0])
    mask = fx["mask"][sel]
    target = np.where(mask[:, :, None] > 0, fx["target"][sel], 0.0)
    ic = float(np.abs(target[:, :, 0]).max())
    kinds = fx["node_kind"]
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    ctx.eos_set(_eos_tables())
    out = ctx.lm_fit_device(fx["nodes0"][sel], target, kinds, 1e-2 * node_scales(kinds), mask=mask, lm_start=1e3,
                            max_iter=int(fx["iters"][0]), delta=_delta(fx), spectral_broadening=w)
    ctx.close()
    ours = out["chi2"] * ic * ic
    ref = fx["fit_chi2"][sel]
    print("device-built broadened fit: chi2 ours / reference", ours / ref, "iterations", out["iters"])
    assert np.all(ours / ref < 1.01) and np.all(ours / ref > 0.8)
    d = out["nodes"] - fx["fit_nodes"][sel]
    d[:, 9] = (d[:, 9] + np.pi / 2) % np.pi - np.pi / 2
    assert np.all(np.abs(d[:, :4]) < 80.0) and np.all(np.abs(d[:, 7]) < 10.0) and np.all(np.abs(d[:, 8:10]) < 0.02)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "golden", "config4_256.npz")),
                    reason="256-pixel reference fit fixture not generated")
def test_lm_device_build_256_pixels_vs_reference(sb):
    """The whole fit on the device for 256 config-4 pixels (seed 404: uneven masks, noisy targets,
    offset starting nodes) against the reference's stokes_lm_fit of the same pixels (the fixture's
    stop rule -- the configuration's DELTA 1e-4 from the patched reference build --, start damping
    1e3, 30 iterations).  Compared as distributions: the reference's semi-analytic responses and our
    finite-difference Jacobian can take a pixel to different local minima.  The worst pixels are
    printed with their node differences (the record for explaining them)."""
    from conftest import load_fixture
    fx = load_fixture("config4_256")
    ic = _ic(fx)
    kinds = fx["node_kind"]
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    ctx.eos_set(_eos_tables())
    out = ctx.lm_fit_device(fx["nodes0"], fx["target"], kinds, 1e-2 * node_scales(kinds), mask=fx["mask"],
                            lm_start=1e3, max_iter=int(fx["iters"][0]), delta=_delta(fx))
    ctx.close()
    ratio = out["chi2"] * ic * ic / fx["fit_chi2"]
    d = out["nodes"] - fx["fit_nodes"]
    d[:, 9] = (d[:, 9] + np.pi / 2) % np.pi - np.pi / 2
    dT = np.abs(d[:, :4]).max(axis=1)
    dB = np.abs(d[:, 7])
    dang = np.abs(d[:, 8:10]).max(axis=1)
    print("256 pixels: chi2 ours / reference: median %.3f, 5/95 %% %.3f / %.3f, max %.3f" % (
        np.median(ratio), np.percentile(ratio, 5), np.percentile(ratio, 95), ratio.max()))
    print("  |dT| median %.1f K, 90 %% %.1f K; |dB| median %.2f G, 90 %% %.2f G; |d angle| 90 %% %.4f rad" % (
        np.median(dT), np.percentile(dT, 90), np.median(dB), np.percentile(dB, 90), np.percentile(dang, 90)))
    for i in np.argsort(ratio)[::-1][:5]:
        print("  pixel %3d: chi2 ratio %.3f, iterations %d, node differences %s" % (
            i, ratio[i], out["iters"][i], np.array2string(d[i], precision=3, max_line_width=200)))
    assert np.median(ratio) <= 1.0
    assert np.mean(ratio < 1.05) >= 0.95
    assert np.mean(dT < 80.0) >= 0.9 and np.mean(dB < 10.0) >= 0.9 and np.mean(dang < 0.02) >= 0.9


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "golden", "config4_256.npz")),
                    reason="256-pixel reference fit fixture not generated")
def test_lm_256_outliers_are_the_iteration_cap(sb):
    """The 256-pixel comparison's worst pixels (20: chi2 13.7x the reference's after 30 iterations,
    18: 4.1x) are not a model difference: at the reference's fitted nodes the device's chi2 is the
    reference's, and with 100 iterations the device's fit ends well below the reference's chi2 --
    the reference's 30-iteration result is not a minimum either (both fits are still descending
    slowly when the iteration cap stops them, along different paths)."""
    from conftest import load_fixture
    fx = load_fixture("config4_256")
    ic = _ic(fx)
    kinds = fx["node_kind"]
    sel = np.array([20, 18])
    tgt, mask = fx["target"][sel], fx["mask"][sel]
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    ctx.eos_set(_eos_tables())
    rec, _, _, st = ctx.build_records(fx["fit_nodes"][sel], tangents=False)
    r = (tgt - ctx.synth(rec)) * mask[:, :, None]
    at_ref = (r * r).sum(axis=(1, 2)) / fx["fit_chi2"][sel]
    out = ctx.lm_fit_device(fx["nodes0"][sel], tgt, kinds, 1e-2 * node_scales(kinds), mask=mask, lm_start=1e3,
                            max_iter=100, delta=_delta(fx))
    ctx.close()
    long_fit = out["chi2"] * ic * ic / fx["fit_chi2"][sel]
    print("chi2 at the reference's nodes / reference's:", at_ref, " 100-iteration fit / reference's:", long_fit,
          "iterations", out["iters"])
    assert np.all(np.abs(at_ref - 1.0) < 1e-2)
    assert np.all(long_fit < 0.5)
