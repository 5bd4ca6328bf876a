"""The oracle (FP64 C restatement) pinned against the compiled reference's outputs.

The golden fixtures were produced by the reference itself (oracle/_ref/snapi_ref_dump, generated
by tests/golden/make_golden.py): the column record after build_from_nodes, the reference's
normalised opacity at 7 wavelengths and its obs_stokes Stokes vectors."""
import numpy as np
import pytest


def _lines(so, fx):
    return so.lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])


def test_opacity_matches_reference(oracle_lib, config1):
    so, fx = oracle_lib, config1
    lines = _lines(so, fx)
    lam = fx["lambda_air"]
    lv = np.array([so.airtovac(x) for x in lam])
    lmid = 0.5 * (lv[0] + lv[-1])
    rec = fx["record"][0]
    worst = 0.0
    for i, l in enumerate(fx["probe_l"].astype(int)):
        for k in range(rec.shape[0]):
            op, em = so.opacity(rec[k], lines, lv[l], lmid)
            ref = fx["opacity_probe"][i, k]
            got = np.concatenate([op.ravel(), em])
            scale = np.concatenate([np.full(16, abs(ref[0])), np.full(4, abs(ref[16]))])
            worst = max(worst, float(np.max(np.abs(got - ref) / scale)))
    assert worst < 1e-12


def _stokes_err(so, fx):
    lines = _lines(so, fx)
    S = so.synth(fx["lambda_air"], fx["tau500"], fx["record"], lines)
    ic = fx["stokes"][:, :, 0].max(axis=1)[:, None, None]
    return float(np.max(np.abs(S - fx["stokes"]) / ic))


def test_stokes_config1(oracle_lib, config1):
    assert _stokes_err(oracle_lib, config1) < 1e-12


def test_stokes_config2(oracle_lib, config2):
    assert _stokes_err(oracle_lib, config2) < 1e-12


def test_stokes_config3(oracle_lib, config3):
    assert _stokes_err(oracle_lib, config3) < 1e-12


def test_stokes_config2_subset(oracle_lib):
    """Config 2's parity subset (64 corner pixels + 1 % of the seeded 256 x 256 cube): the oracle on
    12 of its pixels against the reference's Stokes.  The fixture stores the records in float32
    (what the device takes), so the bound is that rounding's effect, not the FP64 restatement's."""
    import os
    from conftest import GOLDEN, load_fixture
    if not os.path.exists(os.path.join(GOLDEN, "config2_720.npz")):
        pytest.skip("fixture config2_720.npz not generated")
    fx = load_fixture("config2_720")
    assert fx["record"].shape[0] == 719 and np.all(np.diff(fx["pixel_index"]) > 0)
    sel = np.linspace(0, 718, 12).astype(int)
    lines = oracle_lib.lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])
    st = oracle_lib.synth(fx["lambda_air"], fx["tau500"], fx["record"][sel].astype(np.float64), lines)
    ic = fx["stokes"][sel][:, :, 0].max(axis=1)[:, None, None]
    assert (np.abs(st - fx["stokes"][sel]) / ic).max() < 1e-6


def test_stokes_config5_nlte_ca(oracle_lib, config5):
    """Ca II 8542 window with the reference's NLTE populations in the record (10 transitions:
    Ca II H, K and the infrared triplet, the hydrogen far wings, Fe I 6301/6302)."""
    assert _stokes_err(oracle_lib, config5) < 1e-12


def _spec_fixture():
    import os
    from conftest import GOLDEN, load_fixture
    if not os.path.exists(os.path.join(GOLDEN, "config5_spec.npz")):
        pytest.skip("fixture config5_spec.npz not generated")
    return load_fixture("config5_spec")


def test_stokes_config5_spec(oracle_lib):
    """The same window at the configuration's stated settings (100 depths; populations converged
    by the patched reference with the 5-point angle set to 1e-4)."""
    fx = _spec_fixture()
    assert _stokes_err(oracle_lib, fx) < 1e-12


def test_zeeman_pattern_matches_reference(oracle_lib, config1):
    so, fx = oracle_lib, config1
    # Fe I 6301.5 (2J 4 -> 4, g 1.5 / 1.83) and 6302.5 (2J 0 -> 2, g 0 / 2.5): iron_6300.cfg
    cases = {3: (4, 4, 1.5, 1.83), 4: (0, 2, 0.0, 2.5)}
    for j, (ju2, jl2, gu, gl) in cases.items():
        L = so.zeeman_pattern(ju2, jl2, gu, gl)
        assert L.split == int(fx["line_const"][j, 5])
        for g in range(3):
            n = int(fx["line_ncomp"][j, g])
            assert L.ncomp[g] == n
            np.testing.assert_allclose([L.S[g][i] for i in range(n)], fx["line_pattern"][j, g, 0, :n], rtol=1e-14)
            np.testing.assert_allclose([L.D[g][i] for i in range(n)], fx["line_pattern"][j, g, 1, :n], rtol=1e-14,
                                       atol=1e-14)


def test_doppler_and_damping_match_reference(oracle_lib, config1):
    """The record's (T, v_turb, gc) reproduce the reference's own Doppler width and damping."""
    fx = config1
    rec = fx["record"][0]
    lc = fx["line_const"]
    k_B, c = 1.3806503E-16, 2.99792458E10
    for j in range(lc.shape[0]):
        lam0, sf, ar, mass = lc[j, :4]
        dld = np.sqrt(2.0 * k_B * rec[:, 0] / mass + rec[:, 1] ** 2) * lam0 / c
        a = sf * (ar + rec[:, 12 + 3 * j + 2]) / dld
        np.testing.assert_allclose(dld, fx["ref_dld"][0, j], rtol=1e-13)
        np.testing.assert_allclose(a, fx["ref_adamp"][0, j], rtol=1e-13)


def test_voigt_regions_continuous_enough(oracle_lib):
    """W4 region boundaries: the published method is accurate to ~1e-4, so the jump across a
    region boundary stays below that (a guard against a mistyped coefficient)."""
    so = oracle_lib
    for a in (1e-3, 0.05, 0.3):
        for xb in (15.0 - a, 5.5 - a):
            h1 = so.voigt(xb - 1e-9, a)[0]
            h2 = so.voigt(xb + 1e-9, a)[0]
            assert abs(h1 - h2) <= 2e-4 * max(abs(h1), 1e-8) + 1e-7


def test_chi2_fd_gradient_linear_in_step(oracle_lib, config3):
    """The oracle's FD gradient is stable to the step (it is the reference for the adjoint)."""
    so, fx = oracle_lib, config3
    lines = _lines(so, fx)
    nl = fx["lambda_air"].shape[0]
    tan = fx["tangent"][0, :1].astype(np.float64)
    obs = fx["stokes"][0] * 0.97
    _, g1 = so.chi2_grad_fd(fx["lambda_air"], fx["tau500"], fx["record"][0], lines, obs, np.ones(4), np.ones(nl),
                            tan, 0.5)
    _, g2 = so.chi2_grad_fd(fx["lambda_air"], fx["tau500"], fx["record"][0], lines, obs, np.ones(4), np.ones(nl),
                            tan, 0.25)
    assert abs(g1[0] - g2[0]) <= 1e-5 * abs(g1[0])


def test_ali_restatement_matches_reference_iterations(config5):
    """The numpy restatement of the NLTE iteration (oracle/ali_oracle.py) reproduces the
    reference's own first two iterations on a Ca II column."""
    import ali_oracle as ao  # oracle/ is on sys.path (conftest)
    fx = config5
    P = ao.Problem(fx)
    p = fx["ali_pop0"][0].copy()
    for it in range(2):
        p, r, neg = ao.iterate(P, fx, 0, p)
        assert not neg
        assert np.abs(p / fx["ali_pops_iter"][0, it] - 1.0).max() < 1e-9
        assert abs(r / fx["ali_relchange"][0, it] - 1.0) < 1e-9


def test_ali_restatement_matches_reference_iterations_spec():
    """As above at the stated settings (10 ray directions, 100 depths).  The fixture stores the
    background opacity / emissivity in float32 (~6e-8 relative), hence the looser bound."""
    import ali_oracle as ao
    fx = _spec_fixture()
    P = ao.Problem(fx)
    p = fx["ali_pop0"][0].copy()
    for it in range(2):
        p, r, neg = ao.iterate(P, fx, 0, p)
        assert not neg
        assert np.abs(p / fx["ali_pops_iter"][0, it] - 1.0).max() < 1e-6
        assert abs(r / fx["ali_relchange"][0, it] - 1.0) < 1e-5


def test_psf_restatement_matches_reference():
    """The numpy restatement of the Gaussian instrumental broadening (oracle/psf_oracle.py) against
    the reference's convolve_spectra_with_gauss on Stokes spectra and node responses, away from the
    blue end where the reference reads an unset interval width."""
    import os

    import psf_oracle as po
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "psf.npz"))
    lam = z["lambda_air"]
    for fw in (45, 150):
        w = float(z["width_%d" % fw][0])
        inner = lam > lam[1] + 12 * w  # the reference's blue-end values (up to 1e44) leak ~11 w
        for v in (0, 3, 9, 40, 85):
            out = po.convolve_gauss(z["spectra"][v], lam, w)
            ref = z["conv_%d" % fw][v]
            assert np.abs(out - ref)[inner].max() <= 1e-12 * np.abs(ref[inner]).max()
