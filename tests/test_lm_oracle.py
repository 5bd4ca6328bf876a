"""The restated LM iteration (oracle/lm_oracle.py) pinned to the reference's own stokes_lm_fit: fed the
reference's responses and the spectrum of its responses call at each of the reference's models, it
reproduces the trial node vectors the reference printed (model::print, atmos_model.cc:712-760; fixture
trace_trial) for the first three iterations of four config-4 pixels.  CPU only: the reference's
responses come from oracle/_ref/snapi_ref_dump."""
import numpy as np
import pytest

from helpers import node_scales
from ref_builder import RefBuilder, ref_builder_available


@pytest.mark.skipif(not ref_builder_available(), reason="reference builder (oracle/_ref) not built")
def test_lm_restatement_reproduces_reference_trials(config4):
    import lm_oracle as lo
    fx = config4
    if "trace_trial" not in fx:
        pytest.skip("fixture without the reference's trial models")
    sel = np.arange(4)
    kinds = fx["node_kind"]
    scale = node_scales(kinds)
    tgt, mask = fx["target"][sel], fx["mask"][sel]
    ref = fx["trace_trial"][sel]
    rb = RefBuilder(responses=True, history=True)
    cur = lo.bracket(fx["nodes0"][sel], kinds)
    rb(cur, np.ones(sel.size, bool))
    h = rb.history[-1]
    resp, S = h["responses"].copy(), h["stokes_resp"].copy()
    # the two syntheses of the reference differ (the residual's and the judge's)
    ic = np.abs(h["stokes"][:, :, 0]).max(axis=1)
    d = np.abs(h["stokes_resp"] - h["stokes"]).max(axis=(1, 2)) / ic
    print("obs_stokes vs responses-call spectrum, max / I_c:", d)
    chi = np.array([lo.chi2(tgt[p], S[p], mask[p]) for p in sel])
    lm = np.full(sel.size, 1e3)
    for k in range(3):
        t = np.array([lo.trial(cur[p], resp[p], S[p], tgt[p], mask[p], kinds, lm[p]) for p in sel])
        step = np.linalg.norm((ref[:, k] - cur) / scale, axis=1)
        rel = np.linalg.norm((t - ref[:, k]) / scale, axis=1) / step
        print("iteration", k + 1, "restated - reference trial / step:", rel)
        if k == 0:  # the same step fed the obs_stokes spectrum instead (what the device synthesises)
            t_obs = np.array([lo.trial(cur[p], resp[p], h["stokes"][p], tgt[p], mask[p], kinds, lm[p]) for p in sel])
            print("  with the obs_stokes spectrum:", np.linalg.norm((t_obs - ref[:, k]) / scale, axis=1) / step)
        assert np.all(rel < 1e-7), (k, rel)
        # the reference judges the trial by forward_evaluate (obs_stokes) against the current metric
        rb(ref[:, k], np.ones(sel.size, bool))
        h = rb.history[-1]
        for p in sel:
            c = lo.chi2(tgt[p], h["stokes"][p], mask[p])
            acc = c < chi[p]
            lm[p] = lo.update_lm(lm[p], acc)
            if acc:  # the next iteration recomputes spectrum and responses at the accepted model
                cur[p], resp[p], S[p] = ref[p, k], h["responses"][p], h["stokes_resp"][p]
                chi[p] = lo.chi2(tgt[p], S[p], mask[p])
