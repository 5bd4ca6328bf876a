"""The autotuner (snapi_autotune): the launch shapes it picks are timed on the call's own inputs and
compute the same bits as the compiled shapes -- the adjoint (wavelengths per sweep CTA, pixels per
opacity tile), the node build (CTA sizes of the hydrostatic march and the record chemistry) and
their composition snapi_adjoint_nodes; its choices persist in a cache file that a new context
reads instead of repeating the trials.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import snapi_b200
    from snapi_b200 import build as b
    b.build_cuda()
    return snapi_b200


def _ctx(sb, fx, eos=None, **kw):
    from snapi_b200.eos_tables import EosTables
    ctx = sb.Context.from_fixture(fx, stokes_scale=float(fx["stokes"][:, :, 0].max()), **kw)
    if eos is not None:
        ctx.eos_set(EosTables(eos))
    return ctx


def _device_adjoint(ctx, rec, obs, tan):
    import torch
    dev = torch.device("cuda", 0)
    npix, npar = tan.shape[0], tan.shape[1]
    d_rec = torch.from_numpy(np.ascontiguousarray(rec, np.float32)).to(dev)
    d_obs = torch.from_numpy(np.ascontiguousarray(obs, np.float32)).to(dev)
    d_tan = torch.from_numpy(np.ascontiguousarray(tan, np.float32)).to(dev)
    d_st = torch.zeros(npix, obs.shape[1], 4, dtype=torch.float32, device=dev)
    d_chi2 = torch.zeros(npix, dtype=torch.float64, device=dev)
    d_grad = torch.zeros(npix, npar, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    ctx.adjoint_device(npix, d_rec.data_ptr(), d_obs.data_ptr(), npar, d_tan.data_ptr(), d_chi2.data_ptr(),
                       d_grad.data_ptr(), stokes_ptr=d_st.data_ptr())
    torch.cuda.synchronize()
    return d_st.cpu().numpy(), d_chi2.cpu().numpy(), d_grad.cpu().numpy()


def test_tuned_adjoint_bitwise_equal_and_cached(sb, config3, tmp_path):
    fx = config3
    idx = np.arange(64) % fx["record"].shape[0]
    rec, obs, tan = fx["record"][idx], fx["target"][idx], fx["tangent"][idx]
    base = _ctx(sb, fx)
    ref = _device_adjoint(base, rec, obs, tan)
    assert base.tuned_config(64)[1] == 0  # autotuner off: compiled shapes
    base.close()
    cache = tmp_path / "tune.txt"
    ctx = _ctx(sb, fx)
    ctx.autotune(True, cache)
    for _ in range(2):  # the first call tunes, the second reuses
        got = _device_adjoint(ctx, rec, obs, tan)
        for a, b in zip(got, ref):
            np.testing.assert_array_equal(a, b)
    cfg, bits = ctx.tuned_config(64)
    assert bits & 1 and cfg["chunk"] in (32, 64, 128) and cfg["optile"] in (8, 16, 32)
    ctx.close()
    lines = cache.read_text().splitlines()
    assert any("|adj|64|%d|%d|%d" % (cfg["chunk"], cfg["optile"], cfg["rt128"]) in ln for ln in lines)
    # a new context with the same cache knows the choice before any call
    ctx2 = _ctx(sb, fx)
    ctx2.autotune(True, cache)
    cfg2, bits2 = ctx2.tuned_config(64)
    assert bits2 & 1 and cfg2["chunk"] == cfg["chunk"] and cfg2["optile"] == cfg["optile"]
    got = _device_adjoint(ctx2, rec, obs, tan)
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)
    ctx2.close()


@pytest.mark.parametrize("chunk,optile,rt128", [(32, 8, 1), (128, 32, 0), (64, 16, 1)])
def test_every_adjoint_shape_bitwise_equal(sb, config3, tmp_path, chunk, optile, rt128):
    """Each candidate shape, forced through the cache file, gives the compiled shape's bits (the
    tuner may pick any of them)."""
    fx = config3
    idx = np.arange(24) % fx["record"].shape[0]
    rec, obs, tan = fx["record"][idx], fx["target"][idx], fx["tangent"][idx]
    base = _ctx(sb, fx)
    ref = _device_adjoint(base, rec, obs, tan)
    base.close()
    ctx = _ctx(sb, fx)
    key_probe = tmp_path / "probe.txt"
    ctx.autotune(True, key_probe)
    _device_adjoint(ctx, rec, obs, tan)  # writes this shape's key
    key = key_probe.read_text().splitlines()[0].split("|adj|")[0]
    forced = tmp_path / "forced.txt"
    forced.write_text("%s|adj|64|%d|%d|%d\n" % (key, chunk, optile, rt128))
    ctx.autotune(True, forced)
    assert ctx.tuned_config(24)[0]["chunk"] == chunk
    got = _device_adjoint(ctx, rec, obs, tan)
    ctx.close()
    for a, b in zip(got, ref):
        np.testing.assert_array_equal(a, b)


def test_tuned_node_build_and_adjoint_nodes_bitwise_equal(sb, eos3, config3):
    fx = config3
    nodes = np.concatenate([fx["nodes"]] * 4)
    obs = np.concatenate([fx["target"]] * 4)
    base = _ctx(sb, fx, eos3)
    rec0, tan0, nt0, st0 = base.build_records(nodes, tangents=True, want_nt=True)
    out0 = base.adjoint_nodes(nodes, obs)
    base.close()
    ctx = _ctx(sb, fx, eos3)
    ctx.autotune(True)
    rec, tan, nt, st = ctx.build_records(nodes, tangents=True, want_nt=True)
    cfg, bits = ctx.tuned_config(nodes.shape[0])
    assert bits & 2 and cfg["he_threads"] in (32, 64, 128) and cfg["var_threads"] in (64, 128, 256)
    for a, b in ((rec, rec0), (tan, tan0), (nt, nt0), (st, st0)):
        np.testing.assert_array_equal(a, b)
    out = ctx.adjoint_nodes(nodes, obs)
    ctx.close()
    for k in ("stokes", "chi2", "grad", "status"):
        np.testing.assert_array_equal(out[k], out0[k])
