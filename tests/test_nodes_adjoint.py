"""snapi_adjoint_nodes: Stokes, chi2 and d chi2 / d node from node vectors, with the records and
node tangents built on the device (the work of the reference's build_from_nodes + obs_stokes +
obs_stokes_responses_to_nodes, contracted with the residual).

Checked against (a) the two-call path it fuses (snapi_build_records with tangents, then
snapi_adjoint) -- identical, it runs the same kernels; (b) host against device buffers --
identical; (c) the FP64 oracle's central-difference gradient on the reference's own records and
tangents (coherent residual), for both chemistry starts.
"""
import numpy as np
import pytest

from helpers import oracle_grad, scaled_rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import snapi_b200
    from snapi_b200 import build as b
    b.build_cuda()
    return snapi_b200


def _ctx(sb, fx, eos, start, **kw):
    from snapi_b200.eos_tables import EosTables
    ctx = sb.Context.from_fixture(fx, stokes_scale=float(fx["stokes"][:, :, 0].max()), **kw)
    ctx.eos_set(EosTables(eos))
    ctx.eos_chem_start(start)
    return ctx


@pytest.mark.parametrize("start", [0, 1])
def test_adjoint_nodes_equals_build_plus_adjoint(sb, eos3, config3, start):
    fx = config3
    nodes = np.concatenate([fx["nodes"]] * 3)  # 24 pixels in chunks of 10
    obs = np.concatenate([fx["target"]] * 3)
    ctx = _ctx(sb, fx, eos3, start, max_batch=10)
    out = ctx.adjoint_nodes(nodes, obs)
    assert np.all(out["status"] == 0)
    rec, tan, _, status = ctx.build_records(nodes, tangents=True)
    ref = ctx.adjoint(rec, obs, tan)
    ctx.close()
    np.testing.assert_array_equal(out["stokes"], ref["stokes"])
    np.testing.assert_array_equal(out["chi2"], ref["chi2"])
    np.testing.assert_array_equal(out["grad"], ref["grad"])


def test_adjoint_nodes_device_equals_host(sb, eos3, config3):
    import torch
    fx = config3
    nodes, obs = fx["nodes"], fx["target"].astype(np.float32)
    npix, npar = nodes.shape
    nl = fx["lambda_air"].shape[0]
    ctx = _ctx(sb, fx, eos3, 0)
    h = ctx.adjoint_nodes(nodes, obs)
    dev = torch.device("cuda", 0)
    d_nodes = torch.from_numpy(np.ascontiguousarray(nodes)).to(dev)
    d_obs = torch.from_numpy(np.ascontiguousarray(obs)).to(dev)
    d_st = torch.zeros(npix, nl, 4, dtype=torch.float32, device=dev)
    d_chi2 = torch.zeros(npix, dtype=torch.float64, device=dev)
    d_grad = torch.zeros(npix, npar, dtype=torch.float64, device=dev)
    d_status = torch.full((npix,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    ctx.adjoint_nodes_device(npix, d_nodes.data_ptr(), d_obs.data_ptr(), d_chi2.data_ptr(), d_grad.data_ptr(),
                             stokes_ptr=d_st.data_ptr(), status_ptr=d_status.data_ptr())
    torch.cuda.synchronize()
    assert ctx.last_kernel_ms > 0.0 and ctx.last_launches >= 7
    assert all(t > 0.0 for t in ctx.last_phase_ms)
    ctx.close()
    np.testing.assert_array_equal(d_st.cpu().numpy(), h["stokes"])
    np.testing.assert_array_equal(d_chi2.cpu().numpy(), h["chi2"])
    np.testing.assert_array_equal(d_grad.cpu().numpy(), h["grad"])
    np.testing.assert_array_equal(d_status.cpu().numpy(), 0)


@pytest.mark.parametrize("start", [0, 1])
def test_adjoint_nodes_vs_oracle_on_reference_columns(sb, oracle_lib, eos3, config3, start):
    """From the 8 config-3 node vectors: the gradient against FP64 central differences of the
    oracle synthesis along the REFERENCE's records and tangents (coherent residual 0.97 x its
    Stokes).  The device build reproduces those records to ~4e-8 and tangents to ~4e-5 of their
    scale, so the gradient agrees to the FP32 adjoint's 1e-4 plus that."""
    fx = config3
    obs = (fx["stokes"] * 0.97).astype(np.float32)
    ctx = _ctx(sb, fx, eos3, start)
    out = ctx.adjoint_nodes(fx["nodes"], obs)
    ctx.close()
    ic = float(fx["stokes"][:, :, 0].max())
    assert np.abs(out["stokes"] - fx["stokes"]).max() / ic < 1e-5
    for p in range(fx["nodes"].shape[0]):
        _, g_ref = oracle_grad(oracle_lib, fx, p, obs[p].astype(np.float64))
        assert scaled_rel_err(out["grad"][p], g_ref, fx["node_kind"]) < 1e-3


def test_fma_peak_probe(sb):
    """The roofline denominators: positive, and FP32 above FP64 on this part."""
    f32 = sb.api.fma_peak(0, fp64=False)
    f64 = sb.api.fma_peak(0, fp64=True)
    print("FMA peak: FP32 %.1f, FP64 %.1f TFLOP/s" % (f32, f64))
    assert f32 > f64 > 0.0
