"""The master's invert job on the GPU (snapi_cube_invert): an .f0 cube streamed through the
device fit, against the reference's cube steps (the cube_to_invert.f0 its job writes, byte for
byte) and against snapi_lm_fit of the same pixels (the fitted nodes, spectra, chi2)."""
import os

import numpy as np
import pytest

from conftest import load_fixture
from helpers import node_scales

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import snapi_b200
    from snapi_b200 import build as b
    b.build_cuda()
    return snapi_b200


@pytest.fixture(scope="module")
def f0():
    return load_fixture("f0_ref")


def _setup(sb, config4):
    from snapi_b200.eos_tables import EosTables
    fx = config4
    ic = float(np.abs(fx["target"][:, :, 0]).max())
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    ctx.eos_set(EosTables(load_fixture("eos_c3")))
    return ctx


def _subfield_pixels(f0):
    """config-4 pixel of each subfield pixel (x major), and the subfield's size"""
    xl, xh, yl, yh = [int(v) for v in f0["cube_sub"][:4]]
    pix = f0["cube_pix"].reshape(4, 4)
    sel = np.array([pix[x - 1, y - 1] for x in range(xl, xh + 1) for y in range(yl, yh + 1)])
    return sel, xh - xl + 1, yh - yl + 1


def test_cube_invert_matches_lm_fit(sb, config4, f0, tmp_path):
    """float32 cube scaled by 1 / 2, 3 x 3 subfield of a 4 x 4 cube, the 201-wavelength window of
    206, starting nodes from a model cube, chunks of 4 pixels (chunks and file rows cross)."""
    fx = config4
    api = sb.api
    sub = [int(v) for v in f0["cube_sub"]]
    cube = tmp_path / "obs.f0"
    cube.write_bytes(bytes(f0["cube_f32_file"]))
    sel, nx, ny = _subfield_pixels(f0)
    kinds = fx["node_kind"]
    npar = kinds.size
    # model cube as the reference reads it: float32, element (x, y, p) at (p * ny + y) * nx + x
    n0 = fx["nodes0"][sel].astype(np.float32)
    model = np.ascontiguousarray(n0.reshape(nx, ny, npar).transpose(2, 1, 0))
    mpath = tmp_path / "model.f0"
    api.f0_write(str(mpath), model)
    nlf = int(api.f0_stat(str(cube))["dims"][0])
    mask = np.zeros(nlf, np.float32)
    mask[sub[4] - 1:sub[5]] = fx["mask"][0]
    qs = f0["cube_f32_qs"]
    opts = dict(lm_start=1e3, max_iter=10, delta=1e-3)
    ctx = _setup(sb, config4)
    out = ctx.cube_invert(str(cube), kinds, 1e-2 * node_scales(kinds), model_path=str(mpath), subfield=sub[:4],
                          window=sub[4:], obs_qs=qs[0], synth_qs=qs[1], mask=mask,
                          out_nodes=str(tmp_path / "inverted_nodes.f0"),
                          out_spectra=str(tmp_path / "inverted_spectra.f0"),
                          out_cube=str(tmp_path / "cube_to_invert.f0"), chunk=4, **opts)
    st = out["stats"]
    assert (st["pixels"], st["chunks"]) == (nx * ny, 3)
    assert st["bytes_read"] == nx * ny * 4 * nlf * 4
    assert ctx.last_launches > 0
    # the scaled window the job fitted is the reference's cube_to_invert.f0, byte for byte
    assert (tmp_path / "cube_to_invert.f0").read_bytes() == bytes(f0["cube_f32_c2i"])
    # the same pixels through snapi_lm_fit: scaling by 1 / 2 is exact, so the obs are identical
    obs = f0["cube_f32_S"].reshape(nx * ny, 4, -1).transpose(0, 2, 1).astype(np.float32)
    ref = ctx.lm_fit_device(n0.astype(np.float64), obs, kinds, 1e-2 * node_scales(kinds),
                            mask=np.tile(mask[sub[4] - 1:sub[5]], (nx * ny, 1)), **opts)
    ctx.close()
    assert np.array_equal(out["chi2"].ravel(), ref["chi2"])
    assert np.array_equal(out["iters"].ravel(), ref["iters"])
    nodes = api.f0_read(str(tmp_path / "inverted_nodes.f0"))
    assert api.f0_stat(str(tmp_path / "inverted_nodes.f0"))["dims"] == (nx, ny, npar)
    assert np.array_equal(nodes, ref["nodes"].astype(np.float32).reshape(nx, ny, npar).transpose(2, 1, 0))
    spec = api.f0_read(str(tmp_path / "inverted_spectra.f0"))
    assert spec.dtype == np.float64 and spec.shape == (nx, ny, 4, obs.shape[1])
    assert np.array_equal(spec, ref["stokes"].astype(np.float64).reshape(nx, ny, -1, 4).transpose(0, 1, 3, 2))


def test_cube_invert_atmosphere_cube(sb, config4, f0, tmp_path):
    """inverted_atmos.f0: the 12 return_as_array rows of every fitted column, dims (nd, ny, nx, 12),
    equal to snapi_build_atmos of the nodes snapi_lm_fit returns for the same pixels; heights passed
    through."""
    fx = config4
    api = sb.api
    sub = [int(v) for v in f0["cube_sub"]]
    cube = tmp_path / "obs.f0"
    cube.write_bytes(bytes(f0["cube_f32_file"]))
    sel, nx, ny = _subfield_pixels(f0)
    kinds = fx["node_kind"]
    x3 = np.linspace(1.5e8, -8e6, fx["tau500"].size)
    opts = dict(lm_start=1e3, max_iter=3, delta=1e-3)
    ctx = _setup(sb, config4)
    out = ctx.cube_invert(str(cube), kinds, 1e-2 * node_scales(kinds), nodes0=fx["nodes0"][0], subfield=sub[:4],
                          window=sub[4:], obs_qs=2.0, synth_qs=1.0, out_atmos=str(tmp_path / "inverted_atmos.f0"),
                          x3=x3, chunk=4, **opts)
    assert out["stats"]["chunks"] == 3
    h = api.f0_stat(str(tmp_path / "inverted_atmos.f0"))
    assert h["type"] == api.F0_FLOAT64 and h["dims"] == (x3.size, ny, nx, 12)
    atm = api.f0_read(str(tmp_path / "inverted_atmos.f0"))  # [12][nx][ny][nd]
    obs = f0["cube_f32_S"].reshape(nx * ny, 4, -1).transpose(0, 2, 1).astype(np.float32)
    fit = ctx.lm_fit_device(np.tile(fx["nodes0"][0], (nx * ny, 1)), obs, kinds, 1e-2 * node_scales(kinds), **opts)
    ref, st = ctx.build_atmos(fit["nodes"], x3=x3)
    ctx.close()
    assert np.all(st == 0)
    assert np.array_equal(atm.transpose(1, 2, 0, 3).reshape(nx * ny, 12, -1), ref)
    assert np.array_equal(atm[1], np.broadcast_to(x3, (nx, ny, x3.size)))


def test_cube_invert_float64_cube(sb, config4, f0, tmp_path):
    """float64 cube, scale 1.1 / 3 (not a power of two): the window the job fits is the
    reference's to the last bit; one chunk, starting nodes of the job's model for every pixel."""
    fx = config4
    sub = [int(v) for v in f0["cube_sub"]]
    cube = tmp_path / "obs64.f0"
    cube.write_bytes(bytes(f0["cube_f64_file"]))
    kinds = fx["node_kind"]
    qs = f0["cube_f64_qs"]
    ctx = _setup(sb, config4)
    out = ctx.cube_invert(str(cube), kinds, 1e-2 * node_scales(kinds), nodes0=fx["nodes0"][0], subfield=sub[:4],
                          window=sub[4:], obs_qs=qs[0], synth_qs=qs[1], out_cube=str(tmp_path / "c2i.f0"),
                          max_iter=2)
    ctx.close()
    assert (tmp_path / "c2i.f0").read_bytes() == bytes(f0["cube_f64_c2i"])
    assert out["stats"]["chunks"] == 1 and np.all(np.isfinite(out["chi2"]))


def test_cube_invert_errors(sb, config4, f0, tmp_path):
    fx = config4
    api = sb.api
    kinds = fx["node_kind"]
    sub = [int(v) for v in f0["cube_sub"]]
    cube = tmp_path / "obs.f0"
    cube.write_bytes(bytes(f0["cube_f32_file"]))
    ctx = _setup(sb, config4)
    step = 1e-2 * node_scales(kinds)
    with pytest.raises(sb.SnapiError, match="wavelengths"):   # window of 206 against a 201-point grid
        ctx.cube_invert(str(cube), kinds, step, nodes0=fx["nodes0"][0])
    with pytest.raises(sb.SnapiError, match="outside"):
        ctx.cube_invert(str(cube), kinds, step, nodes0=fx["nodes0"][0], subfield=(1, 5, 1, 4), window=sub[4:])
    bad_model = tmp_path / "m.f0"
    api.f0_write(str(bad_model), np.zeros((9, 4, 4), np.float32))
    with pytest.raises(sb.SnapiError, match="model cube"):
        ctx.cube_invert(str(cube), kinds, step, model_path=str(bad_model), window=sub[4:])
    flat = tmp_path / "flat.f0"
    api.f0_write(str(flat), np.zeros((4, 4, 206), np.float32))
    with pytest.raises(sb.SnapiError, match="dimensions"):
        ctx.cube_invert(str(flat), kinds, step, nodes0=fx["nodes0"][0])
    with pytest.raises(sb.SnapiError):
        ctx.cube_invert(str(tmp_path / "missing.f0"), kinds, step, nodes0=fx["nodes0"][0])
    with pytest.raises(sb.SnapiError, match="neither"):
        ctx.cube_invert(str(cube), kinds, step, window=sub[4:])
    ctx.close()


# ---- the synthesis branch of the job: atmosphere cubes ------------------------------------------------

def _spinor_setup(sb, config3):
    from snapi_b200.eos_tables import EosTables
    ic = float(np.abs(config3["stokes"][:, :, 0]).max())
    ctx = sb.Context.from_fixture(config3, stokes_scale=ic)
    ctx.eos_set(EosTables(load_fixture("eos_c3")))
    return ctx


def test_records_from_columns_vs_reference(sb, config3):
    """snapi_records_from_columns on the 8 eos_c3 columns in the 12-row layout (one below the
    3200 K floor) against the records and Stokes of the reference's synthesis branch (read_spinor3d,
    extract, obs_stokes)."""
    d = load_fixture("spinor_c3")
    ctx = _spinor_setup(sb, config3)
    rec, st = ctx.records_from_columns(d["columns"])
    S = ctx.synth(rec)
    ctx.close()
    assert np.all(st == 0)
    np.testing.assert_allclose(rec, d["record"], rtol=3e-7, atol=0)
    ic = d["stokes"][:, :, 0].max(axis=1)[:, None, None]
    assert (np.abs(S - d["stokes"]) / ic).max() < 1e-5


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_cube_synth_streams_the_cube(sb, config3, dtype, tmp_path):
    """snapi_cube_synth over a 4 x 2 atmosphere cube (float64 and float32 files), subfield x 2..4,
    chunks of 4 pixels that cross x rows: the spectra equal snapi_synth of snapi_records_from_columns
    of the same columns, and the file holds them as write_file 4-D does (float64 S[x][y][s][l])."""
    api = sb.api
    d = load_fixture("spinor_c3")
    cols = d["columns"].astype(dtype).astype(np.float64)
    nx, ny = 4, 2
    cube = np.ascontiguousarray(cols.reshape(nx, ny, 12, -1).transpose(2, 0, 1, 3)).astype(dtype)
    path = tmp_path / "atm.f0"
    api.f0_write(str(path), cube)
    ctx = _spinor_setup(sb, config3)
    out = ctx.cube_synth(str(path), subfield=(2, 4, 0, 0), out_spectra=str(tmp_path / "spec.f0"), chunk=4)
    rec, st = ctx.records_from_columns(cols[ny:])
    ref = ctx.synth(rec)
    ctx.close()
    s = out["stats"]
    assert (s["pixels"], s["chunks"], s["flagged"]) == (6, 2, 0)
    assert s["bytes_read"] == 6 * 12 * cols.shape[2] * np.dtype(dtype).itemsize
    assert np.array_equal(out["stokes"].reshape(6, -1, 4), ref)
    spec = api.f0_read(str(tmp_path / "spec.f0"))
    assert spec.dtype == np.float64 and spec.shape == (3, ny, 4, ref.shape[1])
    assert np.array_equal(spec, ref.astype(np.float64).reshape(3, ny, -1, 4).transpose(0, 1, 3, 2))


def test_cube_synth_errors(sb, config3, tmp_path):
    api = sb.api
    d = load_fixture("spinor_c3")
    cols = d["columns"]
    ctx = _spinor_setup(sb, config3)
    p11 = tmp_path / "p11.f0"
    api.f0_write(str(p11), np.zeros((11, 4, 2, cols.shape[2])))
    with pytest.raises(sb.SnapiError, match="12"):
        ctx.cube_synth(str(p11))
    short = tmp_path / "short.f0"
    api.f0_write(str(short), np.zeros((12, 4, 2, 40)))
    with pytest.raises(sb.SnapiError, match="depths"):
        ctx.cube_synth(str(short))
    bad = cols.copy()
    bad[5, 0] += 0.01  # a column on another depth grid
    grid = tmp_path / "grid.f0"
    api.f0_write(str(grid), np.ascontiguousarray(bad.reshape(4, 2, 12, -1).transpose(2, 0, 1, 3)))
    with pytest.raises(sb.SnapiError, match="depth grid"):
        ctx.cube_synth(str(grid))
    ctx.close()


def test_invert_then_synthesise_round_trip(sb, config4, f0, tmp_path):
    """The two branches of the job close on each other through the reference's file formats: the
    atmosphere cube the invert job writes (inverted_atmos.f0), synthesised by the synthesis job,
    gives back the fitted spectra the invert job wrote (inverted_spectra.f0), within 1e-6 I_c (the
    columns' records are rebuilt from the written pressures and angles)."""
    fx = config4
    api = sb.api
    sub = [int(v) for v in f0["cube_sub"]]
    cube = tmp_path / "obs.f0"
    cube.write_bytes(bytes(f0["cube_f32_file"]))
    kinds = fx["node_kind"]
    ctx = _setup(sb, config4)
    ctx.cube_invert(str(cube), kinds, 1e-2 * node_scales(kinds), nodes0=fx["nodes0"][0], subfield=sub[:4],
                    window=sub[4:], obs_qs=2.0, synth_qs=1.0, out_spectra=str(tmp_path / "inv_spec.f0"),
                    out_atmos=str(tmp_path / "inv_atmos.f0"), max_iter=4)
    out = ctx.cube_synth(str(tmp_path / "inv_atmos.f0"), out_spectra=str(tmp_path / "syn_spec.f0"))
    ctx.close()
    assert out["stats"]["flagged"] == 0
    a = api.f0_read(str(tmp_path / "inv_spec.f0"))
    b = api.f0_read(str(tmp_path / "syn_spec.f0"))
    assert a.shape == b.shape
    ic = np.abs(a[:, :, 0]).max()
    assert np.abs(a - b).max() / ic < 1e-6
