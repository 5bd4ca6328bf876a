"""Node model -> column records (build_from_nodes, chemistry, hydrostatic equilibrium, record set-up).

CPU: the FP64 restatement (oracle/eos_oracle.c) against the compiled reference's own outputs
(tests/golden/eos_c1.npz, eos_c3.npz, config3.npz): the chemistry on a (T, Nt) grid, the columns
build_from_nodes leaves, the records and the node tangents.
GPU: snapi_build_records against the oracle and against the reference's records.
"""
import numpy as np
import pytest

from conftest import gpu_available, load_fixture

pytestmark_gpu = pytest.mark.skipif(not gpu_available(), reason="needs a CUDA GPU")
THERMAL = [0, 2, 7, 8, 9, 10, 11]  # + the line fields


def _tables(d):
    import eos_oracle as eo
    return eo.EosTables(d)


def _line_const(fx):
    return fx["line_const"][:, 0].copy(), fx["line_const"][:, 3].copy()


# ---- oracle pins (no GPU) ---------------------------------------------------------------------------

def test_oracle_chemistry_grid(oracle_lib, eos3):
    """chemeq + lte + opacity_continuum on 14 x 12 (T, Nt) points, 3400..20000 K, 1e11..1e18 cm^-3."""
    import eos_oracle as eo
    t = _tables(eos3)
    for i, T in enumerate(eos3["chem_T"]):
        for j, Nt in enumerate(eos3["chem_Nt"]):
            ne, nst, npop, khe, kap, passes = eo.chem(t, T, Nt)
            assert passes > 0
            assert abs(ne / eos3["chem_ne"][i, j] - 1) < 1e-12
            assert abs(khe / eos3["chem_kap_he"][i, j] - 1) < 1e-12
            assert abs(kap / eos3["chem_kap"][i, j] - 1) < 1e-12
            ref = eos3["chem_stage"][i, j]
            m = ref > 1e-200
            np.testing.assert_allclose(nst[m], ref[m], rtol=1e-11)
            ref = eos3["chem_lev"][i, j]
            m = ref > 1e-200
            np.testing.assert_allclose(npop[m], ref[m], rtol=1e-11)


@pytest.mark.parametrize("name", ["eos_c3", "eos_c1"])
def test_oracle_hydrostatic_columns(oracle_lib, name):
    """T and Nt of build_from_nodes for the config-3 node vectors (4 T nodes) and the config-1/2
    vectors (one T node per depth)."""
    import eos_oracle as eo
    d = load_fixture(name)
    t = _tables(d)
    fx = load_fixture("config3" if name == "eos_c3" else "config1")
    lam0, mass = _line_const(fx)
    for p in range(min(6, d["nodes"].shape[0])):
        T, Nt, rec, st = eo.build(t, lam0, mass, d["nodes"][p])
        assert st == 0
        np.testing.assert_allclose(T, d["he_T"][p], rtol=1e-13)
        np.testing.assert_allclose(Nt, d["he_Nt"][p], rtol=1e-11)
        np.testing.assert_allclose(rec[:, 2], d["he_ne"][p], rtol=1e-11)


@pytest.mark.parametrize("name", ["eos_c3", "eos_c1"])
def test_oracle_atmosphere_rows(oracle_lib, name):
    """The restatement's return_as_array rows against the reference's (build_from_nodes +
    compute_op_referent), for every node vector of the fixture."""
    import eos_oracle as eo
    d = load_fixture(name)
    t = _tables(d)
    ref = d["atm_arr"]
    for p in range(ref.shape[0]):
        out, st = eo.atmos(t, d["nodes"][p], x3=ref[p, 1])
        assert st == 0
        np.testing.assert_array_equal(out[[1, 5]], ref[p, [1, 5]])
        np.testing.assert_allclose(out[0], ref[p, 0], rtol=0, atol=1e-14)
        np.testing.assert_allclose(out[[2, 7, 8, 9]], ref[p, [2, 7, 8, 9]], rtol=1e-13, atol=1e-9)
        np.testing.assert_allclose(out[[3, 4, 6]], ref[p, [3, 4, 6]], rtol=1e-10)
        np.testing.assert_allclose(out[10:], ref[p, 10:], rtol=0, atol=1e-12)


def test_oracle_column_records(oracle_lib, config3):
    """Records of given atmosphere columns (the reference's synthesis branch: read_spinor3d, then
    obs_stokes' set-up) from the restatement against the reference's, including a column below the
    3200 K floor."""
    import eos_oracle as eo
    d = load_fixture("spinor_c3")
    t = _tables(load_fixture("eos_c3"))
    lam0, mass = _line_const(config3)
    for p in range(d["columns"].shape[0]):
        rec, st = eo.columns(t, lam0, mass, d["columns"][p])
        assert st == 0
        np.testing.assert_allclose(rec, d["record"][p], rtol=1e-10, atol=1e-300)


def test_oracle_records_and_tangents(oracle_lib, eos3, config3):
    """The full record (27 fields) and the node tangents of config-3 pixels against the reference's
    (the fixture stores them in float32, hence the 1e-7 tolerances)."""
    import eos_oracle as eo
    t = _tables(eos3)
    lam0, mass = _line_const(config3)
    for p in (0, 5):
        T, Nt, rec, st = eo.build(t, lam0, mass, config3["nodes"][p])
        ref = config3["record"][p].astype(np.float64)
        np.testing.assert_allclose(rec, ref, rtol=2e-7, atol=0)
        tan, st = eo.tangents(t, lam0, mass, config3["nodes"][p])
        assert st == 0
        rt = config3["tangent"][p].astype(np.float64)
        for q in range(rt.shape[0]):
            scale = np.abs(rt[q]).max(axis=0)
            # a field whose tangent is pure rounding noise in the reference (inclination w.r.t. |B|)
            # is compared against the field's own scale
            floor = np.maximum(scale, 1e-6 * np.abs(ref).max(axis=0))
            err = np.abs(tan[q] - rt[q]).max(axis=0) / floor
            assert err.max() < 1e-5, (q, err)


def test_oracle_continued_start_vs_reference(oracle_lib, eos3, config3):
    """The continued chemistry start in the hydrostatic march (the CUDA path's default), restated in
    the oracle: particle densities, records and node tangents against the reference's (which
    starts every solve cold) within the size of the reference's own last Newton update."""
    import eos_oracle as eo
    t = _tables(eos3)
    lam0, mass = _line_const(config3)
    old = eo.set_chem_start(eo.CHEM_START_CONTINUE)
    try:
        for p in range(config3["nodes"].shape[0]):
            T, Nt, rec, st = eo.build(t, lam0, mass, config3["nodes"][p])
            assert st == 0
            np.testing.assert_allclose(Nt, eos3["he_Nt"][p], rtol=TOL["continue"]["nt"])
            np.testing.assert_allclose(rec, config3["record"][p], rtol=TOL["continue"]["rec"], atol=0)
            tan, _ = eo.tangents(t, lam0, mass, config3["nodes"][p])
            ref = config3["record"][p].astype(np.float64)
            rt = config3["tangent"][p].astype(np.float64)
            for q in range(rt.shape[0]):
                floor = np.maximum(np.abs(rt[q]).max(axis=0), 1e-6 * np.abs(ref).max(axis=0))
                assert (np.abs(tan[q] - rt[q]).max(axis=0) / floor).max() < TOL["continue"]["tan"]
    finally:
        eo.set_chem_start(old)


def test_oracle_continued_start_dense_nodes(oracle_lib, eos1, config1, config2):
    """As above on the 80-temperature-node model (17 columns): Nt and records against the
    reference's build_from_nodes; the wiggly temperature profile moves the march furthest."""
    import eos_oracle as eo
    t = _tables(eos1)
    lam0, mass = _line_const(config1)
    ref = np.concatenate([config1["record"], config2["record"]]).astype(np.float64)
    old = eo.set_chem_start(eo.CHEM_START_CONTINUE)
    try:
        for p in range(eos1["nodes"].shape[0]):
            T, Nt, rec, st = eo.build(t, lam0, mass, eos1["nodes"][p])
            assert st == 0
            np.testing.assert_allclose(Nt, eos1["he_Nt"][p], rtol=TOL["continue"]["nt"])
            np.testing.assert_allclose(rec, ref[p], rtol=TOL["continue"]["rec"], atol=0)
    finally:
        eo.set_chem_start(old)


# ---- GPU ---------------------------------------------------------------------------------------------

def _gpu_ctx(fx, eos, start="cold", **kw):
    import snapi_b200 as sb
    from snapi_b200.eos_tables import EosTables
    ctx = sb.Context.from_fixture(fx, **kw)
    ctx.eos_set(EosTables(eos))
    ctx.eos_chem_start(sb.api.CHEM_START_COLD if start == "cold" else sb.api.CHEM_START_CONTINUE)
    return ctx


# Tolerances per chemistry start.  The cold start is the reference's (its iterates to rounding).
# The continued start (hydrostatic march only) stops on the same Newton rule from a nearby point
# (the predicted iterate), and the fractions a solve returns are those of its last sweep, before
# the final update (up to 1e-4 of a defect away), so the march differs from the reference by up
# to the size of the two paths' last Newton updates: Nt and n_e ~4e-8 relative on the
# 4-temperature-node model and up to 1.1e-6 on the 80-node one, records ~6e-8 (below their
# float32 rounding) and up to 2.2e-6 on the 80-node model (the H- opacities, which go as
# n_e n_H), node tangents ~4e-5 of each field's scale (the reference's 5 K differences carry that
# much noise from its 1e-4 stop).
TOL = {"cold": {"nt": 1e-10, "rec": 3e-7, "tan": 2e-5, "ne": 1e-9},
       "continue": {"nt": 2e-6, "rec": 5e-6, "tan": 1e-4, "ne": 2e-6}}


@pytest.mark.gpu
@pytestmark_gpu
@pytest.mark.parametrize("start", ["cold", "continue"])
def test_gpu_records_vs_oracle_and_reference(oracle_lib, eos3, config3, start):
    """Records of the 8 config-3 node vectors: FP32 rounding of the FP64 device result against
    the oracle (the same start), and against the reference's own records."""
    import eos_oracle as eo
    tol = TOL[start]
    ctx = _gpu_ctx(config3, eos3, start)
    nodes = config3["nodes"]
    rec, tan, nt, status = ctx.build_records(nodes, tangents=False, want_nt=True)
    assert np.all(status == 0)
    assert ctx.last_launches == 3
    t = _tables(eos3)
    lam0, mass = _line_const(config3)
    old = eo.set_chem_start(eo.CHEM_START_COLD if start == "cold" else eo.CHEM_START_CONTINUE)
    try:
        for p in range(nodes.shape[0]):
            T, Nt, ro, st = eo.build(t, lam0, mass, nodes[p])
            np.testing.assert_allclose(nt[p], Nt, rtol=1e-10)           # the oracle on the same path
            np.testing.assert_allclose(rec[p], ro, rtol=3e-7, atol=0)
            np.testing.assert_allclose(nt[p], eos3["he_Nt"][p], rtol=tol["nt"])  # the reference
            np.testing.assert_allclose(rec[p], config3["record"][p], rtol=tol["rec"], atol=0)
    finally:
        eo.set_chem_start(old)
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
@pytest.mark.parametrize("start", ["cold", "continue"])
def test_gpu_tangents_vs_reference(oracle_lib, eos3, config3, start):
    """Node tangents (central differences with the reference's steps: two full builds per
    temperature node, re-interpolation for the others) against the reference's."""
    ctx = _gpu_ctx(config3, eos3, start)
    nodes = config3["nodes"]
    rec, tan, _, status = ctx.build_records(nodes, tangents=True)
    assert np.all(status == 0)
    for p in range(nodes.shape[0]):
        ref = config3["record"][p].astype(np.float64)
        rt = config3["tangent"][p].astype(np.float64)
        for q in range(rt.shape[0]):
            scale = np.abs(rt[q]).max(axis=0)
            floor = np.maximum(scale, 1e-6 * np.abs(ref).max(axis=0))
            err = np.abs(tan[p, q] - rt[q]).max(axis=0) / floor
            assert err.max() < TOL[start]["tan"], (p, q, err)
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
@pytest.mark.parametrize("start", ["cold", "continue"])
def test_gpu_dense_temperature_nodes(oracle_lib, eos1, config1, config2, start):
    """The config-1/2 model (80 temperature nodes, one per depth, + 5): records of 17 columns
    against the reference's, and the hydrostatic Nt against its build_from_nodes."""
    ctx = _gpu_ctx(config1, eos1, start)
    nodes = eos1["nodes"]
    rec, _, nt, status = ctx.build_records(nodes, tangents=False, want_nt=True)
    assert np.all(status == 0)
    np.testing.assert_allclose(nt, eos1["he_Nt"], rtol=TOL[start]["nt"])
    ref = np.concatenate([config1["record"], config2["record"]]).astype(np.float64)
    np.testing.assert_allclose(rec, ref, rtol=TOL[start]["rec"], atol=0)
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
@pytest.mark.parametrize("name", ["eos_c3", "eos_c1"])
@pytest.mark.parametrize("start", ["cold", "continue"])
def test_gpu_atmosphere_rows_vs_reference(oracle_lib, name, config3, config1, start):
    """snapi_build_atmos against the reference's return_as_array after build_from_nodes and
    compute_op_referent (the columns the master writes to inverted_atmos.f0), for the config-3
    node vectors and the 80-temperature-node config-1/2 ones, heights taken from the reference."""
    d = load_fixture(name)
    fx = config3 if name == "eos_c3" else config1
    ctx = _gpu_ctx(fx, d, start)
    ref = d["atm_arr"]
    atm, status = ctx.build_atmos(d["nodes"], x3=ref[0, 1])
    ctx.close()
    assert np.all(status == 0)
    assert atm.shape == ref.shape
    np.testing.assert_array_equal(atm[:, 5], 0.0)
    np.testing.assert_allclose(atm[:, 0], ref[:, 0], rtol=0, atol=1e-14)          # log10 tau
    np.testing.assert_array_equal(atm[:, 1], ref[:, 1])                           # heights
    np.testing.assert_allclose(atm[:, 2], ref[:, 2], rtol=1e-13)                   # T
    np.testing.assert_allclose(atm[:, 3], ref[:, 3], rtol=TOL[start]["nt"])        # Nt k T
    np.testing.assert_allclose(atm[:, [4, 6]], ref[:, [4, 6]], rtol=TOL[start]["ne"])  # n_e k T, kappa
    np.testing.assert_allclose(atm[:, 7:10], ref[:, 7:10], rtol=1e-13, atol=1e-9)  # |B|, v_turb, v_z
    np.testing.assert_allclose(atm[:, 10:], ref[:, 10:], rtol=0, atol=1e-12)       # angles


@pytest.mark.gpu
@pytestmark_gpu
def test_gpu_active_rows_untouched_and_batches(oracle_lib, eos3, config3):
    """Inactive pixels keep the caller's rows; several device batches give the same records."""
    nodes = np.concatenate([config3["nodes"]] * 3)
    ctx = _gpu_ctx(config3, eos3, max_batch=5)
    active = np.ones(nodes.shape[0], np.int32)
    active[[1, 4, 17]] = 0
    rec, tan, _, status = ctx.build_records(nodes, active=active, tangents=True)
    assert np.all(status == 0)
    assert not rec[[1, 4, 17]].any() and not tan[[1, 4, 17]].any()
    for p in np.flatnonzero(active):
        np.testing.assert_array_equal(rec[p], rec[p % 8] if active[p % 8] else rec[p])
    np.testing.assert_allclose(rec[8], config3["record"][0], rtol=3e-7)
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
def test_gpu_segmented_march_records_equal_records_only_build(oracle_lib, eos3, config3):
    """With tangents the march runs in depth segments (its state carried between launches) with the
    record chemistry of finished segments on a second stream; without tangents in one launch.  The
    node vector's records are the same computation either way: equal bit for bit."""
    nodes = np.concatenate([config3["nodes"]] * 4)
    ctx = _gpu_ctx(config3, eos3)
    rec_t, tan, nt_t, st_t = ctx.build_records(nodes, tangents=True, want_nt=True)
    rec_0, _, nt_0, st_0 = ctx.build_records(nodes, tangents=False, want_nt=True)
    np.testing.assert_array_equal(rec_t, rec_0)
    np.testing.assert_array_equal(nt_t, nt_0)
    np.testing.assert_array_equal(st_t, st_0)
    assert np.all(np.isfinite(tan))
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
def test_gpu_continued_start_tangents_vs_oracle(oracle_lib, eos3, config3):
    """The device's continued start against the oracle's restatement of it: the same path, so the
    cold start's tight tangent tolerance holds."""
    import eos_oracle as eo
    ctx = _gpu_ctx(config3, eos3, "continue")
    nodes = config3["nodes"]
    rec, tan, nt, status = ctx.build_records(nodes, tangents=True, want_nt=True)
    ctx.close()
    assert np.all(status == 0)
    t = _tables(eos3)
    lam0, mass = _line_const(config3)
    old = eo.set_chem_start(eo.CHEM_START_CONTINUE)
    try:
        for p in range(nodes.shape[0]):
            _, _, ro, _ = eo.build(t, lam0, mass, nodes[p])
            to, _ = eo.tangents(t, lam0, mass, nodes[p])
            for q in range(to.shape[0]):
                floor = np.maximum(np.abs(to[q]).max(axis=0), 1e-6 * np.abs(ro).max(axis=0))
                assert (np.abs(tan[p, q] - to[q]).max(axis=0) / floor).max() < TOL["cold"]["tan"]
    finally:
        eo.set_chem_start(old)


def _variant_tables(eos3):
    """The config-3 tables with paths the Fe I 6300 set does not use: aluminium's neutral stage
    with an Irwin partition function (ln U = sum a_i (ln T)^i, U ~ 2.7 at 5000 K), the CO molecule
    with a constant equilibrium constant."""
    d = {k: np.array(v) for k, v in eos3.items()}
    al = 7  # atoms_6300.cfg order: H He C N O Ca Si Al Fe
    d["pf_type"][al, 0] = 3
    d["pf_ncoef"][al, 0] = 3
    d["pf_coef"][al, 0, :3] = [-2.0, 0.35, 0.0]
    d["pf_nterm"][al, 0] = 0
    co = 6  # mol.cfg order: H- H2+ H2 H2O OH CH CO ...
    d["mol_i"][co, 9] = 1
    d["mol_i"][co, 10] = 1
    d["mol_coef"][co, 0] = 121.1  # its polynomial's value at 5000 K
    return d


def _fieldless_tables(eos3):
    """The config-3 tables with a node model of temperature and velocities only (no B, inclination,
    azimuth nodes: the reference's build then puts B = 1e-3 G at angles 1e-3 rad)."""
    d = {k: np.array(v) for k, v in eos3.items()}
    keep = d["node_kind"] <= 3
    d["node_kind"] = d["node_kind"][keep]
    d["node_tau"] = d["node_tau"][keep]
    d["meta"] = d["meta"].copy()
    d["meta"][3] = keep.sum()
    return d, keep


@pytest.mark.gpu
@pytestmark_gpu
def test_gpu_irwin_and_constant_equilibrium_vs_oracle(oracle_lib, eos3, config3):
    import eos_oracle as eo
    import snapi_b200 as sb
    from snapi_b200.eos_tables import EosTables
    d = _variant_tables(eos3)
    t = EosTables(d)
    ctx = sb.Context.from_fixture(config3)
    ctx.eos_set(EosTables(d))
    ctx.eos_chem_start(sb.api.CHEM_START_COLD)  # the table variants against the oracle's path
    nodes = config3["nodes"][:4]
    rec, tan, _, status = ctx.build_records(nodes, tangents=True)
    assert np.all(status == 0)
    lam0, mass = _line_const(config3)
    base = EosTables(eos3)
    for p in range(nodes.shape[0]):
        _, _, ro, st = eo.build(t, lam0, mass, nodes[p])
        assert st == 0
        np.testing.assert_allclose(rec[p], ro, rtol=3e-7, atol=0)
        _, _, r0, _ = eo.build(base, lam0, mass, nodes[p])
        assert np.abs(ro[:, 2] / r0[:, 2] - 1).max() > 1e-6  # the variant tables do change n_e
        to, _ = eo.tangents(t, lam0, mass, nodes[p])
        scale = np.maximum(np.abs(to).max(axis=1, keepdims=True), 1e-6 * np.abs(ro).max(axis=0))
        assert (np.abs(tan[p] - to) / scale).max() < 2e-5
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
def test_gpu_model_without_field_nodes_vs_oracle(oracle_lib, eos3, config3):
    import eos_oracle as eo
    import snapi_b200 as sb
    from snapi_b200.eos_tables import EosTables
    d, keep = _fieldless_tables(eos3)
    t = EosTables(d)
    ctx = sb.Context.from_fixture(config3)
    ctx.eos_set(EosTables(d))
    ctx.eos_chem_start(sb.api.CHEM_START_COLD)
    nodes = np.ascontiguousarray(config3["nodes"][:3][:, keep])
    rec, tan, _, status = ctx.build_records(nodes, tangents=True)
    assert np.all(status == 0)
    lam0, mass = _line_const(config3)
    for p in range(nodes.shape[0]):
        _, _, ro, st = eo.build(t, lam0, mass, nodes[p])
        np.testing.assert_allclose(rec[p], ro, rtol=3e-7, atol=1e-30)
        assert abs(ro[0, 4] - 1e-3) < 1e-12  # |B| = TINY
        to, _ = eo.tangents(t, lam0, mass, nodes[p])
        scale = np.maximum(np.abs(to).max(axis=1, keepdims=True), 1e-6 * np.abs(ro).max(axis=0))
        assert (np.abs(tan[p] - to) / np.maximum(scale, 1e-30)).max() < 2e-5
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
def test_gpu_device_pointers_match_host(oracle_lib, eos3, config3, config4):
    """snapi_build_records and snapi_lm_fit on device memory (SNAPI_MEM_DEVICE) give the host-memory
    results."""
    import ctypes
    import torch
    import snapi_b200 as sb
    from snapi_b200.api import SnapiLmOpts, lib, MEM_DEVICE
    from snapi_b200.eos_tables import EosTables
    from helpers import node_scales
    dev = torch.device("cuda", 0)
    ctx = sb.Context.from_fixture(config3)
    ctx.eos_set(EosTables(eos3))
    nodes = config3["nodes"]
    rec_h, tan_h, _, _ = ctx.build_records(nodes, tangents=True)
    n = nodes.shape[0]
    d_nodes = torch.from_numpy(np.ascontiguousarray(nodes)).to(dev)
    d_rec = torch.zeros((n, ctx.nd, ctx.nfield), dtype=torch.float32, device=dev)
    d_tan = torch.zeros((n, nodes.shape[1], ctx.nd, ctx.nfield), dtype=torch.float32, device=dev)
    ctx.build_records_device(n, d_nodes.data_ptr(), d_rec.data_ptr(), d_tan.data_ptr())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_rec.cpu().numpy(), rec_h)
    np.testing.assert_array_equal(d_tan.cpu().numpy(), tan_h)
    ctx.close()

    fx = config4
    ic = float(np.abs(fx["target"][:, :, 0]).max())
    kinds = np.ascontiguousarray(fx["node_kind"], dtype=np.int32)
    steps = np.ascontiguousarray(1e-2 * node_scales(kinds), dtype=np.float64)
    ctx = sb.Context.from_fixture(fx, stokes_scale=ic)
    ctx.eos_set(EosTables(eos3))
    host = ctx.lm_fit_device(fx["nodes0"], fx["target"], kinds, steps, mask=fx["mask"], lm_start=1e3, max_iter=5,
                             delta=1e-3)
    npix, npar = fx["nodes0"].shape
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dtype=dt)).to(dev)  # noqa: E731
    d_n0, d_obs, d_mask = t(fx["nodes0"], np.float64), t(fx["target"], np.float32), t(fx["mask"], np.float32)
    d_out = torch.zeros((npix, npar), dtype=torch.float64, device=dev)
    d_chi = torch.zeros(npix, dtype=torch.float64, device=dev)
    d_it = torch.zeros(npix, dtype=torch.int32, device=dev)
    d_st = torch.zeros((npix, ctx.nl, 4), dtype=torch.float32, device=dev)
    opts = SnapiLmOpts(npar, kinds.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 1e3, 5, 1e-3, 1e-30,
                       steps.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0.0)
    ws = np.ones(4)
    nsteps = ctypes.c_int(0)
    p = lambda x: ctypes.c_void_p(x.data_ptr())  # noqa: E731
    rc = lib().snapi_lm_fit(ctx._ctx, npix, ctypes.byref(opts), p(d_n0), p(d_obs), ws.ctypes.data_as(ctypes.c_void_p),
                            p(d_mask), p(d_out), p(d_chi), p(d_it), p(d_st), ctypes.byref(nsteps), MEM_DEVICE)
    ctx._check(rc)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_out.cpu().numpy(), host["nodes"])
    np.testing.assert_array_equal(d_chi.cpu().numpy(), host["chi2"])
    np.testing.assert_array_equal(d_it.cpu().numpy(), host["iters"])
    ctx.close()


@pytest.mark.gpu
@pytestmark_gpu
def test_gpu_build_errors(oracle_lib, eos3, config3):
    """Error codes, not faults: building without a model, a model whose depth grid is not the
    problem's, node vectors of the wrong length, an LM whose node kinds are not the model's."""
    import snapi_b200 as sb
    from snapi_b200.api import SnapiError
    from snapi_b200.eos_tables import EosTables
    from helpers import node_scales
    ctx = sb.Context.from_fixture(config3)
    ctx._eos_npar = 10
    with pytest.raises(SnapiError) as e:
        ctx.build_records(config3["nodes"][:1], tangents=False)
    assert e.value.code == -1 and "snapi_eos_set" in str(e.value)
    d = dict(eos3)
    d["meta"] = np.array(d["meta"])
    d["meta"][6] = 1.5  # tau_max: another grid
    with pytest.raises(SnapiError) as e:
        ctx.eos_set(EosTables(d))
    assert e.value.code == -1 and "tau500" in str(e.value)
    ctx.eos_set(EosTables(eos3))
    with pytest.raises(ValueError):
        ctx.build_records(config3["nodes"][:1, :9], tangents=False)
    kinds = config3["node_kind"].copy()
    kinds[4], kinds[5] = 3, 2  # not the model's order
    with pytest.raises(SnapiError) as e:
        ctx.lm_fit_device(config3["nodes"][:2], config3["target"][:2], kinds, 1e-2 * node_scales(kinds), max_iter=2)
    assert e.value.code == -1
    rec, _, _, st = ctx.build_records(config3["nodes"][:1], tangents=False)  # the context still works
    assert st[0] == 0 and np.isfinite(rec).all()
    ctx.close()
