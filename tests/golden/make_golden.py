"""Generate the golden fixtures of the tests from the compiled reference (test infrastructure).

Runs in the development container only (it reads the reference's atom / molecule configs and
its 80-depth atmosphere file from REF and runs oracle/_ref/snapi_ref_dump).  Writes:

  tests/golden/c1.tsk, c3.tsk     task blobs (packed atmosphere column + node model + lambda
                                  grid), the payload the reference's master sends a slave;
                                  c5.tsk, c5_spec.tsk the config-5 tasks (80 / 100 depths)
  tests/golden/config1.npz        one column, 80 depths, 201 lambda: record, reference Stokes,
                                  reference opacity at 7 wavelengths, line constants
  tests/golden/config2.npz        16 pixels of the seeded 256x256 synthesis cube (seed 2)
  tests/golden/config3.npz        8 pixels of the seeded 64x64 node-model cube (seed 3): records,
                                  node tangents, reference Stokes, reference node responses,
                                  noisy target Stokes
  tests/golden/bench_pool.npz     32 more seeded config-3 columns (seed 303) with records, node
                                  tangents and reference Stokes: the thermal structures the
                                  benchmark tiles over its 64x64 pixels
  tests/golden/eos_c1.npz, eos_c3.npz  (--only-eos) node-model tables of the c1 / c3 tasks, the
                                  reference's chemistry on a (T, Nt) grid and the columns its
                                  build_from_nodes leaves for the config-1/2 and config-3 nodes,
                                  with the 12 return_as_array rows of each (atm_arr)
  tests/golden/config4_256.npz    (--only-c4-subset 256) the config-4 fit of 256 seeded pixels
                                  (seed 404) by the reference's stokes_lm_fit
  tests/golden/spinor_c3.npz      (--only-spinor) a 4 x 2 atmosphere cube of the eos_c3 columns in
                                  the 12-row layout (one column below the 3200 K floor at the top)
                                  and the records and Stokes the reference's synthesis branch gives
                                  (read_spinor3d, extract, obs_stokes)
  tests/golden/f0_ref.npz         (--only-f0) ANA .f0 files written by the reference's ana_fzwrite
                                  and what its ana_fzread returns for them, for hand-made headers
                                  (reversed synch pattern, big-endian data) and for the two .f0
                                  files of its test directory; a 4 x 4 pixel observed cube (config-4
                                  targets) with the subfield / window / scaling the master's invert
                                  job applies to it (read_file + transpose + normalize + extract)
                                  and the cube_to_invert.f0 it writes; the node and spectra cubes
                                  its write_file calls produce from given arrays
  tests/golden/config5.npz, config5_spec.npz  (--only-c5 [--spec]) NLTE Ca II columns: the
                                  level-population iteration's inputs and the reference's
                                  iterates; with the set-up tables (alis_*: background
                                  bound-free / bound-bound lists, collisional tables, line
                                  damping, the columns' return_as_array rows; eos_*: the task's
                                  atom tables).  --only-c5-setup adds those to an existing one

Synthetic inputs stand in for observations: seeded numpy generators with the shapes and value
distributions of the benchmark configurations (no dataset is read).

usage:  python tests/golden/make_golden.py [--ref /root/reference]
"""
import argparse
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from sbin import read_sbin  # noqa: E402

DUMP = os.path.join(ROOT, "oracle", "_ref", "snapi_ref_dump")
# the same driver over the reference with the configurations' stated settings patched in
# (oracle/patch_spec.py: stokes_lm_fit's DELTA 1e-4, the 5-point angle set, nltepops' 1e-4 stop)
DUMP_SPEC = os.path.join(ROOT, "oracle", "_ref", "snapi_ref_dump_spec")
CFG_FILES = ["atoms_6300.cfg", "mol.cfg", "hydrogen_3lvl.cfg", "helium.cfg", "carbon.cfg", "nitrogen.cfg",
             "oxygen.cfg", "calcium.cfg", "silicon.cfg", "aluminium.cfg", "iron_6300.cfg", "falc_80z.dat",
             "calcium_ir_rh.cfg"]
# config 5: the Fe I 6300 background atoms with Ca II (5 levels + continuum, NLTE = 1) instead of
# the LTE calcium model
C5_ATOMS = ["hydrogen_3lvl.cfg", "helium.cfg", "carbon.cfg", "nitrogen.cfg", "oxygen.cfg", "calcium_ir_rh.cfg",
            "silicon.cfg", "aluminium.cfg", "iron_6300.cfg"]

ND = 80
NLAMBDA = 201
LOGTAU = np.linspace(-6.0, 1.0, ND)


def config1_temperature(x):
    """Config 1 temperature profile: 4400 K at the minimum, tanh rises to 9000 K at log tau = -6
    and 9500 K at log tau = +1 (closed form defined here)."""
    st = lambda z: 0.5 * (1.0 + np.tanh(z))  # noqa: E731
    return (4400.0 + 4600.0 * st((-4.8 - x) / 0.4) / st((-4.8 + 6.0) / 0.4)
            + 5100.0 * st((x - 0.3) / 0.6) / st((1.0 - 0.3) / 0.6))


def write_cfg(path, t_taus, t_vals, vs_taus, vs_vals, vt=1e5, B=1000.0, theta_deg=45.0, phi_deg=30.0,
              atoms="atoms_6300.cfg", lam="6301.0-6303.4", dlam=0.012, atmos_file="falc_80z.dat"):
    fmt = lambda a: ",".join("%.6f" % v for v in a)  # noqa: E731
    cfg = f"""atmos{{
  ID=col
  TYPE=SPINOR
  FILE={atmos_file}
  GEOMETRY=PLANEPARALLEL
  RTSOLVER=Bezier
  ATOM={atoms}
  MOL=mol.cfg
  TAU_GRID=1
}}
obs{{
  ID=obs1
  EL=3.14159265359
  AZ=0.0
  NAME=none
  LAMBDA={lam}
  DLAMBDA={dlam}
}}
model{{
  ID=m1
  TAUGRID=-6.0,1.0
  parameter{{
    ID=TEMP
    TAU={fmt(t_taus)}
    VALUE={fmt(t_vals)}
  }}
  parameter{{
    ID=VT
    TAU=0
    VALUE={vt:.6f}
  }}
  parameter{{
    ID=VS
    TAU={fmt(vs_taus)}
    VALUE={fmt(vs_vals)}
  }}
  parameter{{
    ID=B
    TAU=0
    VALUE={B:.6f}
  }}
  parameter{{
    ID=THETA
    TAU=0
    VALUE={theta_deg:.6f}
  }}
  parameter{{
    ID=PHI
    TAU=0
    VALUE={phi_deg:.6f}
  }}
}}
"""
    with open(path, "w") as f:
        f.write(cfg)


def run(args, cwd):
    r = subprocess.run(args, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("%s failed:\n%s\n%s" % (args, r.stdout, r.stderr))
    return r.stderr


def dump(tmp, task, nodes, flags, name, dump_bin=None):
    nf = os.path.join(tmp, name + "_nodes.f64")
    np.ascontiguousarray(nodes, dtype="<f8").tofile(nf)
    out = os.path.join(tmp, name + ".sbin")
    log = run([dump_bin or DUMP, "dump", task, nf, str(nodes.shape[0]), str(flags), out], tmp)
    sys.stderr.write(log)
    return read_sbin(out)


def line_arrays(d):
    return {"line_const": d["line_const"], "line_ncomp": d["line_ncomp"], "line_pattern": d["line_pattern"]}


def config2_nodes(npix, seed=2):
    """Seeded config-2 pixels: T = config-1 profile + Gaussian-smoothed N(0, 300 K) (sigma = 5 depth
    points), B log-uniform 10..3000 G, cos(inclination) U(-1,1), azimuth U(0, pi), v_los N(0, 2 km/s),
    v_turb U(0.5, 2) km/s.  Node vector: 80 T nodes (one per depth), v_turb, v_los, B, theta, phi."""
    rng = np.random.default_rng(seed)
    base = config1_temperature(LOGTAU)
    k = np.arange(-15, 16)
    ker = np.exp(-0.5 * (k / 5.0) ** 2)
    ker /= np.sqrt(np.sum(ker ** 2))
    nodes = np.zeros((npix, ND + 5))
    for i in range(npix):
        pert = np.convolve(rng.standard_normal(ND + 30), ker, mode="valid")[:ND] * 300.0
        nodes[i, :ND] = np.clip(base + pert, 3500.0, 11500.0)
        nodes[i, ND] = rng.uniform(0.5e5, 2.0e5)
        nodes[i, ND + 1] = rng.normal(0.0, 2.0e5)
        nodes[i, ND + 2] = 10.0 ** rng.uniform(1.0, np.log10(3000.0))
        nodes[i, ND + 3] = np.arccos(rng.uniform(-1.0, 1.0))
        nodes[i, ND + 4] = rng.uniform(0.0, np.pi)
    return nodes


def config2_subset(seed=22):
    """Indices of config 2's parity subset in its 256 x 256 cube (row-major pixel index): the 4 x 4
    pixels at each corner (64) and a seeded 1 % random sample of the rest (655), sorted."""
    corners = [y * 256 + x for y in (0, 1, 2, 3, 252, 253, 254, 255) for x in (0, 1, 2, 3, 252, 253, 254, 255)]
    rest = np.setdiff1d(np.arange(256 * 256), corners)
    pick = np.random.default_rng(seed).choice(rest, size=655, replace=False)
    return np.sort(np.concatenate([np.array(corners), pick]))


def make_config2_subset(tmp):
    """The reference's synthesis of config 2's parity subset (config2_subset) of the seeded cube
    (config2_nodes over all 65 536 pixels): records as float32 (what the device takes) and the
    reference's Stokes (float64), in config2_720.npz."""
    write_cfg(os.path.join(tmp, "c1.cfg"), LOGTAU, config1_temperature(LOGTAU), [0.0], [0.0])
    run([DUMP, "pack", "c1.cfg", "c1.tsk"], tmp)
    idx = config2_subset()
    nodes = config2_nodes(256 * 256)[idx]
    d = dump(tmp, os.path.join(tmp, "c1.tsk"), nodes, 0, "c2s")
    np.savez_compressed(os.path.join(HERE, "config2_720.npz"), lambda_air=d["lambda_air"], tau500=d["tau500"],
                        pixel_index=idx, record=d["record"].astype(np.float32), stokes=d["stokes"], nodes=d["nodes"],
                        meta=d["meta"], **line_arrays(d))


C3_TTAU = np.array([-4.0, -2.5, -1.0, 0.5])
C3_VSTAU = np.array([-2.0, 0.0])
C3_TRUTH = np.array([4600.0, 4900.0, 5500.0, 7400.0, 1.0e5, 0.0, 0.0, 800.0, np.deg2rad(60.0), np.deg2rad(40.0)])


def config3_nodes(npix, seed=3):
    """Seeded config-3 truth nodes (node order of the reference's model: T x4, v_turb, v_los x2,
    B, theta, phi; velocities in cm/s, angles in rad)."""
    rng = np.random.default_rng(seed)
    nodes = np.tile(C3_TRUTH, (npix, 1))
    nodes[:, 0:4] += rng.normal(0.0, 150.0, (npix, 4))
    nodes[:, 4] = rng.uniform(0.5e5, 2.0e5, npix)
    nodes[:, 5:7] = rng.normal(0.0, 1.0e5, (npix, 2))
    nodes[:, 7] = 10.0 ** rng.uniform(2.0, np.log10(2500.0), npix)
    nodes[:, 8] = rng.uniform(np.deg2rad(20.0), np.deg2rad(160.0), npix)
    nodes[:, 9] = rng.uniform(np.deg2rad(10.0), np.deg2rad(170.0), npix)
    return nodes


C4_OFFSET = np.array([200.0, 200.0, 200.0, 200.0, 3.0e4, 3.0e4, 3.0e4, 200.0, 0.1, 0.1])


def config4_inputs(npix, seed=4):
    """Config-4 LM problem: truth nodes (config-3 model, seed 4), initial guess = truth + fixed
    offsets (T +200 K, velocities +0.3 km/s, B +200 G, angles +0.1 rad) and per-pixel masks keeping
    120..201 of the 201 wavelengths (a random contiguous window, then random single drops)."""
    truth = config3_nodes(npix, seed=seed)
    rng = np.random.default_rng(seed + 40)
    mask = np.zeros((npix, NLAMBDA))
    for i in range(npix):
        keep = int(rng.integers(120, 202))
        width = min(NLAMBDA, keep + int(rng.integers(0, 20)))
        start = int(rng.integers(0, NLAMBDA - width + 1))
        m = np.zeros(NLAMBDA)
        m[start:start + width] = 1.0
        on = np.flatnonzero(m)
        drop = rng.choice(on, size=max(0, on.size - keep), replace=False)
        m[drop] = 0.0
        mask[i] = m
    return truth, truth + C4_OFFSET, mask


def parse_trial_models(path, npar):
    """The trial node vectors of the reference's LM loop, one per iteration, from the model prints
    it writes to standard output (model::print, atmos_model.cc:712-760: one line 'i tau value' per
    node, kinds in the node order; inclination and azimuth in degrees -> radians here)."""
    vals = []
    for ln in open(path):
        f = ln.split()
        if len(f) == 3 and f[0].isdigit():
            try:
                vals.append(float(f[2]))
            except ValueError:
                pass
    a = np.array(vals[:len(vals) // npar * npar]).reshape(-1, npar)
    a[:, -2:] = np.deg2rad(a[:, -2:])
    return a


def make_config4(tmp, npix, iters=30, broadening=0.0, name="config4", seed=4, workers=0, spec=False):
    """Reference LM (stokes_lm_fit, start lambda 1e3) on config-4 pixels, one process per pixel;
    with broadening > 0 [cm] the targets are broadened by the reference's own convolution and the
    fit broadens its synthesis and responses the same way.  The relative chi2 stop rule is the
    compiled DELTA 1e-3, or with spec the configuration's 1e-4 (the patched build)."""
    lmfit_bin, delta = (DUMP_SPEC, 1e-4) if spec else (DUMP, 1e-3)
    task = os.path.join(tmp, "c3.tsk")
    truth, nodes0, mask = config4_inputs(npix, seed=seed)
    d = dump(tmp, task, truth, 0, "c4truth")
    rng = np.random.default_rng(44)
    ic = d["stokes"][:, :, 0].max(axis=1)
    stokes = d["stokes"]
    if broadening > 0.0:
        fin = os.path.join(tmp, "c4b_in.f64")
        np.concatenate([d["lambda_air"], stokes.ravel()]).astype("<f8").tofile(fin)
        fout = os.path.join(tmp, "c4b_out.f64")
        run([DUMP, "conv", fin, str(d["lambda_air"].shape[0]), str(npix), repr(broadening), fout], tmp)
        stokes = np.fromfile(fout, dtype="<f8").reshape(stokes.shape)
    target = stokes + rng.normal(0.0, 1e-3, stokes.shape) * ic[:, None, None]
    procs = []
    for i in range(npix):
        for nm, arr in (("n0", nodes0[i:i + 1]), ("tg", target[i:i + 1]), ("mk", mask[i:i + 1])):
            np.ascontiguousarray(arr, dtype="<f8").tofile(os.path.join(tmp, "c4_%s_%d.f64" % (nm, i)))
        args = [lmfit_bin, "lmfit", task] + [os.path.join(tmp, "c4_%s_%d.f64" % (nm, i)) for nm in ("n0", "tg", "mk")] + \
               ["1", str(iters), os.path.join(tmp, "c4_fit_%d.sbin" % i), repr(broadening)]
        if workers and len(procs) >= workers:  # at most `workers` reference processes at a time
            if procs.pop(0).wait() != 0:
                raise RuntimeError("lmfit failed")
        # the reference prints every trial model of its loop (test_model->print(), atmos_fit.cc:152)
        out_f = open(os.path.join(tmp, "c4_trace_%d.txt" % i), "w")
        procs.append(subprocess.Popen(args, cwd=tmp, stdout=out_f, stderr=subprocess.DEVNULL))
        out_f.close()
    for p in procs:
        if p.wait() != 0:
            raise RuntimeError("lmfit failed")
    fits = [read_sbin(os.path.join(tmp, "c4_fit_%d.sbin" % i)) for i in range(npix)]
    npar = nodes0.shape[1]
    trials = [parse_trial_models(os.path.join(tmp, "c4_trace_%d.txt" % i), npar) for i in range(npix)]
    trace = np.full((npix, iters, npar), np.nan)
    for i, t in enumerate(trials):
        trace[i, :t.shape[0]] = t[:iters]
    # the fitted Stokes only for the small fixtures (the 256-pixel one compares nodes and chi2)
    extra = {} if npix > 64 else {"fit_stokes": np.concatenate([f["fit_stokes"] for f in fits])}
    if npix <= 64:
        extra["trace_trial"] = trace
    np.savez_compressed(os.path.join(HERE, name + ".npz"), lambda_air=d["lambda_air"], tau500=d["tau500"],
                        broadening=np.array([broadening]), delta=np.array([delta]),
                        node_kind=d["node_kind"], truth=truth, nodes0=nodes0, mask=mask, target=target,
                        fit_nodes=np.concatenate([f["fit_nodes"] for f in fits]), **extra,
                        fit_chi2=np.concatenate([f["fit_chi2"] for f in fits]),
                        ref_seconds_per_pixel=np.array([np.mean([f["ref_seconds_per_pixel"][0] for f in fits])]),
                        iters=np.array([iters]), **line_arrays(d))


def write_atmos_resampled(src, dst, nd):
    """The reference's SPINOR-format atmosphere file src resampled to nd depths (every column
    interpolated linearly in the row index).  build_from_nodes takes only the depth count (and the
    heights, for return_as_array) from it; the model's TAUGRID sets the log tau grid."""
    rows = open(src).read().split("\n")
    n0 = int(rows[0].split()[0])
    a = np.array([[float(v) for v in r.split()] for r in rows[1:1 + n0]])
    x0 = np.linspace(0.0, 1.0, n0)
    x1 = np.linspace(0.0, 1.0, nd)
    b = np.stack([np.interp(x1, x0, a[:, k]) for k in range(a.shape[1])], axis=1)
    with open(dst, "w") as f:
        f.write("%d\n" % nd)
        for r in b:
            f.write(" ".join("%.6e" % v for v in r) + "\n")


def config5_task(tmp, spec=False):
    """Write and pack the config-5 task in tmp (c5.tsk); returns the dump binary and the fixture
    name.  Default: the reference as compiled on the 80-depth grid; spec: the patched build on the
    100-depth grid (see make_config5)."""
    with open(os.path.join(tmp, "atoms_c5.cfg"), "w") as f:
        f.write("".join("ATOM=%s\n" % a for a in C5_ATOMS))
    dump_bin, name, afile = DUMP, "config5", "falc_80z.dat"
    if spec:
        dump_bin, name, afile = DUMP_SPEC, "config5_spec", "falc_100z.dat"
        write_atmos_resampled(os.path.join(tmp, "falc_80z.dat"), os.path.join(tmp, afile), 100)
    write_cfg(os.path.join(tmp, "c5.cfg"), C3_TTAU, C3_TRUTH[:4], C3_VSTAU, C3_TRUTH[5:7], atoms="atoms_c5.cfg",
              lam="8538.5-8545.985", dlam=0.025, atmos_file=afile)
    run([dump_bin, "pack", "c5.cfg", "c5.tsk"], tmp)
    return dump_bin, name


def config5_setup_arrays(tmp, dump_bin, nodes):
    """The tables of nltepops' population-independent set-up and the columns of the node vectors
    (snapi_ref_dump alisetup: alis_*), and the task's atom / molecule tables with the reference's
    chemistry (snapi_ref_dump eos: eos_*) -- the inputs of the device set-up (snapi_ali_setup)."""
    nf = os.path.join(tmp, "c5s_nodes.f64")
    np.ascontiguousarray(nodes, dtype="<f8").tofile(nf)
    out = {}
    run([dump_bin, "alisetup", "c5.tsk", nf, str(nodes.shape[0]), os.path.join(tmp, "c5s.sbin")], tmp)
    out.update(read_sbin(os.path.join(tmp, "c5s.sbin")))
    run([dump_bin, "eos", "c5.tsk", nf, "0", os.path.join(tmp, "c5e.sbin")], tmp)
    out.update({"eos_" + k: v for k, v in read_sbin(os.path.join(tmp, "c5e.sbin")).items()})
    return out


def make_config5(tmp, ncol, niter=3, spec=False):
    """NLTE Ca II (config 5): the inputs of the level-population iteration per column, the
    populations after each of the reference's first niter iterations, and the populations its
    nltepops converges to.  Columns: the ten-node model with seeded T / v_los / B (seed 5).
    Default: the reference as compiled (2 rays, the 1e-2 stop) on the 80-depth grid
    (config5.npz).  spec: the configuration's stated settings (config5_spec.npz) -- the patched
    reference build (the 5-point angle set, i.e. 10 ray directions, and a 1e-4 population stop)
    on a 100-depth grid; the background opacity / emissivity stored as float32 to keep the fixture
    small (the device takes them as float64; ~6e-8 relative).  Also the set-up tables
    (config5_setup_arrays)."""
    dump_bin, name = config5_task(tmp, spec)
    shutil.copy(os.path.join(tmp, "c5.tsk"), os.path.join(HERE, "c5_spec.tsk" if spec else "c5.tsk"))
    nodes = config3_nodes(ncol, seed=5)
    nf = os.path.join(tmp, "c5_nodes.f64")
    np.ascontiguousarray(nodes, dtype="<f8").tofile(nf)
    out = os.path.join(tmp, "c5.sbin")
    sys.stderr.write(run([dump_bin, "ali", "c5.tsk", nf, str(ncol), str(niter), out], tmp))
    d = read_sbin(out)
    if spec:
        for k in ("ali_bgop", "ali_bgem"):
            d[k] = d[k].astype(np.float32)
    d.update(config5_setup_arrays(tmp, dump_bin, nodes))
    # the reference's synthesis of the 8542 window with those NLTE populations (obs_stokes runs
    # nltepops itself) and the column records the device synthesis takes
    s = dump(tmp, os.path.join(tmp, "c5.tsk"), nodes, 0, "c5syn", dump_bin=dump_bin)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), nodes=nodes, **{k: v for k, v in d.items()},
                        lambda_air=s["lambda_air"], tau500=s["tau500"], record=s["record"], stokes=s["stokes"],
                        ref_synth_seconds=s["ref_seconds_per_pixel"], **line_arrays(s))


def add_config5_setup(tmp, spec=False):
    """Add the set-up arrays (config5_setup_arrays) to an existing config-5 fixture, for its node
    vectors, without running the reference's iterations again (make_config5 writes the same)."""
    dump_bin, name = config5_task(tmp, spec)
    shutil.copy(os.path.join(tmp, "c5.tsk"), os.path.join(HERE, "c5_spec.tsk" if spec else "c5.tsk"))
    path = os.path.join(HERE, name + ".npz")
    d = dict(np.load(path))
    d.update(config5_setup_arrays(tmp, dump_bin, d["nodes"]))
    np.savez_compressed(path, **d)


def make_psf(tmp):
    """The reference's Gaussian instrumental broadening (convolve_spectra_with_gauss) of the
    config-3 Stokes spectra and node responses at 45 and 150 mA FWHM (cfg SPECTRAL_BROADENING,
    converted to cm and divided by 2.35 as jsub/cfg.cc:107-110 does)."""
    c3 = np.load(os.path.join(HERE, "config3.npz"))
    lam = c3["lambda_air"]
    vec = np.concatenate([c3["stokes"], c3["responses"].reshape(-1, lam.shape[0], 4)])
    out = {"lambda_air": lam, "spectra": vec}
    for fwhm in (45.0, 150.0):
        width = fwhm * 1e-11 / 2.35
        fin = os.path.join(tmp, "psf_in.f64")
        np.concatenate([lam, vec.ravel()]).astype("<f8").tofile(fin)
        fout = os.path.join(tmp, "psf_out.f64")
        run([DUMP, "conv", fin, str(lam.shape[0]), str(vec.shape[0]), repr(width), fout], tmp)
        out["width_%d" % int(fwhm)] = np.array([width])
        out["conv_%d" % int(fwhm)] = np.fromfile(fout, dtype="<f8").reshape(vec.shape)
    np.savez_compressed(os.path.join(HERE, "psf.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("SNAPI_REFERENCE", "/root/reference"),
                    help="the reference checkout (default $SNAPI_REFERENCE, else /root/reference)")
    ap.add_argument("--spec", action="store_true",
                    help="config-4 fits with the configuration's DELTA 1e-4 (patched reference build)")
    ap.add_argument("--c2pix", type=int, default=16)
    ap.add_argument("--c3pix", type=int, default=8)
    ap.add_argument("--pool", type=int, default=32)
    ap.add_argument("--only-pool", action="store_true")
    ap.add_argument("--only-c4", action="store_true")
    ap.add_argument("--c4pix", type=int, default=8)
    ap.add_argument("--only-c5", action="store_true")
    ap.add_argument("--only-psf", action="store_true")
    ap.add_argument("--only-c5-setup", action="store_true",
                    help="add the NLTE set-up tables to the existing config-5 fixture (--spec: config5_spec)")
    ap.add_argument("--only-eos", action="store_true")
    ap.add_argument("--only-f0", action="store_true")
    ap.add_argument("--only-spinor", action="store_true")
    ap.add_argument("--only-c4-subset", type=int, default=0, metavar="N",
                    help="config-4 fit of N pixels by the reference (8 processes at a time)")
    ap.add_argument("--c5col", type=int, default=3)
    ap.add_argument("--workers", type=int, default=8, help="reference processes at a time (config-4 subset)")
    ap.add_argument("--only-c2-subset", action="store_true",
                    help="config 2's parity subset (64 corner pixels + 1 %% of its 256 x 256 cube)")
    a = ap.parse_args()
    if not os.path.exists(DUMP):
        raise SystemExit("build the oracle first: make -C oracle")
    tmp = tempfile.mkdtemp(prefix="snapi_golden_")
    try:
        for f in CFG_FILES:
            shutil.copy(os.path.join(a.ref, "cfg", f), tmp)
        if a.only_eos:
            make_eos(tmp)
            return
        if a.only_c5_setup:
            add_config5_setup(tmp, spec=a.spec)
            return
        if a.only_c2_subset:
            make_config2_subset(tmp)
            return
        if a.only_f0:
            make_f0(tmp, a.ref)
            return
        if a.only_spinor:
            make_spinor(tmp)
            return
        if a.only_c4_subset:
            shutil.copy(os.path.join(HERE, "c3.tsk"), os.path.join(tmp, "c3.tsk"))
            make_config4(tmp, a.only_c4_subset, name="config4_%d" % a.only_c4_subset, seed=404, workers=a.workers,
                         spec=a.spec)
            return
        if a.only_psf:
            make_psf(tmp)
            shutil.copy(os.path.join(HERE, "c3.tsk"), os.path.join(tmp, "c3.tsk"))
            # config 4 with the 45 mA instrumental profile of cfg/invert.cfg
            make_config4(tmp, 4, broadening=45.0 * 1e-11 / 2.35, name="config4_psf", spec=a.spec)
            return
        if a.only_pool or a.only_c4 or a.only_c5:
            shutil.copy(os.path.join(HERE, "c3.tsk"), os.path.join(tmp, "c3.tsk"))
        else:
            make_configs_1_to_3(a, tmp)
        if a.c4pix and not a.only_c5:
            make_config4(tmp, a.c4pix, spec=a.spec)
        if a.c5col and not a.only_c4:
            make_config5(tmp, a.c5col, spec=a.spec)
        if a.pool and not (a.only_c4 or a.only_c5):
            n4 = config3_nodes(a.pool, seed=303)
            d4 = dump(tmp, os.path.join(tmp, "c3.tsk"), n4, 2, "pool")
            np.savez_compressed(os.path.join(HERE, "bench_pool.npz"), lambda_air=d4["lambda_air"],
                                tau500=d4["tau500"], record=d4["record"].astype(np.float32),
                                stokes=d4["stokes"], nodes=d4["nodes"], node_kind=d4["node_kind"],
                                tangent=d4["tangent"].astype(np.float32),
                                ref_seconds_per_pixel=d4["ref_seconds_per_pixel"], meta=d4["meta"],
                                **line_arrays(d4))
        print("fixtures written to", HERE)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


F0_NP = [np.int8, np.int16, np.int32, np.float32, np.float64, np.int64]
MFBD_TO_ANA = {0: 0, 1: 1, 2: 2, 3: 5, 4: 3, 5: 4}  # fileio.h MFBD_* -> ana_io.h type codes


def f0_header_block(synch_bytes, subf, nhb, datyp, dims, text=b""):
    b = bytearray(512)
    b[0:4] = synch_bytes
    b[4], b[6], b[7], b[8] = subf, nhb, datyp, len(dims)
    for i, d in enumerate(dims):
        b[192 + 4 * i:196 + 4 * i] = int(d).to_bytes(4, "little")
    b[256:256 + len(text)] = text
    return bytes(b)


def ref_f0read(tmp, path):
    out = os.path.join(tmp, "f0read.dump")
    run([DUMP, "f0read", path, out], tmp)
    b = open(out, "rb").read()
    t, nd = np.frombuffer(b[:8], "<i4")
    dims = np.frombuffer(b[8:8 + 4 * nd], "<i4").astype(np.int64)
    o = 8 + 4 * nd
    hl = int(np.frombuffer(b[o:o + 4], "<i4")[0])
    hdr = b[o + 4:o + 4 + hl]
    o += 4 + hl
    nb = int(np.frombuffer(b[o:o + 8], "<i8")[0])
    return MFBD_TO_ANA[int(t)], dims, hdr, np.frombuffer(b[o + 8:o + 8 + nb], np.uint8)


def make_f0(tmp, ref):
    out = {}
    rng = np.random.default_rng(50)
    # ana_fzwrite: name, ANA type, C shape (slowest first), header text (None: no header)
    wcases = [("f32_3d", 3, (2, 3, 4), None), ("f64_1d_hdr", 4, (5,), "hello f0"),
              ("i16_2d_3blk", 1, (3, 7), "h" * 600), ("i32_4d_255", 2, (2, 2, 2, 2), "a" * 255),
              ("i32_256", 2, (3,), "b" * 256), ("i8_1d", 0, (10,), None), ("i64_clip", 5, (3,), "c" * 4000)]
    names = []
    for name, t, shape, hdr in wcases:
        dt = F0_NP[t]
        if t in (3, 4):
            data = rng.standard_normal(shape).astype(dt)
        else:
            data = rng.integers(-100, 100, shape).astype(dt)
        dfile = os.path.join(tmp, name + ".bin")
        data.tofile(dfile)
        hfile = "-"
        if hdr is not None:
            hfile = os.path.join(tmp, name + ".hdr")
            open(hfile, "w").write(hdr)
        f0 = os.path.join(tmp, name + ".f0")
        run([DUMP, "f0write", f0, str(t), ",".join(str(v) for v in reversed(shape)), hfile, dfile], tmp)
        out["w_%s_data" % name] = data
        out["w_%s_type" % name] = np.int64(t)
        out["w_%s_header" % name] = np.frombuffer((hdr or "").encode(), np.uint8)
        out["w_%s_has_header" % name] = np.int64(hdr is not None)
        out["w_%s_bytes" % name] = np.frombuffer(open(f0, "rb").read(), np.uint8)
        names.append(name)
    out["w_names"] = np.array(names)
    # ana_fzread on hand-made headers: (name, file bytes)
    v = rng.standard_normal((2, 3)).astype(np.float32)
    v8 = rng.standard_normal((4,)).astype(np.float64)
    norm, rev = bytes([0xaa, 0xaa, 0x55, 0x55]), bytes([0x55, 0x55, 0xaa, 0xaa])
    rcases = [
        ("be_data", f0_header_block(norm, 128, 1, 3, (3, 2)) + v.astype(">f4").tobytes()),
        ("rev_synch", f0_header_block(rev, 0, 1, 3, (3, 2), b"reversed") + v.astype(">f4").tobytes()),
        ("rev_synch_be", f0_header_block(rev, 128, 1, 3, (3, 2)) + v.astype("<f4").tobytes()),
        ("f64_2blk", f0_header_block(norm, 0, 2, 4, (4,), b"x" * 255) +
         f0_header_block(b"\0\0\0\0", 0, 0, 0, (), b"tail") + v8.tobytes()),
    ]
    for fn in ("inverted_atmos.f0", "acoustic_mean.f0"):
        rcases.append(("test_" + fn[:-3], open(os.path.join(ref, "test", fn), "rb").read()))
    rnames = []
    for name, blob in rcases:
        path = os.path.join(tmp, "r_" + name + ".f0")
        open(path, "wb").write(blob)
        t, dims, hdr, data = ref_f0read(tmp, path)
        out["r_%s_file" % name] = np.frombuffer(blob, np.uint8)
        out["r_%s_type" % name] = np.int64(t)
        out["r_%s_dims" % name] = dims
        out["r_%s_header" % name] = np.frombuffer(hdr, np.uint8)
        out["r_%s_data" % name] = data
        rnames.append(name)
    out["r_names"] = np.array(rnames)
    # the invert job's cube steps on a 4 x 4 pixel cube of config-4 targets, 3 + 2 padding wavelengths
    d4 = np.load(os.path.join(HERE, "config4.npz"))
    tgt = d4["target"]
    nx, ny, pad0, pad1 = 4, 4, 3, 2
    nlf = NLAMBDA + pad0 + pad1
    cube = np.zeros((nx, ny, 4, nlf))
    for x in range(nx):
        for y in range(ny):
            s4 = tgt[(x * ny + y) % tgt.shape[0]].T
            cube[x, y, :, pad0:pad0 + NLAMBDA] = s4
            cube[x, y, :, :pad0] = s4[:, :1]
            cube[x, y, :, pad0 + NLAMBDA:] = s4[:, -1:]
    sub = (2, 4, 2, 4, pad0 + 1, pad0 + NLAMBDA)
    for tag, t, qs in (("f32", 3, (2.0, 1.0)), ("f64", 4, (3.0, 1.1))):
        data = (cube * qs[0] / qs[1]).astype(F0_NP[t])
        dfile = os.path.join(tmp, "cube_%s.bin" % tag)
        data.tofile(dfile)
        f0 = os.path.join(tmp, "cube_%s.f0" % tag)
        run([DUMP, "f0write", f0, str(t), "%d,4,%d,%d" % (nlf, ny, nx), "-", dfile], tmp)
        sdump = os.path.join(tmp, "cubeobs_%s.bin" % tag)
        c2i = os.path.join(tmp, "c2i_%s.f0" % tag)
        run([DUMP, "cubeobs", f0] + [str(v) for v in sub] + [repr(qs[0]), repr(qs[1]), sdump, c2i], tmp)
        b = open(sdump, "rb").read()
        hdr = np.frombuffer(b[:16], "<i4")
        out["cube_%s_file" % tag] = np.frombuffer(open(f0, "rb").read(), np.uint8)
        out["cube_%s_qs" % tag] = np.array(qs)
        out["cube_%s_S" % tag] = np.frombuffer(b[16:], "<f8").reshape(tuple(hdr))
        out["cube_%s_c2i" % tag] = np.frombuffer(open(c2i, "rb").read(), np.uint8)
    out["cube_sub"] = np.array(sub)
    out["cube_pix"] = np.array([(x * ny + y) % tgt.shape[0] for x in range(nx) for y in range(ny)])
    # write_file of the node cube (3-D) and the fitted spectra (4-D), job.cc:579, 597
    nxs, nys, npar = 3, 3, 10
    nodes = rng.standard_normal((nxs, nys, npar)) * 1e3
    spec = rng.standard_normal((nxs, nys, 4, 7))
    nf, sf = os.path.join(tmp, "wn.bin"), os.path.join(tmp, "ws.bin")
    nodes.tofile(nf)
    spec.tofile(sf)
    on, osp = os.path.join(tmp, "inverted_nodes.f0"), os.path.join(tmp, "inverted_spectra.f0")
    run([DUMP, "cubewrite", nf, sf, str(nxs), str(nys), str(npar), "7", on, osp], tmp)
    out["cw_nodes"] = nodes
    out["cw_spec"] = spec
    out["cw_nodes_file"] = np.frombuffer(open(on, "rb").read(), np.uint8)
    out["cw_spec_file"] = np.frombuffer(open(osp, "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "f0_ref.npz"), **out)


def make_spinor(tmp):
    """The synthesis branch of the master's job on a small atmosphere cube: the 8 eos_c3 columns
    (return_as_array rows) as a 4 x 2 cube, column 3 set to 3000 K in its top 6 depths (below
    read_spinor3d's 3200 K floor); the reference reads it with read_spinor3d and synthesises every
    column -> tests/golden/spinor_c3.npz."""
    sys.path.insert(0, ROOT)
    from snapi_b200 import api
    d = np.load(os.path.join(HERE, "eos_c3.npz"))
    cols = d["atm_arr"].copy()
    cols[3, 2, :6] = 3000.0
    nx, ny = 4, 2
    cube = np.ascontiguousarray(cols.reshape(nx, ny, 12, -1).transpose(2, 0, 1, 3))  # [12][nx][ny][nd]
    api.f0_write(os.path.join(tmp, "atm.f0"), cube)
    shutil.copy(os.path.join(HERE, "c3.tsk"), os.path.join(tmp, "c3.tsk"))
    run([DUMP, "spinor", "c3.tsk", "atm.f0", "spinor.sbin"], tmp)
    o = read_sbin(os.path.join(tmp, "spinor.sbin"))
    np.savez_compressed(os.path.join(HERE, "spinor_c3.npz"), columns=cols, nx=np.array([nx]), ny=np.array([ny]),
                        record=o["record"], stokes=o["stokes"])


def make_eos(tmp):
    """Node-model tables of the c1 / c3 tasks (atoms, partition functions, levels with their
    bound-free cross-sections, molecules, line ties, nodes), the reference's chemistry on a (T, Nt)
    grid and the columns (T, Nt, n_e, kappa, rho) its build_from_nodes leaves for the config-1/2
    and config-3 node vectors -> tests/golden/eos_c1.npz, eos_c3.npz."""
    c2 = np.load(os.path.join(HERE, "config2.npz"))
    c1 = np.load(os.path.join(HERE, "config1.npz"))
    c3 = np.load(os.path.join(HERE, "config3.npz"))
    for name, task, nodes in (("eos_c1", "c1.tsk", np.concatenate([c1["nodes"], c2["nodes"]])),
                              ("eos_c3", "c3.tsk", c3["nodes"])):
        shutil.copy(os.path.join(HERE, task), os.path.join(tmp, task))
        nf = os.path.join(tmp, name + "_nodes.f64")
        np.ascontiguousarray(nodes, dtype="<f8").tofile(nf)
        out = os.path.join(tmp, name + ".sbin")
        run([DUMP, "eos", task, nf, str(nodes.shape[0]), out], tmp)
        d = read_sbin(out)
        d["nodes"] = nodes
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)


def make_configs_1_to_3(a, tmp):
    if True:
        # config 1: dense temperature nodes (one per depth) reproduce the closed-form profile
        T1 = config1_temperature(LOGTAU)
        write_cfg(os.path.join(tmp, "c1.cfg"), LOGTAU, T1, [0.0], [0.0])
        run([DUMP, "pack", "c1.cfg", "c1.tsk"], tmp)
        shutil.copy(os.path.join(tmp, "c1.tsk"), os.path.join(HERE, "c1.tsk"))
        n1 = np.concatenate([T1, [1e5, 0.0, 1000.0, np.deg2rad(45.0), np.deg2rad(30.0)]])[None, :]
        d1 = dump(tmp, os.path.join(tmp, "c1.tsk"), n1, 4, "c1")
        np.savez_compressed(os.path.join(HERE, "config1.npz"), lambda_air=d1["lambda_air"], tau500=d1["tau500"],
                            record=d1["record"], stokes=d1["stokes"], nodes=d1["nodes"], probe_l=d1["probe_l"],
                            opacity_probe=d1["opacity_probe"], ref_dld=d1["ref_dld"], ref_adamp=d1["ref_adamp"],
                            meta=d1["meta"], **line_arrays(d1))
        # config 2 subset
        n2 = config2_nodes(a.c2pix)
        d2 = dump(tmp, os.path.join(tmp, "c1.tsk"), n2, 0, "c2")
        np.savez_compressed(os.path.join(HERE, "config2.npz"), lambda_air=d2["lambda_air"], tau500=d2["tau500"],
                            record=d2["record"], stokes=d2["stokes"], nodes=d2["nodes"], meta=d2["meta"],
                            **line_arrays(d2))
        # config 3: ten-node model
        write_cfg(os.path.join(tmp, "c3.cfg"), C3_TTAU, C3_TRUTH[:4], C3_VSTAU, C3_TRUTH[5:7])
        run([DUMP, "pack", "c3.cfg", "c3.tsk"], tmp)
        shutil.copy(os.path.join(tmp, "c3.tsk"), os.path.join(HERE, "c3.tsk"))
        n3 = config3_nodes(a.c3pix)
        d3 = dump(tmp, os.path.join(tmp, "c3.tsk"), n3, 3, "c3")
        rng = np.random.default_rng(33)
        Ic = d3["stokes"][:, :, 0].max(axis=1)
        target = d3["stokes"] + rng.normal(0.0, 1e-3, d3["stokes"].shape) * Ic[:, None, None]
        np.savez_compressed(os.path.join(HERE, "config3.npz"), lambda_air=d3["lambda_air"], tau500=d3["tau500"],
                            record=d3["record"], stokes=d3["stokes"], nodes=d3["nodes"], node_kind=d3["node_kind"],
                            tangent=d3["tangent"].astype(np.float32), responses=d3["responses"], target=target,
                            ref_seconds_per_pixel=d3["ref_seconds_per_pixel"], meta=d3["meta"], **line_arrays(d3))


if __name__ == "__main__":
    main()
