"""Algorithmic work of the Stokes synthesis + adjoint per (wavelength, depth) cell and of the node
-> record build per column, counted by the op-count builds (test and measurement infrastructure;
never the product).

  count_oracle.cc  the FP64 restatement oracle/snapi_oracle.c with every double operation counted:
                   the reference's algorithm (opacity at every depth and wavelength, the polarized
                   DELO sweep) -- the forward cell
  count_emu.cc     the CPU emulator of the FP32 kernels (tests/emu/snapi_emu.cc) with every float
                   and double operation counted: emu_synth is the synthesis kernel's algorithm,
                   emu_adjoint the adjoint call's (forward sweep storing its state, reverse DELO
                   sweep, opacity adjoint, chain rule to the record) -- forward + reverse cell
  count_eos.cc     the FP64 node -> record restatement oracle/eos_oracle.c with every double
                   operation counted: one column's build (hydrostatic march with the chemistry at
                   every iteration, the record chemistry at every depth), with the reference's cold
                   chemistry start and with the CUDA path's continued start; a build with node
                   tangents is 1 + 2 x (temperature nodes) such builds (+- 2.5 K per node).  The
                   restatement re-evaluates the partition functions' temperature terms in every
                   ionisation sweep, as the reference does; the kernels evaluate them once per
                   temperature, so this count is an upper bound of the kernels' work.

Run on the config-3 pixels (80 depths, 201 wavelengths, Fe I 6301.5 / 6302.5 with their Zeeman
patterns and the hydrogen far wings; the config-3 node model).  flops = add + mul + div + 2 fma;
square roots, exponentials / logarithms and trigonometric functions are listed separately.  The
figures the benchmark uses are frozen in bench.py (FLOPS) and profiles/flops_per_cell.md.

usage: python oracle/opcount/count_flops.py [--pixels N]
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
sys.path.insert(0, ORACLE)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)
import snapi_oracle as so  # noqa: E402

KEYS = ["add", "mul", "div", "fma", "sqrt", "exp", "trig", "flops"]


def build(out_dir):
    libs = {}
    inc_o = ["-I" + ORACLE, "-I" + os.path.join(ROOT, "include")]
    for name, src, inc in (("oracle", "count_oracle.cc", inc_o), ("emu", "count_emu.cc", []),
                           ("eos", "count_eos.cc", inc_o)):
        out = os.path.join(out_dir, "libopc_%s.so" % name)
        subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared"] + inc + ["-o", out, os.path.join(HERE, src)],
                       check=True)
        L = ctypes.CDLL(out)
        L.opc_get.argtypes = [ctypes.c_void_p]
        libs[name] = L
    return libs


def counts(L):
    c = np.zeros(16, np.int64)
    L.opc_get(c.ctypes.data)
    return {("f32_" if k < 8 else "f64_") + KEYS[k % 8]: int(c[k]) for k in range(16)}


def total(c):
    out = {k: c["f32_" + k] + c["f64_" + k] for k in KEYS}
    out["f32_flops"], out["f64_flops"] = c["f32_flops"], c["f64_flops"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pixels", type=int, default=8)
    a = ap.parse_args()
    fx = dict(np.load(os.path.join(ROOT, "tests", "golden", "config3.npz")))
    npix = min(a.pixels, fx["record"].shape[0])
    lam, tau = fx["lambda_air"], fx["tau500"]
    nl, nd = lam.shape[0], tau.shape[0]
    cells = npix * nl * nd
    d = ctypes.POINTER(ctypes.c_double)
    P = lambda x: x.ctypes.data_as(d)  # noqa: E731
    with tempfile.TemporaryDirectory() as tmp:
        libs = build(tmp)
        # FP64 oracle synthesis (the oracle's line structures: same layout)
        Lo = libs["oracle"]
        Lo.sno_synth_batch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, d, d, d, ctypes.c_int,
                                       ctypes.POINTER(so.SnoLine), ctypes.c_double, d]
        lines = so.lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])
        rec = np.ascontiguousarray(fx["record"][:npix], np.float64)
        st = np.zeros((npix, nl, 4))
        Lo.opc_reset()
        Lo.sno_synth_batch(npix, nd, nl, P(np.ascontiguousarray(lam)), P(np.ascontiguousarray(tau)), P(rec),
                           len(lines), lines, -1.0, P(st))
        fwd64 = total(counts(Lo))
        ref = so.synth(lam, tau, fx["record"][:npix], lines)
        assert np.abs(st - ref).max() < 1e-12 * np.abs(ref).max(), "counting build changed the oracle's results"
        # FP32 kernels through the emulator
        from helpers import emu_lines
        Le = libs["emu"]
        vp, ip, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        Le.emu_synth.argtypes = [ip, ip, ip, vp, vp, dbl, vp, ip, vp, vp]
        Le.emu_adjoint.argtypes = [ip, ip, ip, vp, vp, dbl, vp, dbl, ip, vp, vp, vp, vp, ip, vp, vp, vp, vp, vp]
        el = emu_lines(so, fx)
        r32 = np.ascontiguousarray(fx["record"][:npix], np.float32)
        out = np.zeros((npix, nl, 4), np.float32)
        Le.opc_reset()
        Le.emu_synth(nd, nl, len(el), lam.ctypes.data, tau.ctypes.data, 1.0, ctypes.addressof(el), npix,
                     r32.ctypes.data, out.ctypes.data)
        syn32 = total(counts(Le))
        obs = np.ascontiguousarray(fx["target"][:npix], np.float32)
        tan = np.ascontiguousarray(fx["tangent"][:npix], np.float32)
        npar = tan.shape[1]
        ws = np.ones(4)
        chi2 = np.zeros(npix)
        grad = np.zeros((npix, npar))
        ic = float(fx["stokes"][:, :, 0].max())
        Le.opc_reset()
        Le.emu_adjoint(nd, nl, len(el), lam.ctypes.data, tau.ctypes.data, 1.0, ctypes.addressof(el), ic, npix,
                       r32.ctypes.data, obs.ctypes.data, ws.ctypes.data, None, npar, tan.ctypes.data,
                       out.ctypes.data, chi2.ctypes.data, grad.ctypes.data, None)
        adj32 = total(counts(Le))
        # FP64 node -> record build per column (config-3 node model: 4 temperature nodes)
        from snapi_b200.eos_tables import EosTables
        eos = dict(np.load(os.path.join(ROOT, "tests", "golden", "eos_c3.npz")))
        tab = EosTables(eos)
        Lb = libs["eos"]
        Lb.sne_build.restype = ctypes.c_int
        Lb.sne_build.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, d, d, d, d, d, d]
        Lb.sne_set_chem_start.argtypes = [ctypes.c_int]
        lam0 = np.ascontiguousarray(fx["line_const"][:, 0])
        mass = np.ascontiguousarray(fx["line_const"][:, 3])
        nf = 12 + 3 * tab.nlines
        tn = np.flatnonzero(eos["node_kind"].astype(int) == 1)
        builds = {}
        for mode, tag in ((1, "cold_start"), (0, "continued_start")):
            Lb.sne_set_chem_start(mode)
            per = []
            for p in range(npix):
                Lb.opc_reset()
                variants = [fx["nodes"][p]]
                for q in tn:
                    for sgn in (0.5, -0.5):
                        v = fx["nodes"][p].copy()
                        v[q] += sgn * 5.0
                        variants.append(v)
                one = None
                for k, v in enumerate(variants):
                    T = np.zeros(tab.nd)
                    Nt = np.zeros(tab.nd)
                    r = np.zeros((tab.nd, nf))
                    Lb.sne_build(ctypes.addressof(tab.model), tab.nd, tab.nlines, P(lam0), P(mass),
                                 P(np.ascontiguousarray(v)), P(T), P(Nt), P(r))
                    if k == 0:
                        one = total(counts(Lb))
                per.append((one, total(counts(Lb))))
            builds[tag] = {"records_only_flops_per_column": float(np.mean([x["flops"] for x, _ in per])),
                           "with_tangents_flops_per_column": float(np.mean([y["flops"] for _, y in per])),
                           "with_tangents_special_per_column": {k: float(np.mean([y[k] for _, y in per]))
                                                                for k in ("sqrt", "exp", "trig")},
                           "builds_per_column_with_tangents": 1 + 2 * len(tn)}
        Lb.sne_set_chem_start(1)
    res = {
        "workload": "config-3 pixels: %d depths x %d wavelengths, Fe I 6301.5/6302.5 + H far wings, 10 nodes"
                    % (nd, nl),
        "pixels_counted": npix,
        "cells_per_pixel": nl * nd,
        "forward_cell_fp64_oracle": {k: v / cells for k, v in fwd64.items()},
        "synthesis_cell_fp32_kernel": {k: v / cells for k, v in syn32.items()},
        "adjoint_cell_fp32_kernel": {k: v / cells for k, v in adj32.items()},
        "reverse_cell_fp32_kernel": {k: (adj32[k] - syn32[k]) / cells for k in adj32},
        "synthesis_flops_per_pixel": syn32["flops"] / npix,
        "adjoint_flops_per_pixel": adj32["flops"] / npix,
        "adjoint_fp32_flops_per_pixel": adj32["f32_flops"] / npix,
        "oracle_forward_flops_per_pixel": fwd64["flops"] / npix,
        "node_build_fp64": builds,
    }
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
