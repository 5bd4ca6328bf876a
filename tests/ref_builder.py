"""Host-side node -> record builders for the LM tests (test infrastructure).

RefBuilder: the reference's own build_from_nodes + chemistry + the node tangents (central
differences, atmos_fit.cc:1225-1307), i.e. oracle/_ref/snapi_ref_dump in "dump" mode, run as one
process per core on the pixels still fitting.  This is the caller's side of snapi_lm_step: in
production the reference's islave builds the records with the same code.

LinearBuilder: records that are exactly linear in the nodes (micro-turbulence, line-of-sight
velocity, B, inclination, azimuth enter the record linearly through the node interpolation, and
the azimuth only through 2 phi), so record(n) = record(n0) + sum_p tangent_p (n_p - n0_p).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DUMP = os.path.join(ROOT, "oracle", "_ref", "snapi_ref_dump")
TASK = os.path.join(HERE, "golden", "c3.tsk")
sys.path.insert(0, os.path.join(HERE, "golden"))
from sbin import read_sbin  # noqa: E402


def ref_builder_available():
    return os.path.exists(DUMP) and os.path.exists(TASK)


class RefBuilder:
    """responses: return the reference's own node responses (obs_stokes_responses_to_nodes, the
    Jacobian its stokes_lm_fit uses) instead of the record tangents, for snapi_lm_step_jacobian.
    history: keep, per call, the requested nodes and the reference's spectra there ("stokes" of
    obs_stokes; with responses also "stokes_resp", the spectrum of the responses call, which
    stokes_lm_fit forms its residual with) and the responses."""

    def __init__(self, task=TASK, nproc=None, responses=False, history=False):
        self.task = task
        self.nproc = nproc or os.cpu_count() or 1
        self.calls = 0
        self.responses = responses
        self.history = [] if history else None

    def __call__(self, nodes, active):
        idx = np.flatnonzero(active)
        rec = tan = None
        kept = {}
        with tempfile.TemporaryDirectory(prefix="snapi_build_") as tmp:
            jobs = []
            for k, chunk in enumerate(np.array_split(idx, min(self.nproc, max(1, idx.size)))):
                if chunk.size == 0:
                    continue
                nf = os.path.join(tmp, "n%d.f64" % k)
                out = os.path.join(tmp, "o%d.sbin" % k)
                np.ascontiguousarray(nodes[chunk], dtype="<f8").tofile(nf)
                flags = "1" if self.responses else "2"
                p = subprocess.Popen([DUMP, "dump", self.task, nf, str(chunk.size), flags, out], cwd=tmp,
                                     stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
                jobs.append((chunk, out, p))
            for chunk, out, p in jobs:
                if p.wait() != 0:
                    raise RuntimeError("snapi_ref_dump failed")
                d = read_sbin(out)
                key = "responses" if self.responses else "tangent"
                if rec is None:
                    rec = np.zeros((nodes.shape[0],) + d["record"].shape[1:], np.float32)
                    tan = np.zeros((nodes.shape[0],) + d[key].shape[1:], np.float32)
                rec[chunk] = d["record"]
                tan[chunk] = d[key]
                if self.history is not None:
                    for k in ("stokes", "stokes_resp", "responses"):
                        if k in d:
                            if k not in kept:
                                kept[k] = np.full((nodes.shape[0],) + d[k].shape[1:], np.nan)
                            kept[k][chunk] = d[k]
        self.calls += 1
        if self.history is not None:
            kept["nodes"] = np.array(nodes, np.float64, copy=True)
            kept["active"] = np.array(active, bool, copy=True)
            self.history.append(kept)
        return rec, tan


class LinearBuilder:
    def __init__(self, rec0, tan, nodes0):
        self.rec0 = np.asarray(rec0, np.float64)
        self.tan = np.asarray(tan, np.float64)
        self.nodes0 = np.asarray(nodes0, np.float64)

    def __call__(self, nodes, active):
        d = np.asarray(nodes, np.float64) - self.nodes0
        rec = self.rec0 + np.einsum("np,npzf->nzf", d, self.tan)
        return rec.astype(np.float32), self.tan.astype(np.float32)
