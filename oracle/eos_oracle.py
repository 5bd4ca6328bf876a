"""ctypes binding of the FP64 CPU restatement of the node -> record build (oracle/eos_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker of snapi_build_records.  Only tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline leg import this module; the product never does.
"""
import ctypes
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))
from snapi_b200.eos_tables import MAX_LEVELS, MAX_STAGES, EosTables  # noqa: E402
from snapi_oracle import lib as _lib  # noqa: E402

_D = ctypes.POINTER(ctypes.c_double)
_ready = False


def lib():
    global _ready
    L = _lib()
    if not _ready:
        L.sne_chem.restype = ctypes.c_int
        L.sne_chem.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D, _D, _D, _D, _D]
        L.sne_build.restype = ctypes.c_int
        L.sne_build.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, _D]
        L.sne_columns.restype = ctypes.c_int
        L.sne_columns.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D]
        L.sne_atmos.restype = ctypes.c_int
        L.sne_atmos.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, _D]
        L.sne_set_chem_start.restype = ctypes.c_int
        L.sne_set_chem_start.argtypes = [ctypes.c_int]
        L.sne_tangents.restype = ctypes.c_int
        L.sne_tangents.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D]
        _ready = True
    return L


CHEM_START_CONTINUE, CHEM_START_COLD = 0, 1  # SNAPI_CHEM_START_*


def set_chem_start(mode):
    """The chemistry start of the following builds (the reference's cold start by default, or the
    CUDA path's continued start in the hydrostatic march); returns the previous mode."""
    return lib().sne_set_chem_start(int(mode))


def _p(a):
    return None if a is None else a.ctypes.data_as(_D)


def chem(tables, T, Nt):
    """Ne, stage totals [natom][S], level populations [natom][S][L], kappa_he, kappa, passes."""
    na = tables.model.natom
    ne = np.zeros(1)
    nst = np.zeros((na, MAX_STAGES))
    npop = np.zeros((na, MAX_STAGES, MAX_LEVELS))
    khe = np.zeros(1)
    kap = np.zeros(1)
    passes = lib().sne_chem(ctypes.addressof(tables.model), float(T), float(Nt), _p(ne), _p(nst), _p(npop),
                            _p(khe), _p(kap))
    return ne[0], nst, npop, khe[0], kap[0], passes


def build(tables, lam0, mass, nodes, nd=None):
    """T [nd], Nt [nd], record [nd][nfield] (FP64) and status of one node vector."""
    nd = nd or tables.nd
    nl = tables.nlines
    lam0 = np.ascontiguousarray(lam0, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    nodes = np.ascontiguousarray(nodes, np.float64)
    T = np.zeros(nd)
    Nt = np.zeros(nd)
    rec = np.zeros((nd, 12 + 3 * nl))
    st = lib().sne_build(ctypes.addressof(tables.model), nd, nl, _p(lam0), _p(mass), _p(nodes), _p(T), _p(Nt),
                         _p(rec))
    if st < 0:
        raise ValueError("sne_build: bad sizes")
    return T, Nt, rec, st


def atmos(tables, nodes, x3=None, nd=None):
    """The 12 return_as_array rows [12][nd] of one node vector's column, and the status."""
    nd = nd or tables.nd
    nodes = np.ascontiguousarray(nodes, np.float64)
    h3 = None if x3 is None else np.ascontiguousarray(x3, np.float64)
    out = np.zeros((12, nd))
    st = lib().sne_atmos(ctypes.addressof(tables.model), nd, _p(nodes), _p(h3), _p(out))
    if st < 0:
        raise ValueError("sne_atmos: bad sizes")
    return out, st


def columns(tables, lam0, mass, cols):
    """Record [nd][nfield] (FP64) of one column [12][nd] in the sne_atmos row layout, and the status."""
    cols = np.ascontiguousarray(cols, np.float64)
    nd = cols.shape[1]
    nl = tables.nlines
    rec = np.zeros((nd, 12 + 3 * nl))
    st = lib().sne_columns(ctypes.addressof(tables.model), nd, nl, _p(np.ascontiguousarray(lam0, np.float64)),
                           _p(np.ascontiguousarray(mass, np.float64)), _p(cols), _p(rec))
    if st < 0:
        raise ValueError("sne_columns: bad sizes")
    return rec, st


def tangents(tables, lam0, mass, nodes, step=None, nd=None):
    nd = nd or tables.nd
    nl = tables.nlines
    lam0 = np.ascontiguousarray(lam0, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    nodes = np.ascontiguousarray(nodes, np.float64)
    tan = np.zeros((tables.npar, nd, 12 + 3 * nl))
    st = None if step is None else np.ascontiguousarray(step, np.float64)
    status = lib().sne_tangents(ctypes.addressof(tables.model), nd, nl, _p(lam0), _p(mass), _p(nodes), _p(st),
                                _p(tan))
    return tan, status


def load_tables(path):
    return EosTables(np.load(path))
