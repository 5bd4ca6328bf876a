"""ctypes binding of the FP64 CPU restatement (oracle/snapi_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA path.  Only tests/, __graft_entry__.smoke()
and bench.py's cpu_baseline leg import this module; the product never does.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MAXCOMP = 16


class SnoLine(ctypes.Structure):
    _fields_ = [
        ("lam0", ctypes.c_double),
        ("sf", ctypes.c_double),
        ("ar", ctypes.c_double),
        ("mass", ctypes.c_double),
        ("split", ctypes.c_int),
        ("ncomp", ctypes.c_int * 3),
        ("S", (ctypes.c_double * MAXCOMP) * 3),
        ("D", (ctypes.c_double * MAXCOMP) * 3),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_ref", "libsnapi_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle library missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(path)
        d = ctypes.POINTER(ctypes.c_double)
        L.sno_voigt.argtypes = [ctypes.c_double, ctypes.c_double, d, d]
        L.sno_airtovac.restype = ctypes.c_double
        L.sno_airtovac.argtypes = [ctypes.c_double]
        L.sno_zeeman_pattern.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.POINTER(SnoLine)]
        L.sno_opacity.argtypes = [d, ctypes.c_int, ctypes.POINTER(SnoLine), ctypes.c_double,
                                  ctypes.c_double, d, d]
        L.sno_formal.argtypes = [ctypes.c_int, d, d, d, ctypes.c_double, d]
        L.sno_synth_batch.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, d, d, d, ctypes.c_int,
                                      ctypes.POINTER(SnoLine), ctypes.c_double, d]
        L.sno_chi2_grad_fd.argtypes = [ctypes.c_int, ctypes.c_int, d, d, d, ctypes.c_int,
                                       ctypes.POINTER(SnoLine), ctypes.c_double, d, d, d, ctypes.c_int, d,
                                       ctypes.c_double, d, d]
        L.sno_stokes_jvp_fd.argtypes = [ctypes.c_int, ctypes.c_int, d, d, d, ctypes.c_int,
                                        ctypes.POINTER(SnoLine), ctypes.c_double, ctypes.c_int, d,
                                        ctypes.c_double, d]
        _LIB = L
    return _LIB


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def lines_from_arrays(line_const, line_ncomp, line_pattern):
    """sno_line array from the fixture arrays (line_const [n,8], ncomp [n,3], pattern [n,3,2,16])."""
    n = line_const.shape[0]
    arr = (SnoLine * n)()
    for j in range(n):
        L = arr[j]
        L.lam0, L.sf, L.ar, L.mass = (float(v) for v in line_const[j, :4])
        L.split = int(line_const[j, 5])
        for g in range(3):
            L.ncomp[g] = int(line_ncomp[j, g])
            for i in range(MAXCOMP):
                L.S[g][i] = float(line_pattern[j, g, 0, i])
                L.D[g][i] = float(line_pattern[j, g, 1, i])
    return arr


def voigt(x, a):
    H = ctypes.c_double()
    F = ctypes.c_double()
    lib().sno_voigt(float(x), float(a), ctypes.byref(H), ctypes.byref(F))
    return H.value, F.value


def zeeman_pattern(ju2, jl2, gu, gl):
    L = SnoLine()
    lib().sno_zeeman_pattern(int(ju2), int(jl2), float(gu), float(gl), ctypes.byref(L))
    return L


def airtovac(lam_air_cm):
    return lib().sno_airtovac(float(lam_air_cm))


def opacity(rec_k, lines, lam_vac, lam_mid):
    rec_k = np.ascontiguousarray(rec_k, dtype=np.float64)
    op = np.zeros(16)
    em = np.zeros(4)
    lib().sno_opacity(_p(rec_k), len(lines), lines, float(lam_vac), float(lam_mid), _p(op), _p(em))
    return op.reshape(4, 4), em


def synth(lam_air, tau500, records, lines, ct=-1.0):
    """records [npix, nd, nfield] -> stokes [npix, nl, 4] (FP64)."""
    lam_air = np.ascontiguousarray(lam_air, dtype=np.float64)
    tau500 = np.ascontiguousarray(tau500, dtype=np.float64)
    rec = np.ascontiguousarray(records, dtype=np.float64)
    npix, nd, _ = rec.shape
    nl = lam_air.shape[0]
    out = np.zeros((npix, nl, 4))
    lib().sno_synth_batch(npix, nd, nl, _p(lam_air), _p(tau500), _p(rec), len(lines), lines, float(ct),
                          _p(out))
    return out


def chi2_grad_fd(lam_air, tau500, record, lines, obs, ws, mask, tangent, step, ct=-1.0):
    """Central-difference chi2 gradient along tangent directions [npar, nd, nfield]."""
    lam_air = np.ascontiguousarray(lam_air, dtype=np.float64)
    tau500 = np.ascontiguousarray(tau500, dtype=np.float64)
    rec = np.ascontiguousarray(record, dtype=np.float64)
    obs = np.ascontiguousarray(obs, dtype=np.float64)
    ws = np.ascontiguousarray(ws, dtype=np.float64)
    mask = np.ascontiguousarray(mask, dtype=np.float64)
    tan = np.ascontiguousarray(tangent, dtype=np.float64)
    nd = rec.shape[0]
    nl = lam_air.shape[0]
    npar = tan.shape[0]
    chi2 = ctypes.c_double()
    grad = np.zeros(npar)
    lib().sno_chi2_grad_fd(nd, nl, _p(lam_air), _p(tau500), _p(rec), len(lines), lines, float(ct),
                           _p(obs), _p(ws), _p(mask), npar, _p(tan), float(step), ctypes.byref(chi2),
                           _p(grad))
    return chi2.value, grad


def stokes_jvp_fd(lam_air, tau500, record, lines, tangent, step, ct=-1.0):
    lam_air = np.ascontiguousarray(lam_air, dtype=np.float64)
    tau500 = np.ascontiguousarray(tau500, dtype=np.float64)
    rec = np.ascontiguousarray(record, dtype=np.float64)
    tan = np.ascontiguousarray(tangent, dtype=np.float64)
    nd = rec.shape[0]
    nl = lam_air.shape[0]
    npar = tan.shape[0]
    dS = np.zeros((npar, nl, 4))
    lib().sno_stokes_jvp_fd(nd, nl, _p(lam_air), _p(tau500), _p(rec), len(lines), lines, float(ct), npar,
                            _p(tan), float(step), _p(dS))
    return dS
