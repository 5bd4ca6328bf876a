"""ctypes mirror of the node-model tables of include/snapi_cuda.h (snapi_eos_model and its parts) and
their assembly from flat arrays.

The arrays are what a caller reads from its atom / molecule / model objects (the reference:
atom::abund, ip, partf, nl, g, ee, bf; mol components and equilibrium constants; the node model).
Array layout (S = SNAPI_EOS_MAX_STAGES, T = SNAPI_PF_MAX_TERMS, C = SNAPI_PF_MAX_COEF,
L = SNAPI_EOS_MAX_LEVELS):
  meta [13]       natom, nmol, nlines, npar, nd, tau_min, tau_max, theta, phi, lambda_he,
                  lambda_kappa, grav, nlambda
  atom_f [na][4]  abundance, nstage, nlte, mass;        atom_ip [na][S]
  pf_type, pf_value, pf_zeff, pf_g0, pf_nterm, pf_ncoef [na][S]; pf_m, pf_g2, pf_ee, pf_ll [na][S][T];
  pf_gam, pf_a [na][S][T][C]; pf_coef [na][S][C]
  lev_n [na][S];  lev [na][S][L][6]  g, ee, sigma_he, sigma_kappa, sigma_win, lambda_win
  mol_i [nm][11]  ncomp, comp_atom[4], comp_charge[4], eqc, ncoef;  mol_coef [nm][C]
  line_eos [nlines][9]  atom, stage, lower, upper, Blu, Bul, A, alpha_col, sigma_col
  node_kind [npar], node_tau [npar]
"""
import ctypes

import numpy as np

MAX_ATOMS = 16
MAX_STAGES = 12
MAX_LEVELS = 16
MAX_MOLS = 32
MOL_MAX_COMP = 4
PF_MAX_TERMS = 8
PF_MAX_COEF = 8
MAX_PAR = 128

_d = ctypes.c_double
_i = ctypes.c_int


class SnapiPartition(ctypes.Structure):
    _fields_ = [("type", _i), ("nterm", _i), ("ncoef", _i), ("m", _i * PF_MAX_TERMS),
                ("value", _d), ("zeff", _d), ("g0", _d),
                ("g2", _d * PF_MAX_TERMS), ("ee", _d * PF_MAX_TERMS), ("ll", _d * PF_MAX_TERMS),
                ("gam", (_d * PF_MAX_COEF) * PF_MAX_TERMS), ("a", (_d * PF_MAX_COEF) * PF_MAX_TERMS),
                ("coef", _d * PF_MAX_COEF)]


class SnapiEosLevel(ctypes.Structure):
    _fields_ = [("g", _d), ("ee", _d), ("sigma_he", _d), ("sigma_kappa", _d), ("sigma_win", _d),
                ("lambda_win", _d)]


class SnapiEosAtom(ctypes.Structure):
    _fields_ = [("abundance", _d), ("nstage", _i), ("nlte", _i), ("ip", _d * MAX_STAGES),
                ("nlevel", _i * MAX_STAGES), ("pf", SnapiPartition * MAX_STAGES),
                ("level", (SnapiEosLevel * MAX_LEVELS) * MAX_STAGES)]


class SnapiEosMolecule(ctypes.Structure):
    _fields_ = [("ncomp", _i), ("comp_atom", _i * MOL_MAX_COMP), ("comp_charge", _i * MOL_MAX_COMP),
                ("eqc", _i), ("ncoef", _i), ("coef", _d * PF_MAX_COEF)]


class SnapiEosLine(ctypes.Structure):
    _fields_ = [("atom", _i), ("stage", _i), ("lower", _i), ("upper", _i), ("Blu", _d), ("Bul", _d), ("A", _d),
                ("alpha_col", _d), ("sigma_col", _d)]


class SnapiEosModel(ctypes.Structure):
    _fields_ = [("natom", _i), ("atoms", ctypes.POINTER(SnapiEosAtom)), ("nmol", _i),
                ("mols", ctypes.POINTER(SnapiEosMolecule)), ("lines", ctypes.POINTER(SnapiEosLine)),
                ("lambda_he", _d), ("lambda_kappa", _d), ("grav", _d), ("tau_min", _d), ("tau_max", _d),
                ("theta", _d), ("phi", _d), ("npar", _i), ("node_kind", ctypes.POINTER(_i)),
                ("node_tau", ctypes.POINTER(_d))]


class EosTables:
    """The tables of one node model as ctypes structures (kept alive by this object).

    d: mapping with the arrays listed in the module docstring (e.g. an npz of them)."""

    def __init__(self, d):
        meta = np.asarray(d["meta"], np.float64)
        na, nm, nlines, npar = int(meta[0]), int(meta[1]), int(meta[2]), int(meta[3])
        if na > MAX_ATOMS or nm > MAX_MOLS or npar > MAX_PAR:
            raise ValueError("node model tables exceed the library's limits")
        self.nd = int(meta[4])
        self.nlines = nlines
        self.npar = npar
        self.atoms = (SnapiEosAtom * na)()
        af = np.asarray(d["atom_f"], np.float64)
        for a in range(na):
            A = self.atoms[a]
            A.abundance = af[a, 0]
            A.nstage = int(af[a, 1])
            A.nlte = int(af[a, 2])
            for z in range(A.nstage):
                A.ip[z] = float(d["atom_ip"][a, z])
                A.nlevel[z] = int(d["lev_n"][a, z])
                P = A.pf[z]
                P.type = int(d["pf_type"][a, z])
                P.value = float(d["pf_value"][a, z])
                P.zeff = float(d["pf_zeff"][a, z])
                P.g0 = float(d["pf_g0"][a, z])
                P.nterm = int(d["pf_nterm"][a, z])
                P.ncoef = int(d["pf_ncoef"][a, z])
                for t in range(P.nterm):
                    P.m[t] = int(d["pf_m"][a, z, t])
                    P.g2[t] = float(d["pf_g2"][a, z, t])
                    P.ee[t] = float(d["pf_ee"][a, z, t])
                    P.ll[t] = float(d["pf_ll"][a, z, t])
                    for c in range(P.m[t]):
                        P.gam[t][c] = float(d["pf_gam"][a, z, t, c])
                        P.a[t][c] = float(d["pf_a"][a, z, t, c])
                for c in range(P.ncoef):
                    P.coef[c] = float(d["pf_coef"][a, z, c])
                for lv in range(A.nlevel[z]):
                    L = A.level[z][lv]
                    (L.g, L.ee, L.sigma_he, L.sigma_kappa, L.sigma_win, L.lambda_win) = (
                        float(v) for v in d["lev"][a, z, lv])
        self.mols = (SnapiEosMolecule * max(nm, 1))()
        mi = np.asarray(d["mol_i"]).reshape(nm, 11) if nm else np.zeros((0, 11))
        for k in range(nm):
            M = self.mols[k]
            M.ncomp = int(mi[k, 0])
            for c in range(M.ncomp):
                M.comp_atom[c] = int(mi[k, 1 + c])
                M.comp_charge[c] = int(mi[k, 5 + c])
            M.eqc = int(mi[k, 9])
            M.ncoef = int(mi[k, 10])
            for c in range(M.ncoef):
                M.coef[c] = float(d["mol_coef"][k, c])
        self.lines = (SnapiEosLine * max(nlines, 1))()
        le = np.asarray(d["line_eos"], np.float64).reshape(nlines, 9) if nlines else np.zeros((0, 9))
        for j in range(nlines):
            L = self.lines[j]
            L.atom, L.stage, L.lower, L.upper = (int(v) for v in le[j, :4])
            L.Blu, L.Bul, L.A, L.alpha_col, L.sigma_col = (float(v) for v in le[j, 4:])
        self.node_kind = np.ascontiguousarray(d["node_kind"], dtype=np.int32)
        self.node_tau = np.ascontiguousarray(d["node_tau"], dtype=np.float64)
        m = SnapiEosModel()
        m.natom = na
        m.atoms = ctypes.cast(self.atoms, ctypes.POINTER(SnapiEosAtom))
        m.nmol = nm
        m.mols = ctypes.cast(self.mols, ctypes.POINTER(SnapiEosMolecule))
        m.lines = ctypes.cast(self.lines, ctypes.POINTER(SnapiEosLine))
        m.lambda_he, m.lambda_kappa, m.grav = float(meta[9]), float(meta[10]), float(meta[11])
        m.tau_min, m.tau_max = float(meta[5]), float(meta[6])
        m.theta, m.phi = float(meta[7]), float(meta[8])
        m.npar = npar
        m.node_kind = self.node_kind.ctypes.data_as(ctypes.POINTER(_i))
        m.node_tau = self.node_tau.ctypes.data_as(ctypes.POINTER(_d))
        self.model = m

    def tau500(self):
        lt = self.model.tau_min + (self.model.tau_max - self.model.tau_min) / (self.nd - 1) * np.arange(self.nd)
        return 10.0 ** lt

    def pointer(self):
        return ctypes.byref(self.model)
