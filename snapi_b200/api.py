"""Python host mirror of the C ABI of libsnapi_cuda (include/snapi_cuda.h).

The calls mirror the reference's per-pixel entry points (atmos/atmos.h):
  Context.synth       ~ atmosphere::obs_stokes(theta, phi, lambda, nlambda)
  Context.adjoint     ~ chi2 and d chi2 / d nodes of atmosphere::stokes_lm_fit's inner loop,
                        evaluated by reverse mode instead of obs_stokes_responses_to_nodes
  Context.responses   ~ atmosphere::obs_stokes_responses_to_nodes
  Context.fd_grad     ~ the plain finite-difference gradient the adjoint replaces
but batched over pixels.  Arrays are numpy (host) or raw device pointers (int) with mem=DEVICE.
Errors raise SnapiError with the library's message; there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SNAPI_LIB", os.path.join(_PKG, "libsnapi_cuda.so"))

OK, EINVAL, ECUDA, ETIMEOUT, ENONCONV, ENOMEM = 0, -1, -2, -3, -4, -5
MEM_HOST, MEM_DEVICE = 0, 1
CHEM_START_CONTINUE, CHEM_START_COLD = 0, 1  # SNAPI_CHEM_START_*
JACOBIAN_FD, JACOBIAN_TANGENT = 0, 1  # SNAPI_JACOBIAN_*
NFIELD0 = 12
MAX_LINES = 16  # SNAPI_MAX_LINES
MAX_COMP = 16

# record field indices (include/snapi_cuda.h)
F_T, F_VT, F_NE, F_VLOS, F_B, F_INC, F_AZI, F_KAP, F_HMBF, F_HMFF, F_BFOP, F_BFEM = range(12)
FIELD_NAMES = ["T", "vt", "ne", "vlos", "B", "inc", "azi", "kap500", "hm_bf", "hm_ff", "bf_op", "bf_em"]


class SnapiError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("snapi error %d: %s" % (code, msg))
        self.code = code


class SnapiLine(ctypes.Structure):
    """Mirror of snapi_line."""
    _fields_ = [
        ("lam0", ctypes.c_double),
        ("sf", ctypes.c_double),
        ("ar", ctypes.c_double),
        ("mass", ctypes.c_double),
        ("split", ctypes.c_int),
        ("ncomp", ctypes.c_int * 3),
        ("S", (ctypes.c_double * MAX_COMP) * 3),
        ("D", (ctypes.c_double * MAX_COMP) * 3),
    ]


class SnapiProblem(ctypes.Structure):
    _fields_ = [
        ("nd", ctypes.c_int),
        ("nlambda", ctypes.c_int),
        ("nlines", ctypes.c_int),
        ("lambda_air", ctypes.POINTER(ctypes.c_double)),
        ("tau500", ctypes.POINTER(ctypes.c_double)),
        ("mu", ctypes.c_double),
        ("lines", ctypes.POINTER(SnapiLine)),
        ("stokes_scale", ctypes.c_double),
        ("max_batch", ctypes.c_int),
    ]


class SnapiLmOpts(ctypes.Structure):
    _fields_ = [
        ("npar", ctypes.c_int),
        ("node_kind", ctypes.POINTER(ctypes.c_int)),
        ("lm_start", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("delta", ctypes.c_double),
        ("stopping_chisq", ctypes.c_double),
        ("resp_step", ctypes.POINTER(ctypes.c_double)),
        ("spectral_broadening", ctypes.c_double),
    ]


F0_INT8, F0_INT16, F0_INT32, F0_FLOAT32, F0_FLOAT64, F0_INT64 = range(6)
F0_DTYPES = [np.int8, np.int16, np.int32, np.float32, np.float64, np.int64]


class F0Info(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int),
        ("ndim", ctypes.c_int),
        ("dim", ctypes.c_longlong * 16),
        ("nelem", ctypes.c_longlong),
        ("data_offset", ctypes.c_longlong),
        ("nhb", ctypes.c_int),
        ("swap", ctypes.c_int),
        ("compressed", ctypes.c_int),
        ("reversed_synch", ctypes.c_int),
        ("header", ctypes.c_char * (15 * 256 + 1)),
    ]


class CubeJob(ctypes.Structure):
    _fields_ = [
        ("obs_path", ctypes.c_char_p),
        ("xl", ctypes.c_int), ("xh", ctypes.c_int), ("yl", ctypes.c_int), ("yh", ctypes.c_int),
        ("ll", ctypes.c_int), ("lh", ctypes.c_int),
        ("obs_qs", ctypes.c_double), ("synth_qs", ctypes.c_double),
        ("nodes0", ctypes.c_void_p),
        ("model_path", ctypes.c_char_p),
        ("mask", ctypes.c_void_p),
        ("w_stokes", ctypes.c_void_p),
        ("out_nodes", ctypes.c_char_p), ("out_spectra", ctypes.c_char_p), ("out_cube", ctypes.c_char_p),
        ("chi2", ctypes.c_void_p),
        ("iters", ctypes.c_void_p),
        ("chunk", ctypes.c_int),
        ("out_atmos", ctypes.c_char_p),
        ("x3", ctypes.c_void_p),
    ]


class CubeStats(ctypes.Structure):
    _fields_ = [
        ("pixels", ctypes.c_longlong), ("chunks", ctypes.c_longlong), ("lm_steps", ctypes.c_longlong),
        ("wall_s", ctypes.c_double), ("fit_s", ctypes.c_double), ("read_wait_s", ctypes.c_double),
        ("write_wait_s", ctypes.c_double), ("bytes_read", ctypes.c_longlong), ("bytes_written", ctypes.c_longlong),
        ("kernel_ms", ctypes.c_double), ("launches", ctypes.c_int), ("flagged", ctypes.c_longlong),
    ]


class CubeSynthJob(ctypes.Structure):
    _fields_ = [
        ("atmos_path", ctypes.c_char_p),
        ("xl", ctypes.c_int), ("xh", ctypes.c_int), ("yl", ctypes.c_int), ("yh", ctypes.c_int),
        ("out_spectra", ctypes.c_char_p),
        ("stokes", ctypes.c_void_p),
        ("chunk", ctypes.c_int),
        ("ali", ctypes.c_void_p), ("ali_prob", ctypes.c_void_p), ("ali_tables", ctypes.c_void_p),
        ("line_level", ctypes.c_void_p), ("ali_max_iter", ctypes.c_int), ("ali_tol", ctypes.c_double),
    ]


_LIB = None


def lib():
    """Load libsnapi_cuda.so (raises if it was not built: there is no fallback)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libsnapi_cuda.so is missing: run `python -m snapi_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        vp, dp, fp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p, ctypes.c_int
        L.snapi_create.restype = vp
        L.snapi_create.argtypes = [ctypes.POINTER(SnapiProblem), ip, ctypes.POINTER(ctypes.c_int)]
        L.snapi_destroy.argtypes = [vp]
        L.snapi_last_error.restype = ctypes.c_char_p
        L.snapi_last_error.argtypes = [vp]
        L.snapi_synth.argtypes = [vp, ip, fp, fp, ip]
        L.snapi_adjoint.argtypes = [vp, ip, fp, fp, fp, fp, ip, fp, fp, fp, fp, fp, ip]
        L.snapi_responses.argtypes = [vp, ip, fp, ip, fp, fp, fp, fp, ip]
        L.snapi_fd_grad.argtypes = [vp, ip, fp, fp, fp, fp, ip, fp, fp, fp, fp, ip]
        L.snapi_adjoint_packed.argtypes = [vp, ip, fp, fp, fp, fp, ip, fp, fp, fp, fp, fp, ip]
        L.snapi_spectral_broaden.argtypes = [vp, ip, fp, ctypes.c_double, ip]
        L.snapi_eos_set.argtypes = [vp, vp]
        L.snapi_eos_chem_start.argtypes = [vp, ip]
        L.snapi_adjoint_nodes.argtypes = [vp, ip, fp, fp, fp, fp, fp, fp, fp, fp, ip]
        L.snapi_fma_peak.argtypes = [ip, ip, ctypes.POINTER(ctypes.c_double)]
        L.snapi_lm_step_jacobian.argtypes = [vp, fp, fp, fp, fp, ctypes.POINTER(ctypes.c_int), ip]
        L.snapi_last_phase_ms.restype = ctypes.c_double
        L.snapi_last_phase_ms.argtypes = [vp, ip]
        L.snapi_autotune.argtypes = [vp, ip, ctypes.c_char_p]
        L.snapi_jacobian_mode.argtypes = [vp, ip]
        L.snapi_tuned_config.argtypes = [vp, ip, fp]
        L.snapi_build_records.argtypes = [vp, ip, fp, fp, fp, fp, fp, fp, fp, ip]
        L.snapi_build_atmos.argtypes = [vp, ip, fp, fp, fp, fp, fp, ip]
        L.snapi_records_from_columns.argtypes = [vp, ip, fp, fp, fp, ip]
        L.snapi_lm_fit.argtypes = [vp, ip, ctypes.POINTER(SnapiLmOpts), fp, fp, fp, fp, fp, fp, fp, fp,
                                   ctypes.POINTER(ctypes.c_int), ip]
        L.snapi_zeeman_pattern.argtypes = [ip, ip, ctypes.c_double, ctypes.c_double, ctypes.POINTER(SnapiLine)]
        L.snapi_host_alloc.restype = vp
        L.snapi_host_alloc.argtypes = [ctypes.c_size_t]
        L.snapi_host_free.argtypes = [vp]
        L.snapi_stream.restype = vp
        L.snapi_stream.argtypes = [vp]
        L.snapi_last_kernel_ms.restype = ctypes.c_double
        L.snapi_last_kernel_ms.argtypes = [vp]
        L.snapi_last_launches.restype = ip
        L.snapi_last_launches.argtypes = [vp]
        L.snapi_lm_begin.argtypes = [vp, ip, ctypes.POINTER(SnapiLmOpts), fp, fp, fp, fp, fp, ip]
        L.snapi_lm_step.argtypes = [vp, fp, fp, fp, fp, ctypes.POINTER(ctypes.c_int), ip]
        L.snapi_lm_result.argtypes = [vp, fp, fp, fp, fp, ip]
        ll = ctypes.c_longlong
        L.snapi_f0_stat.argtypes = [ctypes.c_char_p, ctypes.POINTER(F0Info)]
        L.snapi_f0_read.argtypes = [ctypes.c_char_p, ll, ll, vp, ip]
        L.snapi_f0_write.argtypes = [ctypes.c_char_p, vp, ip, ip, ctypes.POINTER(ll), ctypes.c_char_p]
        L.snapi_f0_create.restype = vp
        L.snapi_f0_create.argtypes = [ctypes.c_char_p, ip, ip, ctypes.POINTER(ll), ctypes.c_char_p,
                                      ctypes.POINTER(ctypes.c_int)]
        L.snapi_f0_write_at.argtypes = [vp, ll, ll, vp]
        L.snapi_f0_close.argtypes = [vp]
        L.snapi_f0_error.restype = ctypes.c_char_p
        L.snapi_f0_error.argtypes = []
        L.snapi_cube_invert.argtypes = [vp, ctypes.POINTER(SnapiLmOpts), ctypes.POINTER(CubeJob),
                                        ctypes.POINTER(CubeStats)]
        L.snapi_cube_synth.argtypes = [vp, ctypes.POINTER(CubeSynthJob), ctypes.POINTER(CubeStats)]
        _LIB = L
    return _LIB


def fma_peak(device=0, fp64=False):
    """Measured FMA peak of GPU `device` [TFLOP/s] (snapi_fma_peak): FP32, or FP64 with fp64."""
    out = ctypes.c_double(0.0)
    rc = lib().snapi_fma_peak(int(device), 1 if fp64 else 0, ctypes.byref(out))
    if rc != 0:
        raise SnapiError(rc, "snapi_fma_peak failed")
    return out.value


def zeeman_pattern(ju2, jl2, g_upper, g_lower):
    line = SnapiLine()
    rc = lib().snapi_zeeman_pattern(int(ju2), int(jl2), float(g_upper), float(g_lower), ctypes.byref(line))
    if rc != OK:
        raise SnapiError(rc, "zeeman_pattern")
    return line


def lines_from_arrays(line_const, line_ncomp, line_pattern):
    """snapi_line array from arrays: line_const [n, >=6] = (lam0, sf, ar, mass, A, split),
    line_ncomp [n, 3], line_pattern [n, 3, 2, 16] (strengths, shifts)."""
    n = int(line_const.shape[0])
    arr = (SnapiLine * max(n, 1))()
    for j in range(n):
        L = arr[j]
        L.lam0, L.sf, L.ar, L.mass = (float(v) for v in line_const[j, :4])
        L.split = int(line_const[j, 5])
        for g in range(3):
            L.ncomp[g] = int(line_ncomp[j, g])
            for i in range(MAX_COMP):
                L.S[g][i] = float(line_pattern[j, g, 0, i])
                L.D[g][i] = float(line_pattern[j, g, 1, i])
    return arr, n


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, int):
        return ctypes.c_void_p(a)
    return ctypes.c_void_p(a.ctypes.data)


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


def tangent_field_mask(tangents):
    """Per node, the bit mask of record fields its tangent touches anywhere in the batch:
    tangents [npix, npar, nd, nfield] -> uint64 [npar]."""
    nz = (np.asarray(tangents) != 0).any(axis=(0, 2))
    return np.array([sum(1 << int(f) for f in np.flatnonzero(nz[p])) for p in range(nz.shape[0])], dtype=np.uint64)


def pack_tangents(tangents, field_mask):
    """Dense tangents [npix, npar, nd, nfield] -> packed [npix, ntcol, nd] (node by node, fields in
    increasing order), the layout of snapi_adjoint_packed."""
    t = np.asarray(tangents)
    cols = []
    for p, m in enumerate(np.asarray(field_mask, dtype=np.uint64)):
        for f in range(t.shape[3]):
            if (int(m) >> f) & 1:
                cols.append(t[:, p, :, f])
    return np.ascontiguousarray(np.stack(cols, axis=1), dtype=np.float32)


def _f0_check(rc):
    if rc != 0:
        raise SnapiError(rc, lib().snapi_f0_error().decode())


def f0_stat(path):
    """Header of an ANA .f0 file (snapi_f0_stat): dict of type, dims (fastest first), header, ..."""
    info = F0Info()
    _f0_check(lib().snapi_f0_stat(os.fsencode(path), ctypes.byref(info)))
    return {"type": info.type, "dims": tuple(info.dim[d] for d in range(info.ndim)), "nelem": info.nelem,
            "data_offset": info.data_offset, "nhb": info.nhb, "swap": info.swap, "compressed": info.compressed,
            "reversed_synch": info.reversed_synch, "header": info.header.decode("latin-1")}


def f0_read(path, out_type=None, first=0, count=None):
    """Elements of an .f0 file as a numpy array shaped like the reference's C array (slowest dimension
    first), or a flat range [first, first + count) when count is given."""
    h = f0_stat(path)
    t = h["type"] if out_type is None else out_type
    n = h["nelem"] - first if count is None else count
    out = np.empty(n, F0_DTYPES[t])
    _f0_check(lib().snapi_f0_read(os.fsencode(path), first, n, out.ctypes.data, t))
    if count is None and first == 0:
        out = out.reshape(tuple(reversed(h["dims"])))
    return out


def f0_write(path, data, header=None, type=None):
    """Write an array as the reference's ana_fzwrite does (dims reversed: the last axis varies fastest)."""
    a = np.ascontiguousarray(data)
    t = F0_DTYPES.index(a.dtype.type) if type is None else type
    if 0 <= t < len(F0_DTYPES):
        a = np.ascontiguousarray(a, dtype=F0_DTYPES[t])
    dims = (ctypes.c_longlong * a.ndim)(*reversed(a.shape))
    hb = None if header is None else header.encode("latin-1")
    _f0_check(lib().snapi_f0_write(os.fsencode(path), a.ctypes.data, t, a.ndim, dims, hb))


class Context:
    """A libsnapi_cuda context for one problem geometry (depth grid, wavelengths, line list)."""

    def __init__(self, lambda_air, tau500, lines, nlines, mu=1.0, stokes_scale=1.0, max_batch=4096, device=0):
        self._lam = np.ascontiguousarray(lambda_air, dtype=np.float64)
        self._tau = np.ascontiguousarray(tau500, dtype=np.float64)
        self._lines = lines
        self.nd = int(self._tau.shape[0])
        self.nl = int(self._lam.shape[0])
        self.nlines = int(nlines)
        self.nfield = NFIELD0 + 3 * self.nlines
        prob = SnapiProblem()
        prob.nd, prob.nlambda, prob.nlines = self.nd, self.nl, self.nlines
        prob.lambda_air = self._lam.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        prob.tau500 = self._tau.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        prob.mu = float(mu)
        prob.lines = ctypes.cast(lines, ctypes.POINTER(SnapiLine))
        prob.stokes_scale = float(stokes_scale)
        prob.max_batch = int(max_batch)
        st = ctypes.c_int(0)
        self._ctx = lib().snapi_create(ctypes.byref(prob), int(device), ctypes.byref(st))
        if not self._ctx:
            raise SnapiError(st.value, "snapi_create failed")

    @classmethod
    def from_fixture(cls, fx, **kw):
        """Context from a fixture / problem dict (lambda_air, tau500, line_const, line_ncomp, line_pattern)."""
        lines, n = lines_from_arrays(fx["line_const"], fx["line_ncomp"], fx["line_pattern"])
        return cls(fx["lambda_air"], fx["tau500"], lines, n, **kw)

    def close(self):
        if getattr(self, "_ctx", None):
            lib().snapi_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != OK:
            raise SnapiError(rc, lib().snapi_last_error(self._ctx).decode())

    @property
    def stream(self):
        return lib().snapi_stream(self._ctx)

    @property
    def last_kernel_ms(self):
        return lib().snapi_last_kernel_ms(self._ctx)

    @property
    def last_phase_ms(self):
        """(node build, adjoint) device time [ms] of the last adjoint_nodes call."""
        return lib().snapi_last_phase_ms(self._ctx, 0), lib().snapi_last_phase_ms(self._ctx, 1)

    @property
    def last_launches(self):
        return lib().snapi_last_launches(self._ctx)

    def _npix(self, records):
        r = np.asarray(records)
        if r.ndim != 3 or r.shape[1] != self.nd or r.shape[2] != self.nfield:
            raise ValueError("records must be [npix, %d, %d]" % (self.nd, self.nfield))
        return r.shape[0]

    # --- host-memory API ------------------------------------------------------------------
    def synth(self, records):
        """Stokes [npix, nlambda, 4] from records [npix, nd, nfield] (obs_stokes, batched)."""
        rec = _f32(records)
        npix = self._npix(rec)
        out = np.zeros((npix, self.nl, 4), np.float32)
        self._check(lib().snapi_synth(self._ctx, npix, _ptr(rec), _ptr(out), MEM_HOST))
        return out

    def adjoint(self, records, obs, tangents=None, w_stokes=(1.0, 1.0, 1.0, 1.0), mask=None, want_stokes=True,
                want_rec_grad=False, out=None):
        """chi2 [npix], d chi2/d node [npix, npar] (and Stokes, d chi2 / d record) by one forward and
        one reverse sweep.  out: optional dict of preallocated "stokes" / "chi2" / "grad" arrays
        (e.g. page-locked from snapi_host_alloc) that receive the results."""
        rec = _f32(records)
        npix = self._npix(rec)
        ob = _f32(obs)
        tn = _f32(tangents)
        npar = 0 if tn is None else tn.shape[1]
        mk = _f32(mask)
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        out = out or {}
        st = out.get("stokes", np.zeros((npix, self.nl, 4), np.float32)) if want_stokes else None
        chi2 = out.get("chi2", np.zeros(npix))
        grad = out.get("grad", np.zeros((npix, max(npar, 1))))
        assert st is None or (st.dtype == np.float32 and st.flags.c_contiguous and st.size == npix * self.nl * 4)
        assert chi2.dtype == np.float64 and chi2.size == npix and grad.dtype == np.float64
        assert grad.flags.c_contiguous and grad.size >= npix * max(npar, 1)
        rg = np.zeros((npix, self.nd, self.nfield)) if want_rec_grad else None
        self._check(lib().snapi_adjoint(self._ctx, npix, _ptr(rec), _ptr(ob), _ptr(ws), _ptr(mk), npar, _ptr(tn),
                                        _ptr(st), _ptr(chi2), _ptr(grad), _ptr(rg), MEM_HOST))
        res = {"chi2": chi2, "grad": grad.reshape(npix, -1)[:, :npar]}
        if want_stokes:
            res["stokes"] = st
        if want_rec_grad:
            res["rec_grad"] = rg
        return res

    def fd_grad(self, records, obs, tangents, step, w_stokes=(1.0, 1.0, 1.0, 1.0), mask=None):
        rec = _f32(records)
        npix = self._npix(rec)
        ob = _f32(obs)
        tn = _f32(tangents)
        npar = tn.shape[1]
        mk = _f32(mask)
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        stp = np.ascontiguousarray(np.broadcast_to(step, (npar,)), dtype=np.float64)
        chi2 = np.zeros(npix)
        grad = np.zeros((npix, npar))
        self._check(lib().snapi_fd_grad(self._ctx, npix, _ptr(rec), _ptr(ob), _ptr(ws), _ptr(mk), npar, _ptr(tn),
                                        _ptr(stp), _ptr(chi2), _ptr(grad), MEM_HOST))
        return {"chi2": chi2, "grad": grad}

    # ---- batched Levenberg-Marquardt (stokes_lm_fit) ----------------------------------------
    def lm_begin(self, nodes0, obs, node_kind, resp_step, mask=None, w_stokes=(1.0, 1.0, 1.0, 1.0), lm_start=1e3,
                 max_iter=30, delta=1e-3, stopping_chisq=1e-30, spectral_broadening=0.0):
        """Start a fit of every pixel; returns the (bracketed) node vectors to build first."""
        n0 = np.ascontiguousarray(nodes0, dtype=np.float64)
        npix, npar = n0.shape
        ob = _f32(obs)
        mk = None if mask is None else _f32(mask)
        self._lm_kind = np.ascontiguousarray(node_kind, dtype=np.int32)
        self._lm_step = np.ascontiguousarray(np.broadcast_to(resp_step, (npar,)), dtype=np.float64)
        opts = SnapiLmOpts(npar, self._lm_kind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), float(lm_start),
                           int(max_iter), float(delta), float(stopping_chisq),
                           self._lm_step.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), float(spectral_broadening))
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        req = np.zeros_like(n0)
        self._check(lib().snapi_lm_begin(self._ctx, npix, ctypes.byref(opts), _ptr(n0), _ptr(ob), _ptr(ws), _ptr(mk),
                                         _ptr(req), MEM_HOST))
        self._lm_shape = (npix, npar)
        return req

    def lm_step(self, records, tangents, jacobian=False):
        """One LM iteration for every active pixel, from the records / tangents of the node vectors
        the previous call requested (jacobian: `tangents` is instead the caller's dS/dnode
        [npix, npar, nlambda, 4], snapi_lm_step_jacobian).  Returns (request, active, n_active)."""
        rec = _f32(records)
        tn = _f32(tangents)
        req = np.zeros(self._lm_shape)
        act = np.zeros(self._lm_shape[0], np.int32)
        na = ctypes.c_int(0)
        fn = lib().snapi_lm_step_jacobian if jacobian else lib().snapi_lm_step
        self._check(fn(self._ctx, _ptr(rec), _ptr(tn), _ptr(req), _ptr(act), ctypes.byref(na), MEM_HOST))
        return req, act.astype(bool), na.value

    def lm_result(self):
        npix, npar = self._lm_shape
        nodes = np.zeros((npix, npar))
        chi2 = np.zeros(npix)
        iters = np.zeros(npix, np.int32)
        st = np.zeros((npix, self.nl, 4), np.float32)
        self._check(lib().snapi_lm_result(self._ctx, _ptr(nodes), _ptr(chi2), _ptr(iters), _ptr(st), MEM_HOST))
        return {"nodes": nodes, "chi2": chi2, "iters": iters, "stokes": st}

    def lm_fit_device(self, nodes0, obs, node_kind, resp_step, mask=None, w_stokes=(1.0, 1.0, 1.0, 1.0), lm_start=1e3,
                      max_iter=30, delta=1e-3, stopping_chisq=1e-30, spectral_broadening=0.0):
        """The whole fit with the node -> record map on the GPU (snapi_lm_fit; needs eos_set)."""
        n0 = np.ascontiguousarray(nodes0, dtype=np.float64)
        npix, npar = n0.shape
        ob = _f32(obs)
        mk = None if mask is None else _f32(mask)
        kind = np.ascontiguousarray(node_kind, dtype=np.int32)
        stp = np.ascontiguousarray(np.broadcast_to(resp_step, (npar,)), dtype=np.float64)
        opts = SnapiLmOpts(npar, kind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), float(lm_start), int(max_iter),
                           float(delta), float(stopping_chisq), stp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           float(spectral_broadening))
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        nodes = np.zeros((npix, npar))
        chi2 = np.zeros(npix)
        iters = np.zeros(npix, np.int32)
        st = np.zeros((npix, self.nl, 4), np.float32)
        steps = ctypes.c_int(0)
        self._check(lib().snapi_lm_fit(self._ctx, npix, ctypes.byref(opts), _ptr(n0), _ptr(ob), _ptr(ws), _ptr(mk),
                                       _ptr(nodes), _ptr(chi2), _ptr(iters), _ptr(st), ctypes.byref(steps), MEM_HOST))
        return {"nodes": nodes, "chi2": chi2, "iters": iters, "stokes": st, "steps": steps.value}

    def cube_invert(self, obs_path, node_kind, resp_step, nodes0=None, model_path=None, subfield=(0, 0, 0, 0),
                    window=(0, 0), obs_qs=0.0, synth_qs=0.0, mask=None, w_stokes=(1.0, 1.0, 1.0, 1.0),
                    out_nodes=None, out_spectra=None, out_cube=None, out_atmos=None, x3=None, chunk=0, lm_start=1e3,
                    max_iter=30, delta=1e-3, stopping_chisq=1e-30, spectral_broadening=0.0):
        """The master's invert job over an .f0 cube (snapi_cube_invert; needs eos_set).  subfield
        (xl, xh, yl, yh) and window (ll, lh) are 1-based inclusive, 0 = the cube's extent.  Returns the
        per-pixel chi2 and iterations (x major) and the job's statistics."""
        kind = np.ascontiguousarray(node_kind, dtype=np.int32)
        npar = kind.size
        stp = np.ascontiguousarray(np.broadcast_to(resp_step, (npar,)), dtype=np.float64)
        opts = SnapiLmOpts(npar, kind.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), float(lm_start), int(max_iter),
                           float(delta), float(stopping_chisq), stp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                           float(spectral_broadening))
        dims = f0_stat(obs_path)["dims"]
        nx_full, ny_full = (dims[3], dims[2]) if len(dims) == 4 else (1, 1)  # the library reports the shape
        xl, xh, yl, yh = subfield
        nx = (xh or nx_full) - (xl or 1) + 1
        ny = (yh or ny_full) - (yl or 1) + 1
        n0 = None if nodes0 is None else np.ascontiguousarray(nodes0, dtype=np.float64)
        mk = None if mask is None else _f32(mask)
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        chi2 = np.zeros(max(nx * ny, 1))
        iters = np.zeros(max(nx * ny, 1), np.int32)
        enc = lambda p: None if p is None else os.fsencode(p)
        h3 = None if x3 is None else np.ascontiguousarray(x3, dtype=np.float64)
        job = CubeJob(os.fsencode(obs_path), xl, xh, yl, yh, window[0], window[1], float(obs_qs), float(synth_qs),
                      _ptr(n0), enc(model_path), _ptr(mk), _ptr(ws), enc(out_nodes), enc(out_spectra), enc(out_cube),
                      _ptr(chi2), _ptr(iters), int(chunk), enc(out_atmos), _ptr(h3))
        stats = CubeStats()
        self._check(lib().snapi_cube_invert(self._ctx, ctypes.byref(opts), ctypes.byref(job), ctypes.byref(stats)))
        return {"chi2": chi2.reshape(nx, ny), "iters": iters.reshape(nx, ny),
                "stats": {k: getattr(stats, k) for k, _ in CubeStats._fields_}}

    def lm_fit(self, nodes0, obs, builder, node_kind, resp_step, jacobian=False, trace=None, **kw):
        """Run the fit to the end.  builder(nodes [n, npar], active [n] bool) returns (records,
        tangents) for all n rows (rows of inactive pixels may hold anything); with jacobian, (records,
        dS/dnode [n, npar, nlambda, 4]).  trace: optional list that receives every requested node
        array (the first is the bracketed start, then one trial per LM iteration)."""
        req = self.lm_begin(nodes0, obs, node_kind, resp_step, **kw)
        active = np.ones(req.shape[0], bool)
        steps = 0
        while True:
            if trace is not None:
                trace.append(req.copy())
            rec, tan = builder(req, active)
            req, active, n = self.lm_step(rec, tan, jacobian=jacobian)
            steps += 1
            if n == 0:
                break
        out = self.lm_result()
        out["steps"] = steps
        return out

    def broaden(self, spectra, width):
        """Gaussian instrumental broadening of [nvec, nlambda, 4] spectra (returns a new array)."""
        a = np.array(spectra, dtype=np.float32, order="C", copy=True)
        nvec = a.size // (self.nl * 4)
        self._check(lib().snapi_spectral_broaden(self._ctx, nvec, _ptr(a), float(width), MEM_HOST))
        return a

    def eos_set(self, tables):
        """Attach a node model (snapi_b200.eos_tables.EosTables) for build_records."""
        self._eos = tables  # keep the ctypes tables alive for the call
        self._check(lib().snapi_eos_set(self._ctx, ctypes.addressof(tables.model)))
        self._eos_npar = tables.npar

    def jacobian_mode(self, mode):
        """How responses and the LM Jacobian are formed: JACOBIAN_FD (central differences, default) or
        JACOBIAN_TANGENT (forward-mode sweeps, exact derivative of the FP32 synthesis)."""
        self._check(lib().snapi_jacobian_mode(self._ctx, int(mode)))

    def autotune(self, on=True, cache_path=None):
        """snapi_autotune: pick launch shapes by timing them on the first calls of each batch size
        (on), or use the compiled ones (off); cache_path: optional file shared across processes."""
        self._check(lib().snapi_autotune(self._ctx, 1 if on else 0,
                                         None if cache_path is None else str(cache_path).encode()))

    def tuned_config(self, npix):
        """(shapes dict, tuned bits) of snapi_tuned_config for a batch of npix pixels."""
        cfg = np.zeros(5, np.int32)
        bits = lib().snapi_tuned_config(self._ctx, int(npix), _ptr(cfg))
        keys = ("chunk", "optile", "he_threads", "var_threads", "rt128")
        return {k: int(v) for k, v in zip(keys, cfg)}, int(bits)

    def eos_chem_start(self, mode):
        """How the march's chemistry starts each solve: CHEM_START_CONTINUE (default; Newton from the
        previous solution of the same column) or CHEM_START_COLD (the reference's start every time)."""
        self._check(lib().snapi_eos_chem_start(self._ctx, int(mode)))

    def build_records(self, nodes, active=None, tangents=True, step=None, want_nt=False):
        """Column records [npix, nd, nfield] of node vectors [npix, npar] on the GPU (build_from_nodes +
        chemistry + the record set-up), with node tangents [npix, npar, nd, nfield] if `tangents`.
        Returns (records, tangents or None, Nt or None, pixel status)."""
        nodes = np.ascontiguousarray(np.atleast_2d(nodes), dtype=np.float64)
        npix, npar = nodes.shape
        if npar != self._eos_npar:
            raise ValueError("node vectors have %d entries, the model %d" % (npar, self._eos_npar))
        rec = np.zeros((npix, self.nd, self.nfield), np.float32)
        tan = np.zeros((npix, npar, self.nd, self.nfield), np.float32) if tangents else None
        nt = np.zeros((npix, self.nd), np.float64) if want_nt else None
        act = None if active is None else np.ascontiguousarray(active, dtype=np.int32)
        stp = None if step is None else np.ascontiguousarray(np.broadcast_to(step, (npar,)), dtype=np.float64)
        status = np.zeros(npix, np.int32)
        self._check(lib().snapi_build_records(self._ctx, npix, _ptr(nodes), _ptr(act), _ptr(rec), _ptr(nt), _ptr(tan),
                                              _ptr(stp), _ptr(status), MEM_HOST))
        return rec, tan, nt, status

    def build_atmos(self, nodes, x3=None, active=None):
        """The 12 return_as_array rows of each node vector's column (snapi_build_atmos):
        atmos [npix][12][nd] float64 and the per-pixel status."""
        n = np.ascontiguousarray(nodes, dtype=np.float64)
        npix = n.shape[0]
        atm = np.zeros((npix, 12, self.nd))
        st = np.zeros(npix, np.int32)
        act = None if active is None else np.ascontiguousarray(active, dtype=np.int32)
        h3 = None if x3 is None else np.ascontiguousarray(x3, dtype=np.float64)
        self._check(lib().snapi_build_atmos(self._ctx, npix, _ptr(n), _ptr(act), _ptr(h3), _ptr(atm), _ptr(st),
                                            MEM_HOST))
        return atm, st

    def records_set_populations(self, records, pops, line_level):
        """The opacity / emissivity fields of the lines with line_level[j] = (lower, upper) >= 0 from
        level populations pops [npix][nd][nlevel] (snapi_records_set_populations; needs eos_set);
        returns a new records array."""
        rec = np.array(records, dtype=np.float32, order="C", copy=True)
        p = np.ascontiguousarray(pops, dtype=np.float64)
        ll = np.ascontiguousarray(line_level, dtype=np.int32)
        self._check(_pop_lib().snapi_records_set_populations(self._ctx, rec.shape[0], _ptr(rec), _ptr(p), p.shape[2],
                                                             _ptr(ll), MEM_HOST))
        return rec

    def records_from_columns(self, columns):
        """Records of atmosphere columns [npix][12][nd] in the snapi_build_atmos row layout
        (snapi_records_from_columns; needs eos_set): records [npix][nd][nfield] and the status."""
        c = np.ascontiguousarray(columns, dtype=np.float64)
        npix = c.shape[0]
        rec = np.zeros((npix, self.nd, self.nfield), np.float32)
        st = np.zeros(npix, np.int32)
        self._check(lib().snapi_records_from_columns(self._ctx, npix, _ptr(c), _ptr(rec), _ptr(st), MEM_HOST))
        return rec, st

    def cube_synth(self, atmos_path, subfield=(0, 0, 0, 0), out_spectra=None, chunk=0, want_stokes=True, ali=None,
                   ali_tables=None, line_level=None, ali_max_iter=0, ali_tol=0.0):
        """The synthesis branch of the master's job over an atmosphere .f0 cube (snapi_cube_synth):
        returns the Stokes vectors [nx][ny][nlambda][4] (if want_stokes) and the job's statistics.
        With an NLTE atom: ali (AliContext), ali_tables (AliSetupTables), line_level [nlines][2]."""
        dims = f0_stat(atmos_path)["dims"]
        nx_full, ny_full = (dims[2], dims[1]) if len(dims) == 4 else (1, 1)
        xl, xh, yl, yh = subfield
        nx = min(xh or nx_full, nx_full) - (xl or 1) + 1
        ny = min(yh or ny_full, ny_full) - (yl or 1) + 1
        st = np.zeros((max(nx, 1), max(ny, 1), self.nl, 4), np.float32) if want_stokes else None
        enc = lambda p: None if p is None else os.fsencode(p)
        ll = None if line_level is None else np.ascontiguousarray(line_level, dtype=np.int32)
        job = CubeSynthJob(os.fsencode(atmos_path), xl, xh, yl, yh, enc(out_spectra), _ptr(st), int(chunk),
                           ali._ctx if ali is not None else None,
                           ctypes.addressof(ali._prob) if ali is not None else None,
                           ctypes.addressof(ali_tables.tab) if ali_tables is not None else None, _ptr(ll),
                           int(ali_max_iter), float(ali_tol))
        stats = CubeStats()
        self._check(lib().snapi_cube_synth(self._ctx, ctypes.byref(job), ctypes.byref(stats)))
        return {"stokes": st, "stats": {k: getattr(stats, k) for k, _ in CubeStats._fields_}}

    def build_records_device(self, npix, nodes_ptr, rec_ptr, tan_ptr=0, active_ptr=0, status_ptr=0):
        """build_records on device pointers (int addresses, e.g. torch .data_ptr())."""
        p = lambda a: ctypes.c_void_p(a) if a else None  # noqa: E731
        self._check(lib().snapi_build_records(self._ctx, npix, p(nodes_ptr), p(active_ptr), p(rec_ptr), None,
                                              p(tan_ptr), None, p(status_ptr), MEM_DEVICE))

    def responses(self, records, tangents, step, want_stokes=True):
        """d Stokes / d node [npix, npar, nlambda, 4] (obs_stokes_responses_to_nodes, batched) by
        central differences of the records along the node tangents with steps `step` [npar]."""
        rec = _f32(records)
        npix = self._npix(rec)
        tn = _f32(tangents)
        npar = tn.shape[1]
        stp = np.ascontiguousarray(np.broadcast_to(step, (npar,)), dtype=np.float64)
        st = np.zeros((npix, self.nl, 4), np.float32) if want_stokes else None
        ds = np.zeros((npix, npar, self.nl, 4), np.float32)
        self._check(lib().snapi_responses(self._ctx, npix, _ptr(rec), npar, _ptr(tn), _ptr(stp), _ptr(st), _ptr(ds),
                                          MEM_HOST))
        return (st, ds) if want_stokes else ds

    # --- device-memory API (raw pointers, e.g. torch tensor .data_ptr()) --------------------
    def synth_device(self, npix, rec_ptr, stokes_ptr):
        self._check(lib().snapi_synth(self._ctx, int(npix), _ptr(int(rec_ptr)), _ptr(int(stokes_ptr)), MEM_DEVICE))

    def adjoint_device(self, npix, rec_ptr, obs_ptr, npar, tan_ptr, chi2_ptr, grad_ptr, stokes_ptr=None,
                       mask_ptr=None, w_stokes=(1.0, 1.0, 1.0, 1.0)):
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        self._check(lib().snapi_adjoint(self._ctx, int(npix), _ptr(int(rec_ptr)), _ptr(int(obs_ptr)), _ptr(ws),
                                        _ptr(int(mask_ptr)) if mask_ptr else None, int(npar), _ptr(int(tan_ptr)),
                                        _ptr(int(stokes_ptr)) if stokes_ptr else None, _ptr(int(chi2_ptr)),
                                        _ptr(int(grad_ptr)), None, MEM_DEVICE))

    def adjoint_packed_device(self, npix, rec_ptr, obs_ptr, field_mask, ptan_ptr, chi2_ptr, grad_ptr,
                              stokes_ptr=None, mask_ptr=None, w_stokes=(1.0, 1.0, 1.0, 1.0)):
        fm = np.ascontiguousarray(field_mask, dtype=np.uint64)
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        self._check(lib().snapi_adjoint_packed(self._ctx, int(npix), _ptr(int(rec_ptr)), _ptr(int(obs_ptr)), _ptr(ws),
                                               _ptr(int(mask_ptr)) if mask_ptr else None, len(fm), _ptr(fm),
                                               _ptr(int(ptan_ptr)), _ptr(int(stokes_ptr)) if stokes_ptr else None,
                                               _ptr(int(chi2_ptr)), _ptr(int(grad_ptr)), MEM_DEVICE))

    def adjoint_packed(self, records, obs, field_mask, packed_tangents, w_stokes=(1.0, 1.0, 1.0, 1.0), mask=None,
                       out=None):
        """snapi_adjoint with packed node tangents (see pack_tangents); host arrays."""
        rec = _f32(records)
        npix = self._npix(rec)
        ob = _f32(obs)
        pt = _f32(packed_tangents)
        mk = _f32(mask)
        fm = np.ascontiguousarray(field_mask, dtype=np.uint64)
        npar = len(fm)
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        out = out or {}
        st = out.get("stokes", np.zeros((npix, self.nl, 4), np.float32))
        chi2 = out.get("chi2", np.zeros(npix))
        grad = out.get("grad", np.zeros((npix, npar)))
        self._check(lib().snapi_adjoint_packed(self._ctx, npix, _ptr(rec), _ptr(ob), _ptr(ws), _ptr(mk), npar, _ptr(fm),
                                               _ptr(pt), _ptr(st), _ptr(chi2), _ptr(grad), MEM_HOST))
        return {"stokes": st, "chi2": chi2, "grad": grad.reshape(npix, npar)}

    def adjoint_nodes(self, nodes, obs, w_stokes=(1.0, 1.0, 1.0, 1.0), mask=None, out=None):
        """snapi_adjoint_nodes on host arrays: Stokes, chi2 and d chi2 / d node from node vectors
        [npix, npar] (records and tangents built on the device).  out: optional dict of
        preallocated (e.g. page-locked) result arrays "stokes", "chi2", "grad", "status"."""
        nodes = np.ascontiguousarray(np.atleast_2d(nodes), dtype=np.float64)
        npix, npar = nodes.shape
        if npar != self._eos_npar:
            raise ValueError("nodes have %d columns, the node model %d" % (npar, self._eos_npar))
        ob = _f32(obs)
        mk = _f32(mask)
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        out = out or {}
        st = out.get("stokes", np.zeros((npix, self.nl, 4), np.float32))
        chi2 = out.get("chi2", np.zeros(npix))
        grad = out.get("grad", np.zeros((npix, npar)))
        status = out.get("status", np.zeros(npix, np.int32))
        self._check(lib().snapi_adjoint_nodes(self._ctx, npix, _ptr(nodes), _ptr(ob), _ptr(ws), _ptr(mk), _ptr(st),
                                              _ptr(chi2), _ptr(grad), _ptr(status), MEM_HOST))
        return {"stokes": st, "chi2": chi2, "grad": grad, "status": status}

    def adjoint_nodes_device(self, npix, nodes_ptr, obs_ptr, chi2_ptr, grad_ptr, stokes_ptr=None, mask_ptr=None,
                             status_ptr=None, w_stokes=(1.0, 1.0, 1.0, 1.0)):
        """snapi_adjoint_nodes on device buffers (raw device pointers)."""
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        opt = lambda v: _ptr(int(v)) if v else None  # noqa: E731
        self._check(lib().snapi_adjoint_nodes(self._ctx, int(npix), _ptr(int(nodes_ptr)), _ptr(int(obs_ptr)), _ptr(ws),
                                              opt(mask_ptr), opt(stokes_ptr), _ptr(int(chi2_ptr)),
                                              _ptr(int(grad_ptr)), opt(status_ptr), MEM_DEVICE))

    def fd_grad_device(self, npix, rec_ptr, obs_ptr, npar, tan_ptr, step, chi2_ptr, grad_ptr,
                       w_stokes=(1.0, 1.0, 1.0, 1.0)):
        ws = np.ascontiguousarray(w_stokes, dtype=np.float64)
        stp = np.ascontiguousarray(np.broadcast_to(step, (npar,)), dtype=np.float64)
        self._check(lib().snapi_fd_grad(self._ctx, int(npix), _ptr(int(rec_ptr)), _ptr(int(obs_ptr)), _ptr(ws),
                                        None, int(npar), _ptr(int(tan_ptr)), _ptr(stp), _ptr(int(chi2_ptr)),
                                        _ptr(int(grad_ptr)), MEM_DEVICE))


# ---- NLTE level populations (snapi_ali_*) ---------------------------------------------------
class SnapiAliProblem(ctypes.Structure):
    _fields_ = [("nd", ctypes.c_int), ("nlambda", ctypes.c_int), ("nray", ctypes.c_int), ("nlevel", ctypes.c_int),
                ("ntrans", ctypes.c_int)] + [(n, ctypes.c_void_p) for n in (
                    "grid", "lambda_", "lambda_w", "fudge", "ray_theta", "ray_w", "trans", "line_c", "line_e", "A",
                    "B", "stage", "cont_of", "sigma")]


class SnapiAliColumns(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("T", "ne", "na", "kappa", "vray", "dld", "adamp", "bfratio", "coll",
                                               "bg_op", "bg_em")]


def _ali_lib():
    L = lib()
    if not getattr(L, "_ali_set", False):
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.snapi_ali_create.restype = vp
        L.snapi_ali_create.argtypes = [ctypes.POINTER(SnapiAliProblem), ip, ctypes.POINTER(ctypes.c_int)]
        L.snapi_ali_destroy.argtypes = [vp]
        L.snapi_ali_last_error.restype = ctypes.c_char_p
        L.snapi_ali_last_error.argtypes = [vp]
        L.snapi_ali_iter.argtypes = [vp, ip, ctypes.POINTER(SnapiAliColumns), vp, ip, ctypes.c_double, vp, vp, vp, ip]
        L.snapi_ali_last_kernel_ms.restype = ctypes.c_double
        L.snapi_ali_last_kernel_ms.argtypes = [vp]
        L._ali_set = True
    return L


class AliContext:
    """NLTE populations of one atom in many columns (atmosphere::nltepops, batched).

    transitions: [ntrans, 2] (lower, upper) level pairs; a pair whose upper level is the lower
    level's continuum (cont_of) is bound-free.  line_c [ntrans, 4]: lambda0, A_ul, B_lu, B_ul;
    line_e [ntrans]: E_u - E_l; sigma [ntrans, nlambda]: bound-free cross sections."""

    def __init__(self, grid, lam, lam_w, fudge, ray_theta, ray_w, transitions, line_c, line_e, A, B, stage, cont_of,
                 sigma, device=0):
        d = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        self._keep = [d(grid), d(lam), d(lam_w), d(fudge), d(ray_theta), d(ray_w), i32(transitions), d(line_c),
                      d(line_e), d(A), d(B), i32(stage), i32(cont_of), d(sigma)]
        k = self._keep
        self.nd, self.nl, self.nray, self.nlev = len(k[0]), len(k[1]), len(k[4]), k[9].shape[0]
        self.ntr = k[6].shape[0]
        p = SnapiAliProblem(self.nd, self.nl, self.nray, self.nlev, self.ntr, *[a.ctypes.data for a in k])
        self._prob = p
        self.nline = int(sum(1 for t in range(self.ntr) if k[12][k[6][t, 0]] != k[6][t, 1]))
        self.nbf = self.ntr - self.nline
        st = ctypes.c_int(0)
        self._ctx = _ali_lib().snapi_ali_create(ctypes.byref(p), device, ctypes.byref(st))
        if not self._ctx:
            raise RuntimeError("snapi_ali_create failed (%d)" % st.value)

    @classmethod
    def from_fixture(cls, fx, **kw):
        tr = np.asarray(fx["ali_tr"]).astype(int)  # type, lower, upper, stage of the lower level
        nlev = fx["ali_A"].shape[0]
        stage = np.zeros(nlev, int)
        cont = -np.ones(nlev, int)
        for t, lo, up, z in tr:
            stage[lo] = z
            stage[up] = z + 1 if t == 1 else z
            if t == 1:
                cont[lo] = up
        sig = np.zeros((tr.shape[0], fx["ali_lambda"].shape[0]))
        sig[tr[:, 0] == 1] = fx["ali_sigma"]
        trc = np.asarray(fx["ali_trc"])
        return cls(fx["ali_grid"], fx["ali_lambda"], fx["ali_lw"], fx["ali_fudge"], fx["ali_th"], fx["ali_bin"],
                   tr[:, 1:3], trc[:, :4], trc[:, 4], fx["ali_A"], fx["ali_B"], stage, cont, sig, **kw)

    def close(self):
        if getattr(self, "_ctx", None):
            _ali_lib().snapi_ali_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    @staticmethod
    def columns_from_fixture(fx):
        return {k: fx["ali_" + k] for k in ("T", "ne", "na", "kap", "vray", "dld", "adamp", "bfratio", "coll",
                                             "bgop", "bgem")}

    def iterate(self, cols, pops, max_iter=100, tol=1e-2):
        """Iterate all columns; returns (pops, rel_change, iters, status)."""
        d = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        arrs = [d(cols["T"]), d(cols["ne"]), d(cols["na"]), d(cols["kap"]), d(cols["vray"]), d(cols["dld"]),
                d(cols["adamp"]), d(cols["bfratio"]), d(cols["coll"]), d(cols["bgop"]), d(cols["bgem"])]
        c = SnapiAliColumns(*[a.ctypes.data for a in arrs])
        p = d(pops).copy()
        ncol = p.shape[0]
        rel = np.zeros(ncol)
        it = np.zeros(ncol, np.int32)
        st = np.zeros(ncol, np.int32)
        rc = _ali_lib().snapi_ali_iter(self._ctx, ncol, ctypes.byref(c), p.ctypes.data, int(max_iter), float(tol),
                                       rel.ctypes.data, it.ctypes.data, st.ctypes.data, MEM_HOST)
        if rc != 0:
            raise RuntimeError("snapi_ali_iter: %s" % _ali_lib().snapi_ali_last_error(self._ctx).decode())
        return p, rel, it, st

    def iterate_device(self, ncol, cols, pops_ptr, max_iter=100, tol=1e-2, rel_ptr=0, iters_ptr=0, status_ptr=0):
        """iterate on device arrays: cols maps the SnapiAliColumns field names to device addresses
        (e.g. torch .data_ptr()), pops_ptr [ncol][nd][nlevel] in / out."""
        c = SnapiAliColumns(*[cols[n] for n, _ in SnapiAliColumns._fields_])
        rc = _ali_lib().snapi_ali_iter(self._ctx, int(ncol), ctypes.byref(c), pops_ptr, int(max_iter), float(tol),
                                       rel_ptr or None, iters_ptr or None, status_ptr or None, MEM_DEVICE)
        if rc != 0:
            raise RuntimeError("snapi_ali_iter: %s" % _ali_lib().snapi_ali_last_error(self._ctx).decode())

    def column_shapes(self, ncol):
        """Shapes of the SnapiAliColumns arrays (and 'pops') for ncol columns."""
        nd, nr, nl, nv = self.nd, self.nray, self.nl, self.nlev
        return {"T": (ncol, nd), "ne": (ncol, nd), "na": (ncol, nd), "kappa": (ncol, nd), "vray": (ncol, nr, nd),
                "dld": (ncol, self.nline, nd), "adamp": (ncol, self.nline, nd), "bfratio": (ncol, self.nbf, nd),
                "coll": (ncol, nd, nv, nv), "bg_op": (ncol, nr, nl, nd), "bg_em": (ncol, nr, nl, nd),
                "pops": (ncol, nd, nv)}

    def setup(self, ctx, tables, columns):
        """The population-independent set-up on the device (snapi_ali_setup) of host columns
        [ncol][12][nd] with ctx's atom tables (Context.eos_set) and the set-up tables
        (AliSetupTables): returns (cols, pops0, status) as host arrays, cols keyed like
        columns_from_fixture."""
        cols = np.ascontiguousarray(columns, dtype=np.float64)
        ncol = cols.shape[0]
        sh = self.column_shapes(ncol)
        out = {n: np.zeros(sh[n]) for n in sh}
        st = np.zeros(ncol, np.int32)
        o = SnapiAliSetupOut(*[out[n].ctypes.data for n, _ in SnapiAliSetupOut._fields_])
        rc = _ali_setup_lib().snapi_ali_setup(ctx._ctx, ctypes.byref(self._prob), ctypes.byref(tables.tab), ncol,
                                             cols.ctypes.data, ctypes.byref(o), out["pops"].ctypes.data,
                                             st.ctypes.data, MEM_HOST)
        ctx._check(rc)
        cmap = {"T": "T", "ne": "ne", "na": "na", "kap": "kappa", "vray": "vray", "dld": "dld", "adamp": "adamp",
                "bfratio": "bfratio", "coll": "coll", "bgop": "bg_op", "bgem": "bg_em"}
        return {k: out[v] for k, v in cmap.items()}, out["pops"], st

    def setup_device(self, ctx, tables, ncol, columns_ptr, out, pops_ptr, status_ptr=0):
        """snapi_ali_setup on device arrays: out maps the SnapiAliSetupOut field names to device
        addresses."""
        o = SnapiAliSetupOut(*[out[n] for n, _ in SnapiAliSetupOut._fields_])
        ctx._check(_ali_setup_lib().snapi_ali_setup(ctx._ctx, ctypes.byref(self._prob), ctypes.byref(tables.tab),
                                                    int(ncol), columns_ptr, ctypes.byref(o), pops_ptr,
                                                    status_ptr or None, MEM_DEVICE))

    @property
    def last_kernel_ms(self):
        return _ali_lib().snapi_ali_last_kernel_ms(self._ctx)


def _pop_lib():
    L = lib()
    if not getattr(L, "_pop_set", False):
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.snapi_records_set_populations.argtypes = [vp, ip, vp, vp, ip, vp, ip]
        L._pop_set = True
    return L


def ali_line_levels(line_eos, nlte_atom, level_map):
    """line_level [nlines][2] of snapi_records_set_populations: for each line (the node model's
    line ties, rows atom, stage, lower, upper) of the NLTE atom, the indices of its levels among the
    ALI problem's (level_map [nlevel][2]: stage, level); (-1, -1) for the other lines."""
    lm = {(int(z), int(l)): k for k, (z, l) in enumerate(np.asarray(level_map).astype(int))}
    out = -np.ones((len(line_eos), 2), np.int32)
    for j, r in enumerate(np.asarray(line_eos)):
        a, z, lo, up = (int(v) for v in r[:4])
        if a == nlte_atom:
            out[j] = (lm[(z, lo)], lm[(z, up)])
    return out


class SnapiAliBB(ctypes.Structure):
    _fields_ = [("atom", ctypes.c_int), ("stage", ctypes.c_int), ("lower", ctypes.c_int), ("upper", ctypes.c_int)] + \
        [(n, ctypes.c_double) for n in ("lambda0", "Blu", "Bul", "a_rad", "alpha_col", "sigma_col", "mass")]


class SnapiAliSetupTables(ctypes.Structure):
    _fields_ = [("nbf", ctypes.c_int), ("bf_level", ctypes.c_void_p), ("bf_sigma", ctypes.c_void_p),
                ("nbb", ctypes.c_int), ("bb", ctypes.c_void_p), ("nray_atom", ctypes.c_int),
                ("ray_atom", ctypes.c_void_p), ("atom", ctypes.c_int), ("atom_Z", ctypes.c_int)] + \
        [(n, ctypes.c_void_p) for n in ("level", "line_damp", "sigma_edge", "coll_n", "coll_t", "coll_v")]


class SnapiAliSetupOut(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("T", "ne", "na", "kappa", "vray", "dld", "adamp", "bfratio", "coll",
                                               "bg_op", "bg_em")]


def _ali_setup_lib():
    L = _ali_lib()
    if not getattr(L, "_alis_set", False):
        vp, ip = ctypes.c_void_p, ctypes.c_int
        L.snapi_ali_setup.argtypes = [vp, ctypes.POINTER(SnapiAliProblem), ctypes.POINTER(SnapiAliSetupTables), ip, vp,
                                      ctypes.POINTER(SnapiAliSetupOut), vp, vp, ip]
        L._alis_set = True
    return L


class AliSetupTables:
    """The set-up tables of snapi_ali_setup (snapi_ali_setup_tables), kept alive by this object.

    bf_level [nbf, 3] (atom, stage, level) and bf_sigma [nbf, nlambda]: bound-free levels of the LTE
    atoms; bb [nbb, 11]: atom, stage, lower, upper, lambda0, Blu, Bul, a_rad, alpha_col, sigma_col,
    mass; ray_atom: Rayleigh atoms; atom / atom_Z: the NLTE atom; level [nlevel, 2]: stage and
    level of the problem's levels; line_damp [nline, 4]; sigma_edge [nlevel]; coll_n [nlevel, nlevel],
    coll_t / coll_v [nlevel, nlevel, 8]."""

    def __init__(self, bf_level, bf_sigma, bb, ray_atom, atom, atom_Z, level, line_damp, sigma_edge, coll_n, coll_t,
                 coll_v):
        d = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        bb = np.asarray(bb, np.float64).reshape(-1, 11)
        self._bb = (SnapiAliBB * max(1, bb.shape[0]))()
        for q, r in enumerate(bb):
            self._bb[q] = SnapiAliBB(int(r[0]), int(r[1]), int(r[2]), int(r[3]), *[float(v) for v in r[4:]])
        self._keep = [i32(np.asarray(bf_level).reshape(-1, 3)), d(bf_sigma), i32(np.asarray(ray_atom).reshape(-1)),
                      i32(level), d(line_damp), d(sigma_edge), i32(coll_n), d(coll_t), d(coll_v)]
        k = self._keep
        self.tab = SnapiAliSetupTables(k[0].shape[0], k[0].ctypes.data, k[1].ctypes.data, bb.shape[0],
                                       ctypes.addressof(self._bb), k[2].shape[0], k[2].ctypes.data, int(atom),
                                       int(atom_Z), k[3].ctypes.data, k[4].ctypes.data, k[5].ctypes.data,
                                       k[6].ctypes.data, k[7].ctypes.data, k[8].ctypes.data)

    @classmethod
    def from_fixture(cls, fx):
        m = fx["alis_meta"]
        return cls(fx["alis_bf"].astype(int), fx["alis_bfsig"], fx["alis_bb"], fx["alis_ray"].astype(int), int(m[0]),
                   int(m[1]), fx["alis_lev"].astype(int), fx["alis_line"], fx["alis_sedge"],
                   fx["alis_coll_n"].astype(int), fx["alis_coll_t"], fx["alis_coll_v"])
