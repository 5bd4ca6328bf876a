"""FP64 numpy restatement of one NLTE level-population iteration (test infrastructure).

Follows the reference's atmosphere::nltepops loop body (atmos/atmos_pop.cc:133-214) for one
column, from the population-independent inputs the reference's own set-up produces (the
config-5 fixture made by tests/golden/make_golden.py):

  * active opacity / emissivity per (ray, wavelength, depth): atom::boundbound_op / _em and
    atom::boundfree_op / _em (atmos/atmol/atom/atom_rad.cc:312-400, 437-530), W4 profile / dld
  * normalisation by kappa_500 and the scalar formal solution with the diagonal operator
    (atmos/plpar/atmos_ppbez_rts.cc:21-219: monotone-derivative Bezier optical depth, linear
    weights with the Taylor branch below 1e-2, boundary I = S at the bottom for outgoing rays)
  * atom::add (atmos/atmol/atom/atom.cc:1865-1927): profile norm, J and Lambda* per line,
    photo-ionisation / recombination integrals per bound-free transition
  * atom::newpops (atmos/atmol/atom/atom_pop.cc:27-145) with R_ij_local_ALO / R_ij, R_i_cont,
    R_cont_i (atom_rad.cc:1726-1756, 1842-1855), the most populated level replaced by
    conservation, and atmosphere::newpops' relative change and negative check
    (atmos/atmos_pop.cc:339-412).
"""
import numpy as np

C = 2.99792458E10
H = 6.6260687652E-27
K = 1.3806503E-16
PI = np.pi


def w4(x, a):
    """Humlicek W4 real part / sqrt(pi) (cmlib/profiles.cc:91-115), vectorised."""
    x = np.asarray(x, dtype=np.float64)
    a = np.broadcast_to(np.asarray(a, dtype=np.float64), x.shape)
    s = np.abs(x) + a
    t = a - 1j * x
    u = t * t
    w = np.empty(x.shape, dtype=np.complex128)
    r1 = s >= 15.0
    r2 = (~r1) & (s > 5.5)
    r3 = (~r1) & (~r2) & (a > 0.195 * np.abs(x) - 0.176)
    r4 = ~(r1 | r2 | r3)
    w[r1] = t[r1] * 0.5641896 / (0.5 + u[r1])
    w[r2] = t[r2] * (1.410474 + u[r2] * 0.5641896) / (0.75 + u[r2] * (3.0 + u[r2]))
    tt = t[r3]
    w[r3] = (16.4955 + tt * (20.20933 + tt * (11.96482 + tt * (3.778987 + tt * 0.5642236)))) / \
        (16.4955 + tt * (38.82363 + tt * (39.27121 + tt * (21.69274 + tt * (6.699398 + tt)))))
    tt, uu = t[r4], u[r4]
    num = tt * (36183.31 - uu * (3321.9905 - uu * (1540.787 - uu * (219.0313 - uu * (35.76683 - uu * (1.320522 - uu * 0.56419))))))
    den = 32066.6 - uu * (24322.84 - uu * (9022.228 - uu * (2186.181 - uu * (364.2191 - uu * (61.57037 - uu * (1.841439 - uu))))))
    su = np.sin(uu.imag)
    w[r4] = np.exp(uu.real) * (np.sqrt(1.0 - su * su) + 1j * su) - num / den
    return w.real / 1.77245386399759


class Problem:
    def __init__(self, fx):
        tr = np.asarray(fx["ali_tr"]).astype(int)
        self.lines = [i for i in range(tr.shape[0]) if tr[i, 0] == 0]
        self.bfs = [i for i in range(tr.shape[0]) if tr[i, 0] == 1]
        self.tr = tr
        self.trc = np.asarray(fx["ali_trc"])
        self.A = np.asarray(fx["ali_A"])
        self.B = np.asarray(fx["ali_B"])
        self.m = self.A.shape[0]
        self.stage = np.zeros(self.m, int)
        self.cont = -np.ones(self.m, int)
        self.bf_of = -np.ones(self.m, int)
        for t, lo, up, z in tr:
            self.stage[lo] = z
            self.stage[up] = z + 1 if t == 1 else z
        for b, i in enumerate(self.bfs):
            self.cont[tr[i, 1]] = tr[i, 2]
            self.bf_of[tr[i, 1]] = b
        self.tmap = -np.ones((self.m, self.m), int)
        for k, i in enumerate(self.lines):
            lo, up = tr[i, 1], tr[i, 2]
            self.tmap[lo, up] = self.tmap[up, lo] = k
        self.lam = np.asarray(fx["ali_lambda"])
        self.lw = np.asarray(fx["ali_lw"])
        self.fudge = np.asarray(fx["ali_fudge"])
        self.th = np.asarray(fx["ali_th"])
        self.bin = np.asarray(fx["ali_bin"])
        self.grid = np.asarray(fx["ali_grid"])
        self.sigma = np.asarray(fx["ali_sigma"])


def formal(grid, oo, ee, ct):
    """Scalar formal solution for all wavelengths at once: oo, ee [nl, nd] normalised."""
    nl, nd = oo.shape
    I = np.zeros((nl, nd))
    L = np.zeros((nl, nd))
    dz = 1 if ct > 0 else -1
    zl, zh = (0, nd - 1) if ct > 0 else (nd - 1, 0)
    h = lambda za, zb: (grid[zb] - grid[za]) / (-ct)  # noqa: E731
    d = np.zeros((nl, nd))
    d[:, zl] = (oo[:, zl + dz] - oo[:, zl]) / h(zl, zl + dz)
    d[:, zh] = (oo[:, zh] - oo[:, zh - dz]) / h(zh - dz, zh)
    z = zl + dz
    while z != zh:
        h2, h1 = h(z, z + dz), h(z - dz, z)
        d2 = (oo[:, z + dz] - oo[:, z]) / h2
        d1 = (oo[:, z] - oo[:, z - dz]) / h1
        al = (1.0 + h1 / (h1 + h2)) / 3.0
        with np.errstate(divide="ignore", invalid="ignore"):
            v = d1 * d2 / (al * d1 + (1.0 - al) * d2)
        d[:, z] = np.where(d1 * d2 > 0.0, v, 0.0)
        z += dz
    I[:, zl] = 0.0 if ct > 0 else ee[:, zl] / oo[:, zl]
    L[:, zl] = 0.0 if ct > 0 else 1.0
    z = zl + dz
    while True:
        hz = h(z - dz, z)
        C0 = oo[:, z] - hz / 2.0 * d[:, z]
        C1 = oo[:, z - dz] + hz / 2.0 * d[:, z - dz]
        tb = hz / 3.0 * (oo[:, z - dz] + oo[:, z] + 0.5 * (C0 + C1))
        small = tb < 1e-2
        with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
            etb = np.where(small, 1.0 - tb + tb * tb * 0.5 - tb ** 3 / 6.0, np.exp(-tb))
            w0 = np.where(small, tb * (0.5 - tb * (1.0 / 3.0 - tb / 8.0)), 1.0 / tb - etb * (1.0 + 1.0 / tb))
            w1 = np.where(small, 0.5 * tb * (1.0 - tb / 3.0 * (1.0 - tb / 4.0)), 1.0 - 1.0 / tb + etb / tb)
        I[:, z] = I[:, z - dz] * etb + w0 * ee[:, z - dz] / oo[:, z - dz] + w1 * ee[:, z] / oo[:, z]
        L[:, z] = w1
        if z == zh:
            break
        z += dz
    return I, L


def iterate(P, fx, col, pops):
    """One iteration for column col; returns (new pops [nd, m], max relative change, negative)."""
    T, ne, na, kap = (np.asarray(fx["ali_" + k][col]) for k in ("T", "ne", "na", "kap"))
    nd, m = pops.shape
    nline, nbf = len(P.lines), len(P.bfs)
    dld, ad = np.asarray(fx["ali_dld"][col]), np.asarray(fx["ali_adamp"][col])
    bfr = np.asarray(fx["ali_bfratio"][col])
    lam = P.lam[:, None]
    nrm = np.zeros((nline, nd)); Jl = np.zeros((nline, nd)); Ll = np.zeros((nline, nd))
    Jbu = np.zeros((nbf, nd)); Jbd = np.zeros((nbf, nd))
    e_bf = np.exp(-H * C / (lam * K * T[None, :]))
    with np.errstate(over="ignore"):
        planck = 2.0 * 6.62606957 * 8.9875517E-7 / lam ** 5 / (np.exp(1.4387769 / lam / T[None, :]) - 1.0)
    for r in range(len(P.th)):
        vr = np.asarray(fx["ali_vray"][col, r])
        op = np.array(fx["ali_bgop"][col, r], dtype=np.float64)
        em = np.array(fx["ali_bgem"][col, r], dtype=np.float64)
        phis = []
        for k, i in enumerate(P.lines):
            lo, up = P.tr[i, 1], P.tr[i, 2]
            lam0, Aul, Blu, Bul = P.trc[i, :4]
            x = (lam0 - lam * (1.0 + vr[None, :] / C)) / dld[k][None, :]
            phi = w4(x, ad[k][None, :]) / dld[k][None, :]
            phis.append(phi)
            op += phi * (pops[:, lo] * Blu - pops[:, up] * Bul)[None, :] * H * C / lam / 4.0 / PI
            em += phi * (pops[:, up] * Aul)[None, :] * H * C / lam / 4.0 / PI
        for b, i in enumerate(P.bfs):
            lo, up = P.tr[i, 1], P.tr[i, 2]
            sg = P.sigma[b][:, None] * P.fudge[:, None]
            pm = pops[:, up][None, :] * bfr[b][None, :]
            op += sg * (pops[:, lo][None, :] - pm * e_bf)
            em += sg * pm * (1.0 - e_bf) * planck
        I, L = formal(P.grid, op / kap[None, :], em / kap[None, :], np.cos(P.th[r]))
        w = (P.lw * P.bin[r])[:, None]
        for k, i in enumerate(P.lines):
            lo, up = P.tr[i, 1], P.tr[i, 2]
            phi = phis[k]
            lf = (pops[:, lo] * P.trc[i, 2] - pops[:, up] * P.trc[i, 3])[None, :] * phi * P.trc[i, 4] / 4.0 / PI / op
            nrm[k] += (w * phi / 4.0 / PI).sum(0)
            Jl[k] += (w * I * phi * lf / 4.0 / PI).sum(0)
            Ll[k] += (w * L * phi * lf / 4.0 / PI).sum(0)
        for b, i in enumerate(P.bfs):
            s = w * P.sigma[b][:, None] * lam / H / C
            Jbu[b] += (s * I).sum(0)
            Jbd[b] += (s * (I + 2.0 * H * C * C / lam ** 5) * e_bf).sum(0)

    def solve(alo):
        out = np.zeros((nd, m))
        for z in range(nd):
            n = pops[z]
            Cz = np.asarray(fx["ali_coll"][col, z])
            M = np.zeros((m, m)); bv = np.zeros(m)

            def rad(fr, to, JJ, LL):
                a, bb = P.A[fr, to], P.B[fr, to]
                if not alo:
                    return a + bb * JJ
                if fr == to:
                    return 0.0
                u, lo_ = (to, fr) if to > fr else (fr, to)
                sl = n[u] * P.A[u, lo_] / (n[lo_] * P.B[lo_, u] - n[u] * P.B[u, lo_])
                return a * (1.0 - LL) + bb * (JJ - LL * sl)

            for i in range(m - 1):
                for j in range(m):
                    if P.stage[j] != P.stage[i]:
                        continue
                    k = P.tmap[i, j]
                    JJ = Jl[k, z] / nrm[k, z] if k >= 0 else -1.0
                    LL = Ll[k, z] / nrm[k, z] if k >= 0 else 0.0
                    M[i, i] -= rad(i, j, JJ, LL) + Cz[i, j]
                    M[i, j] += rad(j, i, JJ, LL) + Cz[j, i]
                c = P.cont[i]
                if c >= 0:
                    b = P.bf_of[i]
                    upr = Jbu[b, z] + Cz[i, c]
                    M[i, i] -= upr; M[c, i] += upr
                    dn = Jbd[b, z] * bfr[b, z] + Cz[c, i]
                    M[i, c] += dn; M[c, c] -= dn
            rep = m - 1
            for i in range(m - 1):
                if n[i] > n[rep]:
                    rep = i
            M[rep, :] = 1.0
            bv[rep] = na[z]
            out[z] = np.linalg.solve(M, bv)
        rc = out / pops - 1.0
        return out, np.abs(rc).max(), bool((rc < -1.0).any())

    new, rmax, neg = solve(True)
    if neg:
        new, rmax, neg = solve(False)
    return new, rmax, neg
