"""FP64 numpy restatement of the population-independent set-up of atmosphere::nltepops.

TEST INFRASTRUCTURE ONLY: the checker of snapi_ali_setup.  Only tests/ import this module.

What the reference computes once per column before its level-population iterations
(atmos/atmos_pop.cc:67-240), from a column built by build_from_nodes (T, Nt, v_turb, v_z per
depth) and the tables of its atom objects:

  * the chemistry and LTE populations (ltepops, atmos_pop.cc:31-46: chemeq + atom::lte,
    atom.cc:763-789) -- here eos_oracle.chem, itself pinned to the reference's chemistry;
  * kappa_500 (compute_op_referent), the NLTE atom's total (compute_active_population,
    atom.cc:793-810) and its LTE populations as the iteration's start;
  * per ray the projected velocity (atmosphere::project, atmos_rad.cc:15-30; V_x = V_y = 0);
  * the LTE background per ray, wavelength and depth, opacity_lte / emissivity_lte
    (atmos_rad.cc:225-246): Thomson is zeroed there, so the sum of every LTE atom's free-free
    (atom_rad.cc:203-236), Rayleigh (atom_rad.cc:268-298, only for atoms with Z == 1, with the
    reference's loop reading the first coefficient six times and squaring the cross-section),
    bound-free (atom_rad.cc:312-340) and bound-bound opacity (atom_rad.cc:502-535: every level
    pair of every stage, W4 profile / Doppler width), H- bound-free and free-free (mol.cc:516-632),
    plus the NLTE atom's own free-free and Rayleigh; the emissivity is the opacity times the Planck
    function (emissivity_lte);
  * per line of the NLTE atom the Doppler width and damping (broad_dop, damp_rad, damp_col:
    atom_rad.cc:879-883, atom.cc:926-959);
  * per bound-free transition the LTE ratio factor of boundfree_op (atom_rad.cc:327-335);
  * the collisional rates of the rate matrix (atom_rad.cc:1769-1901: tabulated de-excitation
    rates, linear in T, times n_e, excitation by detailed balance; Seaton's continuum rate and its
    detailed-balance inverse).
"""
import numpy as np

import eos_oracle as eo
from ali_oracle import w4
from snapi_b200.eos_tables import EosTables

PI = 3.141592653589793238462643383279502884197169399375105
C, H, K, ME = 2.99792458E10, 6.6260687652E-27, 1.3806503E-16, 9.1093818872E-28
E, RYD, E0, SAHA = 4.8032042510E-10, 1.097373156853955E5, 7.957747154594775607E-02, 2.0706615382E-16
FCT_FF = (E * E * C * H * H * RYD) / (6.0 * PI * PI * PI * E0 * ME * C) * np.sqrt((2.0 * PI) / (3.0 * K * ME * ME * ME))


def planck(lam, T):
    """Planck_f (cmlib/mathtools.cc:1150-1152)."""
    return 2.0 * 6.62606957 * 8.9875517E-7 / lam ** 5 / (np.exp(1.4387769 / lam / T) - 1.0)


def tab_interp(t, v, T):
    """tbcr::interpol (colr.cc:111-115): linear on the first interval whose upper end exceeds T,
    the last value beyond the table."""
    for i in range(1, len(t)):
        if t[i] > T:
            return (v[i] * (T - t[i - 1]) + v[i - 1] * (t[i] - T)) / (t[i] - t[i - 1])
    return v[-1]


class Setup:
    """The set-up of one fixture (config5 / config5_spec): its task's atom tables (eos_*), the
    set-up tables (alis_*) and the ALI problem (ali_lambda, ali_fudge, ali_th, ali_tr, ali_trc)."""

    def __init__(self, fx):
        self.eos = {k[4:]: np.asarray(v) for k, v in fx.items() if k.startswith("eos_")}
        self.tab = EosTables(self.eos)
        self.d = {k: np.asarray(v) for k, v in fx.items() if k.startswith("alis_")}
        d = self.d
        self.lam = np.asarray(fx["ali_lambda"], np.float64)
        self.fudge = np.asarray(fx["ali_fudge"], np.float64)
        self.th = np.asarray(fx["ali_th"], np.float64)
        self.tr = np.asarray(fx["ali_tr"]).astype(int)
        self.trc = np.asarray(fx["ali_trc"], np.float64)
        self.inlte = int(d["alis_meta"][0])
        self.Z = int(d["alis_meta"][1])
        self.lev = np.asarray(d["alis_lev"]).astype(int)

    def column(self, atm):
        """atm [12][nd] (return_as_array rows) -> dict of the set-up arrays of one column."""
        d, eos, lam, fudge = self.d, self.eos, self.lam, self.fudge
        nd = atm.shape[1]
        na = int(eos["meta"][0])
        nstage = eos["atom_f"][:, 1].astype(int)
        T = atm[2].copy()
        Nt = atm[3] / (K * T)
        vt, vz = atm[8], atm[9]
        nmap = self.lev.shape[0]
        lines = [i for i in range(self.tr.shape[0]) if self.tr[i, 0] == 0]
        bfs = [i for i in range(self.tr.shape[0]) if self.tr[i, 0] == 1]
        nray, nl = self.th.shape[0], lam.shape[0]
        out = {k: np.zeros(s) for k, s in (("ne", nd), ("na", nd), ("kap", nd), ("vray", (nray, nd)),
                                           ("dld", (len(lines), nd)), ("adamp", (len(lines), nd)),
                                           ("bfratio", (len(bfs), nd)), ("coll", (nd, nmap, nmap)),
                                           ("bgop", (nray, nl, nd)), ("bgem", (nray, nl, nd)),
                                           ("pop0", (nd, nmap)))}
        out["T"] = T
        g = eos["lev"][:, :, :, 0]
        ee = eos["lev"][:, :, :, 1]
        ip = eos["atom_ip"]
        a = self.inlte
        for x in range(nd):
            ne, nst, npop, _, kap, _ = eo.chem(self.tab, T[x], Nt[x])
            kT = K * T[x]
            nH0 = nst[0, 0]
            out["ne"][x], out["kap"][x] = ne, kap
            out["na"][x] = npop[a].sum()
            for i in range(nmap):
                out["pop0"][x, i] = npop[a, self.lev[i, 0], self.lev[i, 1]]
            for r in range(nray):
                out["vray"][r, x] = np.cos(PI - self.th[r]) * vz[x]
            for q, t in enumerate(lines):
                lam0 = self.trc[t, 0]
                alpha, sig, mass, ar = d["alis_line"][q]
                dld = np.sqrt(2.0 * K * T[x] / mass + vt[x] * vt[x]) * lam0 / C
                red = 1.66E-24 / (1.0 / 1.008 + 1.66E-24 / mass)
                vm = np.sqrt(8.0 * K * T[x] / PI / red)
                gc = nH0 * vm * (vm / 1E6) ** (-alpha) * sig
                out["dld"][q, x] = dld
                out["adamp"][q, x] = lam0 * lam0 / (4.0 * PI * C) * (ar + gc) / dld
            for q, t in enumerate(bfs):
                z, l = self.lev[self.tr[t, 1]]
                out["bfratio"][q, x] = ne * SAHA * T[x] ** -1.5 * g[a, z, l] / g[a, z + 1, 0] * \
                    np.exp((ip[a, z] - ee[a, z, l]) / kT)
            # collisional rates (the reference's rate-matrix loop, atom_pop.cc:27-145)
            Cm = out["coll"][x]
            gi = 0.3 if self.Z > 2 else (0.2 if self.Z == 2 else 0.1)
            for i in range(nmap - 1):
                z, l = self.lev[i]
                for ll in range(int(eos["lev_n"][a, z])):
                    j = i + (ll - l)
                    if ll == l:
                        Cm[i, j] = 0.0
                        continue
                    n = int(d["alis_coll_n"][i, j])
                    if n == 0:
                        raise ValueError("collisional rate without a table")
                    lu, ld = max(l, ll), min(l, ll)
                    rate = tab_interp(d["alis_coll_t"][i, j, :n], d["alis_coll_v"][i, j, :n], T[x]) * ne
                    if l < ll:
                        u0 = abs(ee[a, z, lu] - ee[a, z, ld]) / kT
                        rate *= np.exp(-u0) * g[a, z, lu] / g[a, z, ld]
                    Cm[i, j] = rate
                dl = int(eos["lev_n"][a, z]) - l
                if dl:
                    dE = ip[a, z] - ee[a, z, l]
                    u0 = dE / kT
                    ci = 1.55E13 / np.sqrt(T[x]) * gi * d["alis_sedge"][i] * np.exp(-u0) / u0 * ne
                    Cm[i, i + dl] = ci
                    Cm[i + dl, i] = ci * g[a, z, l] / g[a, z + 1, 0] * np.exp(dE / kT) * T[x] ** -1.5 * ne * SAHA
            # LTE background (opacity_lte + the NLTE atom's free-free and Rayleigh)
            zsum = sum(z * z * nst[b, z] for b in range(na) for z in range(1, nstage[b]))
            aff = FCT_FF * 1.1 * ne / (np.sqrt(T[x]) * C * C * C) * zsum
            for r in range(nray):
                ll_ = lam * (1.0 + out["vray"][r, x] / C)
                op = aff * ll_ ** 3 * (1.0 - np.exp(-(H * C) / kT / ll_)) * fudge
                # Rayleigh: the listed LTE atoms, and the NLTE atom when its Z is 1 (its Rayleigh
                # opacity joins the background with its free-free)
                for b in list(d["alis_ray"].astype(int)) + ([a] if self.Z == 1 else []):
                    l0 = 1215.67E-8
                    cs = 1.26563 * sum((l0 / lam) ** (2 * ii) for ii in range(6)) * (l0 / lam) ** 4
                    op = op + cs * cs * 6.65E-25 * nst[b, 0]
                for q, (b, z, l) in enumerate(d["alis_bf"].astype(int)):
                    sigma = d["alis_bfsig"][q]
                    pm = npop[b, z + 1, 0] * ne * SAHA * T[x] ** -1.5 * g[b, z, l] / g[b, z + 1, 0] * \
                        np.exp((ip[b, z] - ee[b, z, l] - H * C / lam) / kT)
                    op = op + sigma * (npop[b, z, l] - pm) * fudge
                for row in d["alis_bb"]:
                    b, z, lo, up = (int(v) for v in row[:4])
                    lam0, Blu, Bul, ar, alpha, sig, mass = row[4:]
                    dld = np.sqrt(2.0 * K * T[x] / mass + vt[x] * vt[x]) * lam0 / C
                    red = 1.66E-24 / (1.0 / 1.008 + 1.66E-24 / mass)
                    vm = np.sqrt(8.0 * K * T[x] / PI / red)
                    gc = nH0 * vm * (vm / 1E6) ** (-alpha) * sig
                    av = lam0 * lam0 / (4.0 * PI * C) * (ar + gc) / dld
                    xv = (lam0 - lam * (1.0 + out["vray"][r, x] / C)) / dld
                    prof = w4(xv, av) / dld
                    nlo, nup = npop[b, z, lo], npop[b, z, up]
                    op = op + prof * nlo * Blu * H * C / lam / 4.0 / PI * (1.0 - nup / nlo * Bul / Blu)
                # H- (mol.cc:516-632)
                TP = 5040.0 / T[x]
                alf = sum(c * (lam * 1E8) ** i for i, c in enumerate(
                    (1.99654, -1.18267E-5, 2.64243E-6, -4.40524E-10, 3.23992E-14, -1.39568E-18, 2.78701E-23)))
                op = op + 4.158E-28 * alf * ne * kT * TP ** 2.5 * 10.0 ** (0.754 * TP) * nH0 * \
                    (1.0 - np.exp(-H * C / lam / kT)) * fudge
                lg = np.log10(lam * 1E8)
                f0 = -2.2763 - 1.6850 * lg + 0.76661 * lg * lg - 0.053346 * lg ** 3
                f1 = 15.2827 - 9.2846 * lg + 1.99381 * lg * lg - 0.142631 * lg ** 3
                f2 = -197.789 + 190.266 * lg - 67.9775 * lg * lg + 10.6913 * lg ** 3 - 0.625151 * lg ** 4
                lt = np.log10(TP)
                op = op + 1E-26 * ne * kT * 10.0 ** (f0 + f1 * lt + f2 * lt * lt) * nH0 * fudge
                out["bgop"][r, :, x] = op
                out["bgem"][r, :, x] = op * planck(lam, T[x])
        return out
