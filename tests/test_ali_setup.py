"""The population-independent set-up of the NLTE level-population iteration
(atmosphere::nltepops, atmos/atmos_pop.cc:67-240): chemistry and LTE populations of the column,
kappa_500, the projected velocities, the LTE background opacity / emissivity per ray and
wavelength, line widths and damping, bound-free LTE ratios and collisional rates.

CPU: the FP64 restatement (oracle/ali_setup_oracle.py) against the reference's own set-up arrays
of the config-5 fixtures (the compiled reference, tests/golden/make_golden.py).  GPU:
snapi_ali_setup against the same arrays, and the level populations the device iteration reaches
from the device set-up against the reference's."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_fixture

FIXTURES = ("config5", "config5_spec")
# the set-up arrays: fixture key -> oracle key
KEYS = (("ali_T", "T"), ("ali_ne", "ne"), ("ali_na", "na"), ("ali_kap", "kap"), ("ali_vray", "vray"),
        ("ali_dld", "dld"), ("ali_adamp", "adamp"), ("ali_bfratio", "bfratio"), ("ali_coll", "coll"),
        ("ali_bgop", "bgop"), ("ali_bgem", "bgem"), ("ali_pop0", "pop0"))


def _have(name):
    return os.path.exists(os.path.join(GOLDEN, name + ".npz"))


_params = [pytest.param(n, marks=pytest.mark.skipif(not _have(n), reason="fixture %s.npz not generated" % n))
           for n in FIXTURES]


def _relerr(v, r):
    """Largest relative difference; exact zeros must agree.  An array the fixture stores in float32
    (config5_spec's background) is compared where it is a normal float32 above 1e-30 (the emissivity
    underflows to 0 or to float32 subnormals at the blue end of the grid)."""
    f32 = np.asarray(r).dtype == np.float32
    v, r = np.asarray(v, np.float64), np.asarray(r, np.float64)
    if f32:
        m = np.abs(r) > 1e-30
    else:
        assert np.array_equal(v == 0, r == 0)
        m = r != 0
    return float((np.abs(v - r)[m] / np.abs(r[m])).max()) if m.any() else 0.0


@pytest.mark.parametrize("name", _params)
def test_oracle_setup_matches_reference(name):
    import ali_setup_oracle as aso
    fx = load_fixture(name)
    S = aso.Setup(fx)
    ncol = 2 if name == "config5_spec" else fx["alis_atm"].shape[0]
    for c in range(ncol):
        out = S.column(fx["alis_atm"][c])
        for fk, ok in KEYS:
            err = _relerr(out[ok], fx[fk][c])
            # FP64 restatement of FP64 reference code: 1e-14 measured; the spec fixture stores the
            # background in float32
            tol = 2e-7 if (name == "config5_spec" and fk in ("ali_bgop", "ali_bgem")) else 1e-12
            assert err < tol, (name, c, fk, err)
