"""Rest state on the Guillot (2010) profile (init_PT_profile = guillot).

The CPU test checks the restatement of the reference's guillot_T and of the general rest-state
branch of initial_values (tests/thorx_testlib.py, after src/ESP/ultrahot_thermo.cu:121-161 and
src/ESP/esp_initial.cu:840-1000): the column is in the discrete hydrostatic balance the Newton
iteration solves, and deep in the atmosphere the profile follows its diffusion limit. The GPU test
holds thorx_init_guillot_state against it.
"""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (HOT_JUPITER, RefGrid, grid_dict, guillot_T, guillot_column, make_params,
                           thorx_params)

RT = dict(Tint=100.0, f_lw=0.5, kappa_sw=4e-4, kappa_lw=1e-3)


def column(nv=40):
    p, c = make_params(4, 300.0, **dict(HOT_JUPITER, Tmean=1414.0, Top_altitude=3.5e6))
    g = RefGrid(4, nv, A=c["A"], top=c["Top_altitude"])
    return g, c, guillot_column(g.arrays["Altitude"], g.arrays["Altitudeh"], c, **RT)


def test_guillot_column_restatement():
    g, c, (p, T, rho) = column()
    alt, alth = g.arrays["Altitude"], g.arrays["Altitudeh"]
    g.close()
    assert np.all(np.diff(p) < 0) and np.all(T > 0)
    # the discrete balance of every layer against the one below (the iteration's f = 0)
    grav = c["Gravit"]
    for lev in range(1, len(p)):
        dz = alt[lev] - alt[lev - 1]
        li, ri = (alt[lev] - alth[lev]) / dz, (alth[lev] - alt[lev - 1]) / dz
        f = (p[lev] - p[lev - 1]) / dz + grav * (rho[lev] * ri + rho[lev - 1] * li)
        assert abs(f) * dz <= 1e-10 * p[lev], lev
    # deep limit (large optical depth): T^4 -> 3/4 Tint^4 tau_lw + the absorbed-flux terms;
    # at the top, T tends to the irradiated skin temperature, between Tint and Teq
    assert T[0] > T[-1] > 0.5 * c["Tmean"]
    t_deep = guillot_T(1e9, 0.5, c["Tmean"], c["P_Ref"], grav, **RT)
    assert t_deep > T[0]


@pytest.mark.gpu
def test_product_guillot_state_matches_restatement():
    g, c, (p, T, rho) = column()
    x = thor_b200.Thorx(grid_dict(g), 4, thorx_params(c, 300.0))
    x.init_guillot_state(c["Tmean"], seed=1, noise_amp=0.0, **RT)
    N, nv = g.point_num, len(p)
    got = {f: x.get(f).reshape(N, nv) for f in ("pressure", "temperature", "Rho")}
    x.close(), g.close()
    for f, ref in (("pressure", p), ("temperature", T), ("Rho", rho)):
        err = np.abs(got[f] - ref[None, :]).max() / np.abs(ref).max()
        assert err <= 1e-13, (f, err)
