"""Long run of the bench workload in both forms: Held-Suarez, glevel 6 (40962 columns) x 48
levels, dt = 600 s, 1000 large steps (~6.9 simulated days) from the seeded isothermal rest state.

Checks, for the all-FP64 and the mixed form (FP32 momentum-side stencils):
* global mass (compensated sum of rho x cell volume) conserved to 1e-12 relative in each form;
* the zonal-mean temperature of the mixed run within 1 K of the FP64 run's, and its zonal-mean
  zonal wind within the stated bound (5-degree latitude bands, every level, area-weighted);
* every state field finite, the field errors of the mixed form against the FP64 form stated.
"""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import rel_err

GLEVEL, NV, DT, NSTEPS = 6, 48, 600.0, 1000
PARAMS = dict(A=6.371e6, Omega=7.292e-5, Gravit=9.8, Rd=287.0, Cp=1005.0, P_Ref=1e5,
              Top_altitude=36e3, timestep=DT, Diffc=0.0048, DivDampc=0.0048, HyDiffOrder=4,
              DeepModel=1, NonHydro=1, GravHeightVar=0, HyDiff=1, DivDampP=1, thermo_equation=0,
              core_benchmark=1)
FIELDS = ["Rho", "pressure", "temperature", "Mh", "Wh", "W"]
BANDS = 36


def zonal_means(grid, T, Mh, Rho):
    """Area-weighted means over 5-degree latitude bands of T and of the zonal wind u, [band][lev]."""
    N = grid.point_num
    lon = grid["lonlat"][0::2]
    lat = grid["lonlat"][1::2]
    w = grid["areasT"][:N]
    band = np.clip(((lat + np.pi / 2) / np.pi * BANDS).astype(int), 0, BANDS - 1)
    T = T.reshape(N, NV)
    M = Mh.reshape(N, NV, 3)
    u = (-np.sin(lon)[:, None] * M[:, :, 0] + np.cos(lon)[:, None] * M[:, :, 1]) / Rho.reshape(N, NV)
    tz, uz = np.zeros((BANDS, NV)), np.zeros((BANDS, NV))
    for b in range(BANDS):
        m = band == b
        ww = w[m][:, None]
        tz[b] = (ww * T[m]).sum(0) / ww.sum()
        uz[b] = (ww * u[m]).sum(0) / ww.sum()
    return tz, uz


@pytest.fixture(scope="module")
def runs():
    grid = thor_b200.Icogrid(GLEVEL, NV)
    out = {}
    for name, prec in (("fp64", thor_b200.FP64), ("mixed", thor_b200.MIXED)):
        x = thor_b200.Thorx(grid.as_dict(), GLEVEL, dict(PARAMS, precision=prec))
        x.init_rest_state(300.0, 20260101, 0.1)
        m0 = x.globdiag()[1]
        x.step(NSTEPS)
        x.sync()
        m1 = x.globdiag()[1]
        out[name] = dict(fields={f: x.get(f) for f in FIELDS}, mass=(m0, m1))
        x.close()
    return grid, out


@pytest.mark.gpu
def test_mass_conserved_over_1000_steps(runs):
    _, out = runs
    drift = {k: abs(v["mass"][1] - v["mass"][0]) / v["mass"][0] for k, v in out.items()}
    print("relative mass drift over %d steps:" % NSTEPS, drift)
    for k, d in drift.items():
        assert d <= 1e-12, (k, drift)


@pytest.mark.gpu
def test_mixed_form_zonal_means_and_field_errors_over_1000_steps(runs):
    grid, out = runs
    a, b = out["fp64"]["fields"], out["mixed"]["fields"]
    for k in (a, b):
        for f, v in k.items():
            assert np.all(np.isfinite(v)), f
    errs = {f: rel_err(b[f], a[f]) for f in FIELDS}
    tz_a, uz_a = zonal_means(grid, a["temperature"], a["Mh"], a["Rho"])
    tz_b, uz_b = zonal_means(grid, b["temperature"], b["Mh"], b["Rho"])
    dT, du = np.abs(tz_b - tz_a).max(), np.abs(uz_b - uz_a).max()
    print("mixed vs fp64 after %d steps: fields %s; zonal-mean T max diff %.3e K, zonal-mean u "
          "max diff %.3e m/s (max |u_zm| %.2f m/s)"
          % (NSTEPS, {k: "%.2e" % v for k, v in errs.items()}, dT, du, np.abs(uz_a).max()))
    # the flow has spun up: Held-Suarez forcing drives zonal jets from the rest state
    assert np.abs(uz_a).max() > 1.0
    assert dT <= 1.0
    assert du <= 1.0
