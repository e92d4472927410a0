"""The product against the reference's own FP64 CUDA kernels at the configurations its throughput
is quoted on, not only at the small grids of test_dycore_parity_gpu.py.

* Held-Suarez, glevel 6 (40962 columns) x 48 levels, dt = 600 s (the bench workload): the
  product's grid builder against the reference's (bit for bit), then one large step, eagerly and
  as a graph replay, against the reference's FMA and no-FMA builds.
* Hot Jupiter with double-gray RT, glevel 5 (10242 columns) x 40 levels, dt = 300 s: R = 1e8 m,
  g = 10, Rd = 3714, Cp = 13000, 100 bar at the bottom, top at 1e-3 bar, substellar point at
  longitude 0, gray opacities 4e-4 (SW) and 1e-3 (LW) m^2/kg, Guillot rest state (Tint 100 K,
  T_irr 2000 K) with seeded +-1 K noise; two large steps with the RT module.
* Held-Suarez, glevel 4 (2562 columns) x 32 levels, dt = 1200 s, all 100 large steps.

Tolerances as in the other dynamical-core tests: 1e-12 of max|field| for density, pressure and
temperature after one step, and for the other fields 1e-12 or 4x the spread between the
reference's own FMA and no-FMA builds where that is larger (the vertical momentum and its
tendency are small residuals of hydrostatic balance, where rounding is amplified). Over 100 steps
the two reference builds drift apart as well; the product is held to 4x that drift.
"""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (RefGrid, RefSim, STATE_FIELDS, field_tolerance, grid_dict,
                           initial_state, make_params, rel_err, thorx_params)

TEND = ["SlowMh", "SlowWh", "SlowRho", "Slowpressure"]
TIGHT = {"Rho", "pressure", "temperature"}
GRID_F64 = ["Altitude", "Altitudeh", "lonlat", "areas", "areasT", "areasTr", "nvecoa", "nvecti",
            "nvecte", "div", "grad", "func_r"]
GRID_I32 = ["maps", "point_local"]


def compare(x, sims, fields, floor=1e-12, tight=1e-12):
    s, sn = sims
    res, bad = {}, {}
    for f in fields:
        a, b, bn = x.get(f), s.get(f), sn.get(f)
        err, spread = rel_err(a, b), rel_err(bn, b)
        tol = tight if f in TIGHT else field_tolerance(spread, floor=floor)
        res[f] = (err, spread)
        if not (np.all(np.isfinite(a)) and err <= tol):
            bad[f] = (err, tol)
    return bad, res


@pytest.fixture(scope="module")
def g6_grid():
    g = RefGrid(6, 48)
    yield g
    g.close()


@pytest.mark.gpu
def test_g6_product_grid_is_the_reference_grid(g6_grid):
    """bench.py builds its grid with thorx_grid_build: the same arrays, bit for bit."""
    mine = thor_b200.Icogrid(6, 48)
    for k in GRID_F64 + GRID_I32:
        a, b = np.asarray(mine[k]), np.asarray(g6_grid[k])
        assert a.shape == b.shape and np.array_equal(a, b), k


@pytest.mark.gpu
@pytest.mark.parametrize("use_graph", [False, True])
def test_g6_l48_step_matches_reference(g6_grid, use_graph):
    glevel, dt = 6, 600.0
    p, c = make_params(glevel, dt)
    g = g6_grid
    ic = initial_state(g.arrays, g.point_num, g.nv, c)
    sims = (RefSim(g, p), RefSim(g, p, nofma=True))
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt))
    for k, v in ic.items():
        for h in sims + (x,):
            h.set(k, v)
    for h in sims:
        h.step(1)
    if use_graph:
        x.step(1)
        x.sync()
    else:
        x.profx()
        x.thor()
    bad, res = compare(x, sims, STATE_FIELDS + ["temperature"] + TEND)
    x.close()
    for h in sims:
        h.close()
    print("g6/L48 one step (err, reference spread):", {k: "%.2e %.2e" % v for k, v in res.items()})
    assert not bad, {"failures": bad, "all": res}


# the hot Jupiter of the RT configuration
HJ_T_IRR, HJ_TSTAR, HJ_RSTAR = 2000.0, 4300.0, 0.667 * 695700000.0
HJ_TEQ = HJ_T_IRR / 2 ** 0.5
HJ = dict(A=1e8, Omega=9.09e-5, Gravit=10.0, Rd=3714.0, Cp=13000.0, P_Ref=1e7,
          Top_altitude=3714.0 * HJ_TEQ / 10.0 * np.log(1e7 / 1e2), Tmean=HJ_TEQ, Diffc=0.015,
          DivDampc=0.015, HyDiffOrder=4, DeepModel=1, NonHydro=1, GravHeightVar=0, HyDiff=1,
          DivDampP=1, energy_equation=0, held_suarez=0)
HJ_RT = dict(Tstar=HJ_TSTAR, radius_star=HJ_RSTAR,
             planet_star_dist=HJ_RSTAR * (HJ_TSTAR / HJ_T_IRR) ** 2, diff_ang=0.5, Tint=100.0,
             albedo=0.0, kappa_sw=4e-4, kappa_lw=1e-3, kappa_lw_pole=1e-3, n_sw=1.0, n_lw=2.0,
             f_lw=0.5, sync_rot=1, alpha_i=0.0)
RT_FIELDS = ["cos_zenith", "insol", "ASR", "OLR", "fsw_dn", "flw_up", "flw_dn", "tau", "dtemp",
             "profx_Qheat", "insol_ann"]


@pytest.mark.gpu
def test_hot_jupiter_rt_g5_l40_matches_reference():
    glevel, nv, dt = 5, 40, 300.0
    p, c = make_params(glevel, dt, **HJ)
    g = RefGrid(glevel, nv, A=c["A"], top=c["Top_altitude"])
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt))
    x.init_guillot_state(HJ_TEQ, HJ_RT["Tint"], HJ_RT["f_lw"], HJ_RT["kappa_sw"],
                         HJ_RT["kappa_lw"], 20260101, 1.0)
    N = g.point_num
    ic = {f: x.get(f) for f in ["Rho", "pressure", "temperature", "Mh", "Wh", "W"]}
    ic["Rd"], ic["Cp"] = np.full(N * nv, c["Rd"]), np.full(N * nv, c["Cp"])
    assert np.ptp(ic["temperature"].reshape(N, nv)[:, 0]) > 1.0  # the noise is there
    sims = (RefSim(g, p), RefSim(g, p, nofma=True))
    for h in sims:
        for k, v in ic.items():
            h.set(k, v)
        h.rt(HJ_RT)
    x.rt_enable(HJ_RT)
    # one physics step: the RT fields
    x.profx()
    x.sync()
    for h in sims:
        h.step(1, profx=True, thor=False)
    bad1, res1 = compare(x, sims, RT_FIELDS + ["pressure", "temperature"])
    # synchronous rotation on a circular orbit: the zenith angles of the reference binary's
    # calc_zenith (src/ESP/insolation.cu:128-207), bit for bit
    assert np.array_equal(x.get("cos_zenith"), sims[0].get("cos_zenith"))
    # then the dynamical core of that step and a second full step (graph replay)
    x.thor()
    x.step(1)
    x.sync()
    for h in sims:
        h.step(1, profx=False, thor=True)
        h.step(1)
    bad2, res2 = compare(x, sims, STATE_FIELDS + ["temperature", "profx_Qheat"], floor=1e-11,
                         tight=1e-11)
    tot, rtot = x.rt_totals(), sims[0].rt_totals()
    x.close(), g.close()
    for h in sims:
        h.close()
    print("hot Jupiter g5/L40 RT step:", {k: "%.2e %.2e" % v for k, v in res1.items()})
    print("after two large steps:", {k: "%.2e %.2e" % v for k, v in res2.items()})
    assert not bad1, {"failures": bad1, "all": res1}
    assert not bad2, {"failures": bad2, "all": res2}
    for a, b in zip(tot, rtot):
        assert abs(a - b) <= 1e-11 * abs(b), (tot, rtot)


@pytest.mark.gpu
def test_held_suarez_g4_l32_hundred_steps_match_reference():
    glevel, nv, dt, n = 4, 32, 1200.0, 100
    p, c = make_params(glevel, dt)
    g = RefGrid(glevel, nv)
    ic = initial_state(g.arrays, g.point_num, nv, c)
    sims = (RefSim(g, p), RefSim(g, p, nofma=True))
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt))
    for k, v in ic.items():
        for h in sims + (x,):
            h.set(k, v)
    for h in sims:
        h.step(n)
    x.step(n)
    x.sync()
    fields = STATE_FIELDS + ["temperature"]
    res = {}
    for f in fields:
        a, b, bn = x.get(f), sims[0].get(f), sims[1].get(f)
        res[f] = (rel_err(a, b), rel_err(bn, b))
    x.close(), g.close()
    for h in sims:
        h.close()
    print("g4/L32 after 100 steps (err, reference spread):",
          {k: "%.2e %.2e" % v for k, v in res.items()})
    bad = {f: v for f, v in res.items() if not v[0] <= field_tolerance(v[1], floor=1e-11)}
    assert not bad, res
