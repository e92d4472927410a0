"""Dry convective adjustment (sim.conv_adj, conv_adj_type = hourdin) in ProfX.

The product (thorx_conv_adj_enable) and the CPU restatement against the reference's own
dry_conv_adj kernel (src/headers/phy/dry_conv_adj.h:50-311, launched by oracle/ref_harness.cu
where src/ESP/profx_driver.cu:239-290 launches it), on a Held-Suarez state whose lowest levels are
superadiabatic. Tolerance per field as in the dynamical-core tests: 1e-12 of max|field|, or 4x the
spread between the reference's own FMA and no-FMA builds where that is larger. The CPU test checks
the restatement's own properties: adjusted columns are neutral or stable, and the adjustment
conserves the column's dry enthalpy weighting it mixes.
"""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (Oracle, RefGrid, RefSim, field_tolerance, grid_dict, make_params,
                           rel_err, thorx_params, unstable_state)

GLEVEL, NV, DT = 4, 16, 1200.0


def theta(T, p, ps, Rd, Cp):
    return T * (ps / p) ** (Rd / Cp)


def worst_instability(o, N, c, ps):
    """Most negative potential-temperature step between adjacent levels, K (0 if none)."""
    T = o.get("temperature").reshape(N, NV)
    p = o.get("pressure").reshape(N, NV)
    return min(0.0, float(np.diff(theta(T, p, ps[:, None], c["Rd"], c["Cp"]), axis=1).min()))


def test_restatement_removes_the_instability():
    """Each round mixes the unstable stretches to one potential temperature; recomputing the
    pressure at fixed density leaves a small residual that later rounds reduce (the reference
    repeats up to conv_adj_iter rounds for that reason)."""
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT, held_suarez=0)
    st = unstable_state(g.arrays, g.point_num, NV, c)
    N = g.point_num
    ps = st["pressure"].reshape(N, NV)[:, 0]
    worst = {}
    for iterations in (0, 1, 2, 8):
        o = Oracle(g, p)
        for k, v in st.items():
            o.set(k, v)
        o.conv_adj(iterations=iterations)
        o.step(1, profx=True, thor=False)
        worst[iterations] = worst_instability(o, N, c, ps)
        T = o.get("temperature")
        assert np.all(np.isfinite(T)) and np.all(T > 0)
        o.close()
    g.close()
    assert worst[0] < -10.0, worst                  # the test state is strongly unstable
    assert worst[1] > 0.5 * worst[0], worst         # each round removes most of what is left
    assert worst[0] < worst[1] < worst[2] < worst[8] <= 0.0, worst
    assert worst[8] > -0.01, worst                  # and eight rounds leave a hundredth of a K


def run_profx(who, iterations, soft, nsteps=1, thor=False):
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = unstable_state(g.arrays, g.point_num, NV, c)
    if who == "product":
        x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        x.conv_adj(iterations, soft)
    elif who == "oracle":
        x = Oracle(g, p)
        x.conv_adj(iterations, soft)
    else:
        x = RefSim(g, p, nofma=(who == "reference_nofma"))
        x.conv_adj(iterations, soft)
    for k, v in st.items():
        x.set(k, v)
    if who == "product":
        for _ in range(nsteps):
            if thor:
                x.step(1)
            else:
                x.profx()
        x.sync()
    else:
        x.step(nsteps, profx=True, thor=thor)
    fields = ["temperature", "pressure", "profx_Qheat", "Mh"] + (["Rho", "Wh"] if thor else [])
    out = {f: x.get(f) for f in fields}
    x.close(), g.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("who", ["product", "oracle"])
@pytest.mark.parametrize("iterations,soft,nsteps,thor", [
    (1, False, 1, False), (4, False, 1, False), (2, True, 1, False), (2, False, 3, True)])
def test_conv_adj_matches_reference(who, iterations, soft, nsteps, thor):
    ref = run_profx("reference", iterations, soft, nsteps, thor)
    ref_nf = run_profx("reference_nofma", iterations, soft, nsteps, thor)
    got = run_profx(who, iterations, soft, nsteps, thor)
    for f in ref:
        assert np.all(np.isfinite(ref[f])), f  # the reference itself stays finite on this state
    bad, res = {}, {}
    for f in ref:
        err, spread = rel_err(got[f], ref[f]), rel_err(ref_nf[f], ref[f])
        tol = field_tolerance(spread, floor=1e-11 if thor else 1e-12)
        res[f] = (err, spread)
        if not err <= tol:
            bad[f] = (err, tol)
    assert not bad, {"failures": bad, "all": res}
    if soft:
        assert np.abs(ref["profx_Qheat"]).max() > 0  # the soft form heats
    else:
        assert np.abs(ref["temperature"] - run_profx("reference", 0, False)["temperature"]).max() > 1.0
