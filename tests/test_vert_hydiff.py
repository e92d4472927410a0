"""Vertical hyperdiffusion (VertHyDiff) of the dynamical core.

The product (thorx_vert_hydiff_enable) and the CPU restatement against the reference's own
vertical_diff kernel (src/headers/dyn/thor_diff.h:1198-1426), which oracle/ref_harness.cu
launches inside the hyperdiffusion block as src/ESP/thor_driver.cu:590-612 does, with the
strengths of src/ESP/esp_initial.cu:1327-1335. The test state has winds and seeded noise with
vertical structure, so that the high-order vertical derivatives are far from zero. Tolerances as
in the dynamical-core tests.
"""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (Oracle, RefGrid, RefSim, field_tolerance, grid_dict, initial_state,
                           make_params, rel_err, splitmix64_uniform, thorx_params)

GLEVEL, NV, DT = 4, 20, 1200.0


def wavy_state(g, c, seed=11):
    """Seeded 2 K temperature noise plus horizontal and vertical winds with level-to-level noise."""
    N = g.point_num
    st = initial_state(g.arrays, N, NV, c, amp=2.0)
    lon = g["lonlat"][0::2].repeat(NV)
    lat = g["lonlat"][1::2].repeat(NV)
    rho = st["Rho"]
    u = 30.0 * np.cos(lat) + 4.0 * (2 * splitmix64_uniform(N * NV, seed) - 1)
    v = 4.0 * (2 * splitmix64_uniform(N * NV, seed + 1) - 1)
    ex = np.stack([-np.sin(lon), np.cos(lon), np.zeros_like(lon)], 1)
    ey = np.stack([-np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)], 1)
    st["Mh"] = ((u[:, None] * ex + v[:, None] * ey) * rho[:, None]).reshape(-1)
    wh = 0.3 * (2 * splitmix64_uniform(N * (NV + 1), seed + 2) - 1)
    wh = wh.reshape(N, NV + 1)
    wh[:, 0] = wh[:, NV] = 0.0
    rc = rho.reshape(N, NV)
    rh = np.concatenate([rc[:, :1], 0.5 * (rc[:, 1:] + rc[:, :-1]), rc[:, -1:]], 1)
    st["Wh"] = (wh * rh).reshape(-1)
    return st


def test_restatement_runs_and_acts():
    """The oracle's vertical hyperdiffusion changes the step, leaves the density part zero, and
    its effect shrinks in proportion to Diffc_v (the operator is linear in Kdv6)."""
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT, held_suarez=0)
    st = wavy_state(g, c)
    res = {}
    for dv in (0.0, 1e-3, 2e-3):
        o = Oracle(g, p)
        for k, v in st.items():
            o.set(k, v)
        if dv:
            o.vert_hydiff(dv, 6)
        o.step(1, profx=True, thor=True)
        res[dv] = {f: o.get(f) for f in ("Mh", "Wh", "pressure", "diffrv", "diffmv", "diffprv")}
        o.close()
    g.close()
    assert np.all(res[1e-3]["diffrv"] == 0.0)
    assert np.abs(res[1e-3]["diffmv"]).max() > 0 and np.abs(res[1e-3]["diffprv"]).max() > 0
    d1 = res[1e-3]["Mh"] - res[0.0]["Mh"]
    d2 = res[2e-3]["Mh"] - res[0.0]["Mh"]
    assert np.abs(d1).max() > 0
    # one step: the response to the small diffusion is close to linear
    np.testing.assert_allclose(d2, 2 * d1, rtol=0, atol=0.05 * np.abs(d2).max())


def run(who, order, dv, nsteps, deep, held_suarez):
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT, DeepModel=int(deep), held_suarez=held_suarez)
    st = wavy_state(g, c)
    if who == "product":
        x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        x.vert_hydiff(dv, order)
    elif who == "oracle":
        x = Oracle(g, p)
        x.vert_hydiff(dv, order)
    else:
        x = RefSim(g, p, nofma=(who == "reference_nofma"))
        x.vert_hydiff(dv, order)
    for k, v in st.items():
        x.set(k, v)
    if who == "product":
        x.step(nsteps)
        x.sync()
    else:
        x.step(nsteps, profx=True, thor=True)
    out = {f: x.get(f) for f in ("Rho", "pressure", "Mh", "Wh")}
    x.close(), g.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("who", ["product", "oracle"])
@pytest.mark.parametrize("order,dv,nsteps,deep,hs", [
    (6, 2e-3, 1, True, 1), (6, 2e-3, 3, True, 1), (4, 5e-3, 1, False, 0), (8, 1e-3, 2, True, 0)])
def test_vert_hydiff_matches_reference(who, order, dv, nsteps, deep, hs):
    ref = run("reference", order, dv, nsteps, deep, hs)
    ref_nf = run("reference_nofma", order, dv, nsteps, deep, hs)
    got = run(who, order, dv, nsteps, deep, hs)
    bad, res = {}, {}
    for f in ref:
        assert np.all(np.isfinite(ref[f])), f
        err, spread = rel_err(got[f], ref[f]), rel_err(ref_nf[f], ref[f])
        tol = field_tolerance(spread, floor=1e-11)
        res[f] = (err, spread)
        if not err <= tol:
            bad[f] = (err, tol)
    assert not bad, {"failures": bad, "all": res}
    # the operator acts: the state differs from a run without it
    base = run("oracle", 0, 0.0, nsteps, deep, hs) if who == "oracle" else None
    if base is not None:
        assert rel_err(base["Mh"], ref["Mh"]) > 1e-9
