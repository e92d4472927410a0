"""Uniform thermodynamics (Phys::uniform_thermo).

When every cell's Rd and Cp equal the configured scalars, the dynamical-core kernels use the
scalars instead of loading the fields (and fold Rd / (Cp - Rd) and the like into constants). The
values are the same, so the state must be the same bits as with the per-cell path, which a
context falls back to as soon as a module holds the fields' device pointers. With fields that
really vary from cell to cell (the reference's ultrahot thermodynamics writes them), the per-cell
path must match the reference's kernels.
"""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (RefGrid, RefSim, STATE_FIELDS, field_tolerance, grid_dict,
                           initial_state, make_params, rel_err, splitmix64_uniform, thorx_params)

GLEVEL, NV, DT = 4, 16, 1200.0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [thor_b200.FP64, thor_b200.MIXED])
def test_uniform_path_is_bitwise_the_per_cell_path(precision):
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    ic = initial_state(g.arrays, g.point_num, NV, c, amp=2.0)
    res = []
    for per_cell in (False, True):
        x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT, precision=precision))
        for k, v in ic.items():
            x.set(k, v)
        if per_cell:
            x.device_field("Rd")  # a module could now write the field: per-cell from here on
        x.step(3)
        x.sync()
        res.append({f: x.get(f) for f in STATE_FIELDS + ["temperature"]})
        x.close()
    g.close()
    for f in res[0]:
        assert np.array_equal(res[0][f], res[1][f]), f


@pytest.mark.gpu
def test_varying_gas_constant_matches_reference():
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    ic = initial_state(g.arrays, g.point_num, NV, c, amp=2.0)
    n = g.point_num * NV
    ic["Rd"] = c["Rd"] * (1.0 + 2e-3 * (splitmix64_uniform(n, 7) - 0.5))
    ic["Cp"] = c["Cp"] * (1.0 + 2e-3 * (splitmix64_uniform(n, 8) - 0.5))
    ic["Rho"] = ic["pressure"] / (ic["Rd"] * ic["temperature"])
    sims = (RefSim(g, p), RefSim(g, p, nofma=True))
    x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
    for k, v in ic.items():
        for h in sims + (x,):
            h.set(k, v)
    for h in sims:
        h.step(1)
    x.step(1)
    x.sync()
    bad, res = {}, {}
    for f in STATE_FIELDS + ["temperature"]:
        a, b, bn = x.get(f), sims[0].get(f), sims[1].get(f)
        err, spread = rel_err(a, b), rel_err(bn, b)
        res[f] = (err, spread)
        tol = 1e-12 if f in ("Rho", "pressure", "temperature") else field_tolerance(spread)
        if not err <= tol:
            bad[f] = (err, tol)
    x.close(), g.close()
    for h in sims:
        h.close()
    assert not bad, {"failures": bad, "all": res}
