"""The mixed-precision form (THORX_MIXED) against the all-FP64 form, same grid and seeded state.

In the mixed form the momentum-side horizontal stencils (the hyperdiffusion of v and w, the
divergence damping, and their use in the slow modes and the momentum equation) compute in FP32;
density, pressure and temperature tendencies, the vertical implicit solve and the global sums stay
FP64. The test states the field errors after 1 and 20 large steps and the global mass drift."""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (STATE_FIELDS, RefGrid, grid_dict, initial_state, make_params, rel_err,
                           thorx_params)

FIELDS = STATE_FIELDS + ["temperature"]


def run(glevel, nv, dt, nsteps, precision):
    g = RefGrid(glevel, nv)
    p, c = make_params(glevel, dt)
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt, precision=precision))
    for k, v in initial_state(g.arrays, g.point_num, nv, c).items():
        x.set(k, v)
    m0 = x.globdiag()[1]
    x.step(nsteps)
    x.sync()
    out = {f: x.get(f) for f in FIELDS}
    m1 = x.globdiag()[1]
    x.close(), g.close()
    return out, m0, m1


@pytest.mark.gpu
@pytest.mark.parametrize("nsteps", [1, 20])
def test_mixed_form_field_errors_and_mass(nsteps):
    ref, m0, m1 = run(4, 16, 1200.0, nsteps, thor_b200.FP64)
    mix, n0, n1 = run(4, 16, 1200.0, nsteps, thor_b200.MIXED)
    errs = {f: rel_err(mix[f], ref[f]) for f in FIELDS}
    drift_fp64 = abs(m1 - m0) / m0
    drift_mixed = abs(n1 - n0) / n0
    print("mixed vs fp64 after %d steps: %s; mass drift fp64 %.3g mixed %.3g"
          % (nsteps, {k: "%.2e" % v for k, v in errs.items()}, drift_fp64, drift_mixed))
    for f in FIELDS:
        assert np.all(np.isfinite(mix[f])), f
    # stated bounds (measured on a B200: 1 step 4e-14 / 8e-9, 20 steps 4e-12 / 2.5e-8, drift 0)
    tight, loose = (1e-12, 1e-7) if nsteps == 1 else (1e-10, 1e-6)
    for f in ["Rho", "pressure", "temperature"]:
        assert errs[f] <= tight, (f, errs[f])
    for f in ["Mh", "Wh", "W"]:
        assert errs[f] <= loose, (f, errs[f])
    assert drift_mixed <= 1e-12 and drift_fp64 <= 1e-12
