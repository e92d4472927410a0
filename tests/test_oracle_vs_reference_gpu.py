"""The CPU restatement (oracle) against the reference's own FP64 CUDA kernels, live on the GPU.

Same reference grid, same seeded state, one large step (ProfX Held-Suarez + Thor). The oracle runs
without FMA contraction and is compared with the reference built with --fmad=false; the bound of
a field is 4x the spread between the reference's own FMA and no-FMA builds (1e-12 of max|field|
at least), and for the shallow case half that spread: what is left there is last-bit pow/log
differences between the GPU math library and glibc.
"""
import pytest

from thorx_testlib import (RefGrid, RefSim, Oracle, STATE_FIELDS, field_tolerance,
                           initial_state, make_params, rel_err)

TEND = ["SlowMh", "SlowWh", "SlowRho", "Slowpressure"]


@pytest.mark.gpu
@pytest.mark.parametrize("glevel,nv,dt,over", [
    (4, 8, 1200.0, {}),
    (4, 32, 1200.0, {}),
    (4, 16, 1200.0, dict(DeepModel=0, NonHydro=0, energy_equation=1)),
    (5, 16, 600.0, dict(GravHeightVar=1)),
])
def test_oracle_matches_reference_cuda(glevel, nv, dt, over):
    g = RefGrid(glevel, nv)
    p, c = make_params(glevel, dt, **over)
    ic = initial_state(g.arrays, g.point_num, g.nv, c)
    o, s, sn = Oracle(g, p), RefSim(g, p), RefSim(g, p, nofma=True)
    for k, v in ic.items():
        o.set(k, v)
        s.set(k, v)
        sn.set(k, v)
    o.step(1)
    s.step(1)
    sn.step(1)
    shallow = not over.get("DeepModel", 1)
    bad, all_ = {}, {}
    for f in STATE_FIELDS + ["temperature"] + TEND:
        a, b, bn = o.get(f), s.get(f), sn.get(f)
        spread = rel_err(bn, b)
        e = rel_err(a, bn)
        tol = max(1e-13, 0.5 * spread) if shallow else field_tolerance(spread)
        all_[f] = (e, spread)
        if not e <= tol:
            bad[f] = (e, tol)
    o.close(), s.close(), sn.close(), g.close()
    assert not bad, {"failures": bad, "all": all_}
