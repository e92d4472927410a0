"""Global conserved quantities and the compensated device sum on the GPU.

thorx_globdiag and the reference's own ESP::globdiag kernels (CalcMass et al. +
gpu_sum_on_device<1024>, run by oracle/ref_harness.cu) are held against the CPU restatement on the
same state. The bound is relative to the sum of the magnitudes of the per-cell terms, the scale
of any summation error: the product's sums are compensated (1e-13 covers last-bit differences of
the per-cell transcendental functions), the reference's are plain tree sums (1e-12).
"""
import math

import numpy as np
import pytest

import thor_b200
from thorx_testlib import (RefGrid, RefSim, Oracle, grid_dict, initial_state, make_params,
                           thorx_params)

EPS = np.finfo(np.float64).eps
FIELDS = ["Rho", "temperature", "pressure", "W", "Cp", "Rd", "Mh", "Wh"]


@pytest.mark.gpu
@pytest.mark.parametrize("glevel,nv,over", [
    (4, 8, {}),
    (4, 16, dict(DeepModel=0, NonHydro=0, energy_equation=1)),
    (5, 12, dict(GravHeightVar=1)),
])
def test_globdiag_matches_oracle_and_reference(glevel, nv, over):
    dt = 1200.0
    g = RefGrid(glevel, nv)
    p, c = make_params(glevel, dt, **over)
    o = Oracle(g, p)
    for k, v in initial_state(g.arrays, g.point_num, nv, c).items():
        o.set(k, v)
    o.step(2)
    st = {k: o.get(k) for k in FIELDS}
    want, mag = o.globdiag()
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt))
    s = RefSim(g, p)
    for k, v in st.items():
        x.set(k, v)
        s.set(k, v)
    mine = np.array(x.globdiag())
    again = np.array(x.globdiag())
    sums, cells = x.globdiag_fields()
    ref = s.globdiag()
    # the per-cell terms against the reference's own arrays (CalcTotEnergy, CalcMass, CalcAngMom,
    # CalcEntropy store them per cell for the output files)
    names = ["Etotal", "Mass", "AngMomx", "AngMomy", "AngMomz", "Entropy"]
    for q, n in enumerate(names):
        r = s.get(n)
        scale = np.abs(r).max()
        assert np.abs(cells[q] - r).max() <= 1e-13 * scale, n
    x.close(), s.close(), o.close(), g.close()
    assert np.array_equal(sums, mine)  # the same sums with the per-cell terms kept
    assert np.array_equal(mine, again), "globdiag is not deterministic"
    err = np.abs(mine - want) / mag
    err_ref = np.abs(ref - want) / mag
    assert np.all(err <= 1e-13), dict(err=err, mine=mine, oracle=want)
    assert np.all(err_ref <= 1e-12), dict(err_ref=err_ref, ref=ref, oracle=want)


@pytest.mark.gpu
def test_globdiag_after_product_and_reference_steps_agree():
    """After three steps of the product and of the reference from the same state, the totals agree
    to the accuracy the two states agree (1e-12 in density and pressure)."""
    glevel, nv, dt = 4, 16, 1200.0
    g = RefGrid(glevel, nv)
    p, c = make_params(glevel, dt)
    ic = initial_state(g.arrays, g.point_num, nv, c)
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt))
    s = RefSim(g, p)
    for k, v in ic.items():
        x.set(k, v)
        s.set(k, v)
    x.step(3)
    x.sync()
    s.step(3)
    mine, ref = x.globdiag(), s.globdiag()
    x.close(), s.close(), g.close()
    assert abs(mine[1] - ref[1]) <= 1e-12 * abs(ref[1]), (mine[1], ref[1])
    assert abs(mine[5] - ref[5]) <= 1e-12 * abs(ref[5]), (mine[5], ref[5])


def _exact_bound(x, exact):
    return 2 * EPS * abs(exact) + 4 * x.size * EPS ** 2 * math.fsum(np.abs(x))


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 2, 2047, 2048, 2049, 1_000_003])
def test_device_sum_is_compensated_and_deterministic(n):
    import torch
    rng = np.random.default_rng(n)
    big = rng.standard_normal(n) * 1e12
    x = np.concatenate([big, -big[::-1], rng.standard_normal(n)])
    rng.shuffle(x)
    xd = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    a = thor_b200.device_sum(xd.data_ptr(), x.size)
    b = thor_b200.device_sum(xd.data_ptr(), x.size)
    exact = math.fsum(x)
    assert a == b
    assert abs(a - exact) <= _exact_bound(x, exact), (a, exact)


@pytest.mark.gpu
def test_device_sum_agrees_with_the_reference_reduction():
    from thorx_testlib import ref_lib
    rng = np.random.default_rng(3)
    x = rng.uniform(0.5, 2.0, 3 * 2048 * 7 + 5)  # positive terms: the plain tree sum is accurate
    import torch
    xd = torch.from_numpy(x).cuda()
    torch.cuda.synchronize()
    mine = thor_b200.device_sum(xd.data_ptr(), x.size)
    ref = ref_lib().ref_device_sum(x.ctypes.data, x.size)
    exact = math.fsum(x)
    assert abs(mine - exact) <= 2 * EPS * exact
    assert abs(ref - exact) <= 1e-13 * exact


@pytest.mark.gpu
def test_device_sum_rejects_bad_arguments_before_any_launch():
    import torch
    xd = torch.ones(1000, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert thor_b200.device_sum(xd.data_ptr(), 0) == 0.0
    assert thor_b200.device_sum(xd.data_ptr(), 1000) == 1000.0
    host = np.ones(10)
    for ptr, n, what in [(host.ctypes.data, 10, "not device memory"),
                         (xd.data_ptr(), 10_000_000, "past the end"),
                         (xd.data_ptr(), -1, "negative")]:
        with pytest.raises(thor_b200.ThorxError) as e:
            thor_b200.device_sum(ptr, n)
        assert e.value.code == thor_b200.E_ARG, (what, str(e.value))
    # the context is still healthy
    assert thor_b200.device_sum(xd.data_ptr(), 1000) == 1000.0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [thor_b200.FP64, thor_b200.MIXED])
def test_globdiag_fields_leaves_the_next_steps_unchanged(precision):
    """thorx_globdiag_fields computes its per-cell planes in the hyperdiffusion work buffer; the
    steps after it must give the same bits as steps that never saw the call."""
    glevel, nv, dt = 4, 16, 1200.0
    g = RefGrid(glevel, nv)
    p, c = make_params(glevel, dt)
    ic = initial_state(g.arrays, g.point_num, nv, c)
    out = []
    for call in (False, True):
        x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt, precision=precision))
        for k, v in ic.items():
            x.set(k, v)
        x.step(2)
        if call:
            sums, cells = x.globdiag_fields()
            assert np.all(np.isfinite(sums)) and all(np.all(np.isfinite(v)) for v in cells)
        x.step(3)
        x.sync()
        out.append({f: x.get(f) for f in ["Rho", "pressure", "Mh", "Wh", "W"]})
        x.close()
    g.close()
    for f in out[0]:
        assert np.array_equal(out[0][f], out[1][f]), f
