"""Partitioned step (thorx_set_partition, thorx_set_exchange, thorx_halo_columns,
thorx_copy_columns): the grid's columns divided among several contexts, each computing its own
columns and taking its halo from the others after every kernel.

One GPU stands in for several: each partition is a context with its own stream, stepped by its own
host thread; after every kernel the exchange callback synchronises its stream, meets the other
threads at a barrier (on the host: no kernel ever waits for another), copies its halo columns from
their owners, and meets them again. The state the partitions compute, put together, must be the
unpartitioned context's bit for bit.
"""
import threading

import numpy as np
import pytest

import thor_b200
from thorx_testlib import (RT_WASP43B, RefGrid, STATE_FIELDS, grid_dict, hot_jupiter_params,
                           initial_state, make_params, thorx_params)

FIELDS = STATE_FIELDS + ["temperature"]


def run_partitioned(g, glevel, params, ic, ranges, nsteps, rt=None):
    import torch
    torch.cuda.set_device(0)
    d = grid_dict(g)
    R = len(ranges)
    xs = [thor_b200.Thorx(d, glevel, params) for _ in ranges]
    for x, (a, b) in zip(xs, ranges):
        for k, v in ic.items():
            x.set(k, v)
        if rt:
            x.rt_enable(rt)
        x.set_partition(a, b)

    def owner(c):
        return next(r for r, (a, b) in enumerate(ranges) if a <= c < b)

    cols = []  # cols[r][s]: the halo columns of partition r that partition s computes
    for r, (a, b) in enumerate(ranges):
        h = thor_b200.halo_columns(d, glevel, a, b)
        by = {}
        for c in h:
            by.setdefault(owner(int(c)), []).append(int(c))
        cols.append({s: torch.tensor(v, dtype=torch.int32, device="cuda") for s, v in by.items()})
    barrier = threading.Barrier(R, timeout=120)

    def exchange_of(r):
        def fn(stream, fields):
            st = torch.cuda.ExternalStream(stream)
            st.synchronize()
            barrier.wait()  # every partition has finished the kernel
            for s, t in cols[r].items():
                for f in fields:
                    xs[r].copy_columns(xs[s], f, t.data_ptr(), t.numel())
            st.synchronize()
            barrier.wait()  # every copy is done before any partition writes again
            return 0
        return fn

    for r, x in enumerate(xs):
        x.set_exchange(exchange_of(r))
    errors = [None] * R

    def work(r):
        try:
            xs[r].step(nsteps)
            xs[r].sync()
        except Exception as e:  # noqa: BLE001
            errors[r] = e
            barrier.abort()

    th = [threading.Thread(target=work, args=(r,)) for r in range(R)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not any(errors), errors
    out = {}
    for f in FIELDS:
        parts = [x.get(f).reshape(g.point_num, -1) for x in xs]
        full = np.empty_like(parts[0])
        for (a, b), p in zip(ranges, parts):
            full[a:b] = p[a:b]
        out[f] = full.reshape(-1)
    for x in xs:
        x.close()
    return out


def run_whole(g, glevel, params, ic, nsteps, rt=None):
    x = thor_b200.Thorx(grid_dict(g), glevel, params)
    for k, v in ic.items():
        x.set(k, v)
    if rt:
        x.rt_enable(rt)
    x.step(nsteps)
    x.sync()
    out = {f: x.get(f) for f in FIELDS}
    x.close()
    return out


CASES = {
    # two halves of whole rhombi (5 of the 10 at glevel 4; the poles in the second)
    "hs_fp64_2": (dict(), [(0, 1280), (1280, 2562)], 0),
    # three tile-aligned parts that cut through rhombi, the mixed form
    "hs_mixed_3": (dict(), [(0, 1056), (1056, 2048), (2048, 2562)], 1),
    # shallow, hydrostatic, energy equation (the energy form's extra fields cross the halo)
    "energy_2": (dict(DeepModel=0, NonHydro=0, energy_equation=1), [(0, 768), (768, 2562)], 0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_partitioned_step_is_bitwise_the_whole_step(case):
    over, ranges, precision = CASES[case]
    glevel, nv, dt, n = 4, 16, 1200.0, 2
    p, c = make_params(glevel, dt, **over)
    g = RefGrid(glevel, nv)
    ic = initial_state(g.arrays, g.point_num, nv, c, amp=2.0)
    params = thorx_params(c, dt, precision=precision)
    whole = run_whole(g, glevel, params, ic, n)
    parts = run_partitioned(g, glevel, params, ic, ranges, n)
    g.close()
    for f in FIELDS:
        assert np.array_equal(parts[f], whole[f]), f


@pytest.mark.gpu
def test_partitioned_step_with_radiative_transfer():
    glevel, nv, dt = 4, 20, 300.0
    p, c = hot_jupiter_params(glevel, dt)
    g = RefGrid(glevel, nv, A=c["A"], top=c["Top_altitude"])
    ic = initial_state(g.arrays, g.point_num, nv, c, amp=1.0)
    params = thorx_params(c, dt)
    whole = run_whole(g, glevel, params, ic, 2, rt=RT_WASP43B)
    parts = run_partitioned(g, glevel, params, ic, [(0, 1280), (1280, 2562)], 2, rt=RT_WASP43B)
    g.close()
    for f in FIELDS:
        assert np.array_equal(parts[f], whole[f]), f


@pytest.mark.gpu
def test_partition_arguments_and_whole_grid_calls_are_rejected():
    glevel, nv, dt = 4, 8, 1200.0
    p, c = make_params(glevel, dt)
    g = RefGrid(glevel, nv)
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt))
    x.init_rest_state(300.0)
    for a, b in ((0, 0), (16, 1280), (0, 1000), (-32, 64), (0, 2563)):
        with pytest.raises(thor_b200.ThorxError) as e:
            x.set_partition(a, b)
        assert e.value.code == thor_b200.E_ARG, (a, b)
    x.set_partition(0, 1280)
    with pytest.raises(thor_b200.ThorxError) as e:
        x.globdiag()
    assert e.value.code == thor_b200.E_UNSUPPORTED
    x.set_partition(0, g.point_num)  # the whole grid again: no longer partitioned
    x.globdiag()
    x.close(), g.close()


@pytest.mark.gpu
def test_fp32_divg_of_the_mixed_form():
    """The mixed form keeps divg in FP32 (its values are FP32 results, so the state is the same
    bits as with FP64 storage): modules are refused its device array, which the FP64 form hands
    out; switching forms between steps leaves a usable state (divg is recomputed before every
    use)."""
    glevel, nv, dt = 4, 8, 1200.0
    p, c = make_params(glevel, dt)
    g = RefGrid(glevel, nv)
    ic = initial_state(g.arrays, g.point_num, nv, c, amp=2.0)
    x = thor_b200.Thorx(grid_dict(g), glevel, thorx_params(c, dt, precision=1))
    for k, v in ic.items():
        x.set(k, v)
    with pytest.raises(thor_b200.ThorxError) as e:
        x.device_field("divg")
    assert e.value.code == thor_b200.E_UNSUPPORTED
    x.step(1)
    x.set_precision(0)
    assert x.device_field("divg")[1:3] == (nv, 3)
    x.step(1)
    x.set_precision(1)
    x.step(1)
    x.sync()
    for f in FIELDS:
        assert np.all(np.isfinite(x.get(f))), f
    x.close(), g.close()
