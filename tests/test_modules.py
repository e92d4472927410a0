"""Physics-module interface (thorx_module_add, thorx_rk_register_array, thorx_device_field).

The probe module (tests/modules/probe_module.cu) and the harness's probe (oracle/ref_harness.cu)
do the same things at the reference's module hook points (src/ESP/thor_driver.cu:116,641,1290,
1465; src/ESP/profx_driver.cu:405-416): a two-component tracer with a tendency of 1 per second
carried through the RK array registry, snapshots of Rhos and Whs between Vertical_Eq and
Density_Pressure_Eqs of the last small step, and +0.5 K on the temperature before the pressure
update. The harness's tracer goes through the reference's own device_RK_array_manager and
UpdateRK / UpdateRK2, so the registry's semantics are checked against the reference's code; the
snapshots check that the fast-mode hook sees the state the reference's hook sees.
"""
import ctypes
import os

import numpy as np
import pytest

import thor_b200
from thorx_testlib import (ROOT, RefGrid, RefSim, field_tolerance, grid_dict, initial_state,
                           make_params, rel_err, splitmix64_uniform, thorx_params)

GLEVEL, NV, DT = 4, 16, 1200.0
PROBE_SO = os.path.join(ROOT, "tests", "modules", "_build", "libprobe_module.so")


def test_module_entry_points_are_exported():
    L = thor_b200.lib()
    for f in ("thorx_module_add", "thorx_rk_register_array", "thorx_device_field"):
        assert hasattr(L, f), f


def probe_lib():
    thor_b200.lib()  # libthorx.so first: the probe links against it
    P = ctypes.CDLL(PROBE_SO)
    P.probe_create.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    P.probe_create.restype = ctypes.c_int
    P.probe_io.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p]
    P.probe_io.restype = ctypes.c_int
    P.probe_calls.argtypes = [ctypes.c_void_p, ctypes.c_int]
    P.probe_calls.restype = ctypes.c_longlong
    P.probe_destroy.argtypes = [ctypes.c_void_p]
    return P


def tracer0(N):
    """Seeded initial tracer, component-major [2][nv][N]."""
    return (1.0 + splitmix64_uniform(2 * NV * N, 99)).reshape(2, NV, N)


class Product:
    def __init__(self, g, c, flags):
        self.x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        self.P = probe_lib()
        self.N = g.point_num
        self.p = ctypes.c_void_p()
        if flags is not None:
            assert self.P.probe_create(self.x.h, flags, ctypes.byref(self.p)) == 0
            t = np.ascontiguousarray(tracer0(self.N))
            assert self.P.probe_io(self.p, b"set_tracer", self.N, t.ctypes.data) == 0

    def io(self, what, rows):
        a = np.zeros((rows, self.N))
        assert self.P.probe_io(self.p, what.encode(), self.N, a.ctypes.data) == 0
        return a

    def calls(self):
        return [self.P.probe_calls(self.p, i) for i in range(5)]

    def close(self):
        if self.p:
            self.P.probe_destroy(self.p)
        self.x.close()


def state(g, c):
    return initial_state(g.arrays, g.point_num, NV, c, amp=2.0)


@pytest.mark.gpu
def test_probe_module_matches_the_reference_hooks():
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = state(g, c)
    N = g.point_num
    out = {}
    for who in ("reference", "reference_nofma", "product"):
        if who == "product":
            pr = Product(g, c, 3)
            x = pr.x
        else:
            x = RefSim(g, p, nofma=(who == "reference_nofma"))
            x.probe()
            x.set("tracer", tracer0(N).transpose(2, 1, 0).reshape(-1))  # [col][lev][2]
        for k, v in st.items():
            x.set(k, v)
        x.step(1)
        if who == "product":
            x.sync()
            r = {"tracer": pr.io("tracer", 2 * NV).reshape(2, NV, N),
                 "snap_Rhos": pr.io("snap_Rhos", NV).T.reshape(-1),
                 "snap_Whs": pr.io("snap_Whs", NV + 1).T.reshape(-1)}
            calls = pr.calls()
        else:
            r = {"tracer": x.get("tracer").reshape(N, NV, 2).transpose(2, 1, 0),
                 "snap_Rhos": x.get("snap_Rhos"), "snap_Whs": x.get("snap_Whs")}
        for f in ("Rho", "pressure", "Mh", "Wh"):
            r[f] = x.get(f)
        out[who] = r
        if who == "product":
            pr.close()
        else:
            x.close()
    g.close()
    ref, ref_nf, got = out["reference"], out["reference_nofma"], out["product"]
    # the tracer: a unit tendency over one large step adds dt; the registry's reset and
    # accumulation are elementwise, so product and reference agree to the last bit
    np.testing.assert_allclose(ref["tracer"], tracer0(N) + DT, rtol=1e-13)
    assert np.array_equal(got["tracer"], ref["tracer"])
    assert calls == [1, 3, 10, 1, 1], calls
    bad = {}
    for f in ("snap_Rhos", "snap_Whs", "Rho", "pressure", "Mh", "Wh"):
        err, spread = rel_err(got[f], ref[f]), rel_err(ref_nf[f], ref[f])
        if not err <= field_tolerance(spread, floor=1e-11):
            bad[f] = (err, spread)
    assert not bad, bad
    # the snapshot is Rhos before Density_Pressure_Eqs of the last small step: not the final one
    assert np.abs(ref["snap_Rhos"]).max() > 0


@pytest.mark.gpu
def test_split_vertical_step_is_bitwise_the_fused_one():
    """A fast-mode hook splits the vertical kernel in two launches; the state is the same bits."""
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = state(g, c)
    res = []
    for flags in (None, 2):
        pr = Product(g, c, flags)
        for k, v in st.items():
            pr.x.set(k, v)
        pr.x.step(3)
        pr.x.sync()
        res.append({f: pr.x.get(f) for f in ("Rho", "pressure", "Mh", "Wh", "W")})
        if flags:
            assert pr.x.kernels_per_step() > 49 + 10  # split vertical and the registry kernels
        pr.close()
    g.close()
    for f in res[0]:
        assert np.array_equal(res[0][f], res[1][f]), f


@pytest.mark.gpu
def test_graph_replay_and_eager_calls_agree():
    """thorx_step captures the hooks once and replays their work; thorx_profx + thorx_thor call
    them every step. Both give the same bits."""
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = state(g, c)
    res, calls = [], []
    for eager in (False, True):
        pr = Product(g, c, 3)
        for k, v in st.items():
            pr.x.set(k, v)
        for _ in range(3):
            if eager:
                pr.x.profx()
                pr.x.thor()
            else:
                pr.x.step(1)
        pr.x.sync()
        res.append({f: pr.x.get(f) for f in ("Rho", "pressure", "Mh")})
        res[-1]["tracer"] = pr.io("tracer", 2 * NV)
        calls.append(pr.calls())
        pr.close()
    g.close()
    for f in res[0]:
        assert np.array_equal(res[0][f], res[1][f]), f
    np.testing.assert_allclose(res[0]["tracer"], tracer0(g.point_num).reshape(2 * NV, -1) + 3 * DT,
                               rtol=1e-13)
    assert calls[0] == [1, 3, 10, 1, 1]            # captured once
    assert calls[1] == [3, 9, 30, 3, 3]            # called every step
