"""The thorx_phy shim (include/thorx_phy.h, thor_b200/phy/): physics-module managers written for
the reference's phy_modules_* interface (src/headers/phy_modules.h:57-98) on the thorx dynamical
core, unchanged.

* The reference's own empty manager (src/physics/managers/empty/src/phy_modules.cu), compiled
  unchanged against the shim's headers (tests/modules/Makefile): it links, attaches, and the state
  after two steps is bitwise the state without it.
* The probe of oracle/ref_harness.cu re-expressed as a reference-API manager
  (tests/modules/refapi_probe.cu: reference-layout arrays, device_RK_array_manager, ESP members):
  tracer through the RK registry bitwise equal to the reference's, snapshots at the fast-mode hook
  and the state within the reference's own FMA spread, hook call counts, its configuration key.
"""
import ctypes
import os

import numpy as np
import pytest

import thor_b200
from thorx_testlib import (ROOT, RefGrid, RefSim, field_tolerance, grid_dict, initial_state,
                           make_params, rel_err, splitmix64_uniform, thorx_params)

GLEVEL, NV, DT = 4, 16, 1200.0
BUILD = os.path.join(ROOT, "tests", "modules", "_build")
REFPROBE_SO = os.path.join(BUILD, "libphy_refprobe.so")
EMPTY_SO = os.path.join(BUILD, "libphy_empty.so")


class SetupC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ["A", "Omega", "Gravit", "Rd", "Cp", "Tmean", "P_Ref", "Top_altitude", "Diffc",
                 "Diffc_v", "DivDampc"]] + [
        (n, ctypes.c_int) for n in
        ["GravHeightVar", "DeepModel", "HyDiff", "HyDiffOrder", "DivDampP", "VertHyDiff",
         "VertHyDiffOrder", "NonHydro", "conv_adj", "conv_adj_iter", "soft_adjustment",
         "first_step"]]


def shim_lib(path):
    thor_b200.lib()  # libthorx.so first: the shim links against it
    L = ctypes.CDLL(path)
    L.thorx_phy_attach.argtypes = [ctypes.c_void_p, ctypes.POINTER(thor_b200.GridC),
                                   ctypes.POINTER(SetupC), ctypes.POINTER(ctypes.c_char_p),
                                   ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_void_p)]
    L.thorx_phy_attach.restype = ctypes.c_int
    L.thorx_phy_detach.argtypes = [ctypes.c_void_p]
    L.thorx_phy_name.argtypes = [ctypes.c_char_p, ctypes.c_int]
    return L


def setup_struct(c):
    s = SetupC()
    for n, _ in SetupC._fields_:
        if n in c:
            setattr(s, n, c[n])
    s.Tmean, s.Diffc_v, s.VertHyDiff, s.VertHyDiffOrder = c.get("Tmean", 300.0), 0.0, 0, 6
    s.conv_adj, s.conv_adj_iter, s.soft_adjustment, s.first_step = 0, 1, 0, 1
    return s


class Attached:
    """A thorx context with a shim manager attached (grid arrays kept alive for the call)."""

    def __init__(self, so, g, c, keys=(), values=()):
        self.x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        self.L = shim_lib(so)
        gd = grid_dict(g)
        self.keep = {}
        gc = thor_b200.GridC(g.point_num, g.nv, g.nl_region, g.nr, GLEVEL)
        for k in thor_b200.GRID_KEYS:
            a = np.ascontiguousarray(gd[k], dtype=np.int32 if k in ("maps", "point_local")
                                     else np.float64)
            self.keep[k] = a
            setattr(gc, k, a.ctypes.data)
        self.sim = setup_struct(c)
        ks = (ctypes.c_char_p * max(1, len(keys)))(*[k.encode() for k in keys])
        vs = (ctypes.c_char_p * max(1, len(values)))(*[v.encode() for v in values])
        self.h = ctypes.c_void_p()
        self.rc = self.L.thorx_phy_attach(self.x.h, ctypes.byref(gc), ctypes.byref(self.sim), ks,
                                          vs, len(keys), ctypes.byref(self.h))

    def close(self):
        self.x.close()  # the context first: the manager's arrays are registered with it
        if self.h:
            assert self.L.thorx_phy_detach(self.h) == 0


def test_shim_libraries_link_and_name_their_manager():
    """No GPU needed: the reference's empty manager and the probe manager link against the shim and
    libthorx.so, and export the shim's entry points."""
    for so, name in ((EMPTY_SO, b"empty"), (REFPROBE_SO, b"refapi_probe")):
        L = shim_lib(so)
        for f in ("thorx_phy_attach", "thorx_phy_detach", "thorx_phy_name"):
            assert hasattr(L, f), (so, f)
        buf = ctypes.create_string_buffer(64)
        assert L.thorx_phy_name(buf, 64) == 0
        assert buf.value == name


def tracer0(N):
    """Seeded initial tracer in the reference layout [col][lev][2]."""
    return (1.0 + splitmix64_uniform(2 * NV * N, 99)).reshape(2, NV, N).transpose(2, 1, 0).copy()


@pytest.mark.gpu
def test_reference_empty_manager_leaves_the_state_unchanged():
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = initial_state(g.arrays, g.point_num, NV, c, amp=2.0)
    res = []
    for attach in (False, True):
        if attach:
            a = Attached(EMPTY_SO, g, c)
            assert a.rc == 0
            x = a.x
        else:
            x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        for k, v in st.items():
            x.set(k, v)
        x.step(2)
        x.sync()
        res.append({f: x.get(f) for f in ("Rho", "pressure", "Mh", "Wh", "W")})
        a.close() if attach else x.close()
    g.close()
    for f in res[0]:
        assert np.array_equal(res[0][f], res[1][f]), f


@pytest.mark.gpu
def test_unknown_module_key_is_rejected():
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    a = Attached(REFPROBE_SO, g, c, keys=["no_such_key"], values=["1"])
    assert a.rc == thor_b200.E_ARG and not a.h
    a.close()
    a = Attached(REFPROBE_SO, g, c, keys=["probe_heating"], values=["warm"])
    assert a.rc == thor_b200.E_ARG and not a.h
    a.close()
    g.close()


@pytest.mark.gpu
def test_reference_api_probe_matches_the_reference_hooks():
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = initial_state(g.arrays, g.point_num, NV, c, amp=2.0)
    N = g.point_num
    out = {}
    for who in ("reference", "reference_nofma", "product"):
        if who == "product":
            a = Attached(REFPROBE_SO, g, c, keys=["probe_heating"], values=["0.5"])
            assert a.rc == 0
            x, L = a.x, a.L
            L.refprobe_io.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
            L.refprobe_calls.restype = ctypes.c_longlong
            t = tracer0(N)
            assert L.refprobe_io(b"set_tracer", t.ctypes.data) == 0
        else:
            x = RefSim(g, p, nofma=(who == "reference_nofma"))
            x.probe()
            x.set("tracer", tracer0(N).reshape(-1))
        for k, v in st.items():
            x.set(k, v)
        x.step(1)
        if who == "product":
            x.sync()
            r = {}
            for name, n in (("tracer", 2 * N * NV), ("snap_Rhos", N * NV), ("snap_Whs", N * (NV + 1))):
                r[name] = np.zeros(n)
                assert L.refprobe_io(name.encode(), r[name].ctypes.data) == 0
            calls = [L.refprobe_calls(i) for i in range(5)]
        else:
            r = {f: x.get(f) for f in ("tracer", "snap_Rhos", "snap_Whs")}
        for f in ("Rho", "pressure", "Mh", "Wh", "temperature"):
            r[f] = x.get(f)
        out[who] = r
        a.close() if who == "product" else x.close()
    g.close()
    ref, ref_nf, got = out["reference"], out["reference_nofma"], out["product"]
    np.testing.assert_allclose(ref["tracer"], tracer0(N).reshape(-1) + DT, rtol=1e-13)
    assert np.array_equal(got["tracer"], ref["tracer"])
    assert calls == [1, 3, 10, 1, 1], calls
    bad = {}
    for f in ("snap_Rhos", "snap_Whs", "Rho", "pressure", "Mh", "Wh", "temperature"):
        err, spread = rel_err(got[f], ref[f]), rel_err(ref_nf[f], ref[f])
        if not err <= field_tolerance(spread, floor=1e-11):
            bad[f] = (err, spread)
    assert not bad, bad
    assert np.abs(ref["snap_Rhos"]).max() > 0
