"""Global conserved quantities (ESP::globdiag) and compensated sums: the CPU restatement.

The oracle's per-cell terms follow src/ESP/profx_globdiag.cu:45-252 in the reference's operand
order; its sums are Neumaier-compensated. Here it is checked against an independent numpy
restatement of the same per-cell formulas summed exactly with math.fsum, and its compensated sum
against math.fsum on ill-conditioned data. The GPU tests (test_globdiag_gpu.py) then hold the
product and the reference's own kernels against this oracle.
"""
import math

import numpy as np
import pytest

from thorx_testlib import RefGrid, Oracle, initial_state, make_params, oracle_lib

EPS = np.finfo(np.float64).eps


def numpy_globdiag(g, c, st, deep):
    """Per-cell energy, mass, angular momentum, entropy (reference expressions), exact sums."""
    N, nv = g.point_num, g.nv
    A = c["A"]
    alt, alth = g["Altitude"], g["Altitudeh"]
    areasT = g["areasT"][:, None]
    zup, zlow = alth[1:] + A, alth[:-1] + A
    if deep:
        vol = areasT / A ** 2 * (zup ** 3 - zlow ** 3) / 3
    else:
        vol = areasT * (zup - zlow)
    lon = g["lonlat"][0::2][:, None]
    lat = g["lonlat"][1::2][:, None]
    rho = st["Rho"].reshape(N, nv)
    T = st["temperature"].reshape(N, nv)
    p = st["pressure"].reshape(N, nv)
    W = st["W"].reshape(N, nv)
    Cp = st["Cp"].reshape(N, nv)
    Rd = st["Rd"].reshape(N, nv)
    Mh = st["Mh"].reshape(N, nv, 3)
    m0, m1, m2 = Mh[..., 0], Mh[..., 1], Mh[..., 2]
    wx = W * np.cos(lat) * np.cos(lon)
    wy = W * np.cos(lat) * np.sin(lon)
    wz = W * np.sin(lat)
    Ek = 0.5 * ((m0 + wx) ** 2 + (m1 + wy) ** 2 + (m2 + wz) ** 2) / rho
    E = (Ek + (Cp - Rd) * T * rho + rho * c["Gravit"] * alt[None, :]) * vol
    M = rho * vol
    r = (A + alt)[None, :]
    fr = g["func_r"].reshape(N, 3)
    rx, ry, rz = r * fr[:, 0:1], r * fr[:, 1:2], r * fr[:, 2:3]
    Om = c["Omega"]
    AMx = (ry * m2 - rz * m1 - rho * Om * r * rz * np.cos(lat) * np.cos(lon)) * vol
    AMy = (-rx * m2 + rz * m0 - rho * Om * r * rz * np.cos(lat) * np.sin(lon)) * vol
    AMz = (rx * m1 - ry * m0 + rho * Om * r * r * np.cos(lat) * np.cos(lat)) * vol
    S = Cp * np.log(T * (c["P_Ref"] / p) ** (Rd / Cp)) * vol
    terms = [E, M, AMx, AMy, AMz, S]
    return (np.array([math.fsum(t.ravel()) for t in terms]),
            np.array([math.fsum(np.abs(t).ravel()) for t in terms]))


@pytest.mark.parametrize("over", [{}, dict(DeepModel=0, NonHydro=0, energy_equation=1)])
def test_oracle_globdiag_matches_exact_restatement(over):
    glevel, nv, dt = 4, 8, 1200.0
    g = RefGrid(glevel, nv)
    p, c = make_params(glevel, dt, **over)
    o = Oracle(g, p)
    for k, v in initial_state(g.arrays, g.point_num, nv, c).items():
        o.set(k, v)
    o.step(1)  # winds and vertical velocity no longer zero
    st = {k: o.get(k) for k in ["Rho", "temperature", "pressure", "W", "Cp", "Rd", "Mh"]}
    mine, mag = o.globdiag()
    exact, mag_exact = numpy_globdiag(g, c, st, deep=c["DeepModel"])
    o.close(), g.close()
    assert np.all(mag > 0)
    # per-cell terms: libm vs numpy transcendental functions differ in the last bits
    err = np.abs(mine - exact) / mag_exact
    assert np.all(err <= 1e-13), err
    # shallow-atmosphere mass involves no transcendental function (the deep volume differences
    # zup^3 - zlow^3 amplify libm/numpy pow differences ~500x): exact to a few roundings
    if not c["DeepModel"]:
        assert abs(mine[1] - exact[1]) <= 8 * EPS * mag_exact[1]


def test_oracle_compensated_sum_is_exact_on_ill_conditioned_data():
    rng = np.random.default_rng(7)
    for n in [1, 2, 3, 1000, 100003]:
        big = rng.standard_normal(n) * 1e12
        x = np.concatenate([big, -big[::-1], rng.standard_normal(n)])
        rng.shuffle(x)
        exact = math.fsum(x)
        s = oracle_lib().oracle_sum(x.ctypes.data, x.size)
        bound = 2 * EPS * abs(exact) + 4 * x.size * EPS ** 2 * math.fsum(np.abs(x))
        assert abs(s - exact) <= bound, (n, s, exact)
