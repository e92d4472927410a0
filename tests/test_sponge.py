"""Rayleigh sponge layer (RayleighSponge with raysp_calc_mode = imp) in ProfX.

The product (thorx_sponge_enable) and the CPU restatement against the reference's own kernels:
zonal_uv / zonal_w / zonal_temp, the per-bin sums of gpu_sum_on_device_sponge and sponge_layer
(src/ESP/profx_sponge.cu, src/headers/reduction_add.h:242-288), launched by oracle/ref_harness.cu
where src/ESP/profx_driver.cu:96-194 launches them, with the reference grid's own zonal-mean table
(Icogrid::zonal_mean_tab_f, src/ESP/grid.cu:3203-3260). The test state has a zonal jet plus seeded
noise in the horizontal and vertical winds, so that the means, the interpolation between bins and
the relaxation all act. Tolerances as in the dynamical-core tests: 1e-12 of max|field|, or 4x the
spread between the reference's FMA and no-FMA builds where that is larger.
"""
import numpy as np
import pytest

import thor_b200
from thorx_testlib import (Oracle, RefGrid, RefSim, field_tolerance, grid_dict, initial_state,
                           make_params, rel_err, splitmix64_uniform, thorx_params)

GLEVEL, NV, DT, NLAT = 4, 16, 1200.0, 20


def windy_state(g, c, seed=7):
    """initial_state plus a zonal jet u = 40 cos(lat) m/s, seeded noise of 5 m/s in u and v and of
    0.5 m/s in w at the interfaces (w at the centres from Recompute_W's interpolation)."""
    N = g.point_num
    st = initial_state(g.arrays, N, NV, c)
    lon = g["lonlat"][0::2].repeat(NV)
    lat = g["lonlat"][1::2].repeat(NV)
    rho = st["Rho"]
    u = 40.0 * np.cos(lat) + 5.0 * (2 * splitmix64_uniform(N * NV, seed) - 1)
    v = 5.0 * (2 * splitmix64_uniform(N * NV, seed + 1) - 1)
    ex = np.stack([-np.sin(lon), np.cos(lon), np.zeros_like(lon)], 1)
    ey = np.stack([-np.sin(lat) * np.cos(lon), -np.sin(lat) * np.sin(lon), np.cos(lat)], 1)
    st["Mh"] = ((u[:, None] * ex + v[:, None] * ey) * rho[:, None]).reshape(-1)
    wh = 0.5 * (2 * splitmix64_uniform(N * (NV + 1), seed + 2) - 1)
    wh = wh.reshape(N, NV + 1)
    wh[:, 0] = wh[:, NV] = 0.0  # rigid bottom and top
    rho_c = rho.reshape(N, NV)
    rho_h = np.concatenate([rho_c[:, :1], 0.5 * (rho_c[:, 1:] + rho_c[:, :-1]), rho_c[:, -1:]], 1)
    st["Wh"] = (wh * rho_h).reshape(-1)
    return st


def zonal_table(lat, nlat):
    """Icogrid::zonal_mean_tab_f restated: (bin, members of the bin, slot) per column."""
    des = np.pi / nlat
    edges = [-np.pi / 2.0]
    for _ in range(nlat):
        edges.append(edges[-1] + des)
    N = lat.size
    tab = np.zeros((N, 3), dtype=np.int64)
    count = np.zeros(nlat, dtype=np.int64)
    for i in range(N):
        b = 0
        for j in range(nlat):
            if edges[j] <= lat[i] < edges[j + 1]:
                b = j
                break
        if lat[i] >= edges[nlat]:
            b = nlat - 1
        tab[i, 0], tab[i, 2] = b, count[b]
        count[b] += 1
    tab[:, 1] = count[tab[:, 0]]
    return tab


def test_latitude_bins_match_the_reference_table():
    for nlat in (20, 7):
        g = RefGrid(GLEVEL, NV, nlat=nlat)
        ref = g["zonal_mean_tab"].reshape(-1, 3)
        mine = zonal_table(g["lonlat"][1::2], nlat)
        assert np.array_equal(ref, mine), nlat
        g.close()


def oracle_run(d, nsteps=1, state=None):
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = state or windy_state(g, c)
    o = Oracle(g, p)
    for k, v in st.items():
        o.set(k, v)
    if d is not None:
        o.sponge(d)
    o.step(nsteps, profx=True, thor=False)
    out = {f: o.get(f) for f in ("Mh", "W", "Wh", "pressure")}
    means = o.sponge_means() if d is not None else None
    o.close()
    return g, c, st, out, means


def test_restatement_means_and_relaxation():
    """The oracle's zonal means are the bin averages of u, v, w (and T); without damping to the
    mean, every wind component above ns is divided by 1 + k dt with k = R sin^2(...), and the
    levels below ns are left as they are."""
    d = dict(nlat_bins=NLAT, ns_ray_sponge=0.5, damp_uv_to_mean=0, damp_w_to_mean=0,
             RayleighSpongeT=1, Ruv_sponge=2e-4, Rw_sponge=5e-4)
    g, c, st, out, (vbar, tbar) = oracle_run(d)
    _, _, _, base, _ = oracle_run(None, state=st)
    N = g.point_num
    alt, ztop = g["Altitude"], g["Altitudeh"][NV]
    n = alt / ztop
    k = np.where(n >= 0.5, np.sin(0.5 * np.pi * (n - 0.5) / (1 - 0.5)) ** 2, 0.0)
    Mh0, Mh1 = base["Mh"].reshape(N, NV, 3), out["Mh"].reshape(N, NV, 3)
    W0, W1 = base["W"].reshape(N, NV), out["W"].reshape(N, NV)
    np.testing.assert_allclose(Mh1, Mh0 / (1 + 2e-4 * DT * k)[None, :, None], rtol=0,
                               atol=1e-13 * np.abs(Mh0).max())
    np.testing.assert_allclose(W1, W0 / (1 + 5e-4 * DT * k)[None, :], rtol=0,
                               atol=1e-13 * np.abs(W0).max())
    assert k[0] == 0 and k[-1] > 0.5  # both sides of ns are covered
    # the thermal sponge's mean temperature is the bin average of p / (Rd rho)
    tab = zonal_table(g["lonlat"][1::2], NLAT)
    T = (st["pressure"] / st["Rd"] / st["Rho"]).reshape(N, NV)
    for b in (0, 5, NLAT - 1):
        sel = tab[:, 0] == b
        np.testing.assert_allclose(tbar[b], T[sel].mean(0), rtol=1e-13)
    # damping to the mean: the means are the bin averages of u, v and of w from Recompute_W
    d2 = dict(d, damp_uv_to_mean=1, damp_w_to_mean=1)
    _, _, _, _, (vbar2, _) = oracle_run(d2, state=st)
    lon, lat = g["lonlat"][0::2], g["lonlat"][1::2]
    rho = st["Rho"].reshape(N, NV)
    M = st["Mh"].reshape(N, NV, 3)
    u = (M[..., 0] * -np.sin(lon)[:, None] + M[..., 1] * np.cos(lon)[:, None]) / rho
    for b in (0, 9, NLAT - 1):
        sel = tab[:, 0] == b
        np.testing.assert_allclose(vbar2[b, :, 0], u[sel].mean(0), rtol=1e-12, atol=1e-12)


def run(who, d, nsteps=1, thor=False):
    nlat = d["nlat_bins"]
    g = RefGrid(GLEVEL, NV, nlat=nlat)
    p, c = make_params(GLEVEL, DT)
    st = windy_state(g, c)
    if who == "product":
        x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        x.sponge(d)
    elif who == "oracle":
        x = Oracle(g, p)
        x.sponge(d)
    else:
        x = RefSim(g, p, nofma=(who == "reference_nofma"))
        x.sponge(g, d)
    for k, v in st.items():
        x.set(k, v)
    if who == "product":
        if thor:
            x.step(nsteps)
        else:
            for _ in range(nsteps):
                x.profx()
        x.sync()
    else:
        x.step(nsteps, profx=True, thor=thor)
    fields = ["Mh", "W", "Wh", "pressure", "temperature"] + (["Rho"] if thor else [])
    out = {f: x.get(f) for f in fields}
    out["vbar"], out["Tbar"] = x.sponge_means()
    x.close(), g.close()
    return out


CASES = {
    "defaults": dict(nlat_bins=NLAT),
    "to_zero": dict(nlat_bins=NLAT, damp_uv_to_mean=0, damp_w_to_mean=0, ns_ray_sponge=0.5),
    "thermal": dict(nlat_bins=NLAT, RayleighSpongeT=1, ns_ray_sponge=0.4, Ruv_sponge=3e-4,
                    RT_sponge=2e-4),
    "bins7_w_only": dict(nlat_bins=7, damp_uv_to_mean=0, ns_ray_sponge=0.3, Rw_sponge=1e-3),
    # the sponge at exp(-2) of its strength and weakening from step to step
    "shrinking": dict(nlat_bins=NLAT, shrink_sponge=1, t_shrink=1000, first_step=3000,
                      RayleighSpongeT=1, Ruv_sponge=1e-2, Rw_sponge=1e-2, RT_sponge=1e-2),
    # the explicit modes: tendencies in every RK stage of the dynamical core, means from the
    # first stage (exp1) or every stage (exp3)
    "exp1": dict(nlat_bins=NLAT, raysp_calc_mode=1, ns_ray_sponge=0.5, Ruv_sponge=1e-3,
                 Rw_sponge=1e-3),
    "exp3_thermal_shrinking": dict(nlat_bins=NLAT, raysp_calc_mode=2, RayleighSpongeT=1,
                                   shrink_sponge=1, t_shrink=1000, first_step=3000,
                                   Ruv_sponge=1e-2, Rw_sponge=1e-2, RT_sponge=1e-2),
}


@pytest.mark.gpu
@pytest.mark.parametrize("who", ["product", "oracle"])
@pytest.mark.parametrize("case,nsteps,thor", [
    ("defaults", 1, False), ("to_zero", 1, False), ("thermal", 1, False),
    ("bins7_w_only", 1, False), ("shrinking", 2, False), ("defaults", 3, True),
    ("thermal", 3, True), ("exp1", 2, True), ("exp3_thermal_shrinking", 2, True)])
def test_sponge_matches_reference(who, case, nsteps, thor):
    d = CASES[case]
    ref = run("reference", d, nsteps, thor)
    ref_nf = run("reference_nofma", d, nsteps, thor)
    got = run(who, d, nsteps, thor)
    bad, res = {}, {}
    for f in ref:
        if f == "Tbar" and not d.get("RayleighSpongeT"):
            continue
        if f == "vbar":  # components the configuration does not average stay unchecked
            keep = [k for k, on in ((0, d.get("damp_uv_to_mean", 1)), (1, d.get("damp_uv_to_mean", 1)),
                                    (2, d.get("damp_w_to_mean", 1))) if on]
            if not keep:
                continue
            a, b, bn = got[f][..., keep], ref[f][..., keep], ref_nf[f][..., keep]
        else:
            a, b, bn = got[f], ref[f], ref_nf[f]
        assert np.all(np.isfinite(b)), f
        err, spread = rel_err(a, b), rel_err(bn, b)
        tol = field_tolerance(spread, floor=1e-11 if thor else 1e-12)
        res[f] = (err, spread)
        if not err <= tol:
            bad[f] = (err, tol)
    assert not bad, {"failures": bad, "all": res}
    # the sponge acts: the winds at the top differ from a run without it
    base = run_plain(nsteps, thor)
    assert rel_err(ref["Mh"], base["Mh"]) > 1e-6


def run_plain(nsteps, thor):
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = windy_state(g, c)
    x = Oracle(g, p)
    for k, v in st.items():
        x.set(k, v)
    x.step(nsteps, profx=True, thor=thor)
    out = {"Mh": x.get("Mh")}
    x.close(), g.close()
    return out


@pytest.mark.gpu
def test_sponge_off_again_restores_plain_profx():
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = windy_state(g, c)
    outs = []
    for on_then_off in (False, True):
        x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        if on_then_off:
            x.sponge(dict(nlat_bins=NLAT))
            x.sponge(None)
        for k, v in st.items():
            x.set(k, v)
        x.step(2)
        x.sync()
        outs.append(x.get("Mh"))
        x.close()
    g.close()
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
def test_runner_with_the_sponge(tmp_path):
    """bin/esp with RayleighSponge = true (the keys of the reference's ifile/wasp43b_ex.thr)."""
    import io
    from thor_b200 import esp
    from test_esp_cli import HS_THR
    cfg = tmp_path / "hs_sponge.thr"
    cfg.write_text(HS_THR.replace("RayleighSponge = false", "RayleighSponge = true")
                   + "nlat_bins = 20\nns_ray_sponge = 0.75\nRuv_sponge = 1e-4\n"
                   + "damp_uv_to_mean = true\ndamp_w_to_mean = true\nraysp_calc_mode = imp\n")
    out = io.StringIO()
    assert esp.run([str(cfg), "-o", str(tmp_path / "o")], out) == 0, out.getvalue()
    from thor_b200 import h5
    final = h5.read(str(tmp_path / "o" / "esp_output_TestHS_2.h5"))
    assert int(final["nstep"][0][0]) == 4 and np.all(np.isfinite(final["Mh"][0]))
    planet = h5.read(str(tmp_path / "o" / "esp_output_planet_TestHS.h5"))
    assert planet["RayleighSponge"][0][0] == 1.0 and planet["nlat_bins"][0][0] == 20


@pytest.mark.gpu
def test_reconfiguring_the_sponge_replaces_it():
    """A second thorx_sponge_enable (other bins, after steps with the first) gives the steps of a
    context that had only the second one; the first set-up's tables are released."""
    g = RefGrid(GLEVEL, NV)
    p, c = make_params(GLEVEL, DT)
    st = windy_state(g, c)
    second = dict(nlat_bins=7, ns_ray_sponge=0.4, Ruv_sponge=5e-4)
    outs = []
    for reconfigure in (False, True):
        x = thor_b200.Thorx(grid_dict(g), GLEVEL, thorx_params(c, DT))
        if reconfigure:
            x.sponge(dict(nlat_bins=NLAT))
            for k, v in st.items():
                x.set(k, v)
            x.step(2)
            x.sync()
        x.sponge(second)
        for k, v in st.items():
            x.set(k, v)
        x.step(2)
        x.sync()
        outs.append((x.get("Mh"), x.sponge_means()[0]))
        x.close()
    g.close()
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
