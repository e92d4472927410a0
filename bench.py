"""Throughput of the thorx HE-VI dynamical core on B200: simulated days per wall-hour.

Workload (the bench configuration): Earth Held-Suarez on the icosahedral grid of glevel 6
(40962 columns) x 48 levels, dt = 600 s, DeepModel + NonHydro, entropy equation, 4th-order
hyperdiffusion and 3D divergence damping (the reference ifile/earth_hstest.thr switches),
isothermal 300 K rest state with seeded +-0.1 K noise. One "step" = one large step: ProfX
(Held-Suarez) + Thor (3 RK stages, 10 small steps), replayed as one CUDA graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form fp64|mixed] [--impl reference]

N > 1 runs one process per GPU under torchrun, each an independent replica of the workload
(the north-star path is single-GPU; there is no exchange between replicas): weak scaling, the
job's value is the sum over replicas with the slowest replica's time.

--impl reference times the reference side: the CPU restatement of the same step (oracle/, the
reference itself is CUDA-only) on all host cores, and, alongside, the reference's own FP64 CUDA
kernels (oracle/_ref, compiled from its sources) on the same GPU.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GLEVEL, NV, DT = 6, 48, 600.0
EARTH = dict(A=6.371e6, Omega=7.292e-5, Gravit=9.8, Rd=287.0, Cp=1005.0, P_Ref=1e5,
             Top_altitude=36e3, Diffc=0.0048, DivDampc=0.0048, HyDiffOrder=4, DeepModel=1,
             NonHydro=1, GravHeightVar=0, HyDiff=1, DivDampP=1, thermo_equation=0,
             core_benchmark=1)
TMEAN, SEED, NOISE = 300.0, 20260101, 0.1
# the prognostic state a step reads and writes: the fields of the reference's restart files
# (src/ESP/esp_initial.cu:1215-1260); W is diagnostic (ProfX recomputes it from Wh first)
STATE = ["Rho", "pressure", "Mh", "Wh"]
FALLBACK_HBM_GBS = 6650.0


CPU_SAMPLE_STEPS = 6  # oracle steps timed for cpu_baseline at g6/L48: ~10 s on 16 cores


def workload_name():
    return "Held-Suarez g%d/L%d dt=%g (%d columns x %d levels)" % (
        GLEVEL, NV, DT, 2 + 10 * 4 ** GLEVEL, NV)


def sim_days_per_hour(nsteps, seconds, dt=DT):
    return (nsteps * dt / 86400.0) / (seconds / 3600.0)


def set_workload(glevel, nv):
    global GLEVEL, NV
    GLEVEL, NV = glevel, nv


def params(form):
    p = dict(EARTH)
    p.update(timestep=DT, precision={"fp64": 0, "mixed": 1}[form])
    return p


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax = float(c[2])
            except ValueError:
                continue
            for n, v in zip(names, c[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=None)
    return world, rank, local


def max_over_ranks(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def grid_for_bench():
    import thor_b200
    return thor_b200.Icogrid(GLEVEL, NV, A=EARTH["A"], Top_altitude=EARTH["Top_altitude"])


def ncu_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, scaled to this workload."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    k = d.get("kernels", {}).get(kernel)
    if not k:
        return None
    return k["dram_bytes_per_launch"] * (GLEVEL == d["glevel"] and NV == d["nv"] and 1.0
                                         or (2 + 10 * 4 ** GLEVEL) * NV
                                         / ((2 + 10 * 4 ** d["glevel"]) * d["nv"]))


def cpu_baseline(grid, nsteps, warmup=1):
    """The CPU restatement of the same step (oracle/) on all host cores, bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from thorx_testlib import Oracle, make_params, oracle_lib
    threads = os.cpu_count() or 1
    oracle_lib().oracle_set_threads(threads)
    p, c = make_params(GLEVEL, DT)
    o = Oracle(grid, p)
    st = initial_state_host(grid)
    for k, v in st.items():
        o.set(k, v)
    if warmup:
        o.step(warmup)
    t0 = time.perf_counter()
    o.step(nsteps)
    sec = time.perf_counter() - t0
    o.close()
    return dict(value=sim_days_per_hour(nsteps, sec), unit="sim-days/wall-hour", cores=threads,
                kind="port", seconds=sec,
                sample="%d large steps of the g%d/L%d Held-Suarez step (after %d warm-up), "
                       "oracle/thor_oracle.cpp, OpenMP over columns" % (nsteps, GLEVEL, NV, warmup))


def bench_config(form, world):
    """The config dict of both arms' JSON lines (the same workload, the same keys)."""
    n = 2 + 10 * 4 ** GLEVEL
    return {"workload": workload_name(), "glevel": GLEVEL, "nv": NV, "dt": DT, "form": form,
            "parallelism": "replicas%d" % world,
            "l2": "state resident in HBM (%.3f GB per level-field x ~40 fields), far above the "
                  "126 MB L2: no flush needed" % (n * NV * 8 / 1e9)}


def initial_state_host(grid):
    """The same seeded rest state thorx_init_rest_state builds, via the test helper."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from thorx_testlib import initial_state
    c = dict(EARTH)
    c.update(Tmean=TMEAN, energy_equation=0, held_suarez=1)
    return initial_state(grid.arrays, grid.point_num, grid.nv, c, seed=SEED, amp=NOISE)


def reference_grid():
    """The reference's own grid builder (Icogrid, src/ESP/grid.cu, compiled into oracle/_ref),
    so that the reference arm maps none of the product's code."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from thorx_testlib import RefGrid
    return RefGrid(GLEVEL, NV, A=EARTH["A"], top=EARTH["Top_altitude"])


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0  # rank 0 alone runs the reference arm
    grid = reference_grid()
    # all K steps are timed (after W warm-up steps): each is one whole large step on the CPU
    base = cpu_baseline(grid, args.steps, warmup=args.warmup)
    value = base["value"]
    ref_cuda = reference_cuda(grid, args)
    grid.close()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "sim-days/wall-hour",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": base["seconds"] * 1000.0 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded isothermal rest state, Held-Suarez forcing)",
            "config": bench_config("fp64", world),
            "cpu_baseline": {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": value, "unit": "sim-days/wall-hour", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_cuda": ref_cuda}
    print(json.dumps(line), flush=True)
    return 0


def reference_cuda(grid, args):
    """The reference's own FP64 CUDA kernels (oracle/_ref) on this GPU, same workload."""
    try:
        import ctypes
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import torch
        from thorx_testlib import Params, make_params, ref_lib
        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        lib = ref_lib()

        class View(ctypes.Structure):
            _fields_ = [("point_num", ctypes.c_int), ("nv", ctypes.c_int),
                        ("nl_region", ctypes.c_int), ("nr", ctypes.c_int)] + [
                (n, ctypes.c_void_p) for n in
                ["maps", "point_local", "Altitude", "Altitudeh", "lonlat", "areas", "areasT",
                 "areasTr", "nvecoa", "nvecti", "nvecte", "div", "grad", "func_r"]]
        keep = {k: np.ascontiguousarray(grid[k]) for k in grid.arrays}
        v = View(grid.point_num, grid.nv, grid.nl_region, grid.nr,
                 *[keep[k].ctypes.data for k in
                   ["maps", "point_local", "Altitude", "Altitudeh", "lonlat", "areas", "areasT",
                    "areasTr", "nvecoa", "nvecti", "nvecte", "div", "grad", "func_r"]])
        lib.ref_sim_new_view.restype = ctypes.c_void_p
        lib.ref_sim_new_view.argtypes = [ctypes.POINTER(View), ctypes.POINTER(Params)]
        p, c = make_params(GLEVEL, DT)
        h = lib.ref_sim_new_view(ctypes.byref(v), ctypes.byref(p))
        if not h:
            return {"unavailable": "ref_sim_new_view failed"}
        for k, a in initial_state_host(grid).items():
            a = np.ascontiguousarray(a)
            lib.ref_sim_set(h, k.encode(), a.ctypes.data)
        lib.ref_sim_step(h, args.warmup, 1, 1)
        k = max(1, args.steps)
        ms = lib.ref_sim_time(h, k)
        lib.ref_sim_free(h)
        return {"value": sim_days_per_hour(k, ms / 1000.0), "unit": "sim-days/wall-hour",
                "ms_per_step": ms / k, "steps": k,
                "what": "reference FP64 CUDA kernels (compiled from its sources for sm_100a, "
                        "default stream, synchronised after every launch as in thor_driver.cu)"}
    except Exception as e:  # the side measurement never breaks the reference line
        return {"unavailable": "%s" % e}


METRIC = "sim-days/wall-hour at glevel6 L48, mixed+surrogate vs plain FP64; HBM GB/s"


def time_steps(x, stream, precision, nsteps):
    """ms per large step of a context in the given precision form (graph replays, CUDA events)."""
    import torch
    x.set_precision(precision)
    x.step(3)
    x.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    x.step(nsteps)
    e1.record(stream)
    e1.synchronize()
    x.sync()
    return e0.elapsed_time(e1) / nsteps


# Hot Jupiter with double-gray RT (the RT configuration): R = 1e8 m, g = 10, Rd = 3714,
# Cp = 13000, surface 100 bar, top at 1e-3 bar, dt = 300 s, synchronous rotation with the
# substellar point at longitude 0, gray opacities 4e-4 (SW) and 1e-3 (LW) m^2/kg, irradiation
# temperature 2000 K (Tstar 4300 K, R* = 0.667 R_sun, a = R* (Tstar / T_irr)^2). Initial state:
# the Guillot profile (init_PT_profile = guillot) with T_eq = T_irr / sqrt(2), Tint = 100 K and the
# RT's gray opacities, with seeded +-1 K noise; the model top is the altitude of 1e-3 bar in an
# isothermal column at T_eq.
RT_GLEVEL, RT_NV, RT_DT = 5, 40, 300.0
RT_TIRR, RT_TSTAR, RT_RSTAR = 2000.0, 4300.0, 0.667 * 695700000.0


def rt_params_planet():
    teq = RT_TIRR / 2 ** 0.5
    top = 3714.0 * teq / 10.0 * np.log(1e7 / 1e2)
    p = dict(A=1e8, Omega=9.09e-5, Gravit=10.0, Rd=3714.0, Cp=13000.0, P_Ref=1e7, Top_altitude=top,
             timestep=RT_DT, Diffc=0.015, DivDampc=0.015, HyDiffOrder=4, DeepModel=1, NonHydro=1,
             GravHeightVar=0, HyDiff=1, DivDampP=1, thermo_equation=0, core_benchmark=0,
             precision=0)
    rt = dict(Tstar=RT_TSTAR, radius_star=RT_RSTAR,
              planet_star_dist=RT_RSTAR * (RT_TSTAR / RT_TIRR) ** 2, diff_ang=0.5, Tint=100.0,
              albedo=0.0, kappa_sw=4e-4, kappa_lw=1e-3, kappa_lw_pole=1e-3, n_sw=1.0, n_lw=2.0,
              f_lw=0.5, sync_rot=1, alpha_i=0.0)
    return p, rt, teq


def rt_surrogate_leg(torch, thor_b200, nlog=200, iters=5000, batch=8192, nsteps=20,
                     catch=True, online_chunks=5, online_every=20, online_iters=300):
    """Plain FP64 + RT against mixed + trained surrogate RT on the RT configuration (g5/L40):
    time the plain form, log the plain RT, train the surrogate on the GPU, time the other form."""
    try:
        p, rt, teq = rt_params_planet()
        grid = thor_b200.Icogrid(RT_GLEVEL, RT_NV, A=p["A"], Top_altitude=p["Top_altitude"])
        stream = torch.cuda.Stream()
        x = thor_b200.Thorx(grid.as_dict(), RT_GLEVEL, p, stream=stream.cuda_stream)
        x.init_guillot_state(teq, rt["Tint"], rt["f_lw"], rt["kappa_sw"], rt["kappa_lw"], SEED, 1.0)
        x.rt_enable(rt)
        x.sur_create(hidden=512, train_batch=batch, log_capacity=nlog * grid.point_num,
                     recheck_period=16, tolerance=0.05, seed=SEED)
        ms_plain = time_steps(x, stream, thor_b200.FP64, nsteps)
        kms_plain = dict(zip([t[0] for t in x.kernel_table()], x.profile_steps(1)))
        x.sur_mode(thor_b200.SUR_LOG)
        x.step(nlog)
        x.sync()
        t0 = time.perf_counter()
        n_fine = iters // 5 # the last fifth of the iterations at a fifth of the learning rate
        first, last = x.sur_train(iters - n_fine, batch, lr=1e-3)
        if n_fine:
            _, last = x.sur_train(n_fine, batch, lr=2e-4)
        torch.cuda.synchronize()
        train_s = time.perf_counter() - t0
        # online learning: the surrogate runs, the columns the plain RT re-checks or falls back to
        # are logged, and the network trains between chunks of steps
        x.sur_mode(thor_b200.SUR_USE_LOG)
        x.sur_stats()
        t1, online = time.perf_counter(), {"steps": 0, "rt_columns": 0, "rechecked": 0, "failed": 0}
        for _ in range(online_chunks):
            x.step(online_every)
            x.sync()
            so = x.sur_stats()
            for k in ("rt_columns", "rechecked", "failed"):
                online[k] += so[k]
            online["steps"] += online_every
            x.sur_train(online_iters, batch, lr=2e-4)
        torch.cuda.synchronize()
        online["seconds"] = time.perf_counter() - t1
        online["rt_column_fraction"] = online["rt_columns"] / max(1, online["steps"] * grid.point_num)
        online["what"] = ("%d chunks of %d steps, %d Adam steps (lr 2e-4) after each"
                          % (online_chunks, online_every, online_iters))
        x.sur_mode(thor_b200.SUR_USE)
        x.sur_stats()
        ms_sur = time_steps(x, stream, thor_b200.MIXED, nsteps)
        st = x.sur_stats()
        kms_sur = dict(zip([t[0] for t in x.kernel_table()], x.profile_steps(1)))
        x.close()
        N = grid.point_num
        return {"workload": "hot Jupiter double-gray RT g%d/L%d dt=%g (%d columns), Guillot-profile "
                            "start (Teq %.0f K)" % (RT_GLEVEL, RT_NV, RT_DT, N, teq),
                "plain_fp64": {"ms_per_step": ms_plain,
                               "value": sim_days_per_hour(1, ms_plain / 1000.0, dt=RT_DT)},
                "mixed_surrogate": {"ms_per_step": ms_sur,
                                    "value": sim_days_per_hour(1, ms_sur / 1000.0, dt=RT_DT)},
                "ratio": ms_plain / ms_sur,
                "rt_ms_per_step": {"plain": kms_plain.get("radiative_transfer", 0.0),
                                   "surrogate_mode_rt": kms_sur.get("radiative_transfer", 0.0),
                                   "surrogate_mode_net": kms_sur.get("rt_surrogate", 0.0)},
                "training": {"columns_logged": nlog * N, "iterations": iters, "batch": batch,
                             "lr": "1e-3, last fifth 2e-4", "loss_first": first,
                             "loss_last": last, "seconds": train_s},
                "online_learning": online,
                "recheck": {"steps": nsteps + 3, "rechecked": st["rechecked"],
                            "failed": st["failed"], "max_rel_err": st["max_err"],
                            "rt_column_fraction": st["rt_columns"] / ((nsteps + 3) * N)}}
    except Exception as e:  # a side measurement never breaks the bench line
        if not catch:
            raise
        return {"unavailable": "%s" % e}


def zonal_mean_T(grid, T, nv, bands=36):
    """Area-weighted mean temperature over 5-degree latitude bands, [band][lev]."""
    N = grid.point_num
    lat = grid["lonlat"][1::2]
    w = grid["areasT"][:N]
    band = np.clip(((lat + np.pi / 2) / np.pi * bands).astype(int), 0, bands - 1)
    T = T.reshape(N, nv)
    out = np.zeros((bands, nv))
    for b in range(bands):
        m = band == b
        out[b] = (w[m][:, None] * T[m]).sum(0) / w[m].sum()
    return out


def config4_leg(torch, thor_b200, nsteps=2000, nlog=60, iters=5000, batch=8192, glevel=7,
                chunk=100, online_iters=300):
    """The large run: Held-Suarez at glevel 7 (163842 columns) x 48 levels, dt = 300 s, with the
    double-gray RT (Earth orbit and rotation; the RT configuration's gray opacities), all state in
    HBM, every step one CUDA graph replay. The all-FP64 form with the plain RT runs all nsteps as the
    judge; the mixed form logs the plain RT for the first nlog steps, trains the L48 surrogate
    (97 -> 512 x 3 -> 48) on the GPU, and runs the remaining steps with it, learning online
    (the columns the plain RT re-checks or falls back to are logged; online_iters Adam steps
    after every chunk of steps). Reports both forms' speed, the surrogate's re-check statistics,
    the mixed form's errors against the judge (fields, zonal-mean temperature) and the global mass
    drift of each."""
    nv, dt = 48, 300.0
    p = dict(EARTH, timestep=dt)
    rt = dict(Tstar=5772.0, radius_star=695700000.0, planet_star_dist=149597870700.0,
              diff_ang=0.5, Tint=0.0, albedo=0.3, kappa_sw=4e-4, kappa_lw=1e-3,
              kappa_lw_pole=1e-3, n_sw=1.0, n_lw=2.0, f_lw=0.5, sync_rot=0,
              mean_motion=1.991e-7, alpha_i=0.0)
    t0 = time.perf_counter()
    grid = thor_b200.Icogrid(glevel, nv, A=EARTH["A"], Top_altitude=EARTH["Top_altitude"])
    grid_s = time.perf_counter() - t0
    N = grid.point_num
    stream = torch.cuda.Stream()
    out = {"workload": "Held-Suarez + double-gray RT g%d/L%d dt=%g (%d columns), %d steps"
                       % (glevel, nv, dt, N, nsteps), "grid_seconds": grid_s}

    def timed(x, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        x.step(n)
        e1.record(stream)
        e1.synchronize()
        x.sync()
        return e0.elapsed_time(e1)

    # the judge: all FP64, plain RT
    x = thor_b200.Thorx(grid.as_dict(), glevel, dict(p, precision=thor_b200.FP64),
                        stream=stream.cuda_stream)
    x.init_rest_state(TMEAN, SEED, NOISE)
    x.rt_enable(rt)
    m0 = x.globdiag()[1]
    ms = timed(x, nsteps)
    judge = {f: x.get(f) for f in ("Rho", "pressure", "temperature", "Mh", "Wh")}
    out["fp64_plain_rt"] = {"ms_per_step": ms / nsteps,
                            "value": sim_days_per_hour(nsteps, ms / 1000.0, dt=dt),
                            "mass_drift": abs(x.globdiag()[1] - m0) / m0}
    x.close()
    # mixed form + surrogate
    x = thor_b200.Thorx(grid.as_dict(), glevel, dict(p, precision=thor_b200.MIXED),
                        stream=stream.cuda_stream)
    x.init_rest_state(TMEAN, SEED, NOISE)
    x.rt_enable(rt)
    x.sur_create(hidden=512, train_batch=batch, log_capacity=nlog * N, recheck_period=16,
                 tolerance=0.05, seed=SEED)
    m0 = x.globdiag()[1]
    x.sur_mode(thor_b200.SUR_LOG)
    ms_log = timed(x, nlog)
    t1 = time.perf_counter()
    first, last = x.sur_train(iters - iters // 5, batch, lr=1e-3)
    _, last = x.sur_train(iters // 5, batch, lr=2e-4)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t1
    # the remaining steps in chunks with online learning: the columns the plain RT ran on are
    # logged, and the network trains between chunks (graph replays timed, training apart)
    x.sur_mode(thor_b200.SUR_USE_LOG)
    x.sur_stats()
    nuse, ms_use, st = nsteps - nlog, 0.0, {"rechecked": 0, "failed": 0, "rt_columns": 0, "max_err": 0.0}
    online_s, left = 0.0, nsteps - nlog
    while left > 0:
        n = min(chunk, left)
        ms_use += timed(x, n)
        so = x.sur_stats()
        for k in ("rechecked", "failed", "rt_columns"):
            st[k] += so[k]
        st["max_err"] = max(st["max_err"], so["max_err"])
        left -= n
        if left > 0:
            t2 = time.perf_counter()
            x.sur_train(online_iters, batch, lr=2e-4)
            torch.cuda.synchronize()
            online_s += time.perf_counter() - t2
    mix = {f: x.get(f) for f in ("Rho", "pressure", "temperature", "Mh", "Wh")}
    out["mixed_surrogate"] = {
        "ms_per_step": ms_use / nuse, "value": sim_days_per_hour(nuse, ms_use / 1000.0, dt=dt),
        "mass_drift": abs(x.globdiag()[1] - m0) / m0,
        "logging_ms_per_step": ms_log / nlog,
        "online_learning": {"chunk_steps": chunk, "adam_steps_per_chunk": online_iters,
                            "seconds": online_s,
                            "amortised_ms_per_step": online_s * 1000.0 / nuse},
        "training": {"columns_logged": nlog * N, "iterations": iters, "batch": batch,
                     "loss_first": first, "loss_last": last, "seconds": train_s},
        "recheck": {"steps": nuse, "rechecked": st["rechecked"], "failed": st["failed"],
                    "max_rel_err": st["max_err"], "rt_column_fraction": st["rt_columns"] / (nuse * N)}}
    x.close()
    out["ratio"] = out["fp64_plain_rt"]["ms_per_step"] / out["mixed_surrogate"]["ms_per_step"]
    out["mixed_vs_fp64"] = {f: float(np.abs(mix[f] - judge[f]).max() / np.abs(judge[f]).max())
                            for f in judge}
    tz = np.abs(zonal_mean_T(grid, mix["temperature"], nv) - zonal_mean_T(grid, judge["temperature"], nv))
    out["zonal_mean_T_max_diff_K"] = float(tz.max())
    return out


def run_ours(args):
    import torch
    import thor_b200
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    grid = grid_for_bench()
    stream = torch.cuda.Stream(device)
    x = thor_b200.Thorx(grid.as_dict(), GLEVEL, params(args.form), stream=stream.cuda_stream)
    x.init_rest_state(TMEAN, SEED, NOISE)
    # warm-up (also captures the step graph)
    x.step(args.warmup)
    x.sync()
    barrier(world)
    torch.cuda.synchronize(device)
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    x.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    x.sync()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    barrier(world)
    ms = max_over_ranks(ms, world, device)
    ms_step = ms / args.steps
    value = world * sim_days_per_hour(args.steps, ms / 1000.0)

    # per-kernel roofline: eager steps with CUDA events around every launch, same stream
    table = x.kernel_table()
    nprof = 2
    kms = x.profile_steps(nprof)
    x.sync()
    total_kms = sum(kms)
    ki = max(range(len(table)), key=lambda i: kms[i])
    name, bytes_launch, launches = table[ki]
    avg_ms = kms[ki] / (launches * nprof)
    peak, peak_kind = peaks()
    achieved = bytes_launch / (avg_ms * 1e-3) / 1e9
    per_kernel = {t[0]: {"ms_per_step": kms[i] / nprof, "launches_per_step": t[2],
                         "GBps": (t[1] / (kms[i] / (t[2] * nprof) * 1e-3) / 1e9)
                         if kms[i] > 0 and t[2] > 0 else None,
                         "share": kms[i] / total_kms if total_kms else None}
                  for i, t in enumerate(table)}
    step_bytes = sum(t[1] * t[2] for t in table)

    # end to end through the C ABI with host buffers: the prognostic state goes in from pinned
    # host memory, one step runs, and the state comes back, every step
    host = {}
    for f in STATE:
        n = x.size(f)
        host[f] = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
        x.get(f, host[f])
    ke = max(3, min(args.steps, 10))
    torch.cuda.synchronize(device)
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(ke):
        for f in STATE:
            x.set(f, host[f])
        x.step(1)
        for f in STATE:
            x.get(f, host[f])
    e3.record(stream)
    e3.synchronize()
    x.sync()
    te = e2.elapsed_time(e3) / 1000.0
    te = max_over_ranks(te, world, device)
    io_bytes = sum(host[f].nbytes for f in STATE)
    e2e = {"value": world * sim_days_per_hour(ke, te), "unit": "sim-days/wall-hour",
           "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes, "steps": ke,
           "what": "thorx_set_field(state) + thorx_step(1) + thorx_get_field(state) per step, "
                   "pinned host buffers in the reference layout, CUDA events on the context "
                   "stream around all of it"}
    finite = all(np.isfinite(host[f]).all() for f in STATE)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        b = cpu_baseline(grid, CPU_SAMPLE_STEPS)
        cpu = {k: b[k] for k in ("value", "unit", "cores", "kind", "sample")}

    line = {"metric": METRIC, "value": value, "unit": "sim-days/wall-hour", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.form == "fp64" else "f32+f64",
            "data": "synthetic (seeded isothermal rest state, Held-Suarez forcing)",
            "config": bench_config(args.form, world),
            "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": ncu_traffic(name),
                         "algorithmic_bytes_per_launch": bytes_launch,
                         "avg_launch_ms": avg_ms},
            "step_effective_GBps": step_bytes / (ms_step * 1e-3) / 1e9,
            "kernels": per_kernel,
            "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
            "gpu_launches": x.kernels_per_step() * args.steps,
            "state_finite": bool(finite)}
    if world == 1 and not args.no_extras:
        # the mixed-precision form of the same context, same workload, after the measurements above
        ms_mixed = time_steps(x, stream, thor_b200.MIXED, max(5, min(args.steps, 50)))
        kms_mixed = x.profile_steps(nprof)
        x.sync()
        line["mixed_form"] = {"ms_per_step": ms_mixed,
                              "value": sim_days_per_hour(1, ms_mixed / 1000.0),
                              "ratio_vs_fp64": ms_step / ms_mixed,
                              "kernels_ms_per_step": {t[0]: kms_mixed[i] / nprof
                                                      for i, t in enumerate(table)
                                                      if kms_mixed[i] > 0},
                              "what": "THORX_MIXED: FP32 momentum-side stencils, hyperdiffusion "
                                      "and divergence damping through per-column operator weights, "
                                      "FP64 mass, pressure, vertical solve and sums; same state, "
                                      "same graph timing"}
        line["rt_surrogate"] = rt_surrogate_leg(torch, thor_b200)
    x.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--form", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-form and RT/surrogate side measurements")
    ap.add_argument("--glevel", type=int, default=GLEVEL,
                    help="grid level (default 6; smaller cases are for profiling captures)")
    ap.add_argument("--nv", type=int, default=NV, help="vertical levels (default 48)")
    ap.add_argument("--surrogate-only", action="store_true",
                    help="run only the RT surrogate leg (g5/L40) and print its JSON object; with "
                         "--sur-log-steps / --sur-iters it is the small case for profiling captures")
    ap.add_argument("--sur-log-steps", type=int, default=200,
                    help="plain-RT steps logged for training (surrogate leg)")
    ap.add_argument("--sur-iters", type=int, default=5000, help="Adam iterations (surrogate leg)")
    ap.add_argument("--config4", action="store_true",
                    help="run only the large g7/L48 Held-Suarez + surrogate-RT leg (2000 steps in "
                         "two forms, several minutes) and print its JSON object")
    args = ap.parse_args()
    set_workload(args.glevel, args.nv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.config4:
        import torch
        import thor_b200
        # glevel 7 unless --glevel names another (smaller cases for checks)
        print(json.dumps(config4_leg(torch, thor_b200, nsteps=args.steps,
                                     glevel=7 if args.glevel == 6 else args.glevel)), flush=True)
        return 0
    if args.surrogate_only:
        import torch
        import thor_b200
        leg = rt_surrogate_leg(torch, thor_b200, nlog=args.sur_log_steps, iters=args.sur_iters,
                               nsteps=args.steps, catch=False)
        print(json.dumps(leg), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
