"""Generates tests/golden/*.npz from the reference's OWN FP64 CUDA kernels.

Run on a machine with a GPU after `make -C oracle ref` (the reference sources compiled into
oracle/_ref/libthor_ref.so):

    python tests/golden/make_golden.py OUTDIR [rt]

Each fixture holds, for the seeded initial state of tests/thorx_testlib.initial_state on the
reference's own grid, the state after one large step (ProfX Held-Suarez + Thor) and the slow-mode
tendencies of the last RK stage, on every `stride`-th column (all levels), from the reference
built as it ships (FMA contraction on, keys FIELD) and with --fmad=false (keys nofma_FIELD).
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from thorx_testlib import (RT_WASP43B, RefGrid, RefSim, STATE_FIELDS,  # noqa: E402
                           hot_jupiter_params, initial_state, make_params)

CASES = [  # (name, glevel, nv, timestep, stride, overrides)
    ("hs_g4_l8_dt1200", 4, 8, 1200.0, 9, {}),
    ("hs_g4_l32_dt1200_shallow_hydro_energy", 4, 32, 1200.0, 20,
     dict(DeepModel=0, NonHydro=0, energy_equation=1)),
]
TEND = ["SlowMh", "SlowWh", "SlowRho", "Slowpressure"]


def column_slice(a, N, stride):
    per = a.size // N
    return a.reshape(N, per)[::stride].copy()


def main(outdir):
    os.makedirs(outdir, exist_ok=True)
    for name, glevel, nv, dt, stride, over in CASES:
        g = RefGrid(glevel, nv)
        p, c = make_params(glevel, dt, **over)
        ic = initial_state(g.arrays, g.point_num, g.nv, c)
        out = {"glevel": glevel, "nv": nv, "timestep": dt, "stride": stride,
               "overrides": repr(over), "seed": 20260101}
        for nofma in (False, True):
            s = RefSim(g, p, nofma=nofma)
            for k, v in ic.items():
                s.set(k, v)
            s.step(1)
            for f in STATE_FIELDS + ["temperature"] + TEND:
                out[("nofma_" if nofma else "") + f] = column_slice(s.get(f), g.point_num, stride)
            s.close()
        np.savez_compressed(os.path.join(outdir, name + ".npz"), **out)
        g.close()
        print("wrote", name)


# Double-gray RT case: the reference's ifile/wasp43b_ex.thr planet and RT keys at glevel 4, L20,
# seeded isothermal 1800 K state with +-1 K noise. One physics step (ProfX with insolation + RT,
# no Thor) gives the RT fields; then a full step (Thor included) gives the state.
RT_CASE = ("rt_wasp43b_g4_l20_dt300", 4, 20, 300.0, 7)
RT_FIELDS = ["cos_zenith", "insol", "ASR", "OLR", "fsw_dn", "flw_up", "flw_dn", "tau", "dtemp",
             "profx_Qheat"]


def main_rt(outdir):
    name, glevel, nv, dt, stride = RT_CASE
    p, c = hot_jupiter_params(glevel, dt)
    g = RefGrid(glevel, nv, A=c["A"], top=c["Top_altitude"])
    ic = initial_state(g.arrays, g.point_num, g.nv, c, amp=1.0)
    out = {"glevel": glevel, "nv": nv, "timestep": dt, "stride": stride, "seed": 20260101,
           "rt": repr(sorted(RT_WASP43B.items()))}
    for nofma in (False, True):
        pre = "nofma_" if nofma else ""
        s = RefSim(g, p, nofma=nofma)
        for k, v in ic.items():
            s.set(k, v)
        s.rt(RT_WASP43B)
        s.step(1, profx=True, thor=False)
        for f in RT_FIELDS:
            out[pre + f] = column_slice(s.get(f), g.point_num, stride)
        out[pre + "ASR_tot"], out[pre + "OLR_tot"] = s.rt_totals()
        s.step(1, profx=False, thor=True)
        for f in STATE_FIELDS + ["temperature"]:
            out[pre + "step_" + f] = column_slice(s.get(f), g.point_num, stride)
        s.close()
    np.savez_compressed(os.path.join(outdir, name + ".npz"), **out)
    g.close()
    print("wrote", name)


if __name__ == "__main__":
    outdir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    if len(sys.argv) > 2 and sys.argv[2] == "rt":
        main_rt(outdir)
    else:
        main(outdir)
        main_rt(outdir)
