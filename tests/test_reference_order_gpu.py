"""The all-FP64 form applies the hyperdiffusion and divergence-damping operators through FP64
per-column operator weights: the reference's linear operators summed in another order. This test
keeps the build with the reference's own operation order in those operators
(thor_b200/libthorx_reforder.so, THORX_FP64_DIFF_WEIGHTS=0, THORX_FP64_DIVM_WEIGHTS=0) at the same
per-field tolerances against the reference's kernels, and keeps the two orders of the product
within the reference's own FMA/no-FMA spread of each other.

The variant library runs in a child process (THORX_LIB selects it), so the two builds of the same
ABI never share a process.
"""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
VARIANT = os.path.join(ROOT, "thor_b200", "libthorx_reforder.so")
CASES = [(4, 16, 1200.0, {}), (5, 16, 600.0, dict(DivDampP=0)),
         (4, 12, 1200.0, dict(HyDiffOrder=2, held_suarez=0)),
         (4, 16, 1200.0, dict(DeepModel=0, NonHydro=0, energy_equation=1))]


def child():
    sys.path[:0] = [ROOT, HERE]
    from test_dycore_parity_gpu import run_case
    out = [run_case(*c) for c in CASES]
    print("RESULT " + json.dumps(out))


@pytest.mark.gpu
def test_reference_operation_order_build_matches_reference():
    from thorx_testlib import field_tolerance
    assert os.path.exists(VARIANT), "build thor_b200 first (python -m thor_b200.build)"
    env = dict(os.environ, THORX_LIB=VARIANT,
               PYTHONPATH=os.pathsep.join([ROOT, HERE, os.environ.get("PYTHONPATH", "")]))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--child"], env=env,
                       capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    line = [l for l in r.stdout.splitlines() if l.startswith("RESULT ")][-1]
    results = json.loads(line[len("RESULT "):])
    bad = []
    for case, res in zip(CASES, results):
        for f, (err, spread) in res.items():
            tol = 1e-12 if f in ("Rho", "pressure", "temperature") else field_tolerance(spread)
            if not err <= tol:
                bad.append((case, f, err, tol))
    assert not bad, bad


if __name__ == "__main__" and "--child" in sys.argv:
    child()
