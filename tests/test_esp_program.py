"""thor_b200/bin/esp, the C++ program that runs a simulation from a .thr file over libthorx's C ABI,
against the Python runner (thor_b200/esp.py), which restates the reference's program entry
(src/esp.cu:164-1573), configuration rules (src/utils/config_file.cpp:60-130,
src/headers/parser_helpers.h:77-365) and output layout (src/ESP/esp_output.cu:136-487).

Without a GPU: the two read every configuration of the CLI tests to the same values and print the
same messages and exit codes for every rejected configuration and argument set; the program's HDF5
reader reads the reference-written files as thor_b200/h5.py does, and its writer lays out a file
byte for byte as h5.py does (apart from the modification times). On the GPU: a Held-Suarez run
and a hot-Jupiter run (double-gray RT from the Guillot profile, Rayleigh sponge, convective
adjustment, mixed form) give output files whose every dataset equals the Python runner's bit for
bit and the same logs; the Held-Suarez run also a bitwise continuation, batch mode and the
planet-file check.
"""
import io
import os
import struct
import subprocess

import numpy as np
import pytest

from thor_b200 import build, esp, h5
from test_esp_cli import HS_THR

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "h5")


@pytest.fixture(scope="module")
def program():
    build.build(verbose=False)
    assert os.path.exists(build.ESP_BIN)
    return build.ESP_BIN


def run_program(program, args, cwd):
    r = subprocess.run([program] + [str(a) for a in args], cwd=str(cwd), capture_output=True,
                       text=True, timeout=600)
    return r.returncode, r.stdout, r.stderr


def run_python(args):
    out = io.StringIO()
    rc = esp.run([str(a) for a in args], out)
    return rc, out.getvalue()


def py_str(v):
    return str(v)


VARIANTS = {
    "hs": HS_THR,
    "defaults": "",
    "rt": HS_THR + "radiative_transfer = true\nTstar = 4300\nplanet_star_dist = 0.015\n"
                   "radius_star = 0.667\nthermo_equation = energy\nprecision = mixed\n"
                   "core_benchmark = NoBenchmark\ninit_PT_profile = guillot\necc = 0.2\n",
    "sponge": HS_THR.replace("RayleighSponge = false", "RayleighSponge = true")
              + "nlat_bins = 12\nns_ray_sponge = 0.6\ndamp_w_to_mean = false\n"
                "raysp_calc_mode = exp3\nshrink_sponge = true\nt_shrink = 7\n",
    "crlf": HS_THR.replace("\n", "\r\n") + "Diffc_v = 1e-5\nVertHyDiff = true\n",
}


@pytest.mark.parametrize("name", list(VARIANTS))
def test_configuration_reads_as_the_python_runner(program, tmp_path, name):
    cfg = tmp_path / "x.thr"
    cfg.write_text(VARIANTS[name], newline="")
    rc, out, err = run_program(program, [cfg, "--dump-config"], tmp_path)
    assert rc == 0, out + err
    c, _ = esp.read_config(VARIANTS[name], io.StringIO())
    want = ["%s = %s" % (k, py_str(c[k])) for k in esp.KEYS]
    got = [l for l in out.splitlines() if " = " in l and not l.startswith(("#", " ", "WARNING"))]
    assert got == want
    p, rt = esp.thorx_params(c), esp.rt_config(c, 1)
    assert ("# thorx_params: thermo_equation %d core_benchmark %d precision %d"
            % (p["thermo_equation"], p["core_benchmark"], p["precision"])) in out
    assert ("# thorx_rt_params: planet_star_dist %r radius_star %r"
            % (rt["planet_star_dist"], rt["radius_star"])) in out


BAD_LINES = ["glevel = 4.5", "globdiag = yes", "radius = .5",
             "  # two blanks before the hash are neither a comment nor a key", "glevel 4",
             "DiffSponge = true", "RayleighSponge = true\nraysp_calc_mode = implicit",
             "RayleighSponge = true\nns_ray_sponge = 1.0", "conv_adj_type = rayph",
             "chemistry = true", "init_PT_profile = parmentier", "rt_type = PicketFence",
             "core_benchmark = JetSteady", "HyDiffOrder = 5", "glevel = 9", "glevel = 3",
             "n_out = 0", "precision = fp16", "timestep = -5\nRd = 0",
             "increased_damping_for_n_steps = 3", "vert_refined = true", "Tstar = 1e400x"]


@pytest.mark.parametrize("line", BAD_LINES)
def test_rejected_configurations_print_what_the_python_runner_prints(program, tmp_path, line):
    cfg = tmp_path / "bad.thr"
    cfg.write_text(HS_THR + line + "\n")
    rc, out, _ = run_program(program, [cfg, "-o", tmp_path / "o"], tmp_path)
    prc, pout = run_python([cfg, "-o", tmp_path / "o"])
    assert (rc, out) == (prc, pout) and rc == 255


def test_arguments_and_missing_files_as_the_python_runner(program, tmp_path):
    cfg = tmp_path / "hs.thr"
    cfg.write_text(HS_THR)
    cases = [[cfg, "-c", "x.h5", "-b"], [cfg, "-c", "x.h5", "-i", "y.h5"],
             [tmp_path / "missing.thr"], [cfg, "-i", tmp_path / "nothere.h5", "-o", tmp_path],
             [cfg, "--continue", tmp_path / "nothere.h5", "--output_dir", tmp_path]]
    for args in cases:
        rc, out, _ = run_program(program, args, tmp_path)
        assert (rc, out) == run_python(args), args
    # restart files whose planet file is missing or named outside the scheme
    (tmp_path / "esp_output_T_3.h5").write_bytes(b"")
    (tmp_path / "other.h5").write_bytes(b"")
    for args in ([cfg, "-i", tmp_path / "esp_output_T_3.h5", "-o", tmp_path / "r"],
                 [cfg, "-c", tmp_path / "other.h5", "-o", tmp_path / "r"],
                 [cfg, "-i", tmp_path / "other.h5", "-o", tmp_path / "r"]):
        rc, out, _ = run_program(program, args, tmp_path)
        assert (rc, out) == run_python(args), args
    rc, _, err = run_program(program, [cfg, "--bogus"], tmp_path)
    assert rc == 2 and "unrecognized arguments" in err
    rc, _, err = run_program(program, [cfg, "-N", "abc"], tmp_path)
    assert rc == 2 and "invalid int value" in err


def reference_files():
    return sorted(f for f in os.listdir(GOLDEN) if f.endswith(".h5"))


@pytest.mark.parametrize("name", reference_files())
def test_reader_reads_reference_files_as_h5py(program, tmp_path, name):
    path = os.path.join(GOLDEN, name)
    rc, out, err = run_program(program, ["--h5-dump", path], tmp_path)
    assert rc == 0, out + err
    want = []
    for k, (a, attrs) in sorted(h5.read(path).items()):
        v = [float(x) for x in np.asarray(a).reshape(-1)]
        want.append("\t".join([k, "int" if a.dtype.kind in "iu" else "float", str(len(v)),
                               attrs.get("units", ""), attrs.get("Variable", ""),
                               "%.16g" % v[0] if v else "", "%.16g" % sum(v)]))
    assert out.splitlines() == want


MTIME_HEAD = struct.pack("<HHB3x", 0x12, 8, 0) + bytes([1, 0, 0, 0])


def same_but_mtime(a, b):
    """True if the files differ only in the 4 time bytes of modification-time messages."""
    if len(a) != len(b):
        return False
    ok = set()
    p = a.find(MTIME_HEAD)
    while p >= 0:
        ok.update(range(p + len(MTIME_HEAD), p + len(MTIME_HEAD) + 4))
        p = a.find(MTIME_HEAD, p + 1)
    return all(i in ok for i in range(len(a)) if a[i] != b[i])


@pytest.mark.parametrize("name", reference_files())
def test_writer_lays_out_files_as_h5py(program, tmp_path, name):
    path = os.path.join(GOLDEN, name)
    rc, out, err = run_program(program, ["--h5-copy", path, tmp_path / "cxx.h5"], tmp_path)
    assert rc == 0, out + err
    w = h5.H5Writer(str(tmp_path / "py.h5"))
    for k, (a, attrs) in h5.read(path).items():
        w.table(k, a, attrs.get("units", ""), attrs.get("Variable", ""))
    w.close()
    a, b = (tmp_path / "cxx.h5").read_bytes(), (tmp_path / "py.h5").read_bytes()
    assert same_but_mtime(a, b)
    back = h5.read(str(tmp_path / "cxx.h5"))
    for k, (arr, attrs) in h5.read(path).items():
        assert np.array_equal(back[k][0].reshape(-1), np.asarray(arr).reshape(-1)), k
        assert back[k][1] == attrs


def datasets(path):
    return {k: (a.dtype.str, a.tobytes(), attrs) for k, (a, attrs) in h5.read(path).items()}


# a hot Jupiter with the double-gray RT from the Guillot profile, an implicit Rayleigh sponge,
# dry convective adjustment and the mixed form: the RT's and the sponge's keys and output fields
RT_THR = """\
num_steps = 3
timestep = 300
n_out = 3
globdiag = true
simulation_ID = HotJ
radius = 94400000.0
rotation_rate = 2.06e-5
gravitation = 9.42
Rd = 3714.0
Cp = 13000.0
Tmean = 1400.0
P_ref = 10000000.0
Top_altitude = 4000000.0
glevel = 4
vlevel = 20
core_benchmark = NoBenchmark
init_PT_profile = guillot
radiative_transfer = true
Tstar = 4300.0
planet_star_dist = 0.015
radius_star = 0.667
Tint = 100.0
kappa_sw = 0.00125
kappa_lw = 0.0025
kappa_lw_pole = 0.0025
RayleighSponge = true
ns_ray_sponge = 0.7
conv_adj = true
precision = mixed
"""


@pytest.mark.gpu
def test_rt_sponge_mixed_run_matches_the_python_runner(program, tmp_path):
    cfg = tmp_path / "hj.thr"
    cfg.write_text(RT_THR)
    a, b = tmp_path / "cxx", tmp_path / "py"
    rc, out, err = run_program(program, [cfg, "-o", a], tmp_path)
    assert rc == 0, out + err
    prc, pout = run_python([cfg, "-o", b])
    assert prc == 0, pout
    assert sorted(os.listdir(a)) == sorted(os.listdir(b))
    final = h5.read(str(a / "esp_output_HotJ_1.h5"))
    for k in ("insol", "flw_up", "DGQheat", "ASR", "OLR", "cos_zenith_angles", "GlobalMass"):
        assert k in final, k
    assert np.all(np.isfinite(final["Rho"][0]))
    for n in sorted(os.listdir(a)):
        if n.endswith(".h5"):
            assert datasets(str(a / n)) == datasets(str(b / n)), n
    for n in ("esp_write_log_HotJ.txt", "esp_global_HotJ.txt"):
        assert (a / n).read_text() == (b / n).read_text(), n


@pytest.mark.gpu
def test_run_matches_the_python_runner(program, tmp_path):
    cfg = tmp_path / "hs.thr"
    cfg.write_text(HS_THR)
    a, b = tmp_path / "cxx", tmp_path / "py"
    rc, out, err = run_program(program, [cfg, "-o", a], tmp_path)
    assert rc == 0, out + err
    assert "Starting the model integration" in out and "Time step number = 4/4" in out
    prc, pout = run_python([cfg, "-o", b])
    assert prc == 0, pout
    assert sorted(os.listdir(a)) == sorted(os.listdir(b))
    for n in sorted(os.listdir(a)):
        if n.endswith(".h5"):
            assert datasets(str(a / n)) == datasets(str(b / n)), n
            assert same_but_mtime((a / n).read_bytes(), (b / n).read_bytes()), n
    for n in ("esp_write_log_TestHS.txt", "esp_global_TestHS.txt"):
        assert (a / n).read_text() == (b / n).read_text(), n
    diag = [l.split("\t") for l in (a / "esp_diagnostics_TestHS.txt").read_text().splitlines()]
    assert diag[0][0] == "#current_step" and [int(r[0]) for r in diag[1:]] == [2, 4]
    # continue from the intermediate output: the same final state bit for bit
    c = tmp_path / "cont"
    assert run_program(program, [cfg, "-o", c, "-N", "2"], tmp_path)[0] == 0
    rc, out, err = run_program(program, [cfg, "-o", c, "-c", c / "esp_output_TestHS_1.h5"],
                               tmp_path)
    assert rc == 0, out + err
    final, cont = h5.read(str(a / "esp_output_TestHS_2.h5")), h5.read(str(c / "esp_output_TestHS_2.h5"))
    for f in ("Rho", "Pressure", "Mh", "Wh"):
        assert np.array_equal(cont[f][0], final[f][0]), f
    assert (c / "esp_write_log_TestHS.txt").read_text() == (a / "esp_write_log_TestHS.txt").read_text()
    # batch mode finds the last output and has nothing left to do
    rc, out, _ = run_program(program, [cfg, "-o", c, "-b"], tmp_path)
    assert rc == 0 and "continuing batch run from file" in out
    # existing outputs are not overwritten without -w
    rc, out, _ = run_program(program, [cfg, "-o", a], tmp_path)
    assert rc == 255 and "use -w to overwrite" in out
    # a planet file that does not match the configuration stops a restart, as in the Python runner
    cfg5 = tmp_path / "hs5.thr"
    cfg5.write_text(HS_THR.replace("glevel = 4", "glevel = 5"))
    args = [cfg5, "-o", tmp_path / "d", "-i", c / "esp_output_TestHS_1.h5"]
    rc, out, _ = run_program(program, args, tmp_path)
    assert (rc, out) == run_python(args) and "mismatch for /glevel" in out
