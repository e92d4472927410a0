"""The .thr configuration and bin/esp command line (thor_b200/esp.py) against the reference's rules.

Parse rules restated from src/headers/parser_helpers.h:77-365 and src/utils/config_file.cpp:60-130;
checks from src/esp.cu:574-700; argument handling from src/esp.cu:183-198, 497-570. The GPU test
runs a short Held-Suarez simulation through the runner, checks its files and logs, and that a run
continued from an intermediate output ends bitwise where the uninterrupted run ends.
"""
import io
import os

import numpy as np
import pytest

from thor_b200 import esp

HS_THR = """\
config_version = 1
num_steps = 4
timestep = 1200
n_out = 2
# a comment line
 # one blank before the hash is still a comment
globdiag = true
simulation_ID = TestHS
radius = 6371000.0
rotation_rate = 7.292E-5
gravitation = 9.8
Rd = 287.0
Cp = 1005.0
Tmean = 300.0
P_ref = 100000.0
Top_altitude = 36000.0
glevel = 4
vlevel = 8
spring_dynamics = true
spring_beta = 1.15
NonHydro = true
DeepModel = true
rest = true
core_benchmark = HeldSuarez
thermo_equation = entropy
HyDiff  =    true
DivDampP =    true
Diffc = 0.0048      # trailing comment
DivDampc = 0.0048
RayleighSponge = false
radiative_transfer = false
output_mean = false
some_future_key = 3
"""


def test_value_syntax_follows_the_reference():
    ok = lambda k, t: esp.parse_value(k, t)[0]
    assert ok(bool, "true") and ok(bool, "false") and not ok(bool, "True") and not ok(bool, "1")
    assert ok(int, "-12") and ok(int, "+3") and not ok(int, "1.0") and not ok(int, "1e3")
    for good in ("1", "-2.5", "1e-4", "7.292E-5", "+6.0e+2"):
        assert ok(float, good), good
    for bad in (".5", "1.", "e5", "1e", "0x10", "nan"):
        assert not ok(float, bad), bad
    assert esp.parse_value(float, "7.292E-5")[1] == 7.292e-5
    assert esp.parse_value(str, "ifile/x.h5") == (True, "ifile/x.h5")


def test_config_file_reading():
    out = io.StringIO()
    c, given = esp.read_config(HS_THR, out)
    assert c["glevel"] == 4 and c["vlevel"] == 8 and c["Diffc"] == 0.0048
    assert c["simulation_ID"] == "TestHS" and c["globdiag"] is True
    assert c["HyDiffOrder"] == 4 and c["GravHeightVar"] is False  # defaults
    assert "some_future_key" not in c
    assert "WARNING: config file key [some_future_key] does not exist, skipping" in out.getvalue()
    assert "Diffc" in given and "HyDiffOrder" not in given
    esp.check_config(c, io.StringIO())


@pytest.mark.parametrize("line", [
    "glevel = 4.5",                 # int expected
    "globdiag = yes",               # bool expected
    "radius = .5",                  # the reference's double syntax needs a leading digit
    "  # two blanks before the hash are neither a comment nor a key",
    "glevel 4",                     # no '='
])
def test_bad_lines_fail_the_file(line):
    out = io.StringIO()
    with pytest.raises(esp.ConfigError):
        esp.read_config(HS_THR + line + "\n", out)
    assert "ERROR" in out.getvalue()


@pytest.mark.parametrize("line,what", [
    ("DiffSponge = true", "DiffSponge"),
    ("RayleighSponge = true\nraysp_calc_mode = implicit", "raysp_calc_mode"),
    ("RayleighSponge = true\nns_ray_sponge = 1.0", "ns_ray_sponge"),
    ("conv_adj_type = rayph", "conv_adj_type"),
    ("chemistry = true", "chemistry"),
    ("init_PT_profile = parmentier", "init_PT_profile"),
    ("rt_type = PicketFence", "rt_type"),
    ("core_benchmark = JetSteady", "core_benchmark"),
    ("HyDiffOrder = 5", "HyDiffOrder"),
    ("glevel = 9", "glevel"),
    ("glevel = 3", "glevel"),
    ("n_out = 0", "n_out"),
    ("precision = fp16", "precision"),
])
def test_unsupported_or_invalid_settings_are_rejected(line, what):
    c, _ = esp.read_config(HS_THR + line + "\n", io.StringIO())
    out = io.StringIO()
    with pytest.raises(esp.ConfigError):
        esp.check_config(c, out)
    assert what in out.getvalue()


def test_sponge_keys():
    c, _ = esp.read_config(HS_THR.replace("RayleighSponge = false", "RayleighSponge = true")
                           + "nlat_bins = 12\nns_ray_sponge = 0.6\ndamp_w_to_mean = false\n",
                           io.StringIO())
    esp.check_config(c, io.StringIO())
    d = esp.sponge_config(c, 9)
    assert d["nlat_bins"] == 12 and d["ns_ray_sponge"] == 0.6 and d["first_step"] == 9
    assert d["damp_w_to_mean"] == 0 and d["damp_uv_to_mean"] == 1 and d["Ruv_sponge"] == 1e-4
    # the mode is not checked while the sponge is off (src/esp.cu:757-780)
    c, _ = esp.read_config(HS_THR + "raysp_calc_mode = exp1\n", io.StringIO())
    esp.check_config(c, io.StringIO())


def test_defaults_and_unit_conversions():
    c, _ = esp.read_config("", io.StringIO())
    # the reference's own defaults, including its Tstar/radius_star/planet_star_dist choice
    assert (c["radius"], c["Tmean"], c["timestep"], c["Diffc"]) == (72427000.0, 1400.0, 1800, 0.009973)
    assert (c["Tstar"], c["radius_star"], c["planet_star_dist"]) == (0.002, 0.001, 0.5)
    c2, _ = esp.read_config("Tstar = 4300\nplanet_star_dist = 0.015\nradius_star = 0.667\n"
                            "thermo_equation = energy\ncore_benchmark = NoBenchmark\n"
                            "precision = mixed\n", io.StringIO())
    rt = esp.rt_config(c2, 7)
    assert rt["planet_star_dist"] == 0.015 * 149597870700.0
    assert rt["radius_star"] == 0.667 * 695700000.0 and rt["first_step"] == 7
    p = esp.thorx_params(c2)
    assert p["thermo_equation"] == 1 and p["core_benchmark"] == 0 and p["precision"] == 1


def test_exclusive_arguments(tmp_path):
    cfg = tmp_path / "hs.thr"
    cfg.write_text(HS_THR)
    out = io.StringIO()
    assert esp.run([str(cfg), "-c", "x.npz", "-b"], out) == 255
    assert "options are exclusive" in out.getvalue()
    out = io.StringIO()
    assert esp.run([str(cfg), "-c", "x.npz", "-i", "y.npz"], out) == 255
    out = io.StringIO()
    assert esp.run([str(tmp_path / "missing.thr")], out) == 255
    assert "reading failed" in out.getvalue()
    out = io.StringIO()
    assert esp.run([str(cfg), "-i", str(tmp_path / "nothere.npz"), "-o", str(tmp_path)], out) == 255
    assert "not found" in out.getvalue()


def test_batch_log_lookup(tmp_path):
    (tmp_path / "esp_write_log_X.txt").write_text(
        "#step_number\tfile_number\tfilename\n0\t0\tesp_output_X_0.h5\n20\t1\tesp_output_X_1.h5\n")
    assert esp.last_output(str(tmp_path), "X") == (1, 20, "esp_output_X_1.h5")
    assert esp.last_output(str(tmp_path), "Y") is None


@pytest.mark.gpu
def test_run_outputs_logs_and_bitwise_continuation(tmp_path):
    from thor_b200 import h5
    cfg = tmp_path / "hs.thr"
    cfg.write_text(HS_THR)
    a, b = tmp_path / "a", tmp_path / "b"
    out = io.StringIO()
    assert esp.run([str(cfg), "-o", str(a)], out) == 0, out.getvalue()
    names = sorted(os.listdir(a))
    for n in ("esp_output_TestHS_0.h5", "esp_output_TestHS_1.h5", "esp_output_TestHS_2.h5",
              "esp_write_log_TestHS.txt", "esp_global_TestHS.txt", "esp_diagnostics_TestHS.txt",
              "esp_output_grid_TestHS.h5", "esp_output_planet_TestHS.h5"):
        assert n in names, names
    log = (a / "esp_write_log_TestHS.txt").read_text().splitlines()
    assert log[0] == "#step_number\tfile_number\tfilename"
    assert log[1:] == ["0\t0\tesp_output_TestHS_0.h5", "2\t1\tesp_output_TestHS_1.h5",
                       "4\t2\tesp_output_TestHS_2.h5"]
    glob = [l.split("\t") for l in (a / "esp_global_TestHS.txt").read_text().splitlines()[1:]]
    assert [int(r[0]) for r in glob] == [2, 4] and float(glob[1][1]) == 4 * 1200.0
    m0, m1 = float(glob[0][3]), float(glob[1][3])
    assert abs(m1 - m0) <= 1e-12 * m0  # global mass, compensated sums
    final = h5.read(str(a / "esp_output_TestHS_2.h5"))
    assert int(final["nstep"][0][0]) == 4 and np.all(np.isfinite(final["Rho"][0]))
    assert final["Mh"][0].size == 3 * final["Rho"][0].size
    assert final["Rho"][1] == {"Variable": "Density", "units": "kg/m^3"}
    assert float(final["GlobalMass"][0][0]) == m1  # the file's global sums are the log's
    assert final["Mass"][1] == {"Variable": "Mass", "units": "kg"}
    assert abs(final["Mass"][0].sum() - m1) <= 1e-12 * m1  # the per-cell terms of that sum
    planet = h5.read(str(a / "esp_output_planet_TestHS.h5"))
    assert int(planet["glevel"][0][0]) == 4 and float(planet["A"][0][0]) == 6371000.0
    # run 2 steps, then continue from that output for the remaining 2
    out = io.StringIO()
    assert esp.run([str(cfg), "-o", str(b), "-N", "2"], out) == 0, out.getvalue()
    out = io.StringIO()
    assert esp.run([str(cfg), "-o", str(b), "-c", str(b / "esp_output_TestHS_1.h5")], out) == 0
    cont = h5.read(str(b / "esp_output_TestHS_2.h5"))
    for f in ("Rho", "Pressure", "Mh", "Wh"):
        assert np.array_equal(cont[f][0], final[f][0]), f
    # batch mode finds the last output and has nothing left to do
    out = io.StringIO()
    assert esp.run([str(cfg), "-o", str(b), "-b"], out) == 0
    assert "continuing batch run from file" in out.getvalue()
    # a planet file that does not match the configuration stops a restart
    bad = HS_THR.replace("glevel = 4", "glevel = 5")
    cfg2 = tmp_path / "hs5.thr"
    cfg2.write_text(bad)
    out = io.StringIO()
    assert esp.run([str(cfg2), "-o", str(tmp_path / "c"), "-i",
                    str(b / "esp_output_TestHS_1.h5")], out) == 255
    assert "mismatch for /glevel" in out.getvalue()
