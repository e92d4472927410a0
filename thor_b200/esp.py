"""bin/esp for thorx: run THOR's large step from a .thr configuration file.

    python -m thor_b200.esp [config.thr] [-g GPU] [-o DIR] [-N STEPS] [-i FILE | -c FILE | -b] [-w]

Restates the program entry of the reference (src/esp.cu:164-1573): the same command-line
arguments with the same meaning (src/esp.cu:183-198, overrides at :497-570), the same
configuration syntax (key = value lines, comments, typed values; src/utils/config_file.cpp:60-130,
src/headers/parser_helpers.h:77-365), the same keys and defaults for everything on the path
(src/esp.cu:257-475, src/headers/define.h; the RT module's keys,
src/physics/modules/src/radiative_transfer.cu:1107-1190; the insolation keys,
src/ESP/insolation.cu:239-251), the same checks (src/esp.cu:574-700), the main loop's cadence of
outputs, global diagnostics and log lines (src/esp.cu:1381-1480), batch and continue modes
(src/esp.cu:848-940) and the three text logs (src/utils/log_writer.cpp).

Differences, each stated where it applies:
  * output files are HDF5 with the reference's file names, dataset names, units and descriptions
    and memory layout ([column][level][component]) (src/ESP/esp_output.cu:136-487), written and read
    by thor_b200/h5.py (there is no HDF5 library here); the grid file lacks the curl operator (not
    built here) and the output files the RT's Qheat scaling; restart files may also be the .npz
    archives of earlier versions of this runner;
  * keys for physics that this build does not implement (the diffusive sponge, the RayPH
    convective adjustment, chemistry, boundary layer, ultra-hot thermodynamics, refined vertical grids,
    picket-fence or two-stream RT, the Parmentier and constant-N initial profiles) are accepted at
    their default values
    and rejected with an error naming the key otherwise;
  * output_mean, out_interm_momentum and output_diffusion only add arrays to the output files in
    the reference; here they are accepted and a warning says the arrays are not written;
  * one extension key, `precision` = fp64 (default) | mixed, selects the compute form.
The simulation itself runs on the GPU through the C ABI (include/thorx.h); nothing here computes.
"""
import argparse
import os
import re
import signal
import sys
import time

import numpy as np

AU = 149597870700.0       # src/headers/physical_constants.h:9
R_SUN = 695700000.0       # src/headers/physical_constants.h:15

# ---------------------------------------------------------------------------------------------
# Configuration syntax (src/headers/parser_helpers.h:77-130, 268-360)
# ---------------------------------------------------------------------------------------------
_PUNCT = re.escape("!\"#$%&'()*+,-./:;<=>?@[\\]^_`{|}~")
_EMPTY = re.compile(r"^[ \t]*$")
_COMMENT = re.compile(r"^[ \t]?#.*$")
_KEY_VALUE = re.compile(r"^[ \t]*([A-Za-z0-9_]+)[ \t]*=[ \t]*((?:[A-Za-z0-9]|[" + _PUNCT
                        + r"])+)[ \t]*(#.*)?$")
_BOOL = re.compile(r"^(true|false)$")
_INT = re.compile(r"^((-|\+)?[0-9]+)$")
_DOUBLE = re.compile(r"^((-|\+)?[0-9]+(\.[0-9]+)?((E|e)(-|\+)?[0-9]+)?)$")


def parse_value(kind, text):
    """(ok, value) for one configuration value of type kind (bool, int, float, str)."""
    if kind is bool:
        m = _BOOL.match(text)
        return (True, m.group(1) == "true") if m else (False, None)
    if kind is int:
        m = _INT.match(text)
        return (True, int(m.group(1))) if m else (False, None)
    if kind is float:
        m = _DOUBLE.match(text)
        return (True, float(m.group(1))) if m else (False, None)
    return True, text


# Keys: name -> (type, default, role). Roles: "path" (used), "output" (accepted, output only),
# "fixed" (must keep one of the allowed values: physics outside this build), "ignored" (no effect
# here, e.g. a parameter of a switched-off scheme). Defaults as the reference registers them: the
# planet's from SimulationSetup (src/ESP/simulation_setup.cu:60-76, a hot Jupiter), the switches
# from src/headers/define.h, and its own choice for MetStar, Tstar, radius_star and
# planet_star_dist, which take the defaults of Tint, kappa_lw, kappa_sw and f_lw
# (src/esp.cu:426-430).
KEYS = {
    "config_version": (int, -1, "ignored"),
    "timestep": (int, 1800, "path"),
    "num_steps": (int, 48000, "path"),
    "simulation_ID": (str, "Earth", "path"),
    "radius": (float, 72427000.0, "path"),
    "rotation_rate": (float, 9.09e-5, "path"),
    "gravitation": (float, 47.0, "path"),
    "GravHeightVar": (bool, False, "path"),
    "Rd": (float, 3714.0, "path"),
    "Cp": (float, 13000.0, "path"),
    "Tmean": (float, 1400.0, "path"),
    "P_ref": (float, 10000000.0, "path"),
    "Top_altitude": (float, 1235376.0, "path"),
    "Diffc": (float, 0.009973, "path"),
    "DivDampc": (float, 0.009973, "path"),
    "Diffc_v": (float, 0.0, "path"),
    "spring_dynamics": (bool, True, "path"),
    "glevel": (int, 4, "path"),
    "spring_beta": (float, 1.15, "path"),
    "vlevel": (int, 32, "path"),
    "HyDiff": (bool, True, "path"),
    "HyDiffOrder": (int, 4, "path"),
    "DivDampP": (bool, True, "path"),
    "VertHyDiff": (bool, False, "path"),
    "VertHyDiffOrder": (int, 6, "path"),
    "increased_damping_for_n_steps": (int, 0, "fixed"),
    "NonHydro": (bool, True, "path"),
    "DeepModel": (bool, True, "path"),
    "output_mean": (bool, True, "output"),
    "out_interm_momentum": (bool, False, "output"),
    "output_diffusion": (bool, False, "output"),
    "RayleighSponge": (bool, False, "path"),
    "RayleighSpongeT": (bool, False, "path"),
    "DiffSponge": (bool, False, "fixed"),
    "shrink_sponge": (bool, False, "path"),
    "t_shrink": (int, 144000, "path"),
    "raysp_calc_mode": (str, "imp", "path"),
    "nlat_bins": (int, 20, "path"),
    "Ruv_sponge": (float, 1e-4, "path"),
    "Rw_sponge": (float, 1e-4, "path"),
    "RT_sponge": (float, 1e-4, "path"),
    "ns_ray_sponge": (float, 0.75, "path"),
    "damp_uv_to_mean": (bool, True, "path"),
    "damp_w_to_mean": (bool, True, "path"),
    "Dv_sponge": (float, 0.01, "ignored"),
    "ns_diff_sponge": (float, 0.75, "ignored"),
    "order_diff_sponge": (int, 2, "ignored"),
    "rest": (bool, True, "path"),
    "initial": (str, "ifile/esp_initial.h5", "path"),
    "core_benchmark": (str, "HeldSuarez", "path"),
    "init_PT_profile": (str, "isothermal", "fixed"),
    "conv_adj": (bool, False, "path"),
    "conv_adj_iter": (int, 1, "path"),
    "soft_adjustment": (bool, False, "path"),
    "conv_adj_type": (str, "hourdin", "fixed"),
    "GPU_ID_N": (int, 0, "path"),
    "n_out": (int, 1000, "path"),
    "results_path": (str, "results", "path"),
    "gcm_off": (bool, False, "path"),
    "globdiag": (bool, False, "path"),
    "single_column": (bool, False, "fixed"),
    "custom_global_n_out": (bool, False, "path"),
    "global_n_out": (int, 1000, "path"),
    "custom_log_n_out": (bool, False, "path"),
    "log_n_out": (int, 1000, "path"),
    "Tint": (float, 100.0, "path"),
    "kappa_lw": (float, 0.002, "path"),
    "kappa_sw": (float, 0.001, "path"),
    "f_lw": (float, 0.5, "path"),
    "bv_freq": (float, 0.01, "ignored"),
    "MetStar": (float, 100.0, "ignored"),
    "Tstar": (float, 0.002, "path"),
    "radius_star": (float, 0.001, "path"),
    "planet_star_dist": (float, 0.5, "path"),
    "ultrahot_thermo": (str, "none", "fixed"),
    "ultrahot_heating": (str, "none", "fixed"),
    "thermo_equation": (str, "entropy", "path"),
    "vert_refined": (bool, False, "fixed"),
    "transition_altitude": (float, 1000.0, "ignored"),
    "lowest_layer_thickness": (float, 2.0, "ignored"),
    "vert_dense_around": (bool, False, "fixed"),
    "frac_height_dense": (float, 0.7, "ignored"),
    "a_dense": (float, 1.0, "ignored"),
    "b_dense": (float, 6.0, "ignored"),
    # physics modules (src/physics/managers/multi/src/phy_modules.cu:118-140)
    "radiative_transfer": (bool, False, "path"),
    "chemistry": (bool, False, "fixed"),
    "chem_time_file": (str, "", "ignored"),
    "chem_fEQ_file": (str, "", "ignored"),
    "boundary_layer": (bool, False, "fixed"),
    "bl_type": (str, "RayleighHS", "ignored"),
    "two_streams_radiative_transfer": (bool, False, "fixed"),
    # double-gray RT (radiative_transfer.cu:1146-1190, radiative_transfer.h:98-119)
    "rt_type": (str, "DualbandGray", "fixed"),
    "diff_ang": (float, 0.5, "path"),
    "albedo": (float, 0.18, "path"),
    "latf_lw": (bool, False, "path"),
    "kappa_lw_pole": (float, 0.002, "path"),
    "n_sw": (float, 1.0, "path"),
    "n_lw": (float, 2.0, "path"),
    "rt1Dmode": (bool, False, "path"),
    "surface": (bool, False, "fixed"),
    "Csurf": (float, 1e7, "ignored"),
    "dgrt_spinup_start": (int, -1, "path"),
    "dgrt_spinup_stop": (int, -1, "path"),
    "dgrt_spindown_start": (int, -1, "path"),
    "dgrt_spindown_stop": (int, -1, "path"),
    # insolation (src/ESP/insolation.cu:239-251, src/headers/insolation.h:132-138)
    "sync_rot": (bool, True, "path"),
    "mean_motion": (float, 1.991e-7, "path"),
    "alpha_i": (float, 0.0, "path"),
    "true_long_i": (float, 0.0, "path"),
    "ecc": (float, 0.0, "path"),
    "obliquity": (float, 0.0, "path"),
    "longp": (float, 0.0, "path"),
    "insol_avg": (str, "NoInsolAvg", "fixed"),
    # extension: compute form of this build
    "precision": (str, "fp64", "path"),
}
# values a "fixed" key may take (its default unless listed)
ALLOWED = {"init_PT_profile": ("isothermal", "guillot"), "rt_type": ("DualbandGray",),
           "conv_adj_type": ("hourdin", "Hourdin"),
           "ultrahot_thermo": ("none",), "ultrahot_heating": ("none",),
           "insol_avg": ("NoInsolAvg",)}
CHOICES = {"core_benchmark": ("HeldSuarez", "NoBenchmark", "TidallyLockedEarth",
                              "ShallowHotJupiter"),
           "thermo_equation": ("entropy", "energy"), "precision": ("fp64", "mixed")}


class ConfigError(Exception):
    pass


def read_config(text, out=sys.stdout):
    """Parse a .thr text into {key: value} with defaults, as the reference's config_file does:
    unknown keys warn and are skipped, a malformed line or value fails the whole file."""
    values = {k: v[1] for k, v in KEYS.items()}
    given = set()
    ok = True
    for n, line in enumerate(text.splitlines(), 1):
        if _EMPTY.match(line) or _COMMENT.match(line):
            continue
        m = _KEY_VALUE.match(line)
        if not m:
            out.write("ERROR in config file at line %d :\t [%s]\n" % (n, line))
            ok = False
            continue
        key, value = m.group(1), m.group(2)
        if key not in KEYS:
            out.write("WARNING: config file key [%s] does not exist, skipping\n" % key)
            continue
        good, v = parse_value(KEYS[key][0], value)
        if not good:
            out.write("ERROR: parsing of value [%s] failed for key [%s] \n" % (value, key))
            ok = False
            continue
        values[key] = v
        given.add(key)
    if not ok:
        raise ConfigError("config file reading failed")
    return values, given


def check_config(c, out=sys.stdout):
    """The reference's range checks (src/esp.cu:574-700) plus this build's scope; raises
    ConfigError listing every problem."""
    bad = []
    def need(cond, msg):
        if not cond:
            bad.append(msg)
    need(c["timestep"] > 0, "timestep must be > 0")
    need(c["num_steps"] > 0, "nsmax must be > 0")
    need(c["gravitation"] > 0, "gravitation must be > 0")
    need(c["Rd"] > 0, "Rd must be > 0")
    need(c["Tmean"] > 0, "T_mean must be > 0")
    need(c["P_ref"] > 0, "P_Ref must be > 0")
    need(c["Top_altitude"] > 0, "Top_altitude must be > 0")
    need(3 <= c["glevel"] <= 8, "glevel must be in [3, 8]")
    need(4 <= c["glevel"] <= 7, "glevel = %d: this build's grid takes 4 to 7" % c["glevel"])
    need(c["vlevel"] > 0, "vlevel must be > 0")
    need(c["GPU_ID_N"] > -1, "GPU_ID_N must be > -1")
    need(c["n_out"] > 0, "n_out must be > 0")
    need(len(c["simulation_ID"]) < 160, "Bad value for config variable simulation_ID")
    need(c["HyDiffOrder"] > 2 and c["HyDiffOrder"] % 2 == 0,
         "Bad value for HyDiffOrder! Must be multiple of 2 greater than/equal to 4.")
    need(c["VertHyDiffOrder"] > 2 and c["VertHyDiffOrder"] % 2 == 0,
         "Bad value for VertHyDiffOrder! Must be multiple of 2 greater than/equal to 4.")
    for k, allowed in CHOICES.items():
        need(c[k] in allowed, "%s = %s: this build supports %s" % (k, c[k], " | ".join(allowed)))
    if c["RayleighSponge"]:  # src/esp.cu:757-780: the mode is read only with the sponge on
        need(c["raysp_calc_mode"] in ("imp", "exp1", "exp3"),
             "raysp_calc_mode config item not recognised: [%s]" % c["raysp_calc_mode"])
        need(c["nlat_bins"] >= 1, "nlat_bins must be >= 1")
        need(0.0 <= c["ns_ray_sponge"] < 1.0, "ns_ray_sponge must be in [0, 1)")
    for k, (kind, default, role) in KEYS.items():
        if role == "fixed":
            allowed = ALLOWED.get(k, (default,))
            need(c[k] in allowed, "%s = %s: not implemented in this build (allowed: %s)"
                 % (k, c[k], ", ".join(str(a) for a in allowed)))
    if bad:
        for b in bad:
            out.write("Config error: %s\n" % b)
        raise ConfigError("; ".join(bad))
    for k in ("output_mean", "out_interm_momentum", "output_diffusion"):
        if c[k]:
            out.write("WARNING: %s = true: those arrays are not written by this build\n" % k)


def sponge_config(c, first_step):
    """The Rayleigh-sponge keys as thorx_sponge_params (the Thorx.sponge dict)."""
    return dict(nlat_bins=c["nlat_bins"], Ruv_sponge=c["Ruv_sponge"], Rw_sponge=c["Rw_sponge"],
                RT_sponge=c["RT_sponge"], ns_ray_sponge=c["ns_ray_sponge"],
                damp_uv_to_mean=int(c["damp_uv_to_mean"]), damp_w_to_mean=int(c["damp_w_to_mean"]),
                RayleighSpongeT=int(c["RayleighSpongeT"]), shrink_sponge=int(c["shrink_sponge"]),
                t_shrink=c["t_shrink"], first_step=first_step,
                raysp_calc_mode={"imp": 0, "exp1": 1, "exp3": 2}[c["raysp_calc_mode"]])


def thorx_params(c):
    """The configuration as thorx_params (the Thorx constructor's dict)."""
    return dict(A=c["radius"], Omega=c["rotation_rate"], Gravit=c["gravitation"], Rd=c["Rd"],
                Cp=c["Cp"], P_Ref=c["P_ref"], Top_altitude=c["Top_altitude"],
                timestep=float(c["timestep"]), Diffc=c["Diffc"], DivDampc=c["DivDampc"],
                HyDiffOrder=c["HyDiffOrder"], DeepModel=int(c["DeepModel"]),
                NonHydro=int(c["NonHydro"]), GravHeightVar=int(c["GravHeightVar"]),
                HyDiff=int(c["HyDiff"]), DivDampP=int(c["DivDampP"]),
                thermo_equation=1 if c["thermo_equation"] == "energy" else 0,
                core_benchmark={"NoBenchmark": 0, "HeldSuarez": 1, "TidallyLockedEarth": 2,
                                "ShallowHotJupiter": 3}[c["core_benchmark"]],
                precision=1 if c["precision"] == "mixed" else 0)


def rt_config(c, first_step):
    """The RT module's parameters in the C ABI's units (m, K, degrees): the configuration gives
    the star radius in solar radii and the distance in au (src/ESP/esp_initial.cu:194-196)."""
    return dict(Tstar=c["Tstar"], planet_star_dist=c["planet_star_dist"] * AU,
                radius_star=c["radius_star"] * R_SUN, diff_ang=c["diff_ang"], Tint=c["Tint"],
                albedo=c["albedo"], kappa_sw=c["kappa_sw"], kappa_lw=c["kappa_lw"],
                kappa_lw_pole=c["kappa_lw_pole"], n_sw=c["n_sw"], n_lw=c["n_lw"], f_lw=c["f_lw"],
                latf_lw=int(c["latf_lw"]), rt1Dmode=int(c["rt1Dmode"]),
                sync_rot=int(c["sync_rot"]), surface=0, mean_motion=c["mean_motion"],
                alpha_i=c["alpha_i"], true_long_i=c["true_long_i"], ecc=c["ecc"],
                obliquity=c["obliquity"], longp=c["longp"],
                spinup_start=c["dgrt_spinup_start"], spinup_stop=c["dgrt_spinup_stop"],
                spindown_start=c["dgrt_spindown_start"], spindown_stop=c["dgrt_spindown_stop"],
                first_step=first_step)


# ---------------------------------------------------------------------------------------------
# Files: HDF5 outputs (src/ESP/esp_output.cu) and the text logs (src/utils/log_writer.cpp)
# ---------------------------------------------------------------------------------------------
# what a restart reads (src/ESP/esp_initial.cu:1215-1260): the prognostic fields and the per-cell
# gas constants; dataset names of the output files
STATE = ["Rho", "pressure", "Mh", "Wh", "Rd", "Cp"]
ARCHIVE_NAMES = {"Rho": "Rho", "pressure": "Pressure", "Mh": "Mh", "Wh": "Wh", "W": "W",
                 "Rd": "Rd", "Cp": "Cp"}


def output_name(sim_id, idx):
    return "esp_output_%s_%d.h5" % (sim_id, idx)


def _atomic_h5(path):
    from thor_b200 import h5
    return h5.H5Writer(path + ".tmp")


def write_state(path, x, nstep, sim_time, c, glob=None, rt=None, cells=None):
    """ESP::output's state file (src/ESP/esp_output.cu:306-470) and the RT module's and the
    insolation's store() (radiative_transfer.cu:1286-1336, insolation.cu:484-493)."""
    w = _atomic_h5(path)
    w.value("/nstep", int(nstep), "-", "Step number")
    w.value("/simulation_time", float(sim_time), "s", "Simulation time")
    w.table("/Rho", x.get("Rho"), "kg/m^3", "Density")
    w.table("/Pressure", x.get("pressure"), "Pa", "Pressure")
    w.table("/Mh", x.get("Mh"), "kg m^-2 s^-1", "Horizontal Momentum")
    w.table("/Wh", x.get("Wh"), "kg m^-2 s^-1", "Vertical Momentum")
    if cells is not None:  # the per-cell terms of the global sums (esp_output.cu:410-428)
        w.table("/Etotal", cells[0], "kg m^2/s^2", "Total Energy")
        w.table("/Entropy", cells[5], "kg m^2/s^2 K^-1", "Entropy")
        w.table("/Mass", cells[1], "kg", "Mass")
        w.table("/AngMomx", cells[2], "kg m^2/s", "AngMom in X")
        w.table("/AngMomy", cells[3], "kg m^2/s", "AngMom in Y")
        w.table("/AngMomz", cells[4], "kg m^2/s", "AngMom in Z")
    if glob is not None:
        E, M, AMx, AMy, AMz, Ent = glob
        w.value("/GlobalE", E, "kg m^2/s^2", "Global Total Energy")
        w.value("/GlobalEnt", Ent, "kg m^2/s^2 K^-1", "Global Entropy")
        w.value("/GlobalMass", M, "kg", "Global Mass")
        w.value("/GlobalAMx", AMx, "kg m^2/s", "Global AngMomX")
        w.value("/GlobalAMy", AMy, "kg m^2/s", "Global AngMomY")
        w.value("/GlobalAMz", AMz, "kg m^2/s", "Global AngMomZ")
    w.table("/Qheat", x.get("profx_Qheat"), "W m^-3", "Physics module Qheat")
    w.table("/Rd", x.get("Rd"), "J/K/kg", "Local gas constant")
    w.table("/Cp", x.get("Cp"), "J/K/kg", "Local heat capacity")
    if rt is not None:
        asr, olr = rt
        w.table("/insol", x.get("insol"), "W m^-2", "insolation (instantaneous)")
        w.table("/insol_annual", x.get("insol_ann"), "W m^-2",
                "insolation (annual/orbit averaged)")
        w.table("/flw_up", x.get("flw_up"), "W m^-2", "upward flux (LW)")
        w.table("/fsw_up", x.get("fsw_up"), "W m^-2", "upward flux (SW)")
        w.table("/flw_dn", x.get("flw_dn"), "W m^-2", "downward flux (LW)")
        w.table("/fsw_dn", x.get("fsw_dn"), "W m^-2", "downward flux (SW)")
        w.table("/tau", x.get("tau"), " ", "optical depth across each layer (not total optical depth)")
        w.table("/DGQheat", x.get("DG_Qheat"), " ", "Double Gray Qheat")
        w.value("/ASR", asr, "W", "Absorbed Shortwave Radiation (global total)")
        w.value("/OLR", olr, "W", "Outgoing Longwave Radiation (global total)")
        w.table("/cos_zenith_angles", x.get("cos_zenith"), "-", "cos_zenith_angles per column")
    w.close()
    os.replace(path + ".tmp", path)


def write_grid(path, grid):
    """ESP::output's grid file (src/ESP/esp_output.cu:144-183), without the curl operator."""
    d = grid.as_dict()
    w = _atomic_h5(path)
    w.table("/Altitude", d["Altitude"], "m", "Altitude")
    w.table("/Altitudeh", d["Altitudeh"], "m", "Altitude at the interfaces")
    w.table("/areasT", d["areasT"], "m^2", "Main cells areas")
    w.table("/lonlat", d["lonlat"], "-", "Longitudes and latitudes")
    w.value("/point_num", float(d["point_num"]), "-", "Number of grid points in one level")
    w.value("/nv", float(d["nv"]), "-", "Number of vertical layers")
    w.table("/pntloc", d["point_local"].astype(np.int32), "-", "Neighbours indexes")
    w.table("/grad", d["grad"], "m^-1", "Horizontal gradient operator")
    w.table("/div", d["div"], "m^-1", "Horizontal divergence operator")
    w.close()
    os.replace(path + ".tmp", path)


def write_planet(path, c):
    """ESP::output's planet file (src/ESP/esp_output.cu:186-304) with the module manager's, the
    RT module's and the insolation's store_init (phy_modules.cu:219-237,
    radiative_transfer.cu:1366-1388, insolation.cu:459-479)."""
    b = lambda k: 1.0 if c[k] else 0.0
    w = _atomic_h5(path)
    w.value("/glevel", int(c["glevel"]), "-", "Horizontal subdivision level")
    w.value("/vlevel", int(c["vlevel"]), "-", "Vertical subdivision level")
    w.value("/spring_dynamics", b("spring_dynamics"), "-", "Spring dynamics")
    w.value("/spring_beta", float(c["spring_beta"]), "-", "Spring Beta")
    w.value("/A", float(c["radius"]), "m", "Planet radius")
    w.value("/Rd", float(c["Rd"]), "J/(Kg K)", "Gas constant")
    w.value("/Omega", float(c["rotation_rate"]), "1/s", "Rotation rate")
    w.value("/Gravit", float(c["gravitation"]), "m/s^2", "Surface gravity")
    w.value("/P_Ref", float(c["P_ref"]), "Pa", "Reference pressure")
    w.value("/Top_altitude", float(c["Top_altitude"]), "m", "Top of the model's domain")
    w.value("/Cp", float(c["Cp"]), "J/(Kg K)", "Specific heat capacity")
    w.value("/RayleighSponge", b("RayleighSponge"), "-", "Using Rayleigh SpongeLayer?")
    w.value("/RayleighSpongeT", b("RayleighSpongeT"), "-", "Using thermal SpongeLayer?")
    w.value("/DiffSponge", b("DiffSponge"), "-", "Using Diffusive SpongeLayer?")
    w.value("/DeepModel", b("DeepModel"), "-", "Using Deep Model")
    w.value("/NonHydro", b("NonHydro"), "-", "Using Non Hydrostatic parameter")
    w.value("/output_mean", b("output_mean"), "-", "outputting mean quantities")
    w.value("/output_diffusion", b("output_diffusion"), "-", "outputting diffusion terms")
    w.value("/out_interm_momentum", b("out_interm_momentum"), "-",
            "outputting intermediate momentum values")
    w.value("/DivDampP", b("DivDampP"), "-", "Using Divergence-damping")
    w.value("/HyDiff", b("HyDiff"), "-", "Using Hyper diffusion")
    w.value("/Diffc", float(c["Diffc"]), "-", "Hyperdiffusion strength")
    w.value("/Diffc_v", float(c["Diffc_v"]), "-", "Vertical hyperdiffusion strength")
    w.value("/Tmean", float(c["Tmean"]), "K", "Mean atmospheric temperature")
    w.value("/conv_adj", b("conv_adj"), "-", "Using convection adjustment")
    w.value("/gcm_off", b("gcm_off"), "-", "GCM off")
    w.value("/single_column", b("single_column"), "-", "single column mode")
    w.value("/rest", b("rest"), "-", "Starting from rest")
    w.value("/core_benchmark", int(thorx_params(c)["core_benchmark"]), "-",
            "Using benchmark forcing")
    if c["RayleighSponge"]:
        w.value("/nlat_bins", int(c["nlat_bins"]), "-",
                "number of lat rings for Rayleigh sponge layer")
        w.value("/ns_ray_sponge", float(c["ns_ray_sponge"]), "-", "Bottom of rayleigh sponge layer")
        w.value("/Ruv_sponge", float(c["Ruv_sponge"]), "1/s",
                "Strength of Rayleigh sponge layer (uv components)")
        w.value("/Rw_sponge", float(c["Rw_sponge"]), "1/s",
                "Strength of Rayleigh sponge layer (w component)")
    w.value("/Tint", float(c["Tint"]), "K", "Temperature of interior heat flux")
    w.value("/f_lw", float(c["f_lw"]), "-", "fraction of taulw in well-mixed absorber")
    w.value("/kappa_lw", float(c["kappa_lw"]), "-", "longwave opacity")
    w.value("/kappa_sw", float(c["kappa_sw"]), "-", "shortwave opacity")
    w.value("/phy_module", 0.0, "-", "multi")
    w.value("/surface", 0.0, "-", "include solid/liquid surface")
    w.value("/Csurf", float(c["Csurf"]), "J/K/m^2", "heat capacity of surface by area")
    # the module manager (multi) and its modules
    w.value("/radiative_transfer", b("radiative_transfer"), "-", "Using radiative transfer")
    w.value("/Tstar", float(c["Tstar"]), "K", "Temperature of host star")
    w.value("/planet_star_dist", float(c["planet_star_dist"]), "au",
            "distance b/w host star and planet")
    w.value("/radius_star", float(c["radius_star"]), "R_sun", "radius of host star")
    w.value("/diff_ang", float(c["diff_ang"]), "-", "diffusivity factor")
    w.value("/albedo", float(c["albedo"]), "-", "bond albedo of planet")
    w.value("/latf_lw", b("latf_lw"), "-", "use lat dependent opacity")
    w.value("/kappa_lw_pole", float(c["kappa_lw_pole"]), "-", "gray opacity of longwave at poles")
    w.value("/n_lw", float(c["n_lw"]), "-", "power law exponent for unmixed absorber in LW")
    w.value("/n_sw", float(c["n_sw"]), "-", "power law exponent for mixed/unmixed absorber in SW")
    w.value("/rt_type", 0, "-", "Type of radiative transfer physics")
    w.value("/chemistry", 0.0, "-", "Using relaxation chemistry")
    w.value("/boundary_layer", 0.0, "-", "Using boundary layer")
    if c["radiative_transfer"]:
        w.value("/sync_rot", b("sync_rot"), "-", "enforce synchronous rotation")
        w.value("/mean_motion", float(c["mean_motion"]), "rad/s", "orbital mean motion")
        w.value("/alpha_i", float(c["alpha_i"]), "deg", "initial RA of host star")
        w.value("/true_long_i", float(c["true_long_i"]), "deg",
                "initial orbital position of planet")
        w.value("/ecc", float(c["ecc"]), "-", "orbital eccentricity")
        w.value("/obliquity", float(c["obliquity"]), "deg", "tilt of spin axis")
        w.value("/longp", float(c["longp"]), "deg", "longitude of periastron")
    w.close()
    os.replace(path + ".tmp", path)


def output_numbering(path):
    """(basename, number) of a file named esp_output_<basename>_<number>.h5, else None
    (match_output_file_numbering_scheme, src/utils/directories.cpp:270-311)."""
    if not path.endswith(".h5"):
        return None
    parts = os.path.basename(path)[:-3].split("_")
    if len(parts) < 4 or parts[0] != "esp" or parts[1] != "output":
        return None
    try:
        number = int(parts[-1])
    except ValueError:
        return None
    return ("_".join(parts[2:-1]), number) if number > -1 else None


def planet_file(initial, continuing):
    """The planet file that goes with an initial-conditions file (find_continue_file,
    src/utils/directories.cpp:313-362): esp_output_planet_<basename>.h5 beside an output-named
    file, <stem>_planet.h5 beside any other. None when continuing from a file without the output
    naming."""
    d = os.path.dirname(initial) or "."
    m = output_numbering(initial)
    if m is not None:
        return os.path.join(d, "esp_output_planet_%s.h5" % m[0])
    if continuing:
        return None
    stem = os.path.splitext(os.path.basename(initial))[0]
    return os.path.join(d, stem + "_planet.h5")


def check_planet(path, c, out):
    """The restart check of src/ESP/esp_initial.cu:1147-1205: A, Top_altitude, glevel, vlevel and
    surface of the planet file must equal the configuration's. Returns True when they do."""
    from thor_b200 import h5
    try:
        d = h5.read(path)
    except (OSError, h5.H5FormatError) as e:
        out.write("planet_file %s not readable: %s\n" % (path, e))
        return False
    ok = True
    for key, want in (("A", float(c["radius"])), ("Top_altitude", float(c["Top_altitude"])),
                      ("glevel", int(c["glevel"])), ("vlevel", int(c["vlevel"])),
                      ("surface", 0.0)):
        if key not in d:
            out.write("Error reading key /%s from reload config.\n" % key)
            ok = False
            continue
        have = d[key][0].reshape(-1)[0]
        if have != want:
            out.write("mismatch for /%s value between config value: %s and initial condition "
                      "value %s.\n" % (key, want, have))
            ok = False
    if not ok:
        out.write("Could not reload full configuration.\n")
    return ok


def read_state(path):
    """(fields present in the file, nstep, simulation time) of an output file (HDF5) or of an
    .npz archive of earlier versions of this runner."""
    if path.endswith(".npz"):
        with np.load(path) as d:
            state = {f: np.array(d[ARCHIVE_NAMES[f]]) for f in STATE if ARCHIVE_NAMES[f] in d}
            return state, int(d["nstep"]), float(d["simulation_time"])
    from thor_b200 import h5
    d = h5.read(path)
    state = {f: d[ARCHIVE_NAMES[f]][0] for f in STATE if ARCHIVE_NAMES[f] in d}
    return state, int(d["nstep"][0][0]), float(d["simulation_time"][0][0])


class Logs:
    """esp_write_log_<ID>.txt, esp_global_<ID>.txt, esp_diagnostics_<ID>.txt in the output
    directory, with the reference's headers and columns."""

    def __init__(self, out_dir, sim_id, append, globdiag):
        self.out_dir, self.sim_id = out_dir, sim_id
        mode = "a" if append else "w"
        self.write_log = self._open("esp_write_log_%s.txt" % sim_id, mode,
                                    "#step_number\tfile_number\tfilename")
        self.glob = self._open("esp_global_%s.txt" % sim_id, mode,
                               "#current_step\tsimulation_time\tGlobalE_h\tGlobalMass_h\t"
                               "GlobalAMx_h\tGlobalAMy_h\tGlobalAMz_h\tGlobalEnt_h") \
            if globdiag else None
        self.diag = self._open("esp_diagnostics_%s.txt" % sim_id, mode,
                               "#current_step\tsimulation_time\ttotal_bytes\tfree_bytes\t"
                               "elapsed_time\ttime_left\tmean_delta_per_step\tend_time")

    def _open(self, name, mode, header):
        path = os.path.join(self.out_dir, name)
        fresh = mode == "w" or not os.path.exists(path)
        f = open(path, mode)
        if fresh:
            f.write(header + "\n")
        return f

    def output(self, step, idx, filename):
        self.write_log.write("%d\t%d\t%s\n" % (step, idx, filename))
        self.write_log.flush()

    def globdiag(self, step, t, g):
        self.glob.write("%d\t%s\t%s\n" % (step, _g16(t), "\t".join(_g16(v) for v in g)))
        self.glob.flush()

    def diagnostics(self, step, t, total, free, elapsed, left, mean_delta, end):
        self.diag.write("%d\t%s\t%d\t%d\t%s\t%s\t%s\t%s\n"
                        % (step, _g16(t), total, free, _g16(elapsed), _g16(left),
                           _g16(mean_delta), end))
        self.diag.flush()

    def close(self):
        for f in (self.write_log, self.glob, self.diag):
            if f:
                f.close()


def _g16(v):
    return "%.16g" % v


def last_output(out_dir, sim_id):
    """(file number, step, filename) of the last line of esp_write_log_<ID>.txt, or None
    (log_writer::check_output_log, src/utils/log_writer.cpp:80-136)."""
    path = os.path.join(out_dir, "esp_write_log_%s.txt" % sim_id)
    if not os.path.exists(path):
        return None
    last = None
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 3 and not line.startswith("#"):
                last = (int(parts[1]), int(parts[0]), parts[2])
    return last


# ---------------------------------------------------------------------------------------------
# The run
# ---------------------------------------------------------------------------------------------
_caught = []


def _on_signal(signum, frame):  # the reference's sigterm/sigint handlers (src/esp.cu:99-110)
    _caught.append(signum)


def build_parser():
    ap = argparse.ArgumentParser(prog="esp", description="run THOR GCM simulation (thorx)")
    ap.add_argument("config", nargs="?", default="ifile/earth.thr", help="config filename")
    ap.add_argument("-g", "--gpu_id", type=int, help="GPU_ID to run on")
    ap.add_argument("-o", "--output_dir", help="results directory to store output")
    ap.add_argument("-i", "--initial", help="start from this initial condition instead of rest")
    ap.add_argument("-c", "--continue", dest="cont",
                    help="continue simulation from this output file")
    ap.add_argument("-N", "--numsteps", type=int, help="number of steps to run")
    ap.add_argument("-w", "--overwrite", action="store_true",
                    help="Force overwrite of output file if they exist")
    ap.add_argument("-b", "--batch", action="store_true", help="Run as batch")
    return ap


def run(argv=None, out=sys.stdout):
    """Run a simulation; returns the process exit status (0 ok)."""
    args = build_parser().parse_args(argv)
    try:
        with open(args.config) as f:
            text = f.read()
    except OSError:
        out.write(" Config file %s reading failed, aborting\n" % args.config)
        return 255
    try:
        c, given = read_config(text, out)
    except ConfigError:
        out.write(" Config file %s reading failed, aborting\n" % args.config)
        return 255
    out.write(" Config file %s read\n" % args.config)
    # command-line overrides (src/esp.cu:497-570)
    if args.gpu_id is not None:
        c["GPU_ID_N"] = args.gpu_id
    if args.output_dir is not None:
        c["results_path"] = args.output_dir
    if args.numsteps is not None:
        c["num_steps"] = args.numsteps
    start_file = None
    if args.initial is not None:
        c["rest"] = False
        start_file = args.initial
    if args.cont is not None:
        if args.batch:
            out.write("--continue and --batch options set, options are exclusive, must set only one\n")
            return 255
        if args.initial is not None:
            out.write("--continue and --initial options set, options are exclusive, must set only one\n")
            return 255
        c["rest"] = False
        start_file = args.cont
    if not c["rest"] and start_file is None:
        start_file = c["initial"]
    try:
        check_config(c, out)
    except ConfigError:
        return 255
    if start_file is not None and not os.path.exists(start_file):
        out.write("Initial conditions file \"%s\" not found\n" % start_file)
        return 255

    out_dir, sim_id = c["results_path"], c["simulation_ID"]
    os.makedirs(out_dir, exist_ok=True)
    continuing = args.cont is not None
    first_idx, step_idx, sim_time0 = 0, 1, 0.0
    if args.batch:
        last = last_output(out_dir, sim_id)
        if last is not None:
            start_file = os.path.join(out_dir, last[2])
            continuing = True
            out.write("continuing batch run from file %s\n" % start_file)
        else:
            out.write("No batch file found, initialise simulation.\n")
    if not continuing and not args.overwrite and os.path.exists(
            os.path.join(out_dir, output_name(sim_id, 0))):
        out.write("output files already exist in %s; use -w to overwrite\n" % out_dir)
        return 255
    if start_file is not None and start_file.endswith(".h5"):
        pf = planet_file(start_file, continuing)
        if pf is None:
            out.write("Loading initial conditions: Could not recognise file numbering scheme for "
                      "input %s\n" % start_file)
            return 255
        if not os.path.exists(pf):
            out.write("planet_file %s not found.\n" % pf)
            return 255
        if not check_planet(pf, c, out):
            return 255

    import thor_b200
    # the device: GPU_ID_N (or -g) through CUDA_VISIBLE_DEVICES, before the first CUDA call
    if "CUDA_VISIBLE_DEVICES" in os.environ:
        if c["GPU_ID_N"] != 0:
            out.write("WARNING: CUDA_VISIBLE_DEVICES is set; GPU_ID_N = %d ignored\n"
                      % c["GPU_ID_N"])
    else:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(c["GPU_ID_N"])
    grid = thor_b200.Icogrid(c["glevel"], c["vlevel"], A=c["radius"],
                             Top_altitude=c["Top_altitude"], spring=c["spring_dynamics"],
                             beta=c["spring_beta"])
    x = thor_b200.Thorx(grid.as_dict(), c["glevel"], thorx_params(c))
    handlers = None
    try:
        if start_file is not None:
            state, nstep0, sim_time0 = read_state(start_file)
            missing = [f for f in ("Rho", "pressure", "Mh", "Wh") if f not in state]
            if missing:
                out.write("start file %s lacks %s\n" % (start_file, ", ".join(missing)))
                return 255
            cells = x.size("Rho")
            state.setdefault("Rd", np.full(cells, c["Rd"]))   # files without the gas constants
            state.setdefault("Cp", np.full(cells, c["Cp"]))
            for f, v in state.items():
                x.set(f, v)
            if continuing:
                step_idx = nstep0 + 1
                m = re.search(r"_(\d+)\.(h5|npz)$", start_file)
                first_idx = int(m.group(1)) + 1 if m else 1
        elif c["init_PT_profile"] == "guillot":
            x.init_guillot_state(c["Tmean"], c["Tint"], c["f_lw"], c["kappa_sw"], c["kappa_lw"], 0,
                                 0.0)
        else:
            x.init_rest_state(c["Tmean"], 0, 0.0)
        if c["radiative_transfer"]:
            x.rt_enable(rt_config(c, step_idx))
        if c["conv_adj"]:
            x.conv_adj(c["conv_adj_iter"], c["soft_adjustment"])
        if c["RayleighSponge"]:
            x.sponge(sponge_config(c, step_idx))
        if c["VertHyDiff"]:
            x.vert_hydiff(c["Diffc_v"], c["VertHyDiffOrder"])
        nsmax = c["num_steps"]
        logs = Logs(out_dir, sim_id, continuing, c["globdiag"])
        write_grid(os.path.join(out_dir, "esp_output_grid_%s.h5" % sim_id), grid)
        write_planet(os.path.join(out_dir, "esp_output_planet_%s.h5" % sim_id), c)
        rt_tot = (lambda: x.rt_totals()) if c["radiative_transfer"] else (lambda: None)
        if not continuing:
            name = output_name(sim_id, 0)
            g0, cells0 = x.globdiag_fields() if c["globdiag"] else (None, None)
            write_state(os.path.join(out_dir, name), x, 0, sim_time0, c, g0, rt_tot(), cells0)
            logs.output(0, 0, name)
            first_idx = 1
        del _caught[:]
        handlers = (signal.signal(signal.SIGTERM, _on_signal),
                    signal.signal(signal.SIGINT, _on_signal))
        dt = c["timestep"]
        n_out = c["n_out"]
        g_out = c["global_n_out"] if c["custom_global_n_out"] else n_out
        l_out = c["log_n_out"] if c["custom_log_n_out"] else n_out
        idx, nstep, t0 = first_idx, step_idx - 1, time.time()
        out.write(" Starting the model integration.\n\n")
        while nstep < nsmax:
            # next step at which something is written: run up to it as one call (graph replays)
            nxt = min(nsmax, *(((nstep // k) + 1) * k for k in (n_out, g_out, l_out)),
                      nstep + 64)
            k = nxt - nstep
            if c["gcm_off"]:
                for _ in range(k):
                    x.profx()
            else:
                x.step(k)
            x.sync()
            nstep = nxt
            sim_time = sim_time0 + (nstep - step_idx + 1) * dt
            writing = nstep % n_out == 0 or bool(_caught)
            glob, cells = None, None
            if c["globdiag"]:
                glob, cells = x.globdiag_fields() if writing else (x.globdiag(), None)
            if c["globdiag"] and nstep % g_out == 0:
                logs.globdiag(nstep, sim_time, glob)
            if writing:
                name = output_name(sim_id, idx)
                write_state(os.path.join(out_dir, name), x, nstep, sim_time, c, glob, rt_tot(),
                            cells)
                logs.output(nstep, idx, name)
                idx += 1
            elapsed = time.time() - t0
            done = nstep - step_idx + 1
            mean = elapsed / done
            left = mean * (nsmax - nstep)
            end = time.strftime("%Y-%m-%d %H:%M:%S", time.localtime(time.time() + left))
            if nstep % l_out == 0:
                out.write("\n Time step number = %d/%d || Time = %f days. \n\t Elapsed %.0f s || "
                          "Left: %.0f s || Completion: %s. \n"
                          % (nstep, nsmax, sim_time / 86400.0, elapsed, left, end))
                logs.diagnostics(nstep, sim_time, 0, 0, elapsed, left, mean, end)
            if _caught:
                out.write("\n Caught signal, stopping after step %d.\n" % nstep)
                break
        logs.close()
    finally:
        if handlers:
            signal.signal(signal.SIGTERM, handlers[0])
            signal.signal(signal.SIGINT, handlers[1])
        x.close()
    return 0


def main():
    sys.exit(run())


if __name__ == "__main__":
    main()
