"""Test helpers: ctypes access to the checkers and the seeded initial state.

The checkers are test infrastructure, never the product:
  * oracle/_build/liboracle.so  - the CPU restatement of the reference step (oracle/thor_oracle.cpp)
  * oracle/_ref/libthor_ref.so  - the reference's own grid builder and FP64 CUDA kernels,
                                  compiled from its sources by oracle/Makefile
"""
import ctypes
import math
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libthor_ref.so")
# the same reference sources built with FMA contraction off
REF_NOFMA_SO = os.path.join(ROOT, "oracle", "_ref", "libthor_ref_nofma.so")

# ------------------------------------------------------------------------------------------------
# Configurations (Earth Held-Suarez; the reference's ifile/earth_hstest.thr constants)
# ------------------------------------------------------------------------------------------------
EARTH = dict(A=6.371e6, Omega=7.292e-5, Gravit=9.8, Rd=287.0, Cp=1005.0, P_Ref=1e5,
             Top_altitude=36e3, Tmean=300.0, Diffc=0.0048, DivDampc=0.0048, HyDiffOrder=4,
             DeepModel=1, NonHydro=1, GravHeightVar=0, HyDiff=1, DivDampP=1,
             energy_equation=0, held_suarez=1)

PARAM_FIELDS = [("A", ctypes.c_double), ("Omega", ctypes.c_double), ("Gravit", ctypes.c_double),
                ("Rd", ctypes.c_double), ("Cp", ctypes.c_double), ("P_Ref", ctypes.c_double),
                ("timestep", ctypes.c_double), ("Diffc", ctypes.c_double),
                ("DivDampc", ctypes.c_double), ("HyDiffOrder", ctypes.c_int),
                ("DeepModel", ctypes.c_int), ("NonHydro", ctypes.c_int),
                ("GravHeightVar", ctypes.c_int), ("HyDiff", ctypes.c_int),
                ("DivDampP", ctypes.c_int), ("energy_equation", ctypes.c_int),
                ("held_suarez", ctypes.c_int), ("glevel", ctypes.c_int)]


class Params(ctypes.Structure):
    _fields_ = PARAM_FIELDS


def make_params(glevel, timestep, **over):
    c = dict(EARTH)
    c.update(over)
    p = Params()
    for name, _ in PARAM_FIELDS:
        if name == "timestep":
            p.timestep = timestep
        elif name == "glevel":
            p.glevel = glevel
        else:
            setattr(p, name, c[name])
    return p, c


# Hot Jupiter with double-gray RT: the reference's ifile/wasp43b_ex.thr constants (no sponge, no
# convective adjustment), and its RT/insolation keys with lengths in m.
AU, R_SUN = 149597870700.0, 695700000.0
HOT_JUPITER = dict(A=72427000.0, Omega=9.09e-5, Gravit=47.0, Rd=3714.0, Cp=13000.0, P_Ref=1e7,
                   Top_altitude=1.4e6, Tmean=1800.0, Diffc=0.015, DivDampc=0.015, HyDiffOrder=4,
                   DeepModel=1, NonHydro=1, GravHeightVar=0, HyDiff=1, DivDampP=1,
                   energy_equation=0, held_suarez=0)
RT_WASP43B = dict(Tstar=4300.0, planet_star_dist=0.015 * AU, radius_star=0.667 * R_SUN,
                  diff_ang=0.5, Tint=100.0, albedo=0.18, kappa_sw=0.00125, kappa_lw=0.0025,
                  kappa_lw_pole=0.0025, n_sw=1.0, n_lw=2.0, f_lw=0.5, sync_rot=1)


def hot_jupiter_params(glevel, timestep, **over):
    c = dict(HOT_JUPITER)
    c.update(over)
    return make_params(glevel, timestep, **c)


RT_F64 = ["Tstar", "planet_star_dist", "radius_star", "diff_ang", "Tint", "albedo", "kappa_sw",
          "kappa_lw", "kappa_lw_pole", "n_sw", "n_lw", "f_lw", "mean_motion", "alpha_i",
          "true_long_i", "ecc", "obliquity", "longp"]
RT_INT = ["latf_lw", "rt1Dmode", "sync_rot", "surface", "spinup_start", "spinup_stop",
          "spindown_start", "spindown_stop", "first_step"]
RT_DEFAULTS = dict(latf_lw=0, rt1Dmode=0, sync_rot=1, surface=0, spinup_start=-1, spinup_stop=-1,
                   spindown_start=-1, spindown_stop=-1, first_step=1, mean_motion=1.991e-7,
                   alpha_i=0.0, true_long_i=0.0, ecc=0.0, obliquity=0.0, longp=0.0)


class RtParams(ctypes.Structure):
    """oracle_rt_params / ref_rt_params (the product's thorx_rt_params has the same layout)."""
    _fields_ = [(n, ctypes.c_double) for n in RT_F64] + [(n, ctypes.c_int) for n in RT_INT]


def rt_struct(d):
    v = dict(RT_DEFAULTS)
    v.update(d)
    return RtParams(*[float(v[n]) for n in RT_F64], *[int(v[n]) for n in RT_INT])


SPONGE_FIELDS = [("nlat_bins", ctypes.c_int), ("Ruv_sponge", ctypes.c_double),
                 ("Rw_sponge", ctypes.c_double), ("RT_sponge", ctypes.c_double),
                 ("ns_ray_sponge", ctypes.c_double), ("damp_uv_to_mean", ctypes.c_int),
                 ("damp_w_to_mean", ctypes.c_int), ("RayleighSpongeT", ctypes.c_int),
                 ("shrink_sponge", ctypes.c_int), ("t_shrink", ctypes.c_int),
                 ("first_step", ctypes.c_int), ("raysp_calc_mode", ctypes.c_int)]
# the reference's defaults, src/headers/define.h:59-78
SPONGE_DEFAULTS = dict(nlat_bins=20, Ruv_sponge=1e-4, Rw_sponge=1e-4, RT_sponge=1e-4,
                       ns_ray_sponge=0.75, damp_uv_to_mean=1, damp_w_to_mean=1,
                       RayleighSpongeT=0, shrink_sponge=0, t_shrink=144000, first_step=1,
                       raysp_calc_mode=0)


class SpongeParams(ctypes.Structure):
    """oracle_sponge_params / ref_sponge_params (same layout as thorx_sponge_params)."""
    _fields_ = SPONGE_FIELDS


def sponge_struct(d):
    v = dict(SPONGE_DEFAULTS)
    v.update(d)
    return SpongeParams(*[float(v[n]) if t is ctypes.c_double else int(v[n])
                          for n, t in SPONGE_FIELDS])


# ------------------------------------------------------------------------------------------------
# Reference grid (reference src/ESP/grid.cu, host code, runs on the CPU)
# ------------------------------------------------------------------------------------------------
GRID_NAMES_F64 = ["point_xyz", "point_xyzq", "Altitude", "Altitudeh", "lonlat", "areas", "areasT",
                  "areasTr", "nvec", "nvecoa", "nvecti", "nvecte", "mvec", "div", "grad", "curlz",
                  "func_r"]
GRID_NAMES_I32 = ["pent_ind", "maps", "point_local"]

_ref = {}


def ref_lib(nofma=False):
    if nofma not in _ref:
        lib = ctypes.CDLL(REF_NOFMA_SO if nofma else REF_SO)
        lib.ref_grid_new.restype = ctypes.c_void_p
        lib.ref_grid_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_int, ctypes.c_double]
        lib.ref_grid_new_sponge.restype = ctypes.c_void_p
        lib.ref_grid_new_sponge.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_int]
        lib.ref_sim_sponge.restype = ctypes.c_int
        lib.ref_sim_sponge.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_sim_sponge_means.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_sim_probe.restype = ctypes.c_int
        lib.ref_sim_probe.argtypes = [ctypes.c_void_p]
        lib.ref_sim_vert_hydiff.restype = ctypes.c_int
        lib.ref_sim_vert_hydiff.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        lib.ref_grid_get.restype = ctypes.c_long
        lib.ref_grid_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        lib.ref_grid_dims.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 4
        lib.ref_grid_free.argtypes = [ctypes.c_void_p]
        lib.ref_sim_new.restype = ctypes.c_void_p
        lib.ref_sim_new.argtypes = [ctypes.c_void_p, ctypes.POINTER(Params)]
        lib.ref_sim_set.restype = ctypes.c_long
        lib.ref_sim_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        lib.ref_sim_get.restype = ctypes.c_long
        lib.ref_sim_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        lib.ref_sim_step.restype = ctypes.c_int
        lib.ref_sim_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.ref_sim_time.restype = ctypes.c_double
        lib.ref_sim_time.argtypes = [ctypes.c_void_p, ctypes.c_int]
        lib.ref_sim_free.argtypes = [ctypes.c_void_p]
        lib.ref_sim_globdiag.restype = ctypes.c_int
        lib.ref_sim_globdiag.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_sim_rt.restype = ctypes.c_int
        lib.ref_sim_rt.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_sim_conv_adj.restype = ctypes.c_int
        lib.ref_sim_conv_adj.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        lib.ref_sim_rt_totals.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double)]
        lib.ref_device_sum.restype = ctypes.c_double
        lib.ref_device_sum.argtypes = [ctypes.c_void_p, ctypes.c_long]
        _ref[nofma] = lib
    return _ref[nofma]


class RefGrid:
    """The reference's own Icogrid, built on the host, with its arrays copied out."""

    def __init__(self, glevel, nv, A=EARTH["A"], top=EARTH["Top_altitude"], sprd=1, beta=1.15,
                 nlat=None):
        """nlat: also build the Rayleigh sponge's zonal-mean table with nlat latitude bins."""
        lib = ref_lib()
        if nlat:
            self.h = lib.ref_grid_new_sponge(glevel, nv, A, top, sprd, beta, nlat)
        else:
            self.h = lib.ref_grid_new(glevel, nv, A, top, sprd, beta)
        d = [ctypes.c_int() for _ in range(4)]
        lib.ref_grid_dims(self.h, *[ctypes.byref(x) for x in d])
        self.point_num, self.nv, self.nl_region, self.nr = [x.value for x in d]
        self.glevel = glevel
        self.arrays = {}
        for name in GRID_NAMES_F64 + GRID_NAMES_I32 + (["zonal_mean_tab"] if nlat else []):
            n = lib.ref_grid_get(self.h, name.encode(), None)
            a = np.zeros(n, dtype=np.float64 if name in GRID_NAMES_F64 else np.int32)
            assert n >= 0, name
            lib.ref_grid_get(self.h, name.encode(), a.ctypes.data)
            self.arrays[name] = a

    def __getitem__(self, k):
        return self.arrays[k]

    def close(self):
        if self.h:
            ref_lib().ref_grid_free(self.h)
            self.h = None


# ------------------------------------------------------------------------------------------------
# Seeded initial state: isothermal hydrostatic column (reference src/ESP/esp_initial.cu:507-588)
# plus uniform temperature noise from SplitMix64, p kept, rho = p / (Rd T).
# ------------------------------------------------------------------------------------------------
def splitmix64_uniform(n, seed):
    """n uniform doubles in [0,1) from SplitMix64 (Steele, Lea & Flood 2014), top 53 bits."""
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + (np.arange(1, n + 1, dtype=np.uint64)
                               * np.uint64(0x9E3779B97F4A7C15))
        z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def isothermal_column(Altitude, Altitudeh, c):
    nv = len(Altitude)
    p = np.zeros(nv)
    rho = np.zeros(nv)
    T = np.zeros(nv)
    eps, it_max = 1e-15, 100
    Rd, Tm, g = c["Rd"], c["Tmean"], c["Gravit"]
    for lev in range(nv):
        if lev == 0:
            P_L, rho_L, T_L, dz = c["P_Ref"], c["P_Ref"] / (Rd * Tm), Tm, Altitude[0]
            l_int = r_int = 0.5
        else:
            P_L, rho_L, T_L = p[lev - 1], rho[lev - 1], T[lev - 1]
            dz = Altitude[lev] - Altitude[lev - 1]
            l_int = (Altitude[lev] - Altitudeh[lev]) / dz
            r_int = (Altitudeh[lev] - Altitude[lev - 1]) / dz
        g_L = g
        p[lev], rho[lev], T[lev] = P_L, rho_L, T_L
        ptmp = p[lev] + 2 * eps * p[lev]
        it = 0
        while it < it_max and (ptmp - p[lev]) / p[lev] > eps:
            ptmp = p[lev]
            f = (p[lev] - P_L) / dz + (g * r_int + g_L * l_int) * (rho[lev] * r_int + rho_L * l_int)
            df = 1.0 / dz + (g * r_int + g_L * l_int) * r_int / (Rd * T[lev])
            p[lev] = p[lev] - f / df
            rho[lev] = p[lev] / (Rd * T[lev])
            it += 1
    return p, rho, T


def guillot_T(p, mu, Teq, P_Ref, g, Tint, f_lw, kappa_sw, kappa_lw):
    """Guillot (2010) eq. 27 as the reference evaluates it (src/ESP/ultrahot_thermo.cu:121-161)."""
    tau0 = kappa_lw * P_Ref / g
    eps = 1.0 / f_lw
    x0 = P_Ref / g
    gamma0 = kappa_sw / kappa_lw
    klw = kappa_lw * (1.0 + 2 * (eps - 1) * p / P_Ref)
    x = p / g
    tau = kappa_lw * x
    tau_lw = tau0 * p / P_Ref + (eps - 1) * tau0 * (p / P_Ref) ** 2
    gamma = kappa_sw / klw
    e = math.exp(-gamma0 * tau / mu)
    T4 = (0.75 * Tint ** 4 * (2. / 3 + tau_lw)
          + 3 * mu * Teq ** 4 * (2. / 3 + gamma / (3 * mu) * e + mu / gamma0 * (1.0 - e)
                                 + 2 * (eps - 1) * mu / (gamma0 * kappa_sw * x0)
                                 * (mu - (mu + gamma0 * tau) * e)))
    return T4 ** 0.25


def guillot_column(Altitude, Altitudeh, c, Tint, f_lw, kappa_sw, kappa_lw):
    """Rest column on the Guillot profile: the general branch of initial_values
    (src/ESP/esp_initial.cu:840-1000), Teq = Tmean, mu = 0.5, constant gravity."""
    nv = len(Altitude)
    p, T = np.zeros(nv), np.zeros(nv)
    g, Rd, PR, mu = c["Gravit"], c["Rd"], c["P_Ref"], 0.5
    for lev in range(nv):
        if lev == 0:
            T[0] = guillot_T(PR, mu, c["Tmean"], PR, g, Tint, f_lw, kappa_sw, kappa_lw)
            P_L, T_L, dz, l_int, r_int = PR, T[0], Altitude[0], 0.5, 0.5
        else:
            T[lev] = T[lev - 1]
            P_L, T_L = p[lev - 1], T[lev - 1]
            dz = Altitude[lev] - Altitude[lev - 1]
            l_int = (Altitude[lev] - Altitudeh[lev]) / dz
            r_int = (Altitudeh[lev] - Altitude[lev - 1]) / dz
        p[lev], T[lev] = P_L, T_L
        ptmp = p[lev] + 2 * 1e-15 * p[lev]
        it = 0
        while it < 100 and (ptmp - p[lev]) / p[lev] > 1e-15:
            ptmp = p[lev]
            f = (p[lev] - P_L) / dz + (g * r_int + g * l_int) / Rd * (p[lev] * r_int / T[lev]
                                                                     + P_L * l_int / T_L)
            df = 1.0 / dz + (g * r_int + g * l_int) * r_int / (Rd * T[lev])
            p[lev] = p[lev] - f / df
            T[lev] = guillot_T(p[lev], mu, c["Tmean"], PR, g, Tint, f_lw, kappa_sw, kappa_lw)
            it += 1
    return p, T, p / (T * Rd)


def hydrostatic_column(Altitude, Altitudeh, c, Tprof):
    """Pressure and density of a column with temperature profile Tprof in the model's discrete
    hydrostatic balance (the Newton iteration of isothermal_column, the temperature given)."""
    nv = len(Altitude)
    p, rho = np.zeros(nv), np.zeros(nv)
    Rd, g = c["Rd"], c["Gravit"]
    for lev in range(nv):
        if lev == 0:
            P_L, rho_L, dz = c["P_Ref"], c["P_Ref"] / (Rd * Tprof[0]), Altitude[0]
            l_int = r_int = 0.5
        else:
            P_L, rho_L = p[lev - 1], rho[lev - 1]
            dz = Altitude[lev] - Altitude[lev - 1]
            l_int = (Altitude[lev] - Altitudeh[lev]) / dz
            r_int = (Altitudeh[lev] - Altitude[lev - 1]) / dz
        p[lev], rho[lev] = P_L, P_L / (Rd * Tprof[lev])
        for _ in range(100):
            f = (p[lev] - P_L) / dz + g * (rho[lev] * r_int + rho_L * l_int)
            df = 1.0 / dz + g * r_int / (Rd * Tprof[lev])
            step = f / df
            p[lev] -= step
            rho[lev] = p[lev] / (Rd * Tprof[lev])
            if abs(step) <= 1e-15 * p[lev]:
                break
    return p, rho


def unstable_state(grid_arrays, N, nv, c, seed=20260101, lapse=0.015, nlow=4, amp=2.0):
    """A rest state whose lowest nlow levels are cooled superadiabatically (lapse in K/m, against
    the dry adiabat g/Cp), in discrete hydrostatic balance, with +-amp K of seeded noise at fixed
    pressure: many statically unstable stretches for the convective adjustment."""
    alt = np.asarray(grid_arrays["Altitude"])
    Tprof = c["Tmean"] - lapse * np.minimum(alt, alt[min(nlow, nv) - 1])
    p0, _ = hydrostatic_column(alt, np.asarray(grid_arrays["Altitudeh"]), c, Tprof)
    noise = (2.0 * splitmix64_uniform(N * nv, seed) - 1.0) * amp
    T = np.tile(Tprof, N) + noise
    p = np.tile(p0, N)
    return dict(Rho=p / (c["Rd"] * T), pressure=p, temperature=T, Mh=np.zeros(3 * N * nv),
                Wh=np.zeros(N * (nv + 1)), W=np.zeros(N * nv), Rd=np.full(N * nv, c["Rd"]),
                Cp=np.full(N * nv, c["Cp"]))


def initial_state(grid_arrays, N, nv, c, seed=20260101, amp=0.1):
    """Reference-layout initial state: dict of Rho, pressure, temperature, Mh, Wh, W, Rd, Cp."""
    p0, rho0, T0 = isothermal_column(grid_arrays["Altitude"], grid_arrays["Altitudeh"], c)
    noise = (2.0 * splitmix64_uniform(N * nv, seed) - 1.0) * amp
    T = np.tile(T0, N) + noise
    p = np.tile(p0, N)
    rho = p / (c["Rd"] * T)
    return dict(Rho=rho, pressure=p, temperature=T, Mh=np.zeros(3 * N * nv),
                Wh=np.zeros(N * (nv + 1)), W=np.zeros(N * nv), Rd=np.full(N * nv, c["Rd"]),
                Cp=np.full(N * nv, c["Cp"]))


# ------------------------------------------------------------------------------------------------
# The CPU restatement (oracle)
# ------------------------------------------------------------------------------------------------
class OracleGrid(ctypes.Structure):
    _fields_ = [("point_num", ctypes.c_int), ("nv", ctypes.c_int), ("nl_region", ctypes.c_int),
                ("nr", ctypes.c_int), ("maps", ctypes.c_void_p), ("point_local", ctypes.c_void_p),
                ("Altitude", ctypes.c_void_p), ("Altitudeh", ctypes.c_void_p),
                ("lonlat", ctypes.c_void_p), ("areas", ctypes.c_void_p),
                ("areasTr", ctypes.c_void_p), ("nvecoa", ctypes.c_void_p),
                ("nvecti", ctypes.c_void_p), ("nvecte", ctypes.c_void_p),
                ("div", ctypes.c_void_p), ("grad", ctypes.c_void_p), ("func_r", ctypes.c_void_p),
                ("areasT", ctypes.c_void_p)]


_oracle = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_new.restype = ctypes.c_void_p
        lib.oracle_new.argtypes = [ctypes.POINTER(OracleGrid), ctypes.POINTER(Params)]
        lib.oracle_set.restype = ctypes.c_long
        lib.oracle_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        lib.oracle_get.restype = ctypes.c_long
        lib.oracle_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]
        lib.oracle_step.restype = ctypes.c_int
        lib.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.oracle_globdiag.restype = ctypes.c_int
        lib.oracle_globdiag.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_rt.restype = ctypes.c_int
        lib.oracle_rt.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_conv_adj.restype = ctypes.c_int
        lib.oracle_conv_adj.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        lib.oracle_vert_hydiff.restype = ctypes.c_int
        lib.oracle_vert_hydiff.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        lib.oracle_sponge.restype = ctypes.c_int
        lib.oracle_sponge.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_sponge_means.restype = ctypes.c_int
        lib.oracle_sponge_means.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.oracle_rt_totals.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_double)]
        lib.oracle_sum.restype = ctypes.c_double
        lib.oracle_sum.argtypes = [ctypes.c_void_p, ctypes.c_long]
        lib.oracle_set_threads.argtypes = [ctypes.c_int]
        lib.oracle_free.argtypes = [ctypes.c_void_p]
        _oracle = lib
    return _oracle


class Oracle:
    def __init__(self, grid, params):
        """grid: object with point_num, nv, nl_region, nr and reference-layout arrays."""
        lib = oracle_lib()
        names = ["maps", "point_local", "Altitude", "Altitudeh", "lonlat", "areas", "areasTr",
                 "nvecoa", "nvecti", "nvecte", "div", "grad", "func_r", "areasT"]
        self._keep = {k: np.ascontiguousarray(grid[k]) for k in names}
        g = OracleGrid(grid.point_num, grid.nv, grid.nl_region, grid.nr,
                       *[self._keep[k].ctypes.data for k in names])
        self.h = lib.oracle_new(ctypes.byref(g), ctypes.byref(params))
        self._nv = grid.nv

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        n = oracle_lib().oracle_set(self.h, name.encode(), a.ctypes.data)
        assert n == a.size, (name, n, a.size)

    def get(self, name):
        n = oracle_lib().oracle_get(self.h, name.encode(), None)
        assert n >= 0, name
        a = np.zeros(n)
        oracle_lib().oracle_get(self.h, name.encode(), a.ctypes.data)
        return a

    def step(self, n=1, profx=True, thor=True):
        assert oracle_lib().oracle_step(self.h, n, int(profx), int(thor)) == 0

    def rt(self, d):
        self._rt = rt_struct(d)
        assert oracle_lib().oracle_rt(self.h, ctypes.byref(self._rt)) == 0

    def conv_adj(self, iterations=1, soft=False):
        assert oracle_lib().oracle_conv_adj(self.h, iterations, int(soft)) == 0

    def sponge(self, d):
        self._sp = sponge_struct(d)
        assert oracle_lib().oracle_sponge(self.h, ctypes.byref(self._sp)) == 0

    def vert_hydiff(self, Diffc_v, order=6):
        assert oracle_lib().oracle_vert_hydiff(self.h, Diffc_v, order) == 0

    def sponge_means(self):
        nlat, nv = self._sp.nlat_bins, self._nv
        vbar, tbar = np.zeros((nlat, nv, 3)), np.zeros((nlat, nv))
        assert oracle_lib().oracle_sponge_means(self.h, vbar.ctypes.data, tbar.ctypes.data) == 0
        return vbar, tbar

    def rt_totals(self):
        a, o = ctypes.c_double(), ctypes.c_double()
        oracle_lib().oracle_rt_totals(self.h, ctypes.byref(a), ctypes.byref(o))
        return a.value, o.value

    def globdiag(self):
        """(sums, sums of magnitudes) of energy, mass, AMx, AMy, AMz, entropy."""
        out, mag = np.zeros(6), np.zeros(6)
        assert oracle_lib().oracle_globdiag(self.h, out.ctypes.data, mag.ctypes.data) == 0
        return out, mag

    def close(self):
        if self.h:
            oracle_lib().oracle_free(self.h)
            self.h = None


class RefSim:
    """The reference's own FP64 CUDA kernels driven by oracle/ref_harness.cu (needs a GPU)."""

    def __init__(self, refgrid, params, nofma=False):
        self.lib = ref_lib(nofma)
        self.h = self.lib.ref_sim_new(refgrid.h, ctypes.byref(params))
        assert self.h, "ref_sim_new failed"
        self._nv = refgrid.nv

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        n = self.lib.ref_sim_set(self.h, name.encode(), a.ctypes.data)
        assert n == a.size, (name, n, a.size)

    def get(self, name):
        n = self.lib.ref_sim_get(self.h, name.encode(), None)
        assert n >= 0, name
        a = np.zeros(n)
        assert self.lib.ref_sim_get(self.h, name.encode(), a.ctypes.data) == n
        return a

    def step(self, n=1, profx=True, thor=True):
        assert self.lib.ref_sim_step(self.h, n, int(profx), int(thor)) == 0

    def time(self, n):
        return self.lib.ref_sim_time(self.h, n)

    def rt(self, d):
        self._rt = rt_struct(d)
        assert self.lib.ref_sim_rt(self.h, ctypes.byref(self._rt)) == 0

    def conv_adj(self, iterations=1, soft=False):
        assert self.lib.ref_sim_conv_adj(self.h, iterations, int(soft)) == 0

    def vert_hydiff(self, Diffc_v, order=6):
        assert self.lib.ref_sim_vert_hydiff(self.h, Diffc_v, order) == 0

    def probe(self):
        """The harness's probe module (oracle/ref_harness.cu): a tracer through the reference's
        RK array registry, snapshots at the fast-mode hook, +0.5 K in phy_loop."""
        assert self.lib.ref_sim_probe(self.h) == 0

    def sponge(self, refgrid, d):
        """refgrid: a RefGrid built with nlat = d's nlat_bins."""
        self._sp = sponge_struct(d)
        assert self.lib.ref_sim_sponge(self.h, refgrid.h, ctypes.byref(self._sp)) == 0

    def sponge_means(self):
        nlat, nv = self._sp.nlat_bins, self._nv
        vbar, tbar = np.zeros((nlat, nv, 3)), np.zeros((nlat, nv))
        self.lib.ref_sim_sponge_means(self.h, vbar.ctypes.data, tbar.ctypes.data)
        return vbar, tbar

    def rt_totals(self):
        a, o = ctypes.c_double(), ctypes.c_double()
        self.lib.ref_sim_rt_totals(self.h, ctypes.byref(a), ctypes.byref(o))
        return a.value, o.value

    def globdiag(self):
        out = np.zeros(6)
        assert self.lib.ref_sim_globdiag(self.h, out.ctypes.data) == 0
        return out

    def close(self):
        if self.h:
            self.lib.ref_sim_free(self.h)
            self.h = None


def rel_err(a, b):
    """max|a-b| / max|b| (b the reference), 0 when both vanish."""
    den = np.max(np.abs(b))
    num = np.max(np.abs(a - b))
    if den == 0.0:
        return float(num)
    return float(num / den)


STATE_FIELDS = ["Rho", "pressure", "Mh", "Wh", "W"]


# ------------------------------------------------------------------------------------------------
# Product handles
# ------------------------------------------------------------------------------------------------
def thorx_params(c, timestep, precision=0):
    """thorx_params dict from a configuration dict as returned by make_params."""
    return dict(A=c["A"], Omega=c["Omega"], Gravit=c["Gravit"], Rd=c["Rd"], Cp=c["Cp"],
                P_Ref=c["P_Ref"], Top_altitude=c["Top_altitude"], timestep=timestep,
                Diffc=c["Diffc"], DivDampc=c["DivDampc"], HyDiffOrder=c["HyDiffOrder"],
                DeepModel=c["DeepModel"], NonHydro=c["NonHydro"],
                GravHeightVar=c["GravHeightVar"], HyDiff=c["HyDiff"], DivDampP=c["DivDampP"],
                thermo_equation=c["energy_equation"], core_benchmark=c["held_suarez"],
                precision=precision)


def grid_dict(g):
    d = dict(point_num=g.point_num, nv=g.nv, nl_region=g.nl_region, nr=g.nr)
    d.update(g.arrays)
    return d


def field_tolerance(spread, floor=1e-12, factor=4.0):
    """Tolerance of a field: 1e-12, or `factor` x the reference's own FMA / no-FMA spread where
    cancellation makes the reference itself that uncertain."""
    return max(floor, factor * spread)


# ------------------------------------------------------------------------------------------------
# The surrogate MLP restated on the CPU (oracle_mlp)
# ------------------------------------------------------------------------------------------------
def oracle_mlp(nv, H, Ws, bs, x, t=None):
    """float64 forward (and backward if t is given) of the surrogate network with the GPU's bf16
    rounding points. Ws, bs: the four padded layers as float32 arrays. Returns y, loss, gW, gb."""
    lib = oracle_lib()
    lib.oracle_mlp.restype = ctypes.c_int
    lib.oracle_mlp.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    Ws = [np.ascontiguousarray(w, dtype=np.float32) for w in Ws]
    bs = [np.ascontiguousarray(b, dtype=np.float32) for b in bs]
    Wp = (ctypes.c_void_p * 4)(*[w.ctypes.data for w in Ws])
    bp = (ctypes.c_void_p * 4)(*[b.ctypes.data for b in bs])
    x = np.ascontiguousarray(x, dtype=np.float32)
    B = x.shape[0]
    y = np.zeros((B, nv))
    loss = ctypes.c_double()
    gW = [np.zeros(w.shape) for w in Ws]
    gb = [np.zeros(b.shape) for b in bs]
    gWp = (ctypes.c_void_p * 4)(*[g.ctypes.data for g in gW])
    gbp = (ctypes.c_void_p * 4)(*[g.ctypes.data for g in gb])
    tt = None if t is None else np.ascontiguousarray(t, dtype=np.float32)
    assert lib.oracle_mlp(nv, H, Wp, bp, x.ctypes.data, None if tt is None else tt.ctypes.data, B,
                          y.ctypes.data, ctypes.byref(loss), gWp if tt is not None else None,
                          gbp if tt is not None else None) == 0
    return y, loss.value, gW, gb
