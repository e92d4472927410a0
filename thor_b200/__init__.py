"""thor_b200: Python handle on the thorx C ABI (include/thorx.h, thor_b200/libthorx.so).

The compute path is the CUDA library; this module only marshals host arrays in the reference
THOR layouts across the C ABI. There is no CPU fallback: importing works without a GPU, but
creating a context needs the library and a CUDA device and raises otherwise.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# THORX_LIB selects another build of the same ABI (e.g. libthorx_reforder.so, the FP64 form with
# the reference's operation order in the hyperdiffusion and divergence damping)
LIB_PATH = os.environ.get("THORX_LIB") or os.path.join(HERE, "libthorx.so")

FP64, MIXED = 0, 1
ENTROPY, ENERGY = 0, 1
NO_BENCHMARK, HELD_SUAREZ = 0, 1

E_ARG, E_CUDA, E_NAN, E_UNSUPPORTED, E_STATE, E_CONVERGENCE = -1, -2, -3, -4, -5, -6
ERRORS = {-1: "THORX_E_ARG", -2: "THORX_E_CUDA", -3: "THORX_E_NAN", -4: "THORX_E_UNSUPPORTED",
          -5: "THORX_E_STATE", -6: "THORX_E_CONVERGENCE"}


class ThorxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "?"), code, msg))
        self.code = code


class GridC(ctypes.Structure):
    _fields_ = [("point_num", ctypes.c_int), ("nv", ctypes.c_int), ("nl_region", ctypes.c_int),
                ("nr", ctypes.c_int), ("glevel", ctypes.c_int)] + [
        (n, ctypes.c_void_p) for n in
        ["maps", "point_local", "Altitude", "Altitudeh", "lonlat", "areas", "areasTr", "areasT",
         "nvecoa", "nvecti", "nvecte", "div", "grad", "func_r"]]


RT_F64 = ["Tstar", "planet_star_dist", "radius_star", "diff_ang", "Tint", "albedo", "kappa_sw",
          "kappa_lw", "kappa_lw_pole", "n_sw", "n_lw", "f_lw", "mean_motion", "alpha_i",
          "true_long_i", "ecc", "obliquity", "longp"]
RT_INT = ["latf_lw", "rt1Dmode", "sync_rot", "surface", "spinup_start", "spinup_stop",
          "spindown_start", "spindown_stop", "first_step"]


class RtParamsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in RT_F64] + [(n, ctypes.c_int) for n in RT_INT]


def rt_params(d):
    """thorx_rt_params from a dict (lengths in m, angles in degrees); missing switches off."""
    defaults = dict(latf_lw=0, rt1Dmode=0, sync_rot=1, surface=0, spinup_start=-1,
                    spinup_stop=-1, spindown_start=-1, spindown_stop=-1, first_step=1,
                    mean_motion=1.991e-7, alpha_i=0.0, true_long_i=0.0, ecc=0.0, obliquity=0.0,
                    longp=0.0)
    v = dict(defaults)
    v.update(d)
    return RtParamsC(*[float(v[n]) for n in RT_F64], *[int(v[n]) for n in RT_INT])


SPONGE_FIELDS = [("nlat_bins", ctypes.c_int), ("Ruv_sponge", ctypes.c_double),
                 ("Rw_sponge", ctypes.c_double), ("RT_sponge", ctypes.c_double),
                 ("ns_ray_sponge", ctypes.c_double), ("damp_uv_to_mean", ctypes.c_int),
                 ("damp_w_to_mean", ctypes.c_int), ("RayleighSpongeT", ctypes.c_int),
                 ("shrink_sponge", ctypes.c_int), ("t_shrink", ctypes.c_int),
                 ("first_step", ctypes.c_int), ("raysp_calc_mode", ctypes.c_int)]


class SpongeParamsC(ctypes.Structure):
    _fields_ = SPONGE_FIELDS


def sponge_params(d):
    """thorx_sponge_params from a dict; missing keys take the reference's defaults
    (src/headers/define.h:59-78)."""
    v = dict(nlat_bins=20, Ruv_sponge=1e-4, Rw_sponge=1e-4, RT_sponge=1e-4, ns_ray_sponge=0.75,
             damp_uv_to_mean=1, damp_w_to_mean=1, RayleighSpongeT=0, shrink_sponge=0,
             t_shrink=144000, first_step=1, raysp_calc_mode=0)
    v.update(d)
    return SpongeParamsC(*[float(v[n]) if t is ctypes.c_double else int(v[n])
                           for n, t in SPONGE_FIELDS])


class SurrogateParamsC(ctypes.Structure):
    _fields_ = [("hidden", ctypes.c_int), ("train_batch", ctypes.c_int),
                ("log_capacity", ctypes.c_longlong), ("recheck_period", ctypes.c_int),
                ("tolerance", ctypes.c_double), ("seed", ctypes.c_ulonglong)]


SUR_OFF, SUR_LOG, SUR_USE, SUR_USE_LOG = 0, 1, 2, 3


class ParamsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ["A", "Omega", "Gravit", "Rd", "Cp", "P_Ref", "Top_altitude", "timestep", "Diffc",
                 "DivDampc"]] + [
        (n, ctypes.c_int) for n in
        ["HyDiffOrder", "DeepModel", "NonHydro", "GravHeightVar", "HyDiff", "DivDampP",
         "thermo_equation", "core_benchmark", "precision"]]


_lib = None


def lib():
    """The loaded libthorx.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("%s is missing: run `python -m thor_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        vp, cp, ci = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int
        L.thorx_create.argtypes = [ctypes.POINTER(GridC), ctypes.POINTER(ParamsC), vp,
                                   ctypes.POINTER(vp)]
        L.thorx_create.restype = ci
        L.thorx_destroy.argtypes = [vp]
        L.thorx_last_error.argtypes = [vp]
        L.thorx_last_error.restype = cp
        L.thorx_field_size.argtypes = [vp, cp]
        L.thorx_field_size.restype = ctypes.c_long
        for f in ("thorx_set_field", "thorx_get_field"):
            getattr(L, f).argtypes = [vp, cp, vp]
            getattr(L, f).restype = ci
        for f in ("thorx_profx", "thorx_thor", "thorx_sync"):
            getattr(L, f).argtypes = [vp]
            getattr(L, f).restype = ci
        L.thorx_step.argtypes = [vp, ci]
        L.thorx_step.restype = ci
        L.thorx_kernels_per_step.argtypes = [vp]
        L.thorx_kernels_per_step.restype = ci
        L.thorx_grid_build.argtypes = [ci, ci, ctypes.c_double, ctypes.c_double, ci,
                                       ctypes.c_double, ctypes.POINTER(vp)]
        L.thorx_grid_build.restype = ci
        L.thorx_grid_info.argtypes = [vp] + [ctypes.POINTER(ci)] * 5
        L.thorx_grid_info.restype = ci
        L.thorx_grid_get.argtypes = [vp, cp, vp]
        L.thorx_grid_get.restype = ctypes.c_long
        L.thorx_grid_free.argtypes = [vp]
        L.thorx_init_rest_state.argtypes = [vp, ctypes.c_double, ctypes.c_ulonglong,
                                            ctypes.c_double]
        L.thorx_init_rest_state.restype = ci
        L.thorx_kernel_classes.argtypes = [vp]
        L.thorx_kernel_classes.restype = ci
        L.thorx_kernel_info.argtypes = [vp, ci, ctypes.POINTER(cp), ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ci)]
        L.thorx_kernel_info.restype = ci
        L.thorx_profile_steps.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_double)]
        L.thorx_profile_steps.restype = ci
        L.thorx_globdiag.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.thorx_globdiag.restype = ci
        L.thorx_device_sum.argtypes = [vp, ctypes.c_longlong, vp, ctypes.POINTER(ctypes.c_double)]
        L.thorx_device_sum.restype = ci
        L.thorx_device_sum_noalloc.argtypes = [vp, ctypes.c_longlong, vp,
                                               ctypes.POINTER(ctypes.c_double)]
        L.thorx_device_sum_noalloc.restype = ci
        L.thorx_set_precision.argtypes = [vp, ci]
        L.thorx_set_precision.restype = ci
        L.thorx_conv_adj_enable.argtypes = [vp, ci, ci]
        L.thorx_conv_adj_enable.restype = ci
        L.thorx_sponge_enable.argtypes = [vp, ctypes.POINTER(SpongeParamsC)]
        L.thorx_sponge_enable.restype = ci
        L.thorx_sponge_means.argtypes = [vp, vp, vp]
        L.thorx_sponge_means.restype = ci
        L.thorx_device_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(vp),
                                         ctypes.POINTER(ci), ctypes.POINTER(ci),
                                         ctypes.POINTER(ctypes.c_long)]
        L.thorx_device_field.restype = ci
        L.thorx_vert_hydiff_enable.argtypes = [vp, ctypes.c_double, ci]
        L.thorx_vert_hydiff_enable.restype = ci
        L.thorx_check_thomas.argtypes = [vp, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_longlong)]
        L.thorx_check_thomas.restype = ci
        L.thorx_globdiag_fields.argtypes = [vp, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_void_p)]
        L.thorx_globdiag_fields.restype = ci
        L.thorx_init_guillot_state.argtypes = [vp] + [ctypes.c_double] * 5 + [ctypes.c_ulonglong,
                                                                             ctypes.c_double]
        L.thorx_init_guillot_state.restype = ci
        L.thorx_bf16_gemm.argtypes = [vp, vp, ci, ci, ci, vp]
        L.thorx_bf16_gemm.restype = ci
        L.thorx_surrogate_last_error.restype = cp
        L.thorx_check_division.argtypes = [ctypes.c_longlong, ctypes.c_ulonglong,
                                           ctypes.POINTER(ctypes.c_longlong)]
        L.thorx_check_division.restype = ci
        L.thorx_surrogate_create.argtypes = [vp, ctypes.POINTER(SurrogateParamsC)]
        L.thorx_surrogate_set_mode.argtypes = [vp, ci]
        L.thorx_surrogate_logged.argtypes = [vp]
        L.thorx_surrogate_logged.restype = ctypes.c_longlong
        L.thorx_surrogate_train.argtypes = [vp, ci, ci, ctypes.c_double,
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]
        L.thorx_surrogate_stats.argtypes = [vp, vp]
        L.thorx_surrogate_layer.argtypes = [vp, ci, ctypes.POINTER(ci), ctypes.POINTER(ci), vp, vp,
                                            ci]
        L.thorx_surrogate_layer_grad.argtypes = [vp, ci, vp, vp]
        L.thorx_surrogate_normalisation.argtypes = [vp, vp, vp, vp, vp, ci]
        L.thorx_surrogate_forward_host.argtypes = [vp, vp, ci, vp]
        L.thorx_surrogate_gradients_host.argtypes = [vp, vp, vp, ci, ctypes.POINTER(ctypes.c_double)]
        for f in ["thorx_surrogate_create", "thorx_surrogate_set_mode", "thorx_surrogate_train",
                  "thorx_surrogate_stats", "thorx_surrogate_layer", "thorx_surrogate_layer_grad",
                  "thorx_surrogate_normalisation", "thorx_surrogate_forward_host",
                  "thorx_surrogate_gradients_host"]:
            getattr(L, f).restype = ci
        L.thorx_rt_enable.argtypes = [vp, ctypes.POINTER(RtParamsC)]
        L.thorx_rt_enable.restype = ci
        L.thorx_rt_totals.argtypes = [vp, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double)]
        L.thorx_rt_totals.restype = ci
        L.thorx_set_partition.argtypes = [vp, ci, ci]
        L.thorx_set_partition.restype = ci
        L.thorx_set_exchange.argtypes = [vp, EXCHANGE_FN, vp]
        L.thorx_set_exchange.restype = ci
        L.thorx_halo_columns.argtypes = [ctypes.POINTER(GridC), ci, ci, vp, ci]
        L.thorx_halo_columns.restype = ci
        L.thorx_copy_columns.argtypes = [vp, vp, cp, vp, ci]
        L.thorx_copy_columns.restype = ci
        for f in ("thorx_pack_columns", "thorx_unpack_columns"):
            getattr(L, f).argtypes = [vp, cp, vp, ci, vp]
            getattr(L, f).restype = ci
        L.thorx_set_graph_mode.argtypes = [vp, ci]
        L.thorx_set_graph_mode.restype = ci
        _lib = L
    return _lib


# thorx_exchange_fn: (user, ctx, stream, fields, nfields) -> status
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.POINTER(ctypes.c_char_p), ctypes.c_int)


def grid_struct(grid, glevel):
    """(thorx_grid, the arrays it points to) from a mapping of reference-layout arrays."""
    g = GridC(int(grid["point_num"]), int(grid["nv"]), int(grid["nl_region"]), int(grid["nr"]),
              int(glevel))
    keep = {}
    for k in GRID_KEYS:
        a = np.ascontiguousarray(grid[k], dtype=np.int32 if k in ("maps", "point_local")
                                 else np.float64)
        keep[k] = a
        setattr(g, k, a.ctypes.data)
    return g, keep


def halo_columns(grid, glevel, col_begin, col_end):
    """The halo of the columns [col_begin, col_end) of a grid (thorx_halo_columns; host only)."""
    g, keep = grid_struct(grid, glevel)
    n = lib().thorx_halo_columns(ctypes.byref(g), col_begin, col_end, None, 0)
    if n < 0:
        raise ThorxError(n, "thorx_halo_columns")
    out = np.zeros(max(n, 1), dtype=np.int32)
    lib().thorx_halo_columns(ctypes.byref(g), col_begin, col_end, out.ctypes.data, n)
    return out[:n]


EXPORTED = ["thorx_create", "thorx_destroy", "thorx_last_error", "thorx_field_size",
            "thorx_set_field", "thorx_get_field", "thorx_profx", "thorx_thor", "thorx_step",
            "thorx_sync", "thorx_kernels_per_step", "thorx_grid_build", "thorx_grid_info",
            "thorx_grid_get", "thorx_grid_describe", "thorx_grid_free", "thorx_init_rest_state",
            "thorx_kernel_classes", "thorx_kernel_info", "thorx_profile_steps", "thorx_globdiag",
            "thorx_device_sum", "thorx_device_sum_noalloc", "thorx_rt_enable",
            "thorx_rt_totals", "thorx_set_precision", "thorx_bf16_gemm", "thorx_surrogate_last_error",
            "thorx_surrogate_create", "thorx_surrogate_set_mode", "thorx_surrogate_logged",
            "thorx_surrogate_train", "thorx_surrogate_stats", "thorx_surrogate_layer",
            "thorx_surrogate_layer_grad", "thorx_surrogate_normalisation",
            "thorx_surrogate_forward_host", "thorx_surrogate_gradients_host",
            "thorx_check_division", "thorx_conv_adj_enable", "thorx_init_guillot_state",
            "thorx_sponge_enable", "thorx_sponge_means", "thorx_module_add",
            "thorx_rk_register_array", "thorx_device_field", "thorx_vert_hydiff_enable",
            "thorx_check_thomas", "thorx_globdiag_fields", "thorx_set_partition",
            "thorx_set_exchange", "thorx_halo_columns", "thorx_copy_columns",
            "thorx_pack_columns", "thorx_unpack_columns", "thorx_set_graph_mode"]

def device_sum(ptr, n, stream=0):
    """Compensated sum of n doubles at device address `ptr` (thorx_device_sum)."""
    out = ctypes.c_double()
    rc = lib().thorx_device_sum(ctypes.c_void_p(ptr), n, ctypes.c_void_p(stream), ctypes.byref(out))
    if rc:
        raise ThorxError(rc, lib().thorx_last_error(None).decode())
    return out.value


def bf16_bits(a):
    """float array -> bf16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def bf16_value(bits):
    """bf16 bit patterns -> float32 values."""
    return (np.asarray(bits, dtype=np.uint32) << 16).view(np.float32)


def bf16_gemm(A_bits, B_bits):
    """D = A . B^T on the tensor cores (thorx_bf16_gemm); A [M x K], B [N x K] bf16 bit patterns."""
    A_bits = np.ascontiguousarray(A_bits, dtype=np.uint16)
    B_bits = np.ascontiguousarray(B_bits, dtype=np.uint16)
    M, K = A_bits.shape
    N = B_bits.shape[0]
    D = np.zeros((M, N), dtype=np.float32)
    rc = lib().thorx_bf16_gemm(A_bits.ctypes.data, B_bits.ctypes.data, M, N, K, D.ctypes.data)
    if rc:
        raise ThorxError(rc, lib().thorx_surrogate_last_error().decode())
    return D


def check_division(n, seed=1):
    """thorx_check_division: (double, float) counts of n random pairs whose reciprocal-based
    quotient (the stencil kernels' area divisions) differs from the IEEE quotient."""
    out = (ctypes.c_longlong * 2)()
    rc = lib().thorx_check_division(n, seed, out)
    if rc:
        raise ThorxError(rc, lib().thorx_last_error(None).decode())
    return out[0], out[1]


NOALLOC_SUM_MAX_N = 134217728


def device_sum_noalloc(ptr, n, stream=0):
    """thorx_device_sum_noalloc: the same sum with no allocation (fixed 1 MiB device scratch,
    n <= NOALLOC_SUM_MAX_N, calls on one device must not overlap)."""
    out = ctypes.c_double()
    rc = lib().thorx_device_sum_noalloc(ctypes.c_void_p(ptr), n, ctypes.c_void_p(stream),
                                        ctypes.byref(out))
    if rc:
        raise ThorxError(rc, lib().thorx_last_error(None).decode())
    return out.value


GRID_F64 = ["point_xyz", "point_xyzq", "Altitude", "Altitudeh", "lonlat", "areas", "areasT",
            "areasTr", "nvec", "nvecoa", "nvecti", "nvecte", "div", "grad", "func_r"]
GRID_I32 = ["maps", "point_local", "pent_ind"]


class Icogrid:
    """THOR's icosahedral grid built by thorx_grid_build (host code, no GPU needed)."""

    def __init__(self, glevel, nv, A=6.371e6, Top_altitude=36e3, spring=True, beta=1.15):
        L = lib()
        h = ctypes.c_void_p()
        rc = L.thorx_grid_build(glevel, nv, A, Top_altitude, int(spring), beta, ctypes.byref(h))
        if rc != 0:
            raise ThorxError(rc, "thorx_grid_build(glevel=%d, nv=%d)" % (glevel, nv))
        self.h = h.value
        d = [ctypes.c_int() for _ in range(5)]
        L.thorx_grid_info(self.h, *[ctypes.byref(x) for x in d])
        self.point_num, self.nv, self.nl_region, self.nr, self.spring_iterations = [
            x.value for x in d]
        self.glevel = glevel
        self.arrays = {}
        for name in GRID_F64 + GRID_I32:
            n = L.thorx_grid_get(self.h, name.encode(), None)
            a = np.empty(n, dtype=np.int32 if name in GRID_I32 else np.float64)
            L.thorx_grid_get(self.h, name.encode(), a.ctypes.data)
            self.arrays[name] = a
        L.thorx_grid_free(self.h)
        self.h = None

    def __getitem__(self, k):
        return self.arrays[k]

    def as_dict(self):
        d = dict(point_num=self.point_num, nv=self.nv, nl_region=self.nl_region, nr=self.nr)
        d.update(self.arrays)
        return d

GRID_KEYS = ["maps", "point_local", "Altitude", "Altitudeh", "lonlat", "areas", "areasTr",
             "areasT", "nvecoa", "nvecti", "nvecte", "div", "grad", "func_r"]


class Thorx:
    """One simulation context (thorx_create .. thorx_destroy)."""

    def __init__(self, grid, glevel, params, stream=None):
        """grid: mapping with point_num, nv, nl_region, nr and the reference-layout arrays;
        params: dict of thorx_params fields."""
        L = lib()
        keep = {}
        g = GridC(int(grid["point_num"]), int(grid["nv"]), int(grid["nl_region"]),
                  int(grid["nr"]), int(glevel))
        for k in GRID_KEYS:
            dt = np.int32 if k in ("maps", "point_local") else np.float64
            a = np.ascontiguousarray(grid[k], dtype=dt)
            keep[k] = a
            setattr(g, k, a.ctypes.data)
        p = ParamsC()
        for name, _ in ParamsC._fields_:
            setattr(p, name, params[name])
        h = ctypes.c_void_p()
        rc = L.thorx_create(ctypes.byref(g), ctypes.byref(p), stream, ctypes.byref(h))
        self.h = h.value
        if rc != 0:
            msg = L.thorx_last_error(self.h).decode() if self.h else ""
            if self.h:
                L.thorx_destroy(self.h)
                self.h = None
            raise ThorxError(rc, msg)
        self.N = int(grid["point_num"])
        self.nv = int(grid["nv"])

    def _check(self, rc):
        if rc != 0:
            raise ThorxError(rc, lib().thorx_last_error(self.h).decode())

    def size(self, name):
        return lib().thorx_field_size(self.h, name.encode())

    def set(self, name, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        n = self.size(name)
        if n != a.size:
            raise ValueError("%s: expected %d values, got %d" % (name, n, a.size))
        self._check(lib().thorx_set_field(self.h, name.encode(), a.ctypes.data))

    def get(self, name, out=None):
        n = self.size(name)
        if n < 0:
            raise KeyError(name)
        if out is None:
            out = np.empty(n)
        self._check(lib().thorx_get_field(self.h, name.encode(), out.ctypes.data))
        return out

    def init_rest_state(self, Tmean, seed=20260101, noise_amp=0.1):
        self._check(lib().thorx_init_rest_state(self.h, Tmean, seed, noise_amp))

    def init_guillot_state(self, Tmean, Tint, f_lw, kappa_sw, kappa_lw, seed=20260101, noise_amp=0.0):
        """Rest state on the Guillot (2010) profile (Teq = Tmean), as init_PT_profile = guillot."""
        self._check(lib().thorx_init_guillot_state(self.h, Tmean, Tint, f_lw, kappa_sw, kappa_lw,
                                                   seed, noise_amp))

    def profx(self):
        self._check(lib().thorx_profx(self.h))

    def thor(self):
        self._check(lib().thorx_thor(self.h))

    def step(self, n=1):
        self._check(lib().thorx_step(self.h, n))

    def sync(self):
        self._check(lib().thorx_sync(self.h))

    def kernels_per_step(self):
        return lib().thorx_kernels_per_step(self.h)

    def kernel_table(self):
        """[(name, algorithmic bytes per launch, launches per step)] for each kernel class."""
        L = lib()
        out = []
        for k in range(L.thorx_kernel_classes(self.h)):
            name, b, n = ctypes.c_char_p(), ctypes.c_double(), ctypes.c_int()
            self._check(L.thorx_kernel_info(self.h, k, ctypes.byref(name), ctypes.byref(b),
                                            ctypes.byref(n)))
            out.append((name.value.decode(), b.value, n.value))
        return out

    def profile_steps(self, n):
        """Summed ms per kernel class over n eager steps timed with CUDA events."""
        k = lib().thorx_kernel_classes(self.h)
        ms = (ctypes.c_double * k)()
        self._check(lib().thorx_profile_steps(self.h, n, ms))
        return list(ms)

    def rt_enable(self, d):
        """Double-gray RT + insolation in every following ProfX (dict as for rt_params)."""
        self._rt = rt_params(d)
        self._check(lib().thorx_rt_enable(self.h, ctypes.byref(self._rt)))

    def rt_totals(self):
        """(ASR, OLR) of the last RT call, globally summed."""
        a, o = ctypes.c_double(), ctypes.c_double()
        self._check(lib().thorx_rt_totals(self.h, ctypes.byref(a), ctypes.byref(o)))
        return a.value, o.value

    def set_precision(self, precision):
        self._check(lib().thorx_set_precision(self.h, precision))

    def conv_adj(self, iterations=1, soft=False):
        """Dry convective adjustment in every following ProfX (0 iterations: off)."""
        self._check(lib().thorx_conv_adj_enable(self.h, iterations, int(soft)))

    def sponge(self, d=None):
        """Implicit Rayleigh sponge in every following ProfX (dict as for sponge_params; None:
        off)."""
        if d is None:
            self._sponge = None
            self._check(lib().thorx_sponge_enable(self.h, None))
            return
        self._sponge = sponge_params(d)
        self._check(lib().thorx_sponge_enable(self.h, ctypes.byref(self._sponge)))

    def globdiag_fields(self):
        """(the six global sums, the six per-cell term arrays [col][lev]) of thorx_globdiag_fields."""
        out = (ctypes.c_double * 6)()
        n = self.size("Rho")
        arrs = [np.zeros(n) for _ in range(6)]
        ptrs = (ctypes.c_void_p * 6)(*[a.ctypes.data for a in arrs])
        self._check(lib().thorx_globdiag_fields(self.h, out, ptrs))
        return np.array(list(out)), arrs

    def check_thomas(self, epsilon=1e-8):
        """(largest relative residual, interfaces above epsilon) of the last vertical solve."""
        m, n = ctypes.c_double(), ctypes.c_longlong()
        self._check(lib().thorx_check_thomas(self.h, epsilon, ctypes.byref(m), ctypes.byref(n)))
        return m.value, n.value

    def vert_hydiff(self, Diffc_v, order=6):
        """Vertical hyperdiffusion (VertHyDiff) in every following step; order 0: off."""
        self._check(lib().thorx_vert_hydiff_enable(self.h, Diffc_v, order))

    def device_field(self, name):
        """(device address, levels, components, plane stride) of a context array, for module
        kernels (thorx_device_field)."""
        d, lv, k, pl = ctypes.c_void_p(), ctypes.c_int(), ctypes.c_int(), ctypes.c_long()
        self._check(lib().thorx_device_field(self.h, name.encode(), ctypes.byref(d),
                                             ctypes.byref(lv), ctypes.byref(k), ctypes.byref(pl)))
        return d.value, lv.value, k.value, pl.value

    def set_partition(self, col_begin, col_end):
        """Compute only the columns [col_begin, col_end) (thorx_set_partition)."""
        self._check(lib().thorx_set_partition(self.h, col_begin, col_end))

    def set_exchange(self, fn):
        """fn(stream, [field names]) -> 0 after every kernel (thorx_set_exchange); None removes."""
        if fn is None:
            self._xfn = None
            self._check(lib().thorx_set_exchange(self.h, EXCHANGE_FN(), None))
            return

        def cb(user, ctx, stream, fields, n):
            try:
                return int(fn(stream, [fields[i].decode() for i in range(n)]))
            except Exception:  # an exception ends the step with an error, not the process
                return -100
        self._xfn = EXCHANGE_FN(cb)  # kept alive as long as the context uses it
        self._check(lib().thorx_set_exchange(self.h, self._xfn, None))

    def copy_columns(self, src, field, dev_cols, n):
        """All levels of the n columns at device address dev_cols of `field`, from context src
        (thorx_copy_columns, on this context's stream)."""
        self._check(lib().thorx_copy_columns(self.h, src.h, field.encode(), dev_cols, n))

    def sponge_means(self):
        """(vbar [bin][lev][3], Tbar [bin][lev]) of the last sponge step."""
        nlat, nv = self._sponge.nlat_bins, self.nv
        vbar = np.zeros((nlat, nv, 3))
        tbar = np.zeros((nlat, nv))
        self._check(lib().thorx_sponge_means(self.h, vbar.ctypes.data, tbar.ctypes.data))
        return vbar, tbar

    # ---- RT surrogate ----
    def sur_create(self, hidden=512, train_batch=8192, log_capacity=0, recheck_period=16,
                   tolerance=0.05, seed=1):
        self._sp = SurrogateParamsC(hidden, train_batch, log_capacity, recheck_period, tolerance,
                                    seed)
        self._check(lib().thorx_surrogate_create(self.h, ctypes.byref(self._sp)))

    def sur_mode(self, mode):
        self._check(lib().thorx_surrogate_set_mode(self.h, mode))

    def sur_logged(self):
        n = lib().thorx_surrogate_logged(self.h)
        if n < 0:
            self._check(int(n))
        return n

    def sur_train(self, iterations, batch, lr=1e-3):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(lib().thorx_surrogate_train(self.h, iterations, batch, lr, ctypes.byref(a),
                                                ctypes.byref(b)))
        return a.value, b.value

    def sur_stats(self):
        out = (ctypes.c_uint * 4)()
        self._check(lib().thorx_surrogate_stats(self.h, out))
        return dict(rechecked=out[0], failed=out[1], max_err=out[2] * 1e-6, rt_columns=out[3])

    def sur_layer(self, layer):
        n, k = ctypes.c_int(), ctypes.c_int()
        self._check(lib().thorx_surrogate_layer(self.h, layer, ctypes.byref(n), ctypes.byref(k),
                                                None, None, 0))
        W = np.zeros((n.value, k.value), dtype=np.float32)
        b = np.zeros(n.value, dtype=np.float32)
        self._check(lib().thorx_surrogate_layer(self.h, layer, None, None, W.ctypes.data,
                                                b.ctypes.data, 0))
        return W, b

    def sur_set_layer(self, layer, W, b):
        W = np.ascontiguousarray(W, dtype=np.float32)
        b = np.ascontiguousarray(b, dtype=np.float32)
        self._check(lib().thorx_surrogate_layer(self.h, layer, None, None, W.ctypes.data,
                                                b.ctypes.data, 1))

    def sur_grad(self, layer):
        W, b = self.sur_layer(layer)
        gW, gb = np.zeros_like(W), np.zeros_like(b)
        self._check(lib().thorx_surrogate_layer_grad(self.h, layer, gW.ctypes.data,
                                                     gb.ctypes.data))
        return gW, gb

    def sur_set_normalisation(self, in_mean, in_std, out_mean, out_std):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (in_mean, in_std, out_mean,
                                                                     out_std)]
        self._check(lib().thorx_surrogate_normalisation(self.h, *[a.ctypes.data for a in arrs], 1))

    def sur_normalisation(self, n_in, nv):
        arrs = [np.zeros(n, dtype=np.float32) for n in (n_in, n_in, nv, nv)]
        self._check(lib().thorx_surrogate_normalisation(self.h, *[a.ctypes.data for a in arrs], 0))
        return arrs

    def sur_forward(self, x, nv):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], nv), dtype=np.float32)
        self._check(lib().thorx_surrogate_forward_host(self.h, x.ctypes.data, x.shape[0],
                                                       y.ctypes.data))
        return y

    def sur_gradients(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = ctypes.c_double()
        self._check(lib().thorx_surrogate_gradients_host(self.h, x.ctypes.data, t.ctypes.data,
                                                         x.shape[0], ctypes.byref(loss)))
        return loss.value

    def globdiag(self):
        """Global energy, mass, angular momentum (x, y, z) and entropy of the current state."""
        out = (ctypes.c_double * 6)()
        self._check(lib().thorx_globdiag(self.h, out))
        return list(out)

    def close(self):
        if self.h:
            lib().thorx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
