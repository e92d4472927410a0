/* thorx — B200-native HE-VI dynamical core and double-gray RT for THOR, C ABI.
 *
 * One context owns one simulation on one GPU: the grid geometry, the prognostic state and the
 * scratch of the dynamical core, all resident in device memory in a column-index-fastest
 * layout. Host buffers passed across this interface use the reference THOR layouts:
 *   cell scalar    [col][lev]            (ESP::Rho_d, pressure_d, ...   src/headers/esp.h:226-371)
 *   cell vector    [col][lev][xyz]       (ESP::Mh_d)
 *   interface      [col][lev+1]          (ESP::Wh_d)
 *   grid arrays    as built by Icogrid   (src/ESP/grid.cu:84-302)
 * so that ESP can hand its own arrays over unchanged.
 *
 * Every function returns 0 on success and a negative THORX_E* code on error; the message of the
 * last error of a context is available from thorx_last_error(). Nothing calls exit().
 * One host thread per context. All work is ordered on the context's CUDA stream.
 */
#ifndef THORX_H
#define THORX_H

#ifdef __cplusplus
extern "C" {
#endif

#define THORX_OK 0
#define THORX_E_ARG -1      /* bad argument (null pointer, bad size, unknown name)        */
#define THORX_E_CUDA -2     /* a CUDA call failed (message has the CUDA error string)     */
#define THORX_E_NAN -3      /* the NaN check after the physics step tripped               */
#define THORX_E_UNSUPPORTED -4 /* option outside what this build implements               */
#define THORX_E_STATE -5    /* call out of order (e.g. stepping before the state is set)  */
#define THORX_E_CONVERGENCE -6 /* a column's convective adjustment exceeded its pass bound    */

typedef struct thorx_ctx thorx_ctx;

/* Grid geometry, reference layouts (Icogrid members, src/headers/grid.h:66-117).
 * The pointers are read during thorx_create only. */
typedef struct {
    int           point_num;  /* 2 + 10 * 4^glevel                                    */
    int           nv;         /* vertical layers                                       */
    int           nl_region;  /* rhombus side (16 for glevel 4..7)                     */
    int           nr;         /* number of rhombi                                      */
    int           glevel;
    const int*    maps;        /* [nr][(nl_region+2)^2]                                 */
    const int*    point_local; /* [point_num][6]                                        */
    const double* Altitude;    /* [nv]                                                  */
    const double* Altitudeh;   /* [nv+1]                                                */
    const double* lonlat;      /* [point_num][2]                                        */
    const double* areas;       /* [point_num][6][3]                                     */
    const double* areasTr;     /* [point_num][6]                                        */
    const double* areasT;      /* [point_num]                                           */
    const double* nvecoa;      /* [point_num][6][3]                                     */
    const double* nvecti;      /* [point_num][6][3]                                     */
    const double* nvecte;      /* [point_num][6][3]                                     */
    const double* div;         /* [point_num][7][3]                                     */
    const double* grad;        /* [point_num][7][3]                                     */
    const double* func_r;      /* [point_num][3]                                        */
} thorx_grid;

/* Precision forms of the dynamical core. */
#define THORX_FP64 0  /* every operation in FP64                                                */
#define THORX_MIXED 1 /* horizontal stencils and tendencies in FP32; Thomas solve, pressure and
                         density update, hydrostatic/effective-gravity integration and global
                         sums in FP64                                                          */

/* Thermodynamic equation (reference .thr key thermo_equation). */
#define THORX_ENTROPY 0
#define THORX_ENERGY 1

/* Benchmark forcing (reference .thr key core_benchmark; the values of the reference's
 * benchmark_types, src/headers/define.h:151-160). */
#define THORX_NO_BENCHMARK 0
#define THORX_HELD_SUAREZ 1
#define THORX_TIDALLY_LOCKED_EARTH 2 /* tidalearth, src/headers/phy/profx_tidalearth.h:49-126   */
#define THORX_SHALLOW_HOT_JUPITER 3  /* shallowHJ, src/headers/phy/profx_shallowHJ.h:50-128     */

/* Simulation switches: the SimulationSetup members the step reads
 * (src/headers/simulation_setup.h) and the .thr keys they come from. */
typedef struct {
    double A;            /* radius [m]                        (radius)          */
    double Omega;        /* rotation rate [1/s]               (rotation_rate)   */
    double Gravit;       /* gravity [m/s^2]                   (gravitation)     */
    double Rd;           /* gas constant [J/kg/K]             (Rd)              */
    double Cp;           /* heat capacity [J/kg/K]            (Cp)              */
    double P_Ref;        /* reference pressure [Pa]           (P_ref)           */
    double Top_altitude; /* model top [m]                     (Top_altitude)    */
    double timestep;     /* large step [s]                    (timestep)        */
    double Diffc;        /* hyperdiffusion coefficient        (Diffc)           */
    double DivDampc;     /* divergence damping coefficient    (DivDampc)        */
    int    HyDiffOrder;  /* even, >= 4                        (HyDiffOrder)     */
    int    DeepModel;    /*                                   (DeepModel)       */
    int    NonHydro;     /*                                   (NonHydro)        */
    int    GravHeightVar;/*                                   (GravHeightVar)   */
    int    HyDiff;       /*                                   (HyDiff)          */
    int    DivDampP;     /*                                   (DivDampP)        */
    int    thermo_equation; /* THORX_ENTROPY | THORX_ENERGY   (thermo_equation) */
    int    core_benchmark;  /* THORX_NO_BENCHMARK .. THORX_SHALLOW_HOT_JUPITER   */
    int    precision;       /* THORX_FP64 | THORX_MIXED                         */
} thorx_params;

/* Creates a context on the current CUDA device. `stream` is a cudaStream_t (NULL: the context
 * creates its own non-blocking stream). Replaces the device allocation and geometry upload of
 * ESP::ESP / ESP::alloc_data / initial_values (src/ESP/esp_initial.cu:68-484,1292-1393). */
int thorx_create(const thorx_grid* grid, const thorx_params* params, void* stream,
                 thorx_ctx** out);
void thorx_destroy(thorx_ctx* ctx);
const char* thorx_last_error(const thorx_ctx* ctx);

/* Copies a named field between a host buffer in the reference layout and the device.
 * Names are the reference ESP member names without the _d suffix: "Rho", "pressure", "Mh",
 * "Wh", "W", "temperature", "Rd", "Cp", "profx_Qheat", and the slow-mode tendencies of the last
 * RK stage "SlowMh", "SlowWh", "SlowRho", "Slowpressure". thorx_field_size gives the element
 * count of a name (negative if unknown). */
long thorx_field_size(const thorx_ctx* ctx, const char* name);
int thorx_set_field(thorx_ctx* ctx, const char* name, const double* host);
int thorx_get_field(thorx_ctx* ctx, const char* name, double* host);

/* Initial state at rest (src/ESP/esp_initial.cu:507-588, isothermal branch): the isothermal
 * hydrostatic column at Tmean from the Newton-Raphson solve of the reference, the same in every
 * column, plus a seeded uniform temperature perturbation in [-noise_amp, noise_amp) K from
 * SplitMix64(seed) on index col*nv + lev, at fixed pressure (rho = p / (Rd T)); Mh = W = Wh = 0,
 * Rd and Cp uniform. noise_amp = 0 gives the reference's noise-free rest state. */
int thorx_init_rest_state(thorx_ctx* ctx, double Tmean, unsigned long long seed, double noise_amp);
/* Rest state on the Guillot (2010) radiative-equilibrium profile (.thr init_PT_profile = guillot):
 * the general rest-state branch of initial_values (src/ESP/esp_initial.cu:840-1000) with
 * guillot_T (src/ESP/ultrahot_thermo.cu:121-161), Teq = Tmean, mu = 0.5 and the given internal
 * temperature and gray opacities (the .thr keys Tint, f_lw, kappa_sw, kappa_lw), in discrete
 * hydrostatic balance; then the seeded +-noise_amp K perturbation of thorx_init_rest_state. */
int thorx_init_guillot_state(thorx_ctx* ctx, double Tmean, double Tint, double f_lw,
                             double kappa_sw, double kappa_lw, unsigned long long seed,
                             double noise_amp);

/* Switches the precision form (THORX_FP64 / THORX_MIXED) between steps; the state and everything
 * else of the context carry over (both forms store FP64). A captured step graph is re-captured. */
int thorx_set_precision(thorx_ctx* ctx, int precision);

/* Dry convective adjustment in every following ProfX (sim.conv_adj with conv_adj_type = hourdin:
 * dry_conv_adj, src/headers/phy/dry_conv_adj.h:50-311, called at src/ESP/profx_driver.cu:239-290):
 * up to `iterations` rounds per step (the reference's conv_adj_iter; 0 switches it off);
 * soft_adjustment != 0 turns the adjustment into heating in profx_Qheat (soft_adjustment).
 * A column that exceeds the pass bound (the reference's loops have none) makes the next
 * thorx_sync return THORX_E_CONVERGENCE. */
int thorx_conv_adj_enable(thorx_ctx* ctx, int iterations, int soft_adjustment);

/* ---- Rayleigh sponge layer at the top of the model (RayleighSponge: sponge_layer with its zonal
 * means, src/ESP/profx_sponge.cu, run by ESP::ProfX at src/ESP/profx_driver.cu:96-194 in the
 * implicit mode and by ESP::Thor at src/ESP/thor_driver.cu:749-866 in the explicit ones; latitude
 * bins of Icogrid::zonal_mean_tab_f, src/ESP/grid.cu:3203-3260). The .thr keys of the same
 * names. ---- */
typedef struct {
    int    nlat_bins;       /* latitude bins over which the zonal means are taken (>= 1)     */
    double Ruv_sponge;      /* damping rate of the horizontal wind at the top [1/s]          */
    double Rw_sponge;       /* damping rate of the vertical wind at the top [1/s]            */
    double RT_sponge;       /* damping rate of the temperature (thermal sponge) [1/s]        */
    double ns_ray_sponge;   /* bottom of the sponge as a fraction of the model top, [0, 1)   */
    int    damp_uv_to_mean; /* damp u, v toward their zonal mean (else toward zero)          */
    int    damp_w_to_mean;  /* damp w toward its zonal mean (else toward zero)               */
    int    RayleighSpongeT; /* also damp the temperature toward its zonal mean               */
    int    shrink_sponge;   /* weaken the sponge exponentially after t_shrink steps          */
    int    t_shrink;        /* steps after which the sponge shrinks                          */
    int    first_step;      /* step number of the next physics step (1 at a fresh start)     */
    int    raysp_calc_mode; /* 0 imp: implicit, in ProfX; 1 exp1 / 2 exp3: explicit tendencies
                               in every RK stage of Thor, zonal means from the first stage (exp1)
                               or every stage (exp3) (src/ESP/thor_driver.cu:749-866)           */
} thorx_sponge_params;

/* Adds the Rayleigh sponge to every following step: the implicit one in ProfX between Recompute_W
 * and the temperature, the explicit ones before the slow modes of every RK stage; NULL switches it
 * off. A step graph captured earlier is re-captured. THORX_E_ARG for nlat_bins < 1, ns_ray_sponge
 * outside [0, 1) or an unknown raysp_calc_mode. */
int thorx_sponge_enable(thorx_ctx* ctx, const thorx_sponge_params* sp);
/* The zonal means of the last sponge step: vbar [bin][lev][3] (u, v, w; the reference's vbar_h;
 * zero where damp_*_to_mean is off) and Tbar [bin][lev] (zero without RayleighSpongeT); either
 * may be NULL. THORX_E_STATE when the sponge is off. */
int thorx_sponge_means(thorx_ctx* ctx, double* vbar, double* Tbar);

/* ---- Physics modules: the reference's phy_modules_* interface (src/headers/phy_modules.h:57-98)
 * as C callbacks, called where ESP calls the module manager: dyn_core_loop_init after Thor's
 * initial copies (src/ESP/thor_driver.cu:116), dyn_core_loop_slow_modes after the hyperdiffusion of
 * every RK stage (:641), dyn_core_loop_fast_modes between Vertical_Eq and Density_Pressure_Eqs of
 * every small step (:1290), dyn_core_loop_end after Thor's final copies (:1465), phy_loop in ProfX
 * after the benchmark forcing and the built-in RT, before Compute_pressure
 * (src/ESP/profx_driver.cu:405-416). Every hook may be NULL. A hook enqueues its device work on
 * `stream` (the context's stream) and returns 0, or a nonzero code that the enqueuing call
 * returns. thorx_step captures one step as a CUDA graph, so there the hooks run once, at capture,
 * and what they enqueued is replayed every step: their work must be stream-ordered device work
 * (kernels, device-to-device copies and sets) that keeps any per-step state on the device.
 * thorx_profx and thorx_thor call the hooks every time. rk (0..2) and ns (small step) locate the
 * call; times is the reference's `times` (the RK stage's small time step). ---- */
typedef struct {
    void* user;
    int (*dyn_core_loop_init)(void* user, thorx_ctx* ctx, void* stream);
    int (*dyn_core_loop_slow_modes)(void* user, thorx_ctx* ctx, void* stream, int rk, double times);
    int (*dyn_core_loop_fast_modes)(void* user, thorx_ctx* ctx, void* stream, int rk, int ns,
                                    double times);
    int (*dyn_core_loop_end)(void* user, thorx_ctx* ctx, void* stream);
    int (*phy_loop)(void* user, thorx_ctx* ctx, void* stream, double time_step);
} thorx_module;
/* Adds a module (at most 8; hooks run in the order modules were added). A step graph captured
 * earlier is re-captured. */
int thorx_module_add(thorx_ctx* ctx, const thorx_module* m);
/* device_RK_array_manager::register_array (src/ESP/phy_modules_device.cu:53-67): the RK stages
 * reset array = arrayi - arrayk at the start of stages 2 and 3 (UpdateRK) and accumulate
 * arrayk += array at the end of every stage (UpdateRK2), elementwise over
 * dimensions * nv * plane doubles (plane from thorx_device_field). At most 10 arrays. */
int thorx_rk_register_array(thorx_ctx* ctx, double* array, double* arrayk, double* arrayi,
                            int dimensions);
/* The same registry for arrays of any layout: the RK stages update `count` doubles of each array
 * elementwise (for a module that keeps its arrays in the reference layout, [col][lev][dim] of
 * point_num * nv * dimensions doubles; the register_array of the thorx_phy shim,
 * thor_b200/phy/). At most 10 arrays in all. */
int thorx_rk_register_array_n(thorx_ctx* ctx, double* array, double* arrayk, double* arrayi,
                              long long count);
/* use_graph = 0: thorx_step enqueues every step's kernels and calls every module hook each step,
 * instead of capturing the step once as a CUDA graph and replaying it; for modules whose hooks do
 * host work or launch on the legacy default stream (the reference's phy_modules_* managers through
 * the thorx_phy shim). 1 (the default) restores graph replay. */
int thorx_set_graph_mode(thorx_ctx* ctx, int use_graph);
/* ---- Partitioned step: the grid's columns divided among several contexts (one per GPU, or several
 * on one GPU), each computing its own columns and taking its halo (the neighbours of its columns
 * that others compute) from the others after every kernel. The decomposition the reference sketches
 * for multi-GPU runs (rhombi per rank, a one-cell halo exchanged before every horizontal stencil);
 * the reference itself runs on one GPU. Every context holds whole-grid arrays; only its own columns
 * (and, after an exchange, its halo) are current. The state after a step is bit for bit the
 * unpartitioned one. Not with the Rayleigh sponge, the surrogate, physics modules or
 * thorx_globdiag (whole-grid sums). ---- */
/* Restricts ctx to columns [col_begin, col_end): col_begin a multiple of 32, col_end a multiple of
 * 32 or point_num (whole rhombi qualify: 256 columns each at glevel >= 4; the two poles are the last
 * columns). A step graph captured earlier is re-captured. */
int thorx_set_partition(thorx_ctx* ctx, int col_begin, int col_end);
/* Called after every kernel of a step with the names (as for thorx_device_field) of the fields the
 * kernel wrote; the callee brings the halo columns of those fields up to date (thorx_copy_columns
 * between contexts of one process, or thorx_pack_columns / thorx_unpack_columns around a transfer
 * between processes), stream-ordered on `stream`, and returns 0 (else the step stops with that
 * code). Setting it makes thorx_step enqueue every step eagerly (thorx_set_graph_mode(ctx, 0)).
 * NULL removes it. */
typedef int (*thorx_exchange_fn)(void* user, thorx_ctx* ctx, void* stream,
                                 const char* const* fields, int nfields);
int thorx_set_exchange(thorx_ctx* ctx, thorx_exchange_fn fn, void* user);
/* Host only (no GPU needed): the halo of the columns [col_begin, col_end) of a grid, the columns
 * outside the range whose values the step's stencils read at those columns, ascending. Writes at
 * most cap of them to cols (which may be NULL) and returns how many there are, or a negative
 * status. */
int thorx_halo_columns(const thorx_grid* grid, int col_begin, int col_end, int* cols, int cap);
/* All levels and components of the n columns dev_cols (a device array) of a field: copied from src
 * to dst (contexts of the same grid whose devices can reach each other's memory), or packed to /
 * unpacked from dev_buf [n][levels * components] (device). Enqueued on dst's / ctx's stream; the
 * source's last write must be complete (the caller synchronises src). In the mixed form the
 * intermediate "divg" holds FP32 values (the buffer of dev_buf stays doubles, exact both ways);
 * both contexts of a copy must use the same form. */
int thorx_copy_columns(thorx_ctx* dst, thorx_ctx* src, const char* field, const int* dev_cols,
                       int n);
int thorx_pack_columns(thorx_ctx* ctx, const char* field, const int* dev_cols, int n,
                       double* dev_buf);
int thorx_unpack_columns(thorx_ctx* ctx, const char* field, const int* dev_cols, int n,
                         const double* dev_buf);
/* The context's device array of a field, for module kernels: *dev, its levels (nv or nv+1), its
 * components (1 or 3) and the plane stride (doubles): element (lev, col, comp) is at
 * dev[(comp * levels + lev) * plane + col]. Names: the thorx_get_field names and the dycore's
 * stage and deviation arrays "Rhok", "Rhos", "Mhk", "Mhs", "Whk", "Whs", "Wk", "pressurek",
 * "pressures", and "profx_dMh", "profx_dWh" (module tendencies of the slow modes). A field held
 * in FP32 (divg in the mixed form) returns THORX_E_UNSUPPORTED. */
int thorx_device_field(thorx_ctx* ctx, const char* name, double** dev, int* levels,
                       int* components, long* plane);

/* Sixth-order (or any even order >= 4) vertical hyperdiffusion in every following step (VertHyDiff
 * with Diffc_v and VertHyDiffOrder: vertical_diff, src/headers/dyn/thor_diff.h:1198-1426, called
 * in the hyperdiffusion block of ESP::Thor, src/ESP/thor_driver.cu:590-612; strengths
 * Kdv6 = Diffc_v dz^order / dt, src/ESP/esp_initial.cu:1327-1335). Like the reference it acts only
 * with HyDiff on. order 0 switches it off. A step graph captured earlier is re-captured. */
int thorx_vert_hydiff_enable(thorx_ctx* ctx, double Diffc_v, int order);

/* The check of the vertical solve that the reference compiles in with
 * DIAG_CHECK_THOR_VERTICAL_INT_THOMAS_RESULT (src/headers/dyn/thor_vertical_int.h:486-523): for
 * the last small step's tridiagonal system, the largest residual relative to the right-hand side
 * (absolute where it is 0) over the interior interfaces 2..nv-1 of all columns, and the number of
 * interfaces above epsilon (the reference uses 1e-8). Synchronises the context's stream. */
int thorx_check_thomas(thorx_ctx* ctx, double epsilon, double* max_rel, long long* n_bad);

/* One physics step, ESP::ProfX (src/ESP/profx_driver.cu:70-474): W from Wh, T and potential
 * temperature from p and rho, Held-Suarez forcing when core_benchmark says so, p = rho Rd T,
 * and the NaN check (reported at the next synchronising call as THORX_E_NAN). */
int thorx_profx(thorx_ctx* ctx);
/* One dynamical-core large step, ESP::Thor (src/ESP/thor_driver.cu:70-1466). */
int thorx_thor(thorx_ctx* ctx);
/* `nsteps` x (ProfX, Thor), the inner part of the main loop of src/esp.cu:1382-1398. The first
 * call captures one step as a CUDA graph; every step is a replay of it. */
int thorx_step(thorx_ctx* ctx, int nsteps);
/* Waits for the context's stream; returns THORX_E_NAN if a NaN check tripped since the last
 * synchronisation. */
int thorx_sync(thorx_ctx* ctx);
/* Number of kernels one thorx_step(ctx, 1) launches. */
int thorx_kernels_per_step(const thorx_ctx* ctx);

/* Kernel classes of a step, for roofline accounting: name, algorithmic bytes of one launch
 * (every element the kernel must read or write counted once, geometry included) and launches per
 * step. thorx_profile_steps runs `nsteps` steps eagerly with a CUDA event pair on the context's
 * stream around every launch and returns the summed milliseconds of each class in
 * ms_per_class[0 .. thorx_kernel_classes()-1]. */
int thorx_kernel_classes(const thorx_ctx* ctx);
int thorx_kernel_info(const thorx_ctx* ctx, int k, const char** name, double* bytes_per_launch,
                      int* launches_per_step);
int thorx_profile_steps(thorx_ctx* ctx, int nsteps, double* ms_per_class);

/* ---- Double-gray radiative transfer (radiative_transfer module with rt_type = DualbandGray,
 * src/physics/modules/src/radiative_transfer.cu, kernel rtm_dual_band
 * src/physics/modules/inc/profx_RT.h:316-587) and the insolation it uses (Insolation,
 * src/ESP/insolation.cu). The .thr keys of the same names; lengths in m (the .thr file gives
 * planet_star_dist in au and radius_star in solar radii), angles in degrees. ---- */
typedef struct {
    double Tstar;            /* stellar effective temperature [K]                      */
    double planet_star_dist; /* semi-major axis [m]                                   */
    double radius_star;      /* stellar radius [m]                                    */
    double diff_ang;         /* 1 / diffusivity factor                                */
    double Tint;             /* internal temperature [K]                              */
    double albedo;           /* Bond albedo                                           */
    double kappa_sw, kappa_lw, kappa_lw_pole; /* gray opacities [m^2/kg]              */
    double n_sw, n_lw;       /* pressure-scaling exponents of the optical depths      */
    double f_lw;             /* fraction of the LW optical depth that is uniform      */
    double mean_motion;      /* orbital mean motion [rad/s] (sync_rot: Omega is used) */
    double alpha_i;          /* initial right ascension of the star [deg]             */
    double true_long_i;      /* initial true longitude of the planet [deg]            */
    double ecc;              /* orbital eccentricity, 0 <= ecc < 1                    */
    double obliquity;        /* [deg]                                                 */
    double longp;            /* longitude of periastron [deg]                         */
    int    latf_lw;          /* sin^2(lat) variation of kappa_lw toward kappa_lw_pole */
    int    rt1Dmode;         /* cos(zenith) fixed at 0.5                              */
    int    sync_rot;         /* synchronous rotation                                  */
    int    surface;          /* must be 0: the surface layer is not implemented       */
    int    spinup_start, spinup_stop, spindown_start, spindown_stop; /* steps, -1 = off */
    int    first_step;       /* step number of the next physics step (1 at a fresh start) */
} thorx_rt_params;

/* Adds insolation + double-gray RT to every following ProfX, between the benchmark forcing and
 * the pressure update, heating into profx_Qheat (replaces the module's initialise_memory /
 * initial_conditions / phy_loop, radiative_transfer.cu:384-460,769-1105, and
 * Insolation::initial_conditions / phy_loop, insolation.cu:292-490). Call once, after
 * thorx_create; a step graph captured earlier is re-captured. Adds the fields "cos_zenith",
 * "insol", "insol_ann", "ASR", "OLR" ([col]), "phtemp", "thtemp", "fsw_up", "fsw_dn",
 * "flw_up", "flw_dn" ([col][lev+1]), "tau" ([col][lev][2]: SW, LW), "ttemp", "dtemp",
 * "DG_Qheat" ([col][lev]). THORX_E_UNSUPPORTED for surface != 0 and for GravHeightVar (whose
 * reference shortwave code reads past the end of Altitudeh). */
int thorx_rt_enable(thorx_ctx* ctx, const thorx_rt_params* rt);
/* Absorbed shortwave and outgoing longwave power of the last RT call, summed over the globe
 * (the reference's ASR_tot / OLR_tot, radiative_transfer.cu:1083-1084), compensated sums. */
int thorx_rt_totals(thorx_ctx* ctx, double* asr, double* olr);

/* ---- BF16 tensor-core GEMM (tcgen05, FP32 accumulate), the building block of the RT surrogate.
 * No counterpart in the reference. D[M x N] = A[M x K] . B[N x K]^T with A, B bf16 (raw 16-bit
 * patterns, row-major, K contiguous) and D float32, all host buffers. M a multiple of 128, N of
 * 64, K of 64. Context-free; on error thorx_surrogate_last_error() has the message. */
int thorx_bf16_gemm(const unsigned short* A, const unsigned short* B, int M, int N, int K, float* D);
const char* thorx_surrogate_last_error(void);

/* ---- Self-check of the division the stencil kernels use for the cell-area divisions: 1/b
 * rounded once per column, then each a/b from it by fused multiply-adds (Markstein's theorem),
 * which must equal the IEEE quotient bit for bit. n random (a, b) pairs per type, drawn on the
 * device from seed (exponents over +-300 in double, +-60 in float; half of them with near-exact
 * quotients), compared with a / b; mismatches[0] (double) and [1] (float) count the differing
 * pairs. Context-free, current device, default stream. */
int thorx_check_division(long long n, unsigned long long seed, long long mismatches[2]);

/* ---- Learned RT surrogate. No counterpart in the reference. ----
 * A per-column MLP from (T per level, ln p per level, cos zenith) to the double-gray RT heating
 * rates per level as temperature tendencies dT/dt = Q / (rho c_v) in K/s (Q in W m^-3 is what
 * rtm_dual_band adds to profx_Qheat; the surrogate's output is multiplied back by rho c_v before
 * it is added), 2 nv + 1 inputs, three hidden
 * layers of `hidden` units with GELU, nv outputs; BF16 weights and activations, FP32
 * accumulation on the tensor cores, FP32 master weights trained with Adam on the GPU. Inputs and
 * outputs are standardised with the mean and standard deviation of the logged training data
 * (fitted on the first thorx_surrogate_train call, or set with thorx_surrogate_normalisation).
 * Modes, set between steps (a captured step graph is re-captured):
 *   THORX_SUR_LOG  every physics step runs the plain RT and appends each column's inputs and
 *                  heating rates to a ring of log_capacity columns (the training set);
 *   THORX_SUR_USE  every physics step runs the surrogate on all columns and the plain RT only on
 *                  the columns it re-checks this step (the blocks of 32 columns with
 *                  (column / 32) % recheck_period == step % recheck_period, so a warp of the RT
 *                  kernel re-checks all its columns or none) and on those that have fallen back:
 *                  a re-checked column whose
 *                  relative error max|q_sur - q_rt| / max|q_rt| (q in K/s, maxima over the
 *                  column's levels) exceeds `tolerance` falls back
 *                  to the plain RT until a later re-check passes; re-checked columns use the
 *                  plain RT's heating. The cooling limiter and profx_Qheat coupling of the plain
 *                  RT apply to the chosen heating. ASR/OLR are current only on the columns the
 *                  plain RT ran on.
 *   THORX_SUR_USE_LOG as THORX_SUR_USE, and every column the plain RT ran on (re-checked or
 *                  fallen back) is appended to the log ring, so that training between steps
 *                  follows the states the run reaches (online learning; needs log_capacity > 0).
 * Requires thorx_rt_enable first. */
#define THORX_SUR_OFF 0
#define THORX_SUR_LOG 1
#define THORX_SUR_USE 2
#define THORX_SUR_USE_LOG 3
typedef struct {
    int                hidden;         /* hidden width, a multiple of 256 (512)               */
    int                train_batch;    /* largest training batch, a multiple of 128 (8192)     */
    long long          log_capacity;   /* logged columns kept (ring), 0 = no logging           */
    int                recheck_period; /* plain-RT re-check of 1/recheck_period columns (16)   */
    double             tolerance;      /* relative heating error that triggers fallback (0.05) */
    unsigned long long seed;           /* weight initialisation and batch sampling             */
} thorx_surrogate_params;
int thorx_surrogate_create(thorx_ctx* ctx, const thorx_surrogate_params* sp);
int thorx_surrogate_set_mode(thorx_ctx* ctx, int mode);
/* Columns logged so far (may exceed log_capacity: the ring keeps the latest). */
long long thorx_surrogate_logged(thorx_ctx* ctx);
/* `iterations` Adam steps (lr, batch rows drawn uniformly from the log); the mean squared error
 * (standardised units) of the first and the last batch. */
int thorx_surrogate_train(thorx_ctx* ctx, int iterations, int batch, double lr, double* loss_first,
                          double* loss_last);
/* Since the previous call: columns re-checked, re-checks that failed, the largest re-check error
 * (in units of 1e-6), and column-steps heated by the plain RT. Resets the counters. */
int thorx_surrogate_stats(thorx_ctx* ctx, unsigned int out[4]);
/* Weights of layer 0..3 (padded shapes N x K from the call; W [N][K], b [N]), get or set. */
int thorx_surrogate_layer(thorx_ctx* ctx, int layer, int* N, int* K, float* W, float* b, int set);
/* Gradients of the last thorx_surrogate_gradients_host / training batch (padded shapes). */
int thorx_surrogate_layer_grad(thorx_ctx* ctx, int layer, float* gW, float* gb);
/* Standardisation: in_* [2 nv + 1], out_* [nv]; get or set (set marks the surrogate usable). */
int thorx_surrogate_normalisation(thorx_ctx* ctx, float* in_mean, float* in_std, float* out_mean,
                                  float* out_std, int set);
/* Network output (standardised) for B standardised input rows x [B][2 nv + 1] -> y [B][nv]. */
int thorx_surrogate_forward_host(thorx_ctx* ctx, const float* x, int B, float* y);
/* Forward and backward pass of the MSE loss on (x [B][2 nv + 1], t [B][nv]) standardised rows,
 * B a multiple of 128, without an optimiser step; gradients via thorx_surrogate_layer_grad. */
int thorx_surrogate_gradients_host(thorx_ctx* ctx, const float* x, const float* t, int B,
                                   double* loss);

/* ---- Global conserved quantities (replaces ESP::globdiag, src/ESP/profx_driver.cu:476-569,
 * with the per-cell terms of CalcTotEnergy / CalcMass / CalcAngMom / CalcEntropy,
 * src/ESP/profx_globdiag.cu:45-252; no surface term) ----
 * out[0] total energy (J), out[1] mass (kg), out[2..4] angular momentum x, y, z (kg m^2 s^-1),
 * out[5] entropy (J K^-1) of the current state. Each is a compensated sum whose order of
 * addition is fixed: the same state gives the same bits on every call. Synchronises the
 * context's stream. */
int thorx_globdiag(thorx_ctx* ctx, double* out);
/* thorx_globdiag plus the per-cell terms the sums are made of, as the reference keeps them for its
 * output files (Etotal_d, Mass_d, AngMomx_d, AngMomy_d, AngMomz_d, Entropy_d of CalcTotEnergy /
 * CalcMass / CalcAngMom / CalcEntropy, src/ESP/profx_globdiag.cu:45-252): fields[q] (host, [col][lev],
 * q in the order of out; NULL entries are skipped). */
int thorx_globdiag_fields(thorx_ctx* ctx, double* out, double* const fields[6]);

/* Compensated sum of n doubles in device memory of the current device
 * (replaces gpu_sum_on_device<1024>, src/headers/reduction_add.h:96-128). x must point into one
 * device or managed allocation of the current device whose extent the driver reports
 * (cudaMalloc, cudaMallocManaged, cudaMallocAsync) and which holds n doubles from x on; both
 * are checked before any kernel runs (THORX_E_ARG otherwise). The sum runs on
 * `stream` (NULL: the legacy default stream), which is synchronised before *out is written.
 * Like the reference it allocates its partial sums with cudaMalloc for the call and frees them
 * after. Context-free: on error, thorx_last_error(NULL) gives this thread's message. */
int thorx_device_sum(const double* x, long long n, void* stream, double* out);

/* Allocation-free twin of thorx_device_sum. No counterpart in the reference.
 *
 * Same kernels, same order of addition, so the same bits as thorx_device_sum, but it allocates
 * no memory at all: the partial sums go to a fixed 1 MiB array in the library's own device
 * memory instead of a cudaMalloc per call. It is for callers that must not allocate:
 *  - a time loop whose device memory is fully budgeted (the model's arrays plus a framework's
 *    caching pool can leave no free megabyte, and a failed cudaMalloc mid-run loses the run);
 *  - a loop that keeps other streams busy (output copies, physics on a second stream): cudaFree
 *    synchronises the whole device and would stall that overlap at every diagnostic step.
 * Limits and rules:
 *  - n <= THORX_NOALLOC_SUM_MAX_N (134,217,728 doubles = 1 GiB of input); a larger n returns
 *    THORX_E_ARG with a message saying so (use thorx_device_sum);
 *  - there is one scratch per device per process: calls that overlap in time on the same device
 *    (e.g. from two host threads at once) race on it and can return wrong sums; serialise them;
 *  - the first call on each device sets the scratch up (it looks up the array's device address
 *    with cudaGetSymbolAddress, with that device current); make that first call before any stream
 *    capture begins;
 *  - nothing in the scratch has to start at zero: every entry a call reads, that call has
 *    written first.
 * Argument checks, stream and error reporting as thorx_device_sum. */
#define THORX_NOALLOC_SUM_MAX_N 134217728LL
int thorx_device_sum_noalloc(const double* x, long long n, void* stream, double* out);

/* ---- Icosahedral grid (replaces Icogrid::Icogrid, src/ESP/grid.cu:84-302) ----
 * Builds THOR's grid on the host: same point order, neighbours, rhombus maps, spring-dynamics
 * relaxation (beta = spring_beta, when spring_dynamics != 0), control volumes and operators,
 * uniform vertical levels up to Top_altitude. glevel 4..7. */
typedef struct thorx_icogrid thorx_icogrid;
int thorx_grid_build(int glevel, int vlevel, double A, double Top_altitude, int spring_dynamics,
                     double spring_beta, thorx_icogrid** out);
int thorx_grid_info(const thorx_icogrid* g, int* point_num, int* nv, int* nl_region, int* nr,
                    int* spring_iterations);
/* Copies a named array (the Icogrid member names: "point_xyz", "point_xyzq", "maps",
 * "point_local", "pent_ind", "Altitude", "Altitudeh", "lonlat", "areas", "areasT", "areasTr",
 * "nvec", "nvecoa", "nvecti", "nvecte", "div", "grad", "func_r") into `out` (int32 for the
 * first three integer arrays, double otherwise). Returns the element count; out may be NULL. */
long thorx_grid_get(const thorx_icogrid* g, const char* name, void* out);
/* Fills a thorx_grid with pointers into `g` (valid until thorx_grid_free), for thorx_create. */
int thorx_grid_describe(const thorx_icogrid* g, thorx_grid* out);
void thorx_grid_free(thorx_icogrid* g);

#ifdef __cplusplus
}
#endif

#endif /* THORX_H */
