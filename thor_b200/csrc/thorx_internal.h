// Internal definitions of the thorx dynamical core: device layout and kernel argument blocks.
//
// Device layout (column-index fastest, one plane per level):
//   Np            point_num rounded up to a multiple of 32 (planes start on 256-byte boundaries)
//   cell scalar   x[lev * Np + col]
//   cell vector   x[(k * nv + lev) * Np + col], k = 0,1,2 (three planes per level)
//   interface     x[lev * Np + col], lev = 0..nv
//   div, grad     x[(j * 3 + k) * Np + col], j = 0..6 stencil point (self, pt1..pt6), k = xyz
//   areas, nvec*  x[(j * 3 + k) * Np + col], j = 0..5 triangle / edge
//   areasTr       x[j * Np + col]
//   func_r        x[k * Np + col]
// Columns keep the reference ordering (rhombus r, row j, column i -> r*nl^2 + j*nl + i; the two
// poles last), so that a rhombus row of 16 columns is one 128-byte line of a plane.
//
// Neighbours are explicit per-column tables built from the rhombus maps
// (reference src/headers/kernel_halo_helpers.h:47-128) and, for the poles, from point_local:
//   nb[j * Np + col], j = 0..5  the stencil points pt1..pt6 of the reference kernels
//                               (tile offsets (x,y+1) (x+1,y+1) (x+1,y) (x,y-1) (x-1,y-1)
//                               (x-1,y); at a pentagon pt5 -> (x-1,y); -1 = a hole whose
//                               value is 0, as the reference's zero-filled tile corner)
//   ring[j * Np + col], j = 0..5 the neighbours in the order the Laplacian and the divergence
//                               damping walk them (5 entries at pentagons and poles)
//   cflag[col]                   bit 0: pole, bit 1: five-entry ring
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace thorx {

constexpr int kColAlign = 32;

enum : uint8_t { kPole = 1, kRing5 = 2 };

struct Geometry {
    int            N, Np, nv, nvi;
    // The columns this context computes (a partition of the grid among several contexts or GPUs,
    // thorx_set_partition): 32-column tiles tile0 .. tile0 + ntile - 1, and the columns below
    // col_end; all tiles and N without a partition. The arrays stay whole-grid.
    int            tile0, ntile, col_end;
    const int*     nb;
    const int*     ring;
    const uint8_t* cflag;
    const int*     special;  // the columns with a five-entry ring (pentagons, poles)
    int            nspecial; // 12
    const double*  div;
    const double*  grad;
    const double*  areas;
    const double*  areasTr;
    const double*  nvecoa;
    const double*  nvecti;
    const double*  nvecte;
    const double*  func_r;
    const double*  lat;
    const double*  lon;
    const double*  areasT;
    const double*  Altitude;
    const double*  Altitudeh;
    const double*  Kdh4;
    const double*  Kdhz;
    const double*  Kdv6;     // vertical hyperdiffusion strength per level (null: off)
    const double*  lt; // per-level tables, lt[t * nvi + i] (LevelTable below)
    // Operator weights of the mixed form (stencil_weights_kernel), per column:
    // lapw [7][Np]: hyperdiffusion Laplacian at rscale = 1; entry 0 = the sum of all seven
    //   weights, entries 1..6 = the ring's, so lap = w0 a0 + sum_k wk (ak - a0).
    // dmw [84][Np]: divergence damping, output o (x, y, z) at o * 28: the (Mh) vector part at
    //   rscale = 1, entries 3 k + comp (k = 0 the centre, as the sum over all points, 1..6 the
    //   ring), then 7 entries for (Wh below - Wh above) at points 0..6 at rscale = dz = 1.
    const double*  lapw;
    const float*   dmw;
    const double*  dmw64; // dmw in double, for the FP64 form
    // Shared-memory windows of the momentum kernel, per 32-column tile (whole grid): the first
    // column of each of kWinSpans spans of kWinW columns that hold the tile's stencil points, or
    // -1 for an unused span ([tiles][kWinSpans]).
    const int*     wspan;
};
// The mixed form stores the divergence-damping intermediate divg in FP32 (its values are FP32
// results, so the state is the same bits either way); the planes keep their [3][nv][Np]
// indexing within the FP64-sized allocation. THORX_DIVG_F32=0 keeps FP64 storage.
#ifndef THORX_DIVG_F32
#define THORX_DIVG_F32 1
#endif
constexpr bool kDivgF32 = THORX_DIVG_F32 != 0;

// Columns of a tile (the lanes of a warp); width (columns, even: every box row starts on a
// 16-byte boundary) and number of the window spans.
constexpr int kTileCols = 32, kWinW = 36, kWinSpans = 3;

// Per-level quantities that every column shares, tabulated once on the device at context
// creation with the same expressions the kernels would evaluate per cell (so the values are
// the same bits). "centre" entries are indexed by level 0..nv-1, "interface" entries by
// interface 0..nv (only 1..nv-1 where marked interior).
enum LevelTable : int {
    kLtRscale, // centre: DeepModel ? A / (Alt + A) : 1
    kLtR2cD,   // centre: pow(Alt + A, 2.0)
    kLtDr2dz,  // centre: (pow(Alth[l+1] + A, 3.0) - pow(Alth[l] + A, 3.0)) / 3.0
    kLtGhv,    // centre: pow(A / (A + Alt), 2)
    kLtCIntt,  // centre from its interfaces: (Alt - Alth[l+1]) / (Alth[l] - Alth[l+1])
    kLtCIntl,  // centre from its interfaces: (Alt - Alth[l]) / (Alth[l+1] - Alth[l])
    kLtR2hD,   // interface: pow(Alth + A, 2.0)
    kLtR2hI,   // interface: pow(Alth + A, 2)
    kLtOr2,    // interface: 1 / pow(Alth + A, 2)
    kLtTor3,   // interface: 2 / pow(Alth + A, 3)
    kLtDzp,    // interior interface: 1 / (Alth[i+1] - Alth[i])
    kLtDzh,    // interior interface: 1 / (Alt[i] - Alt[i-1])
    kLtDzm,    // interior interface: 1 / (Alth[i] - Alth[i-1])
    kLtIntl,   // interior interface: (Alt[i] - Alth[i]) * dzp * dzh
    kLtInttm,  // interior interface: -(Alt[i-1] - Alth[i]) * dzm * dzh
    kLtHIntt,  // interior interface from centres: (Alth[i] - Alt[i]) / (Alt[i-1] - Alt[i])
    kLtHIntl,  // interior interface from centres: (Alth[i] - Alt[i-1]) / (Alt[i] - Alt[i-1])
    // reciprocals of level-constant divisors, RN(1 / divisor), for div_rcp (the IEEE quotient)
    kLtRDz,    // centre: 1 / (Alth[l+1] - Alth[l])
    kLtRDr2dz, // centre: 1 / kLtDr2dz
    kLtRDzR2m, // centre: 1 / ((Alth[l+1] - Alth[l]) * kLtR2cD)
    kLtCount
};

struct Phys {
    double A, Omega, Gravit, Rd, Cp, P_Ref, timestep;
    double rP_Ref; // RN(1 / P_Ref), for div_rcp
    int    HyDiffOrder;
    bool   DeepModel, NonHydro, GravHeightVar, HyDiff, DivDampP, energy, held_suarez;
    int    benchmark; // THORX_NO_BENCHMARK .. THORX_SHALLOW_HOT_JUPITER (forcing in ProfX)
    bool   mixed; // momentum-side horizontal stencils computed in FP32 (THORX_MIXED)
    int    conv_adj_iter; // dry convective adjustment: iterations per step (0: off)
    int    vhd_order;     // vertical hyperdiffusion order (VertHyDiffOrder; 0: off)
    bool   conv_soft;     // its soft form (heating into profx_Qheat instead of T and p)
    // every cell's Rd and Cp fields hold exactly Rd and Cp above (kept by the context: set from the
    // host arrays given to thorx_set_field, off for good once a module holds the fields' device
    // pointers); the dynamical-core kernels then use the scalars (rd_at, cp_at)
    bool   uniform_thermo;
};

// Prognostic state (start of large step "x", RK stage "xk", small-step deviation "xs"),
// diagnostics and tendencies. All device pointers in the layout above.
struct State {
    double *Mh, *Mhk, *Mhs;       // 3 planes per level
    double *Rho, *Rhok, *Rhos;
    double *p, *pk, *ps;
    double *Wh, *Whk, *Whs;       // interfaces
    double *W, *Wk;
    double *T, *Rd, *Cp;
    double *h, *hh, *pt, *pth, *gtil, *gtilh;
    double *ep, *eph, *ek, *ekh, *Etotal; // energy equation only
    double *Adv;                  // 3 planes
    double *diff;                 // 6 planes (intermediate hyperdiffusion passes)
    double *diffmh, *diffw, *diffrh, *diffpr;
    double *divg;                 // 3 planes
    double *vrows;                // 4 x (nv+1) planes: tridiagonal rows of the vertical solve,
                                  // then 6 x nv scratch planes of the vertical kernel
    double *SlowMh, *SlowWh, *SlowRho, *Slowp;
    double *Qheat, *dMh, *dWh;    // physics-module coupling (profx_Qheat_d, profx_dMh_d, ...)
    unsigned int* flags;          // device status word (kFlagNaN, kFlagConvAdj)
};

// device-side error flags (State::flags), read by thorx_sync: a NaN in the temperature after
// the physics step; a column whose convective adjustment exceeded its pass bound; a copy into
// shared memory that did not complete within its wait bound
enum : unsigned int { kFlagNaN = 1u, kFlagConvAdj = 2u, kFlagWait = 4u };

// Largest nv the kernels take (levels per thread are unrolled into registers).
int max_levels();
// Dynamic shared memory of the vertical implicit kernel.
size_t vertical_smem_bytes(const Geometry& g);

// Fills the per-level tables lt[kLtCount * (nv+1)] (thor_b200/csrc/dyn_fp64.cu).
void launch_level_tables(const Geometry& g, const Phys& P, double* lt, cudaStream_t st);
void launch_stencil_weights(const Geometry& g, double* lapw, float* dmw, double* dmw64,
                            cudaStream_t st);

// Rayleigh sponge layer at the top of the model (RayleighSponge with raysp_calc_mode = imp,
// reference src/ESP/profx_sponge.cu, called at src/ESP/profx_driver.cu:96-194): winds (and with
// temp, the temperature) above the fractional height ns are relaxed implicitly toward the zonal
// mean of their latitude bin (or toward zero). nlat == 0: off.
struct SpongeStep { // device-resident so that a captured step graph advances it
    long long nstep;  // step number of the next physics step
    double    rv_fac; // strength factor of the current step (shrink_sponge)
};
struct Sponge {
    int           nlat;            // latitude bins of the zonal means
    double        Ruv, Rw, RT, ns; // damping rates [1/s]; bottom of the sponge (z / ztop)
    bool          uv_mean, w_mean; // damp toward the zonal mean (else toward zero)
    bool          temp;            // thermal sponge (RayleighSpongeT)
    bool          shrink;          // shrink_sponge
    int           mode;            // raysp_calc_mode: 0 imp (in ProfX), 1 exp1, 2 exp3 (in Thor)
    long long     t_shrink;        // steps after which the sponge shrinks
    const int*    bin;             // [Np] latitude bin of each column
    const int*    start;           // [nlat + 1] first entry of each bin in members
    const int*    members;         // [N] the columns of each bin, in increasing index
    const double* trig;            // [4][Np] sin(lon), cos(lon) (lon in [0, 2 pi)), sin(lat), cos(lat)
    double*       vbar;            // [3][nlat][nv] zonal means of u, v, w: (k * nlat + bin) * nv + lev
    double*       Tbar;            // [nlat][nv] zonal mean temperature
    SpongeStep*   step;
};

// What the sponge's zonal means read: the step's fields (ProfX: Mh, Rho, Wh interpolated to the
// centres, p) or the RK stage's (explicit modes: Mhk, Rhok, Wk, pk); advance: this call starts a
// step (the step counter and the shrink factor move on).
struct SpongeIn {
    const double *M, *Rho, *W, *Wh, *p, *Rd;
    bool          advance;
};

// Kernel launchers (thor_b200/csrc/dyn_fp64.cu).
// The sponge's zonal means and step factor (sp.nlat > 0 only); the explicit sponge of an RK stage;
// and the per-column trigonometric table they use, once at set-up.
void launch_sponge_means(const Geometry& g, const Phys& P, const Sponge& sp, const SpongeIn& in,
                         cudaStream_t st);
void launch_sponge_explicit(const Geometry& g, const Phys& P, const Sponge& sp, const State& s,
                            cudaStream_t st);
void launch_sponge_trig(const Geometry& g, double* trig, cudaStream_t st);
// ProfX up to the physics modules; with finish, also the pressure update and NaN check, which
// launch_profx_finish does separately when modules run in between. The sponge (sp.nlat > 0) runs
// between Recompute_W and the temperature.
void launch_profx(const Geometry& g, const Phys& P, const Sponge& sp, const State& s, bool finish,
                  cudaStream_t st);
void launch_profx_finish(const Geometry& g, const State& s, cudaStream_t st);
void launch_adv_temp(const Geometry& g, const Phys& P, const State& s, cudaStream_t st);
// Vertical hyperdiffusion of one RK stage, added into diffmh, diffw and diffpr (P.vhd_order > 0).
void launch_vertical_diff(const Geometry& g, const Phys& P, const State& s, cudaStream_t st);
void launch_diffusion(const Geometry& g, const Phys& P, const State& s, int stepnum, bool last,
                      cudaStream_t st);
void launch_divm0(const Geometry& g, const Phys& P, const State& s, bool small_step,
                  cudaStream_t st);
void launch_slow_modes(const Geometry& g, const Phys& P, const State& s, bool update_rk,
                       cudaStream_t st);
void launch_momentum(const Geometry& g, const Phys& P, const State& s, double dt,
                     cudaStream_t st);
// part 0: Prepare_Implicit_Vertical + Vertical_Eq + Density_Pressure_Eqs in one launch; 1 and 2:
// the same split before and after Density_Pressure_Eqs (for a module's fast-mode hook).
void launch_vertical(const Geometry& g, const Phys& P, const State& s, double dt, int part,
                     cudaStream_t st);
// Physics-module arrays that the RK stages update (device_RK_array_manager): at most
// kMaxRkArrays, each `count` doubles.
constexpr int kMaxRkArrays = 10;
struct RkArrays {
    int       n;
    double*   array[kMaxRkArrays];
    double*   arrayk[kMaxRkArrays];
    double*   arrayi[kMaxRkArrays];
    long long count[kMaxRkArrays];
};
// Residual of the last vertical solve's tridiagonal system per column (colmax [N]) and the count
// of interfaces above eps (nbad, added to).
void launch_thomas_residual(const Geometry& g, const State& s, double eps, double* colmax,
                            unsigned int* nbad, cudaStream_t st);
// mode 0: UpdateRK's deviation reset (array = arrayi - arrayk); 1: UpdateRK2 (arrayk += array).
void launch_rk_arrays(const RkArrays& t, int mode, cudaStream_t st);
void launch_update_rk2(const Geometry& g, const Phys& P, const State& s, cudaStream_t st);
// cnt[0..1] += pairs whose reciprocal-based quotient differs from the IEEE one (double, float)
void launch_div_check(long long n, unsigned long long seed, unsigned long long* cnt,
                      cudaStream_t st);

// Double-gray radiative transfer with its insolation (thor_b200/csrc/rt.cu).
struct RtConst { // set once by thorx_rt_enable; angles in radians, lengths in m
    double incflx, diff_ang, Tint, albedo, kappa_sw, kappa_lw, kappa_lw_pole, n_sw, n_lw, f_lw;
    double mean_motion, mean_anomaly_i, true_long_i, ecc, obliquity, alpha_i, longp;
    int    latf_lw, rt1Dmode, sync_rot;
    int    spinup_start, spinup_stop, spindown_start, spindown_stop;
};
struct RtStep { // per-step scalars, device-resident so that a captured step graph advances them
    long long nstep;  // step number of the next physics step
    long long cur;    // step number of the current one
    double    r_orb, sin_decl, cos_decl, alpha; // Insolation state (member defaults 1, 0, 1, 0)
    double    Qheat_scaling;
    int       run;
};
// The surrogate's plain-RT re-check: the columns of every period-th block of 32 (one warp's
// columns in the RT kernels), rotating with the step, so that every column is re-checked once in
// `period` steps and the warps of the other blocks have no re-check to run.
__host__ __device__ inline bool recheck_column(int id, int period, long long step) {
    return (id >> 5) % period == (int)(step % period);
}
struct RtFields { // column-fastest device arrays (interfaces nv+1 planes, tau 2 x nv planes)
    double *phtemp, *thtemp, *ttemp, *dtemp, *qheat, *tau, *fsw_up, *fsw_dn, *flw_up, *flw_dn;
    double *insol, *insol_ann, *ASR, *OLR, *cos_zenith;
    RtStep* step;
    // Surrogate mode (fallback != nullptr): the RT runs only on the columns it re-checks this step
    // (column % period == step % period) and on the columns that have fallen back to it
    // (fallback[col] != 0), leaves dtemp unlimited and does not touch profx_Qheat: the surrogate's
    // combine kernel chooses, limits and couples. nullptr: plain RT on every column.
    const uint8_t* fallback;
    int            period;
};
// Insolation::phy_loop + radiative_transfer::phy_loop (DualbandGray) of one physics step.
void launch_rt(const Geometry& g, const Phys& P, const RtConst& c, const RtFields& f,
               const State& s, cudaStream_t st);

// Global sums (thor_b200/csrc/globdiag.cu).
// Partials the global-diagnostics reduction writes (double2 each, per quantity).
int  globdiag_partials(const Geometry& g);
// Energy, mass, AMx, AMy, AMz, entropy of the current state into out6 (device), using
// 6 * globdiag_partials(g) double2 of scratch at part.
// cells (optional): the six per-cell terms, six cell planes (energy, mass, AMx, AMy, AMz,
// entropy).
void launch_globdiag(const Geometry& g, const Phys& P, const State& s, double2* part, double* out6,
                     cudaStream_t st, double* cells = nullptr);
// Partials a compensated sum of n doubles writes.
long long device_sum_partials(long long n);
// Compensated sum of x[0..n-1] (device) into *out (device), device_sum_partials(n) double2 of
// scratch at part.
void launch_device_sum(const double* x, long long n, double2* part, double* out, cudaStream_t st);
// Largest n of the allocation-free sum, and its scratch on the current device (set up on the
// first call per device): partials at *part, the result at *result.
long long   noalloc_sum_max_n();
cudaError_t noalloc_sum_scratch(double2** part, double** result);

} // namespace thorx
