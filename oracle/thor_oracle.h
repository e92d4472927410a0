// CPU restatement of THOR's HE-VI dynamical-core step and Held-Suarez ProfX step.
// TEST INFRASTRUCTURE ONLY: the oracle for parity tests and the timed CPU baseline. The product
// (thor_b200/) never links, loads or calls it.
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

// Physical and numerical switches, as in the reference's SimulationSetup
// (src/headers/simulation_setup.h) and ESP members (src/headers/esp.h).
typedef struct {
    double A, Omega, Gravit, Rd, Cp, P_Ref, timestep, Diffc, DivDampc;
    int    HyDiffOrder;
    // held_suarez: the benchmark forcing, benchmark_types values (0 none, 1 Held-Suarez,
    // 2 tidally locked Earth, 3 shallow hot Jupiter)
    int    DeepModel, NonHydro, GravHeightVar, HyDiff, DivDampP, energy_equation, held_suarez;
    int    glevel;
} oracle_params;

// Grid arrays in the reference layout (src/ESP/grid.cu): maps [nr][(nl+2)^2], point_local [N][6],
// div/grad [N][7][3], areas/nvecoa/nvecti/nvecte [N][6][3], areasTr [N][6], func_r [N][3],
// lonlat [N][2], Altitude [nv], Altitudeh [nv+1], areasT [N]. Copied at creation.
typedef struct {
    int           point_num, nv, nl_region, nr;
    const int*    maps;
    const int*    point_local;
    const double *Altitude, *Altitudeh, *lonlat, *areas, *areasTr, *nvecoa, *nvecti, *nvecte,
        *div, *grad, *func_r;
    const double* areasT; // may be null when oracle_globdiag is not used
} oracle_grid;

// Double-gray radiative transfer module with the insolation it needs (radiative_transfer,
// DualbandGray, src/physics/modules/src/radiative_transfer.cu; Insolation, src/ESP/insolation.cu).
// Lengths in m, angles in degrees (as in the .thr file), spin-up/down in steps (-1 = off).
typedef struct {
    double Tstar, planet_star_dist, radius_star, diff_ang, Tint, albedo;
    double kappa_sw, kappa_lw, kappa_lw_pole, n_sw, n_lw, f_lw;
    double mean_motion, alpha_i, true_long_i, ecc, obliquity, longp;
    int    latf_lw, rt1Dmode, sync_rot, surface;
    int    spinup_start, spinup_stop, spindown_start, spindown_stop;
    int    first_step;
} oracle_rt_params;

void* oracle_new(const oracle_grid* g, const oracle_params* p);
// Enables the RT module in ProfX (between the benchmark forcing and Compute_pressure, as
// src/ESP/profx_driver.cu:405-416). Returns 0, or -1 for an option the restatement lacks.
int oracle_rt(void* h, const oracle_rt_params* rp);
// Enables the dry convective adjustment in ProfX (after the temperature, before the forcing, as
// src/ESP/profx_driver.cu:239-290): up to `iterations` rounds per step; soft != 0 for the soft form.
// A column that exceeds the pass bound makes oracle_step return -3.
int oracle_conv_adj(void* h, int iterations, int soft);
// Rayleigh sponge, implicit form (RayleighSponge with raysp_calc_mode = imp; sponge_layer with its
// zonal means, src/ESP/profx_sponge.cu, run in ProfX after Recompute_W, src/ESP/profx_driver.cu:96-194).
// Same fields as thorx_sponge_params.
typedef struct {
    int    nlat_bins;
    double Ruv_sponge, Rw_sponge, RT_sponge, ns_ray_sponge;
    int    damp_uv_to_mean, damp_w_to_mean, RayleighSpongeT, shrink_sponge, t_shrink, first_step;
    int    raysp_calc_mode; // 0 imp (ProfX), 1 exp1, 2 exp3 (explicit, in the dynamical core)
} oracle_sponge_params;
// Enables the sponge (NULL: off). Returns 0.
int oracle_sponge(void* h, const oracle_sponge_params* sp);
// Zonal means of the last sponge step: vbar [bin][lev][3] (u, v, w), Tbar [bin][lev].
int oracle_sponge_means(void* h, double* vbar, double* Tbar);
// Enables the vertical hyperdiffusion of the dynamical core (VertHyDiff, vertical_diff,
// src/headers/dyn/thor_diff.h:1198-1426) with strength Diffc_v and the given even order (0: off).
int oracle_vert_hydiff(void* h, double Diffc_v, int order);
// Global absorbed shortwave and outgoing longwave of the last RT call (the reference's
// ASR_tot / OLR_tot), compensated sums.
void oracle_rt_totals(void* h, double* asr, double* olr);
// Copy a named field in/out (reference layout). Returns element count, -1 if unknown.
long oracle_set(void* h, const char* name, const double* src);
long oracle_get(void* h, const char* name, double* dst);
// nsteps x (ProfX if do_profx, then Thor if do_thor), as src/esp.cu:1382-1398.
int  oracle_step(void* h, int nsteps, int do_profx, int do_thor);
// Global conserved quantities of the current state (ESP::globdiag, src/ESP/profx_driver.cu:476-560):
// out = {energy, mass, AMx, AMy, AMz, entropy}, each a compensated sum; if abs_out is not null it
// receives the sums of the magnitudes of the per-cell terms (the scale of the rounding error).
int    oracle_globdiag(void* h, double* out, double* abs_out);
// Compensated (Neumaier) sum of x[0..n-1] in index order.
double oracle_sum(const double* x, long n);
// The RT surrogate MLP (thor_b200/csrc/surrogate.cu) in float64 on the CPU, with the GPU's
// bf16 rounding points: inputs, weights and hidden activations rounded to bf16, the GELU
// derivatives rounded to bf16 (as stored for the backward pass), the output gradient and the
// pre-activation gradients rounded to bf16 where the GPU feeds them to a GEMM. GELU in its tanh form.
// Shapes padded as on the GPU: layer l has W[l] [N_l][K_l], b[l] [N_l] (N = H, H, H, Nout;
// K = Kin, H, H, H). x [B][n_in], t [B][nv] standardised; outputs y [B][nv], loss (mean squared
// error), gradients gW[l] (same shape as W[l]) and gb[l]. t, gW, gb may be null (forward only).
int oracle_mlp(int nv, int H, const float* const* W, const float* const* b, const float* x,
               const float* t, int B, double* y, double* loss, double* const* gW,
               double* const* gb);
void oracle_set_threads(int n);
void oracle_free(void* h);

#ifdef __cplusplus
}
#endif
