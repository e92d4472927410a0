// Reference harness: TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own grid builder (src/ESP/grid.cu) and its own dynamical-core and
// physics kernels (src/headers/dyn/*.h, src/headers/phy/profx_*.h, src/ESP/profx_sponge.cu) into
// oracle/_ref/libthor_ref.so, and drives them with the launch sequence of
//   ESP::Thor   src/ESP/thor_driver.cu:70-1466
//   ESP::ProfX  src/ESP/profx_driver.cu:70-474   (the options listed below)
// on one GPU, all FP64, default stream, one launch after another. It is the "reference's own FP64
// CUDA build" against which the CPU restatement (oracle/thor_oracle.cpp) and the product kernels
// are checked, and it is the timing of the reference's CUDA kernels on the same B200.
//
// Only tests/ (and bench.py's reference-CUDA side leg) load this library. The product never does.
//
// Subset mirrored (the configurations this repository measures): entropy or energy equation,
// HyDiff of any even order, DivDampP on/off, DeepModel, NonHydro, GravHeightVar, the Rayleigh
// sponge in its implicit form (raysp_calc_mode = imp), no diffusive sponge, no vertical
// hyperdiffusion, no ultrahot thermodynamics, dry convective adjustment on/off, no increased
// damping, the benchmark forcings (Held-Suarez, tidally locked Earth, shallow hot Jupiter), the
// double-gray RT module.

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "vector_operations.h"

#include "dyn/phy_modules_device.h"

#include "dyn/thor_adv_cor.h"
#include "dyn/thor_auxiliary.h"
// The RK-array registry itself is defined by the reference's src/ESP/phy_modules_device.cu:47-48,
// compiled alongside (relocatable device code). It stays empty in every configuration here.
#include "dyn/thor_diff.h"
#include "dyn/thor_div.h"
#include "dyn/thor_fastmodes.h"
#include "dyn/thor_slowmodes.h"
#include "dyn/thor_vertical_int.h"
#include "phy/dry_conv_adj.h"
#include "phy/profx_auxiliary.h"
#include "phy/profx_globdiag.h"
#include "phy/profx_held_suarez.h"
#include "phy/profx_shallowHJ.h"
#include "phy/profx_sponge.h"
#include "phy/profx_tidalearth.h"
#include "physical_constants.h"
#include "profx_RT.h"
#include "reduction_add.h"

#include "grid.h"
#include "log_writer.h"

FILE* log::pFILE = nullptr;

#define REF_CHECK(call)                                                                           \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            std::fprintf(stderr, "ref harness: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
                         __LINE__);                                                               \
            return -1;                                                                            \
        }                                                                                         \
    } while (0)

// ---------------------------------------------------------------------------------------------
// Grid
// ---------------------------------------------------------------------------------------------
struct RefGrid {
    Icogrid* g = nullptr;
    int      glevel;
    int      nv;
    int      nlat      = 0; // latitude bins of the zonal-mean table (0: built without)
    int      max_count = 0;
};

extern "C" void* ref_grid_new(int    glevel,
                              int    vlevel,
                              double A,
                              double top_altitude,
                              int    sprd,
                              double spring_beta) {
    RefGrid* r   = new RefGrid;
    int max_count = 0;
    // output path without a cached aux_grid_constructs.h5: the grid is always built from scratch
    r->g      = new Icogrid(sprd != 0, spring_beta, glevel, vlevel, 20, A, top_altitude, false,
                       &max_count, false, 2.0, 1000.0, false, 0.7, 1.0, 6.0,
                       std::string("/nonexistent-thorx-ref-cache"));
    r->glevel = glevel;
    r->nv     = vlevel;
    return r;
}

// The same grid with the Rayleigh sponge's zonal-mean table (Icogrid with sponge = true and
// nlat latitude bins, src/ESP/grid.cu:295-299).
extern "C" void* ref_grid_new_sponge(int glevel, int vlevel, double A, double top_altitude,
                                     int sprd, double spring_beta, int nlat) {
    RefGrid* r    = new RefGrid;
    r->max_count  = 0;
    r->g          = new Icogrid(sprd != 0, spring_beta, glevel, vlevel, nlat, A, top_altitude, true,
                       &r->max_count, false, 2.0, 1000.0, false, 0.7, 1.0, 6.0,
                       std::string("/nonexistent-thorx-ref-cache"));
    r->glevel = glevel;
    r->nv     = vlevel;
    r->nlat   = nlat;
    return r;
}

extern "C" void ref_grid_dims(void* h, int* point_num, int* nv, int* nl_region, int* nr) {
    RefGrid* r = (RefGrid*)h;
    *point_num = r->g->point_num;
    *nv        = r->g->nv;
    *nl_region = r->g->nl_region;
    *nr        = r->g->nr;
}

// Copies one named grid array into `out`. Returns the number of elements, or -1 for an unknown
// name. Pass out == nullptr to query the size.
extern "C" long ref_grid_get(void* h, const char* name, void* out) {
    RefGrid* r  = (RefGrid*)h;
    Icogrid* g  = r->g;
    int      N  = g->point_num;
    int      nl = g->nl_region;
    struct Item {
        const void* p;
        long        n;
        size_t      es;
    };
    std::map<std::string, Item> m = {
        {"point_xyz", {g->point_xyz, 3L * N, 8}},
        {"point_xyzq", {g->point_xyzq, 18L * N, 8}},
        {"pent_ind", {g->pent_ind, 12, 4}},
        {"maps", {g->maps, (long)(nl + 2) * (nl + 2) * g->nr, 4}},
        {"point_local", {g->point_local, 6L * N, 4}},
        {"Altitude", {g->Altitude, g->nv, 8}},
        {"Altitudeh", {g->Altitudeh, g->nvi, 8}},
        {"lonlat", {g->lonlat, 2L * N, 8}},
        {"areas", {g->areas, 18L * N, 8}},
        {"areasT", {g->areasT, N, 8}},
        {"areasTr", {g->areasTr, 6L * N, 8}},
        {"nvec", {g->nvec, 18L * N, 8}},
        {"nvecoa", {g->nvecoa, 18L * N, 8}},
        {"nvecti", {g->nvecti, 18L * N, 8}},
        {"nvecte", {g->nvecte, 18L * N, 8}},
        {"mvec", {g->mvec, 18L * N, 8}},
        {"div", {g->div, 21L * N, 8}},
        {"grad", {g->grad, 21L * N, 8}},
        {"curlz", {g->curlz, 21L * N, 8}},
        {"func_r", {g->func_r, 3L * N, 8}},
    };
    if (r->nlat > 0) // [col][3]: latitude bin, members of the bin, slot in the bin
        m["zonal_mean_tab"] = {g->zonal_mean_tab, 3L * N, 4};
    auto it = m.find(name);
    if (it == m.end())
        return -1;
    if (out)
        std::memcpy(out, it->second.p, it->second.n * it->second.es);
    return it->second.n;
}

extern "C" void ref_grid_free(void* h) {
    RefGrid* r = (RefGrid*)h;
    r->g->free_memory();
    delete r->g;
    delete r;
}

// ---------------------------------------------------------------------------------------------
// Simulation state on the device, reference layout ([col][lev], [col][lev][xyz], [col][lev+1])
// ---------------------------------------------------------------------------------------------
struct ref_params {
    double A, Omega, Gravit, Rd, Cp, P_Ref, timestep, Diffc, DivDampc;
    int    HyDiffOrder;
    int    DeepModel, NonHydro, GravHeightVar, HyDiff, DivDampP, energy_equation, held_suarez;
    int    glevel;
};

// Double-gray RT module and its insolation; same field order as oracle_rt_params.
struct ref_rt_params {
    double Tstar, planet_star_dist, radius_star, diff_ang, Tint, albedo;
    double kappa_sw, kappa_lw, kappa_lw_pole, n_sw, n_lw, f_lw;
    double mean_motion, alpha_i, true_long_i, ecc, obliquity, longp;
    int    latf_lw, rt1Dmode, sync_rot, surface;
    int    spinup_start, spinup_stop, spindown_start, spindown_stop;
    int    first_step;
};

// Rayleigh sponge; same field order as oracle_sponge_params.
struct ref_sponge_params {
    int    nlat_bins;
    double Ruv_sponge, Rw_sponge, RT_sponge, ns_ray_sponge;
    int    damp_uv_to_mean, damp_w_to_mean, RayleighSpongeT, shrink_sponge, t_shrink, first_step;
    int    raysp_calc_mode; // 0 IMP, 1 EXP1, 2 EXP3 (define.h:169)
};

struct RefSim {
    ref_params                     p;
    // the probe module (ref_sim_probe): a tracer through the reference's RK array registry
    bool                           probe = false;
    device_RK_array_manager        rkm;
    bool                           sponge = false;
    int                            vhd_order = 0; // vertical hyperdiffusion (VertHyDiff)
    ref_sponge_params              S{};
    int                            max_count = 0, sp_step = 1;
    int*                           zonal_mean_tab_d = nullptr;
    double *                       vbar_h = nullptr, *Tbar_h = nullptr;
    int                            conv_adj_iter = 0; // dry_conv_adj when > 0
    bool                           conv_soft     = false;
    bool                           rt = false;
    ref_rt_params                  R{};
    double incflx = 0, mean_motion = 0, mean_anomaly_i = 0, true_long_i = 0, ecc = 0,
           obliquity = 0, alpha_i = 0, longp = 0;
    double r_orb = 1, sin_decl = 0, cos_decl = 1, alpha = 0; // Insolation member defaults
    int    nstep = 1;
    double ASR_tot = 0, OLR_tot = 0;
    int                            N, nv, nvi, nl_region, nr;
    std::map<std::string, double*> f;    // device fields
    std::map<std::string, long>    size; // element counts
    int*                           maps_d        = nullptr;
    int*                           point_local_d = nullptr;
    unsigned int*                  diag_flag_d   = nullptr;
    diag_data*                     diag_data_d   = nullptr;
    double*                        Altitude_h    = nullptr;
};

static int sim_alloc(RefSim* s, const char* name, long n) {
    double* d = nullptr;
    REF_CHECK(cudaMalloc(&d, n * sizeof(double)));
    REF_CHECK(cudaMemset(d, 0, n * sizeof(double)));
    s->f[name]    = d;
    s->size[name] = n;
    return 0;
}

// Grid arrays handed over directly (reference layouts), e.g. from a grid built elsewhere.
struct ref_grid_view {
    int           point_num, nv, nl_region, nr;
    const int*    maps;
    const int*    point_local;
    const double *Altitude, *Altitudeh, *lonlat, *areas, *areasT, *areasTr, *nvecoa, *nvecti,
        *nvecte, *div, *grad, *func_r;
};

static void* sim_new(const ref_grid_view* g, const ref_params* p);

extern "C" void* ref_sim_new(void* gh, const ref_params* p) {
    Icogrid*      ig = ((RefGrid*)gh)->g;
    ref_grid_view v{ig->point_num, ig->nv,         ig->nl_region, ig->nr,      ig->maps,
                    ig->point_local, ig->Altitude, ig->Altitudeh, ig->lonlat,  ig->areas,
                    ig->areasT,     ig->areasTr,   ig->nvecoa,    ig->nvecti,  ig->nvecte,
                    ig->div,        ig->grad,      ig->func_r};
    return sim_new(&v, p);
}

extern "C" void* ref_sim_new_view(const ref_grid_view* g, const ref_params* p) {
    return sim_new(g, p);
}

static void* sim_new(const ref_grid_view* g, const ref_params* p) {
    RefSim* s    = new RefSim;
    s->p         = *p;
    s->N         = g->point_num;
    s->nv        = g->nv;
    s->nvi       = g->nv + 1;
    s->nl_region = g->nl_region;
    s->nr        = g->nr;
    long N = s->N, nv = s->nv, nvi = s->nvi;

    const char* cell1[] = {"Rho", "Rhok", "Rhos", "pressure", "pressurek", "pressures",
                           "temperature", "W", "Wk", "Ws", "h", "pt", "gtil", "SlowRho",
                           "Slowpressure", "Sp", "Sd", "diffw", "diffrh", "diffpr", "diffwv",
                           "diffrv", "diffprv", "epotential", "ekinetic", "Etotal", "Cp", "Rd",
                           "profx_Qheat", "profx_dW", "Mass", "AngMomx", "AngMomy", "AngMomz",
                           "Entropy"};
    const char* cell3[] = {"Mh", "Mhk", "Mhs", "Adv", "v", "SlowMh", "DivM", "divg_Mh",
                           "diffmh", "diffmv", "profx_dMh"};
    const char* iface[] = {"Wh", "Whk", "Whs", "hh", "pth", "gtilh", "SlowWh", "epotentialh",
                           "ekinetich", "profx_dWh"};
    const char* cell6[] = {"diff", "diff_sponge", "diff2", "boundary_flux"};
    for (auto n : cell1)
        if (sim_alloc(s, n, N * nv))
            return nullptr;
    for (auto n : cell3)
        if (sim_alloc(s, n, 3 * N * nv))
            return nullptr;
    for (auto n : iface)
        if (sim_alloc(s, n, N * nvi))
            return nullptr;
    for (auto n : cell6)
        if (sim_alloc(s, n, 6 * N * nv))
            return nullptr;
    for (auto n : {"Kdh4", "Kdhz", "Kdh2"})
        if (sim_alloc(s, n, nv))
            return nullptr;

    // geometry (reference layout, copied as built by Icogrid)
    struct G {
        const char*   n;
        const double* h;
        long          c;
    } geo[] = {{"Altitude", g->Altitude, nv},  {"Altitudeh", g->Altitudeh, nvi},
               {"lonlat", g->lonlat, 2 * N},   {"areas", g->areas, 18 * N},
               {"areasT", g->areasT, N},       {"areasTr", g->areasTr, 6 * N},
               {"nvecoa", g->nvecoa, 18 * N},  {"nvecti", g->nvecti, 18 * N},
               {"nvecte", g->nvecte, 18 * N},  {"div", g->div, 21 * N},
               {"grad", g->grad, 21 * N},      {"func_r", g->func_r, 3 * N}};
    for (auto& x : geo) {
        if (sim_alloc(s, x.n, x.c))
            return nullptr;
        if (cudaMemcpy(s->f[x.n], x.h, x.c * 8, cudaMemcpyHostToDevice) != cudaSuccess)
            return nullptr;
    }
    long nmaps = (long)(s->nl_region + 2) * (s->nl_region + 2) * s->nr;
    if (cudaMalloc(&s->maps_d, nmaps * sizeof(int)) != cudaSuccess)
        return nullptr;
    cudaMemcpy(s->maps_d, g->maps, nmaps * sizeof(int), cudaMemcpyHostToDevice);
    if (cudaMalloc(&s->point_local_d, 6 * N * sizeof(int)) != cudaSuccess)
        return nullptr;
    cudaMemcpy(s->point_local_d, g->point_local, 6 * N * sizeof(int), cudaMemcpyHostToDevice);
    cudaMalloc(&s->diag_flag_d, sizeof(unsigned int));
    cudaMemset(s->diag_flag_d, 0, sizeof(unsigned int));
    cudaMalloc(&s->diag_data_d, N * nvi * sizeof(diag_data));

    s->Altitude_h = new double[nv];
    std::memcpy(s->Altitude_h, g->Altitude, nv * 8);

    // Hyperdiffusion and divergence-damping strengths (src/ESP/esp_initial.cu:1292-1335,
    // no diffusive sponge).
    std::vector<double> kdh4(nv), kdhz(nv);
    for (int lev = 0; lev < nv; lev++) {
        double dbar = sqrt(2 * M_PI / 5) * p->A / (pow(2, p->glevel));
        kdh4[lev]   = (p->Diffc) * pow(dbar, 1.0 * p->HyDiffOrder) / p->timestep;
        kdhz[lev]   = (p->DivDampc) * pow(dbar, 4.) / p->timestep;
    }
    cudaMemcpy(s->f["Kdh4"], kdh4.data(), nv * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(s->f["Kdhz"], kdhz.data(), nv * 8, cudaMemcpyHostToDevice);
    int zero = 0;
    cudaMemcpyToSymbol(num_dynamical_arrays, &zero, sizeof(int));
    if (cudaDeviceSynchronize() != cudaSuccess)
        return nullptr;
    return s;
}

extern "C" long ref_sim_set(void* h, const char* name, const double* host) {
    RefSim* s  = (RefSim*)h;
    auto    it = s->f.find(name);
    if (it == s->f.end())
        return -1;
    long n = s->size[name];
    if (cudaMemcpy(it->second, host, n * 8, cudaMemcpyHostToDevice) != cudaSuccess)
        return -2;
    return n;
}

extern "C" long ref_sim_get(void* h, const char* name, double* host) {
    RefSim* s  = (RefSim*)h;
    auto    it = s->f.find(name);
    if (it == s->f.end())
        return -1;
    long n = s->size[name];
    if (host && cudaMemcpy(host, it->second, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return -2;
    return n;
}

// One ProfX call, Held-Suarez branch (src/ESP/profx_driver.cu:70-474).

// ---------------------------------------------------------------------------------------------
// RT module. rtm_dual_band and annual_insol are the reference's own kernels
// (src/physics/modules/inc/profx_RT.h); the argument list and the host logic around them follow
// radiative_transfer::phy_loop (src/physics/modules/src/radiative_transfer.cu:769-1105) and
// RTSetup (:1393-1437). The orbit and zenith arithmetic is the reference's own, compiled from
// src/ESP/insolation.cu (oracle/Makefile builds it with a copy of its header whose storage include
// resolves to the shim): the free functions solve_kepler, calc_r_orb, ecc2true_anomaly,
// true2ecc_anomaly and the kernel compute_cos_zenith_angles (calc_zenith, insolation.cu:128-207).
// Only Insolation::update_spin_orbit (insolation.cu:514-529), a private member of a class whose
// object needs a whole ESP, is restated here, on those functions.
// ---------------------------------------------------------------------------------------------
double solve_kepler(double mean_anomaly, double ecc);
double calc_r_orb(double ecc_anomaly, double ecc);
double ecc2true_anomaly(double ecc_anomaly, double ecc);
double true2ecc_anomaly(double true_anomaly, double ecc);
__global__ void compute_cos_zenith_angles(double* cos_zenith_angles, double* lonlat_d, double alpha,
                                          double alpha_i, double sin_decl, double cos_decl,
                                          double ecc, double obliquity, bool sync_rot,
                                          int num_points);
static void h_update_spin_orbit(RefSim* s, double time) { // insolation.cu:514-529
    double M         = fmod((s->mean_motion * time + s->mean_anomaly_i), (2 * M_PI));
    double E         = fmod(solve_kepler(M, s->ecc), (2 * M_PI));
    s->r_orb         = calc_r_orb(E, s->ecc);
    double true_long = fmod((ecc2true_anomaly(E, s->ecc) + s->longp), (2 * M_PI));
    s->sin_decl      = sin(s->obliquity) * sin(true_long);
    s->cos_decl      = sqrt(1.0 - s->sin_decl * s->sin_decl);
    s->alpha         = -s->p.Omega * time + true_long - s->true_long_i + s->alpha_i;
}

extern "C" int ref_sim_rt(void* h, const ref_rt_params* rp) {
    RefSim* s = (RefSim*)h;
    if (rp->surface || s->p.GravHeightVar)
        return -1;
    s->R   = *rp;
    s->rt  = true;
    long N = s->N, nv = s->nv, nvi = s->nvi;
    for (auto n : {"flw_up", "flw_dn", "fsw_up", "fsw_dn", "phtemp", "thtemp"})
        if (sim_alloc(s, n, N * nvi))
            return -2;
    if (sim_alloc(s, "tau", N * nv * 2))
        return -2;
    for (auto n : {"ttemp", "dtemp", "DG_Qheat"})
        if (sim_alloc(s, n, N * nv))
            return -2;
    for (auto n : {"insol", "insol_ann", "ASR", "OLR", "cos_zenith", "surf_flux", "Tsurface",
                   "dTsurf_dt"})
        if (sim_alloc(s, n, N))
            return -2;
    double resc_flx   = pow(rp->radius_star / rp->planet_star_dist, 2.0);
    s->incflx         = resc_flx * SIGMA_SB_th * rp->Tstar * rp->Tstar * rp->Tstar * rp->Tstar;
    s->mean_motion    = rp->sync_rot ? s->p.Omega : rp->mean_motion;
    s->true_long_i    = rp->true_long_i * M_PI / 180.0;
    s->longp          = rp->longp * M_PI / 180.0;
    s->ecc            = rp->ecc;
    double f_i        = fmod(s->true_long_i - s->longp, (2 * M_PI));
    double E_i        = true2ecc_anomaly(f_i, s->ecc);
    s->mean_anomaly_i = fmod(E_i - s->ecc * sin(E_i), (2 * M_PI));
    s->alpha_i        = rp->alpha_i * M_PI / 180.0;
    s->obliquity      = rp->obliquity * M_PI / 180.0;
    s->nstep          = rp->first_step;
    return 0;
}

// The dry convective adjustment in ProfX (sim.conv_adj, conv_adj_type hourdin): the reference's
// dry_conv_adj kernel as profx_driver.cu:239-290 launches it.
extern "C" int ref_sim_conv_adj(void* h, int iterations, int soft) {
    RefSim* s = (RefSim*)h;
    if (!s->f.count("pressureh") && sim_alloc(s, "pressureh", (long)s->N * s->nvi))
        return -2;
    s->conv_adj_iter = iterations;
    s->conv_soft     = soft != 0;
    return 0;
}

// The Rayleigh sponge in ProfX (sim.RayleighSponge with raysp_calc_mode = imp), launched as
// profx_driver.cu:96-194 launches it, with the grid's zonal-mean table (gh from
// ref_grid_new_sponge with the same nlat_bins).
// Vertical hyperdiffusion (sim.VertHyDiff): Kdv6 as src/ESP/esp_initial.cu:1327-1335, and the
// reference's scratch diff2 of 6 (nv + 2) planes per column that vertical_diff needs.
extern "C" int ref_sim_vert_hydiff(void* h, double Diffc_v, int order) {
    RefSim*    s = (RefSim*)h;
    const long N = s->N, nv = s->nv;
    if (!s->f.count("Kdv6") && sim_alloc(s, "Kdv6", nv))
        return -2;
    if (!s->f.count("diff2v") && sim_alloc(s, "diff2v", 6 * N * (nv + 2)))
        return -2;
    std::vector<double> k(nv);
    std::vector<double> alth(nv + 1);
    REF_CHECK(cudaMemcpy(alth.data(), s->f["Altitudeh"], (nv + 1) * 8, cudaMemcpyDeviceToHost));
    for (int lev = 0; lev < nv; lev++) {
        double dz = alth[lev + 1] - alth[lev];
        k[lev]    = Diffc_v * pow(dz, 1.0 * order) / s->p.timestep;
    }
    REF_CHECK(cudaMemcpy(s->f["Kdv6"], k.data(), nv * 8, cudaMemcpyHostToDevice));
    s->vhd_order = order;
    return 0;
}

extern "C" int ref_sim_sponge(void* h, void* gh, const ref_sponge_params* sp) {
    RefSim*  s = (RefSim*)h;
    RefGrid* r = (RefGrid*)gh;
    if (!r->g->zonal_mean_tab || r->nlat != sp->nlat_bins || r->g->point_num != s->N)
        return -1;
    s->S         = *sp;
    s->sponge    = true;
    s->max_count = r->max_count;
    s->sp_step   = sp->first_step;
    const long N = s->N, nv = s->nv, nlat = sp->nlat_bins, mc = r->max_count;
    REF_CHECK(cudaMalloc(&s->zonal_mean_tab_d, 3 * N * sizeof(int)));
    REF_CHECK(cudaMemcpy(s->zonal_mean_tab_d, r->g->zonal_mean_tab, 3 * N * sizeof(int),
                         cudaMemcpyHostToDevice));
    for (auto n : {"utmp", "vtmp", "wtmp", "Ttmp"})
        if (sim_alloc(s, n, nlat * nv * mc))
            return -2;
    if (sim_alloc(s, "vbar", 3 * nlat * nv) || sim_alloc(s, "Tbar", nlat * nv))
        return -2;
    s->vbar_h = new double[3 * nlat * nv]();
    s->Tbar_h = new double[nlat * nv]();
    return 0;
}

extern "C" void ref_sim_sponge_means(void* h, double* vbar, double* Tbar) {
    RefSim*    s = (RefSim*)h;
    const long n = (long)s->S.nlat_bins * s->nv;
    if (vbar)
        std::memcpy(vbar, s->vbar_h, 3 * n * sizeof(double));
    if (Tbar)
        std::memcpy(Tbar, s->Tbar_h, n * sizeof(double));
}

// The explicit sponge of one RK stage (raysp_calc_mode exp1 / exp3), thor_driver.cu:749-866.
static int ref_sponge_explicit(RefSim* s, int rk) {
    auto&      F   = s->f;
    const int  NTH = 256;
    const int  N = s->N, nv = s->nv, nvi = s->nvi, nlat_bins = s->S.nlat_bins;
    const int  max_count = s->max_count;
    const bool uvm = s->S.damp_uv_to_mean != 0, wm = s->S.damp_w_to_mean != 0;
    dim3       NB((N / NTH) + 1, nv, 1);
    dim3       NBRT((N / NTH) + 1, 1, 1);
    REF_CHECK(cudaMemset(F["profx_dMh"], 0, sizeof(double) * 3 * N * nv));
    REF_CHECK(cudaMemset(F["profx_dWh"], 0, sizeof(double) * N * nvi));
    REF_CHECK(cudaMemset(F["profx_dW"], 0, sizeof(double) * N * nv));
    if (rk == 0 || s->S.raysp_calc_mode == 2) {
        if (uvm) {
            REF_CHECK(cudaMemset(F["utmp"], 0, sizeof(double) * nlat_bins * nv * max_count));
            REF_CHECK(cudaMemset(F["vtmp"], 0, sizeof(double) * nlat_bins * nv * max_count));
            zonal_uv<<<NB, NTH>>>(F["Mhk"], F["Rhok"], s->zonal_mean_tab_d, F["lonlat"], N,
                                  F["utmp"], F["vtmp"], max_count);
            REF_CHECK(cudaDeviceSynchronize());
        }
        if (wm) {
            REF_CHECK(cudaMemset(F["wtmp"], 0, sizeof(double) * nlat_bins * nv * max_count));
            zonal_w<<<NB, NTH>>>(F["Wk"], F["Rhok"], s->zonal_mean_tab_d, N, F["wtmp"], max_count);
            REF_CHECK(cudaDeviceSynchronize());
        }
        if (uvm) {
            gpu_sum_on_device_sponge<1024>(F["utmp"], max_count, s->vbar_h, nv, nlat_bins, 0);
            gpu_sum_on_device_sponge<1024>(F["vtmp"], max_count, s->vbar_h, nv, nlat_bins, 1);
        }
        if (wm)
            gpu_sum_on_device_sponge<1024>(F["wtmp"], max_count, s->vbar_h, nv, nlat_bins, 2);
        if (uvm || wm) {
            REF_CHECK(cudaMemset(F["vbar"], 0, sizeof(double) * 3 * nlat_bins * nv));
            REF_CHECK(cudaMemcpy(F["vbar"], s->vbar_h, 3 * nlat_bins * nv * sizeof(double),
                                 cudaMemcpyHostToDevice));
        }
        if (s->S.RayleighSpongeT) {
            zonal_temp<<<NB, NTH>>>(F["pressurek"], F["Rhok"], F["Tbar"], s->zonal_mean_tab_d,
                                    F["lonlat"], N, F["Ttmp"], F["Rd"], max_count);
            REF_CHECK(cudaDeviceSynchronize());
            for (int ilat = 0; ilat < nlat_bins; ilat++)
                for (int lev = 0; lev < nv; lev++)
                    s->Tbar_h[ilat * nv + lev] = gpu_sum_on_device<1024>(
                        &(F["Ttmp"][ilat * nv * max_count + lev * max_count]), max_count);
            REF_CHECK(cudaMemcpy(F["Tbar"], s->Tbar_h, nlat_bins * nv * sizeof(double),
                                 cudaMemcpyHostToDevice));
        }
    }
    const double timestep = s->p.timestep;
    const int    current_step = s->sp_step;
    double       Rv_fac = 1;
    if (s->S.shrink_sponge) {
        if (current_step * timestep >= s->S.t_shrink * timestep) {
            double shrink_scale = timestep * 1000;
            Rv_fac = exp(-(current_step * timestep - s->S.t_shrink * timestep) / shrink_scale);
        }
    }
    sponge_layer<<<NBRT, NTH>>>(F["Mhk"], F["Rhok"], F["Wk"], F["Whk"], F["pressurek"], F["vbar"],
                                F["Tbar"], s->zonal_mean_tab_d, F["lonlat"], F["Altitude"],
                                F["Altitudeh"], s->S.Ruv_sponge, s->S.Rw_sponge, s->S.RT_sponge,
                                Rv_fac, s->S.ns_ray_sponge, uvm, wm, false, timestep, F["Rd"],
                                nlat_bins, N, nv, s->S.RayleighSpongeT != 0, F["profx_dMh"],
                                F["profx_dWh"], F["profx_dW"], F["profx_Qheat"]);
    REF_CHECK(cudaDeviceSynchronize());
    return 0;
}

static int ref_sponge_step(RefSim* s) {
    auto&      F   = s->f;
    const int  NTH = 256;
    const int  N = s->N, nv = s->nv, nlat_bins = s->S.nlat_bins, max_count = s->max_count;
    const bool uvm = s->S.damp_uv_to_mean != 0, wm = s->S.damp_w_to_mean != 0;
    dim3       NB((N / NTH) + 1, nv, 1);
    dim3       NBRT((N / NTH) + 1, 1, 1);
    if (uvm) {
        REF_CHECK(cudaMemset(F["utmp"], 0, sizeof(double) * nlat_bins * nv * max_count));
        REF_CHECK(cudaMemset(F["vtmp"], 0, sizeof(double) * nlat_bins * nv * max_count));
        zonal_uv<<<NB, NTH>>>(F["Mh"], F["Rho"], s->zonal_mean_tab_d, F["lonlat"], N, F["utmp"],
                              F["vtmp"], max_count);
        REF_CHECK(cudaDeviceSynchronize());
    }
    if (wm) {
        REF_CHECK(cudaMemset(F["wtmp"], 0, sizeof(double) * nlat_bins * nv * max_count));
        zonal_w<<<NB, NTH>>>(F["W"], F["Rho"], s->zonal_mean_tab_d, N, F["wtmp"], max_count);
        REF_CHECK(cudaDeviceSynchronize());
    }
    if (uvm) {
        gpu_sum_on_device_sponge<1024>(F["utmp"], max_count, s->vbar_h, nv, nlat_bins, 0);
        gpu_sum_on_device_sponge<1024>(F["vtmp"], max_count, s->vbar_h, nv, nlat_bins, 1);
    }
    if (wm)
        gpu_sum_on_device_sponge<1024>(F["wtmp"], max_count, s->vbar_h, nv, nlat_bins, 2);
    if (uvm || wm) {
        REF_CHECK(cudaMemset(F["vbar"], 0, sizeof(double) * 3 * nlat_bins * nv));
        REF_CHECK(cudaMemcpy(F["vbar"], s->vbar_h, 3 * nlat_bins * nv * sizeof(double),
                             cudaMemcpyHostToDevice));
    }
    if (s->S.RayleighSpongeT) {
        zonal_temp<<<NB, NTH>>>(F["pressure"], F["Rho"], F["Tbar"], s->zonal_mean_tab_d,
                                F["lonlat"], N, F["Ttmp"], F["Rd"], max_count);
        REF_CHECK(cudaDeviceSynchronize());
        for (int ilat = 0; ilat < nlat_bins; ilat++)
            for (int lev = 0; lev < nv; lev++)
                s->Tbar_h[ilat * nv + lev] = gpu_sum_on_device<1024>(
                    &(F["Ttmp"][ilat * nv * max_count + lev * max_count]), max_count);
        REF_CHECK(cudaMemcpy(F["Tbar"], s->Tbar_h, nlat_bins * nv * sizeof(double),
                             cudaMemcpyHostToDevice));
    }
    const double timestep = s->p.timestep;
    const int    current_step = s->sp_step++;
    double       Rv_fac = 1;
    if (s->S.shrink_sponge) {
        if (current_step * timestep >= s->S.t_shrink * timestep) {
            double shrink_scale = timestep * 1000;
            Rv_fac = exp(-(current_step * timestep - s->S.t_shrink * timestep) / shrink_scale);
        }
    }
    sponge_layer<<<NBRT, NTH>>>(F["Mh"], F["Rho"], F["W"], F["Wh"], F["pressure"], F["vbar"],
                                F["Tbar"], s->zonal_mean_tab_d, F["lonlat"], F["Altitude"],
                                F["Altitudeh"], s->S.Ruv_sponge, s->S.Rw_sponge, s->S.RT_sponge,
                                Rv_fac, s->S.ns_ray_sponge, uvm, wm, true, timestep, F["Rd"],
                                nlat_bins, N, nv, s->S.RayleighSpongeT != 0, F["profx_dMh"],
                                F["profx_dWh"], F["profx_dW"], F["profx_Qheat"]);
    REF_CHECK(cudaDeviceSynchronize());
    return 0;
}

// ---------------------------------------------------------------------------------------------
// Probe module: a physics module of this harness (not of the reference), called at the points
// where ESP calls the module manager (src/ESP/thor_driver.cu:116,641,1290,1465;
// src/ESP/profx_driver.cu:405-416). It carries a two-component tracer through the reference's own
// RK array registry (device_RK_array_manager, consumed by UpdateRK/UpdateRK2) with a tendency of 1
// per second, snapshots Rhos and Whs at the fast-mode hook of the last small step, and adds 0.5 K
// to the temperature in phy_loop. The product's test module does the same through its C ABI.
// ---------------------------------------------------------------------------------------------
__global__ void probe_add(double* x, long n, double v) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        x[i] += v;
}

extern "C" int ref_sim_probe(void* h) {
    RefSim*    s = (RefSim*)h;
    const long N = s->N, nv = s->nv;
    for (auto n : {"tracer", "tracerk", "tracers"})
        if (sim_alloc(s, n, 2 * N * nv))
            return -2;
    if (sim_alloc(s, "snap_Rhos", N * nv) || sim_alloc(s, "snap_Whs", N * s->nvi))
        return -2;
    if (!s->rkm.register_array(s->f["tracers"], s->f["tracerk"], s->f["tracer"], 2))
        return -1;
    s->probe = true;
    return 0;
}

static void probe_phy_loop(RefSim* s) {
    probe_add<<<256, 256>>>(s->f["temperature"], (long)s->N * s->nv, 0.5);
}
static void probe_init(RefSim* s) {
    const long n = 2L * s->N * s->nv;
    cudaMemcpy(s->f["tracerk"], s->f["tracer"], n * 8, cudaMemcpyDeviceToDevice);
    cudaMemset(s->f["tracers"], 0, n * 8);
}
static void probe_fast(RefSim* s, int rk, int ns, int ns_it, double times) {
    probe_add<<<256, 256>>>(s->f["tracers"], 2L * s->N * s->nv, times);
    if (rk == 2 && ns == ns_it - 1) {
        cudaMemcpy(s->f["snap_Rhos"], s->f["Rhos"], (size_t)s->N * s->nv * 8,
                   cudaMemcpyDeviceToDevice);
        cudaMemcpy(s->f["snap_Whs"], s->f["Whs"], (size_t)s->N * s->nvi * 8,
                   cudaMemcpyDeviceToDevice);
    }
    cudaDeviceSynchronize();
}
static void probe_end(RefSim* s) {
    cudaMemcpy(s->f["tracer"], s->f["tracerk"], 2L * s->N * s->nv * 8, cudaMemcpyDeviceToDevice);
}

extern "C" void ref_sim_rt_totals(void* h, double* asr, double* olr) {
    RefSim* s = (RefSim*)h;
    *asr      = s->ASR_tot;
    *olr      = s->OLR_tot;
}

// Insolation::phy_loop + radiative_transfer::phy_loop (DualbandGray), in ProfX order.
static int ref_rt_step(RefSim* s) {
    auto&        F = s->f;
    const int    NTH = 256, N = s->N, nv = s->nv, nvi = s->nvi, nstep = s->nstep;
    const double dt = s->p.timestep;
    dim3         NBRT((N / NTH) + 1, 1, 1);
    if (s->R.sync_rot) {
        if (s->ecc > 1e-10)
            h_update_spin_orbit(s, nstep * dt);
    }
    else
        h_update_spin_orbit(s, nstep * dt);
    compute_cos_zenith_angles<<<(N / NTH) + 1, NTH>>>(F["cos_zenith"], F["lonlat"], s->alpha,
                                                      s->alpha_i, s->sin_decl, s->cos_decl, s->ecc,
                                                      s->obliquity, s->R.sync_rot, N);
    REF_CHECK(cudaDeviceSynchronize());
    bool   run           = true;
    double Qheat_scaling = 1.0;
    const ref_rt_params& R = s->R;
    if (R.spinup_start > -1 && R.spinup_stop > -1) {
        if (nstep < R.spinup_start) {
            run           = false;
            Qheat_scaling = 0.0;
        }
        else if ((nstep >= R.spinup_start) && (nstep <= R.spinup_stop)) {
            double x = (double)(nstep - R.spinup_start) / (double)(R.spinup_stop - R.spinup_start);
            Qheat_scaling = (1 + sin(M_PI * x - M_PI / 2.0)) / 2.0;
            run           = true;
        }
    }
    if (R.spindown_start > -1 && R.spindown_stop > -1) {
        if ((nstep >= R.spindown_start) && (nstep <= R.spindown_stop)) {
            double x = (double)(nstep - R.spindown_start) / (double)(R.spindown_stop - R.spindown_start);
            Qheat_scaling = 1.0 - (1 + sin(M_PI * x - M_PI / 2.0)) / 2.0;
            run           = true;
        }
        else if (nstep >= R.spindown_stop) {
            run           = false;
            Qheat_scaling = 0.0;
        }
    }
    if (run) {
        rtm_dual_band<<<NBRT, NTH>>>(
            F["pressure"], F["Rho"], F["temperature"], F["flw_up"], F["flw_dn"], F["fsw_up"],
            F["fsw_dn"], F["tau"], s->p.Gravit, F["Cp"], F["lonlat"], F["Altitude"],
            F["Altitudeh"], F["phtemp"], F["dtemp"], F["ttemp"], F["thtemp"], dt, R.Tstar,
            R.planet_star_dist, R.radius_star, R.diff_ang, R.Tint, R.albedo, R.kappa_sw,
            R.kappa_lw, R.latf_lw, R.kappa_lw_pole, R.n_sw, R.n_lw, R.f_lw, s->incflx, s->p.P_Ref,
            N, nv, nvi, s->p.A, s->r_orb, F["cos_zenith"], F["insol"], false, 1e7, F["Tsurface"],
            F["dTsurf_dt"], F["surf_flux"], F["areasT"], F["ASR"], F["OLR"], F["profx_Qheat"],
            F["DG_Qheat"], F["Rd"], Qheat_scaling, false, R.rt1Dmode, s->p.DeepModel,
            s->p.GravHeightVar);
        REF_CHECK(cudaGetLastError());
        s->ASR_tot = gpu_sum_on_device<1024>(F["ASR"], N);
        s->OLR_tot = gpu_sum_on_device<1024>(F["OLR"], N);
        if (nstep * dt < (2 * M_PI / s->mean_motion))
            annual_insol<<<NBRT, NTH>>>(F["insol_ann"], F["insol"], nstep, N);
    }
    REF_CHECK(cudaDeviceSynchronize());
    s->nstep++;
    return 0;
}

static int ref_profx(RefSim* s) {
    auto&     F   = s->f;
    const int NTH = 256;
    int       N = s->N, nv = s->nv;
    dim3      NB((N / NTH) + 1, nv, 1);
    REF_CHECK(cudaMemset(F["profx_Qheat"], 0, sizeof(double) * N * nv));
    Recompute_W<<<NB, NTH>>>(F["W"], F["Wh"], F["Altitude"], F["Altitudeh"], N);
    REF_CHECK(cudaDeviceSynchronize());
    if (s->sponge && s->S.raysp_calc_mode == 0 && ref_sponge_step(s))
        return -1;
    Compute_temperature<<<NB, NTH>>>(F["temperature"], F["pt"], F["pressure"], F["Rho"],
                                     s->p.P_Ref, F["Rd"], F["Cp"], N, true);
    REF_CHECK(cudaDeviceSynchronize());
    if (s->conv_adj_iter > 0) {
        const int NBRT = (N / NTH) + 1;
        dry_conv_adj<<<NBRT, NTH>>>(F["pressure"], F["pressureh"], F["temperature"],
                                    F["profx_Qheat"], F["pt"], F["Rho"], F["Cp"], F["Rd"],
                                    s->p.Gravit, F["Altitude"], F["Altitudeh"], s->p.timestep,
                                    s->p.A, s->conv_adj_iter, s->conv_soft, N, nv,
                                    s->p.GravHeightVar);
        REF_CHECK(cudaDeviceSynchronize());
    }
    // benchmark forcing, profx_driver.cu:300-360 (held_suarez carries the benchmark_types value)
    if (s->p.held_suarez == 1) {
        held_suarez<<<NB, NTH>>>(F["Mh"], F["pressure"], F["Rho"], F["temperature"], s->p.Gravit,
                                 s->p.Cp, s->p.Rd, F["Altitude"], F["Altitudeh"], F["lonlat"],
                                 s->p.timestep, N);
        REF_CHECK(cudaDeviceSynchronize());
    }
    else if (s->p.held_suarez == 2) {
        tidalearth<<<NB, NTH>>>(F["Mh"], F["pressure"], F["Rho"], F["temperature"], s->p.Gravit,
                                s->p.Cp, s->p.Rd, F["Altitude"], F["Altitudeh"], F["lonlat"],
                                s->p.timestep, N);
        REF_CHECK(cudaDeviceSynchronize());
    }
    else if (s->p.held_suarez == 3) {
        shallowHJ<<<NB, NTH>>>(F["Mh"], F["pressure"], F["Rho"], F["temperature"], s->p.Gravit,
                               s->p.Cp, s->p.Rd, F["Altitude"], F["Altitudeh"], F["lonlat"],
                               s->p.timestep, N);
        REF_CHECK(cudaDeviceSynchronize());
    }
    if (s->rt && ref_rt_step(s))
        return -1;
    if (s->probe) {
        probe_phy_loop(s);
        REF_CHECK(cudaDeviceSynchronize());
    }
    Compute_pressure<<<NB, NTH>>>(F["pressure"], F["temperature"], F["Rho"], F["Rd"], N);
    REF_CHECK(cudaDeviceSynchronize());
    return 0;
}

// One ESP::Thor call (src/ESP/thor_driver.cu:70-1466) for the subset described above.
static int ref_thor(RefSim* s) {
    auto&      F  = s->f;
    ref_params P  = s->p;
    const int  NTH = 256;
    const int  num_th_vertical_eq = 32;
    const int  LN                 = 16;
    int        N = s->N, nv = s->nv, nvi = s->nvi, nl_region = s->nl_region, nr = s->nr;
    dim3       NT(nl_region, nl_region, 1);
    dim3       NB(nr, nv, 1);
    dim3       NBD(nr, nv, 6);
    dim3       NBDP(2, nv, 6);
    dim3       NBP(2, nv, 1);
    dim3       NBALL1((N / NTH) + 1, nv, 1);
    int*       maps = s->maps_d;
    int*       loc  = s->point_local_d;
    bool       deep = P.DeepModel, nonh = P.NonHydro, ghv = P.GravHeightVar;
    bool       eeq  = P.energy_equation;
    double     A = P.A, dt = P.timestep;

    REF_CHECK(cudaDeviceSynchronize());
    // the RK array registry is one set of constants per library: load this simulation's
    if (s->probe)
        s->rkm.allocate_device_array();
    else {
        int zero = 0;
        cudaMemcpyToSymbol(num_dynamical_arrays, &zero, sizeof(int));
    }
    cudaMemcpy(F["Mhk"], F["Mh"], N * nv * 3 * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["Whk"], F["Wh"], N * nvi * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["Wk"], F["W"], N * nv * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["Rhok"], F["Rho"], N * nv * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["pressurek"], F["pressure"], N * nv * 8, cudaMemcpyDeviceToDevice);
    cudaMemset(F["Mhs"], 0, 8 * 3 * N * nv);
    cudaMemset(F["Rhos"], 0, 8 * N * nv);
    cudaMemset(F["Whs"], 0, 8 * N * nvi);
    cudaMemset(F["Ws"], 0, 8 * N * nv);
    cudaMemset(F["pressures"], 0, 8 * N * nv);
    if (s->probe)
        probe_init(s);

    for (int rk = 0; rk < 3; rk++) {
        int    ns_it = (rk == 0) ? 1 : (rk == 1 ? 3 : 6);
        double times = (rk == 0) ? dt / 3.0 : dt / 6.0;

        cudaMemset(F["Adv"], 0, 8 * 3 * N * nv);
        REF_CHECK(cudaDeviceSynchronize());
        Compute_Advec_Cori1<LN, LN><<<NB, NT>>>(
            (double3*)F["Adv"], (double3*)F["v"], (double3*)F["Mhk"], (double3*)F["div"], F["Wk"],
            F["Rhok"], F["Altitude"], A, (double3*)F["func_r"], maps, nl_region, deep);
        Compute_Advec_Cori_Poles<6><<<2, 1>>>(F["Adv"], F["v"], F["Mhk"], F["div"], F["Wk"],
                                              F["Rhok"], F["Altitude"], A, F["func_r"], loc, N, nv,
                                              deep);
        REF_CHECK(cudaDeviceSynchronize());
        Compute_Advec_Cori2<<<(N / NTH) + 1, NTH>>>(F["Adv"], F["v"], F["Whk"], F["Rhok"],
                                                    F["Altitude"], F["Altitudeh"], F["func_r"],
                                                    P.Omega, A, nv, N, deep);
        REF_CHECK(cudaDeviceSynchronize());
        Compute_Temperature_H_Pt_Geff<<<(N / NTH) + 1, NTH>>>(
            F["temperature"], F["pressurek"], F["Rhok"], F["Mhk"], F["h"], F["hh"], F["pt"],
            F["pth"], F["gtil"], F["gtilh"], F["Whk"], F["Wk"], F["epotential"], F["epotentialh"],
            F["ekinetic"], F["ekinetich"], F["Etotal"], P.P_Ref, P.Gravit, F["Cp"], F["Rd"],
            F["Altitude"], F["Altitudeh"], A, N, nv, true, eeq, ghv);
        REF_CHECK(cudaDeviceSynchronize());
        cudaMemset(F["SlowMh"], 0, 8 * 3 * N * nv);
        cudaMemset(F["SlowWh"], 0, 8 * N * nvi);
        cudaMemset(F["SlowRho"], 0, 8 * N * nv);
        cudaMemset(F["Slowpressure"], 0, 8 * N * nv);

        if (P.HyDiff) {
            cudaMemset(F["diff"], 0, 8 * 6 * N * nv);
            REF_CHECK(cudaDeviceSynchronize());
            int stepnum = 0;
            for (int ihyp = 0; ihyp < P.HyDiffOrder / 2 - 1; ihyp++) {
                Diffusion_Op<LN, LN><<<NBD, NT>>>(
                    F["diffmh"], F["diffw"], F["diffrh"], F["diffpr"], F["diff"], F["diff_sponge"],
                    F["Mhk"], F["Rhok"], F["temperature"], F["Wk"], F["areasTr"], F["areas"],
                    F["nvecoa"], F["nvecti"], F["nvecte"], F["func_r"], F["Kdh4"], F["Altitude"], A,
                    F["Rd"], F["Cp"], maps, nl_region, stepnum, false, deep, false, 2, F["Kdh2"],
                    F["boundary_flux"], eeq, P.HyDiffOrder);
                Diffusion_Op_Poles<5><<<NBDP, 1>>>(
                    F["diffmh"], F["diffw"], F["diffrh"], F["diffpr"], F["diff"], F["diff_sponge"],
                    F["Mhk"], F["Rhok"], F["temperature"], F["Wk"], F["func_r"], F["areasTr"],
                    F["areas"], F["nvecoa"], F["nvecti"], F["nvecte"], F["Kdh4"], F["Altitude"],
                    F["Altitudeh"], A, F["Rd"], F["Cp"], loc, N, stepnum, false, deep, false, 2,
                    F["Kdh2"], F["boundary_flux"], eeq, P.HyDiffOrder);
                REF_CHECK(cudaDeviceSynchronize());
                stepnum += 1;
            }
            cudaMemset(F["diffrh"], 0, 8 * N * nv);
            cudaMemset(F["boundary_flux"], 0, 8 * 6 * N * nv);
            Diffusion_Op<LN, LN><<<NBD, NT>>>(
                F["diffmh"], F["diffw"], F["diffrh"], F["diffpr"], F["diff"], F["diff_sponge"],
                F["Mhk"], F["Rhok"], F["temperature"], F["Wk"], F["areasTr"], F["areas"],
                F["nvecoa"], F["nvecti"], F["nvecte"], F["func_r"], F["Kdh4"], F["Altitude"], A,
                F["Rd"], F["Cp"], maps, nl_region, stepnum, true, deep, false, 2, F["Kdh2"],
                F["boundary_flux"], eeq, P.HyDiffOrder);
            Diffusion_Op_Poles<5><<<NBDP, 1>>>(
                F["diffmh"], F["diffw"], F["diffrh"], F["diffpr"], F["diff"], F["diff_sponge"],
                F["Mhk"], F["Rhok"], F["temperature"], F["Wk"], F["func_r"], F["areasTr"],
                F["areas"], F["nvecoa"], F["nvecti"], F["nvecte"], F["Kdh4"], F["Altitude"],
                F["Altitudeh"], A, F["Rd"], F["Cp"], loc, N, stepnum, true, deep, false, 2,
                F["Kdh2"], F["boundary_flux"], eeq, P.HyDiffOrder);
            REF_CHECK(cudaDeviceSynchronize());
            if (s->vhd_order > 0) { // thor_driver.cu:590-612
                cudaMemset(F["diff"], 0, sizeof(double) * 6 * N * nv);
                cudaMemset(F["diff2v"], 0, sizeof(double) * 6 * N * (nv + 2));
                dim3 NBALL0((N / NTH) + 1, 1, 6);
                vertical_diff<<<NBALL0, NTH>>>(F["diffmv"], F["diffwv"], F["diffrv"], F["diffprv"],
                                               F["diff"], F["diff2v"], F["Mhk"], F["Rhok"],
                                               F["temperature"], F["Wk"], F["Kdv6"], F["Altitude"],
                                               F["Altitudeh"], A, P.Rd, s->vhd_order, deep, N, nv);
                REF_CHECK(cudaDeviceSynchronize());
            }
            Correct_Horizontal<<<NBALL1, NTH>>>(F["diffmh"], F["diffmv"], F["func_r"], N);
            REF_CHECK(cudaDeviceSynchronize());
        }

        cudaMemset(F["DivM"], 0, 8 * N * 3 * nv);
        cudaMemset(F["divg_Mh"], 0, 8 * N * 3 * nv);
        if (P.DivDampP) {
            REF_CHECK(cudaDeviceSynchronize());
            for (int pass = 0; pass < 2; pass++) {
                DivM_Op<LN, LN><<<NB, NT>>>(F["DivM"], F["divg_Mh"], F["Mhk"], F["Whk"],
                                            F["Kdhz"], F["areasTr"], F["areas"], F["nvecoa"],
                                            F["nvecti"], F["nvecte"], F["func_r"], F["Altitudeh"],
                                            F["Altitude"], A, maps, nl_region, pass, deep);
                DivM_Op_Poles<5><<<NBP, 1>>>(F["DivM"], F["divg_Mh"], F["Mhk"], F["Whk"],
                                             F["Kdhz"], F["areasTr"], F["areas"], F["nvecoa"],
                                             F["nvecti"], F["nvecte"], F["func_r"], F["Altitudeh"],
                                             F["Altitude"], A, loc, N, pass, deep);
                REF_CHECK(cudaDeviceSynchronize());
            }
        }
        REF_CHECK(cudaDeviceSynchronize());
        if (s->sponge && s->S.raysp_calc_mode != 0 && ref_sponge_explicit(s, rk))
            return -1;
        Compute_Slow_Modes<LN, LN><<<NB, NT>>>(
            F["SlowMh"], F["SlowWh"], F["SlowRho"], F["Slowpressure"], F["Mhk"], F["Whk"],
            F["Rhok"], F["Adv"], F["DivM"], F["diffmh"], F["diffw"], F["diffrh"], F["diffpr"],
            F["diffmv"], F["diffwv"], F["diffrv"], F["diffprv"], F["pressurek"], F["h"], F["hh"],
            F["gtil"], F["grad"], F["div"], F["Altitude"], F["Altitudeh"], A, P.Gravit, F["Cp"],
            F["Rd"], F["func_r"], maps, nl_region, deep, nonh, F["profx_dMh"], F["profx_dWh"],
            F["profx_Qheat"], eeq, ghv);
        REF_CHECK(cudaDeviceSynchronize());
        Compute_Slow_Modes_Poles<6><<<2, 1>>>(
            F["SlowMh"], F["SlowWh"], F["SlowRho"], F["Slowpressure"], F["Mhk"], F["Whk"],
            F["Rhok"], F["Adv"], F["DivM"], F["diffmh"], F["diffw"], F["diffrh"], F["diffpr"],
            F["diffmv"], F["diffwv"], F["diffrv"], F["diffprv"], F["pressurek"], F["h"], F["hh"],
            F["gtil"], F["grad"], F["div"], F["Altitude"], F["Altitudeh"], A, P.Gravit, F["Cp"],
            F["Rd"], F["func_r"], loc, nv, N, deep, nonh, F["profx_dMh"], F["profx_dWh"],
            F["profx_Qheat"], eeq, ghv);
        REF_CHECK(cudaDeviceSynchronize());

        if (rk > 0) {
            UpdateRK<<<(N / NTH) + 1, NTH>>>(F["Mhs"], F["Mhk"], F["Mh"], F["Whs"], F["Whk"],
                                             F["Wh"], F["Ws"], F["Rhos"], F["Rhok"], F["Rho"],
                                             F["pressures"], F["pressurek"], F["pressure"],
                                             F["func_r"], F["Altitude"], F["Altitudeh"], N, nv);
            REF_CHECK(cudaDeviceSynchronize());
        }

        for (int ns = 0; ns < ns_it; ns++) {
            cudaMemset(F["DivM"], 0, 8 * N * 3 * nv);
            cudaMemset(F["divg_Mh"], 0, 8 * N * 3 * nv);
            if (P.DivDampP) {
                REF_CHECK(cudaDeviceSynchronize());
                for (int pass = 0; pass < 2; pass++) {
                    DivM_Op<LN, LN><<<NB, NT>>>(F["DivM"], F["divg_Mh"], F["Mhs"], F["Whs"],
                                                F["Kdhz"], F["areasTr"], F["areas"], F["nvecoa"],
                                                F["nvecti"], F["nvecte"], F["func_r"],
                                                F["Altitudeh"], F["Altitude"], A, maps, nl_region,
                                                pass, deep);
                    DivM_Op_Poles<5><<<NBP, 1>>>(F["DivM"], F["divg_Mh"], F["Mhs"], F["Whs"],
                                                 F["Kdhz"], F["areasTr"], F["areas"], F["nvecoa"],
                                                 F["nvecti"], F["nvecte"], F["func_r"],
                                                 F["Altitudeh"], F["Altitude"], A, loc, N, pass,
                                                 deep);
                    REF_CHECK(cudaDeviceSynchronize());
                }
            }
            REF_CHECK(cudaDeviceSynchronize());
            Momentum_Eq<LN, LN><<<NB, NT>>>(F["Mhs"], F["pressures"], F["SlowMh"], F["grad"],
                                            F["Altitude"], F["DivM"], A, F["func_r"], times, maps,
                                            nl_region, deep);
            Momentum_Eq_Poles<6><<<2, 1>>>(F["Mhs"], F["pressures"], F["SlowMh"], F["grad"],
                                           F["Altitude"], F["DivM"], A, F["func_r"], times, loc,
                                           nv, N, deep);
            REF_CHECK(cudaDeviceSynchronize());
            Prepare_Implicit_Vertical<LN, LN><<<NB, NT>>>(
                F["Mhs"], F["h"], F["div"], F["Slowpressure"], F["SlowRho"], F["Sp"], F["Sd"],
                F["Altitude"], F["Cp"], F["Rd"], A, maps, nl_region, deep);
            REF_CHECK(cudaDeviceSynchronize());
            Prepare_Implicit_Vertical_Poles<6><<<2, 1>>>(
                F["Mhs"], F["h"], F["div"], F["Slowpressure"], F["SlowRho"], F["Sp"], F["Sd"],
                F["Altitude"], F["Cp"], F["Rd"], A, loc, N, nv, deep);
            REF_CHECK(cudaDeviceSynchronize());
            Vertical_Eq<<<(N / num_th_vertical_eq) + 1, num_th_vertical_eq,
                          2 * num_th_vertical_eq * nvi * sizeof(double)>>>(
                F["Whs"], F["Ws"], F["pressures"], F["h"], F["hh"], F["Rhos"], F["gtil"],
                F["gtilh"], F["Sp"], F["Sd"], F["SlowWh"], F["Cp"], F["Rd"], times, P.Gravit,
                F["Altitude"], F["Altitudeh"], A, nonh, N, nv, nvi, deep, ghv, s->diag_flag_d,
                s->diag_data_d);
            REF_CHECK(cudaDeviceSynchronize());
            REF_CHECK(cudaGetLastError());
            if (s->probe)
                probe_fast(s, rk, ns, ns_it, times);
            Density_Pressure_Eqs<LN, LN><<<NB, NT>>>(
                F["pressures"], F["pressurek"], F["Rhos"], F["Rhok"], F["Mhs"], F["Mhk"],
                F["Whs"], F["Whk"], F["pt"], F["pth"], F["epotential"], F["epotentialh"],
                F["ekinetic"], F["ekinetich"], F["Etotal"], F["h"], F["hh"], F["SlowRho"],
                F["profx_Qheat"], F["diffpr"], F["diffprv"], F["div"], F["Altitude"],
                F["Altitudeh"], F["Cp"], F["Rd"], A, P.P_Ref, P.Gravit, times, maps, nl_region,
                deep, eeq, ghv, s->diag_flag_d, s->diag_data_d);
            REF_CHECK(cudaDeviceSynchronize());
            Density_Pressure_Eqs_Poles<6><<<2, 1>>>(
                F["pressures"], F["pressurek"], F["Rhos"], F["Rhok"], F["Mhs"], F["Mhk"],
                F["Whs"], F["Whk"], F["pt"], F["pth"], F["epotential"], F["epotentialh"],
                F["ekinetic"], F["ekinetich"], F["Etotal"], F["h"], F["hh"], F["SlowRho"],
                F["profx_Qheat"], F["diffpr"], F["diffprv"], F["div"], F["Altitude"],
                F["Altitudeh"], F["Cp"], F["Rd"], A, P.P_Ref, P.Gravit, times, loc, N, nv, deep,
                eeq, ghv, s->diag_flag_d, s->diag_data_d);
            REF_CHECK(cudaDeviceSynchronize());
        }
        UpdateRK2<<<(N / NTH) + 1, NTH>>>(F["Mhs"], F["Mhk"], F["Whs"], F["Whk"], F["Wk"],
                                          F["Rhos"], F["Rhok"], F["pressures"], F["pressurek"],
                                          F["func_r"], F["Altitude"], F["Altitudeh"], N, nv);
        REF_CHECK(cudaDeviceSynchronize());
    }
    REF_CHECK(cudaDeviceSynchronize());
    cudaMemcpy(F["Mh"], F["Mhk"], N * nv * 3 * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["Wh"], F["Whk"], N * nvi * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["W"], F["Wk"], N * nv * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["Rho"], F["Rhok"], N * nv * 8, cudaMemcpyDeviceToDevice);
    cudaMemcpy(F["pressure"], F["pressurek"], N * nv * 8, cudaMemcpyDeviceToDevice);
    if (s->probe)
        probe_end(s);
    if (s->sponge && s->S.raysp_calc_mode != 0)
        s->sp_step++; // the explicit sponge's step number moves on with the large step
    REF_CHECK(cudaDeviceSynchronize());
    return 0;
}

// Runs `nsteps` large steps (ProfX then Thor, as the main loop of src/esp.cu:1382-1398).
extern "C" int ref_sim_step(void* h, int nsteps, int do_profx, int do_thor) {
    RefSim* s = (RefSim*)h;
    for (int i = 0; i < nsteps; i++) {
        if (do_profx && ref_profx(s))
            return -1;
        if (do_thor && ref_thor(s))
            return -1;
    }
    return 0;
}

// Global conserved quantities of the current state: the kernel sequence of ESP::globdiag
// (src/ESP/profx_driver.cu:476-560, no surface) with the reference's own per-cell kernels
// (src/ESP/profx_globdiag.cu) and its own reduction gpu_sum_on_device<1024>
// (src/headers/reduction_add.h:96-128). out = {energy, mass, AMx, AMy, AMz, entropy}.
extern "C" int ref_sim_globdiag(void* h, double* out) {
    RefSim*   s   = (RefSim*)h;
    auto&     f   = s->f;
    const int NTH = 256;
    dim3      NB((s->N / NTH) + 1, s->nv, 1);
    const ref_params& p = s->p;
    CalcMass<<<NB, NTH>>>(f["Mass"], nullptr, f["Rho"], p.A, f["Altitudeh"], f["lonlat"],
                          f["areasT"], s->N, p.DeepModel);
    CalcTotEnergy<<<NB, NTH>>>(f["Etotal"], nullptr, f["Mh"], f["W"], f["Rho"], f["temperature"],
                               p.Gravit, f["Cp"], f["Rd"], p.A, f["Altitude"], f["Altitudeh"],
                               f["lonlat"], f["areasT"], f["func_r"], s->N, p.DeepModel);
    CalcAngMom<<<NB, NTH>>>(f["AngMomx"], f["AngMomy"], f["AngMomz"], nullptr, nullptr, nullptr,
                            f["Mh"], f["Rho"], p.A, p.Omega, f["Altitude"], f["Altitudeh"],
                            f["lonlat"], f["areasT"], f["func_r"], s->N, p.DeepModel);
    CalcEntropy<<<NB, NTH>>>(f["Entropy"], f["pressure"], f["temperature"], f["Cp"], f["Rd"], p.A,
                             p.P_Ref, f["Altitude"], f["Altitudeh"], f["lonlat"], f["areasT"],
                             f["func_r"], s->N, p.DeepModel);
    REF_CHECK(cudaGetLastError());
    const long n = (long)s->N * s->nv;
    out[0]       = gpu_sum_on_device<1024>(f["Etotal"], n);
    out[1]       = gpu_sum_on_device<1024>(f["Mass"], n);
    out[2]       = gpu_sum_on_device<1024>(f["AngMomx"], n);
    out[3]       = gpu_sum_on_device<1024>(f["AngMomy"], n);
    out[4]       = gpu_sum_on_device<1024>(f["AngMomz"], n);
    out[5]       = gpu_sum_on_device<1024>(f["Entropy"], n);
    REF_CHECK(cudaDeviceSynchronize());
    return 0;
}

// The reference's reduction on a host array copied to the device (gpu_sum_on_device<1024>).
extern "C" double ref_device_sum(const double* host, long n) {
    double* d = nullptr;
    if (cudaMalloc(&d, (n > 0 ? n : 1) * sizeof(double)) != cudaSuccess)
        return 0.0 / 0.0;
    cudaMemcpy(d, host, n * sizeof(double), cudaMemcpyHostToDevice);
    double r = gpu_sum_on_device<1024>(d, n);
    cudaFree(d);
    return r;
}

// Times `nsteps` large steps with CUDA events; returns milliseconds (negative on error).
extern "C" double ref_sim_time(void* h, int nsteps) {
    RefSim*     s = (RefSim*)h;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    for (int i = 0; i < nsteps; i++) {
        if (ref_profx(s) || ref_thor(s))
            return -1.0;
    }
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

extern "C" void ref_sim_free(void* h) {
    RefSim* s = (RefSim*)h;
    for (auto& kv : s->f)
        cudaFree(kv.second);
    cudaFree(s->maps_d);
    cudaFree(s->point_local_d);
    cudaFree(s->diag_flag_d);
    cudaFree(s->diag_data_d);
    delete[] s->Altitude_h;
    cudaFree(s->zonal_mean_tab_d);
    if (s->probe) { // leave the registry empty for the next simulation of this library
        int zero = 0;
        cudaMemcpyToSymbol(num_dynamical_arrays, &zero, sizeof(int));
    }
    delete[] s->vbar_h;
    delete[] s->Tbar_h;
    delete s;
}
