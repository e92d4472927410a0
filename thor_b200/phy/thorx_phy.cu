// thorx_phy: runs a physics-module manager written for the reference's phy_modules_* interface
// (src/headers/phy_modules.h:57-98) on a thorx context (include/thorx_phy.h).
//
// The manager sees an ESP (include/esp.h of this directory) whose device arrays are in the
// reference layouts. Around every hook the shim copies the dynamical core's planes
// ([comp][lev][col], column fastest) into those arrays ([col][lev][comp]), synchronises the
// context's stream, calls the hook (whose kernels run on the legacy default stream), waits for the
// device, and copies the arrays back, so whatever the hook changed reaches the dynamical core. The
// copies are exact, so a hook that changes nothing leaves the state bitwise as it was.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "phy_modules.h"
#include "thorx_phy.h"

// Defaults for the hooks a manager does not define: the reference's managers define the functions
// they need (the empty one, src/physics/managers/empty/src/phy_modules.cu, has phy_loop without the
// kernel_diagnostics argument that phy_modules.h declares).
__attribute__((weak)) std::string phy_modules_get_name() { return "none"; }
__attribute__((weak)) void        phy_modules_print_config() {}
__attribute__((weak)) bool        phy_modules_generate_config(config_file&) { return true; }
__attribute__((weak)) bool phy_modules_init_mem(const ESP&, device_RK_array_manager&) { return true; }
__attribute__((weak)) bool phy_modules_free_mem() { return true; }
__attribute__((weak)) bool phy_modules_init_data(const ESP&, const SimulationSetup&, storage*) {
    return true;
}
__attribute__((weak)) bool phy_modules_dyn_core_loop_init(const ESP&) { return true; }
__attribute__((weak)) bool phy_modules_dyn_core_loop_slow_modes(const ESP&, const SimulationSetup&,
                                                                int, double) {
    return true;
}
__attribute__((weak)) bool phy_modules_dyn_core_loop_fast_modes(const ESP&, const SimulationSetup&,
                                                                int, double) {
    return true;
}
__attribute__((weak)) bool phy_modules_dyn_core_loop_end(const ESP&) { return true; }
__attribute__((weak)) bool phy_modules_phy_loop(ESP&, const SimulationSetup&, kernel_diagnostics&,
                                                int, double) {
    return true;
}
__attribute__((weak)) bool phy_modules_phy_loop(ESP&, const SimulationSetup&, int, double) {
    return true;
}
__attribute__((weak)) bool phy_modules_store(const ESP&, storage&) { return true; }
__attribute__((weak)) bool phy_modules_store_init(storage&) { return true; }

bool device_RK_array_manager::register_array(double* array_d, double* arrayk_d, double* arrayi_d,
                                             int dimensions) {
    if (dimensions < 1 || registered >= NUM_PHY_MODULES_DYN_CORE_ARRAYS)
        return false;
    if (thorx_rk_register_array_n(ctx, array_d, arrayk_d, arrayi_d, cells * dimensions) != 0)
        return false;
    registered++;
    return true;
}

namespace {

// plane (comp * L + lev) * P + col  <->  reference (col * L + lev) * K + comp
__global__ void plane_to_ref(const double* __restrict__ plane, double* __restrict__ ref, int N,
                             int L, int K, long P) {
    const long n = (long)N * L * K;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long col = i / ((long)L * K), r = i % ((long)L * K);
        const int  lev = (int)(r / K), k = (int)(r % K);
        ref[i]         = plane[((long)k * L + lev) * P + col];
    }
}
__global__ void ref_to_plane(const double* __restrict__ ref, double* __restrict__ plane, int N,
                             int L, int K, long P) {
    const long n = (long)N * L * K;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const long col = i / ((long)L * K), r = i % ((long)L * K);
        const int  lev = (int)(r / K), k = (int)(r % K);
        plane[((long)k * L + lev) * P + col] = ref[i];
    }
}

struct Mirror {
    double* plane; // the context's array
    double* ref;   // the ESP member's array
    int     L, K;
    long    P;
};

struct Shim {
    thorx_ctx*          ctx = nullptr;
    ESP                 esp;
    SimulationSetup     sim;
    kernel_diagnostics  diag;
    std::vector<Mirror> mirrors;
    std::vector<void*>  allocs;
    int                 nstep = 1;
    Shim(thorx_ctx* c, const thorx_grid* g) :
        ctx(c), esp(g->point_num, g->nv, g->nl_region, g->nr, g->glevel) {}
};

// the reference's ESP members the shim provides, by thorx field name
struct FieldMember {
    const char* name;
    double* ESP::*member;
};
const FieldMember kFields[] = {
    {"temperature", &ESP::temperature_d}, {"Mh", &ESP::Mh_d},
    {"W", &ESP::W_d},                     {"Wh", &ESP::Wh_d},
    {"Rho", &ESP::Rho_d},                 {"pressure", &ESP::pressure_d},
    {"Rd", &ESP::Rd_d},                   {"Cp", &ESP::Cp_d},
    {"Rhos", &ESP::Rhos_d},               {"pressures", &ESP::pressures_d},
    {"Mhs", &ESP::Mhs_d},                 {"Whs", &ESP::Whs_d},
    {"Rhok", &ESP::Rhok_d},               {"pressurek", &ESP::pressurek_d},
    {"Mhk", &ESP::Mhk_d},                 {"Wk", &ESP::Wk_d},
    {"Whk", &ESP::Whk_d},                 {"profx_Qheat", &ESP::profx_Qheat_d},
    {"profx_dMh", &ESP::profx_dMh_d},     {"profx_dWh", &ESP::profx_dWh_d}};

int launch_dims(long n) { return (int)std::min<long>((n + 255) / 256, 148L * 8); }

// Copies the context's arrays into the ESP arrays, runs `hook` with the device idle, and copies
// the arrays back; a CUDA error anywhere is the hook's return code.
template<class F> int around(Shim* sh, cudaStream_t st, F hook) {
    const int N = sh->esp.point_num;
    for (auto& m : sh->mirrors)
        plane_to_ref<<<launch_dims((long)N * m.L * m.K), 256, 0, st>>>(m.plane, m.ref, N, m.L, m.K, m.P);
    if (cudaStreamSynchronize(st) != cudaSuccess)
        return THORX_E_CUDA;
    hook(); // the reference's callers ignore the hooks' bool (src/ESP/thor_driver.cu:641,1290)
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return THORX_E_CUDA;
    for (auto& m : sh->mirrors)
        ref_to_plane<<<launch_dims((long)N * m.L * m.K), 256, 0, st>>>(m.ref, m.plane, N, m.L, m.K, m.P);
    return cudaGetLastError() == cudaSuccess ? 0 : THORX_E_CUDA;
}

int h_init(void* u, thorx_ctx*, void* st) {
    Shim* sh = (Shim*)u;
    return around(sh, (cudaStream_t)st, [&] { phy_modules_dyn_core_loop_init(sh->esp); });
}
int h_slow(void* u, thorx_ctx*, void* st, int, double times) {
    Shim* sh = (Shim*)u;
    return around(sh, (cudaStream_t)st,
                  [&] { phy_modules_dyn_core_loop_slow_modes(sh->esp, sh->sim, sh->nstep, times); });
}
int h_fast(void* u, thorx_ctx*, void* st, int, int, double times) {
    Shim* sh = (Shim*)u;
    return around(sh, (cudaStream_t)st,
                  [&] { phy_modules_dyn_core_loop_fast_modes(sh->esp, sh->sim, sh->nstep, times); });
}
int h_end(void* u, thorx_ctx*, void* st) {
    Shim*     sh = (Shim*)u;
    const int rc = around(sh, (cudaStream_t)st, [&] { phy_modules_dyn_core_loop_end(sh->esp); });
    sh->nstep++; // Thor ends the step (src/esp.cu:1398, then the step counter moves on)
    sh->esp.current_step = sh->nstep;
    return rc;
}
int h_phy(void* u, thorx_ctx*, void* st, double time_step) {
    Shim* sh = (Shim*)u;
    return around(sh, (cudaStream_t)st, [&] {
        phy_modules_phy_loop(sh->esp, sh->sim, sh->diag, sh->nstep, time_step);
        phy_modules_phy_loop(sh->esp, sh->sim, sh->nstep, time_step);
    });
}

template<class T> int upload(Shim* sh, T*& dst, const T* src, size_t n) {
    dst = nullptr;
    if (!src || n == 0)
        return 0;
    if (cudaMalloc((void**)&dst, n * sizeof(T)) != cudaSuccess)
        return THORX_E_CUDA;
    sh->allocs.push_back(dst);
    return cudaMemcpy(dst, src, n * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess ? 0
                                                                                      : THORX_E_CUDA;
}

void release(Shim* sh) {
    for (void* p : sh->allocs)
        cudaFree(p);
    delete sh;
}

} // namespace

extern "C" int thorx_phy_attach(thorx_ctx* ctx, const thorx_grid* grid, const thorx_phy_setup* s,
                                const char* const* keys, const char* const* values, int nkeys,
                                void** handle) {
    if (!ctx || !grid || !s || !handle || nkeys < 0 || (nkeys > 0 && (!keys || !values)))
        return THORX_E_ARG;
    *handle  = nullptr;
    Shim* sh = new Shim(ctx, grid);
    // SimulationSetup
    SimulationSetup& sim = sh->sim;
    sim.A = s->A, sim.Omega = s->Omega, sim.Gravit = s->Gravit, sim.Rd = s->Rd, sim.Cp = s->Cp;
    sim.Tmean = s->Tmean, sim.P_Ref = s->P_Ref, sim.Top_altitude = s->Top_altitude;
    sim.Diffc = s->Diffc, sim.Diffc_v = s->Diffc_v, sim.DivDampc = s->DivDampc;
    sim.GravHeightVar = s->GravHeightVar, sim.DeepModel = s->DeepModel, sim.HyDiff = s->HyDiff;
    sim.HyDiffOrder = s->HyDiffOrder, sim.DivDampP = s->DivDampP, sim.VertHyDiff = s->VertHyDiff;
    sim.VertHyDiffOrder = s->VertHyDiffOrder, sim.NonHydro = s->NonHydro;
    sim.conv_adj = s->conv_adj, sim.conv_adj_iter = s->conv_adj_iter;
    sim.soft_adjustment = s->soft_adjustment;
    sh->nstep = sh->esp.current_step = s->first_step;
    // configuration
    config_file cfg;
    phy_modules_generate_config(cfg);
    for (int i = 0; i < nkeys; i++)
        if (!keys[i] || !values[i] || !cfg.set(keys[i], values[i])) {
            std::fprintf(stderr, "thorx_phy_attach: module key %s not set\n", keys[i] ? keys[i] : "?");
            release(sh);
            return THORX_E_ARG;
        }
    // geometry, reference layouts
    ESP&         e  = sh->esp;
    const size_t N  = grid->point_num, nv = grid->nv, nr = grid->nr;
    const size_t nm = (size_t)(grid->nl_region + 2) * (grid->nl_region + 2);
    int          rc = upload(sh, e.point_local_d, grid->point_local, N * 6);
    rc              = rc ? rc : upload(sh, e.maps_d, grid->maps, nr * nm);
    rc              = rc ? rc : upload(sh, e.Altitude_d, grid->Altitude, nv);
    rc              = rc ? rc : upload(sh, e.Altitudeh_d, grid->Altitudeh, nv + 1);
    rc              = rc ? rc : upload(sh, e.lonlat_d, grid->lonlat, N * 2);
    rc              = rc ? rc : upload(sh, e.areas_d, grid->areas, N * 18);
    rc              = rc ? rc : upload(sh, e.areasTr_d, grid->areasTr, N * 6);
    rc              = rc ? rc : upload(sh, e.areasT_d, grid->areasT, N);
    rc              = rc ? rc : upload(sh, e.nvecoa_d, grid->nvecoa, N * 18);
    rc              = rc ? rc : upload(sh, e.nvecti_d, grid->nvecti, N * 18);
    rc              = rc ? rc : upload(sh, e.nvecte_d, grid->nvecte, N * 18);
    rc              = rc ? rc : upload(sh, e.div_d, grid->div, N * 21);
    rc              = rc ? rc : upload(sh, e.grad_d, grid->grad, N * 21);
    rc              = rc ? rc : upload(sh, e.func_r_d, grid->func_r, N * 3);
    // state mirrors
    for (const FieldMember& f : kFields) {
        if (rc)
            break;
        Mirror m{};
        if ((rc = thorx_device_field(ctx, f.name, &m.plane, &m.L, &m.K, &m.P)))
            break;
        if (cudaMalloc((void**)&m.ref, N * m.L * m.K * sizeof(double)) != cudaSuccess) {
            rc = THORX_E_CUDA;
            break;
        }
        sh->allocs.push_back(m.ref);
        e.*(f.member) = m.ref;
        sh->mirrors.push_back(m);
    }
    if (rc) {
        release(sh);
        return rc;
    }
    // the manager's set-up (src/ESP/esp_initial.cu:1462-1476)
    phy_modules_print_config();
    device_RK_array_manager rk(ctx, (long long)N * nv);
    phy_modules_init_mem(e, rk);
    phy_modules_init_data(e, sim, nullptr);
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        release(sh);
        return THORX_E_CUDA;
    }
    thorx_module m;
    std::memset(&m, 0, sizeof m);
    m.user                     = sh;
    m.dyn_core_loop_init       = h_init;
    m.dyn_core_loop_slow_modes = h_slow;
    m.dyn_core_loop_fast_modes = h_fast;
    m.dyn_core_loop_end        = h_end;
    m.phy_loop                 = h_phy;
    if ((rc = thorx_set_graph_mode(ctx, 0)) || (rc = thorx_module_add(ctx, &m))) {
        release(sh);
        return rc;
    }
    *handle = sh;
    return 0;
}

extern "C" int thorx_phy_detach(void* handle) {
    if (!handle)
        return THORX_E_ARG;
    phy_modules_free_mem();
    release((Shim*)handle);
    return cudaGetLastError() == cudaSuccess ? 0 : THORX_E_CUDA;
}

extern "C" int thorx_phy_name(char* buf, int n) {
    if (!buf || n < 1)
        return THORX_E_ARG;
    const std::string s = phy_modules_get_name();
    std::snprintf(buf, n, "%s", s.c_str());
    return 0;
}
