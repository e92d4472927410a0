// thorx C ABI: context creation, layout conversion, and the ProfX / Thor launch sequence.
//
// The large step reproduces the stage structure of ESP::Thor (src/ESP/thor_driver.cu:70-1466):
// three RK stages with 1 / 3 / 6 forward-backward small steps of dt/3, dt/6, dt/6. Per stage:
//   adv_temp                  Compute_Advec_Cori1/_Poles/2 + Compute_Temperature_H_Pt_Geff
//   diffusion x (order/2)     Diffusion_Op/_Poles (+ Correct_Horizontal on the last pass)
//   divm0                     DivM_Op/_Poles pass 0 on (Mhk, Whk)
//   slow_modes                DivM pass 1 + Compute_Slow_Modes/_Poles (+ UpdateRK, stages 2,3)
//   per small step:
//     divm0                   DivM pass 0 on (Mhs, Whs)
//     momentum                DivM pass 1 + Momentum_Eq/_Poles
//     vertical                Prepare_Implicit_Vertical + Vertical_Eq + Density_Pressure_Eqs
//   update_rk2                UpdateRK2
// with no host synchronisation inside a step; thorx_step replays the whole step as a CUDA graph.

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <cuda.h>

#include "../../include/thorx.h"
#include "surrogate.h"
#include "thorx_internal.h"

using namespace thorx;

struct FieldDesc {
    double** dev;       // address of the device pointer in State
    int      L;         // levels (nv or nv+1)
    int      K;         // components (1 or 3)
    int      esize = 8; // bytes per element: 4 for divg in the mixed form (kDivgF32)
};

struct thorx_ctx {
    Geometry     g{};
    std::vector<double> Altitude_h, Altitudeh_h;
    Phys         P{};
    State        s{};
    cudaStream_t stream     = nullptr;
    bool         own_stream = false;
    int          glevel     = 0;
    int          hydiff_order = 4;
    // device allocations
    std::vector<void*>               allocs;
    std::map<std::string, FieldDesc> fields;
    double*                          staging     = nullptr; // layout conversion buffer
    size_t                           staging_len = 0;       // doubles
    bool                             rt_enabled  = false;   // double-gray RT in ProfX
    Sponge                           sp{};                   // Rayleigh sponge (nlat 0: off)
    std::vector<thorx_module>        modules;                // physics modules, in call order
    bool                             eager = false;          // thorx_step without a graph
    // a partition (thorx_set_partition): the five-neighbour columns of the whole grid, and the
    // halo exchange called after every kernel (thorx_set_exchange)
    std::vector<int>                 special_all;
    bool                             partitioned = false;
    thorx_exchange_fn                xfn         = nullptr;
    void*                            xuser       = nullptr;
    // uniform thermodynamics (Phys::uniform_thermo): the last host arrays set for Rd and Cp were
    // uniform at the scalar values; thermo_escaped: a module holds their device pointers
    bool                             rd_uniform = false, cp_uniform = false, thermo_escaped = false;
    RkArrays                         rk_arrays{};            // their RK-updated arrays
    Surrogate*                       sur         = nullptr; // RT surrogate (thorx_surrogate_create)
    int                              sur_mode    = THORX_SUR_OFF;
    RtConst                          rt_c{};
    RtFields                         rt_f{};
    double2*                         gd_part     = nullptr; // global-sum partials (6 quantities)
    double*                          gd_out      = nullptr; // the six global sums
    unsigned int*                    flags_host  = nullptr; // pinned
    cudaGraphExec_t                  graph_exec  = nullptr;
    cudaGraph_t                      graph       = nullptr;
    std::string                      err;
    bool                             state_set = false;
    // per-launch CUDA events of a profiled (eager) step, grouped by kernel class
    bool                                                 profiling = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof;
    std::vector<cudaEvent_t>                             event_pool;
    size_t                                               event_next = 0;
};

namespace {
// the surrogate heats the columns this step (THORX_SUR_USE, or with online logging)
bool sur_using(const thorx_ctx* ctx) {
    return ctx->sur_mode == THORX_SUR_USE || ctx->sur_mode == THORX_SUR_USE_LOG;
}

int fail(thorx_ctx* c, int code, const std::string& msg) {
    if (c)
        c->err = msg;
    return code;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(ctx, THORX_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));  \
    } while (0)

template<class T> int dev_alloc(thorx_ctx* ctx, T** p, size_t n) {
    void* d = nullptr;
    CK(cudaMalloc(&d, n * sizeof(T)));
    CK(cudaMemset(d, 0, n * sizeof(T)));
    ctx->allocs.push_back(d);
    *p = (T*)d;
    return 0;
}
// Frees one allocation of dev_alloc before the context's end (null: nothing).
void dev_free(thorx_ctx* ctx, const void* p) {
    if (!p)
        return;
    for (size_t i = 0; i < ctx->allocs.size(); i++)
        if (ctx->allocs[i] == p) {
            cudaFree(ctx->allocs[i]);
            ctx->allocs.erase(ctx->allocs.begin() + (long)i);
            return;
        }
}

// ref layout [N][L][K] <-> device layout [K][L][Np], through 32x32 shared-memory tiles of the
// matrix view ref = [N rows][L*K columns].
__global__ void ref_to_dev_kernel(const double* __restrict__ ref, double* __restrict__ dev, int N,
                                  int Np, int L, int K) {
    __shared__ double tile[32][33];
    const int         Q  = L * K;
    const int         c0 = blockIdx.x * 32, q0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int col = c0 + r, q = q0 + threadIdx.x;
        tile[r][threadIdx.x] = (col < N && q < Q) ? ref[(size_t)col * Q + q] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int q = q0 + r, col = c0 + threadIdx.x;
        if (q < Q && col < N) {
            int l = q / K, k = q % K;
            dev[((size_t)k * L + l) * Np + col] = tile[threadIdx.x][r];
        }
    }
}

__global__ void dev_to_ref_kernel(const double* __restrict__ dev, double* __restrict__ ref, int N,
                                  int Np, int L, int K) {
    __shared__ double tile[32][33];
    const int         Q  = L * K;
    const int         c0 = blockIdx.x * 32, q0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int q = q0 + r, col = c0 + threadIdx.x;
        if (q < Q && col < N) {
            int l = q / K, k = q % K;
            tile[r][threadIdx.x] = dev[((size_t)k * L + l) * Np + col];
        }
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        int col = c0 + r, q = q0 + threadIdx.x;
        if (col < N && q < Q)
            ref[(size_t)col * Q + q] = tile[threadIdx.x][r];
    }
}

// Upload a reference-layout geometry array [N][J] to the device layout [J][Np].
int upload_geo(thorx_ctx* ctx, const double* host, int J, const double** out) {
    const int N = ctx->g.N, Np = ctx->g.Np;
    std::vector<double> t((size_t)J * Np, 0.0);
    for (int c = 0; c < N; c++)
        for (int j = 0; j < J; j++)
            t[(size_t)j * Np + c] = host[(size_t)c * J + j];
    double* d;
    if (dev_alloc(ctx, &d, t.size()))
        return THORX_E_CUDA;
    CK(cudaMemcpy(d, t.data(), t.size() * sizeof(double), cudaMemcpyHostToDevice));
    *out = d;
    return 0;
}

// Neighbour tables from the rhombus maps (halo tile of src/headers/kernel_halo_helpers.h:47-128)
// and, for the two poles, point_local (the *_Poles kernels' neighbour lists), on the host:
// nb, ring [6][Np], flag [Np]. An empty string on success, else what is wrong with the grid.
std::string neighbour_tables(const thorx_grid* gr, int Np, std::vector<int>& nb,
                             std::vector<int>& ring, std::vector<uint8_t>& flag) {
    const int N = gr->point_num, nl = gr->nl_region, nhl = nl + 2, nhl2 = nhl * nhl;
    nb.assign((size_t)6 * Np, -1);
    ring.assign((size_t)6 * Np, -1);
    flag.assign(Np, 0);
    std::vector<char> seen(N, 0);
    for (int r = 0; r < gr->nr; r++) {
        const int* m = gr->maps + (size_t)r * nhl2;
        for (int y = 0; y < nl; y++)
            for (int x = 0; x < nl; x++) {
                const int id = m[(y + 1) * nhl + x + 1];
                if (id < 0 || id >= N - 2 || seen[id])
                    return "maps: bad or repeated interior index";
                seen[id]      = 1;
                const bool pe = (x == 0 && y == 0 && m[0] == -1);
                const int  N0 = m[(y + 2) * nhl + x + 1], N1 = m[(y + 2) * nhl + x + 2],
                          N2 = m[(y + 1) * nhl + x + 2], N3 = m[y * nhl + x + 1],
                          N4 = m[y * nhl + x], N5 = m[(y + 1) * nhl + x];
                const int p[6] = {N0, N1, N2, N3, pe ? N5 : N4, N5};
                for (int j = 0; j < 6; j++) {
                    if (p[j] >= N)
                        return "maps: neighbour index out of range";
                    nb[(size_t)j * Np + id] = p[j];
                }
                const int rg[6] = {N0, N1, N2, N3, pe ? N5 : N4, pe ? -1 : N5};
                for (int j = 0; j < 6; j++)
                    ring[(size_t)j * Np + id] = rg[j];
                flag[id] = pe ? kRing5 : 0;
            }
    }
    for (int id = N - 2; id < N; id++) {
        for (int i = 0; i < 5; i++) {
            int v = gr->point_local[(size_t)id * 6 + i];
            if (v < 0 || v >= N)
                return "point_local: bad pole neighbour";
            nb[(size_t)i * Np + id]   = v;
            ring[(size_t)i * Np + id] = v;
        }
        nb[(size_t)5 * Np + id] = -1;
        flag[id]                = kPole | kRing5;
        seen[id]                = 1;
    }
    for (int id = 0; id < N; id++)
        if (!seen[id])
            return "maps do not cover every column";
    return "";
}

// The momentum kernel's shared-memory windows (Geometry::wspan) from the neighbour tables: for
// each tile, every reference its computed columns make (the column itself, its 6 stencil points,
// its 6 ring points) is sorted by column, swept into spans of kWinW columns (a span starts at the
// first uncovered reference, rounded down to even and kept inside the grid), and the kWinSpans
// spans with the most references are kept. References outside them are read from global memory.
std::vector<int> window_spans(int N, int Np, const std::vector<int>& nb,
                              const std::vector<int>& ring, const std::vector<uint8_t>& flag) {
    const int        tiles = (N + kTileCols - 1) / kTileCols;
    std::vector<int> span((size_t)tiles * kWinSpans, -1);
    if (Np < kWinW)
        return span;
    std::vector<int>                 refs;
    std::vector<std::pair<int, int>> found; // (references, first column)
    for (int t = 0; t < tiles; t++) {
        refs.clear();
        for (int c = t * kTileCols; c < std::min(N, (t + 1) * kTileCols); c++) {
            if (flag[c] & kRing5)
                continue;
            refs.push_back(c);
            for (int j = 0; j < 6; j++) {
                if (nb[(size_t)j * Np + c] >= 0)
                    refs.push_back(nb[(size_t)j * Np + c]);
                if (ring[(size_t)j * Np + c] >= 0)
                    refs.push_back(ring[(size_t)j * Np + c]);
            }
        }
        std::sort(refs.begin(), refs.end());
        found.clear();
        for (size_t i = 0; i < refs.size();) {
            const int x0 = std::min(refs[i] & ~1, Np - kWinW);
            size_t    k  = i;
            while (k < refs.size() && refs[k] < x0 + kWinW)
                k++;
            found.push_back({(int)(k - i), x0});
            i = k;
        }
        std::stable_sort(found.begin(), found.end(),
                         [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
                             return a.first > b.first;
                         });
        for (int s = 0; s < kWinSpans && s < (int)found.size(); s++)
            span[(size_t)t * kWinSpans + s] = found[s].second;
    }
    return span;
}

int build_neighbours(thorx_ctx* ctx, const thorx_grid* gr) {
    const int            N = gr->point_num, Np = ctx->g.Np;
    std::vector<int>     nb, ring;
    std::vector<uint8_t> flag;
    const std::string    err = neighbour_tables(gr, Np, nb, ring, flag);
    if (!err.empty())
        return fail(ctx, THORX_E_ARG, err);
    std::vector<int> special;
    for (int id = 0; id < N; id++)
        if (flag[id] & kRing5)
            special.push_back(id);
    if (special.size() > 32)
        return fail(ctx, THORX_E_ARG, "more five-neighbour columns than one tile holds");
    int*     d_nb;
    int*     d_ring;
    uint8_t* d_flag;
    int*     d_special;
    if (dev_alloc(ctx, &d_nb, nb.size()) || dev_alloc(ctx, &d_ring, ring.size())
        || dev_alloc(ctx, &d_flag, flag.size()) || dev_alloc(ctx, &d_special, 32))
        return THORX_E_CUDA;
    CK(cudaMemcpy(d_special, special.data(), special.size() * sizeof(int), cudaMemcpyHostToDevice));
    ctx->g.special   = d_special;
    ctx->g.nspecial  = (int)special.size();
    ctx->special_all = special;
    CK(cudaMemcpy(d_nb, nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_ring, ring.data(), ring.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_flag, flag.data(), flag.size(), cudaMemcpyHostToDevice));
    ctx->g.nb    = d_nb;
    ctx->g.ring  = d_ring;
    ctx->g.cflag = d_flag;
    const std::vector<int> wspan = window_spans(N, Np, nb, ring, flag);
    int*                   d_wspan;
    if (dev_alloc(ctx, &d_wspan, wspan.size()))
        return THORX_E_CUDA;
    CK(cudaMemcpy(d_wspan, wspan.data(), wspan.size() * sizeof(int), cudaMemcpyHostToDevice));
    ctx->g.wspan = d_wspan;
    return 0;
}

int check_flags(thorx_ctx* ctx) {
    CK(cudaMemcpyAsync(ctx->flags_host, ctx->s.flags, sizeof(unsigned int),
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    unsigned int f = *ctx->flags_host;
    if (f)
        CK(cudaMemsetAsync(ctx->s.flags, 0, sizeof(unsigned int), ctx->stream));
    if (f & kFlagNaN)
        return fail(ctx, THORX_E_NAN, "NaN in temperature after the physics step");
    if (f & kFlagConvAdj)
        return fail(ctx, THORX_E_CONVERGENCE,
                    "convective adjustment: a column exceeded the pass bound");
    if (f & kFlagWait)
        return fail(ctx, THORX_E_CUDA, "a copy into shared memory did not complete in time");
    return 0;
}

// Kernel classes of one step, for thorx_kernel_info / thorx_profile_steps.
enum KClass { KProfx = 0, KAdvTemp, KDiffFirst, KDiffLast, KDivm0, KSlow, KMomentum, KVertical,
              KUpdateRk2, KRt, KSurrogate, KSponge, KVertDiff, KNumClasses };
const char* const kClassName[KNumClasses] = {"profx", "adv_temp", "diffusion_first",
                                             "diffusion_last", "divm0", "slow_modes", "momentum",
                                             "vertical", "update_rk2", "radiative_transfer",
                                             "rt_surrogate", "sponge_means",
                                             "vertical_hyperdiffusion"};

cudaEvent_t next_event(thorx_ctx* ctx) {
    if (ctx->event_next == ctx->event_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        ctx->event_pool.push_back(e);
    }
    return ctx->event_pool[ctx->event_next++];
}

// Brackets one launch with events when the context is profiling.
struct KScope {
    thorx_ctx*  ctx;
    int         cls;
    cudaEvent_t a = nullptr;
    KScope(thorx_ctx* c, int k) : ctx(c), cls(k) {
        if (ctx->profiling) {
            a = next_event(ctx);
            cudaEventRecord(a, ctx->stream);
        }
    }
    ~KScope() {
        if (ctx->profiling) {
            cudaEvent_t b = next_event(ctx);
            cudaEventRecord(b, ctx->stream);
            ctx->prof.push_back({cls, {a, b}});
        }
    }
};

// Calls one hook of every module that has it; a nonzero return ends the enqueuing call.
#define THORX_HOOK(name, ...)                                                                      \
    do {                                                                                          \
        for (const thorx_module& m_ : ctx->modules)                                               \
            if (m_.name) {                                                                        \
                const int rc_ = m_.name(m_.user, ctx, (void*)ctx->stream, ##__VA_ARGS__);         \
                if (rc_)                                                                          \
                    return fail(ctx, rc_, "module hook " #name " returned " + std::to_string(rc_)); \
            }                                                                                     \
    } while (0)

bool has_fast_hook(const thorx_ctx* ctx) {
    for (const thorx_module& m : ctx->modules)
        if (m.dyn_core_loop_fast_modes)
            return true;
    return false;
}
bool has_phy_loop(const thorx_ctx* ctx) {
    for (const thorx_module& m : ctx->modules)
        if (m.phy_loop)
            return true;
    return false;
}

// Algorithmic bytes of one launch of a kernel class: every element the kernel must read or
// write, counted once (neighbour re-reads are not counted), geometry included.
double class_bytes(const thorx_ctx* ctx, int k) {
    const double N = ctx->g.N, nv = ctx->g.nv, nvi = ctx->g.nvi;
    const double S = 8.0 * N * nv, Si = 8.0 * N * nvi, G = 8.0 * N, I = 4.0 * N;
    const Phys&  P = ctx->P;
    const double ring_geo = 78 * G + 6 * I + N; // areas, areasTr, nvecoa/ti/te, ring, flag
    // the Rd and Cp fields, which the dynamical core reads only without uniform thermodynamics
    const double RdCp = P.uniform_thermo ? 0.0 : 2 * S;
    switch (k) {
    case KProfx: // Wh, p, Rd, Rho, Mh | W, T, p, Mh (+ with the sponge: Mh, sponge tables | Wh)
        return Si + 3 * S + (P.benchmark || ctx->sp.nlat ? 3 * S : 0) + G + 3 * S
               + (P.benchmark || ctx->sp.nlat ? 3 * S : 0) + (ctx->sp.nlat ? 5 * G + I + Si : 0);
    case KAdvTemp: // Mhk, Rhok, Wk, Whk, pk, Rd, Cp | Adv, T, h, hh, pt, pth, gtil, gtilh
        return 5 * S + RdCp + Si + 21 * G + 3 * G + 6 * I + 7 * S + 3 * Si
               + (P.energy ? 3 * S + 2 * Si - 2 * S - Si : 0);
    case KDiffFirst: // Rhok, Mhk, Wk, T, Rd (Cp) | diff (6)
        return (5 + (P.energy ? 1 : 0)) * S + RdCp / 2 + ring_geo + 6 * S;
    case KDiffLast: // diff (6), Rhok | diffrh, diffmh, diffw, diffpr
        return 7 * S + ring_geo + 3 * G + 6 * S;
    case KDivm0: // Mh, Wh | divg
        return 3 * S + Si + ring_geo + 3 * S;
    case KSlow: // divg, Cp, Rd, Adv, Rhok, pk, Mhk, h, Whk, hh, diffmh, dMh, diffw, dWh, diffrh,
                // gtil, Qheat, diffpr (+ Mh, Rho, p, Wh) | SlowMh, SlowWh, SlowRho, Slowp (+ Mhs,
                // Rhos, ps, Whs)
        return (P.DivDampP ? 3 * S + ring_geo : 0) + 19 * S + RdCp + 3 * Si + 45 * G + 6 * I
               + 5 * S + Si;
    case KMomentum: // divg, ps, SlowMh, Mhs | Mhs
        return (P.DivDampP ? 3 * S + ring_geo : 0) + 7 * S + 24 * G + 6 * I + 3 * S;
    case KVertical: // Mhs, h, Slowp, SlowRho, hh, gtilh, ps, Rhos, SlowWh, Whs, Cp, Rd, Mhk, pt,
                    // pth, Rhok, pk, Whk, Qheat, diffpr | Whs, Rhos, ps
        return 17 * S + RdCp + 6 * Si + 21 * G + 6 * I + N + Si + 2 * S;
    case KUpdateRk2: // Mhs, Mhk, Rhok, Rhos, pk, ps, Whk, Whs | Mhk, Rhok, pk, Whk, Wk
        return 10 * S + 2 * Si + 3 * G + 6 * S + Si;
    case KRt: // p, Rho, T, Rd, Cp, Qheat, lat, lon, areasT, insol_ann | phtemp, thtemp, fsw/flw
              // up/down, tau (2), ttemp, dtemp, DG_Qheat, Qheat, insol, insol_ann, ASR, OLR, coszen
        return ctx->rt_enabled ? 6 * S + 4 * G + 6 * Si + 6 * S + 6 * G : 0;
    case KSurrogate: // T, p, coszen | features; weights; dtemp (RT columns), Y | dtemp, DG_Qheat,
                     // Qheat (bf16 activations between the layers stay in L2)
        return (ctx->sur && sur_using(ctx))
                   ? 2 * S + G + 2.0 * ctx->sur->net.Kin * N + 4.0 * ctx->sur->net.Nout * N
                         + 2.0 * (ctx->sur->net.Kin + 2.0 * ctx->sur->net.H + ctx->sur->net.Nout)
                               * ctx->sur->net.H
                         + 5 * S
                   : 0;
    case KSponge: // Mh, Rho, Wh (+ p, Rd with the thermal sponge), members, trig | means
        return ctx->sp.nlat ? 4 * S + Si + (ctx->sp.temp ? 2 * S : 0) + I + 4 * G : 0;
    case KVertDiff: // Mhk, Rhok, Wk, T, func_r, diffmh, diffw, diffpr | diff (3), diffmh, diffw,
                    // diffpr
        return P.vhd_order ? 11 * S + 3 * G + 3 * S + 5 * S : 0;
    }
    return 0;
}

int class_launches(const thorx_ctx* ctx, int k) {
    const Phys& P      = ctx->P;
    const int   passes = P.HyDiff ? P.HyDiffOrder / 2 : 0;
    switch (k) {
    case KProfx: // ProfX, then its pressure update after RT or the modules' phy_loop
        return ctx->rt_enabled || has_phy_loop(ctx) ? 2 : 1;
    case KRt: return ctx->rt_enabled ? 1 : 0;     // one bracket: orbit kernel + column kernel
    case KSurrogate: return (ctx->sur && sur_using(ctx)) ? 1 : 0;
    case KSponge: // ProfX's means, or per RK stage the explicit sponge (and, exp3, its means)
        return !ctx->sp.nlat ? 0 : ctx->sp.mode == 0 ? 1 : ctx->sp.mode == 1 ? 4 : 6;
    case KVertDiff: return (P.HyDiff && P.vhd_order) ? 3 : 0;
    case KAdvTemp: return 3;
    case KDiffFirst: return 3 * (passes - (passes > 0 ? 1 : 0));
    case KDiffLast: return passes > 0 ? 3 : 0;
    case KDivm0: return P.DivDampP ? 3 + 10 : 0;
    case KSlow: return 3;
    case KMomentum: return 10;
    case KVertical: return has_fast_hook(ctx) ? 20 : 10; // split around the fast-mode hook
    case KUpdateRk2: return 3;
    }
    return 0;
}

// After a kernel of a partitioned step: the caller's exchange brings the halo columns of the fields
// the kernel wrote up to date (thorx_set_exchange); the energy form's extra fields are added where
// eq is set.
int exchange(thorx_ctx* ctx, std::initializer_list<const char*> f, bool eq = false) {
    if (!ctx->xfn)
        return 0;
    std::vector<const char*> v(f);
    if (eq && ctx->P.energy)
        for (const char* e : {"ep", "eph", "ek", "ekh", "Etotal"})
            v.push_back(e);
    const int rc = ctx->xfn(ctx->xuser, ctx, (void*)ctx->stream, v.data(), (int)v.size());
    return rc ? fail(ctx, rc, "halo exchange returned " + std::to_string(rc)) : 0;
}
#define THORX_XCHG(...)                                                                            \
    do {                                                                                          \
        if (const int rc_ = exchange(ctx, __VA_ARGS__))                                           \
            return rc_;                                                                           \
    } while (0)

// what a partitioned context cannot run: whole-grid sums and module hooks on whole-grid arrays
int partition_check(thorx_ctx* ctx) {
    if (ctx->partitioned && (ctx->sp.nlat > 0 || ctx->sur || !ctx->modules.empty()))
        return fail(ctx, THORX_E_UNSUPPORTED,
                    "a partitioned context runs without the sponge, the surrogate and modules");
    return 0;
}

// ESP::ProfX
int enqueue_profx(thorx_ctx* ctx) {
    if (int rc = partition_check(ctx))
        return rc;
    CK(cudaMemsetAsync(ctx->s.Qheat, 0, sizeof(double) * ctx->g.nv * ctx->g.Np, ctx->stream));
    Sponge sp = ctx->sp; // the implicit sponge runs in ProfX, the explicit ones in Thor
    if (sp.mode != 0)
        sp.nlat = 0;
    if (sp.nlat > 0) {
        KScope k(ctx, KSponge);
        const State& s = ctx->s;
        launch_sponge_means(ctx->g, ctx->P, sp, SpongeIn{s.Mh, s.Rho, nullptr, s.Wh, s.p, s.Rd, true},
                            ctx->stream);
    }
    if (!ctx->rt_enabled && !has_phy_loop(ctx)) {
        {
            KScope k(ctx, KProfx);
            launch_profx(ctx->g, ctx->P, sp, ctx->s, true, ctx->stream);
        }
        THORX_XCHG({"W", "temperature", "pressure", "Mh", "pt"}, true);
    }
    else { // the physics modules run before Compute_pressure (profx_driver.cu:405-432)
        {
            KScope k(ctx, KProfx);
            launch_profx(ctx->g, ctx->P, sp, ctx->s, false, ctx->stream);
        }
        THORX_XCHG({"W", "temperature", "Mh", "pt"}, true);
        if (!ctx->rt_enabled) {
        }
        else if (ctx->sur && sur_using(ctx)) {
            RtFields fm = ctx->rt_f; // plain RT only on re-checked and fallen-back columns
            fm.fallback = ctx->sur->fallback;
            fm.period   = ctx->sur->period;
            {
                KScope k(ctx, KRt);
                launch_rt(ctx->g, ctx->P, ctx->rt_c, fm, ctx->s, ctx->stream);
            }
            {
                KScope k(ctx, KSurrogate);
                if (ctx->sur_mode == THORX_SUR_USE_LOG) // before the combine limits dtemp
                    ctx->sur->log_used(ctx->g, ctx->s, fm, ctx->stream);
                ctx->sur->step_features(ctx->g, ctx->s, fm, ctx->stream);
                ctx->sur->step_combine(ctx->g, ctx->P, ctx->s, fm, ctx->stream);
            }
        }
        else {
            {
                KScope k(ctx, KRt);
                launch_rt(ctx->g, ctx->P, ctx->rt_c, ctx->rt_f, ctx->s, ctx->stream);
            }
            if (ctx->sur && ctx->sur_mode == THORX_SUR_LOG)
                ctx->sur->log_step(ctx->g, ctx->s, ctx->rt_f, ctx->stream);
        }
        THORX_HOOK(phy_loop, ctx->P.timestep);
        {
            KScope k(ctx, KProfx);
            launch_profx_finish(ctx->g, ctx->s, ctx->stream);
        }
        THORX_XCHG({"pressure", "profx_Qheat"});
    }
    CK(cudaGetLastError());
    return 0;
}

// ESP::Thor
int enqueue_thor(thorx_ctx* ctx) {
    const Geometry& g  = ctx->g;
    const Phys&     P  = ctx->P;
    State&          s  = ctx->s;
    cudaStream_t    st = ctx->stream;
    const size_t    cell = (size_t)g.nv * g.Np * sizeof(double), iface = (size_t)g.nvi * g.Np * sizeof(double);
    if (int rc = partition_check(ctx))
        return rc;
    CK(cudaMemcpyAsync(s.Mhk, s.Mh, 3 * cell, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.Whk, s.Wh, iface, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.Wk, s.W, cell, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.Rhok, s.Rho, cell, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.pk, s.p, cell, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(s.Mhs, 0, 3 * cell, st));
    CK(cudaMemsetAsync(s.Rhos, 0, cell, st));
    CK(cudaMemsetAsync(s.Whs, 0, iface, st));
    CK(cudaMemsetAsync(s.ps, 0, cell, st));
    THORX_HOOK(dyn_core_loop_init);
    const bool split = has_fast_hook(ctx);
    for (int rk = 0; rk < 3; rk++) {
        const int    ns_it = (rk == 0) ? 1 : (rk == 1 ? 3 : 6);
        const double times = (rk == 0) ? P.timestep / 3.0 : P.timestep / 6.0;
        {
            KScope k(ctx, KAdvTemp);
            launch_adv_temp(g, P, s, st);
        }
        THORX_XCHG({"Adv", "temperature", "h", "hh", "pt", "pth", "gtil", "gtilh"}, true);
        if (P.HyDiff) {
            int passes = P.HyDiffOrder / 2;
            for (int i = 0; i < passes; i++) {
                {
                    KScope k(ctx, i == passes - 1 ? KDiffLast : KDiffFirst);
                    launch_diffusion(g, P, s, i, i == passes - 1, st);
                }
                if (i == passes - 1)
                    THORX_XCHG({"diffrh", "diffmh", "diffw", "diffpr"});
                else
                    THORX_XCHG({"diff"});
            }
            if (P.vhd_order) { // thor_driver.cu:590-612, inside the hyperdiffusion block
                {
                    KScope k(ctx, KVertDiff);
                    launch_vertical_diff(g, P, s, st);
                }
                THORX_XCHG({"diffmh", "diffw", "diffpr"});
            }
        }
        THORX_HOOK(dyn_core_loop_slow_modes, rk, times);
        if (P.DivDampP) {
            {
                KScope k(ctx, KDivm0);
                launch_divm0(g, P, s, false, st);
            }
            THORX_XCHG({"divg"});
        }
        if (ctx->sp.nlat > 0 && ctx->sp.mode != 0) { // thor_driver.cu:749-866
            KScope k(ctx, KSponge);
            if (rk == 0 || ctx->sp.mode == 2)
                launch_sponge_means(g, P, ctx->sp,
                                    SpongeIn{s.Mhk, s.Rhok, s.Wk, nullptr, s.pk, s.Rd, rk == 0}, st);
            launch_sponge_explicit(g, P, ctx->sp, s, st);
        }
        {
            KScope k(ctx, KSlow);
            launch_slow_modes(g, P, s, rk > 0, st);
        }
        if (rk > 0)
            THORX_XCHG({"SlowMh", "SlowWh", "SlowRho", "Slowpressure", "Mhs", "Rhos", "pressures",
                        "Whs"});
        else
            THORX_XCHG({"SlowMh", "SlowWh", "SlowRho", "Slowpressure"});
        if (rk > 0)
            launch_rk_arrays(ctx->rk_arrays, 0, st);
        for (int ns = 0; ns < ns_it; ns++) {
            if (P.DivDampP) {
                {
                    KScope k(ctx, KDivm0);
                    launch_divm0(g, P, s, true, st);
                }
                THORX_XCHG({"divg"});
            }
            {
                KScope k(ctx, KMomentum);
                launch_momentum(g, P, s, times, st);
            }
            THORX_XCHG({"Mhs"});
            if (!split) {
                {
                    KScope k(ctx, KVertical);
                    launch_vertical(g, P, s, times, 0, st);
                }
                THORX_XCHG({"Whs", "Rhos", "pressures"}, true);
            }
            else { // the modules' fast-mode hooks between Vertical_Eq and Density_Pressure_Eqs
                {
                    KScope k(ctx, KVertical);
                    launch_vertical(g, P, s, times, 1, st);
                }
                THORX_HOOK(dyn_core_loop_fast_modes, rk, ns, times);
                {
                    KScope k(ctx, KVertical);
                    launch_vertical(g, P, s, times, 2, st);
                }
            }
        }
        {
            KScope k(ctx, KUpdateRk2);
            launch_update_rk2(g, P, s, st);
        }
        THORX_XCHG({"Mhk", "Rhok", "pressurek", "Whk", "Wk"});
        launch_rk_arrays(ctx->rk_arrays, 1, st);
    }
    CK(cudaMemcpyAsync(s.Mh, s.Mhk, 3 * cell, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.Wh, s.Whk, iface, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.W, s.Wk, cell, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.Rho, s.Rhok, cell, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s.p, s.pk, cell, cudaMemcpyDeviceToDevice, st));
    THORX_HOOK(dyn_core_loop_end);
    CK(cudaGetLastError());
    return 0;
}

// drops the captured step graph: the next thorx_step captures the step again
int drop_graph(thorx_ctx* ctx) {
    if (ctx->graph_exec) {
        CK(cudaGraphExecDestroy(ctx->graph_exec));
        ctx->graph_exec = nullptr;
    }
    if (ctx->graph) {
        CK(cudaGraphDestroy(ctx->graph));
        ctx->graph = nullptr;
    }
    return 0;
}
} // namespace

namespace {

// Message of the last failed call of this host thread that takes no context.
thread_local std::string g_free_err;

int free_fail(int code, const std::string& msg) {
    g_free_err = msg;
    return code;
}

// Largest n a device sum takes: its partial count must fit the final pass's int index.
constexpr long long kDeviceSumMaxN = 2048LL * 0x7fffffffLL;

// x must be memory of the current device (device or managed) that holds n doubles, inside one
// allocation whose extent the driver reports (cuMemGetAddressRange); checked before any kernel
// reads it, so that a host pointer or a short buffer is an error, not a fault.
int check_device_range(const char* fn, const double* x, long long n) {
    cudaPointerAttributes a{};
    cudaError_t           e = cudaPointerGetAttributes(&a, x);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return free_fail(THORX_E_ARG, std::string(fn) + ": x is not a CUDA pointer");
    }
    int dev = -1;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess)
        return free_fail(THORX_E_CUDA, std::string(fn) + ": cudaGetDevice: " + cudaGetErrorString(e));
    if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != dev)
        return free_fail(THORX_E_ARG,
                         std::string(fn) + ": x is not device memory of the current device");
    using RangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
    static RangeFn range = [] {
        void*                            f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess
            || q != cudaDriverEntryPointSuccess)
            f = nullptr;
        cudaGetLastError();
        return (RangeFn)f;
    }();
    CUdeviceptr base = 0;
    size_t      size = 0;
    if (!range || range(&base, &size, (CUdeviceptr)x) != CUDA_SUCCESS)
        return free_fail(THORX_E_ARG,
                         std::string(fn) + ": the driver reports no allocation extent for x");
    const unsigned long long end = (unsigned long long)base + size;
    if ((unsigned long long)(uintptr_t)x + (unsigned long long)n * sizeof(double) > end)
        return free_fail(THORX_E_ARG, std::string(fn) + ": n = " + std::to_string(n)
                                          + " runs past the end of x's allocation");
    return 0;
}

int check_sum_args(const char* fn, const double* x, long long n, double* out) {
    if (!out || n < 0 || (n > 0 && !x))
        return free_fail(THORX_E_ARG, std::string(fn) + ": null pointer or negative n");
    if (n > kDeviceSumMaxN)
        return free_fail(THORX_E_ARG, std::string(fn) + ": n too large");
    if (n == 0) {
        *out = 0.0;
        return 0;
    }
    return check_device_range(fn, x, n);
}

} // namespace

extern "C" {

int thorx_create(const thorx_grid* gr, const thorx_params* pr, void* stream, thorx_ctx** out) {
    if (!out)
        return THORX_E_ARG;
    *out          = nullptr;
    thorx_ctx* ctx = new thorx_ctx;
    if (!gr || !pr || !gr->maps || !gr->point_local || !gr->Altitude || !gr->Altitudeh
        || !gr->lonlat || !gr->areas || !gr->areasTr || !gr->nvecoa || !gr->nvecti || !gr->nvecte
        || !gr->div || !gr->grad || !gr->func_r || !gr->areasT) {
        *out = ctx;
        return fail(ctx, THORX_E_ARG, "thorx_create: null grid or params pointer");
    }
    *out = ctx;
    const int N = gr->point_num, nv = gr->nv;
    if (N < 12 || nv < 3 || gr->nl_region < 2 || gr->nr < 1
        || (long)gr->nr * gr->nl_region * gr->nl_region != N - 2)
        return fail(ctx, THORX_E_ARG, "thorx_create: inconsistent grid sizes");
    if (nv > max_levels())
        return fail(ctx, THORX_E_UNSUPPORTED, "nv above the supported maximum");
    if (pr->HyDiffOrder < 2 || pr->HyDiffOrder % 2)
        return fail(ctx, THORX_E_UNSUPPORTED, "HyDiffOrder must be even and >= 2");
    if (pr->precision != THORX_FP64 && pr->precision != THORX_MIXED)
        return fail(ctx, THORX_E_ARG, "precision: THORX_FP64 or THORX_MIXED");
    if (pr->thermo_equation != THORX_ENTROPY && pr->thermo_equation != THORX_ENERGY)
        return fail(ctx, THORX_E_ARG, "thermo_equation");
    if (pr->core_benchmark < THORX_NO_BENCHMARK || pr->core_benchmark > THORX_SHALLOW_HOT_JUPITER)
        return fail(ctx, THORX_E_UNSUPPORTED, "core_benchmark");
    if (pr->timestep <= 0 || pr->A <= 0)
        return fail(ctx, THORX_E_ARG, "timestep and radius must be positive");

    if (stream) {
        ctx->stream = (cudaStream_t)stream;
    }
    else {
        CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    ctx->glevel       = gr->glevel;
    Geometry& g       = ctx->g;
    g.N               = N;
    g.Np              = (N + kColAlign - 1) / kColAlign * kColAlign;
    g.tile0           = 0; // every tile: no partition
    g.ntile           = g.Np / kColAlign;
    g.col_end         = N;
    g.nv              = nv;
    g.nvi             = nv + 1;
    const int Np      = g.Np;
    Phys& P           = ctx->P;
    P.A               = pr->A;
    P.Omega           = pr->Omega;
    P.Gravit          = pr->Gravit;
    P.Rd              = pr->Rd;
    P.Cp              = pr->Cp;
    P.P_Ref           = pr->P_Ref;
    P.rP_Ref          = 1.0 / pr->P_Ref;
    P.timestep        = pr->timestep;
    P.HyDiffOrder     = pr->HyDiffOrder;
    P.DeepModel       = pr->DeepModel != 0;
    P.NonHydro        = pr->NonHydro != 0;
    P.GravHeightVar   = pr->GravHeightVar != 0;
    P.HyDiff          = pr->HyDiff != 0;
    P.DivDampP        = pr->DivDampP != 0;
    P.energy          = pr->thermo_equation == THORX_ENERGY;
    P.held_suarez     = pr->core_benchmark == THORX_HELD_SUAREZ;
    P.benchmark       = pr->core_benchmark;
    P.mixed           = pr->precision == THORX_MIXED;
    P.conv_adj_iter   = 0; // thorx_conv_adj_enable
    P.vhd_order       = 0; // thorx_vert_hydiff_enable
    P.conv_soft       = false;

    int rc;
    if ((rc = build_neighbours(ctx, gr)))
        return rc;
    if ((rc = upload_geo(ctx, gr->div, 21, &g.div)) || (rc = upload_geo(ctx, gr->grad, 21, &g.grad))
        || (rc = upload_geo(ctx, gr->areas, 18, &g.areas))
        || (rc = upload_geo(ctx, gr->areasTr, 6, &g.areasTr))
        || (rc = upload_geo(ctx, gr->nvecoa, 18, &g.nvecoa))
        || (rc = upload_geo(ctx, gr->nvecti, 18, &g.nvecti))
        || (rc = upload_geo(ctx, gr->nvecte, 18, &g.nvecte))
        || (rc = upload_geo(ctx, gr->func_r, 3, &g.func_r)))
        return rc;
    {
        std::vector<double> lat(Np, 0.0), lon(Np, 0.0), areasT(Np, 0.0);
        for (int c = 0; c < N; c++) {
            lon[c]    = gr->lonlat[2 * c];
            lat[c]    = gr->lonlat[2 * c + 1];
            areasT[c] = gr->areasT[c];
        }
        double *d, *d2, *d3;
        if (dev_alloc(ctx, &d, Np) || dev_alloc(ctx, &d2, Np) || dev_alloc(ctx, &d3, Np))
            return THORX_E_CUDA;
        CK(cudaMemcpy(d, lat.data(), Np * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d2, lon.data(), Np * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d3, areasT.data(), Np * sizeof(double), cudaMemcpyHostToDevice));
        g.lat    = d;
        g.lon    = d2;
        g.areasT = d3;
    }
    {
        // hyperdiffusion and divergence damping strengths (src/ESP/esp_initial.cu:1292-1335,
        // without the diffusive sponge)
        std::vector<double> kdh4(nv), kdhz(nv);
        for (int lev = 0; lev < nv; lev++) {
            double dbar = sqrt(2 * M_PI / 5) * P.A / (pow(2, gr->glevel));
            kdh4[lev]   = (pr->Diffc) * pow(dbar, 1.0 * pr->HyDiffOrder) / P.timestep;
            kdhz[lev]   = (pr->DivDampc) * pow(dbar, 4.) / P.timestep;
        }
        // Altitude gets one zero entry past the top layer: Compute_Temperature_H_Pt_Geff reads
        // Altitude[nv] at the top boundary with GravHeightVar (src/headers/dyn/thor_auxiliary.h:
        // 195-198, lev == nv), one past the reference's nv-entry array, where its fresh device
        // allocation holds zero; here the read stays in bounds and sees that value
        double *a, *b, *alt, *alth;
        if (dev_alloc(ctx, &a, nv) || dev_alloc(ctx, &b, nv) || dev_alloc(ctx, &alt, nv + 1)
            || dev_alloc(ctx, &alth, nv + 1))
            return THORX_E_CUDA;
        CK(cudaMemcpy(a, kdh4.data(), nv * 8, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(b, kdhz.data(), nv * 8, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(alt, gr->Altitude, nv * 8, cudaMemcpyHostToDevice));
        ctx->Altitude_h.assign(gr->Altitude, gr->Altitude + nv);
        ctx->Altitudeh_h.assign(gr->Altitudeh, gr->Altitudeh + nv + 1);
        CK(cudaMemcpy(alth, gr->Altitudeh, (nv + 1) * 8, cudaMemcpyHostToDevice));
        double* lt;
        if (dev_alloc(ctx, &lt, (size_t)kLtCount * (nv + 1)))
            return THORX_E_CUDA;
        g.lt = lt;
        g.Kdh4      = a;
        g.Kdhz      = b;
        g.Altitude  = alt;
        g.Altitudeh = alth;
        launch_level_tables(g, P, lt, ctx->stream);
        CK(cudaGetLastError());
    }
    {
        // operator weights of the mixed form, from the geometry just uploaded
        double* lapw;
        float*  dmw;
        double* dmw64;
        if (dev_alloc(ctx, &lapw, (size_t)7 * Np) || dev_alloc(ctx, &dmw, (size_t)84 * Np)
            || dev_alloc(ctx, &dmw64, (size_t)84 * Np))
            return THORX_E_CUDA;
        g.lapw = lapw;
        g.dmw   = dmw;
        g.dmw64 = dmw64;
        launch_stencil_weights(g, lapw, dmw, dmw64, ctx->stream);
        CK(cudaGetLastError());
    }

    // state
    State&       s     = ctx->s;
    const size_t cell  = (size_t)nv * Np, iface = (size_t)(nv + 1) * Np;
    struct A {
        double** p;
        size_t   n;
    } al[] = {{&s.Mh, 3 * cell},    {&s.Mhk, 3 * cell},  {&s.Mhs, 3 * cell},   {&s.Rho, cell},
              {&s.Rhok, cell},      {&s.Rhos, cell},     {&s.p, cell},         {&s.pk, cell},
              {&s.ps, cell},        {&s.Wh, iface},      {&s.Whk, iface},      {&s.Whs, iface},
              {&s.W, cell},         {&s.Wk, cell},       {&s.T, cell},         {&s.Rd, cell},
              {&s.Cp, cell},        {&s.h, cell},        {&s.hh, iface},       {&s.pt, cell},
              {&s.pth, iface},      {&s.gtil, cell},     {&s.gtilh, iface},    {&s.Adv, 3 * cell},
              {&s.diff, 12 * cell}, {&s.diffmh, 3 * cell}, {&s.diffw, cell},   {&s.diffrh, cell},
              {&s.diffpr, cell},    {&s.divg, 3 * cell}, {&s.vrows, 4 * iface + 6 * cell}, {&s.SlowMh, 3 * cell},
              {&s.SlowWh, iface},
              {&s.SlowRho, cell},   {&s.Slowp, cell},    {&s.Qheat, cell},     {&s.dMh, 3 * cell},
              {&s.dWh, iface}};
    for (auto& x : al)
        if (dev_alloc(ctx, x.p, x.n))
            return THORX_E_CUDA;
    if (P.energy) {
        if (dev_alloc(ctx, &s.ep, cell) || dev_alloc(ctx, &s.eph, iface)
            || dev_alloc(ctx, &s.ek, cell) || dev_alloc(ctx, &s.ekh, iface)
            || dev_alloc(ctx, &s.Etotal, cell))
            return THORX_E_CUDA;
    }
    if (dev_alloc(ctx, &s.flags, 1))
        return THORX_E_CUDA;
    CK(cudaMallocHost(&ctx->flags_host, sizeof(unsigned int)));
    ctx->staging_len = (size_t)N * (nv + 1) * 3;
    if (dev_alloc(ctx, &ctx->staging, ctx->staging_len))
        return THORX_E_CUDA;
    if (dev_alloc(ctx, &ctx->gd_part, (size_t)6 * globdiag_partials(g))
        || dev_alloc(ctx, &ctx->gd_out, 6))
        return THORX_E_CUDA;

    auto& F          = ctx->fields;
    F["Rho"]         = {&s.Rho, nv, 1};
    F["pressure"]    = {&s.p, nv, 1};
    F["Mh"]          = {&s.Mh, nv, 3};
    F["Wh"]          = {&s.Wh, nv + 1, 1};
    F["W"]           = {&s.W, nv, 1};
    F["temperature"] = {&s.T, nv, 1};
    F["Rd"]          = {&s.Rd, nv, 1};
    F["Cp"]          = {&s.Cp, nv, 1};
    F["profx_Qheat"] = {&s.Qheat, nv, 1};
    F["SlowMh"]      = {&s.SlowMh, nv, 3};
    F["SlowWh"]      = {&s.SlowWh, nv + 1, 1};
    F["SlowRho"]     = {&s.SlowRho, nv, 1};
    F["Slowpressure"] = {&s.Slowp, nv, 1};
    F["h"]           = {&s.h, nv, 1};
    F["hh"]          = {&s.hh, nv + 1, 1};
    F["pt"]          = {&s.pt, nv, 1};
    F["pth"]         = {&s.pth, nv + 1, 1};
    F["gtil"]        = {&s.gtil, nv, 1};
    F["gtilh"]       = {&s.gtilh, nv + 1, 1};
    F["Adv"]         = {&s.Adv, nv, 3};
    F["diffmh"]      = {&s.diffmh, nv, 3};
    F["diffw"]       = {&s.diffw, nv, 1};
    F["diffrh"]      = {&s.diffrh, nv, 1};
    F["diffpr"]      = {&s.diffpr, nv, 1};
    CK(cudaDeviceSynchronize());
    return 0;
}

void thorx_destroy(thorx_ctx* ctx) {
    if (!ctx)
        return;
    if (ctx->graph_exec)
        cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->graph)
        cudaGraphDestroy(ctx->graph);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    for (cudaEvent_t e : ctx->event_pool)
        cudaEventDestroy(e);
    if (ctx->sur) {
        ctx->sur->release();
        delete ctx->sur;
    }
    for (void* p : ctx->allocs)
        cudaFree(p);
    if (ctx->flags_host)
        cudaFreeHost(ctx->flags_host);
    if (ctx->own_stream && ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* thorx_last_error(const thorx_ctx* ctx) {
    return ctx ? ctx->err.c_str() : g_free_err.c_str();
}

long thorx_field_size(const thorx_ctx* ctx, const char* name) {
    if (!ctx || !name)
        return THORX_E_ARG;
    auto it = ctx->fields.find(name);
    if (it == ctx->fields.end())
        return THORX_E_ARG;
    return (long)ctx->g.N * it->second.L * it->second.K;
}

namespace {
// Phys::uniform_thermo from the context's record; a change re-captures the step graph (its kernels
// were instantiated for the other form)
int update_thermo(thorx_ctx* ctx) {
    const bool u = ctx->rd_uniform && ctx->cp_uniform && !ctx->thermo_escaped;
    if (u == ctx->P.uniform_thermo)
        return 0;
    ctx->P.uniform_thermo = u;
    return drop_graph(ctx);
}

bool all_bits_equal(const double* a, size_t n, double v) {
    for (size_t i = 0; i < n; i++)
        if (std::memcmp(a + i, &v, sizeof v) != 0)
            return false;
    return true;
}
} // namespace

int thorx_set_field(thorx_ctx* ctx, const char* name, const double* host) {
    if (!ctx)
        return THORX_E_ARG;
    if (!name || !host)
        return fail(ctx, THORX_E_ARG, "thorx_set_field: null argument");
    auto it = ctx->fields.find(name);
    if (it == ctx->fields.end())
        return fail(ctx, THORX_E_ARG, std::string("thorx_set_field: unknown field ") + name);
    const FieldDesc& f = it->second;
    const size_t     n = (size_t)ctx->g.N * f.L * f.K;
    CK(cudaMemcpyAsync(ctx->staging, host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    dim3 grid((ctx->g.N + 31) / 32, (f.L * f.K + 31) / 32), block(32, 8);
    ref_to_dev_kernel<<<grid, block, 0, ctx->stream>>>(ctx->staging, *f.dev, ctx->g.N, ctx->g.Np,
                                                      f.L, f.K);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->state_set = true;
    if (!std::strcmp(name, "Rd") || !std::strcmp(name, "Cp")) {
        const bool rd = !std::strcmp(name, "Rd");
        (rd ? ctx->rd_uniform : ctx->cp_uniform) = all_bits_equal(host, n, rd ? ctx->P.Rd : ctx->P.Cp);
        return update_thermo(ctx);
    }
    return 0;
}

int thorx_get_field(thorx_ctx* ctx, const char* name, double* host) {
    if (!ctx)
        return THORX_E_ARG;
    if (!name || !host)
        return fail(ctx, THORX_E_ARG, "thorx_get_field: null argument");
    auto it = ctx->fields.find(name);
    if (it == ctx->fields.end())
        return fail(ctx, THORX_E_ARG, std::string("thorx_get_field: unknown field ") + name);
    const FieldDesc& f = it->second;
    const size_t     n = (size_t)ctx->g.N * f.L * f.K;
    dim3 grid((ctx->g.N + 31) / 32, (f.L * f.K + 31) / 32), block(32, 8);
    dev_to_ref_kernel<<<grid, block, 0, ctx->stream>>>(*f.dev, ctx->staging, ctx->g.N, ctx->g.Np,
                                                      f.L, f.K);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(host, ctx->staging, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int thorx_init_rest_state(thorx_ctx* ctx, double Tmean, unsigned long long seed,
                          double noise_amp) {
    if (!ctx)
        return THORX_E_ARG;
    if (!(Tmean > 0) || !(noise_amp >= 0) || noise_amp >= Tmean)
        return fail(ctx, THORX_E_ARG, "thorx_init_rest_state: bad Tmean or noise amplitude");
    const int  N = ctx->g.N, nv = ctx->g.nv;
    const Phys& P = ctx->P;
    const double* Alt  = ctx->Altitude_h.data();
    const double* Alth = ctx->Altitudeh_h.data();
    // isothermal hydrostatic column: Newton-Raphson on the discrete hydrostatic balance between
    // consecutive levels (src/ESP/esp_initial.cu:518-587, GravHeightVar as configured)
    std::vector<double> p0(nv), r0(nv), T0(nv);
    const double        eps = 1e-15;
    const int           it_max = 100;
    for (int lev = 0; lev < nv; lev++) {
        double P_L, rho_L, T_L, dz, g_L, l_int, r_int;
        if (lev == 0) {
            P_L   = P.P_Ref;
            rho_L = P.P_Ref / (P.Rd * Tmean);
            T_L   = Tmean;
            dz    = Alt[0];
            g_L   = P.GravHeightVar ? P.Gravit * pow(P.A / (P.A + Alt[0]), 2) : P.Gravit;
            l_int = 0.5;
            r_int = 0.5;
        }
        else {
            P_L   = p0[lev - 1];
            rho_L = r0[lev - 1];
            T_L   = T0[lev - 1];
            dz    = Alt[lev] - Alt[lev - 1];
            g_L   = P.GravHeightVar ? P.Gravit * pow(P.A / (P.A + Alt[lev - 1]), 2) : P.Gravit;
            l_int = (Alt[lev] - Alth[lev]) / dz;
            r_int = (Alth[lev] - Alt[lev - 1]) / dz;
        }
        p0[lev]     = P_L;
        r0[lev]     = rho_L;
        T0[lev]     = T_L;
        double ptmp = p0[lev] + 2 * eps * p0[lev];
        double g    = P.GravHeightVar ? P.Gravit * pow(P.A / (P.A + Alt[lev]), 2) : P.Gravit;
        for (int it = 0; it < it_max && (ptmp - p0[lev]) / p0[lev] > eps; it++) {
            ptmp      = p0[lev];
            double f  = (p0[lev] - P_L) / dz + (g * r_int + g_L * l_int) * (r0[lev] * r_int + rho_L * l_int);
            double df = 1.0 / dz + (g * r_int + g_L * l_int) * r_int / (P.Rd * T0[lev]);
            p0[lev]   = p0[lev] - f / df;
            r0[lev]   = p0[lev] / (P.Rd * T0[lev]);
        }
    }
    // per-column fields with the seeded perturbation (SplitMix64: Steele, Lea & Flood 2014)
    const size_t        n = (size_t)N * nv;
    std::vector<double> T(n), p(n), rho(n), Rd(n, P.Rd), Cp(n, P.Cp), zero3(3 * n, 0.0),
        zeroi((size_t)N * (nv + 1), 0.0), zero(n, 0.0);
    uint64_t x = seed;
    for (size_t i = 0; i < n; i++) {
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = x;
        z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z          = z ^ (z >> 31);
        double u   = (double)(z >> 11) * (1.0 / 9007199254740992.0);
        int    lev = (int)(i % nv);
        T[i]       = T0[lev] + (2.0 * u - 1.0) * noise_amp;
        p[i]       = p0[lev];
        rho[i]     = p[i] / (P.Rd * T[i]);
    }
    int rc;
    if ((rc = thorx_set_field(ctx, "temperature", T.data())) || (rc = thorx_set_field(ctx, "pressure", p.data()))
        || (rc = thorx_set_field(ctx, "Rho", rho.data())) || (rc = thorx_set_field(ctx, "Rd", Rd.data()))
        || (rc = thorx_set_field(ctx, "Cp", Cp.data())) || (rc = thorx_set_field(ctx, "Mh", zero3.data()))
        || (rc = thorx_set_field(ctx, "Wh", zeroi.data())) || (rc = thorx_set_field(ctx, "W", zero.data())))
        return rc;
    return 0;
}

namespace {
// Temperature of Guillot's (2010) radiative-equilibrium profile, eq. 27, in the form of the
// reference's guillot_T (src/ESP/ultrahot_thermo.cu:121-161): gray LW opacity increasing with
// pressure (f_lw the well-mixed fraction), gray SW absorption, irradiation angle mu.
double guillot_T(double pressure, double mu, double Teq, double P_Ref, double Gravit, double Tint,
                 double f_lw, double kappa_sw, double kappa_lw) {
    const double tau0   = kappa_lw * P_Ref / Gravit;
    const double eps    = 1.0 / f_lw;
    const double x0     = P_Ref / Gravit;
    const double gamma0 = kappa_sw / kappa_lw;
    const double klw    = kappa_lw * (1.0 + 2 * (eps - 1) * pressure / P_Ref);
    const double x      = pressure / Gravit;
    const double tau    = kappa_lw * x;
    const double tau_lw = tau0 * pressure / P_Ref + (eps - 1) * tau0 * pow(pressure / P_Ref, 2);
    const double gamma  = kappa_sw / klw;
    const double T4 =
        0.75 * pow(Tint, 4) * (2. / 3 + tau_lw)
        + 3 * mu * pow(Teq, 4)
              * (2. / 3 + gamma / (3 * mu) * exp(-gamma0 * tau / mu)
                 + mu / gamma0 * (1.0 - exp(-gamma0 * tau / mu))
                 + 2 * (eps - 1) * mu / (gamma0 * kappa_sw * x0)
                       * (mu - (mu + gamma0 * tau) * exp(-gamma0 * tau / mu)));
    return pow(T4, 0.25);
}
} // namespace

int thorx_init_guillot_state(thorx_ctx* ctx, double Tmean, double Tint, double f_lw,
                             double kappa_sw, double kappa_lw, unsigned long long seed,
                             double noise_amp) {
    if (!ctx)
        return THORX_E_ARG;
    if (!(Tmean > 0) || !(Tint >= 0) || !(f_lw > 0) || !(kappa_sw > 0) || !(kappa_lw > 0)
        || !(noise_amp >= 0))
        return fail(ctx, THORX_E_ARG, "thorx_init_guillot_state: bad profile parameter");
    const int     N = ctx->g.N, nv = ctx->g.nv;
    const Phys&   P = ctx->P;
    const double* Alt  = ctx->Altitude_h.data();
    const double* Alth = ctx->Altitudeh_h.data();
    // one column, the general rest-state branch of initial_values (src/ESP/esp_initial.cu:840-1000):
    // Newton-Raphson on the discrete hydrostatic balance with T re-evaluated from the profile at
    // every iterate; Teq = Tmean, mu = 0.5, Rd and Cp constant
    std::vector<double> p0(nv), T0(nv);
    const double        eps = 1e-15, mu = 0.5;
    const int           it_max = 100;
    auto grav = [&](double alt) { return P.GravHeightVar ? P.Gravit * pow(P.A / (P.A + alt), 2) : P.Gravit; };
    for (int lev = 0; lev < nv; lev++) {
        double g_L, P_L, T_L, dz, l_int, r_int;
        if (lev == 0) {
            g_L   = grav(Alt[0]);
            T0[0] = guillot_T(P.P_Ref, mu, Tmean, P.P_Ref, g_L, Tint, f_lw, kappa_sw, kappa_lw);
            P_L   = P.P_Ref;
            T_L   = T0[0];
            dz    = Alt[0];
            l_int = 0.5;
            r_int = 0.5;
        }
        else {
            g_L     = grav(Alt[lev - 1]);
            T0[lev] = T0[lev - 1];
            P_L     = p0[lev - 1];
            T_L     = T0[lev - 1];
            dz      = Alt[lev] - Alt[lev - 1];
            l_int   = (Alt[lev] - Alth[lev]) / dz;
            r_int   = (Alth[lev] - Alt[lev - 1]) / dz;
        }
        p0[lev]            = P_L;
        T0[lev]            = T_L;
        double       ptmp  = p0[lev] + 2 * eps * p0[lev];
        const double g     = grav(Alt[lev]);
        for (int it = 0; it < it_max && (ptmp - p0[lev]) / p0[lev] > eps; it++) {
            ptmp            = p0[lev];
            const double f  = (p0[lev] - P_L) / dz
                             + (g * r_int + g_L * l_int) / P.Rd
                                   * (p0[lev] * r_int / T0[lev] + P_L * l_int / T_L);
            const double df = 1.0 / dz + (g * r_int + g_L * l_int) * r_int / (P.Rd * T0[lev]);
            p0[lev]         = p0[lev] - f / df;
            T0[lev] = guillot_T(p0[lev], mu, Tmean, P.P_Ref, g, Tint, f_lw, kappa_sw, kappa_lw);
        }
    }
    const size_t        n = (size_t)N * nv;
    std::vector<double> T(n), p(n), rho(n), Rd(n, P.Rd), Cp(n, P.Cp), zero3(3 * n, 0.0),
        zeroi((size_t)N * (nv + 1), 0.0), zero(n, 0.0);
    uint64_t x = seed; // the perturbation of thorx_init_rest_state
    for (size_t i = 0; i < n; i++) {
        x += 0x9E3779B97F4A7C15ull;
        uint64_t z = x;
        z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z          = z ^ (z >> 31);
        double u   = (double)(z >> 11) * (1.0 / 9007199254740992.0);
        int    lev = (int)(i % nv);
        T[i]       = T0[lev] + (2.0 * u - 1.0) * noise_amp;
        p[i]       = p0[lev];
        rho[i]     = p[i] / (T[i] * P.Rd);
    }
    int rc;
    if ((rc = thorx_set_field(ctx, "temperature", T.data())) || (rc = thorx_set_field(ctx, "pressure", p.data()))
        || (rc = thorx_set_field(ctx, "Rho", rho.data())) || (rc = thorx_set_field(ctx, "Rd", Rd.data()))
        || (rc = thorx_set_field(ctx, "Cp", Cp.data())) || (rc = thorx_set_field(ctx, "Mh", zero3.data()))
        || (rc = thorx_set_field(ctx, "Wh", zeroi.data())) || (rc = thorx_set_field(ctx, "W", zero.data())))
        return rc;
    return 0;
}

int thorx_profx(thorx_ctx* ctx) {
    if (!ctx)
        return THORX_E_ARG;
    int rc = enqueue_profx(ctx);
    if (rc)
        return rc;
    return check_flags(ctx);
}

int thorx_thor(thorx_ctx* ctx) {
    if (!ctx)
        return THORX_E_ARG;
    int rc = enqueue_thor(ctx);
    if (rc)
        return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int thorx_step(thorx_ctx* ctx, int nsteps) {
    if (!ctx || nsteps < 0)
        return THORX_E_ARG;
    if (ctx->eager) { // thorx_set_graph_mode(ctx, 0): every step enqueued, every hook called
        for (int i = 0; i < nsteps; i++) {
            int rc = enqueue_profx(ctx);
            if (!rc)
                rc = enqueue_thor(ctx);
            if (rc)
                return rc;
        }
        return 0;
    }
    if (!ctx->graph_exec) {
        CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_profx(ctx);
        if (!rc)
            rc = enqueue_thor(ctx);
        cudaGraph_t graph = nullptr;
        cudaError_t e     = cudaStreamEndCapture(ctx->stream, &graph);
        if (rc) {
            if (graph)
                cudaGraphDestroy(graph);
            return rc;
        }
        if (e != cudaSuccess)
            return fail(ctx, THORX_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
        ctx->graph = graph;
        CK(cudaGraphInstantiate(&ctx->graph_exec, graph, 0));
    }
    for (int i = 0; i < nsteps; i++)
        CK(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    return 0;
}

int thorx_sync(thorx_ctx* ctx) {
    if (!ctx)
        return THORX_E_ARG;
    return check_flags(ctx);
}

int thorx_kernels_per_step(const thorx_ctx* ctx) {
    if (!ctx)
        return THORX_E_ARG;
    int n = 0;
    for (int k = 0; k < KNumClasses; k++)
        n += class_launches(ctx, k);
    n += ctx->rt_enabled ? 1 : 0; // the RT bracket holds two kernels
    if (ctx->rk_arrays.n > 0)
        n += 5; // UpdateRK's reset in stages 2 and 3, UpdateRK2's accumulation in all three
    if (ctx->sur && sur_using(ctx))
        n += 5; // features, four GEMMs and the combine in one bracket
    if (ctx->sur && ctx->sur_mode == THORX_SUR_LOG)
        n += 2; // log slot reservation and write
    return n;
}

int thorx_kernel_classes(const thorx_ctx* ctx) { return ctx ? (int)KNumClasses : THORX_E_ARG; }

int thorx_kernel_info(const thorx_ctx* ctx, int k, const char** name, double* bytes_per_launch,
                      int* launches_per_step) {
    if (!ctx || k < 0 || k >= KNumClasses)
        return THORX_E_ARG;
    if (name)
        *name = kClassName[k];
    if (bytes_per_launch)
        *bytes_per_launch = class_bytes(ctx, k);
    if (launches_per_step)
        *launches_per_step = class_launches(ctx, k);
    return 0;
}

int thorx_profile_steps(thorx_ctx* ctx, int nsteps, double* ms_per_class) {
    if (!ctx || nsteps < 1 || !ms_per_class)
        return THORX_E_ARG;
    ctx->profiling  = true;
    ctx->event_next = 0;
    ctx->prof.clear();
    int rc = 0;
    for (int i = 0; i < nsteps && !rc; i++) {
        rc = enqueue_profx(ctx);
        if (!rc)
            rc = enqueue_thor(ctx);
    }
    ctx->profiling = false;
    if (rc)
        return rc;
    CK(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < KNumClasses; k++)
        ms_per_class[k] = 0.0;
    for (auto& e : ctx->prof) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e.second.first, e.second.second));
        ms_per_class[e.first] += ms;
    }
    return 0;
}

int thorx_rt_enable(thorx_ctx* ctx, const thorx_rt_params* r) {
    if (!ctx)
        return THORX_E_ARG;
    if (!r)
        return fail(ctx, THORX_E_ARG, "thorx_rt_enable: null argument");
    if (ctx->rt_enabled)
        return fail(ctx, THORX_E_STATE, "thorx_rt_enable: RT is already enabled");
    if (r->surface)
        return fail(ctx, THORX_E_UNSUPPORTED, "thorx_rt_enable: surface = true is not implemented");
    if (ctx->P.GravHeightVar)
        return fail(ctx, THORX_E_UNSUPPORTED,
                    "thorx_rt_enable: GravHeightVar with RT reads past Altitudeh in the reference "
                    "(profx_RT.h:68); not supported");
    if (!(r->planet_star_dist > 0) || !(r->radius_star > 0) || !(r->Tstar >= 0) || !(r->f_lw > 0)
        || !(r->diff_ang > 0) || !(r->ecc >= 0 && r->ecc < 1) || r->first_step < 1
        || (!r->sync_rot && !(r->mean_motion > 0)))
        return fail(ctx, THORX_E_ARG, "thorx_rt_enable: parameter out of range");
    const int N = ctx->g.N, nv = ctx->g.nv, nvi = nv + 1, Np = ctx->g.Np;
    (void)N;
    RtConst& c = ctx->rt_c;
    // RTSetup (radiative_transfer.cu:1431-1432); Insolation::initial_conditions (insolation.cu:292-313)
    const double resc_flx = pow(r->radius_star / r->planet_star_dist, 2.0);
    c.incflx   = resc_flx * 5.6703744191844314e-08 * r->Tstar * r->Tstar * r->Tstar * r->Tstar;
    c.diff_ang = r->diff_ang;
    c.Tint     = r->Tint;
    c.albedo   = r->albedo;
    c.kappa_sw = r->kappa_sw;
    c.kappa_lw = r->kappa_lw;
    c.kappa_lw_pole = r->kappa_lw_pole;
    c.n_sw     = r->n_sw;
    c.n_lw     = r->n_lw;
    c.f_lw     = r->f_lw;
    c.mean_motion = r->sync_rot ? ctx->P.Omega : r->mean_motion;
    c.true_long_i = r->true_long_i * M_PI / 180.0;
    c.longp       = r->longp * M_PI / 180.0;
    c.ecc         = r->ecc;
    {
        double f = fmod(c.true_long_i - c.longp, (2 * M_PI));
        while (f < 0.0)
            f += 2 * M_PI;
        while (f >= 2 * M_PI)
            f -= 2 * M_PI;
        const double cosE = (cos(f) + c.ecc) / (1.0 + c.ecc * cos(f));
        const double E_i  = f < M_PI ? acos(cosE) : 2 * M_PI - acos(cosE);
        c.mean_anomaly_i  = fmod(E_i - c.ecc * sin(E_i), (2 * M_PI));
    }
    c.alpha_i        = r->alpha_i * M_PI / 180.0;
    c.obliquity      = r->obliquity * M_PI / 180.0;
    c.latf_lw        = r->latf_lw;
    c.rt1Dmode       = r->rt1Dmode;
    c.sync_rot       = r->sync_rot;
    c.spinup_start   = r->spinup_start;
    c.spinup_stop    = r->spinup_stop;
    c.spindown_start = r->spindown_start;
    c.spindown_stop  = r->spindown_stop;

    RtFields& f = ctx->rt_f;
    const size_t cell = (size_t)nv * Np, iface = (size_t)nvi * Np;
    if (dev_alloc(ctx, &f.phtemp, iface) || dev_alloc(ctx, &f.thtemp, iface)
        || dev_alloc(ctx, &f.fsw_up, iface) || dev_alloc(ctx, &f.fsw_dn, iface)
        || dev_alloc(ctx, &f.flw_up, iface) || dev_alloc(ctx, &f.flw_dn, iface)
        || dev_alloc(ctx, &f.tau, 2 * cell) || dev_alloc(ctx, &f.ttemp, cell)
        || dev_alloc(ctx, &f.dtemp, cell) || dev_alloc(ctx, &f.qheat, cell)
        || dev_alloc(ctx, &f.insol, (size_t)Np) || dev_alloc(ctx, &f.insol_ann, (size_t)Np)
        || dev_alloc(ctx, &f.ASR, (size_t)Np) || dev_alloc(ctx, &f.OLR, (size_t)Np)
        || dev_alloc(ctx, &f.cos_zenith, (size_t)Np) || dev_alloc(ctx, &f.step, 1))
        return THORX_E_CUDA;
    RtStep st{};
    st.nstep         = r->first_step;
    st.r_orb         = 1.0; // Insolation member defaults (insolation.h:112-118)
    st.sin_decl      = 0.0;
    st.cos_decl      = 1.0;
    st.alpha         = 0.0;
    st.Qheat_scaling = 1.0;
    st.run           = 1;
    CK(cudaMemcpy(f.step, &st, sizeof(st), cudaMemcpyHostToDevice));
    auto& F         = ctx->fields;
    F["phtemp"]     = {&f.phtemp, nvi, 1};
    F["thtemp"]     = {&f.thtemp, nvi, 1};
    F["fsw_up"]     = {&f.fsw_up, nvi, 1};
    F["fsw_dn"]     = {&f.fsw_dn, nvi, 1};
    F["flw_up"]     = {&f.flw_up, nvi, 1};
    F["flw_dn"]     = {&f.flw_dn, nvi, 1};
    F["tau"]        = {&f.tau, nv, 2};
    F["ttemp"]      = {&f.ttemp, nv, 1};
    F["dtemp"]      = {&f.dtemp, nv, 1};
    F["DG_Qheat"]   = {&f.qheat, nv, 1};
    F["insol"]      = {&f.insol, 1, 1};
    F["insol_ann"]  = {&f.insol_ann, 1, 1};
    F["ASR"]        = {&f.ASR, 1, 1};
    F["OLR"]        = {&f.OLR, 1, 1};
    F["cos_zenith"] = {&f.cos_zenith, 1, 1};
    // a step graph captured before this call lacks the module: capture again on the next step
    if (ctx->graph_exec) {
        CK(cudaGraphExecDestroy(ctx->graph_exec));
        ctx->graph_exec = nullptr;
    }
    if (ctx->graph) {
        CK(cudaGraphDestroy(ctx->graph));
        ctx->graph = nullptr;
    }
    ctx->rt_enabled = true;
    return 0;
}

int thorx_rt_totals(thorx_ctx* ctx, double* asr, double* olr) {
    if (!ctx)
        return THORX_E_ARG;
    if (!asr || !olr)
        return fail(ctx, THORX_E_ARG, "thorx_rt_totals: null argument");
    if (!ctx->rt_enabled)
        return fail(ctx, THORX_E_STATE, "thorx_rt_totals: RT is not enabled");
    launch_device_sum(ctx->rt_f.ASR, ctx->g.N, ctx->gd_part, ctx->gd_out, ctx->stream);
    launch_device_sum(ctx->rt_f.OLR, ctx->g.N, ctx->gd_part, ctx->gd_out + 1, ctx->stream);
    CK(cudaGetLastError());
    double out[2];
    CK(cudaMemcpyAsync(out, ctx->gd_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *asr = out[0];
    *olr = out[1];
    return 0;
}

int thorx_set_precision(thorx_ctx* ctx, int precision) {
    if (!ctx)
        return THORX_E_ARG;
    if (precision != THORX_FP64 && precision != THORX_MIXED)
        return fail(ctx, THORX_E_ARG, "thorx_set_precision: THORX_FP64 or THORX_MIXED");
    const bool mixed = precision == THORX_MIXED;
    if (mixed != ctx->P.mixed) {
        if (ctx->graph_exec) {
            CK(cudaGraphExecDestroy(ctx->graph_exec));
            ctx->graph_exec = nullptr;
        }
        if (ctx->graph) {
            CK(cudaGraphDestroy(ctx->graph));
            ctx->graph = nullptr;
        }
        ctx->P.mixed = mixed;
    }
    return 0;
}

int thorx_conv_adj_enable(thorx_ctx* ctx, int iterations, int soft_adjustment) {
    if (!ctx)
        return THORX_E_ARG;
    if (iterations < 0)
        return fail(ctx, THORX_E_ARG, "thorx_conv_adj_enable: negative iteration count");
    ctx->P.conv_adj_iter = iterations;
    ctx->P.conv_soft     = soft_adjustment != 0;
    if (ctx->graph_exec) { // the captured step holds the previous parameters
        CK(cudaGraphExecDestroy(ctx->graph_exec));
        ctx->graph_exec = nullptr;
    }
    if (ctx->graph) {
        CK(cudaGraphDestroy(ctx->graph));
        ctx->graph = nullptr;
    }
    return 0;
}

int thorx_sponge_enable(thorx_ctx* ctx, const thorx_sponge_params* p) {
    if (!ctx)
        return THORX_E_ARG;
    const Geometry& g = ctx->g;
    if (p) {
        if (p->nlat_bins < 1)
            return fail(ctx, THORX_E_ARG, "thorx_sponge_enable: nlat_bins must be >= 1");
        if (!(p->ns_ray_sponge >= 0.0 && p->ns_ray_sponge < 1.0))
            return fail(ctx, THORX_E_ARG, "thorx_sponge_enable: ns_ray_sponge outside [0, 1)");
        if (p->raysp_calc_mode < 0 || p->raysp_calc_mode > 2)
            return fail(ctx, THORX_E_ARG, "thorx_sponge_enable: raysp_calc_mode not 0, 1 or 2");
    }
    // the step graph holds the previous set-up: drop it, then release that set-up's tables
    CK(cudaStreamSynchronize(ctx->stream));
    if (ctx->graph_exec) {
        CK(cudaGraphExecDestroy(ctx->graph_exec));
        ctx->graph_exec = nullptr;
    }
    if (ctx->graph) {
        CK(cudaGraphDestroy(ctx->graph));
        ctx->graph = nullptr;
    }
    {
        Sponge& old = ctx->sp;
        for (const void* q : {(const void*)old.bin, (const void*)old.start, (const void*)old.members,
                              (const void*)old.trig, (const void*)old.vbar, (const void*)old.Tbar,
                              (const void*)old.step})
            dev_free(ctx, q);
        old = Sponge{};
    }
    if (p) {
        const int N = g.N, Np = g.Np, nv = g.nv, nlat = p->nlat_bins;
        // latitude bins as Icogrid::zonal_mean_tab_f (src/ESP/grid.cu:3203-3260): bin j holds
        // lat_array[j] <= lat < lat_array[j + 1], the edges accumulated from -pi/2 in steps of
        // pi / nlat; lat >= lat_array[nlat] goes to the last bin. A latitude below -pi/2 (which
        // the reference leaves without a slot) goes to bin 0.
        std::vector<double> lat(Np), lat_array(nlat + 1);
        CK(cudaMemcpy(lat.data(), g.lat, Np * sizeof(double), cudaMemcpyDeviceToHost));
        const double des_lat = M_PI / nlat;
        lat_array[0]         = -M_PI / 2.0;
        for (int j = 1; j < nlat + 1; j++)
            lat_array[j] = lat_array[j - 1] + des_lat;
        std::vector<int> bin(Np, 0), start(nlat + 1, 0), members(N), fill(nlat, 0);
        for (int c = 0; c < N; c++) {
            int b = 0;
            for (int j = 0; j < nlat; j++)
                if (lat[c] >= lat_array[j] && lat[c] < lat_array[j + 1]) {
                    b = j;
                    break;
                }
            if (lat[c] >= lat_array[nlat])
                b = nlat - 1;
            bin[c] = b;
            start[b + 1]++;
        }
        for (int j = 0; j < nlat; j++)
            start[j + 1] += start[j];
        for (int c = 0; c < N; c++)
            members[start[bin[c]] + fill[bin[c]]++] = c;
        Sponge sp{};
        int *  dbin, *dstart, *dmem;
        double *trig, *vbar, *Tbar;
        if (dev_alloc(ctx, &dbin, (size_t)Np) || dev_alloc(ctx, &dstart, (size_t)nlat + 1)
            || dev_alloc(ctx, &dmem, (size_t)N) || dev_alloc(ctx, &trig, (size_t)4 * Np)
            || dev_alloc(ctx, &vbar, (size_t)3 * nlat * nv) || dev_alloc(ctx, &Tbar, (size_t)nlat * nv)
            || dev_alloc(ctx, &sp.step, 1))
            return THORX_E_CUDA;
        CK(cudaMemcpy(dbin, bin.data(), Np * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dstart, start.data(), (nlat + 1) * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dmem, members.data(), N * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemset(vbar, 0, (size_t)3 * nlat * nv * sizeof(double)));
        CK(cudaMemset(Tbar, 0, (size_t)nlat * nv * sizeof(double)));
        const SpongeStep st0{p->first_step, 1.0};
        CK(cudaMemcpy(sp.step, &st0, sizeof(st0), cudaMemcpyHostToDevice));
        launch_sponge_trig(g, trig, ctx->stream);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(ctx->stream));
        sp.nlat     = nlat;
        sp.Ruv      = p->Ruv_sponge;
        sp.Rw       = p->Rw_sponge;
        sp.RT       = p->RT_sponge;
        sp.ns       = p->ns_ray_sponge;
        sp.uv_mean  = p->damp_uv_to_mean != 0;
        sp.w_mean   = p->damp_w_to_mean != 0;
        sp.temp     = p->RayleighSpongeT != 0;
        sp.shrink   = p->shrink_sponge != 0;
        sp.t_shrink = p->t_shrink;
        sp.mode     = p->raysp_calc_mode;
        sp.bin      = dbin;
        sp.start    = dstart;
        sp.members  = dmem;
        sp.trig     = trig;
        sp.vbar     = vbar;
        sp.Tbar     = Tbar;
        ctx->sp     = sp;
    }
    else
        ctx->sp.nlat = 0;
    // an explicit sponge leaves its tendencies in profx_dMh / profx_dWh: start from zero
    CK(cudaMemset(ctx->s.dMh, 0, sizeof(double) * 3 * g.nv * g.Np));
    CK(cudaMemset(ctx->s.dWh, 0, sizeof(double) * g.nvi * g.Np));
    return 0;
}

int thorx_sponge_means(thorx_ctx* ctx, double* vbar, double* Tbar) {
    if (!ctx)
        return THORX_E_ARG;
    const Sponge& sp = ctx->sp;
    if (sp.nlat == 0)
        return fail(ctx, THORX_E_STATE, "thorx_sponge_means: the sponge is off");
    const int nlat = sp.nlat, nv = ctx->g.nv;
    CK(cudaStreamSynchronize(ctx->stream));
    if (vbar) {
        std::vector<double> t((size_t)3 * nlat * nv);
        CK(cudaMemcpy(t.data(), sp.vbar, t.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int k = 0; k < 3; k++)
            for (int b = 0; b < nlat; b++)
                for (int lev = 0; lev < nv; lev++)
                    vbar[((size_t)b * nv + lev) * 3 + k] = t[((size_t)k * nlat + b) * nv + lev];
    }
    if (Tbar)
        CK(cudaMemcpy(Tbar, sp.Tbar, (size_t)nlat * nv * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

// ---- RT surrogate ------------------------------------------------------------------------------
namespace {
int sur_check(thorx_ctx* ctx, const char* fn) {
    if (!ctx->sur)
        return fail(ctx, THORX_E_STATE, std::string(fn) + ": no surrogate (thorx_surrogate_create)");
    return 0;
}
int sur_err(thorx_ctx* ctx, const char* fn) {
    unsigned int e = 0;
    CK(cudaMemcpyAsync(&e, ctx->sur->err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (e)
        return fail(ctx, THORX_E_CUDA, std::string(fn) + ": tensor-core wait timed out");
    return 0;
}
// Host rows -> a device copy the caller frees (test entry points only).
int stage_host(thorx_ctx* ctx, const float* h, size_t n, float** d) {
    CK(cudaMalloc(d, n * 4));
    CK(cudaMemcpyAsync(*d, h, n * 4, cudaMemcpyHostToDevice, ctx->stream));
    return 0;
}
} // namespace

int thorx_surrogate_create(thorx_ctx* ctx, const thorx_surrogate_params* sp) {
    if (!ctx)
        return THORX_E_ARG;
    if (!sp)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_create: null argument");
    if (ctx->sur)
        return fail(ctx, THORX_E_STATE, "thorx_surrogate_create: already created");
    if (sp->hidden < 256 || sp->hidden % 256 || sp->train_batch < 128 || sp->log_capacity < 0
        || sp->recheck_period < 1 || !(sp->tolerance > 0))
        return fail(ctx, THORX_E_ARG,
                    "thorx_surrogate_create: hidden must be a positive multiple of 256, "
                    "train_batch >= 128, log_capacity >= 0, recheck_period >= 1, tolerance > 0");
    Surrogate* S   = new Surrogate;
    S->period      = sp->recheck_period;
    S->tol         = sp->tolerance;
    const int rows = std::max(sp->train_batch, ctx->g.N);
    const int rc   = S->init(ctx->g.nv, sp->hidden, sp->log_capacity, rows, ctx->g.N, sp->seed);
    if (rc) {
        S->release();
        delete S;
        return fail(ctx, THORX_E_CUDA, "thorx_surrogate_create: device allocation failed");
    }
    ctx->sur = S;
    return 0;
}

int thorx_surrogate_set_mode(thorx_ctx* ctx, int mode) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_set_mode")))
        return rc;
    if (mode != THORX_SUR_OFF && mode != THORX_SUR_LOG && mode != THORX_SUR_USE
        && mode != THORX_SUR_USE_LOG)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_set_mode: unknown mode");
    if (mode != THORX_SUR_OFF && !ctx->rt_enabled)
        return fail(ctx, THORX_E_STATE, "thorx_surrogate_set_mode: RT is not enabled");
    if ((mode == THORX_SUR_LOG || mode == THORX_SUR_USE_LOG) && ctx->sur->log.cap == 0)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_set_mode: log_capacity is 0");
    const bool using_now = sur_using(ctx);
    const bool use       = mode == THORX_SUR_USE || mode == THORX_SUR_USE_LOG;
    if (use && !ctx->sur->norm_fitted)
        return fail(ctx, THORX_E_STATE, "thorx_surrogate_set_mode: the surrogate is not trained");
    if (use && !using_now) // entering the surrogate mode: no column has fallen back yet
        CK(cudaMemsetAsync(ctx->sur->fallback, 0, ctx->g.N, ctx->stream));
    if (mode != ctx->sur_mode && (rc = drop_graph(ctx)))
        return rc;
    ctx->sur_mode = mode;
    return 0;
}

long long thorx_surrogate_logged(thorx_ctx* ctx) {
    if (!ctx || !ctx->sur)
        return THORX_E_ARG;
    long long n = 0;
    if (cudaMemcpyAsync(&n, ctx->sur->log.count, 8, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess
        || cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        return fail(ctx, THORX_E_CUDA, "thorx_surrogate_logged: copy failed");
    return n;
}

int thorx_surrogate_train(thorx_ctx* ctx, int iterations, int batch, double lr, double* loss_first,
                          double* loss_last) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_train")))
        return rc;
    Surrogate* S = ctx->sur;
    if (iterations < 1 || batch < 128 || batch % 128 || batch > S->Bcap || !(lr > 0))
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_train: bad iterations, batch or lr");
    const long long logged = thorx_surrogate_logged(ctx);
    if (logged < batch)
        return fail(ctx, THORX_E_STATE, "thorx_surrogate_train: fewer logged columns than a batch");
    const long long nrows = std::min(logged, S->log.cap);
    if (!S->norm_fitted) {
        S->fit_normalisation(nrows, ctx->stream);
        S->norm_fitted = true;
    }
    std::vector<double> part;
    auto batch_loss = [&](double* out) -> int {
        part.resize(S->lpart_n);
        CK(cudaMemcpyAsync(part.data(), S->lpart, part.size() * 8, cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        double t = 0;
        for (double v : part)
            t += v;
        *out = t / ((double)batch * S->net.nv);
        return 0;
    };
    for (int it = 0; it < iterations; it++) {
        S->train_batch(nrows, batch, (float)lr, ctx->stream);
        CK(cudaGetLastError());
        if (it == 0 && loss_first && (rc = batch_loss(loss_first)))
            return rc;
    }
    if (loss_last && (rc = batch_loss(loss_last)))
        return rc;
    return sur_err(ctx, "thorx_surrogate_train");
}

int thorx_surrogate_stats(thorx_ctx* ctx, unsigned int* out) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_stats")))
        return rc;
    if (!out)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_stats: null argument");
    CK(cudaMemcpyAsync(out, ctx->sur->stats, 16, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemsetAsync(ctx->sur->stats, 0, 16, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int thorx_surrogate_layer(thorx_ctx* ctx, int layer, int* N, int* K, float* W, float* b, int set) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_layer")))
        return rc;
    if (layer < 0 || layer > 3)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_layer: layer out of range");
    SurLayer& L = ctx->sur->lay[layer];
    if (N)
        *N = L.N;
    if (K)
        *K = L.K;
    const size_t         nw   = (size_t)L.N * L.K;
    const cudaMemcpyKind kind = set ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    if (W)
        CK(cudaMemcpyAsync(set ? (void*)L.W : (void*)W, set ? (const void*)W : (const void*)L.W,
                           nw * 4, kind, ctx->stream));
    if (b)
        CK(cudaMemcpyAsync(set ? (void*)L.b : (void*)b, set ? (const void*)b : (const void*)L.b,
                           L.N * 4, kind, ctx->stream));
    if (set)
        ctx->sur->cast_all(ctx->stream);
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int thorx_surrogate_layer_grad(thorx_ctx* ctx, int layer, float* gW, float* gb) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_layer_grad")))
        return rc;
    if (layer < 0 || layer > 3)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_layer_grad: layer out of range");
    SurLayer& L = ctx->sur->lay[layer];
    if (gW)
        CK(cudaMemcpyAsync(gW, L.gW, (size_t)L.N * L.K * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (gb)
        CK(cudaMemcpyAsync(gb, L.gb, L.N * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int thorx_surrogate_normalisation(thorx_ctx* ctx, float* in_mean, float* in_std, float* out_mean,
                                  float* out_std, int set) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_normalisation")))
        return rc;
    if (!in_mean || !in_std || !out_mean || !out_std)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_normalisation: null argument");
    SurNet&              n    = ctx->sur->net;
    const cudaMemcpyKind kind = set ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    struct Pair {
        float* d;
        float* h;
        int    c;
    } ps[] = {{n.in_mean, in_mean, n.n_in},
              {n.in_std, in_std, n.n_in},
              {n.out_mean, out_mean, n.nv},
              {n.out_std, out_std, n.nv}};
    for (auto& x : ps)
        CK(cudaMemcpyAsync(set ? (void*)x.d : (void*)x.h, set ? (const void*)x.h : (const void*)x.d,
                           (size_t)x.c * 4, kind, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (set)
        ctx->sur->norm_fitted = true;
    return 0;
}

int thorx_surrogate_forward_host(thorx_ctx* ctx, const float* x, int B, float* y) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_forward_host")))
        return rc;
    Surrogate* S = ctx->sur;
    if (!x || !y || B < 1 || B > S->Bcap)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_forward_host: bad arguments");
    const int Bp = ((B + 127) / 128) * 128;
    float*    dx = nullptr;
    if ((rc = stage_host(ctx, x, (size_t)B * S->net.n_in, &dx)))
        return rc;
    S->load_host_batch(dx, nullptr, B, ctx->stream);
    S->forward(Bp, ctx->stream);
    std::vector<float> Y((size_t)Bp * S->net.Nout);
    CK(cudaMemcpyAsync(Y.data(), S->Y, Y.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(dx);
    for (int r = 0; r < B; r++)
        for (int j = 0; j < S->net.nv; j++)
            y[(size_t)r * S->net.nv + j] = Y[(size_t)r * S->net.Nout + j];
    return sur_err(ctx, "thorx_surrogate_forward_host");
}

int thorx_surrogate_gradients_host(thorx_ctx* ctx, const float* x, const float* t, int B,
                                   double* loss) {
    if (!ctx)
        return THORX_E_ARG;
    int rc;
    if ((rc = sur_check(ctx, "thorx_surrogate_gradients_host")))
        return rc;
    Surrogate* S = ctx->sur;
    if (!x || !t || B < 128 || B % 128 || B > S->Bcap)
        return fail(ctx, THORX_E_ARG, "thorx_surrogate_gradients_host: B must be a multiple of 128");
    float *dx = nullptr, *dt = nullptr;
    if ((rc = stage_host(ctx, x, (size_t)B * S->net.n_in, &dx))
        || (rc = stage_host(ctx, t, (size_t)B * S->net.nv, &dt)))
        return rc;
    S->load_host_batch(dx, dt, B, ctx->stream);
    S->forward(B, ctx->stream);
    S->backward(B, ctx->stream);
    std::vector<double> part(S->lpart_n);
    CK(cudaMemcpyAsync(part.data(), S->lpart, part.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(dx), cudaFree(dt);
    if (loss) {
        double sum = 0;
        for (double v : part)
            sum += v;
        *loss = sum / ((double)B * S->net.nv);
    }
    return sur_err(ctx, "thorx_surrogate_gradients_host");
}

int thorx_globdiag(thorx_ctx* ctx, double* out) {
    if (!ctx)
        return THORX_E_ARG;
    if (ctx->partitioned)
        return fail(ctx, THORX_E_UNSUPPORTED, "global sums need the whole state, not a partition");
    if (!out)
        return fail(ctx, THORX_E_ARG, "thorx_globdiag: null argument");
    if (!ctx->state_set)
        return fail(ctx, THORX_E_STATE, "thorx_globdiag: the state has not been set");
    launch_globdiag(ctx->g, ctx->P, ctx->s, ctx->gd_part, ctx->gd_out, ctx->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->gd_out, 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int thorx_globdiag_fields(thorx_ctx* ctx, double* out, double* const fields[6]) {
    if (!ctx)
        return THORX_E_ARG;
    if (ctx->partitioned)
        return fail(ctx, THORX_E_UNSUPPORTED, "global sums need the whole state, not a partition");
    if (!out || !fields)
        return fail(ctx, THORX_E_ARG, "thorx_globdiag_fields: null argument");
    if (!ctx->state_set)
        return fail(ctx, THORX_E_STATE, "thorx_globdiag_fields: the state has not been set");
    // the hyperdiffusion scratch (12 cell planes, idle between steps) holds the six planes
    double* cells = ctx->s.diff;
    launch_globdiag(ctx->g, ctx->P, ctx->s, ctx->gd_part, ctx->gd_out, ctx->stream, cells);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->gd_out, 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    const int    N = ctx->g.N, Np = ctx->g.Np, nv = ctx->g.nv;
    const size_t plane = (size_t)nv * Np;
    dim3         grid((N + 31) / 32, (nv + 31) / 32), block(32, 8);
    for (int q = 0; q < 6; q++) {
        if (!fields[q])
            continue;
        dev_to_ref_kernel<<<grid, block, 0, ctx->stream>>>(cells + q * plane, ctx->staging, N, Np,
                                                          nv, 1);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(fields[q], ctx->staging, (size_t)N * nv * sizeof(double),
                           cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream)); // the staging buffer is reused by the next plane
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int thorx_device_sum(const double* x, long long n, void* stream, double* out) {
    int rc = check_sum_args("thorx_device_sum", x, n, out);
    if (rc || n == 0)
        return rc;
    cudaStream_t    st = (cudaStream_t)stream;
    const long long np = device_sum_partials(n);
    double2*        part = nullptr;
    cudaError_t     e    = cudaMalloc(&part, (size_t)(np + 1) * sizeof(double2));
    if (e != cudaSuccess)
        return free_fail(THORX_E_CUDA, std::string("thorx_device_sum: cudaMalloc: ") + cudaGetErrorString(e));
    double* res = (double*)(part + np);
    launch_device_sum(x, n, part, res, st);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    cudaError_t ef = cudaFree(part);
    if (e == cudaSuccess)
        e = ef;
    if (e != cudaSuccess)
        return free_fail(THORX_E_CUDA, std::string("thorx_device_sum: ") + cudaGetErrorString(e));
    return 0;
}

int thorx_device_sum_noalloc(const double* x, long long n, void* stream, double* out) {
    const char* fn = "thorx_device_sum_noalloc";
    if (n > noalloc_sum_max_n())
        return free_fail(THORX_E_ARG, std::string(fn) + ": n = " + std::to_string(n)
                                          + " exceeds the fixed scratch limit of "
                                          + std::to_string(noalloc_sum_max_n())
                                          + " doubles; use thorx_device_sum");
    int rc = check_sum_args(fn, x, n, out);
    if (rc || n == 0)
        return rc;
    double2*    part   = nullptr;
    double*     result = nullptr;
    cudaError_t e      = noalloc_sum_scratch(&part, &result);
    if (e != cudaSuccess)
        return free_fail(THORX_E_CUDA, std::string(fn) + ": scratch set-up (cudaGetSymbolAddress): "
                                           + cudaGetErrorString(e));
    cudaStream_t st = (cudaStream_t)stream;
    launch_device_sum(x, n, part, result, st);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, result, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return free_fail(THORX_E_CUDA, std::string(fn) + ": " + cudaGetErrorString(e));
    return 0;
}

int thorx_check_division(long long n, unsigned long long seed, long long mismatches[2]) {
    const char* fn = "thorx_check_division";
    if (n < 0 || !mismatches)
        return free_fail(THORX_E_ARG, std::string(fn) + ": negative n or null output");
    unsigned long long* cnt = nullptr;
    unsigned long long  h[2] = {0, 0};
    cudaError_t         e    = cudaMalloc(&cnt, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMemset(cnt, 0, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess && n > 0) {
        launch_div_check(n, seed, cnt, 0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(h, cnt, sizeof h, cudaMemcpyDeviceToHost);
    if (cnt) {
        cudaError_t ef = cudaFree(cnt);
        if (e == cudaSuccess)
            e = ef;
    }
    if (e != cudaSuccess)
        return free_fail(THORX_E_CUDA, std::string(fn) + ": " + cudaGetErrorString(e));
    mismatches[0] = (long long)h[0];
    mismatches[1] = (long long)h[1];
    return 0;
}

int thorx_module_add(thorx_ctx* ctx, const thorx_module* m) {
    if (!ctx)
        return THORX_E_ARG;
    if (!m)
        return fail(ctx, THORX_E_ARG, "thorx_module_add: null module");
    if (ctx->modules.size() >= 8)
        return fail(ctx, THORX_E_ARG, "thorx_module_add: at most 8 modules");
    ctx->modules.push_back(*m);
    return drop_graph(ctx);
}

int thorx_rk_register_array(thorx_ctx* ctx, double* array, double* arrayk, double* arrayi,
                            int dimensions) {
    if (!ctx)
        return THORX_E_ARG;
    RkArrays& t = ctx->rk_arrays;
    if (!array || !arrayk || !arrayi || dimensions < 1)
        return fail(ctx, THORX_E_ARG, "thorx_rk_register_array: null array or dimensions < 1");
    if (t.n >= kMaxRkArrays)
        return fail(ctx, THORX_E_ARG, "thorx_rk_register_array: at most 10 arrays");
    t.array[t.n]  = array;
    t.arrayk[t.n] = arrayk;
    t.arrayi[t.n] = arrayi;
    t.count[t.n]  = (long long)dimensions * ctx->g.nv * ctx->g.Np;
    t.n++;
    return drop_graph(ctx);
}

int thorx_rk_register_array_n(thorx_ctx* ctx, double* array, double* arrayk, double* arrayi,
                              long long count) {
    if (!ctx)
        return THORX_E_ARG;
    RkArrays& t = ctx->rk_arrays;
    if (!array || !arrayk || !arrayi || count < 1)
        return fail(ctx, THORX_E_ARG, "thorx_rk_register_array_n: null array or count < 1");
    if (t.n >= kMaxRkArrays)
        return fail(ctx, THORX_E_ARG, "thorx_rk_register_array_n: at most 10 arrays");
    t.array[t.n]  = array;
    t.arrayk[t.n] = arrayk;
    t.arrayi[t.n] = arrayi;
    t.count[t.n]  = count;
    t.n++;
    return drop_graph(ctx);
}

int thorx_set_graph_mode(thorx_ctx* ctx, int use_graph) {
    if (!ctx)
        return THORX_E_ARG;
    ctx->eager = !use_graph;
    return drop_graph(ctx);
}

namespace {
// A field by name: the thorx_get_field fields, the dynamical core's stage, deviation and work
// arrays, and the module tendencies; false when unknown (or not allocated in this form).
bool find_field(thorx_ctx* ctx, const char* name, FieldDesc* out) {
    State&    s  = ctx->s;
    const int nv = ctx->g.nv;
    auto      it = ctx->fields.find(name);
    if (it != ctx->fields.end()) {
        *out = it->second;
        return *out->dev != nullptr;
    }
    const std::map<std::string, FieldDesc> stage = {
        {"Rhok", {&s.Rhok, nv, 1}},       {"Rhos", {&s.Rhos, nv, 1}},
        {"Mhk", {&s.Mhk, nv, 3}},         {"Mhs", {&s.Mhs, nv, 3}},
        {"Whk", {&s.Whk, nv + 1, 1}},     {"Whs", {&s.Whs, nv + 1, 1}},
        {"Wk", {&s.Wk, nv, 1}},           {"pressurek", {&s.pk, nv, 1}},
        {"pressures", {&s.ps, nv, 1}},    {"profx_dMh", {&s.dMh, nv, 3}},
        {"profx_dWh", {&s.dWh, nv + 1, 1}}, {"divg", {&s.divg, nv, 3}},
        {"diff", {&s.diff, nv, 12}},      {"Etotal", {&s.Etotal, nv, 1}},
        {"ep", {&s.ep, nv, 1}},           {"ek", {&s.ek, nv, 1}},
        {"eph", {&s.eph, nv + 1, 1}},     {"ekh", {&s.ekh, nv + 1, 1}}};
    auto jt = stage.find(name);
    if (jt == stage.end())
        return false;
    *out = jt->second;
    if (jt->first == "divg" && kDivgF32 && ctx->P.mixed)
        out->esize = 4;
    return *out->dev != nullptr;
}

extern "C++" { // templates: C++ linkage inside the C ABI block
template<class T>
__global__ void copy_columns_kernel(T* __restrict__ dst, const T* __restrict__ src,
                                    const int* __restrict__ cols, int n, int Q, int Np) {
    const long long total = (long long)n * Q;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int    q = (int)(t / n), i = (int)(t % n);
        const size_t k = (size_t)q * Np + cols[i];
        dst[k]         = src[k];
    }
}
// pack (dir 0): buf[i][q] = field[q][cols[i]]; unpack (dir 1): the reverse (the buffer holds
// doubles; an FP32 field's values convert exactly both ways)
template<class T>
__global__ void pack_columns_kernel(T* __restrict__ field, double* __restrict__ buf,
                                    const int* __restrict__ cols, int n, int Q, int Np, int dir) {
    const long long total = (long long)n * Q;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int    q = (int)(t / n), i = (int)(t % n);
        const size_t k = (size_t)q * Np + cols[i];
        if (dir == 0)
            buf[(size_t)i * Q + q] = field[k];
        else
            field[k] = (T)buf[(size_t)i * Q + q];
    }
}
} // extern "C++"
unsigned column_blocks(long long total) {
    return (unsigned)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 16));
}
} // namespace

int thorx_device_field(thorx_ctx* ctx, const char* name, double** dev, int* levels,
                       int* components, long* plane) {
    if (!ctx)
        return THORX_E_ARG;
    if (!name || !dev)
        return fail(ctx, THORX_E_ARG, "thorx_device_field: null argument");
    if (!std::strcmp(name, "Rd") || !std::strcmp(name, "Cp")) { // a module may write them
        ctx->thermo_escaped = true;
        if (int rc = update_thermo(ctx))
            return rc;
    }
    FieldDesc f;
    if (!find_field(ctx, name, &f))
        return fail(ctx, THORX_E_ARG, std::string("thorx_device_field: unknown field ") + name);
    if (f.esize != 8)
        return fail(ctx, THORX_E_UNSUPPORTED,
                    std::string("thorx_device_field: ") + name + " holds FP32 values in the mixed form");
    *dev = *f.dev;
    if (levels)
        *levels = f.L;
    if (components)
        *components = f.K;
    if (plane)
        *plane = ctx->g.Np;
    return 0;
}

int thorx_set_partition(thorx_ctx* ctx, int col_begin, int col_end) {
    if (!ctx)
        return THORX_E_ARG;
    const int N = ctx->g.N;
    if (col_begin < 0 || col_end > N || col_begin >= col_end || col_begin % kColAlign
        || (col_end % kColAlign && col_end != N))
        return fail(ctx, THORX_E_ARG, "thorx_set_partition: the range must be whole 32-column "
                                      "tiles of the grid (the end may be point_num)");
    if (ctx->sp.nlat > 0 || ctx->sur || !ctx->modules.empty())
        return fail(ctx, THORX_E_UNSUPPORTED,
                    "thorx_set_partition: not with the sponge, the surrogate or modules");
    std::vector<int> sp;
    for (int c : ctx->special_all)
        if (c >= col_begin && c < col_end)
            sp.push_back(c);
    int* d_special;
    if (dev_alloc(ctx, &d_special, 32))
        return THORX_E_CUDA;
    if (!sp.empty())
        CK(cudaMemcpy(d_special, sp.data(), sp.size() * sizeof(int), cudaMemcpyHostToDevice));
    ctx->g.special     = d_special;
    ctx->g.nspecial    = (int)sp.size();
    ctx->g.tile0       = col_begin / kColAlign;
    ctx->g.ntile       = (col_end + kColAlign - 1) / kColAlign - ctx->g.tile0;
    ctx->g.col_end     = col_end;
    ctx->partitioned   = col_begin > 0 || col_end < N;
    return drop_graph(ctx);
}

int thorx_set_exchange(thorx_ctx* ctx, thorx_exchange_fn fn, void* user) {
    if (!ctx)
        return THORX_E_ARG;
    ctx->xfn   = fn;
    ctx->xuser = user;
    if (fn)
        ctx->eager = true;
    return drop_graph(ctx);
}

int thorx_halo_columns(const thorx_grid* gr, int col_begin, int col_end, int* cols, int cap) {
    if (!gr || !gr->maps || !gr->point_local || gr->point_num < 3 || cap < 0
        || col_begin < 0 || col_end > gr->point_num || col_begin >= col_end)
        return free_fail(THORX_E_ARG, "thorx_halo_columns: bad grid or range");
    const int            N = gr->point_num, Np = (N + kColAlign - 1) / kColAlign * kColAlign;
    std::vector<int>     nb, ring;
    std::vector<uint8_t> flag;
    const std::string    err = neighbour_tables(gr, Np, nb, ring, flag);
    if (!err.empty())
        return free_fail(THORX_E_ARG, "thorx_halo_columns: " + err);
    std::vector<char> need(N, 0);
    for (int c = col_begin; c < col_end; c++)
        for (int j = 0; j < 6; j++)
            for (const std::vector<int>* t : {&nb, &ring}) {
                const int v = (*t)[(size_t)j * Np + c];
                if (v >= 0 && (v < col_begin || v >= col_end))
                    need[v] = 1;
            }
    int n = 0;
    for (int c = 0; c < N; c++)
        if (need[c]) {
            if (cols && n < cap)
                cols[n] = c;
            n++;
        }
    return n;
}

int thorx_copy_columns(thorx_ctx* dst, thorx_ctx* src, const char* field, const int* dev_cols,
                       int n) {
    if (!dst || !src)
        return THORX_E_ARG;
    FieldDesc fd, fs;
    if (!field || n < 0 || (n > 0 && !dev_cols) || !find_field(dst, field, &fd)
        || !find_field(src, field, &fs) || dst->g.Np != src->g.Np || dst->g.nv != src->g.nv
        || fd.esize != fs.esize)
        return fail(dst, THORX_E_ARG, "thorx_copy_columns: bad arguments or field");
    if (n == 0)
        return 0;
    const int      Q  = fd.L * fd.K;
    const unsigned nb = column_blocks((long long)n * Q);
    if (fd.esize == 4)
        copy_columns_kernel<<<nb, 256, 0, dst->stream>>>(
            reinterpret_cast<float*>(*fd.dev), reinterpret_cast<const float*>(*fs.dev), dev_cols, n,
            Q, dst->g.Np);
    else
        copy_columns_kernel<<<nb, 256, 0, dst->stream>>>(*fd.dev, *fs.dev, dev_cols, n, Q,
                                                         dst->g.Np);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0
                            : fail(dst, THORX_E_CUDA,
                                   std::string("thorx_copy_columns: ") + cudaGetErrorString(e));
}

static int pack_unpack(thorx_ctx* ctx, const char* field, const int* dev_cols, int n,
                       double* dev_buf, int dir) {
    if (!ctx)
        return THORX_E_ARG;
    FieldDesc f;
    if (!field || n < 0 || (n > 0 && (!dev_cols || !dev_buf)) || !find_field(ctx, field, &f))
        return fail(ctx, THORX_E_ARG, "thorx_pack_columns: bad arguments or field");
    if (n == 0)
        return 0;
    const int      Q  = f.L * f.K;
    const unsigned nb = column_blocks((long long)n * Q);
    if (f.esize == 4)
        pack_columns_kernel<<<nb, 256, 0, ctx->stream>>>(reinterpret_cast<float*>(*f.dev), dev_buf,
                                                         dev_cols, n, Q, ctx->g.Np, dir);
    else
        pack_columns_kernel<<<nb, 256, 0, ctx->stream>>>(*f.dev, dev_buf, dev_cols, n, Q,
                                                         ctx->g.Np, dir);
    CK(cudaGetLastError());
    return 0;
}
int thorx_pack_columns(thorx_ctx* ctx, const char* field, const int* dev_cols, int n,
                       double* dev_buf) {
    return pack_unpack(ctx, field, dev_cols, n, dev_buf, 0);
}
int thorx_unpack_columns(thorx_ctx* ctx, const char* field, const int* dev_cols, int n,
                         const double* dev_buf) {
    return pack_unpack(ctx, field, dev_cols, n, const_cast<double*>(dev_buf), 1);
}

int thorx_vert_hydiff_enable(thorx_ctx* ctx, double Diffc_v, int order) {
    if (!ctx)
        return THORX_E_ARG;
    if (order != 0 && (order < 4 || order % 2))
        return fail(ctx, THORX_E_ARG, "thorx_vert_hydiff_enable: order must be even and >= 4");
    const int nv = ctx->g.nv;
    if (order && nv < 2)
        return fail(ctx, THORX_E_ARG, "thorx_vert_hydiff_enable: needs at least two levels");
    if (order) {
        // Kdv6 = Diffc_v dz^order / dt per level (src/ESP/esp_initial.cu:1327-1335)
        std::vector<double> k(nv);
        for (int lev = 0; lev < nv; lev++) {
            const double dz = ctx->Altitudeh_h[lev + 1] - ctx->Altitudeh_h[lev];
            k[lev]          = Diffc_v * pow(dz, 1.0 * order) / ctx->P.timestep;
        }
        double* d;
        if (!ctx->g.Kdv6) {
            if (dev_alloc(ctx, &d, nv))
                return THORX_E_CUDA;
            ctx->g.Kdv6 = d;
        }
        CK(cudaMemcpy((void*)ctx->g.Kdv6, k.data(), nv * sizeof(double), cudaMemcpyHostToDevice));
    }
    ctx->P.vhd_order = order;
    return drop_graph(ctx);
}

int thorx_check_thomas(thorx_ctx* ctx, double epsilon, double* max_rel, long long* n_bad) {
    if (!ctx)
        return THORX_E_ARG;
    if (!max_rel || !n_bad)
        return fail(ctx, THORX_E_ARG, "thorx_check_thomas: null output");
    const int     N = ctx->g.N;
    double*       colmax = nullptr;
    unsigned int* nbad   = nullptr;
    CK(cudaMalloc(&colmax, (size_t)N * sizeof(double)));
    cudaError_t e = cudaMalloc(&nbad, sizeof(unsigned int));
    if (e == cudaSuccess)
        e = cudaMemsetAsync(nbad, 0, sizeof(unsigned int), ctx->stream);
    if (e == cudaSuccess) {
        launch_thomas_residual(ctx->g, ctx->s, epsilon, colmax, nbad, ctx->stream);
        e = cudaGetLastError();
    }
    std::vector<double> h(N);
    unsigned int        hb = 0;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), colmax, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost,
                            ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&hb, nbad, sizeof(unsigned int), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(ctx->stream);
    cudaFree(colmax);
    if (nbad)
        cudaFree(nbad);
    if (e != cudaSuccess)
        return fail(ctx, THORX_E_CUDA, std::string("thorx_check_thomas: ") + cudaGetErrorString(e));
    double m = 0.0;
    for (double v : h)
        m = v > m ? v : m;
    *max_rel = m;
    *n_bad   = hb;
    return 0;
}

} // extern "C"
