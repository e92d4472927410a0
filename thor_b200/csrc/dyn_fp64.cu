// thorx dynamical-core kernels for sm_100a: the all-FP64 form and the mixed form.
//
// Each kernel is a fusion of reference kernels (file:line in the comment above it). In the FP64
// form the arithmetic of every fused piece follows the reference operation for operation (same
// operand order and association, same math-library calls; quotients by the cell areas come from
// a staged reciprocal but are the IEEE quotients, div_rcp), so that the only differences from the
// reference build are the FMA contractions the compiler chooses. The mixed form (template
// compute type float) runs the momentum-side stencils in FP32 and applies the hyperdiffusion and
// divergence-damping operators through per-column weights (stencil_weights_kernel).
//
// Work decomposition: every kernel except ProfX runs on tiles of 32 consecutive columns (one per
// lane, so that each plane access of a warp is one or two 128-byte lines) times all levels, the
// levels spread over kLevGroups warps (lane x = column, warp y = levels y, y+8, ...). What a
// column needs from the grid (stencil weights, ring geometry) is staged once per tile in shared
// memory, [quantity][32 columns], and shared by the 8 level groups.
// Where the reference carries values down a column loop (Compute_Temperature_H_Pt_Geff,
// Vertical_Eq, UpdateRK2) each level recomputes what it needs from the neighbouring levels
// instead, with the same operations, so that all levels run in parallel; only the Thomas
// elimination itself stays sequential, one warp per tile, overlapped with the other warps' work.
// Neighbours come from the per-column tables described in thorx_internal.h; a hole (-1) reads 0.
// Stencils are templated on the ring size (6, or 5 at pentagons and poles) so that every index
// is static and the ring values stay in registers.

#include <algorithm>
#include <mutex>
#include <type_traits>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "thorx.h"
#include "thorx_internal.h"

namespace thorx {
namespace {

#ifndef THORX_LEVGROUPS
#define THORX_LEVGROUPS 8
#endif
constexpr int kTile      = kTileCols;       // columns per tile (lanes)
constexpr int kLevGroups = THORX_LEVGROUPS; // warps per tile, each taking every kLevGroups-th level
constexpr int kColBlock  = 128;

// Register budget of each tiled kernel (__maxnreg__), chosen by timing the g6/L48 step on a B200
// (caps of 64, 72, 80, 96, 112, 128 and 160 for every kernel in both forms): the kernels are
// latency-bound, and a cap of 80 registers lets 3 CTAs of 256 threads (24 warps) share an SM where
// the uncapped code fits one or two; adv_temp does best at 72; the FP64 divm0 keeps 128 (2 CTAs),
// where tighter caps spill more than the extra warps win back, and the mixed form's divm0 (which
// applies operator weights) 96. Overridable with -DTHORX_REGS_<KERNEL>=n.
#ifndef THORX_REGS_ADV
#define THORX_REGS_ADV 72
#endif
#ifndef THORX_REGS_DIFF
#define THORX_REGS_DIFF 80
#endif
#ifndef THORX_REGS_DIVM
#define THORX_REGS_DIVM 128
#endif
#ifndef THORX_REGS_DIVM_MIXED
#define THORX_REGS_DIVM_MIXED 96
#endif
#ifndef THORX_REGS_SLOW
#define THORX_REGS_SLOW 80
#endif
#ifndef THORX_REGS_MOM
#define THORX_REGS_MOM 80
#endif
#ifndef THORX_REGS_VERT
#define THORX_REGS_VERT 80
#endif
#define THORX_KATTR_ADV __maxnreg__(THORX_REGS_ADV)
#define THORX_KATTR_DIFF __maxnreg__(THORX_REGS_DIFF)
#define THORX_KATTR_DIVM __maxnreg__(sizeof(R) < sizeof(double) ? THORX_REGS_DIVM_MIXED : THORX_REGS_DIVM)
#define THORX_KATTR_SLOW __maxnreg__(THORX_REGS_SLOW)
#define THORX_KATTR_MOM __maxnreg__(THORX_REGS_MOM)
#define THORX_KATTR_VERT __maxnreg__(THORX_REGS_VERT)

__device__ __forceinline__ double gz(const double* __restrict__ plane, int id) {
    return id >= 0 ? __ldg(plane + id) : 0.0;
}
__device__ __forceinline__ double gz(const float* __restrict__ plane, int id) {
    return id >= 0 ? (double)__ldg(plane + id) : 0.0;
}

// DeepModel ? A / (Altitude + A) : 1, from the level table that holds that expression's value
__device__ __forceinline__ double rscale_of(const Phys&, const Geometry& g, int lev) {
    return g.lt[kLtRscale * g.nvi + lev];
}

// Gas constant and heat capacity of a cell. kUni (Phys::uniform_thermo: every cell's Rd and Cp
// are Phys::Rd and Phys::Cp, which the context checks whenever the fields are set): the scalars, so
// the compiler folds the expressions built from them (Rd / (Cp - Rd) and the like) into per-thread
// constants; they are the same values, so the results are the same bits as the per-cell loads.
template<bool kUni> __device__ __forceinline__ double rd_at(const Phys& P, const State& s, int i) {
    if constexpr (kUni)
        return P.Rd;
    else
        return s.Rd[i];
}
template<bool kUni> __device__ __forceinline__ double cp_at(const Phys& P, const State& s, int i) {
    if constexpr (kUni)
        return P.Cp;
    else
        return s.Cp[i];
}

// Copies rows 0..Q-1 of a [q][Np] grid array for the tile's 32 columns into smem [q][32].
__device__ __forceinline__ void stage(double* sm, const double* __restrict__ src, int Q, int Np,
                                      int c0) {
    for (int q = threadIdx.y; q < Q; q += blockDim.y)
        sm[q * kTile + threadIdx.x] = __ldg(src + (size_t)q * Np + c0 + threadIdx.x);
}

// Column of lane x in a stencil kernel with a five-entry-ring tail CTA. The regular tiles cover
// columns c0..c0+31 and skip the 10 pentagons and 2 poles; the last CTA of the grid takes exactly
// those 12 columns (g.special), one per lane, with the n = 5 stencil code. Returns -1 for an
// idle lane.
__device__ __forceinline__ bool tail_cta() { return blockIdx.x == gridDim.x - 1; }
__device__ __forceinline__ int lane_column(const Geometry& g) {
    const int x = threadIdx.x;
    if (tail_cta())
        return x < g.nspecial ? g.special[x] : -1;
    const int c = (g.tile0 + blockIdx.x) * kTile + x;
    return (c < g.N && !(g.cflag[c] & kRing5)) ? c : -1;
}
// Copies rows 0..Q-1 of a [q][Np] grid array for the lanes' columns into smem [q][32].
__device__ __forceinline__ void stage_cols(double* sm, const double* __restrict__ src, int Q,
                                           int Np, int col) {
    for (int q = threadIdx.y; q < Q; q += blockDim.y)
        sm[q * kTile + threadIdx.x] = col >= 0 ? __ldg(src + (size_t)q * Np + col) : 0.0;
}

// a / b rounded to nearest, from y = 1/b rounded to nearest, with fused multiply-adds only.
// Markstein's theorem (P. W. Markstein, IBM J. Res. Develop. 34(1):111-119, 1990; J.-M. Muller et
// al., Handbook of Floating-Point Arithmetic, 2nd ed., 2018, sect. 4.7): if y = RN(1/b) and q is
// within one ulp of a/b, the remainder a - b q is exact in one fma and RN(q + (a - b q) y) =
// RN(a/b). q0 = RN(a y) is only within 1.5 ulp, so one correction step comes first. The result is
// the IEEE quotient a / b bit for bit while a, b, the quotient and the remainders are normal
// numbers (every field and grid quantity divided here); a zero numerator returns RN(a y), the
// signed zero a / b has. Used where one divisor (a cell's sub-triangle area) serves many divisions,
// so the one IEEE division of the reciprocal is paid once per column.
__device__ __forceinline__ double div_rcp(double a, double b, double y) {
    const double q0 = __dmul_rn(a, y);
    const double q1 = __fma_rn(__fma_rn(-q0, b, a), y, q0);
    const double q2 = __fma_rn(__fma_rn(-q1, b, a), y, q1);
    return a == 0.0 ? q0 : q2;
}
__device__ __forceinline__ float div_rcp(float a, float b, float y) {
    const float q0 = __fmul_rn(a, y);
    const float q1 = __fmaf_rn(__fmaf_rn(-q0, b, a), y, q0);
    const float q2 = __fmaf_rn(__fmaf_rn(-q1, b, a), y, q1);
    return a == 0.0f ? q0 : q2;
}

// Shared-memory view of one column's ring geometry, [quantity][32].
struct SGeo {
    const double *ar, *at, *ti, *te, *oa, *rat;
    int           x;
    __device__ double AR(int q) const { return ar[q * kTile + x]; }
    __device__ double AT(int q) const { return at[q * kTile + x]; }
    __device__ double TI(int q) const { return ti[q * kTile + x]; }
    __device__ double TE(int q) const { return te[q * kTile + x]; }
    __device__ double OA(int q) const { return oa[q * kTile + x]; }
    // 1 / areasTr rounded to nearest
    __device__ double RAT(int q) const { return rat[q * kTile + x]; }
    // the column's operator weights (Geometry::lapw, Geometry::dmw, dmw64), [entry][32]
    const double* lw;
    const float * lwf, *dm;
    const double* dm64;
};

// The mixed form (compute type float) applies the operators through per-column weights.
template<class R> constexpr bool kOperatorWeights = sizeof(R) < sizeof(double);
// Storage type of divg (kDivgF32): FP32 in the mixed form (glevel 6, 48 levels: momentum 1.03
// -> 0.97, divm0 1.13 -> 1.11, slow_modes 0.89 -> 0.87 ms per step, the same bits).
template<class R>
using DivgT = std::conditional_t<(kDivgF32 && sizeof(R) < sizeof(double)), float, double>;
// The FP64 form's hyperdiffusion and divergence damping through FP64 operator weights (the same
// linear operators as the reference's triangle sequences, summed in another order); 0 restores
// the reference's operation order.
#ifndef THORX_FP64_DIFF_WEIGHTS
#define THORX_FP64_DIFF_WEIGHTS 1
#endif
#ifndef THORX_FP64_DIVM_WEIGHTS
#define THORX_FP64_DIVM_WEIGHTS 1
#endif
constexpr bool kDiffWeightsF64 = THORX_FP64_DIFF_WEIGHTS != 0;
constexpr bool kDivmWeightsF64 = THORX_FP64_DIVM_WEIGHTS != 0;

// areas 18, areasTr 6, nvecti 18, nvecte 18, nvecoa 18, 1/areasTr 6
constexpr int kRingGeoRows = 84;
static_assert(7 * 8 + 7 * 4 <= kRingGeoRows * 8 && 84 * 4 <= kRingGeoRows * 8,
              "operator weights must fit the ring-geometry buffer");

__device__ __forceinline__ SGeo stage_ring_geo(double* sm, const Geometry& g, int col) {
    stage_cols(sm, g.areas, 18, g.Np, col);
    stage_cols(sm + 18 * kTile, g.areasTr, 6, g.Np, col);
    stage_cols(sm + 24 * kTile, g.nvecti, 18, g.Np, col);
    stage_cols(sm + 42 * kTile, g.nvecte, 18, g.Np, col);
    stage_cols(sm + 60 * kTile, g.nvecoa, 18, g.Np, col);
    for (int q = threadIdx.y; q < 6; q += blockDim.y) {
        // a pentagon's sixth entry is 0 and never read; its reciprocal (inf) is not either
        const double at = col >= 0 ? __ldg(g.areasTr + (size_t)q * g.Np + col) : 1.0;
        sm[(78 + q) * kTile + threadIdx.x] = 1.0 / at;
    }
    return SGeo{sm,       sm + 18 * kTile, sm + 24 * kTile, sm + 42 * kTile, sm + 60 * kTile,
                sm + 78 * kTile, (int)threadIdx.x, nullptr, nullptr, nullptr};
}

// Mixed form: the Laplacian weights of the lanes' columns in place of the ring geometry
// (double [7][32], then float [7][32]; fits the ring-geometry buffer).
__device__ __forceinline__ SGeo stage_lap_weights(double* sm, const Geometry& g, int col) {
    float* smf = reinterpret_cast<float*>(sm + 7 * kTile);
    for (int q = threadIdx.y; q < 7; q += blockDim.y) {
        const double w = col >= 0 ? __ldg(g.lapw + (size_t)q * g.Np + col) : 0.0;
        sm[q * kTile + threadIdx.x]  = w;
        smf[q * kTile + threadIdx.x] = (float)w;
    }
    SGeo G{};
    G.x   = threadIdx.x;
    G.lw  = sm;
    G.lwf = smf;
    return G;
}
// Mixed form: the divergence-damping weights, float [84][32] (fits the ring-geometry buffer).
__device__ __forceinline__ SGeo stage_divm_weights(double* sm, const Geometry& g, int col) {
    float* smf = reinterpret_cast<float*>(sm);
    for (int q = threadIdx.y; q < 84; q += blockDim.y)
        smf[q * kTile + threadIdx.x] = col >= 0 ? __ldg(g.dmw + (size_t)q * g.Np + col) : 0.0f;
    SGeo G{};
    G.x  = threadIdx.x;
    G.dm = smf;
    return G;
}
// FP64 form: the divergence-damping weights in double, [84][32] (the size of the ring geometry).
__device__ __forceinline__ SGeo stage_divm_weights64(double* sm, const Geometry& g, int col) {
    for (int q = threadIdx.y; q < 84; q += blockDim.y)
        sm[q * kTile + threadIdx.x] = col >= 0 ? __ldg(g.dmw64 + (size_t)q * g.Np + col) : 0.0;
    SGeo G{};
    G.x    = threadIdx.x;
    G.dm64 = sm;
    return G;
}
// What a kernel with divergence damping stages: float weights (mixed form), double weights or the
// ring geometry (FP64 form).
template<class R>
__device__ __forceinline__ SGeo stage_divm_geo(double* sm, const Geometry& g, int col) {
    if constexpr (kOperatorWeights<R>)
        return stage_divm_weights(sm, g, col);
    else if constexpr (kDivmWeightsF64)
        return stage_divm_weights64(sm, g, col);
    else
        return stage_ring_geo(sm, g, col);
}


// ---------------------------------------------------------------------------------------------
// Per-level tables (LevelTable in thorx_internal.h), one thread per level/interface index. The
// expressions are those the kernels evaluate per cell in the reference (same calls, same operand
// order), so a table entry is the value each cell would have computed.
// ---------------------------------------------------------------------------------------------
__global__ void level_tables_kernel(Geometry g, Phys P, double* lt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nv = g.nv, nvi = g.nvi;
    if (i > nv)
        return;
    const double  A    = P.A;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    for (int t = 0; t < kLtCount; t++)
        lt[t * nvi + i] = 0.0;
    // interfaces (thor_vertical_int.h:188-420, thor_fastmodes.h:617-633, thor_adv_cor.h:330-336)
    lt[kLtR2hD * nvi + i] = pow(Alth[i] + A, 2.0);
    lt[kLtR2hI * nvi + i] = pow(Alth[i] + A, 2);
    lt[kLtOr2 * nvi + i]  = 1 / pow(Alth[i] + A, 2);
    lt[kLtTor3 * nvi + i] = 2 / pow(Alth[i] + A, 3);
    if (i >= 1 && i <= nv - 1) {
        const double dzp        = 1.0 / (Alth[i + 1] - Alth[i]);
        const double dzh        = 1.0 / (Alt[i] - Alt[i - 1]);
        const double dzm        = 1.0 / (Alth[i] - Alth[i - 1]);
        lt[kLtDzp * nvi + i]    = dzp;
        lt[kLtDzh * nvi + i]    = dzh;
        lt[kLtDzm * nvi + i]    = dzm;
        lt[kLtIntl * nvi + i]   = (Alt[i] - Alth[i]) * dzp * dzh;
        lt[kLtInttm * nvi + i]  = -(Alt[i - 1] - Alth[i]) * dzm * dzh;
        lt[kLtHIntt * nvi + i]  = (Alth[i] - Alt[i]) / (Alt[i - 1] - Alt[i]);
        lt[kLtHIntl * nvi + i]  = (Alth[i] - Alt[i - 1]) / (Alt[i] - Alt[i - 1]);
    }
    // layer centres
    if (i < nv) {
        lt[kLtRscale * nvi + i] = P.DeepModel ? P.A / (Alt[i] + P.A) : 1.0;
        lt[kLtR2cD * nvi + i]   = pow(Alt[i] + A, 2.0);
        lt[kLtDr2dz * nvi + i]  = (pow(Alth[i + 1] + A, 3.0) - pow(Alth[i] + A, 3.0)) / 3.0;
        lt[kLtGhv * nvi + i]    = pow(A / (A + Alt[i]), 2);
        lt[kLtCIntt * nvi + i]  = (Alt[i] - Alth[i + 1]) / (Alth[i] - Alth[i + 1]);
        lt[kLtCIntl * nvi + i]  = (Alt[i] - Alth[i]) / (Alth[i + 1] - Alth[i]);
        lt[kLtRDz * nvi + i]    = 1.0 / (Alth[i + 1] - Alth[i]);
        lt[kLtRDr2dz * nvi + i] = 1.0 / lt[kLtDr2dz * nvi + i];
        lt[kLtRDzR2m * nvi + i] = 1.0 / ((Alth[i + 1] - Alth[i]) * lt[kLtR2cD * nvi + i]);
    }
}

// ---------------------------------------------------------------------------------------------
// ProfX: Recompute_W (reference src/headers/phy/profx_auxiliary.h:109-130), Compute_temperature
// (:64-92), the dry convective adjustment when enabled (above), the benchmark forcing (held_suarez,
// src/headers/phy/profx_held_suarez.h:51-117; tidalearth; shallowHJ), Compute_pressure (:94-107)
// and the NaN check on temperature (:132-146, src/ESP/profx_driver.cu:389-396,451-458).
// One thread per column (1% of a step).
// ---------------------------------------------------------------------------------------------
// ---------------------------------------------------------------------------------------------
// Dry convective adjustment of one column, dry_conv_adj (src/headers/phy/dry_conv_adj.h:50-311),
// the reference's operation sequence: potential temperature referred to the extrapolated surface
// pressure; repeatedly the lowest unstable layer is found, the unstable stretch above it mixed to
// the enthalpy-weighted mean (extended while the mean is unstable against the layer below or
// above), then T and p recomputed; at most conv_adj_iter rounds. The interface pressures the
// reference also stores are not used on this path and not written. The potential temperature
// uses the pt plane as scratch (the dynamical core recomputes it before reading it). The
// reference's loops end by construction; here each is also bounded (a mixing pass per layer, an
// extension per layer), and a column that reaches a bound sets kFlagConvAdj and stops.
// ---------------------------------------------------------------------------------------------
__device__ void conv_adj_column(const Geometry& g, const Phys& P, const State& s, int c) {
    const int     Np = g.Np, nv = g.nv;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    const double  stable = 0.0;
    double*       pt  = s.pt;
    double*       T   = s.T;
    double*       p   = s.p;
    const double* rho = s.Rho;
    const double* Rd  = s.Rd;
    const double* Cp  = s.Cp;
    auto          at  = [&](int lev) { return lev * Np + c; };
    int           iter   = 0;
    bool          repeat = true;
    while (repeat && iter < P.conv_adj_iter) {
        double psm;
        if (P.GravHeightVar)
            psm = p[at(1)] - rho[at(0)] * P.Gravit * pow(P.A / (P.A + Alt[0]), 2) * (-Alt[0] - Alt[1]);
        else
            psm = p[at(1)] - rho[at(0)] * P.Gravit * (-Alt[0] - Alt[1]);
        const double ps = 0.5 * (p[at(0)] + psm);
        for (int lev = 0; lev < nv; lev++)
            pt[at(lev)] = T[at(lev)] * pow(ps / p[at(lev)], Rd[at(lev)] / Cp[at(lev)]);
        bool done_col = false;
        int  passes   = 0;
        while (!done_col) {
            if (++passes > 2 * nv + 2) {
                atomicOr(s.flags, kFlagConvAdj);
                return;
            }
            int top = 0, bot = nv - 1;
            for (int lev = 0; lev < nv - 1; lev++)
                if (pt[at(lev + 1)] - pt[at(lev)] < stable && bot > lev)
                    bot = lev;
            for (int lev = bot; lev < nv - 1; lev++) {
                if (pt[at(lev + 1)] - pt[at(lev)] > stable) {
                    top = lev;
                    break;
                }
                top = nv - 1;
            }
            if (bot < nv - 1) {
                bool   extend = true;
                int    ext    = 0;
                double thnew  = 0.0;
                while (extend) {
                    if (++ext > nv + 2) {
                        atomicOr(s.flags, kFlagConvAdj);
                        return;
                    }
                    double h = 0.0, sum = 0.0;
                    extend   = false;
                    for (int lev = bot; lev <= top; lev++) {
                        const double pi = pow(p[at(lev)] / ps, Rd[at(lev)] / Cp[at(lev)]);
                        const double rho_g_dz = rho[at(lev)] * P.Gravit * (Alth[lev + 1] - Alth[lev]);
                        h   = h + pt[at(lev)] * pi * rho_g_dz;
                        sum = sum + pi * rho_g_dz;
                    }
                    thnew = h / sum;
                    if (bot > 0 && (thnew - pt[at(bot - 1)]) < stable) {
                        bot    = bot - 1;
                        extend = true;
                    }
                    if (top < nv - 1 && (pt[at(top + 1)] - thnew) < stable) {
                        top    = top + 1;
                        extend = true;
                    }
                }
                for (int lev = bot; lev <= top; lev++)
                    pt[at(lev)] = thnew;
            }
            else
                done_col = true;
        }
        repeat = false;
        iter += 1;
        if (P.conv_soft) {
            for (int lev = 0; lev < nv; lev++) {
                const int    i    = at(lev);
                const double Ttmp = pt[i] * pow(p[i] / ps, Rd[i] / Cp[i]);
                const double Ptmp = Ttmp * Rd[i] * rho[i];
                pt[i]             = T[i] * pow(p[i] / ps, -Rd[i] / Cp[i]);
                s.Qheat[i] += (Cp[i] - Rd[i]) / Rd[i] * (Ptmp - p[i]) / P.timestep;
            }
        }
        else {
            for (int lev = 0; lev < nv; lev++) {
                const int i = at(lev);
                T[i]        = pt[i] * pow(p[i] / ps, Rd[i] / Cp[i]);
                p[i]        = T[i] * Rd[i] * rho[i];
                pt[i]       = T[i] * pow(p[i] / ps, -Rd[i] / Cp[i]);
                if (lev > 0 && pt[i] - pt[at(lev - 1)] < stable)
                    repeat = true;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Rayleigh sponge, implicit form (sponge_layer with implicit = true, src/ESP/profx_sponge.cu:144-431,
// and the zonal means of zonal_uv / zonal_w / zonal_temp, :50-130, summed per bin and level by
// gpu_sum_on_device_sponge, src/headers/reduction_add.h:242-288). Columns are binned by latitude
// at set-up (Icogrid::zonal_mean_tab_f, src/ESP/grid.cu:3203-3260). The means kernel takes one
// CTA per (bin, level) and sums the bin's members in a fixed order (thread-strided, then a fixed
// tree), so the means are deterministic; W is recomputed from Wh there with Recompute_W's
// arithmetic, as the reference's means read W after Recompute_W.
// ---------------------------------------------------------------------------------------------
constexpr int kSpongeThreads = 256;

__global__ void sponge_trig_kernel(Geometry g, double* trig) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int Np  = g.Np;
    double    lon = g.lon[c];
    if (lon < 0)
        lon = lon + 2.0 * M_PI;
    trig[c]          = sin(lon);
    trig[Np + c]     = cos(lon);
    trig[2 * Np + c] = sin(g.lat[c]);
    trig[3 * Np + c] = cos(g.lat[c]);
}

__global__ void __launch_bounds__(kSpongeThreads) sponge_means_kernel(Geometry g, Phys P,
                                                                      Sponge sp, SpongeIn in) {
    const int b = blockIdx.x, lev = blockIdx.y;
    if (in.advance && b == 0 && lev == 0 && threadIdx.x == 0) { // step factor (profx_driver.cu:154-160)
        const long long n  = sp.step->nstep;
        const double    dt = P.timestep;
        double          rv = 1;
        if (sp.shrink && n * dt >= sp.t_shrink * dt) {
            const double shrink_scale = dt * 1000;
            rv = exp(-(n * dt - sp.t_shrink * dt) / shrink_scale);
        }
        sp.step->rv_fac = rv;
        sp.step->nstep  = n + 1;
    }
    if (!(sp.uv_mean || sp.w_mean || sp.temp))
        return;
    const int     Np = g.Np, nv = g.nv;
    const int     m0 = sp.start[b], m1 = sp.start[b + 1];
    const double  cnt  = (double)(m1 - m0);
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    const double  xi = Alt[lev], xim = Alth[lev], xip = Alth[lev + 1];
    const double  intt = (xi - xip) / (xim - xip);
    const double  intl = (xi - xim) / (xip - xim);
    double        acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int m = m0 + threadIdx.x; m < m1; m += kSpongeThreads) {
        const int    c   = sp.members[m];
        const int    i   = lev * Np + c;
        const double rho = in.Rho[i];
        if (sp.uv_mean) {
            const double slon = sp.trig[c], clon = sp.trig[Np + c];
            const double slat = sp.trig[2 * Np + c], clat = sp.trig[3 * Np + c];
            const double mx = in.M[i], my = in.M[nv * Np + i], mz = in.M[2 * nv * Np + i];
            const double u = (mx * (-slon) + my * (clon) + mz * 0) / rho;
            const double v = (mx * (-slat * clon) + my * (-slat * slon) + mz * (clat)) / rho;
            acc[0] += u / cnt;
            acc[1] += v / cnt;
        }
        if (sp.w_mean) {
            const double w = in.W ? in.W[i]
                                  : in.Wh[lev * Np + c] * intt + in.Wh[(lev + 1) * Np + c] * intl;
            acc[2] += (w / rho) / cnt;
        }
        if (sp.temp)
            acc[3] += in.p[i] / in.Rd[i] / rho / cnt;
    }
    __shared__ double red[kSpongeThreads / 32][4];
    const int         lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double x = acc[q];
        for (int o = 16; o > 0; o >>= 1)
            x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0)
            red[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        const int q   = threadIdx.x;
        double    sum = 0.0;
        for (int w = 0; w < kSpongeThreads / 32; w++)
            sum += red[w][q];
        if (q < 3)
            sp.vbar[(q * sp.nlat + b) * nv + lev] = sum;
        else
            sp.Tbar[b * nv + lev] = sum;
    }
}

// The implicit sponge on one column: winds toward the zonal mean of the column's latitude
// (interpolated between the two nearest bin centres; the polar halves of the outermost bins take
// their bin's mean), with the rate Rv_fac R sin^2(pi/2 (z/ztop - ns) / (1 - ns)) above ns; then
// Wh at the interior interfaces from the new W; with the thermal sponge, p from the relaxed T.
struct SpongeLat { // the means at a column's latitude: bin b's, or wa x bin ba + wb x bin bb
    bool   interp;
    int    b, ba, bb;
    double wa, wb;
    __device__ double mean(const double* tab, int nv, int lev) const {
        return interp ? tab[ba * nv + lev] * wa + tab[bb * nv + lev] * wb : tab[b * nv + lev];
    }
};
__device__ SpongeLat sponge_lat(const Geometry& g, const Sponge& sp, int c) {
    const int     nlat    = sp.nlat;
    const int     b       = sp.bin[c];
    const double  des_lat = M_PI / nlat;
    const double  lat1    = -M_PI / 2 + 0.5 * des_lat + des_lat * (b - 1);
    const double  lat2    = -M_PI / 2 + 0.5 * des_lat + des_lat * (b);
    const double  lat3    = -M_PI / 2 + 0.5 * des_lat + des_lat * (b + 1);
    const double  lat     = g.lat[c];
    // which means, and their weights: (ba, bb, wa, wb); interp = false takes bin b's mean. A
    // latitude outside both half-intervals of its bin (only rounding at a bin edge can give one;
    // the reference leaves the mean unset there) takes its bin's mean too.
    bool   interp = false;
    int    ba = b, bb = b;
    double wa = 0.0, wb = 0.0;
    if (lat <= -M_PI / 2 + 0.5 * des_lat) {
    }
    else if (lat >= -M_PI / 2 + 0.5 * des_lat + des_lat * (nlat - 1)) {
    }
    else if (lat >= lat1 && lat < lat2) {
        interp = true;
        ba = b - 1;
        wa = (lat - lat2) / (lat1 - lat2);
        wb = (lat - lat1) / (lat2 - lat1);
    }
    else if (lat >= lat2 && lat < lat3) {
        interp = true;
        bb = b + 1;
        wa = (lat - lat3) / (lat2 - lat3);
        wb = (lat - lat2) / (lat3 - lat2);
    }
    return SpongeLat{interp, b, ba, bb, wa, wb};
}

__device__ void sponge_column(const Geometry& g, const Phys& P, const Sponge& sp, const State& s,
                              int c) {
    const int       Np = g.Np, nv = g.nv, nlat = sp.nlat;
    const double*   Alt  = g.Altitude;
    const double*   Alth = g.Altitudeh;
    const double    ztop = Alth[nv];
    const double    dt   = P.timestep;
    const double    rv   = sp.step->rv_fac;
    const double    slon = sp.trig[c], clon = sp.trig[Np + c];
    const double    slat = sp.trig[2 * Np + c], clat = sp.trig[3 * Np + c];
    const SpongeLat L    = sponge_lat(g, sp, c);
    auto            mean = [&](const double* tab, int lev) { return L.mean(tab, nv, lev); };
    const double* ubar = sp.vbar;
    const double* vbar = sp.vbar + nlat * nv;
    const double* wbar = sp.vbar + 2 * nlat * nv;
    for (int lev = 0; lev < nv; lev++) {
        const int    i   = lev * Np + c;
        const double rho = s.Rho[i];
        const double mx = s.Mh[i], my = s.Mh[nv * Np + i], mz = s.Mh[2 * nv * Np + i];
        const double u = (mx * (-slon) + my * (clon) + mz * 0) / rho;
        const double v = (mx * (-slat * clon) + my * (-slat * slon) + mz * (clat)) / rho;
        const double w = s.W[i] / rho;
        const double n = Alt[lev] / ztop;
        double       kuv = 0.0, kw = 0.0, kvT = 0.0;
        if (n >= sp.ns) {
            const double sn = pow(sin(0.5 * M_PI * (n - sp.ns) * (1.0) / (1.0 - sp.ns)), 2.0);
            kuv             = rv * sp.Ruv * sn;
            kw              = rv * sp.Rw * sn;
            kvT             = rv * sp.RT * sn;
        }
        double unew, vnew, wnew;
        if (sp.uv_mean) {
            unew = (u / dt + kuv * mean(ubar, lev)) / (1.0 / dt + kuv);
            vnew = (v / dt + kuv * mean(vbar, lev)) / (1.0 / dt + kuv);
        }
        else {
            unew = (u / dt) / (1.0 / dt + kuv);
            vnew = (v / dt) / (1.0 / dt + kuv);
        }
        if (sp.w_mean)
            wnew = (w / dt + kw * mean(wbar, lev)) / (1.0 / dt + kw);
        else
            wnew = (w / dt) / (1.0 / dt + kw);
        const double vx = unew * (-slon) + vnew * (-slat * clon);
        const double vy = unew * (clon) + vnew * (-slat * slon);
        const double vz = vnew * (clat);
        s.Mh[i]              = vx * rho;
        s.Mh[nv * Np + i]     = vy * rho;
        s.Mh[2 * nv * Np + i] = vz * rho;
        s.W[i]               = wnew * rho;
        if (sp.temp) {
            const double temperature = s.p[i] / s.Rd[i] / rho;
            s.p[i] = rho * s.Rd[i] * (temperature / dt + kvT * mean(sp.Tbar, lev)) / (1.0 / dt + kvT);
        }
    }
    const int nvi = g.nvi;
    for (int lev = 1; lev < nv; lev++) {
        const double intt = g.lt[kLtHIntt * nvi + lev], intl = g.lt[kLtHIntl * nvi + lev];
        s.Wh[lev * Np + c] = s.W[(lev - 1) * Np + c] * intt + s.W[lev * Np + c] * intl;
    }
}

// The explicit sponge (sponge_layer with implicit = false, raysp_calc_mode exp1 / exp3,
// src/ESP/thor_driver.cu:749-866) on the RK stage's fields: the damping rates become tendencies,
// profx_dMh (horizontal momentum), profx_dWh (the vertical one, interpolated to the interior
// interfaces; zero at the bottom and the top) and, with the thermal sponge, heating added to
// profx_Qheat (which the reference does not reset between RK stages either). One thread per column.
__global__ void __launch_bounds__(kColBlock) sponge_explicit_kernel(Geometry g, Phys P, Sponge sp,
                                                                   State s) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int       Np = g.Np, nv = g.nv, nvi = g.nvi;
    const double*   Alt  = g.Altitude;
    const double    ztop = g.Altitudeh[nv];
    const double    rv   = sp.step->rv_fac;
    const double    slon = sp.trig[c], clon = sp.trig[Np + c];
    const double    slat = sp.trig[2 * Np + c], clat = sp.trig[3 * Np + c];
    const SpongeLat L    = sponge_lat(g, sp, c);
    const double*   ubar = sp.vbar;
    const double*   vbar = sp.vbar + sp.nlat * nv;
    const double*   wbar = sp.vbar + 2 * sp.nlat * nv;
    double          dw_prev = 0.0;
    s.dWh[c]                = 0.0;
    s.dWh[nv * Np + c]      = 0.0;
    for (int lev = 0; lev < nv; lev++) {
        const int    i   = lev * Np + c;
        const double rho = s.Rhok[i];
        const double mx = s.Mhk[i], my = s.Mhk[nv * Np + i], mz = s.Mhk[2 * nv * Np + i];
        const double u = (mx * (-slon) + my * (clon) + mz * 0) / rho;
        const double v = (mx * (-slat * clon) + my * (-slat * slon) + mz * (clat)) / rho;
        const double w = s.Wk[i] / rho;
        const double n = Alt[lev] / ztop;
        double       kuv = 0.0, kw = 0.0, kvT = 0.0;
        if (n >= sp.ns) {
            const double sn = pow(sin(0.5 * M_PI * (n - sp.ns) * (1.0) / (1.0 - sp.ns)), 2.0);
            kuv             = rv * sp.Ruv * sn;
            kw              = rv * sp.Rw * sn;
            kvT             = rv * sp.RT * sn;
        }
        double du, dv, dw;
        if (sp.uv_mean) {
            du = -kuv * (u - L.mean(ubar, nv, lev));
            dv = -kuv * (v - L.mean(vbar, nv, lev));
        }
        else {
            du = -kuv * u;
            dv = -kuv * v;
        }
        const double vx = du * (-slon) + dv * (-slat * clon);
        const double vy = du * (clon) + dv * (-slat * slon);
        const double vz = dv * (clat);
        s.dMh[i]              = vx * rho;
        s.dMh[nv * Np + i]     = vy * rho;
        s.dMh[2 * nv * Np + i] = vz * rho;
        if (sp.w_mean)
            dw = -kw * (w - L.mean(wbar, nv, lev));
        else
            dw = -kw * (w);
        const double dW = dw * rho;
        if (lev > 0) {
            const double intt = g.lt[kLtHIntt * nvi + lev], intl = g.lt[kLtHIntl * nvi + lev];
            s.dWh[lev * Np + c] = dw_prev * intt + dW * intl;
        }
        dw_prev = dW;
        if (sp.temp) {
            const double temperature = s.pk[i] / s.Rd[i] / s.Rhok[i];
            const double dT          = -kvT * (temperature - L.mean(sp.Tbar, nv, lev));
            s.Qheat[i] += s.Rd[i] * s.Rhok[i] * dT;
        }
    }
}

// 32 columns x kProfxGroups level groups per block: the level-local parts run level-parallel
// (group y: levels y, y + kProfxGroups, ...); the column-serial ones (sponge, convective
// adjustment) run on group 0 between barriers.
constexpr int kProfxCols = 32, kProfxGroups = 8;
__global__ void __launch_bounds__(kProfxCols* kProfxGroups) profx_kernel(Geometry g, Phys P,
                                                                        Sponge sp, State s,
                                                                        bool finish) {
    const int  c     = (g.tile0 + blockIdx.x) * kProfxCols + threadIdx.x;
    const bool valid = c < g.N;
    const int  y0 = threadIdx.y, dy = kProfxGroups;
    const int     Np = g.Np, nv = g.nv;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    for (int lev = y0; valid && lev < nv; lev += dy) {
        double whl = s.Wh[lev * Np + c], wht = s.Wh[(lev + 1) * Np + c];
        double xi = Alt[lev], xim = Alth[lev], xip = Alth[lev + 1];
        double intt = (xi - xip) / (xim - xip);
        double intl = (xi - xim) / (xip - xim);
        s.W[lev * Np + c] = whl * intt + wht * intl;
    }
    if (sp.nlat > 0) { // after Recompute_W, before the temperature (profx_driver.cu:96-194)
        __syncthreads();
        if (valid && y0 == 0)
            sponge_column(g, P, sp, s, c);
        __syncthreads();
    }
    for (int lev = y0; valid && lev < nv; lev += dy) {
        int i  = lev * Np + c;
        s.T[i] = s.p[i] / (s.Rd[i] * s.Rho[i]);
    }
    if (P.conv_adj_iter > 0) { // after the temperature, before the forcing (profx_driver.cu:239-290)
        __syncthreads();
        if (valid && y0 == 0)
            conv_adj_column(g, P, s, c);
        __syncthreads();
    }

    if (P.held_suarez) {
        const double sigmab = 0.7, ka = (1.0 / 40.0) * (1.0 / 86400.0), kf = 1.0 / 86400.0;
        const double ks = (1.0 / 4.0) * (1.0 / 86400.0), kappa = P.Rd / P.Cp, dTy = 60.0,
                     dthetaz = 10.0, p0 = 100000.0;
        const double lat  = g.lat[c];
        const double psm1 = s.p[Np + c] - s.Rho[c] * P.Gravit * (-Alt[0] - Alt[1]);
        const double ps   = 0.5 * (s.p[c] + psm1);
        for (int lev = y0; valid && lev < nv; lev += dy) {
            int    i      = lev * Np + c;
            double pre    = s.p[i];
            double sigma  = (pre / ps);
            double sigma0 = (pre / p0);
            double Teq    = fmax(200.0, (315.0 - dTy * pow(sin(lat), 2.0)
                                      - dthetaz * log(sigma0) * pow(cos(lat), 2.0))
                                         * pow(sigma0, kappa));
            double kt = ka
                        + (ks - ka) * fmax(0.0, (sigma - sigmab) / (1.0 - sigmab))
                              * pow(cos(lat), 4.0);
            double kv = kf * fmax(0.0, (sigma - sigmab) / (1.0 - sigmab));
            for (int k = 0; k < 3; k++) {
                int j   = (k * nv + lev) * Np + c;
                s.Mh[j] = s.Mh[j] / (1.0 + kv * P.timestep);
            }
            s.T[i] -= kt * P.timestep * (s.T[i] - Teq);
        }
    }
    else if (P.benchmark == THORX_TIDALLY_LOCKED_EARTH) {
        // tidalearth (src/headers/phy/profx_tidalearth.h:49-126): Held-Suarez with the
        // equilibrium temperature of Heng, Menou & Phillips (2011), eq. 21, centred on the
        // substellar point (longitude pi)
        const double sigmab = 0.7, ka = (1.0 / 40.0) * (1.0 / 86400.0), kf = 1.0 / 86400.0;
        const double ks = (1.0 / 4.0) * (1.0 / 86400.0), kappa = P.Rd / P.Cp, dTy = 60.0,
                     dthetaz = 10.0, p0 = 100000.0;
        const double lat  = g.lat[c], lon = g.lon[c];
        const double psm1 = s.p[Np + c] - s.Rho[c] * P.Gravit * (-Alt[0] - Alt[1]);
        const double ps   = 0.5 * (s.p[c] + psm1);
        for (int lev = y0; valid && lev < nv; lev += dy) {
            int    i      = lev * Np + c;
            double pre    = s.p[i];
            double sigma  = (pre / ps);
            double sigma0 = (pre / p0);
            double Teq    = fmax(200.0, (315.0 + dTy * cos(lon - M_PI) * cos(lat)
                                      - dthetaz * log(sigma0) * pow(cos(lat), 2.0))
                                         * pow(sigma0, kappa));
            double kt = ka
                        + (ks - ka) * fmax(0.0, (sigma - sigmab) / (1.0 - sigmab))
                              * pow(cos(lat), 4.0);
            double kv = kf * fmax(0.0, (sigma - sigmab) / (1.0 - sigmab));
            for (int k = 0; k < 3; k++) {
                int j   = (k * nv + lev) * Np + c;
                s.Mh[j] = s.Mh[j] / (1.0 + kv * P.timestep);
            }
            s.T[i] -= kt * P.timestep * (s.T[i] - Teq);
        }
    }
    else if (P.benchmark == THORX_SHALLOW_HOT_JUPITER) {
        // shallowHJ (src/headers/phy/profx_shallowHJ.h:50-128): Newtonian cooling towards the
        // hot-Jupiter profile of Heng, Menou & Phillips (2011), eqs. 23-25; no friction
        const double dTy = 300.0, zstra = 2e6, sigma_stra = 0.12, Gamma_trop = 2e-4,
                     T_surf = 1600, Delta_Tstra = 10;
        const double lat  = g.lat[c], lon = g.lon[c];
        const double psm1 = s.p[Np + c] - s.Rho[c] * P.Gravit * (-Alt[0] - Alt[1]);
        const double ps   = 0.5 * (s.p[c] + psm1);
        for (int lev = y0; valid && lev < nv; lev += dy) {
            int    i     = lev * Np + c;
            double sigma = (s.p[i] / ps);
            double beta_trop, T_vert;
            if (Alt[lev] <= zstra) {
                beta_trop = sin(0.5 * M_PI * (sigma - sigma_stra) / (1.0 - sigma_stra));
                T_vert    = T_surf - Gamma_trop * (zstra + 0.5 * (Alt[lev] - zstra))
                         + sqrt(pow(0.5 * Gamma_trop * (Alt[lev] - zstra), 2)
                                + Delta_Tstra * Delta_Tstra);
            }
            else {
                beta_trop = 0.0;
                T_vert    = T_surf - Gamma_trop * zstra + Delta_Tstra;
            }
            const double Teq = T_vert + beta_trop * dTy * cos(lon - M_PI) * cos(lat);
            const double kt  = 1 / (1.5e5);
            const double kv  = 0.0;
            for (int k = 0; k < 3; k++) {
                int j   = (k * nv + lev) * Np + c;
                s.Mh[j] = s.Mh[j] / (1.0 + kv * P.timestep);
            }
            s.T[i] -= kt * P.timestep * (s.T[i] - Teq);
        }
    }
    if (!finish) // physics modules run before the pressure update (profx_driver.cu:405-416)
        return;
    __syncthreads(); // the forcings read p at levels 0 and 1 of the column before this writes p
    bool bad = false;
    for (int lev = y0; valid && lev < nv; lev += dy) {
        int i  = lev * Np + c;
        s.p[i] = s.T[i] * s.Rd[i] * s.Rho[i];
        bad |= isnan(s.T[i]);
    }
    if (bad)
        atomicOr(s.flags, kFlagNaN);
}

// Compute_pressure (profx_auxiliary.h:94-107) and the NaN check, after the physics modules.
__global__ void __launch_bounds__(kColBlock) profx_finish_kernel(Geometry g, State s) {
    const int c = g.tile0 * kTile + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.col_end)
        return;
    bool bad = false;
    for (int lev = 0; lev < g.nv; lev++) {
        int i  = lev * g.Np + c;
        s.p[i] = s.T[i] * s.Rd[i] * s.Rho[i];
        bad |= isnan(s.T[i]);
    }
    if (bad)
        atomicOr(s.flags, kFlagNaN);
}

// ---------------------------------------------------------------------------------------------
// Advection + Coriolis + thermodynamic diagnostics of one RK stage:
//   Compute_Advec_Cori1 / _Poles (src/headers/dyn/thor_adv_cor.h:51-362),
//   Compute_Advec_Cori2 (:366-536) and Compute_Temperature_H_Pt_Geff
//   (src/headers/dyn/thor_auxiliary.h:55-309, calcT = true).
// The cartesian velocity v of the reference is recomputed where it is used instead of stored.
// ---------------------------------------------------------------------------------------------
struct ColLevel { // thermodynamic quantities of one column at one level
    double p, rho, Rd, Cp;
};

template<bool kUni>
__device__ __forceinline__ ColLevel col_level(const Phys& P, const State& s, int Np, int lev, int c) {
    const int i = lev * Np + c;
    return ColLevel{s.pk[i], s.Rhok[i], rd_at<kUni>(P, s, i), cp_at<kUni>(P, s, i)};
}
// enthalpy h = Cv T + p / rho (thor_auxiliary.h:111,130,140)
__device__ __forceinline__ double enthalpy(const ColLevel& q) {
    const double Cv = q.Cp - q.Rd;
    const double T  = q.p / (q.rho * q.Rd);
    return Cv * T + q.p / q.rho;
}
// potential temperature (thor_auxiliary.h:111-112,163)
__device__ __forceinline__ double pot_temp(const ColLevel& q, double P_Ref) {
    const double Cv    = q.Cp - q.Rd;
    const double CvoCp = Cv / q.Cp;
    return (P_Ref / (q.Rd * q.rho)) * pow(q.p / P_Ref, CvoCp);
}

template<bool kUni>
__global__ void THORX_KATTR_ADV adv_temp_kernel(Geometry g, Phys P, State s) {
    __shared__ double sdiv[21 * kTile];
    __shared__ double sfr[21 * kTile]; // func_r of the 7 stencil points, [point * 3 + k][32]
    const int         c0 = (g.tile0 + blockIdx.x) * kTile, x = threadIdx.x, c = c0 + x;
    const int         Np = g.Np, nv = g.nv;
    stage(sdiv, g.div, 21, Np, c0);
    for (int q = threadIdx.y; q < 21; q += blockDim.y) {
        const int j = q / 3, k = q % 3;
        int       id = -1;
        if (c < g.N)
            id = j == 0 ? c : g.nb[(j - 1) * Np + c];
        sfr[q * kTile + x] = gz(g.func_r + k * Np, id);
    }
    __syncthreads();
    if (c >= g.N)
        return;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    const double  A = P.A, Omega = P.Omega, P_Ref = P.P_Ref, Gravit = P.Gravit;
    const bool    eeq = P.energy, ghv = P.GravHeightVar;

    const double* lt = g.lt;
    const int     nvi = g.nvi;
    int           nb[7];
    nb[0] = c;
    for (int j = 0; j < 6; j++)
        nb[j + 1] = g.nb[j * Np + c];
    auto fr = [&](int j, int k) { return sfr[(j * 3 + k) * kTile + x]; };
    // v = M / rho + (w / rho) r^, the quotients from one reciprocal of rho (div_rcp: IEEE quotients)
    auto vel = [&](const double* M, double rho, double w, int j, double* v) {
        const double yr = 1.0 / rho, wr = div_rcp(w, rho, yr);
        for (int k = 0; k < 3; k++)
            v[k] = div_rcp(M[k], rho, yr) + wr * fr(j, k);
    };
    auto vown = [&](int lev, double* v) {
        const double M[3] = {s.Mhk[(0 * nv + lev) * Np + c], s.Mhk[(1 * nv + lev) * Np + c],
                             s.Mhk[(2 * nv + lev) * Np + c]};
        vel(M, s.Rhok[lev * Np + c], s.Wk[lev * Np + c], 0, v);
    };
    // kinetic energy per mass of the column at a level (thor_auxiliary.h:152-157)
    auto ekin = [&](int lev) {
        const int    i  = lev * Np + c;
        const double m0 = s.Mhk[(0 * nv + lev) * Np + c], m1 = s.Mhk[(1 * nv + lev) * Np + c],
                     m2 = s.Mhk[(2 * nv + lev) * Np + c], w = s.Wk[i], r = s.Rhok[i];
        return 0.5 * (m0 * m0 + m1 * m1 + m2 * m2 + w * w) / (r * r);
    };
    auto epot = [&](int lev) {
        return ghv ? Gravit * lt[kLtGhv * nvi + lev] * Alt[lev] : Gravit * Alt[lev];
    };
    // velocity-weighted effective gravity at interior interface i (thor_auxiliary.h:288-289)
    auto gtil_w = [&](int i) -> double {
        if (i <= 0 || i >= nv)
            return 0.0;
        const ColLevel lo = col_level<kUni>(P, s, Np, i - 1, c), hi = col_level<kUni>(P, s, Np, i, c);
        const double   dz    = Alt[i] - Alt[i - 1];
        const double   dp_dz = (hi.p - lo.p) / dz;
        const double   intt = lt[kLtHIntt * nvi + i], intl = lt[kLtHIntl * nvi + i];
        const double   rhoh = lo.rho * intt + hi.rho * intl;
        return -(s.Whk[i * Np + c] / rhoh) * dp_dz;
    };

    for (int lev = threadIdx.y; lev < nv; lev += kLevGroups) {
        const int    i      = lev * Np + c;
        const double rscale = rscale_of(P, g, lev);
        // ---- horizontal flux divergence of v (x) M over the 7-point stencil: nine running sums
        // sum[kk][cc] over the points j in order, one point's M and v at a time ----
        double sum[3][3], vcur[3];
#pragma unroll
        for (int j = 0; j < 7; j++) {
            const int id = nb[j];
            double    M[3] = {0.0, 0.0, 0.0}, V[3] = {0.0, 0.0, 0.0};
            if (id >= 0) {
#pragma unroll
                for (int k = 0; k < 3; k++)
                    M[k] = s.Mhk[(k * nv + lev) * Np + id];
                vel(M, s.Rhok[lev * Np + id], s.Wk[lev * Np + id], j, V);
            }
            if (j == 0)
                for (int k = 0; k < 3; k++)
                    vcur[k] = V[k];
#pragma unroll
            for (int kk = 0; kk < 3; kk++)
#pragma unroll
                for (int cc = 0; cc < 3; cc++) {
                    const double t = sdiv[(j * 3 + kk) * kTile + x] * V[cc] * M[kk];
                    sum[kk][cc]    = (j == 0) ? t : sum[kk][cc] + t;
                }
        }
        double nflx[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int kk = 0; kk < 3; kk++)
#pragma unroll
            for (int cc = 0; cc < 3; cc++)
                nflx[cc] += rscale * sum[kk][cc];
        // ---- vertical flux of v w at the interfaces + Coriolis ----
        double        vprev[3] = {0, 0, 0}, vnext[3] = {0, 0, 0};
        const double  altht = Alth[lev + 1], althl = Alth[lev], alt = Alt[lev];
        double        dvwl[3] = {0, 0, 0}, dvwt[3] = {0, 0, 0};
        if (lev > 0) {
            vown(lev - 1, vprev);
            const double intt = lt[kLtHIntt * nvi + lev], intl = lt[kLtHIntl * nvi + lev];
            const double whl = s.Whk[lev * Np + c];
            for (int k = 0; k < 3; k++)
                dvwl[k] = (vprev[k] * intt + vcur[k] * intl) * whl;
        }
        if (lev < nv - 1) {
            vown(lev + 1, vnext);
            const double intt = lt[kLtHIntt * nvi + lev + 1], intl = lt[kLtHIntl * nvi + lev + 1];
            const double wht = s.Whk[(lev + 1) * Np + c];
            for (int k = 0; k < 3; k++)
                dvwt[k] = (vcur[k] * intt + vnext[k] * intl) * wht;
        }
        double r2p = 1.0, r2m = 1.0, r2l = 1.0;
        if (P.DeepModel) {
            r2p = lt[kLtR2hD * nvi + lev + 1];
            r2m = lt[kLtR2cD * nvi + lev];
            r2l = lt[kLtR2hD * nvi + lev];
        }
        const double dz  = 1.0 / ((althl - altht) * r2m);
        const double rho = s.Rhok[i];
        double       C[3];
        if (P.DeepModel) {
            C[0] = -2.0 * Omega * vcur[1] * rho;
            C[1] = 2.0 * Omega * vcur[0] * rho;
            C[2] = 0.0;
        }
        else {
            const double f[3] = {fr(0, 0), fr(0, 1), fr(0, 2)};
            C[0] = 2 * Omega * (vcur[2] * f[2] * f[1] - vcur[1] * pow(f[2], 2)) * rho;
            C[1] = -2 * Omega * (vcur[2] * f[2] * f[0] - vcur[0] * pow(f[2], 2)) * rho;
            C[2] = 2 * Omega * (vcur[1] * f[2] * f[0] - vcur[0] * f[2] * f[1]) * rho;
        }
        for (int k = 0; k < 3; k++) {
            const double dav               = (dvwl[k] * r2l - dvwt[k] * r2p) * dz;
            s.Adv[(k * nv + lev) * Np + c] = nflx[k] + (dav + C[k]);
        }

        // ---- Compute_Temperature_H_Pt_Geff at this level (and its interface below) ----
        const ColLevel q  = col_level<kUni>(P, s, Np, lev, c);
        const double   Cv = q.Cp - q.Rd;
        const double   T  = q.p / (q.rho * q.Rd);
        const double   h  = Cv * T + q.p / q.rho;
        s.T[i]            = T;
        s.h[i]            = h;
        double ep = 0, ek = 0, pt = 0;
        if (eeq) {
            ep          = epot(lev);
            ek          = ekin(lev);
            s.ep[i]     = ep;
            s.ek[i]     = ek;
            s.Etotal[i] = q.rho * (ep + ek) + Cv / q.Rd * q.p;
        }
        else {
            pt      = pot_temp(q, P_Ref);
            s.pt[i] = pt;
        }
        if (lev > 0) { // interior interface `lev`
            const ColLevel lo    = col_level<kUni>(P, s, Np, lev - 1, c);
            const double   dzl   = alt - Alt[lev - 1];
            const double   dp_dz = (q.p - lo.p) / dzl;
            const double   intt = lt[kLtHIntt * nvi + lev], intl = lt[kLtHIntl * nvi + lev];
            s.hh[i] = enthalpy(lo) * intt + h * intl;
            if (eeq) {
                s.eph[i] = epot(lev - 1) * intt + ep * intl;
                s.ekh[i] = ekin(lev - 1) * intt + ek * intl;
            }
            else
                s.pth[i] = pot_temp(lo, P_Ref) * intt + pt * intl;
            const double rhoh = lo.rho * intt + q.rho * intl;
            s.gtilh[i]        = -(1.0 / rhoh) * dp_dz;
        }
        else { // bottom boundary, extrapolated (thor_auxiliary.h:167-187)
            const ColLevel up   = col_level<kUni>(P, s, Np, 1, c);
            const double   extr = (-alt - Alt[1]) / (Alt[1] - alt);
            s.hh[c]             = h;
            double pl;
            if (ghv)
                pl = up.p - q.rho * Gravit * pow(A / (A + Alt[0]), 2) * (-alt - Alt[1]);
            else
                pl = up.p - q.rho * Gravit * (-alt - Alt[1]);
            const double rhol = up.rho + (up.rho - q.rho) * extr;
            const double rhoh = 0.5 * (q.rho + rhol);
            const double dzb  = 2.0 * Alt[0];
            const double dpdz = (q.p - pl) / dzb;
            s.gtilh[c]        = -(1.0 / rhoh) * dpdz;
        }
        // effective gravity at the layer centre (thor_auxiliary.h:293-300; :259-266 at the top,
        // where the reference interpolates with the top layer's own geometry)
        {
            const int    L1   = (lev < nv - 1) ? lev + 1 : lev;
            const double intt = lt[kLtCIntt * nvi + L1], intl = lt[kLtCIntl * nvi + L1];
            const double gw0  = gtil_w(lev);
            const double gw1  = (lev < nv - 1) ? gtil_w(lev + 1) : 0.0;
            s.gtil[i]         = gw0 * intt + gw1 * intl;
        }
        if (lev == nv - 1) { // top boundary and the bottom extrapolations (thor_auxiliary.h:188-258)
            const ColLevel lo2  = col_level<kUni>(P, s, Np, nv - 2, c);
            const ColLevel top  = q;
            const double   extr = (2 * Alth[nv] - alt - Alt[nv - 2]) / (Alt[nv - 1] - Alt[nv - 2]);
            s.hh[nv * Np + c]   = h;
            double pp;
            if (ghv)
                pp = lo2.p - top.rho * Gravit * pow(A / (A + Alt[nv]), 2) * (2 * Alth[nv] - alt - Alt[nv - 2]);
            else
                pp = lo2.p - top.rho * Gravit * (2 * Alth[nv] - alt - Alt[nv - 2]);
            if (pp < 0)
                pp = 0;
            const double rhop = lo2.rho + (top.rho - lo2.rho) * extr;
            const double rhoh = 0.5 * (top.rho + rhop);
            if (eeq) {
                if (ghv) {
                    s.eph[nv * Np + c] = Gravit * pow(A / (A + Alth[nv]), 2) * Alth[nv];
                    s.eph[c]           = Gravit * pow(A / (A + Alth[0]), 2) * Alth[0];
                }
                else {
                    s.eph[nv * Np + c] = Gravit * Alth[nv];
                    s.eph[c]           = Gravit * Alth[0];
                }
                const double ek2 = ekin(nv - 2), ek0 = ekin(0), ek1 = ekin(1);
                s.ekh[nv * Np + c] = ek2 + (ek - ek2) * extr;
                s.ekh[c]           = ek1 + (ek1 - ek0) * (Alth[0] - Alt[1]) / (Alt[1] - Alt[0]);
            }
            else {
                const double pt2 = pot_temp(lo2, P_Ref);
                const double pt0 = pot_temp(col_level<kUni>(P, s, Np, 0, c), P_Ref);
                const double pt1 = pot_temp(col_level<kUni>(P, s, Np, 1, c), P_Ref);
                s.pth[nv * Np + c] = pt2 + (pt - pt2) * extr;
                s.pth[c]           = pt1 + (pt1 - pt0) * (Alth[0] - Alt[1]) / (Alt[1] - Alt[0]);
            }
            const double dzt = 2.0 * (Alth[nv] - Alt[nv - 1]);
            double       pp2;
            if (ghv)
                pp2 = lo2.p - top.rho * Gravit * pow(A / (A + Alt[nv - 1]), 2)
                                  * (2 * Alth[nv] - Alt[nv - 1] - Alt[nv - 2]);
            else
                pp2 = lo2.p - top.rho * Gravit * (2 * Alth[nv] - Alt[nv - 1] - Alt[nv - 2]);
            const double dpdz    = (pp2 - top.p) / dzt;
            s.gtilh[nv * Np + c] = -(1.0 / rhoh) * dpdz;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// FV Laplacian around a ring of n neighbours (Diffusion_Op, src/headers/dyn/thor_diff.h:306-451;
// the pole kernel :735-820 is the same sequence with a five-entry ring).
// ---------------------------------------------------------------------------------------------
template<int n, class R>
__device__ __forceinline__ R laplacian(const SGeo& G, const R* a, R a0, R rscale) {
    static_assert(sizeof(R) == sizeof(double), "the FP32 stencils apply the operator weights");
    auto AR = [&](int q) { return (R)G.AR(q); };
    auto AT = [&](int q) { return (R)G.AT(q); };
    auto TI = [&](int q) { return (R)G.TI(q); };
    auto TE = [&](int q) { return (R)G.TE(q); };
    auto OA = [&](int q) { return (R)G.OA(q); };
    auto RAT = [&](int q) { return G.RAT(q); };
    const R h = (R)0.5;
    R       lap = 0;
    R       lap1 = 0, lap2 = 0, lap3 = 0, lapx1 = 0, lapx2 = 0, lapy1 = 0, lapy2 = 0, lapz1 = 0,
      lapz2 = 0, AT1 = 0;
#pragma unroll
    for (int j = 0; j < n; j++) {
        const int jp1 = (j + 1) % n, jp2 = (j + 2) % n;
        const R   p1 = a[j], p2 = a[jp1], p3 = a[jp2];
        const R   vdiff = h * rscale;
        R         astar;
        if (j == 0) {
            AT1   = div_rcp(rscale, AT(j), RAT(j));
            astar = div_rcp(AR(j * 3 + 0) * a0 + AR(j * 3 + 1) * p1 + AR(j * 3 + 2) * p2, AT(j), RAT(j));
            lap1  = (h * (p1 + a0) - astar);
            lap2  = (h * (p1 + p2) - astar);
            lap3  = (h * (a0 + p2) - astar);
        }
        const R AT2 = div_rcp(rscale, AT(jp1), RAT(jp1));
        astar = div_rcp(AR(jp1 * 3 + 0) * a0 + AR(jp1 * 3 + 1) * p2 + AR(jp1 * 3 + 2) * p3, AT(jp1), RAT(jp1));
        const R lap4 = (h * (a0 + p2) - astar);
        const R lap5 = (h * (p2 + p3) - astar);
        const R lap6 = (h * (a0 + p3) - astar);
        if (j == 0) {
            lapx1 = (-lap1 * TI(j * 3 + 0) + lap2 * TE(j * 3 + 0) + lap3 * TI(jp1 * 3 + 0)) * AT1;
            lapy1 = (-lap1 * TI(j * 3 + 1) + lap2 * TE(j * 3 + 1) + lap3 * TI(jp1 * 3 + 1)) * AT1;
            lapz1 = (-lap1 * TI(j * 3 + 2) + lap2 * TE(j * 3 + 2) + lap3 * TI(jp1 * 3 + 2)) * AT1;
        }
        else {
            lapx1 = lapx2;
            lapy1 = lapy2;
            lapz1 = lapz2;
        }
        lapx2 = (-lap4 * TI(jp1 * 3 + 0) + lap5 * TE(jp1 * 3 + 0) + lap6 * TI(jp2 * 3 + 0)) * AT2;
        lapy2 = (-lap4 * TI(jp1 * 3 + 1) + lap5 * TE(jp1 * 3 + 1) + lap6 * TI(jp2 * 3 + 1)) * AT2;
        lapz2 = (-lap4 * TI(jp1 * 3 + 2) + lap5 * TE(jp1 * 3 + 2) + lap6 * TI(jp2 * 3 + 2)) * AT2;
        lap += ((lapx1 + lapx2) * OA(j * 3 + 0) + (lapy1 + lapy2) * OA(j * 3 + 1)
                + (lapz1 + lapz2) * OA(j * 3 + 2))
               * vdiff;
    }
    return lap;
}

// Laplacian from the weights: (w0 a0 + sum_k wk (ak - a0)) rscale^2, products and sums in R.
template<int n, class R>
__device__ __forceinline__ double laplacian_w(const SGeo& G, const double* a, double rscale) {
    const int x = G.x;
    if constexpr (sizeof(R) < sizeof(double)) {
        float acc = G.lwf[x] * (float)a[0];
#pragma unroll
        for (int k = 1; k <= n; k++)
            acc = fmaf(G.lwf[k * kTile + x], (float)(a[k] - a[0]), acc);
        return (double)(acc * (float)(rscale * rscale));
    }
    else {
        double acc = G.lw[x] * a[0];
#pragma unroll
        for (int k = 1; k <= n; k++)
            acc = fma(G.lw[k * kTile + x], a[k] - a[0], acc);
        return acc * (rscale * rscale);
    }
}

// ---------------------------------------------------------------------------------------------
// Hyperdiffusion pass: Diffusion_Op + Diffusion_Op_Poles (src/headers/dyn/thor_diff.h:54-880)
// on the six variables rho, v(3), w, Rd T (or Cv T), without the diffusive sponge; the final pass
// applies Correct_Horizontal (:882-915) to the momentum result.
//   first pass  (stepnum 0): argument = the fields                     -> diff planes (6)
//   middle pass           : argument = diff of the previous pass       -> diff planes (6)
//   final pass (last)     : argument = diff (rho-weighted for v, w, T), scaled by -Kdh4 (-1)^(o/2)
//                            -> diffrh, diffmh(3), diffw, diffpr
// ---------------------------------------------------------------------------------------------
template<int n, class R, bool kUni>
__device__ __forceinline__ void diffusion_point(const Geometry& g, const Phys& P, const State& s,
                                                const SGeo& G, const double* fr, const int* ring,
                                                const double* __restrict__ diff_in,
                                                double* __restrict__ diff_out, int stepnum,
                                                bool last, int c, int lev, double sign4) {
    const int    Np = g.Np, nv = g.nv;
    const double rscale = rscale_of(P, g, lev);
    const double sdiff  = -g.Kdh4[lev] * sign4;
    const bool   eeq    = P.energy;
    int          ids[n + 1];
    double       rho[n + 1];
    ids[0] = c;
#pragma unroll
    for (int j = 0; j < n; j++)
        ids[j + 1] = ring[j];
#pragma unroll
    for (int j = 0; j <= n; j++)
        rho[j] = gz(s.Rhok + lev * Np, ids[j]);
    const int i = lev * Np + c;
    double    m1 = 0, m2 = 0, m3 = 0; // momentum results, combined after the third
#pragma unroll 1
    for (int var = 0; var < 6; var++) {
        double a[n + 1];
#pragma unroll
        for (int j = 0; j <= n; j++) {
            const int id = ids[j];
            double    v  = 0.0;
            if (id >= 0) {
                const int q = lev * Np + id;
                if (stepnum == 0) {
                    if (var == 0)
                        v = s.Rhok[q];
                    else if (var <= 3)
                        v = s.Mhk[((var - 1) * nv + lev) * Np + id];
                    else if (var == 4)
                        v = s.Wk[q];
                    else
                        v = eeq ? (cp_at<kUni>(P, s, q) - rd_at<kUni>(P, s, q)) * s.T[q] : rd_at<kUni>(P, s, q) * s.T[q];
                    if (var >= 1 && var <= 4)
                        v = v / rho[j];
                }
                else if (last)
                    v = (var == 0) ? diff_in[(var * nv + lev) * Np + id]
                                   : diff_in[(var * nv + lev) * Np + id] * rho[j];
                else
                    v = diff_in[(var * nv + lev) * Np + id];
            }
            a[j] = v;
        }
        double lap = laplacian<n, double>(G, a + 1, a[0], rscale);
        if (!last) {
            diff_out[(var * nv + lev) * Np + c] = lap;
            continue;
        }
        lap *= sdiff;
        if (var == 0)
            s.diffrh[i] = lap;
        else if (var == 1)
            m1 = lap;
        else if (var == 2)
            m2 = lap;
        else if (var == 3) {
            m3 = lap;
            // Correct_Horizontal: remove the radial component of the momentum diffusion
            const double dmhr = fr[0] * m1 + fr[1] * m2 + fr[2] * m3;
            s.diffmh[(0 * nv + lev) * Np + c] = m1 + -fr[0] * dmhr;
            s.diffmh[(1 * nv + lev) * Np + c] = m2 + -fr[1] * dmhr;
            s.diffmh[(2 * nv + lev) * Np + c] = m3 + -fr[2] * dmhr;
        }
        else if (var == 4)
            s.diffw[i] = lap;
        else
            s.diffpr[i] = lap;
    }
}

// The six Laplacians of one (column, level) in one pass over the stencil points. With the operator
// weights each Laplacian is a running sum, so the values of all six variables at a point are
// loaded together; each sum keeps laplacian_w's order (centre weight, then the ring in order).
// kF32 (mixed form): v and w in float, rho and T in double; otherwise all six in double.
template<int n, bool kF32, bool kUni>
__device__ __forceinline__ void diffusion_point_w(const Geometry& g, const Phys& P, const State& s,
                                                  const SGeo& G, const double* fr, const int* ring,
                                                  const double* __restrict__ diff_in,
                                                  double* __restrict__ diff_out, int stepnum,
                                                  bool last, int c, int lev, double sign4) {
    const int    Np = g.Np, nv = g.nv, x = G.x;
    const double rscale = rscale_of(P, g, lev);
    const bool   eeq    = P.energy;
    // the six variables at point id (0 at a hole), as the FP64 form forms them
    auto point = [&](int id, double* v) {
#pragma unroll
        for (int var = 0; var < 6; var++)
            v[var] = 0.0;
        if (id < 0)
            return;
        const int q = lev * Np + id;
        if (stepnum == 0) { // quotients by rho from one reciprocal (div_rcp: IEEE quotients)
            const double rho = s.Rhok[q], yr = 1.0 / rho;
            v[0]             = rho;
#pragma unroll
            for (int k = 0; k < 3; k++)
                v[1 + k] = div_rcp(s.Mhk[(k * nv + lev) * Np + id], rho, yr);
            v[4] = div_rcp(s.Wk[q], rho, yr);
            v[5] = eeq ? (cp_at<kUni>(P, s, q) - rd_at<kUni>(P, s, q)) * s.T[q] : rd_at<kUni>(P, s, q) * s.T[q];
        }
        else {
#pragma unroll
            for (int var = 0; var < 6; var++)
                v[var] = diff_in[(var * nv + lev) * Np + id];
            if (last) {
                const double rho = s.Rhok[q];
#pragma unroll
                for (int var = 1; var < 6; var++)
                    v[var] = v[var] * rho;
            }
        }
    };
    double a0[6];
    point(c, a0);
    const double sc = rscale * rscale;
    double       lap[6];
    if constexpr (kF32) {
        double accd0 = G.lw[x] * a0[0], accd5 = G.lw[x] * a0[5];
        float  accf[4];
#pragma unroll
        for (int k = 0; k < 4; k++)
            accf[k] = G.lwf[x] * (float)a0[1 + k];
#pragma unroll 2
        for (int j = 1; j <= n; j++) {
            double v[6];
            point(__ldg(g.ring + (j - 1) * Np + c), v);
            const double w  = G.lw[j * kTile + x];
            const float  wf = G.lwf[j * kTile + x];
            accd0           = fma(w, v[0] - a0[0], accd0);
            accd5           = fma(w, v[5] - a0[5], accd5);
#pragma unroll
            for (int k = 0; k < 4; k++)
                accf[k] = fmaf(wf, (float)(v[1 + k] - a0[1 + k]), accf[k]);
        }
        lap[0] = accd0 * sc;
        lap[5] = accd5 * sc;
#pragma unroll
        for (int k = 0; k < 4; k++)
            lap[1 + k] = (double)(accf[k] * (float)sc);
    }
    else {
        double acc[6];
#pragma unroll
        for (int var = 0; var < 6; var++)
            acc[var] = G.lw[x] * a0[var];
#pragma unroll 2
        for (int j = 1; j <= n; j++) {
            double v[6];
            point(__ldg(g.ring + (j - 1) * Np + c), v);
            const double w = G.lw[j * kTile + x];
#pragma unroll
            for (int var = 0; var < 6; var++)
                acc[var] = fma(w, v[var] - a0[var], acc[var]);
        }
#pragma unroll
        for (int var = 0; var < 6; var++)
            lap[var] = acc[var] * sc;
    }
    if (!last) {
#pragma unroll
        for (int var = 0; var < 6; var++)
            diff_out[(var * nv + lev) * Np + c] = lap[var];
        return;
    }
    const double sdiff = -g.Kdh4[lev] * sign4;
    const int    i     = lev * Np + c;
#pragma unroll
    for (int var = 0; var < 6; var++)
        lap[var] *= sdiff;
    s.diffrh[i] = lap[0];
    // Correct_Horizontal: remove the radial component of the momentum diffusion
    const double dmhr = fr[0] * lap[1] + fr[1] * lap[2] + fr[2] * lap[3];
    s.diffmh[(0 * nv + lev) * Np + c] = lap[1] + -fr[0] * dmhr;
    s.diffmh[(1 * nv + lev) * Np + c] = lap[2] + -fr[1] * dmhr;
    s.diffmh[(2 * nv + lev) * Np + c] = lap[3] + -fr[2] * dmhr;
    s.diffw[i]                        = lap[4];
    s.diffpr[i]                       = lap[5];
}

template<int n, class R, bool kUni>
__device__ __forceinline__ void diffusion_body(const Geometry& g, const Phys& P, const State& s,
                                               const SGeo& G, const double* __restrict__ diff_in,
                                               double* __restrict__ diff_out, int stepnum,
                                               bool last, int c) {
    const int Np = g.Np;
    double    fr[3];
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    int ring[6];
    for (int j = 0; j < 6; j++)
        ring[j] = g.ring[j * Np + c];
    const double sign4 = pow(-1.0, P.HyDiffOrder / 2); // (-1)^(order/2) of the last pass
    for (int lev = threadIdx.y; lev < g.nv; lev += kLevGroups)
        if constexpr (kOperatorWeights<R>)
            diffusion_point_w<n, true, kUni>(g, P, s, G, fr, ring, diff_in, diff_out, stepnum, last, c,
                                       lev, sign4);
        else if constexpr (kDiffWeightsF64)
            diffusion_point_w<n, false, kUni>(g, P, s, G, fr, ring, diff_in, diff_out, stepnum, last, c,
                                        lev, sign4);
        else
            diffusion_point<n, R, kUni>(g, P, s, G, fr, ring, diff_in, diff_out, stepnum, last, c, lev, sign4);
}

// R: compute type of the momentum and w Laplacians (double; float in the mixed form).
template<class R, bool kUni>
__global__ void THORX_KATTR_DIFF
    diffusion_kernel(Geometry g, Phys P, State s, const double* __restrict__ diff_in,
                     double* __restrict__ diff_out, int stepnum, bool last) {
    __shared__ double sgeo[kRingGeoRows * kTile];
    const int         c = lane_column(g);
    SGeo              G;
    if constexpr (kOperatorWeights<R> || kDiffWeightsF64)
        G = stage_lap_weights(sgeo, g, c);
    else
        G = stage_ring_geo(sgeo, g, c);
    __syncthreads();
    if (c < 0)
        return;
    if (tail_cta())
        diffusion_body<5, R, kUni>(g, P, s, G, diff_in, diff_out, stepnum, last, c);
    else
        diffusion_body<6, R, kUni>(g, P, s, G, diff_in, diff_out, stepnum, last, c);
}

// ---------------------------------------------------------------------------------------------
// Divergence damping (DivM_Op / DivM_Op_Poles, src/headers/dyn/thor_div.h:49-535).
// Pass 0: grad of the 3D divergence of (Mh, Wh) -> divg; pass 1 (divm_final): the tangential
// part of grad(div) of divg scaled by -Kdhz. The poles' corner mean of w uses the second
// sub-area in place of the third (thor_div.h:443-454), restated as it is (c2 = 1).
// ---------------------------------------------------------------------------------------------
template<int n, class R>
__device__ __forceinline__ void divm_core(const SGeo& G, const R* a0, const R (*ar)[3], bool with_w,
                                          R wl0, R wt0, const R* wl, const R* wt, R dz, R rscale,
                                          int c2, R* lapo) {
    static_assert(sizeof(R) == sizeof(double), "the FP32 stencils apply the operator weights");
    auto    AR = [&](int q) { return (R)G.AR(q); };
    auto    AT = [&](int q) { return (R)G.AT(q); };
    auto    TI = [&](int q) { return (R)G.TI(q); };
    auto    TE = [&](int q) { return (R)G.TE(q); };
    auto    OA = [&](int q) { return (R)G.OA(q); };
    auto    RAT = [&](int q) { return G.RAT(q); };
    const R h   = (R)0.5;
    const R AT0 = h * rscale;
    R       lapx = 0, lapy = 0, lapz = 0;
    R       a01x = 0, a01y = 0, a01z = 0, a12x = 0, a12y = 0, a12z = 0, AT1 = 0, lap1 = 0, lap2 = 0;
#pragma unroll
    for (int j = 0; j < n; j++) {
        const int     jp1 = (j + 1) % n, jp2 = (j + 2) % n;
        const R *p1 = ar[j], *p2 = ar[jp1], *p3 = ar[jp2];
        R        dwdz = 0, dwdz2 = 0;
        if (with_w) {
            const R meanwl = div_rcp(AR(j * 3 + 0) * wl0 + AR(j * 3 + 1) * wl[j] + AR(j * 3 + c2) * wl[jp1], AT(j), RAT(j));
            const R meanwt = div_rcp(AR(j * 3 + 0) * wt0 + AR(j * 3 + 1) * wt[j] + AR(j * 3 + c2) * wt[jp1], AT(j), RAT(j));
            const R meanwl2 = div_rcp(AR(jp1 * 3 + 0) * wl0 + AR(jp1 * 3 + 1) * wl[jp1] + AR(jp1 * 3 + c2) * wl[jp2], AT(jp1), RAT(jp1));
            const R meanwt2 = div_rcp(AR(jp1 * 3 + 0) * wt0 + AR(jp1 * 3 + 1) * wt[jp1] + AR(jp1 * 3 + c2) * wt[jp2], AT(jp1), RAT(jp1));
            dwdz  = (meanwl - meanwt) * dz;
            dwdz2 = (meanwl2 - meanwt2) * dz;
        }
        if (j == 0) {
            a01x = (a0[0] + p1[0]);
            a01y = (a0[1] + p1[1]);
            a01z = (a0[2] + p1[2]);
            a12x = (p1[0] + p2[0]);
            a12y = (p1[1] + p2[1]);
            a12z = (p1[2] + p2[2]);
            AT1  = div_rcp(h * rscale, AT(j), RAT(j));
        }
        const R AT2  = div_rcp(h * rscale, AT(jp1), RAT(jp1));
        const R a02x = (a0[0] + p2[0]), a02y = (a0[1] + p2[1]), a02z = (a0[2] + p2[2]);
        const R a23x = (p2[0] + p3[0]), a23y = (p2[1] + p3[1]), a23z = (p2[2] + p3[2]);
        const R a03x = (a0[0] + p3[0]), a03y = (a0[1] + p3[1]), a03z = (a0[2] + p3[2]);
        if (j == 0)
            lap1 = (-a01x * TI(j * 3 + 0) - a01y * TI(j * 3 + 1) - a01z * TI(j * 3 + 2)
                    + a12x * TE(j * 3 + 0) + a12y * TE(j * 3 + 1) + a12z * TE(j * 3 + 2)
                    + a02x * TI(jp1 * 3 + 0) + a02y * TI(jp1 * 3 + 1) + a02z * TI(jp1 * 3 + 2))
                   * AT1;
        else
            lap1 = lap2;
        lap2 = (-a02x * TI(jp1 * 3 + 0) - a02y * TI(jp1 * 3 + 1) - a02z * TI(jp1 * 3 + 2)
                + a23x * TE(jp1 * 3 + 0) + a23y * TE(jp1 * 3 + 1) + a23z * TE(jp1 * 3 + 2)
                + a03x * TI(jp2 * 3 + 0) + a03y * TI(jp2 * 3 + 1) + a03z * TI(jp2 * 3 + 2))
               * AT2;
        lapx += (lap1 + dwdz + lap2 + dwdz2) * OA(j * 3 + 0) * AT0;
        lapy += (lap1 + dwdz + lap2 + dwdz2) * OA(j * 3 + 1) * AT0;
        lapz += (lap1 + dwdz + lap2 + dwdz2) * OA(j * 3 + 2) * AT0;
    }
    lapo[0] = lapx;
    lapo[1] = lapy;
    lapo[2] = lapz;
}

// ---------------------------------------------------------------------------------------------
// Operator weights of the mixed form. Both stencil operators are linear in the point values, so
// each is fixed per column by its response to unit inputs, computed here once per context with
// the FP64 operator code above (laplacian, divm_core) at rscale = 1 (and dz = 1 for the w part of
// the damping): the Laplacian scales with rscale^2 (rscale / areasTr and 0.5 rscale), the damping's
// Mh part with rscale^2 and its w part with rscale dz. The centre entry is stored as the sum of
// all the point weights and the ring entries as they are, so that at run time
//   op(a) = (sum_k w_k) a_0 + sum_{k>=1} w_k (a_k - a_0),
// the same linear operator; the differences a_k - a_0 are formed in FP64 before the FP32
// multiply-adds, so the float arithmetic does not see the large common part of the values.
// One thread per column; a column with a five-entry ring gets zero sixth weights.
// ---------------------------------------------------------------------------------------------
template<int n>
__device__ void stencil_weights_of(const SGeo& G, int c2, int c, int Np, double* lapw, float* dmw,
                                   double* dmw64) {
    // Laplacian
    double w[7] = {0, 0, 0, 0, 0, 0, 0}, wsum = 0.0;
    for (int k = 0; k <= n; k++) {
        double a[n + 1];
        for (int j = 0; j <= n; j++)
            a[j] = (j == k) ? 1.0 : 0.0;
        w[k] = laplacian<n, double>(G, a + 1, a[0], 1.0);
        wsum += w[k];
    }
    lapw[c] = wsum;
    for (int k = 1; k < 7; k++)
        lapw[(size_t)k * Np + c] = w[k];
    // divergence damping, Mh part: response to a unit component comp at point k
    double wm[3][7][3] = {};
    for (int k = 0; k <= n; k++)
        for (int comp = 0; comp < 3; comp++) {
            double a0[3] = {0, 0, 0}, ar[n][3], out[3];
            for (int j = 0; j < n; j++)
                ar[j][0] = ar[j][1] = ar[j][2] = 0.0;
            if (k == 0)
                a0[comp] = 1.0;
            else
                ar[k - 1][comp] = 1.0;
            divm_core<n, double>(G, a0, ar, false, 0.0, 0.0, nullptr, nullptr, 0.0, 1.0, c2, out);
            for (int o = 0; o < 3; o++)
                wm[o][k][comp] = out[o];
        }
    for (int o = 0; o < 3; o++)
        for (int comp = 0; comp < 3; comp++) {
            double sum = 0.0;
            for (int k = 0; k <= n; k++)
                sum += wm[o][k][comp];
            dmw[(size_t)(o * 28 + comp) * Np + c]   = (float)sum;
            dmw64[(size_t)(o * 28 + comp) * Np + c] = sum;
            for (int k = 1; k < 7; k++) {
                dmw[(size_t)(o * 28 + k * 3 + comp) * Np + c]   = (float)wm[o][k][comp];
                dmw64[(size_t)(o * 28 + k * 3 + comp) * Np + c] = wm[o][k][comp];
            }
        }
    // divergence damping, w part: response to a unit (Wh below - Wh above) at point k
    for (int k = 0; k < 7; k++) {
        double out[3] = {0, 0, 0};
        if (k <= n) {
            double a0[3] = {0, 0, 0}, ar[n][3], wl[n], wt[n];
            for (int j = 0; j < n; j++) {
                ar[j][0] = ar[j][1] = ar[j][2] = 0.0;
                wl[j] = (j == k - 1) ? 1.0 : 0.0;
                wt[j] = 0.0;
            }
            divm_core<n, double>(G, a0, ar, true, k == 0 ? 1.0 : 0.0, 0.0, wl, wt, 1.0, 1.0, c2,
                                 out);
        }
        for (int o = 0; o < 3; o++) {
            dmw[(size_t)(o * 28 + 21 + k) * Np + c]   = (float)out[o];
            dmw64[(size_t)(o * 28 + 21 + k) * Np + c] = out[o];
        }
    }
}

__global__ void __launch_bounds__(kTile) stencil_weights_kernel(Geometry g, double* lapw, float* dmw,
                                                                double* dmw64) {
    __shared__ double sgeo[kRingGeoRows * kTile];
    const int         c   = blockIdx.x * kTile + threadIdx.x;
    const int         col = c < g.N ? c : -1;
    const SGeo        G   = stage_ring_geo(sgeo, g, col);
    __syncthreads();
    if (col < 0)
        return;
    const int c2 = (g.cflag[c] & kPole) ? 1 : 2;
    if (g.cflag[c] & kRing5)
        stencil_weights_of<5>(G, c2, c, g.Np, lapw, dmw, dmw64);
    else
        stencil_weights_of<6>(G, c2, c, g.Np, lapw, dmw, dmw64);
}

// Divergence damping from the weights, in float: a0 [3] and ar [n][3] the Mh (or divg) vectors
// at the centre and the ring; dw [n + 1] the (below - above) Wh differences when with_w.
// T: float (mixed form, Geometry::dmw) or double (FP64 form, Geometry::dmw64).
__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
template<int n, class T>
__device__ __forceinline__ void divm_w(const SGeo& G, const double* a0, const double (*ar)[3],
                                       bool with_w, const double* dw, double rscale, double dz,
                                       T* out) {
    const int x = G.x;
    T         d[n][3], c0[3];
#pragma unroll
    for (int comp = 0; comp < 3; comp++) {
        c0[comp] = (T)a0[comp];
#pragma unroll
        for (int j = 0; j < n; j++)
            d[j][comp] = (T)(ar[j][comp] - a0[comp]);
    }
    const T sv = (T)(rscale * rscale), sw = (T)(rscale * dz);
#pragma unroll
    for (int o = 0; o < 3; o++) {
        const T* W;
        if constexpr (sizeof(T) < sizeof(double))
            W = G.dm + o * 28 * kTile + x;
        else
            W = G.dm64 + o * 28 * kTile + x;
        T acc = (T)0;
#pragma unroll
        for (int comp = 0; comp < 3; comp++)
            acc = fma_t(W[comp * kTile], c0[comp], acc);
#pragma unroll
        for (int j = 0; j < n; j++)
#pragma unroll
            for (int comp = 0; comp < 3; comp++)
                acc = fma_t(W[((j + 1) * 3 + comp) * kTile], d[j][comp], acc);
        acc *= sv;
        if (with_w) {
            T accw = (T)0;
#pragma unroll
            for (int k = 0; k <= n; k++)
                accw = fma_t(W[(21 + k) * kTile], (T)dw[k], accw);
            acc = fma_t(accw, sw, acc);
        }
        out[o] = acc;
    }
}

template<int n, class R>
__device__ __forceinline__ void divm0_point(const Geometry& g, const Phys& P, const SGeo& G,
                                            const int* ring, int c2, const double* __restrict__ Mh,
                                            const double* __restrict__ Wh,
                                            DivgT<R>* __restrict__ divg, int c, int lev) {
    const int    Np = g.Np, nv = g.nv;
    const double rscale = rscale_of(P, g, lev);
    const double dz     = 1.0 / (g.Altitudeh[lev] - g.Altitudeh[lev + 1]);
    if constexpr (kOperatorWeights<R> || kDivmWeightsF64) {
        using T = std::conditional_t<kOperatorWeights<R>, float, double>;
        double a0[3], ar[n][3], dw[n + 1];
#pragma unroll
        for (int k = 0; k < 3; k++)
            a0[k] = Mh[(k * nv + lev) * Np + c];
        dw[0] = Wh[lev * Np + c] - Wh[(lev + 1) * Np + c];
#pragma unroll
        for (int j = 0; j < n; j++) {
#pragma unroll
            for (int k = 0; k < 3; k++)
                ar[j][k] = gz(Mh + (k * nv + lev) * Np, ring[j]);
            dw[j + 1] = gz(Wh + lev * Np, ring[j]) - gz(Wh + (lev + 1) * Np, ring[j]);
        }
        T out[3];
        divm_w<n, T>(G, a0, ar, true, dw, rscale, dz, out);
#pragma unroll
        for (int k = 0; k < 3; k++)
            divg[(k * nv + lev) * Np + c] = (DivgT<R>)out[k];
    }
    else {
        R            a0[3], ar[n][3], wl[n], wt[n];
#pragma unroll
        for (int k = 0; k < 3; k++)
            a0[k] = (R)Mh[(k * nv + lev) * Np + c];
#pragma unroll
        for (int j = 0; j < n; j++) {
#pragma unroll
            for (int k = 0; k < 3; k++)
                ar[j][k] = (R)gz(Mh + (k * nv + lev) * Np, ring[j]);
            wl[j] = (R)gz(Wh + lev * Np, ring[j]);
            wt[j] = (R)gz(Wh + (lev + 1) * Np, ring[j]);
        }
        R out[3];
        divm_core<n, R>(G, a0, ar, true, (R)Wh[lev * Np + c], (R)Wh[(lev + 1) * Np + c], wl, wt, (R)dz,
                        (R)rscale, c2, out);
#pragma unroll
        for (int k = 0; k < 3; k++)
            divg[(k * nv + lev) * Np + c] = (DivgT<R>)out[k];
    }
}

// Pass 0 through the operator weights at kL consecutive levels lev .. lev + kL - 1 of column c
// (levels at or above nv are computed on the top level and not stored). The stencil points are
// streamed: at each point the Mh vector of every level and the Wh values of the kL + 1 interfaces
// are loaded once, and each weight read from shared memory serves all kL levels. For each output
// the multiply-adds run in divm_w's order (the centre's components, then the ring point by point,
// the Wh differences in their own sum), so every value is divm0_point's bit for bit.
// Levels per thread: 3 in the FP64 form (glevel 6, 48 levels: divm0 1.245 -> 1.16 ms per step
// against one level; 2: 1.19, 4: 1.36), 1 in the mixed form (1.13 ms; 2: 1.20, 3: 1.18).
#ifndef THORX_DIVM_LEVELS
#define THORX_DIVM_LEVELS 3
#endif
#ifndef THORX_DIVM_LEVELS_MIXED
#define THORX_DIVM_LEVELS_MIXED 1
#endif
template<class R>
constexpr int kDivmLevels = sizeof(R) < sizeof(double) ? THORX_DIVM_LEVELS_MIXED : THORX_DIVM_LEVELS;
template<int n, class T, int kL>
__device__ __forceinline__ void divm0_levels(const Geometry& g, const Phys& P, const SGeo& G,
                                             const int* ring, const double* __restrict__ Mh,
                                             const double* __restrict__ Wh,
                                             double* __restrict__ divg, int c, int lev) {
    const int Np = g.Np, nv = g.nv;
    const T*  W;
    if constexpr (sizeof(T) < sizeof(double))
        W = G.dm + G.x;
    else
        W = G.dm64 + G.x;
    auto w = [&](int o, int e) { return W[(o * 28 + e) * kTile]; };
    int  lv[kL], li[kL + 1]; // the levels and interfaces read, clamped to the column
#pragma unroll
    for (int l = 0; l < kL; l++)
        lv[l] = min(lev + l, nv - 1);
#pragma unroll
    for (int l = 0; l <= kL; l++)
        li[l] = min(lev + l, nv);
    double a0[kL][3], wv[kL + 1];
    T      acc[kL][3], accw[kL][3];
#pragma unroll
    for (int l = 0; l < kL; l++)
#pragma unroll
        for (int k = 0; k < 3; k++)
            a0[l][k] = Mh[(k * nv + lv[l]) * Np + c];
#pragma unroll
    for (int l = 0; l <= kL; l++)
        wv[l] = Wh[li[l] * Np + c];
#pragma unroll
    for (int o = 0; o < 3; o++) {
#pragma unroll
        for (int l = 0; l < kL; l++) {
            acc[l][o]  = (T)0;
            accw[l][o] = (T)0;
        }
#pragma unroll
        for (int comp = 0; comp < 3; comp++) {
            const T wc = w(o, comp);
#pragma unroll
            for (int l = 0; l < kL; l++)
                acc[l][o] = fma_t(wc, (T)a0[l][comp], acc[l][o]);
        }
        const T ww = w(o, 21);
#pragma unroll
        for (int l = 0; l < kL; l++)
            accw[l][o] = fma_t(ww, (T)(wv[l] - wv[l + 1]), accw[l][o]);
    }
#pragma unroll
    for (int j = 0; j < n; j++) {
        double m[kL][3], wr[kL + 1];
#pragma unroll
        for (int l = 0; l < kL; l++)
#pragma unroll
            for (int k = 0; k < 3; k++)
                m[l][k] = gz(Mh + (k * nv + lv[l]) * Np, ring[j]);
#pragma unroll
        for (int l = 0; l <= kL; l++)
            wr[l] = gz(Wh + li[l] * Np, ring[j]);
#pragma unroll
        for (int o = 0; o < 3; o++) {
#pragma unroll
            for (int comp = 0; comp < 3; comp++) {
                const T wc = w(o, (j + 1) * 3 + comp);
#pragma unroll
                for (int l = 0; l < kL; l++)
                    acc[l][o] = fma_t(wc, (T)(m[l][comp] - a0[l][comp]), acc[l][o]);
            }
            const T ww = w(o, 22 + j);
#pragma unroll
            for (int l = 0; l < kL; l++)
                accw[l][o] = fma_t(ww, (T)(wr[l] - wr[l + 1]), accw[l][o]);
        }
    }
#pragma unroll
    for (int l = 0; l < kL; l++) {
        if (lev + l >= nv)
            break;
        const double rscale = rscale_of(P, g, lev + l);
        const double dz     = 1.0 / (g.Altitudeh[lev + l] - g.Altitudeh[lev + l + 1]);
        const T      sv = (T)(rscale * rscale), sw = (T)(rscale * dz);
#pragma unroll
        for (int o = 0; o < 3; o++) {
            T a = acc[l][o];
            a *= sv;
            a = fma_t(accw[l][o], sw, a);
            divg[(o * nv + lev + l) * Np + c] = (double)a;
        }
    }
}

// Pass 0 of the divergence damping on (Mh, Wh) -> divg.
template<int n, class R>
__device__ __forceinline__ void divm0_body(const Geometry& g, const Phys& P, const SGeo& G,
                                           const double* __restrict__ Mh,
                                           const double* __restrict__ Wh,
                                           DivgT<R>* __restrict__ divg, int c) {
    const int Np = g.Np;
    int       ring[6];
    for (int j = 0; j < 6; j++)
        ring[j] = g.ring[j * Np + c];
    if constexpr ((kOperatorWeights<R> || kDivmWeightsF64) && kDivmLevels<R> > 1) {
        using T        = std::conditional_t<kOperatorWeights<R>, float, double>;
        constexpr int L = kDivmLevels<R>;
        for (int lev = threadIdx.y * L; lev < g.nv; lev += kLevGroups * L)
            divm0_levels<n, T, L>(g, P, G, ring, Mh, Wh, divg, c, lev);
    }
    else {
        const int c2 = (g.cflag[c] & kPole) ? 1 : 2;
        for (int lev = threadIdx.y; lev < g.nv; lev += kLevGroups)
            divm0_point<n, R>(g, P, G, ring, c2, Mh, Wh, divg, c, lev);
    }
}

template<class R>
__global__ void THORX_KATTR_DIVM
    divm0_kernel(Geometry g, Phys P, const double* __restrict__ Mh, const double* __restrict__ Wh,
                 double* __restrict__ divg) {
    __shared__ double sgeo[kRingGeoRows * kTile];
    const int         c = lane_column(g);
    const SGeo        G = stage_divm_geo<R>(sgeo, g, c);
    __syncthreads();
    if (c < 0)
        return;
    if (tail_cta())
        divm0_body<5, R>(g, P, G, Mh, Wh, reinterpret_cast<DivgT<R>*>(divg), c);
    else
        divm0_body<6, R>(g, P, G, Mh, Wh, reinterpret_cast<DivgT<R>*>(divg), c);
}

// The end of pass 1: the radial component removed, scaled by -Kdhz.
template<class R>
__device__ __forceinline__ void divm_finish(const Geometry& g, int lev, const double* fr,
                                            const R* lap, R* DivM) {
    const R sdiff = (R)g.Kdhz[lev];
    const R lapr  = (R)fr[0] * lap[0] + (R)fr[1] * lap[1] + (R)fr[2] * lap[2];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const R l = lap[k] - (R)fr[k] * lapr;
        DivM[k]   = -l * sdiff;
    }
}

// Pass 1 of the divergence damping at (column, level): DivM from divg.
template<int n, class R>
__device__ __forceinline__ void divm_final(const Geometry& g, const Phys& P, const SGeo& G,
                                           const int* ring, const DivgT<R>* __restrict__ divg, int c,
                                           int lev, const double* fr, R* DivM) {
    const int Np = g.Np, nv = g.nv;
    R         lap[3];
    if constexpr (kOperatorWeights<R> || kDivmWeightsF64) {
        double a0[3], ar[n][3];
#pragma unroll
        for (int k = 0; k < 3; k++)
            a0[k] = divg[(k * nv + lev) * Np + c];
#pragma unroll
        for (int j = 0; j < n; j++)
#pragma unroll
            for (int k = 0; k < 3; k++)
                ar[j][k] = gz(divg + (k * nv + lev) * Np, ring[j]);
        divm_w<n, R>(G, a0, ar, false, nullptr, rscale_of(P, g, lev), 0.0, lap);
    }
    else {
        R a0[3], ar[n][3];
#pragma unroll
        for (int k = 0; k < 3; k++)
            a0[k] = (R)divg[(k * nv + lev) * Np + c];
#pragma unroll
        for (int j = 0; j < n; j++)
#pragma unroll
            for (int k = 0; k < 3; k++)
                ar[j][k] = (R)gz(divg + (k * nv + lev) * Np, ring[j]);
        divm_core<n, R>(G, a0, ar, false, (R)0, (R)0, nullptr, nullptr, (R)0,
                        (R)rscale_of(P, g, lev), 2, lap);
    }
    divm_finish<R>(g, lev, fr, lap, DivM);
}

// Pass 1 from values already gathered (a0: divg at the column; ar: at its ring), operator weights.
template<int n, class R>
__device__ __forceinline__ void divm_final_vals(const Geometry& g, const Phys& P, const SGeo& G,
                                                const double* a0, const double (*ar)[3], int lev,
                                                const double* fr, R* DivM) {
    R lap[3];
    divm_w<n, R>(G, a0, ar, false, nullptr, rscale_of(P, g, lev), 0.0, lap);
    divm_finish<R>(g, lev, fr, lap, DivM);
}

// ---------------------------------------------------------------------------------------------
// Slow modes of one RK stage: divergence-damping pass 1 on (Mhk, Whk) + Compute_Slow_Modes /
// _Poles (src/headers/dyn/thor_slowmodes.h:48-683) + UpdateRK
// (src/headers/dyn/thor_auxiliary.h:311-418, without module arrays and without the never-read
// Ws). DivM is consumed where it is produced and not stored.
// ---------------------------------------------------------------------------------------------
template<int n, class R, bool kUni>
__device__ __forceinline__ void slow_modes_body(const Geometry& g, const Phys& P, const State& s,
                                                const SGeo& G, const double* sdiv,
                                                const double* sgrad, bool update_rk, int c) {
    const int     x = threadIdx.x;
    const int     Np = g.Np, nv = g.nv, nvi = g.nvi;
    const double  A = P.A, Gravit = P.Gravit;
    const double* lt = g.lt;
    int           nb[7], ring[6];
    nb[0] = c;
    for (int j = 0; j < 6; j++) {
        nb[j + 1] = g.nb[j * Np + c];
        ring[j]   = g.ring[j * Np + c];
    }
    double fr[3];
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    const bool pole = (g.cflag[c] & kPole) != 0;

    for (int lev = threadIdx.y; lev < nv; lev += kLevGroups) {
        const int i       = lev * Np + c;
        R         DivM[3] = {0, 0, 0};
        if (P.DivDampP)
            divm_final<n, R>(g, P, G, ring, reinterpret_cast<const DivgT<R>*>(s.divg), c, lev, fr,
                              DivM);
        const double Cv = cp_at<kUni>(P, s, i) - rd_at<kUni>(P, s, i);
        double       adv[3];
        for (int k = 0; k < 3; k++)
            adv[k] = s.Adv[(k * nv + lev) * Np + c];
        const double rho = s.Rhok[i];
        double       rhol = 0, altl = 0, pressurel = 0, advrl = 0;
        if (lev != 0) {
            advrl = s.Adv[(0 * nv + lev - 1) * Np + c] * fr[0] + s.Adv[(1 * nv + lev - 1) * Np + c] * fr[1]
                    + s.Adv[(2 * nv + lev - 1) * Np + c] * fr[2];
            rhol      = s.Rhok[i - Np];
            altl      = g.Altitude[lev - 1];
            pressurel = s.pk[i - Np];
        }
        double advr = adv[0] * fr[0] + adv[1] * fr[1] + adv[2] * fr[2];
        for (int k = 0; k < 3; k++)
            adv[k] += -advr * fr[k];
        const double altht = g.Altitudeh[lev + 1], althl = g.Altitudeh[lev], alt = g.Altitude[lev];
        double       M0[3];
        for (int k = 0; k < 3; k++)
            M0[k] = s.Mhk[(k * nv + lev) * Np + c];
        if (!P.NonHydro) {
            advr = (pow(M0[0], 2) + pow(M0[1], 2) + pow(M0[2], 2)) / (rho * (alt + A));
            if (lev != 0)
                advrl = (pow(s.Mhk[(0 * nv + lev - 1) * Np + c], 2) + pow(s.Mhk[(1 * nv + lev - 1) * Np + c], 2)
                         + pow(s.Mhk[(2 * nv + lev - 1) * Np + c], 2))
                        / (rhol * (altl + A));
        }
        const double dz = altht - althl;
        double       r2p, r2m, r2l, rscale, dr2dz;
        if (P.DeepModel) { // the level tables hold these expressions' values
            r2p    = lt[kLtR2hD * nvi + lev + 1];
            r2m    = lt[kLtR2cD * nvi + lev];
            r2l    = lt[kLtR2hD * nvi + lev];
            rscale = lt[kLtRscale * nvi + lev];
            dr2dz  = lt[kLtDr2dz * nvi + lev];
        }
        else {
            r2p = r2m = r2l = rscale = 1.0;
            dr2dz                    = r2m * dz;
        }
        // horizontal stencils at this level: running sums over the points in order, one point's
        // p, h and M at a time
        double sg[3], sd[3], sp3[3], pv0 = 0.0;
#pragma unroll
        for (int j = 0; j < 7; j++) {
            const double pv = gz(s.pk + lev * Np, nb[j]), hv = gz(s.h + lev * Np, nb[j]);
            if (j == 0)
                pv0 = pv;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double Mv = gz(s.Mhk + (k * nv + lev) * Np, nb[j]);
                const double dk = sdiv[(j * 3 + k) * kTile + x], gk = sgrad[(j * 3 + k) * kTile + x];
                if (j == 0) {
                    sg[k]  = gk * pv;
                    sd[k]  = dk * Mv;
                    sp3[k] = dk * Mv * hv;
                }
                else {
                    sg[k]  = sg[k] + gk * pv;
                    sd[k]  = sd[k] + dk * Mv;
                    sp3[k] = sp3[k] + dk * Mv * hv;
                }
            }
        }
        double nflxv[3], nflxr = 0.0, nflxp = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            nflxv[k] = rscale * sg[k];
            nflxr += rscale * sd[k];
            nflxp += rscale * sp3[k];
        }
        double whl, wht, hhl, hht;
        if (lev == 0) {
            whl = 0.0;
            wht = s.Whk[(lev + 1) * Np + c];
            hhl = 0.0;
            hht = s.hh[(lev + 1) * Np + c];
        }
        else {
            whl = s.Whk[lev * Np + c];
            wht = s.Whk[(lev + 1) * Np + c];
            hhl = s.hh[lev * Np + c];
            hht = s.hh[(lev + 1) * Np + c];
        }
        const double dwdz  = pole ? (wht * r2p - whl * r2l) / (dz * r2m) : (wht * r2p - whl * r2l) / (dr2dz);
        const double dwhdz = (wht * r2p * hht - whl * r2l * hhl) / (dz * r2m);
        const double dpr   = nflxv[0] * fr[0] + nflxv[1] * fr[1] + nflxv[2] * fr[2];
        // the level's results are stored at its end, after every load of the level, so that no
        // store orders the loads behind it (glevel 6, 48 levels: 0.88 -> 0.84 ms per step, the
        // same bits)
        double smh[3], swh_out = 0.0;
        for (int k = 0; k < 3; k++) {
            const int j = (k * nv + lev) * Np + c;
            smh[k]      = -(nflxv[k] - dpr * fr[k]) - adv[k] + (double)DivM[k] + s.diffmh[j] + s.dMh[j];
        }
        if (lev != 0) {
            const double intt = lt[kLtHIntt * nvi + lev], intl = lt[kLtHIntl * nvi + lev];
            double       swr;
            if (P.DeepModel) {
                if (P.GravHeightVar)
                    swr = (advrl + rhol * Gravit * lt[kLtGhv * nvi + lev - 1]) * intt
                          + (advr + rho * Gravit * lt[kLtGhv * nvi + lev]) * intl;
                else
                    swr = (advrl + rhol * Gravit) * intt + (advr + rho * Gravit) * intl;
            }
            else {
                if (P.GravHeightVar)
                    swr = (rhol * Gravit * lt[kLtGhv * nvi + lev - 1]) * intt
                          + (rho * Gravit * lt[kLtGhv * nvi + lev]) * intl;
                else
                    swr = (rhol * Gravit) * intt + (rho * Gravit) * intl;
            }
            if (P.NonHydro)
                swr += (-s.diffw[i - Np]) * intt + (-s.diffw[i]) * intl;
            const double dz2  = alt - altl;
            const double dpdz = (pv0 - pressurel) / dz2;
            swr += dpdz;
            swr -= s.dWh[lev * Np + c];
            swh_out = -swr;
        }
        nflxr += dwdz;
        const double srho = -nflxr + s.diffrh[i];
        const double r_  = 1.0 / rho;
        const double vgp = (nflxv[0] - dpr * fr[0]) * M0[0] * r_ + (nflxv[1] - dpr * fr[1]) * M0[1] * r_
                           + (nflxv[2] - dpr * fr[2]) * M0[2] * r_;
        double sp = (rd_at<kUni>(P, s, i) / Cv) * (-nflxp - s.gtil[i] - dwhdz + vgp + s.Qheat[i]);
        if (P.energy)
            sp += rd_at<kUni>(P, s, i) / Cv * (s.diffpr[i]);
        else
            sp += s.diffpr[i];
        double mhs[3], rhos = 0.0, pss = 0.0, whs = 0.0;
        if (update_rk) {
            // deviations from the start of the large step
            const double Mx  = s.Mh[(0 * nv + lev) * Np + c] - M0[0];
            const double My  = s.Mh[(1 * nv + lev) * Np + c] - M0[1];
            const double Mz  = s.Mh[(2 * nv + lev) * Np + c] - M0[2];
            const double aux = Mx * fr[0] + My * fr[1] + Mz * fr[2];
            mhs[0]           = Mx - aux * fr[0];
            mhs[1]           = My - aux * fr[1];
            mhs[2]           = Mz - aux * fr[2];
            rhos             = s.Rho[i] - rho;
            pss              = s.p[i] - s.pk[i];
            whs              = (lev == 0) ? 0.0 : s.Wh[lev * Np + c] - s.Whk[lev * Np + c];
        }
        for (int k = 0; k < 3; k++)
            s.SlowMh[(k * nv + lev) * Np + c] = smh[k];
        if (lev == 0) {
            s.SlowWh[c]           = 0.0;
            s.SlowWh[nv * Np + c] = 0.0;
        }
        else
            s.SlowWh[lev * Np + c] = swh_out;
        s.SlowRho[i] = srho;
        s.Slowp[i]   = sp;
        if (update_rk) {
            for (int k = 0; k < 3; k++)
                s.Mhs[(k * nv + lev) * Np + c] = mhs[k];
            s.Rhos[i]           = rhos;
            s.ps[i]             = pss;
            s.Whs[lev * Np + c] = whs;
            if (lev == nv - 1)
                s.Whs[nv * Np + c] = 0.0;
        }
    }
}

template<class R, bool kUni>
__global__ void THORX_KATTR_SLOW
    slow_modes_kernel(Geometry g, Phys P, State s, bool update_rk) {
    __shared__ double sgeo[kRingGeoRows * kTile];
    __shared__ double sdiv[21 * kTile];
    __shared__ double sgrad[21 * kTile];
    const int         c = lane_column(g);
    SGeo              G{};
    if (P.DivDampP)
        G = stage_divm_geo<R>(sgeo, g, c);
    stage_cols(sdiv, g.div, 21, g.Np, c);
    stage_cols(sgrad, g.grad, 21, g.Np, c);
    __syncthreads();
    if (c < 0)
        return;
    if (tail_cta())
        slow_modes_body<5, R, kUni>(g, P, s, G, sdiv, sgrad, update_rk, c);
    else
        slow_modes_body<6, R, kUni>(g, P, s, G, sdiv, sgrad, update_rk, c);
}

// ---------------------------------------------------------------------------------------------
// Small step, horizontal momentum: divergence-damping pass 1 on the deviations (Mhs, Whs) +
// Momentum_Eq / _Poles (src/headers/dyn/thor_fastmodes.h:54-253).
// ---------------------------------------------------------------------------------------------
// The update of Mhs at (c, lev) from ps at the 7 stencil points (pv) and the damping term DivM.
template<class R>
__device__ __forceinline__ void momentum_apply(const Geometry& g, const Phys& P, const State& s,
                                               const double* sgrad, double dt, int c, int lev,
                                               const double* fr, const double* pv, const R* DivM,
                                               const double* slow = nullptr,
                                               const double* mold = nullptr) {
    const int    x = threadIdx.x, Np = g.Np, nv = g.nv;
    const double rscale = rscale_of(P, g, lev);
    double       Mv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        double sg = sgrad[k * kTile + x] * pv[0];
#pragma unroll
        for (int j = 1; j < 7; j++)
            sg = sg + sgrad[(j * 3 + k) * kTile + x] * pv[j];
        const double nflxv = rscale * sg;
        const double sl    = slow ? slow[k] : s.SlowMh[(k * nv + lev) * Np + c];
        Mv[k]              = (-nflxv + sl + (double)DivM[k]) * dt;
    }
    const double vr = Mv[0] * fr[0] + Mv[1] * fr[1] + Mv[2] * fr[2];
    for (int k = 0; k < 3; k++) {
        Mv[k] += -vr * fr[k];
        const int j = (k * nv + lev) * Np + c;
        s.Mhs[j]    = (mold ? mold[k] : s.Mhs[j]) + Mv[k];
    }
}

template<int n, class R>
__device__ __forceinline__ void momentum_body(const Geometry& g, const Phys& P, const State& s,
                                              const SGeo& G, const double* sgrad, double dt,
                                              int c) {
    const int Np = g.Np, nv = g.nv;
    int       nb[7], ring[6];
    nb[0] = c;
    for (int j = 0; j < 6; j++) {
        nb[j + 1] = g.nb[j * Np + c];
        ring[j]   = g.ring[j * Np + c];
    }
    double fr[3];
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    for (int lev = threadIdx.y; lev < nv; lev += kLevGroups) {
        // the cell's own SlowMh and Mhs loaded first, so that their latency overlaps the damping
        // (glevel 6, 48 levels: 1.18 -> 1.09 ms per step, mixed 0.98 -> 0.87; the same bits)
        double slow[3], mold[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            slow[k] = s.SlowMh[(k * nv + lev) * Np + c];
            mold[k] = s.Mhs[(k * nv + lev) * Np + c];
        }
        R DivM[3] = {0, 0, 0};
        if (P.DivDampP)
            divm_final<n, R>(g, P, G, ring, reinterpret_cast<const DivgT<R>*>(s.divg), c, lev, fr,
                              DivM);
        double pv[7];
#pragma unroll
        for (int j = 0; j < 7; j++)
            pv[j] = gz(s.ps + lev * Np, nb[j]);
        momentum_apply<R>(g, P, s, sgrad, dt, c, lev, fr, pv, DivM, slow, mold);
    }
}

template<class R>
__global__ void THORX_KATTR_MOM
    momentum_kernel(Geometry g, Phys P, State s, double dt) {
    __shared__ double sgeo[kRingGeoRows * kTile];
    __shared__ double sgrad[21 * kTile];
    const int         c = lane_column(g);
    SGeo              G{};
    if (P.DivDampP)
        G = stage_divm_geo<R>(sgeo, g, c);
    stage_cols(sgrad, g.grad, 21, g.Np, c);
    __syncthreads();
    if (c < 0)
        return;
    if (tail_cta())
        momentum_body<5, R>(g, P, s, G, sgrad, dt, c);
    else
        momentum_body<6, R>(g, P, s, G, sgrad, dt, c);
}

// The same update with the neighbour values staged in shared memory by the tensor-memory
// accelerator: per round of 8 levels (one per warp), one thread copies, for each of the tile's
// window spans (Geometry::wspan), a box of kWinW columns x 8 levels of ps and of the 3 divg
// components (boxes of this GPU's own planes, no multicast), completing on an mbarrier; the warps
// then read their stencil points from the window, and the few outside it (rhombus edges) from
// global memory. kMomBuf windows: with 2, the copy of the next round overlaps this one's compute.
// The values and the arithmetic are those of momentum_body. The five-neighbour tile reads
// directly. A wait that runs past its bound sets kFlagWait and the CTA ends its work.
// Off by default (THORX_MOM_TMA=1 builds it): on the glevel-6, 48-level step the staged kernel
// took 1.58 ms per step with one window (2.09 ms with two: 2 CTAs per SM instead of 3) against
// 1.18 ms for the direct gathers, the same bits. A CTA waits for a whole round's boxes before any
// warp computes and meets at two barriers per round, where the gathering warps each run ahead on
// their own loads; the neighbour reads hit L1 already.
#ifndef THORX_MOM_TMA
#define THORX_MOM_TMA 0
#endif
#ifndef THORX_MOM_TMA_BUF
#define THORX_MOM_TMA_BUF 1
#endif
#if THORX_MOM_TMA
constexpr int      kMomBuf     = THORX_MOM_TMA_BUF;
constexpr int      kWinFields  = 4; // ps, divg x, y, z
constexpr int      kWinField   = kWinSpans * kLevGroups * kWinW; // doubles of one field's window
constexpr int      kWinDoubles = kWinFields * kWinField;
constexpr uint32_t kWinPolls   = 1u << 22;
// the staged kernel serves the operator-weight forms (the default FP64 form and the mixed form)
template<class R>
constexpr bool kMomTma = THORX_MOM_TMA && (kOperatorWeights<R> || kDivmWeightsF64)
                         && std::is_same_v<DivgT<R>, double>;
size_t momentum_smem_bytes() { return sizeof(double) * kMomBuf * kWinDoubles + 128; }
static_assert(kWinW * kLevGroups * sizeof(double) % 128 == 0, "window boxes keep 128-byte alignment");

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void win_bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void win_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
// phase `parity` of the mbarrier completed within `limit` polls
__device__ __forceinline__ bool win_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(smem_addr(bar)), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}
// one box {kWinW columns, 8 levels, 1 plane} at (x, y, z) of a 3-D map into shared memory
__device__ __forceinline__ void win_copy(double* dst, const CUtensorMap* map, int x, int y, int z,
                                         uint64_t* bar) {
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
                 : "memory");
}

template<class R>
__global__ void THORX_KATTR_MOM
    momentum_tma_kernel(Geometry g, Phys P, State s, double dt,
                        const __grid_constant__ CUtensorMap map_ps,
                        const __grid_constant__ CUtensorMap map_divg) {
    __shared__ double              sgeo[kRingGeoRows * kTile];
    __shared__ double              sgrad[21 * kTile];
    __shared__ uint64_t            bar[kMomBuf];
    extern __shared__ double       win_raw[];
    // [kMomBuf][kWinFields][kWinSpans][8][kWinW], from the first 128-byte boundary (a box's
    // destination must be 128-byte aligned; every box is 2304 bytes)
    double* const win = win_raw + ((128u - (smem_addr(win_raw) & 127u)) & 127u) / sizeof(double);
    const int     c   = lane_column(g);
    SGeo                           G{};
    if (P.DivDampP)
        G = stage_divm_geo<R>(sgeo, g, c);
    stage_cols(sgrad, g.grad, 21, g.Np, c);
    if (tail_cta()) {
        __syncthreads();
        if (c >= 0)
            momentum_body<5, R>(g, P, s, G, sgrad, dt, c);
        return;
    }
    const int  Np = g.Np, nv = g.nv, tile = g.tile0 + blockIdx.x;
    const int  nst    = (nv + kLevGroups - 1) / kLevGroups;
    const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
    int        xs[kWinSpans], nsp = 0;
#pragma unroll
    for (int sp = 0; sp < kWinSpans; sp++) {
        xs[sp] = g.wspan[tile * kWinSpans + sp];
        nsp += xs[sp] >= 0;
    }
    const uint32_t bytes = nsp * kWinFields * kLevGroups * kWinW * sizeof(double);
    auto           issue = [&](int st) {
        double*   w = win + (st % kMomBuf) * kWinDoubles;
        uint64_t* b = &bar[st % kMomBuf];
        win_expect(b, bytes);
#pragma unroll
        for (int sp = 0; sp < kWinSpans; sp++) {
            if (xs[sp] < 0)
                continue;
            double* d = w + sp * kLevGroups * kWinW;
            win_copy(d, &map_ps, xs[sp], st * kLevGroups, 0, b);
#pragma unroll
            for (int k = 0; k < 3; k++)
                win_copy(d + (1 + k) * kWinField, &map_divg, xs[sp], st * kLevGroups, k, b);
        }
    };
    if (leader) {
        for (int b = 0; b < kMomBuf; b++)
            win_bar_init(&bar[b]);
    }
    __syncthreads();
    int issued = 0;
    if (leader)
        for (; issued < kMomBuf && issued < nst; issued++)
            issue(issued);
    // window offset (span * 8 * kWinW + column - span start) of each point, -1 outside the window
    auto woff = [&](int id) {
        int o = -1;
#pragma unroll
        for (int sp = kWinSpans - 1; sp >= 0; sp--)
            if (xs[sp] >= 0 && id >= xs[sp] && id < xs[sp] + kWinW)
                o = sp * kLevGroups * kWinW + id - xs[sp];
        return o;
    };
    int    onb[7], org[6];
    double fr[3];
    if (c >= 0) {
        onb[0] = woff(c);
#pragma unroll
        for (int j = 0; j < 6; j++) {
            onb[j + 1] = woff(g.nb[j * Np + c]);
            org[j]     = woff(g.ring[j * Np + c]);
        }
#pragma unroll
        for (int k = 0; k < 3; k++)
            fr[k] = g.func_r[k * Np + c];
    }
    for (int st = 0; st < nst; st++) {
        const int b  = st % kMomBuf;
        const bool ok =
            __syncthreads_and(win_wait(&bar[b], (uint32_t)((st / kMomBuf) & 1), kWinPolls));
        if (!ok) {
            if (leader) {
                atomicOr(s.flags, kFlagWait);
                for (int q = st; q < issued; q++) // the copies still in flight
                    win_wait(&bar[q % kMomBuf], (uint32_t)((q / kMomBuf) & 1), kWinPolls);
            }
            return;
        }
        const int lev = st * kLevGroups + threadIdx.y;
        if (c >= 0 && lev < nv) {
            const double* w = win + b * kWinDoubles + threadIdx.y * kWinW;
            double        pv[7];
#pragma unroll
            for (int j = 0; j < 7; j++)
                pv[j] = onb[j] >= 0 ? w[onb[j]]
                                    : gz(s.ps + lev * Np, j == 0 ? c : g.nb[(j - 1) * Np + c]);
            R DivM[3] = {0, 0, 0};
            if (P.DivDampP) {
                double a0[3], ar[6][3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const double* dg = s.divg + (k * nv + lev) * Np;
                    a0[k] = onb[0] >= 0 ? w[(1 + k) * kWinField + onb[0]] : dg[c];
#pragma unroll
                    for (int j = 0; j < 6; j++)
                        ar[j][k] = org[j] >= 0 ? w[(1 + k) * kWinField + org[j]]
                                               : gz(dg, g.ring[j * Np + c]);
                }
                divm_final_vals<6, R>(g, P, G, a0, ar, lev, fr, DivM);
            }
            momentum_apply<R>(g, P, s, sgrad, dt, c, lev, fr, pv, DivM);
        }
        __syncthreads(); // the window of this round is read; the next copy may overwrite it
        if (leader && issued < nst)
            issue(issued++);
    }
}
#endif // THORX_MOM_TMA

// ---------------------------------------------------------------------------------------------
// Small step, vertically implicit part:
//   Prepare_Implicit_Vertical / _Poles (src/headers/dyn/thor_vertical_int.h:566-771),
//   Vertical_Eq (:52-563, Thomas forward elimination and back substitution, FP64),
//   Density_Pressure_Eqs / _Poles (src/headers/dyn/thor_fastmodes.h:255-847).
// Phase 1 (all levels in parallel): Sp, Sd at every level -> shared memory.
// Phase 2 (all interfaces in parallel): the tridiagonal row (aa, bb, cc, -C0) of every interior
//   interface, from the column's values at the two adjacent levels and Sp, Sd -> s.vrows.
// Phase 3 (warp 0, lane = column): the Thomas elimination and back substitution over the rows
//   of its column, with the reference's operation sequence; Whs -> global. Meanwhile warps 1..7
//   compute the horizontal flux divergences of phase 4 (they do not depend on the solve).
// Phase 4 (all levels in parallel): the density and pressure update.
// The rows go through global memory (they stay in L1/L2: the same CTA writes and reads them
// across a barrier); the eliminated coefficients c', d' go to shared memory, so that no global
// store orders the sweep's row loads. Shared memory: div [21][32], Sp/Sd (then the flux
// divergences) [2][nv][32] and c'/d' [2][nv][32], 55 KB at nv = 48, three CTAs per SM.
// Level-only factors come from the per-level tables.
// ---------------------------------------------------------------------------------------------
// ---------------------------------------------------------------------------------------------
// Vertical hyperdiffusion (VertHyDiff: vertical_diff, src/headers/dyn/thor_diff.h:1198-1426, and
// its radial correction in Correct_Horizontal, :882-915). One thread per column: the variables
// u, v, w (momentum over density) and T in turn; each goes through order/2 - 1 applications of the
// reference's second-derivative stencil (values at the ghost levels 0 and nv+1 copied from the
// end levels), the last one scaled by sign Kdv6 rho, and a final application (times Rd for T).
// The column sits in shared memory (two planes of nv+2 values per column). The density part of
// the reference is discarded there (include_rho = false) and is not computed. The results, the
// momentum part with its radial component removed, are added into diffmh, diffw and diffpr,
// where the reference keeps them in diffmv, diffwv and diffprv and every consumer adds the pairs.
// ---------------------------------------------------------------------------------------------
constexpr int kVdCols = 32;

__global__ void __launch_bounds__(kVdCols) vertical_diff_kernel(Geometry g, Phys P, State s) {
    extern __shared__ double vsm[];
    const int nv = g.nv, Np = g.Np, x = threadIdx.x;
    const int c  = (g.tile0 + blockIdx.x) * kVdCols + x;
    double*   b2 = vsm;                       // [nv + 2][kVdCols]
    double*   d  = vsm + (nv + 2) * kVdCols;  // [nv][kVdCols]
    if (c >= g.N)
        return;
    const double* Alt   = g.Altitude;
    const double* Alth  = g.Altitudeh;
    const int     order = P.vhd_order;
    const double  sign  = pow(-1.0, order / 2 + 1);
    const double  A     = P.A;
    const int     max_l = order / 2 - 1;
    const double* fr    = nullptr;
    // one application of the stencil to b2 into d; scale_rd for the temperature's last one
    auto stencil = [&](bool scale_rd) {
        for (int lev = 0; lev < nv; lev++) {
            const double dzi = 1.0 / (Alth[lev + 1] - Alth[lev]);
            double       ri, rup, rlow, dzup, dzlow;
            if (P.DeepModel) {
                ri   = A + Alt[lev];
                rup  = A + Alth[lev + 1];
                rlow = A + Alth[lev];
            }
            else {
                ri = rup = rlow = 1.0;
            }
            if (lev == 0) {
                dzup  = 1.0 / (Alt[1] - Alt[0]);
                dzlow = 1.0 / (2.0 * Alt[0]);
            }
            else if (lev == nv - 1) {
                dzup  = 1.0 / (2 * (Alth[lev + 1] - Alt[lev]));
                dzlow = 1.0 / (Alt[lev] - Alt[lev - 1]);
            }
            else {
                dzup  = 1.0 / (Alt[lev + 1] - Alt[lev]);
                dzlow = 1.0 / (Alt[lev] - Alt[lev - 1]);
            }
            const double up  = b2[(lev + 2) * kVdCols + x], mid = b2[(lev + 1) * kVdCols + x];
            const double low = b2[lev * kVdCols + x];
            const double t   = pow(rup, 2) * (up - mid) * dzup - pow(rlow, 2) * (mid - low) * dzlow;
            d[lev * kVdCols + x] = scale_rd ? t * dzi * P.Rd / pow(ri, 2) : t * dzi / pow(ri, 2);
        }
    };
    double* out[3] = {nullptr, nullptr, nullptr};
    for (int var = 1; var <= 5; var++) {
        for (int lev = 0; lev < nv + 2; lev++) {
            const int    l = lev == 0 ? 0 : (lev == nv + 1 ? nv - 1 : lev - 1);
            const int    i = l * Np + c;
            const double r = s.Rhok[i];
            double       v;
            if (var <= 3)
                v = s.Mhk[((var - 1) * nv + l) * Np + c] / r;
            else if (var == 4)
                v = s.Wk[i] / r;
            else
                v = s.T[i];
            b2[lev * kVdCols + x] = v;
        }
        for (int l = 0; l < max_l; l++) {
            stencil(false);
            const bool last = l == max_l - 1;
            for (int lev = 0; lev < nv; lev++) {
                const double dv = d[lev * kVdCols + x];
                b2[(lev + 1) * kVdCols + x] = last ? sign * s.Rhok[lev * Np + c] * g.Kdv6[lev] * dv : dv;
            }
            b2[x]                   = b2[kVdCols + x];
            b2[(nv + 1) * kVdCols + x] = b2[nv * kVdCols + x];
        }
        stencil(var == 5);
        if (var <= 3) { // the momentum components: kept (planes 0..2 of diff) until all three exist
            out[var - 1] = s.diff + (size_t)(var - 1) * nv * Np;
            for (int lev = 0; lev < nv; lev++)
                out[var - 1][lev * Np + c] = d[lev * kVdCols + x];
            if (var == 3) {
                fr = g.func_r;
                const double f0 = fr[c], f1 = fr[Np + c], f2 = fr[2 * Np + c];
                for (int lev = 0; lev < nv; lev++) {
                    const int i   = lev * Np + c;
                    double    v0 = out[0][i], v1 = out[1][i], v2 = out[2][i];
                    const double dmvr = f0 * v0 + f1 * v1 + f2 * v2;
                    v0 += -f0 * dmvr;
                    v1 += -f1 * dmvr;
                    v2 += -f2 * dmvr;
                    s.diffmh[(0 * nv + lev) * Np + c] += v0;
                    s.diffmh[(1 * nv + lev) * Np + c] += v1;
                    s.diffmh[(2 * nv + lev) * Np + c] += v2;
                }
            }
        }
        else if (var == 4)
            for (int lev = 0; lev < nv; lev++)
                s.diffw[lev * Np + c] += d[lev * kVdCols + x];
        else
            for (int lev = 0; lev < nv; lev++)
                s.diffpr[lev * Np + c] += d[lev * kVdCols + x];
    }
}

// kPart: 0 = the whole fused sequence; 1 = Prepare_Implicit_Vertical and Vertical_Eq only (Whs
// written); 2 = Density_Pressure_Eqs only (horizontal flux divergences on every warp, then the
// update, reading the Whs a part-1 launch wrote). Parts 1 and 2 bracket a physics module's
// fast-mode hook, which the reference calls between Vertical_Eq and Density_Pressure_Eqs
// (src/ESP/thor_driver.cu:1222-1304); they compute what the fused kernel computes, value for value.
//
// Shared memory, [quantity][32 columns]: the div stencil (21 rows), then four nv-row arrays.
// kVertMerge (the default): one gather pass per level computes Prepare_Implicit_Vertical's Sp and
// Sd and Density_Pressure_Eqs' horizontal flux divergences Fr and Fpt together (Mhs is gathered
// once for both; Sd's flux term is exactly -Fr: the same products summed in the same order,
// negated); the arrays are Sp, Sd, Fr, Fpt, and the Thomas sweep writes its eliminated
// coefficients over Sp and Sd, which the rows no longer need. Without kVertMerge the flux
// divergences are gathered by warps 1-7 while warp 0 solves, into the Sp/Sd arrays, and the
// eliminated coefficients have arrays of their own.
#ifndef THORX_VERT_MERGE
#define THORX_VERT_MERGE 1
#endif
#ifndef THORX_VERT_PF
#define THORX_VERT_PF 4
#endif
#ifndef THORX_VERT_SMEM
#define THORX_VERT_SMEM 2
#endif
#ifndef THORX_VG
#define THORX_VG 0
#endif
#if THORX_VG >= 1
#define VLD(p) __ldg(p)
#else
#define VLD(p) (*(p))
#endif
constexpr bool kVertMerge = THORX_VERT_MERGE != 0;
// Where the per-level work arrays live: 2 all in shared memory; 1 Sp and Sd in shared memory, Fr,
// Fpt and the eliminated coefficients in global scratch planes; 0 all in global scratch (shared
// memory holds the div stencil only, and the rest of the SM's 256 KB serves as L1 for the gathers).
constexpr int kVertSmem = THORX_VERT_SMEM;

// One per-level array of a tile: element lev of column lane x at p[lev * ld + ci] (shared memory:
// ld 32, ci the lane; a global scratch plane set: ld Np, ci the column).
struct LevArr {
    double* p;
    int     ld, ci;
    __device__ double& operator[](int lev) const { return p[(size_t)lev * ld + ci]; }
};
constexpr int  kThomasPf  = THORX_VERT_PF; // rows loaded ahead of the elimination (0: none)
constexpr int  kVertPre   = 8;             // levels whose pressure factor warps 1-7 precompute


// The 7-point gathers of one level (rows of sdiv: point j, component k at (j * 3 + k)).
// kSpSd: Sp and Sd of Prepare_Implicit_Vertical (thor_vertical_int.h:566-771);
// kFlux: rscale div(Mhs) and rscale div((Mhs + Mhk) pt) (or the energy form's h + ep + ek) of
// Density_Pressure_Eqs (thor_fastmodes.h:255-847). Each sum runs over the points in the
// reference's order.
template<bool kSpSd, bool kFlux, bool kUni>
__device__ __forceinline__ void vert_gathers(const Geometry& g, const Phys& P, const State& s,
                                             const double* sdiv, const int* nb, int c, int lev,
                                             double& Sp, double& Sd, double& Fr, double& Fpt) {
    const int     Np = g.Np, nv = g.nv, x = threadIdx.x;
    const bool    eeq    = P.energy;
    const double  rscale = g.lt[kLtRscale * g.nvi + lev]; // 1 in the shallow model
    double        sdv[3], spv[3], st[3];
    const double* h   = s.h + lev * Np;
#if THORX_VG >= 2
    // every gather of the level issued before any is used
    double LH[7], LM[7][3], LK[7][3], LP[7], LE[7], LEK[7];
#pragma unroll
    for (int j = 0; j < 7; j++) {
        const int id = nb[j];
        const int q  = lev * Np + (id >= 0 ? id : 0);
        LH[j]        = (kSpSd || (kFlux && eeq)) && id >= 0 ? VLD(s.h + q) : 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            LM[j][k] = id >= 0 ? VLD(s.Mhs + (size_t)k * nv * Np + q) : 0.0;
            LK[j][k] = kFlux && id >= 0 ? VLD(s.Mhk + (size_t)k * nv * Np + q) : 0.0;
        }
        LP[j]  = kFlux && !eeq && id >= 0 ? VLD(s.pt + q) : 0.0;
        LE[j]  = kFlux && eeq && id >= 0 ? VLD(s.ep + q) : 0.0;
        LEK[j] = kFlux && eeq && id >= 0 ? VLD(s.ek + q) : 0.0;
    }
#endif
#pragma unroll
    for (int j = 0; j < 7; j++) {
        const int id = nb[j];
        double    hv = 0.0, ms[3] = {0.0, 0.0, 0.0}, v1[3] = {0.0, 0.0, 0.0}, ptv = 0.0;
#if THORX_VG >= 2
        if (id >= 0) {
            hv = LH[j];
#pragma unroll
            for (int k = 0; k < 3; k++)
                ms[k] = LM[j][k];
            if (kFlux) {
#pragma unroll
                for (int k = 0; k < 3; k++)
                    v1[k] = ms[k] + LK[j][k];
                ptv = eeq ? (hv + LE[j] + LEK[j]) : LP[j];
            }
        }
#else
        {   // every load unconditional (a hole reads this column and is zeroed after), so the
            // compiler may schedule the points' loads together
            const bool ok  = id >= 0;
            const int  idv = ok ? id : c;
            const int  q   = lev * Np + idv;
            if (kSpSd || (kFlux && eeq))
                hv = VLD(h + idv);
            double mk[3];
#pragma unroll
            for (int k = 0; k < 3; k++)
                ms[k] = VLD(s.Mhs + (k * nv + lev) * Np + idv);
            if (kFlux) {
#pragma unroll
                for (int k = 0; k < 3; k++)
                    mk[k] = VLD(s.Mhk + (k * nv + lev) * Np + idv);
                ptv = eeq ? (hv + VLD(s.ep + q) + VLD(s.ek + q)) : VLD(s.pt + q);
            }
            if (!ok) {
                hv  = 0.0;
                ptv = 0.0;
#pragma unroll
                for (int k = 0; k < 3; k++)
                    ms[k] = mk[k] = 0.0;
            }
            if (kFlux)
#pragma unroll
                for (int k = 0; k < 3; k++)
                    v1[k] = ms[k] + mk[k];
        }
#endif
        // explicit roundings: the fused and the split launches (and every instantiation) give the
        // same bits whatever the compiler would contract
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const double d  = sdiv[(j * 3 + k) * kTile + x];
            const double dm = __dmul_rn(d, ms[k]);
            if (j == 0) {
                sdv[k] = dm;
                if (kSpSd)
                    spv[k] = __dmul_rn(dm, hv);
                if (kFlux)
                    st[k] = __dmul_rn(__dmul_rn(d, v1[k]), ptv);
            }
            else {
                sdv[k] = __dadd_rn(sdv[k], dm);
                if (kSpSd)
                    spv[k] = __fma_rn(dm, hv, spv[k]);
                if (kFlux)
                    st[k] = __fma_rn(__dmul_rn(d, v1[k]), ptv, st[k]);
            }
        }
    }
    double fr = 0.0, fpt = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        fr = __fma_rn(rscale, sdv[k], fr);
        if (kFlux)
            fpt = __fma_rn(rscale, st[k], fpt);
    }
    Fr  = fr;
    Fpt = fpt;
    if (kSpSd) {
        const int    i   = lev * Np + c;
        const double RoC = rd_at<kUni>(P, s, i) / (cp_at<kUni>(P, s, i) - rd_at<kUni>(P, s, i));
        double       nflxp = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++)
            nflxp = __fma_rn(-__dmul_rn(RoC, rscale), spv[k], nflxp);
        Sp = nflxp + s.Slowp[i];
        Sd = __dadd_rn(-fr, s.SlowRho[i]);
    }
}

// x^y of the entropy form's pressure update. THORX_VPOW_EXPLOG=1 evaluates it as exp(y log x)
// with CUDA's exp and log (inlined, within a few ulp of pow) instead of pow.
#ifndef THORX_VPOW_EXPLOG
#define THORX_VPOW_EXPLOG 0
#endif
__device__ __forceinline__ double vpow(double x, double y) {
#if THORX_VPOW_EXPLOG
    return exp(y * log(x));
#else
    return pow(x, y);
#endif
}

// The entropy form's potential-temperature factor of Density_Pressure_Eqs at (c, lev): ptc =
// (P_Ref / (Rd r)) (p / P_Ref)^(Cv / Cp) with the state before the update. It does not depend on
// the vertical solve, so warps 1-7 evaluate it while warp 0 runs the Thomas sweep.
template<bool kUni>
__device__ __forceinline__ double vert_ptc(const Phys& P, const State& s, int i) {
    const double Cv = cp_at<kUni>(P, s, i) - rd_at<kUni>(P, s, i);
    const double r  = s.Rhok[i] + s.Rhos[i];
    return (P.P_Ref / (rd_at<kUni>(P, s, i) * r)) * vpow(div_rcp(s.ps[i] + s.pk[i], P.P_Ref, P.rP_Ref), Cv / cp_at<kUni>(P, s, i));
}

// Density_Pressure_Eqs at (c, lev): the vertical flux terms from the solved Whs, the update of
// Rhos and ps (thor_fastmodes.h:255-847). Divisions by level constants go through div_rcp with
// tabulated reciprocals (the IEEE quotients). ptc_pre: vert_ptc's value if precomputed.
// The state values one level's update reads (the cell's and its two interfaces'), all loaded
// before any arithmetic, so that their latencies overlap: glevel 6, 48 levels: vertical 2.57 ->
// 2.34 ms per step (the update phase 21.6 -> ~16 us per CTA) against loads issued where the
// arithmetic first uses them, behind its branches; the same bits. Loading the next level's values ahead of the current
// level's update as well (registers for two levels) spills and gains nothing more.
struct VIn {
    double rk, rs, srho, pk, dpr, qh, et; // Rhok, Rhos, SlowRho, pk, diffpr, Qheat, Etotal
    double whl, wht, whkl, whkt, phl, pht; // Whs, Whk, the interfaces' potential temperature (or
                                           // enthalpy) below and above
};
__device__ __forceinline__ VIn vert_load(const Geometry& g, const Phys& P, const State& s, int c,
                                         int lev) {
    const int  Np = g.Np;
    const bool eeq = P.energy;
    const int  i   = lev * Np + c;
    auto       phv = [&](int l) -> double {
        const int q = l * Np + c;
        return eeq ? (s.hh[q] + s.eph[q] + s.ekh[q]) : s.pth[q];
    };
    VIn v;
    v.rk   = s.Rhok[i];
    v.rs   = s.Rhos[i];
    v.srho = s.SlowRho[i];
    v.pk   = s.pk[i];
    v.dpr  = s.diffpr[i];
    v.qh   = s.Qheat[i];
    v.et   = eeq ? s.Etotal[i] : 0.0;
    v.whl  = lev == 0 ? 0.0 : s.Whs[lev * Np + c];
    v.wht  = s.Whs[(lev + 1) * Np + c];
    v.whkl = lev == 0 ? 0.0 : s.Whk[lev * Np + c];
    v.whkt = s.Whk[(lev + 1) * Np + c];
    v.phl  = lev == 0 ? 0.0 : phv(lev);
    v.pht  = phv(lev + 1);
    return v;
}

template<bool kUni>
__device__ __forceinline__ void vert_update(const Geometry& g, const Phys& P, const State& s,
                                            double deltat, int c, int lev, bool pole,
                                            double nflxr, double nflxpt, const double* ptc_pre,
                                            const VIn* in = nullptr) {
    const int     Np = g.Np, nvi = g.nvi, nv = g.nv;
    const double* lt   = g.lt;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    const bool    deep = P.DeepModel, eeq = P.energy, ghv = P.GravHeightVar;
    const VIn     v    = in ? *in : vert_load(g, P, s, c, lev);
    const int     i    = lev * Np + c;
    const double  Cv   = cp_at<kUni>(P, s, i) - rd_at<kUni>(P, s, i);
    const double  dz   = Alth[lev + 1] - Alth[lev];
    double        r2p, r2m, r2l, dr2dz, rdr2dz, rdzr2m;
    if (deep) {
        r2p    = lt[kLtR2hD * nvi + lev + 1];
        r2m    = lt[kLtR2cD * nvi + lev];
        r2l    = lt[kLtR2hD * nvi + lev];
        dr2dz  = lt[kLtDr2dz * nvi + lev];
        rdr2dz = lt[kLtRDr2dz * nvi + lev];
        rdzr2m = lt[kLtRDzR2m * nvi + lev];
    }
    else {
        r2p = r2m = r2l = 1.0;
        dr2dz           = r2m * dz;
        rdr2dz = rdzr2m = lt[kLtRDz * nvi + lev]; // dz r2m = dz exactly
    }
    double whl, wht, whl2, wht2, phl, pht;
    if (lev == 0) {
        whl  = 0.0;
        wht  = v.wht;
        whl2 = 0.0;
        wht2 = wht + v.whkt;
        phl  = 0.0;
        pht  = v.pht;
    }
    else {
        whl  = v.whl;
        wht  = v.wht;
        whl2 = whl + v.whkl;
        wht2 = wht + v.whkt;
        phl  = v.phl;
        pht  = v.pht;
    }
    const double dwdz   = pole ? div_rcp(wht * r2p - whl * r2l, dz * r2m, rdzr2m)
                               : div_rcp(wht * r2p - whl * r2l, dr2dz, rdr2dz);
    const double dwptdz = div_rcp(wht2 * pht * r2p - whl2 * phl * r2l, dz * r2m, rdzr2m);
    double       aux    = -(nflxpt + dwptdz) * deltat;
    const double rk_    = v.rk;
    const double rs     = v.rs;
    const double r      = rk_ + rs;
    // the entropy form's factor from the state before the update (Rhos is overwritten next)
    const double ptc = eeq ? 0.0 : (ptc_pre ? *ptc_pre : vert_ptc<kUni>(P, s, i));
    nflxr += dwdz;
    const double rhos_new = rs + (v.srho - nflxr) * deltat;
    s.Rhos[i]             = rhos_new;
    if (eeq) {
        const double Gravit = P.Gravit;
        aux += v.et + (v.dpr) * deltat + v.qh * deltat;
        s.Etotal[i] = aux;
        const double m0 = s.Mhs[(0 * nv + lev) * Np + c] + s.Mhk[(0 * nv + lev) * Np + c];
        const double m1 = s.Mhs[(1 * nv + lev) * Np + c] + s.Mhk[(1 * nv + lev) * Np + c];
        const double m2 = s.Mhs[(2 * nv + lev) * Np + c] + s.Mhk[(2 * nv + lev) * Np + c];
        const double w  = div_rcp(whl2 * (Alth[lev + 1] - Alt[lev]) + wht2 * (Alt[lev] - Alth[lev]),
                                  Alth[lev + 1] - Alth[lev], lt[kLtRDz * nvi + lev]);
        double Epot_kin;
        if (ghv)
            Epot_kin = (rhos_new + rk_) * Gravit * lt[kLtGhv * nvi + lev] * Alt[lev]
                       + 0.5 * (pow(m0, 2) + pow(m1, 2) + pow(m2, 2) + pow(w, 2)) / (rhos_new + rk_);
        else
            Epot_kin = (rhos_new + rk_) * Gravit * Alt[lev]
                       + 0.5 * (pow(m0, 2) + pow(m1, 2) + pow(m2, 2) + pow(w, 2)) / (rhos_new + rk_);
        s.ps[i] = rd_at<kUni>(P, s, i) / Cv * (aux - Epot_kin) - v.pk;
    }
    else {
        aux += ptc * r;
        const double pn = P.P_Ref * vpow(div_rcp(rd_at<kUni>(P, s, i) * aux, P.P_Ref, P.rP_Ref), cp_at<kUni>(P, s, i) / Cv);
        s.ps[i]         = pn - v.pk + (v.dpr) * deltat + rd_at<kUni>(P, s, i) / Cv * v.qh * deltat;
    }
}

// Rows of the elimination staged through shared memory by cp.async, kThomasRing interfaces
// ahead (0: the register prefetch of kThomasPf interfaces instead). The copies hold no registers
// while in flight, so the ring runs further ahead of the chain than registers allow. glevel 6,
// 48 levels: vertical 2.84 ms per step with the register prefetch, 2.57 with a ring of 8 (the
// sweep 14.2 -> 10.0 us per CTA; the register prefetch's spills gone), 2.59 with 4, 2.95 with 16
// (70.5 KB of shared memory per CTA leave the gathers less L1); the same bits.
#ifndef THORX_THOMAS_RING
#define THORX_THOMAS_RING 8
#endif
constexpr int kThomasRing = THORX_THOMAS_RING;
static_assert(kThomasRing == 0 || (kThomasRing & (kThomasRing - 1)) == 0, "a power of two");
// doubles of the vertical kernel's dynamic shared memory before the ring: sdiv [21][32] and the
// per-level arrays of the columns ([4][nv][32] with THORX_VERT_SMEM=2)
__host__ __device__ inline size_t vertical_ring_offset(int nv) {
    return (size_t)kTile * (21 + (kVertSmem == 2 ? 4 : kVertSmem == 1 ? 2 : 0) * nv);
}
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                     (unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template<int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The Thomas elimination and back substitution of one column (Vertical_Eq,
// thor_vertical_int.h:463-484, same operations) from the row planes, the eliminated coefficients in
// shared memory sc/sd [nv][32]; rows are loaded ahead of their use (kThomasRing interfaces through
// the shared-memory ring `ring` [kThomasRing][4][32], else kThomasPf into registers), so the chain
// of dependent divisions does not wait on memory.
__device__ __forceinline__ void thomas_column(const Geometry& g, const State& s, LevArr sc,
                                              LevArr sd, int c, double* ring) {
    const int     nv = g.nv, Np = g.Np, nvi = g.nvi;
    const double* ra = s.vrows;
    const double* rb = ra + (size_t)nvi * Np;
    const double* rc = rb + (size_t)nvi * Np;
    const double* rd = rc + (size_t)nvi * Np;
    double        cprev = 0, dprev = 0;
    if constexpr (kThomasRing > 0) {
        const int x     = threadIdx.x;
        auto      fetch = [&](int lev) { // interface lev into slot (lev - 1) % kThomasRing
            if (lev < nv) {
                double*   r = ring + ((lev - 1) & (kThomasRing - 1)) * 4 * kTile + x;
                const int q = lev * Np + c;
                cp_async8(r, ra + q);
                cp_async8(r + kTile, rb + q);
                cp_async8(r + 2 * kTile, rc + q);
                cp_async8(r + 3 * kTile, rd + q);
            }
            cp_async_commit(); // one group per interface, empty past the top
        };
        for (int k = 0; k < kThomasRing; k++)
            fetch(1 + k);
        for (int lev = 1; lev < nv; lev++) {
            cp_async_wait<kThomasRing - 1>(); // the group of interface lev is complete
            const double* r  = ring + ((lev - 1) & (kThomasRing - 1)) * 4 * kTile + x;
            const double  aa = r[0], bb = r[kTile];
            double        ccv = r[2 * kTile], ddv = r[3 * kTile];
            if (lev == 1) {
                ccv = ccv / bb;
                ddv = ddv / bb;
            }
            else {
                const double t = 1.0 / (bb - cprev * aa);
                ccv *= t;
                ddv = (ddv - dprev * aa) * t;
            }
            sc[lev] = ccv;
            sd[lev] = ddv;
            cprev = ccv;
            dprev = ddv;
            fetch(lev + kThomasRing); // the slot's values are used: refill it
        }
        cp_async_wait<0>();
    }
    else if constexpr (kThomasPf > 0) {
        constexpr int kQ = kThomasPf > 0 ? kThomasPf : 1;
        double        qa[kQ], qb[kQ], qc[kQ], qd[kQ];
#pragma unroll
        for (int k = 0; k < kThomasPf; k++) {
            const int l = 1 + k;
            if (l < nv) {
                const int q = l * Np + c;
                qa[k] = ra[q], qb[k] = rb[q], qc[k] = rc[q], qd[k] = rd[q];
            }
        }
        for (int base = 1; base < nv; base += kThomasPf) {
#pragma unroll
            for (int k = 0; k < kThomasPf; k++) {
                const int lev = base + k;
                if (lev < nv) {
                    const double aa = qa[k], bb = qb[k];
                    double       ccv = qc[k], ddv = qd[k];
                    const int    ln  = lev + kThomasPf;
                    if (ln < nv) {
                        const int q = ln * Np + c;
                        qa[k] = ra[q], qb[k] = rb[q], qc[k] = rc[q], qd[k] = rd[q];
                    }
                    if (lev == 1) {
                        ccv = ccv / bb;
                        ddv = ddv / bb;
                    }
                    else {
                        const double t = 1.0 / (bb - cprev * aa);
                        ccv *= t;
                        ddv = (ddv - dprev * aa) * t;
                    }
                    sc[lev] = ccv;
                    sd[lev] = ddv;
                    cprev = ccv;
                    dprev = ddv;
                }
            }
        }
    }
    else {
#pragma unroll 2
        for (int lev = 1; lev < nv; lev++) {
            const int    q  = lev * Np + c;
            const double aa = ra[q], bb = rb[q];
            double       ccv = rc[q], ddv = rd[q];
            if (lev == 1) {
                ccv = ccv / bb;
                ddv = ddv / bb;
            }
            else {
                const double t = 1.0 / (bb - cprev * aa);
                ccv *= t;
                ddv = (ddv - dprev * aa) * t;
            }
            sc[lev] = ccv;
            sd[lev] = ddv;
            cprev = ccv;
            dprev = ddv;
        }
    }
    double w           = 0.0;
    s.Whs[nv * Np + c] = 0.0;
    for (int lev = nv - 1; lev > 0; lev--) {
        const double cc = sc[lev], dd = sd[lev];
        w               = (lev == nv - 1) ? dd : (-cc * w + dd);
        s.Whs[lev * Np + c] = w;
    }
    s.Whs[c] = 0.0;
}

#ifndef THORX_VERT_CLOCK
#define THORX_VERT_CLOCK 0
#endif
#if THORX_VERT_CLOCK
// phase timestamps of each CTA of the last launch: [cta][8] = smid, globaltimer at the start,
// clock64 at the start and after phases 1, 2, 3, the latest warp end, the end of the sweep
// (warp 0), the latest end of the other warps' phase-3 work
__device__ unsigned long long g_vclock[16384 * 8];
__device__ __forceinline__ unsigned long long vclk() { return clock64(); }
#define VCLOCK(slot)                                                                              \
    do {                                                                                           \
        if (threadIdx.x == 0 && threadIdx.y == 0 && blockIdx.x < 16384)                           \
            g_vclock[blockIdx.x * 8 + (slot)] = vclk();                                            \
    } while (0)
#else
#define VCLOCK(slot) do {} while (0)
#endif
template<int kPart, bool kUni>
__global__ void THORX_KATTR_VERT
    vertical_kernel(Geometry g, Phys P, State s, double deltat) {
    extern __shared__ double smem[];
    const int nv = g.nv, nvi = g.nvi, Np = g.Np;
    const int c0 = (g.tile0 + blockIdx.x) * kTile, x = threadIdx.x, c = c0 + x;
    double*   sdiv = smem;
    // the four per-level arrays: in shared memory after sdiv, or global scratch planes after the
    // four row planes of s.vrows (kVertSmem)
    double*   gscr = s.vrows + (size_t)4 * nvi * Np;
    auto      arr  = [&](int k) -> LevArr {
        const bool in_smem = kVertSmem == 2 || (kVertSmem == 1 && k < 2);
        return in_smem ? LevArr{sdiv + 21 * kTile + (size_t)k * nv * kTile, kTile, x}
                            : LevArr{gscr + (size_t)k * nv * Np, Np, c};
    };
    const LevArr sSp = arr(0), sSd = arr(1), sX = arr(2), sY = arr(3);
    // merged: Fr, Fpt in X, Y, eliminated c', d' over Sp, Sd; otherwise c', d' in X, Y and Fr,
    // Fpt over Sp, Sd (global scratch keeps them apart: planes 4 and 5 for c', d')
    const LevArr sFr  = kVertMerge ? sX : sSp;
    const LevArr sFpt = kVertMerge ? sY : sSd;
    const LevArr sCp  = kVertSmem < 2 ? arr(4) : (kVertMerge ? sSp : sX);
    const LevArr sDp  = kVertSmem < 2 ? arr(5) : (kVertMerge ? sSd : sY);
    stage(sdiv, g.div, 21, Np, c0);
    __syncthreads();
#if THORX_VERT_CLOCK
    if (threadIdx.x == 0 && threadIdx.y == 0 && blockIdx.x < 16384) {
        unsigned smid, gt_lo, gt_hi;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        unsigned long long gt;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(gt));
        (void)gt_lo, (void)gt_hi;
        g_vclock[blockIdx.x * 8 + 0] = smid;
        g_vclock[blockIdx.x * 8 + 1] = gt;
        g_vclock[blockIdx.x * 8 + 6] = 0;
        g_vclock[blockIdx.x * 8 + 7] = 0;
    }
#endif
    VCLOCK(2);
    const bool    active = c < g.N;
    const double  Gravit = P.Gravit;
    const bool    deep = P.DeepModel, nonh = P.NonHydro, ghv = P.GravHeightVar;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    const double* lt   = g.lt;
    double*       ra   = s.vrows;                      // rows: a, b, c, d planes
    double*       rb   = ra + (size_t)nvi * Np;
    double*       rc   = rb + (size_t)nvi * Np;
    double*       rd   = rc + (size_t)nvi * Np;
    int           nb[7];
    bool          pole = false;
    if (active) {
        nb[0] = c;
        for (int j = 0; j < 6; j++)
            nb[j + 1] = g.nb[j * Np + c];
        pole = (g.cflag[c] & kPole) != 0;
    }

    // ---- phase 1: Sp, Sd (Prepare_Implicit_Vertical), merged: also Fr, Fpt ----
    if (kPart != 2 && active)
        for (int lev = threadIdx.y; lev < nv; lev += kLevGroups) {
            double Sp, Sd, Fr, Fpt;
            if (kVertMerge && kPart == 0) {
                vert_gathers<true, true, kUni>(g, P, s, sdiv, nb, c, lev, Sp, Sd, Fr, Fpt);
                sFr[lev]  = Fr;
                sFpt[lev] = Fpt;
            }
            else
                vert_gathers<true, false, kUni>(g, P, s, sdiv, nb, c, lev, Sp, Sd, Fr, Fpt);
            sSp[lev] = Sp;
            sSd[lev] = Sd;
        }
    if (kPart != 2)
        __syncthreads();
    VCLOCK(3);

    // ---- phase 2: tridiagonal rows at the interior interfaces ----
    if (kPart != 2 && active) {
        const double dt2 = pow(deltat, 2.0);
        for (int lev = 1 + threadIdx.y; lev < nv; lev += kLevGroups) {
            const double alth = Alth[lev];
            const double alt = Alt[lev], altl = Alt[lev - 1];
            double       hp = s.hh[(lev + 1) * Np + c], h = s.hh[lev * Np + c], hm = s.hh[(lev - 1) * Np + c];
            const double gp = s.gtilh[(lev + 1) * Np + c], gg = s.gtilh[lev * Np + c], gm = s.gtilh[(lev - 1) * Np + c];
            const int    iu = lev * Np + c, il = (lev - 1) * Np + c;
            const double p = s.ps[iu], pl = s.ps[il], r = s.Rhos[iu], rl = s.Rhos[il];
            // every state value of the row loaded before the arithmetic's branches
            const double Srh = s.SlowWh[lev * Np + c], whs_v = s.Whs[lev * Np + c];
            const double Sp = sSp[lev], Spl = sSp[lev - 1];
            const double Sd = sSd[lev], Sdl = sSd[lev - 1];
            const double CRddl = (cp_at<kUni>(P, s, il) - rd_at<kUni>(P, s, il)) / (rd_at<kUni>(P, s, il) * deltat * deltat);
            const double CRddu = (cp_at<kUni>(P, s, iu) - rd_at<kUni>(P, s, iu)) / (rd_at<kUni>(P, s, iu) * deltat * deltat);
            double       GCoRl, GCoRu;
            if (ghv) {
                GCoRl = Gravit * lt[kLtGhv * nvi + lev - 1] * (cp_at<kUni>(P, s, il) - rd_at<kUni>(P, s, il)) / rd_at<kUni>(P, s, il);
                GCoRu = Gravit * lt[kLtGhv * nvi + lev] * (cp_at<kUni>(P, s, iu) - rd_at<kUni>(P, s, iu)) / rd_at<kUni>(P, s, iu);
            }
            else {
                GCoRl = Gravit * (cp_at<kUni>(P, s, il) - rd_at<kUni>(P, s, il)) / rd_at<kUni>(P, s, il);
                GCoRu = Gravit * (cp_at<kUni>(P, s, iu) - rd_at<kUni>(P, s, iu)) / rd_at<kUni>(P, s, iu);
            }
            const double dzp   = lt[kLtDzp * nvi + lev];
            const double dzh   = lt[kLtDzh * nvi + lev]; // RN(1 / (alt - altl))
            const double dzm   = lt[kLtDzm * nvi + lev];
            const double dzph  = dzp * dzh;
            const double dzmh  = dzm * dzh;
            const double intl  = lt[kLtIntl * nvi + lev];
            const double inttm = lt[kLtInttm * nvi + lev];
            double       aa, bb, ccv;
            const double CRdd = div_rcp(CRddl * (alt - alth) + CRddu * (alth - altl), alt - altl, dzh);
            const double GCoR = div_rcp(GCoRl * (alt - alth) + GCoRu * (alth - altl), alt - altl, dzh);
            if (deep) {
                hp                = hp * lt[kLtR2hI * nvi + lev + 1];
                h                 = h * lt[kLtR2hI * nvi + lev];
                hm                = hm * lt[kLtR2hI * nvi + lev - 1];
                const double or2  = lt[kLtOr2 * nvi + lev];
                const double tor3 = lt[kLtTor3 * nvi + lev];
                ccv               = -dzph * or2 * hp - inttm * (gp + GCoR - tor3 * hp);
                if (nonh)
                    bb = CRdd + (dzph + dzmh) * or2 * h + (intl - inttm) * (gg + GCoR - tor3 * h);
                else
                    bb = (dzph + dzmh) * or2 * h + (intl - inttm) * (gg + GCoR - tor3 * h);
                aa = -dzmh * or2 * hm + intl * (gm + GCoR - tor3 * hm);
            }
            else {
                ccv = -dzph * hp - inttm * (gp + GCoR);
                if (nonh)
                    bb = CRdd + (dzph + dzmh) * h + (intl - inttm) * (gg + GCoR);
                else
                    bb = (dzph + dzmh) * h + (intl - inttm) * (gg + GCoR);
                aa = -dzmh * hm + intl * (gm + GCoR);
            }
            const double dSpdz = (Sp - Spl) * dzh;
            const double dPdz  = (p - pl) * dzh;
            const double intt2 = lt[kLtHIntt * nvi + lev];
            const double intl2 = lt[kLtHIntl * nvi + lev];
            const double rhohs = rl * intt2 + r * intl2;
            const double Sdh   = Sdl * intt2 + Sd * intl2;
            const double whs   = nonh ? whs_v : 0.0;
            double       C0;
            if (!nonh) {
                if (ghv) {
                    const double gh = lt[kLtGhv * nvi + lev];
                    C0 = (dt2 * dSpdz + dt2 * Gravit * gh * Sdh + Gravit * gh * deltat * rhohs
                          + deltat * dPdz - deltat * Srh)
                         * (CRdd);
                }
                else
                    C0 = (dt2 * dSpdz + dt2 * Gravit * Sdh + Gravit * deltat * rhohs + deltat * dPdz
                          - deltat * Srh)
                         * (CRdd);
            }
            else {
                if (ghv) {
                    const double gh = lt[kLtGhv * nvi + lev];
                    C0 = (-whs + dt2 * dSpdz + dt2 * Gravit * gh * Sdh + Gravit * gh * deltat * rhohs
                          + deltat * dPdz - deltat * Srh)
                         * (CRdd);
                }
                else
                    C0 = (-whs + dt2 * dSpdz + dt2 * Gravit * Sdh + Gravit * deltat * rhohs
                          + deltat * dPdz - deltat * Srh)
                         * (CRdd);
            }
            ra[lev * Np + c] = aa;
            rb[lev * Np + c] = bb;
            rc[lev * Np + c] = ccv;
            rd[lev * Np + c] = -C0;
        }
    }
    if (kPart != 2)
        __syncthreads();
    VCLOCK(4);

    // ---- phase 3: the Thomas sweep (warp 0); meanwhile the other warps compute what the update
    // needs and the solve does not change: merged, the pressure factor of their update levels;
    // otherwise the horizontal flux divergences (all warps in part 2) ----
    const bool eeq = P.energy;
    double     pre[kVertPre];
    if (kPart != 2 && threadIdx.y == 0) {
        if (active)
            thomas_column(g, s, sCp, sDp, c, smem + vertical_ring_offset(nv));
        VCLOCK(5);
    }
    else if (kPart == 0 && kVertMerge) {
        if (active && !eeq) {
#pragma unroll
            for (int k = 0; k < kVertPre; k++) {
                const int lev = (int)threadIdx.y - 1 + k * (kLevGroups - 1);
                if (lev < nv)
                    pre[k] = vert_ptc<kUni>(P, s, lev * Np + c);
            }
        }
    }
    else if (kPart != 1 && active) {
        const int first = kPart == 2 ? (int)threadIdx.y : (int)threadIdx.y - 1;
        const int step  = kPart == 2 ? kLevGroups : kLevGroups - 1;
        for (int lev = first; lev < nv; lev += step) {
            double Sp, Sd, Fr, Fpt;
            vert_gathers<false, true, kUni>(g, P, s, sdiv, nb, c, lev, Sp, Sd, Fr, Fpt);
            sFr[lev]  = Fr;
            sFpt[lev] = Fpt;
        }
    }
#if THORX_VERT_CLOCK
    if (threadIdx.y != 0 && threadIdx.x == 0 && blockIdx.x < 16384)
        atomicMax(&g_vclock[blockIdx.x * 8 + 7], vclk());
#endif
    __syncthreads();
#if THORX_VERT_CLOCK
    struct EndMark {
        __device__ ~EndMark() {
            if (threadIdx.x == 0 && blockIdx.x < 16384)
                atomicMax(&g_vclock[blockIdx.x * 8 + 6], vclk());
        }
    } end_mark;
#endif
    if (kPart == 1 || !active)
        return;

    // ---- phase 4: Density_Pressure_Eqs, vertical terms and the update ----
    if (kPart == 0 && kVertMerge) {
        // warps 1-7, the levels whose pressure factor they computed during the sweep
        if (threadIdx.y == 0)
            return;
#pragma unroll
        for (int k = 0; k < kVertPre; k++) {
            const int lev = (int)threadIdx.y - 1 + k * (kLevGroups - 1);
            if (lev < nv)
                vert_update<kUni>(g, P, s, deltat, c, lev, pole, sFr[lev], sFpt[lev],
                            eeq ? nullptr : &pre[k]);
        }
        for (int lev = (int)threadIdx.y - 1 + kVertPre * (kLevGroups - 1); lev < nv;
             lev += kLevGroups - 1)
            vert_update<kUni>(g, P, s, deltat, c, lev, pole, sFr[lev], sFpt[lev], nullptr);
    }
    else
        for (int lev = threadIdx.y; lev < nv; lev += kLevGroups)
            vert_update<kUni>(g, P, s, deltat, c, lev, pole, sFr[lev], sFpt[lev], nullptr);
}

// ---------------------------------------------------------------------------------------------
// End of an RK stage: UpdateRK2 (src/headers/dyn/thor_auxiliary.h:420-529, no module arrays).
// ---------------------------------------------------------------------------------------------
// A CTA is one 32-column tile; warp y owns the contiguous levels [y chunk, (y + 1) chunk). Before a
// barrier each warp reads the interface just above its chunk (the next warp writes it); then it
// walks its chunk upward, so every other interface it reads is one it has not written yet. Eight
// warps of 6 levels at 48 levels (glevel 6: 0.204 ms per step; 4 warps of 12 levels: 0.235, 6:
// 0.239, 12: 0.223, 16: 0.278; the same bits): more warps keep more loads in flight per SM.
// The interpolation weights are the level tables' values of the same expressions (level 0, whose
// lower interface the reference takes as 0, evaluates them here).
#ifndef THORX_RK2_GROUPS
#define THORX_RK2_GROUPS 8
#endif
constexpr int kRk2Groups = THORX_RK2_GROUPS;

__global__ void __launch_bounds__(kTile* kRk2Groups) update_rk2_kernel(Geometry g, Phys P, State s) {
    const int  c  = (g.tile0 + blockIdx.x) * kTile + threadIdx.x;
    const int  Np = g.Np, nv = g.nv, nvi = g.nvi;
    const bool active = c < g.N;
    const int  chunk  = (nv + kRk2Groups - 1) / kRk2Groups;
    const int  l0 = threadIdx.y * chunk, l1 = min(nv, l0 + chunk);
    auto       whk_after = [&](int i) -> double { // interface value after the update
        return (i == 0 || i == nv) ? 0.0 : s.Whk[i * Np + c] + s.Whs[i * Np + c];
    };
    double top = 0.0, whl = 0.0;
    if (active && l0 < l1) {
        top = whk_after(l1);
        whl = whk_after(l0);
    }
    __syncthreads();
    if (!active || l0 >= l1)
        return;
    double fr[3];
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    const double* lt = g.lt;
#pragma unroll 2
    for (int lev = l0; lev < l1; lev++) {
        const double wht = (lev + 1 == l1) ? top : whk_after(lev + 1);
        double       intt, intl;
        if (lev == 0) {
            const double xi = g.Altitude[0], xim = 0.0, xip = g.Altitudeh[1];
            intt = (xi - xip) / (xim - xip);
            intl = (xi - xim) / (xip - xim);
        }
        else {
            intt = lt[kLtCIntt * nvi + lev];
            intl = lt[kLtCIntl * nvi + lev];
        }
        const int    i   = lev * Np + c;
        const double Mx  = s.Mhs[(0 * nv + lev) * Np + c] + s.Mhk[(0 * nv + lev) * Np + c];
        const double My  = s.Mhs[(1 * nv + lev) * Np + c] + s.Mhk[(1 * nv + lev) * Np + c];
        const double Mz  = s.Mhs[(2 * nv + lev) * Np + c] + s.Mhk[(2 * nv + lev) * Np + c];
        const double aux = Mx * fr[0] + My * fr[1] + Mz * fr[2];
        s.Mhk[(0 * nv + lev) * Np + c] = Mx - aux * fr[0];
        s.Mhk[(1 * nv + lev) * Np + c] = My - aux * fr[1];
        s.Mhk[(2 * nv + lev) * Np + c] = Mz - aux * fr[2];
        s.Rhok[i] += s.Rhos[i];
        s.pk[i] += s.ps[i];
        s.Wk[i]  = whl * intt + wht * intl;
        s.Whk[i] = whl; // whk_after(lev)
        whl      = wht;
    }
    if (l1 == nv)
        s.Whk[nv * Np + c] = 0.0;
}

// the context's tiles (all of them without a partition), and the same plus the five-neighbour tail
inline dim3 tile_grid(const Geometry& g) { return dim3(g.ntile); }
inline dim3 tile_grid_tail(const Geometry& g) { return dim3(g.ntile + 1); }
inline dim3 tile_block() { return dim3(kTile, kLevGroups); }

// ---------------------------------------------------------------------------------------------
// Self-check of div_rcp against the IEEE quotient: n random pairs per type from SplitMix64 on
// (seed, index); exponents over +-300 (double) and +-60 (float); every second pair has a near-exact
// quotient (a = b c rounded), where a wrong last bit would show first. cnt[0] / cnt[1] count the
// double / float pairs whose bits differ.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long splitmix(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double rand_double(unsigned long long r, unsigned long long e, int emin,
                                              int emax) {
    const int          ex   = emin + (int)(e % (unsigned long long)(emax - emin + 1));
    unsigned long long bits = ((unsigned long long)(ex + 1023) << 52) | (r & ((1ull << 52) - 1));
    return __longlong_as_double((long long)(bits | ((r >> 63) << 63)));
}
__device__ __forceinline__ float rand_float(unsigned long long r, unsigned long long e, int emin,
                                            int emax) {
    const int    ex   = emin + (int)(e % (unsigned long long)(emax - emin + 1));
    unsigned int bits = ((unsigned int)(ex + 127) << 23) | (unsigned int)(r & ((1u << 23) - 1));
    return __int_as_float((int)(bits | (unsigned int)((r >> 63) << 31)));
}
__global__ void div_check_kernel(long long n, unsigned long long seed, unsigned long long* cnt) {
    unsigned long long bad_d = 0, bad_f = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        unsigned long long k = seed ^ ((unsigned long long)i * 0xD1B54A32D192ED03ull);
        const unsigned long long r0 = splitmix(k), r1 = splitmix(r0), r2 = splitmix(r1),
                                 r3 = splitmix(r2);
        double a, b;
        float  af, bf;
        if (i & 1) {
            b  = rand_double(r0, r1 >> 40, -2, 2);
            a  = b * rand_double(r2, r3 >> 40, -2, 2);
            bf = rand_float(r1, r0 >> 40, -2, 2);
            af = bf * rand_float(r3, r2 >> 40, -2, 2);
        }
        else {
            a  = rand_double(r0, r1 >> 40, -300, 300);
            b  = rand_double(r2, r3 >> 40, -300, 300);
            af = rand_float(r1, r0 >> 40, -60, 60);
            bf = rand_float(r3, r2 >> 40, -60, 60);
        }
        const double q = a / b, qr = div_rcp(a, b, 1.0 / b);
        bad_d += __double_as_longlong(q) != __double_as_longlong(qr);
        const float qf = af / bf, qfr = div_rcp(af, bf, 1.0f / bf);
        bad_f += __float_as_int(qf) != __float_as_int(qfr);
    }
    if (bad_d)
        atomicAdd(cnt, bad_d);
    if (bad_f)
        atomicAdd(cnt + 1, bad_f);
}

} // namespace

int max_levels() { return 128; }

void launch_level_tables(const Geometry& g, const Phys& P, double* lt, cudaStream_t st) {
    level_tables_kernel<<<(g.nvi + 127) / 128, 128, 0, st>>>(g, P, lt);
}
void launch_stencil_weights(const Geometry& g, double* lapw, float* dmw, double* dmw64,
                            cudaStream_t st) {
    stencil_weights_kernel<<<(g.N + kTile - 1) / kTile, kTile, 0, st>>>(g, lapw, dmw, dmw64);
}

void launch_sponge_trig(const Geometry& g, double* trig, cudaStream_t st) {
    sponge_trig_kernel<<<(g.N + kColBlock - 1) / kColBlock, kColBlock, 0, st>>>(g, trig);
}
void launch_sponge_means(const Geometry& g, const Phys& P, const Sponge& sp, const SpongeIn& in,
                         cudaStream_t st) {
    sponge_means_kernel<<<dim3(sp.nlat, g.nv), kSpongeThreads, 0, st>>>(g, P, sp, in);
}
void launch_sponge_explicit(const Geometry& g, const Phys& P, const Sponge& sp, const State& s,
                            cudaStream_t st) {
    sponge_explicit_kernel<<<(g.N + kColBlock - 1) / kColBlock, kColBlock, 0, st>>>(g, P, sp, s);
}
void launch_profx(const Geometry& g, const Phys& P, const Sponge& sp, const State& s, bool finish,
                  cudaStream_t st) {
    static_assert(kProfxCols == kTile, "ProfX blocks are tiles");
    profx_kernel<<<g.ntile, dim3(kProfxCols, kProfxGroups), 0, st>>>(
        g, P, sp, s, finish);
}
void launch_profx_finish(const Geometry& g, const State& s, cudaStream_t st) {
    profx_finish_kernel<<<(g.ntile * kTile + kColBlock - 1) / kColBlock, kColBlock, 0, st>>>(g, s);
}
void launch_adv_temp(const Geometry& g, const Phys& P, const State& s, cudaStream_t st) {
    if (P.uniform_thermo)
        adv_temp_kernel<true><<<tile_grid(g), tile_block(), 0, st>>>(g, P, s);
    else
        adv_temp_kernel<false><<<tile_grid(g), tile_block(), 0, st>>>(g, P, s);
}
void launch_diffusion(const Geometry& g, const Phys& P, const State& s, int stepnum, bool last,
                      cudaStream_t st) {
    // passes alternate between the two halves of the diff buffer
    const size_t  plane6 = (size_t)6 * g.nv * g.Np;
    const double* in     = s.diff + ((stepnum + 1) % 2) * plane6;
    double*       out    = s.diff + (stepnum % 2) * plane6;
    const dim3 gr = tile_grid_tail(g), bl = tile_block();
    if (P.mixed)
        P.uniform_thermo ? diffusion_kernel<float, true><<<gr, bl, 0, st>>>(g, P, s, in, out, stepnum, last)
                         : diffusion_kernel<float, false><<<gr, bl, 0, st>>>(g, P, s, in, out, stepnum, last);
    else
        P.uniform_thermo ? diffusion_kernel<double, true><<<gr, bl, 0, st>>>(g, P, s, in, out, stepnum, last)
                         : diffusion_kernel<double, false><<<gr, bl, 0, st>>>(g, P, s, in, out, stepnum, last);
}
void launch_divm0(const Geometry& g, const Phys& P, const State& s, bool small_step,
                  cudaStream_t st) {
    if (P.mixed)
        divm0_kernel<float><<<tile_grid_tail(g), tile_block(), 0, st>>>(g, P, small_step ? s.Mhs : s.Mhk,
                                                        small_step ? s.Whs : s.Whk, s.divg);
    else
        divm0_kernel<double><<<tile_grid_tail(g), tile_block(), 0, st>>>(g, P, small_step ? s.Mhs : s.Mhk,
                                                        small_step ? s.Whs : s.Whk, s.divg);
}
void launch_slow_modes(const Geometry& g, const Phys& P, const State& s, bool update_rk,
                       cudaStream_t st) {
    const dim3 gr = tile_grid_tail(g), bl = tile_block();
    if (P.mixed)
        P.uniform_thermo ? slow_modes_kernel<float, true><<<gr, bl, 0, st>>>(g, P, s, update_rk)
                         : slow_modes_kernel<float, false><<<gr, bl, 0, st>>>(g, P, s, update_rk);
    else
        P.uniform_thermo ? slow_modes_kernel<double, true><<<gr, bl, 0, st>>>(g, P, s, update_rk)
                         : slow_modes_kernel<double, false><<<gr, bl, 0, st>>>(g, P, s, update_rk);
}
size_t vertical_smem_bytes(const Geometry& g) {
    return sizeof(double) * (vertical_ring_offset(g.nv) + (size_t)kThomasRing * 4 * kTile);
}

// The largest dynamic shared memory a kernel has been opened to, per device (the attribute is a
// per-device setting; a process may hold contexts on several devices, and host threads may launch
// concurrently). A size is recorded only once the driver has accepted it; a refusal is returned
// (and stays the runtime's last error, which the caller's error check reports), and the next
// launch asks again.
constexpr int kMaxDevices = 64;
struct SmemOptIn {
    std::mutex mu;
    size_t     bytes[kMaxDevices] = {};
    template<class Kernel>
    cudaError_t ensure(Kernel* kernel, size_t smem) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess)
            dev = -1;
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 0 && dev < kMaxDevices && smem <= bytes[dev])
            return cudaSuccess;
        const cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess && dev >= 0 && dev < kMaxDevices)
            bytes[dev] = smem;
        return e;
    }
};
#if THORX_MOM_TMA
// A 3-D tensor map over planes [planes][nv][Np] of doubles, boxes {kWinW, 8, 1}; false if the
// driver's entry point is missing or the map is rejected (alignment, sizes).
bool window_map(CUtensorMap* map, const double* base, int Np, int nv, int planes) {
    static PFN_cuTensorMapEncodeTiled encode = nullptr;
    static std::mutex                 mu;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!encode) {
            void*                           fn = nullptr;
            cudaDriverEntryPointQueryResult q;
            if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q)
                    != cudaSuccess
                || q != cudaDriverEntryPointSuccess || !fn)
                return false;
            encode = (PFN_cuTensorMapEncodeTiled)fn;
        }
    }
    const cuuint64_t dims[3]    = {(cuuint64_t)Np, (cuuint64_t)nv, (cuuint64_t)planes};
    const cuuint64_t strides[2] = {(cuuint64_t)Np * sizeof(double),
                                   (cuuint64_t)Np * nv * sizeof(double)};
    const cuuint32_t box[3]     = {(cuuint32_t)kWinW, (cuuint32_t)kLevGroups, 1};
    const cuuint32_t estr[3]    = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(base), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
           == CUDA_SUCCESS;
}
#endif

template<class R>
void launch_momentum_t(const Geometry& g, const Phys& P, const State& s, double dt,
                       cudaStream_t st) {
#if THORX_MOM_TMA
    if constexpr (kMomTma<R>) {
        CUtensorMap mps, mdivg;
        if (g.Np >= kWinW && window_map(&mps, s.ps, g.Np, g.nv, 1)
            && window_map(&mdivg, s.divg, g.Np, g.nv, 3)) {
            const size_t     smem = momentum_smem_bytes();
            static SmemOptIn opt;
            if (opt.ensure(momentum_tma_kernel<R>, smem) != cudaSuccess)
                return;
            momentum_tma_kernel<R>
                <<<tile_grid_tail(g), tile_block(), smem, st>>>(g, P, s, dt, mps, mdivg);
            return;
        }
    }
#endif
    momentum_kernel<R><<<tile_grid_tail(g), tile_block(), 0, st>>>(g, P, s, dt);
}
void launch_momentum(const Geometry& g, const Phys& P, const State& s, double dt,
                     cudaStream_t st) {
    if (P.mixed)
        launch_momentum_t<float>(g, P, s, dt, st);
    else
        launch_momentum_t<double>(g, P, s, dt, st);
}
template<int kPart, bool kUni>
void launch_vertical_part_t(const Geometry& g, const Phys& P, const State& s, double dt,
                          cudaStream_t st) {
    const size_t     smem = vertical_smem_bytes(g);
    static SmemOptIn opt;
    if (opt.ensure(vertical_kernel<kPart, kUni>, smem) != cudaSuccess)
        return;
    // the carveout: shared memory for the 3 CTAs an SM holds (register-limited), the rest is L1
    // for the neighbour gathers (a hint; 228 KB is the most shared memory an SM has)
    static bool carve = false;
    if (!carve) {
        const int pct = (int)std::min<size_t>(100, (3 * (smem + 1024) * 100 + 233471) / 233472);
        cudaFuncSetAttribute(vertical_kernel<kPart, kUni>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             pct);
        carve = true;
    }
    vertical_kernel<kPart, kUni><<<tile_grid(g), tile_block(), smem, st>>>(g, P, s, dt);
}
template<int kPart>
void launch_vertical_part(const Geometry& g, const Phys& P, const State& s, double dt,
                          cudaStream_t st) {
    if (P.uniform_thermo)
        launch_vertical_part_t<kPart, true>(g, P, s, dt, st);
    else
        launch_vertical_part_t<kPart, false>(g, P, s, dt, st);
}
void launch_vertical(const Geometry& g, const Phys& P, const State& s, double dt, int part,
                     cudaStream_t st) {
    if (part == 1)
        launch_vertical_part<1>(g, P, s, dt, st);
    else if (part == 2)
        launch_vertical_part<2>(g, P, s, dt, st);
    else
        launch_vertical_part<0>(g, P, s, dt, st);
}

// The check of the Thomas solution that the reference compiles in with
// DIAG_CHECK_THOR_VERTICAL_INT_THOMAS_RESULT (src/headers/dyn/thor_vertical_int.h:486-523): at the
// interior interfaces 2..nv-1, the residual of a w(l-1) + b w(l) + c w(l+1) = d for the rows and
// the solution of the last vertical solve, relative to |d| (absolute where d == 0). Per column the
// largest residual and the number of interfaces above epsilon (1e-8 in the reference).
__global__ void thomas_residual_kernel(Geometry g, State s, double eps, double* colmax,
                                       unsigned int* nbad) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int     Np = g.Np, nv = g.nv, nvi = g.nvi;
    const double* ra = s.vrows;
    const double* rb = ra + (size_t)nvi * Np;
    const double* rc = rb + (size_t)nvi * Np;
    const double* rd = rc + (size_t)nvi * Np;
    double        worst = 0.0;
    unsigned int  bad   = 0;
    for (int lev = 2; lev < nv; lev++) {
        const double dd  = rd[lev * Np + c];
        const double out = ra[lev * Np + c] * s.Whs[(lev - 1) * Np + c]
                           + rb[lev * Np + c] * s.Whs[lev * Np + c]
                           + rc[lev * Np + c] * s.Whs[(lev + 1) * Np + c];
        const double r = dd == 0.0 ? fabs(out - dd) : fabs((out - dd) / dd);
        worst          = fmax(worst, r);
        bad += r > eps ? 1u : 0u;
    }
    colmax[c] = worst;
    if (bad)
        atomicAdd(nbad, bad);
}
void launch_thomas_residual(const Geometry& g, const State& s, double eps, double* colmax,
                            unsigned int* nbad, cudaStream_t st) {
    thomas_residual_kernel<<<(g.N + 127) / 128, 128, 0, st>>>(g, s, eps, colmax, nbad);
}

// Registered module arrays (device_RK_array_manager, src/ESP/phy_modules_device.cu:47-77): the
// deviation reset of UpdateRK, array = arrayi - arrayk (src/headers/dyn/thor_auxiliary.h:376-387),
// and the accumulation of UpdateRK2, arrayk += array (:483-494), elementwise.
__global__ void rk_arrays_kernel(RkArrays t, int mode) {
    const int       a = blockIdx.y;
    const long long n = t.count[a];
    double*         x = t.array[a];
    double*         k = t.arrayk[a];
    const double*   i = t.arrayi[a];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        if (mode == 0)
            x[e] = i[e] - k[e];
        else
            k[e] += x[e];
    }
}
void launch_rk_arrays(const RkArrays& t, int mode, cudaStream_t st) {
    if (t.n > 0)
        rk_arrays_kernel<<<dim3(148 * 4, t.n), 256, 0, st>>>(t, mode);
}
void launch_vertical_diff(const Geometry& g, const Phys& P, const State& s, cudaStream_t st) {
    const size_t  smem       = sizeof(double) * kVdCols * (2 * g.nv + 2);
    static SmemOptIn opt;
    if (opt.ensure(vertical_diff_kernel, smem) != cudaSuccess)
        return;
    static_assert(kVdCols == kTile, "vertical hyperdiffusion blocks are tiles");
    vertical_diff_kernel<<<g.ntile, kVdCols, smem, st>>>(g, P, s);
}
void launch_update_rk2(const Geometry& g, const Phys& P, const State& s, cudaStream_t st) {
    update_rk2_kernel<<<tile_grid(g), dim3(kTile, kRk2Groups), 0, st>>>(g, P, s);
}
void launch_div_check(long long n, unsigned long long seed, unsigned long long* cnt,
                      cudaStream_t st) {
    div_check_kernel<<<148 * 8, 256, 0, st>>>(n, seed, cnt);
}

} // namespace thorx

#if THORX_VERT_CLOCK
extern "C" int thorx_debug_vclock(unsigned long long* host, int n) {
    return (int)cudaMemcpyFromSymbol(host, thorx::g_vclock, sizeof(unsigned long long) * n);
}
#endif
