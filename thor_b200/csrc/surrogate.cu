// RT surrogate: a per-column MLP that maps (T, log p per level, cos zenith) to the heating rates
// of the double-gray RT as temperature tendencies dT/dt = Q / (rho c_v) in K/s, trained on the
// GPU from columns the plain RT produced, run inside the physics step with the plain RT
// re-checking a rotating 1/period of the columns and taking over wherever the surrogate's
// relative error exceeds a tolerance. No counterpart in the reference.
//
// Network: in = 2 nv + 1 features -> H -> H -> H -> nv, GELU after the hidden layers, BF16
// weights and activations, FP32 accumulation (the tcgen05 GEMM of umma.cuh), FP32 master weights
// with Adam. Every dimension is padded to the GEMM tile rules (batch to 128, in to a multiple of
// 64, out to 64); padded weights, biases and their gradients are exactly zero and stay zero.
// Features and targets are standardised per feature / per level with statistics of the logged
// training data.
//
// Device layouts: batch-major, row = one column of the grid (or one training sample):
//   X0 [B][Kin] bf16, Z_l [B][H] f32 (pre-activations), A_l [B][H] bf16, Y [B][Nout] f32.
// Layer l: W [N][K] (f32 master, bf16 copy for the forward GEMM, bf16 transpose [K][N] for the
// input-gradient GEMM), b [N].
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/thorx.h"
#include "surrogate.h"
#include "thorx_internal.h"
#include "umma.cuh"

namespace thorx {
namespace {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint64_t mix64(uint64_t z) { // SplitMix64 finaliser
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t i) {
    return (double)(mix64(seed + 0x9E3779B97F4A7C15ull * (i + 1)) >> 11) * (1.0 / 9007199254740992.0);
}

// ---- parameters -----------------------------------------------------------------------------
// W ~ U(-a, a), a = sqrt(6 / (fan_in + fan_out)) on the valid block, zero elsewhere; b = 0.
__global__ void init_layer_kernel(float* W, float* b, int N, int K, int n_valid, int k_valid,
                                  uint64_t seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N * K) {
        const int    n = i / K, k = i % K;
        const double a = sqrt(6.0 / (double)(n_valid + k_valid));
        W[i] = (n < n_valid && k < k_valid) ? (float)((2.0 * uniform01(seed, i) - 1.0) * a) : 0.0f;
    }
    if (i < N)
        b[i] = 0.0f;
}

// bf16 copies of a layer: Wbf [N][K] and its transpose Wt [K][N].
__global__ void cast_layer_kernel(const float* W, bf16* Wbf, bf16* Wt, int N, int K) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * K)
        return;
    const int  n = i / K, k = i % K;
    const bf16 v = __float2bfloat16_rn(W[i]);
    Wbf[i]       = v;
    Wt[(size_t)k * N + n] = v;
}

// Adam (Kingma & Ba 2015) on one tensor, bias-corrected with step t (c1 = 1 - b1^t, c2 = 1 - b2^t).
__global__ void adam_kernel(float* w, float* m, float* v, const float* g, int n, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i]           = mi;
    v[i]           = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ---- batch assembly -------------------------------------------------------------------------
// Standardised bf16 features of the grid columns at the physics step: T, log p per level, and
// cos zenith; rows >= N and features >= n_in are zero.
// Standardised bf16 features of the columns in the step (rows >= N: zero), 32 columns per block:
// the warps compute with lanes across columns (coalesced level planes) into a shared tile, then
// write each column's row of Kin features contiguously.
constexpr int kFeatCols = 32, kFeatWarps = 8;
__global__ void __launch_bounds__(kFeatCols* kFeatWarps)
    features_state_kernel(SurNet net, Geometry g, State s, const double* cos_zenith, bf16* X0,
                          int Brows) {
    extern __shared__ bf16 tile[]; // [32][Kin + 2]: an odd number of 4-byte words per row
    const int pitch = net.Kin + 2;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int r0 = blockIdx.x * kFeatCols, r = r0 + lane;
    const int nv = net.nv;
    for (int j = w; j < net.Kin; j += kFeatWarps) {
        float x = 0.0f;
        if (r < g.N && j < net.n_in) {
            double raw;
            if (j < nv)
                raw = s.T[(size_t)j * g.Np + r];
            else if (j < 2 * nv)
                raw = log(s.p[(size_t)(j - nv) * g.Np + r]);
            else
                raw = cos_zenith[r];
            x = (float)((raw - net.in_mean[j]) / net.in_std[j]);
        }
        tile[lane * pitch + j] = __float2bfloat16_rn(x);
    }
    __syncthreads();
    for (int rr = w; rr < kFeatCols; rr += kFeatWarps) {
        if (r0 + rr >= Brows)
            break;
        bf16* dst = X0 + (size_t)(r0 + rr) * net.Kin;
        for (int j = 2 * lane; j < net.Kin; j += 64)
            *reinterpret_cast<__nv_bfloat162*>(dst + j) =
                __halves2bfloat162(tile[rr * pitch + j], tile[rr * pitch + j + 1]);
    }
}

// Random training batch from the log: standardised bf16 features and f32 targets.
__global__ void features_log_kernel(SurNet net, SurLog lg, long long nlogged, uint64_t seed,
                                    bf16* X0, float* tgt, int B) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B)
        return;
    const long long row = (long long)(uniform01(seed, r) * (double)nlogged) % nlogged;
    const float*    x   = lg.X + (size_t)row * net.n_in;
    const float*    y   = lg.Y + (size_t)row * net.nv;
    for (int j = 0; j < net.Kin; j++) {
        const float v = j < net.n_in ? (float)((x[j] - net.in_mean[j]) / net.in_std[j]) : 0.0f;
        X0[(size_t)r * net.Kin + j] = __float2bfloat16_rn(v);
    }
    for (int j = 0; j < net.Nout; j++)
        tgt[(size_t)r * net.Nout + j] =
            j < net.nv ? (float)((y[j] - net.out_mean[j]) / net.out_std[j]) : 0.0f;
}

// Features and targets given on the host (tests), already standardised.
__global__ void features_host_kernel(SurNet net, const float* x, const float* t, int B, bf16* X0,
                                     float* tgt) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= B)
        return;
    for (int j = 0; j < net.Kin; j++)
        X0[(size_t)r * net.Kin + j] =
            __float2bfloat16_rn(j < net.n_in ? x[(size_t)r * net.n_in + j] : 0.0f);
    if (t)
        for (int j = 0; j < net.Nout; j++)
            tgt[(size_t)r * net.Nout + j] = j < net.nv ? t[(size_t)r * net.nv + j] : 0.0f;
}

// MSE loss over the valid outputs of the first B rows: dY = 2 (Y - T) / (B nv) as f32 and bf16,
// per-block partial losses into part[blockIdx.x] (summed in a fixed order on the host).
__global__ void loss_grad_kernel(SurNet net, const float* Y, const float* tgt, int B, float* dYf,
                                 bf16* dY, double* part) {
    __shared__ double sh[256];
    const int         i     = blockIdx.x * blockDim.x + threadIdx.x;
    const int         total = B * net.Nout;
    double            l     = 0.0;
    if (i < total) {
        const int   j  = i % net.Nout;
        const float d  = (j < net.nv) ? Y[i] - tgt[i] : 0.0f;
        const float gd = 2.0f * d / (float)(B * net.nv);
        dYf[i]         = gd;
        dY[i]          = __float2bfloat16_rn(gd);
        l              = (double)d * d;
    }
    sh[threadIdx.x] = l;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            sh[threadIdx.x] += sh[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        part[blockIdx.x] = sh[0];
}

// Column sums of G [B][N] (bias gradients) in two passes with a fixed order: block (32 columns
// x 8 row lanes) of row chunk blockIdx.y writes part[blockIdx.y][n]; colsum_final adds the chunks.
constexpr int kColsumChunks = 64;
template<class T> __global__ void colsum_kernel(const T* G, int B, int N, float* part) {
    __shared__ float sh[8][33];
    const int        n = blockIdx.x * 32 + threadIdx.x;
    const int        rows = (B + kColsumChunks - 1) / kColsumChunks;
    const int        r0 = blockIdx.y * rows, r1 = min(B, r0 + rows);
    float            acc = 0.0f;
    if (n < N)
        for (int r = r0 + threadIdx.y; r < r1; r += 8)
            acc += (float)G[(size_t)r * N + n];
    sh[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && n < N) {
        float t = 0.0f;
        for (int y = 0; y < 8; y++)
            t += sh[y][threadIdx.x];
        part[(size_t)blockIdx.y * N + n] = t;
    }
}
__global__ void colsum_final_kernel(const float* part, int N, float* db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N)
        return;
    float t = 0.0f;
    for (int z = 0; z < kColsumChunks; z++)
        t += part[(size_t)z * N + n];
    db[n] = t;
}

// out[i] = sum over z of part[z * stride + i] (split-K partial products), z in order.
__global__ void splitk_reduce_kernel(const float* part, int splits, size_t stride, size_t n,
                                     float* out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    float t = 0.0f;
    for (int z = 0; z < splits; z++)
        t += part[(size_t)z * stride + i];
    out[i] = t;
}

// dst [C][ldd] = src [R][C]^T for bf16, 32 x 32 tiles through shared memory (R, C multiples of
// 32); columns R..ldd-1 of the destination are left as they are.
__global__ void transpose_bf16_kernel(const bf16* src, bf16* dst, int R, int C, int ldd) {
    __shared__ bf16 t[32][33];
    const int       r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        t[y][threadIdx.x] = src[(size_t)(r0 + y) * C + c0 + threadIdx.x];
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y)
        dst[(size_t)(c0 + y) * ldd + r0 + threadIdx.x] = t[threadIdx.x][y];
}

// ---- the physics step in surrogate mode -----------------------------------------------------
// Per column: the surrogate's heating (de-standardised), or the plain RT's where the column was
// re-checked this step or has fallen back; a re-checked column falls back (or returns to the
// surrogate) according to its relative error max|Qs - Qrt| / max|Qrt|. Then the cooling limiter
// and the coupling into profx_Qheat as the plain RT does (profx_RT.h:560-584).
// 32 columns per block (lane = column) x kCombGroups warps over the levels (warp y: levels y,
// y + kCombGroups, ...); the re-check's column maxima are reduced over the warps in shared memory.
constexpr int kCombGroups = 8;
__global__ void __launch_bounds__(32 * kCombGroups)
    combine_kernel(SurNet net, Geometry g, Phys P, State s, RtFields f, const float* Yt, int ldy,
                   uint8_t* fallback, int period, double tol, unsigned int* stats) {
    __shared__ double snum[kCombGroups][32], sden[kCombGroups][32];
    __shared__ int    s_use[32];
    const int    lane = threadIdx.x & 31, y = threadIdx.x >> 5;
    const int    id = blockIdx.x * 32 + lane;
    const RtStep st = *f.step;
    if (!st.run) // uniform: the RT does not run this step
        return;
    const bool valid   = id < g.N;
    const int  nv = g.nv, Np = g.Np;
    const bool recheck = valid && recheck_column(id, period, st.cur);
    // heating rates compared as temperature tendencies (K/s): the thin upper layers, whose
    // W/m^3 are small, weigh as much as their temperature change does
    auto rho_cv = [&](int lev) {
        const size_t i = (size_t)lev * Np + id;
        return s.Rho[i] * (s.Cp[i] - s.Rd[i]);
    };
    auto sur = [&](int lev) { // the network's heating rate at this level, K/s
        return (double)Yt[(size_t)lev * ldy + id] * net.out_std[lev] + net.out_mean[lev];
    };
    double num = 0.0, den = 0.0;
    if (recheck)
        for (int lev = y; lev < nv; lev += kCombGroups) {
            const double qr = f.dtemp[(size_t)lev * Np + id] / rho_cv(lev);
            num             = fmax(num, fabs(sur(lev) - qr));
            den             = fmax(den, fabs(qr));
        }
    snum[y][lane] = num;
    sden[y][lane] = den;
    __syncthreads();
    if (y == 0) {
        unsigned int err_e6 = 0;
        bool         failed = false;
        if (recheck) {
            for (int k = 1; k < kCombGroups; k++) {
                num = fmax(num, snum[k][lane]);
                den = fmax(den, sden[k][lane]);
            }
            const double err = den > 0.0 ? num / den : (num > 0.0 ? 1.0e300 : 0.0);
            failed           = err > tol;
            fallback[id]     = failed ? 1 : 0;
            err_e6           = (unsigned)fmin(err * 1e6, 4.0e9);
        }
        const bool use_rt = valid && (fallback[id] != 0 || recheck);
        s_use[lane]       = use_rt;
        // statistics, one atomic per block: re-checked, failed, largest error (1e-6), plain RT
        const unsigned n_re = __popc(__ballot_sync(0xffffffffu, recheck));
        const unsigned n_fa = __popc(__ballot_sync(0xffffffffu, failed));
        const unsigned n_rt = __popc(__ballot_sync(0xffffffffu, use_rt));
        const unsigned mx   = __reduce_max_sync(0xffffffffu, err_e6);
        if (lane == 0) {
            if (n_re)
                atomicAdd(&stats[0], n_re);
            if (n_fa)
                atomicAdd(&stats[1], n_fa);
            if (n_re)
                atomicMax(&stats[2], mx);
            if (n_rt)
                atomicAdd(&stats[3], n_rt);
        }
    }
    __syncthreads();
    if (!valid)
        return;
    const bool use_rt = s_use[lane] != 0;
    for (int lev = y; lev < nv; lev += kCombGroups) {
        const int i = lev * Np + id;
        double    d = use_rt ? f.dtemp[i] : sur(lev) * rho_cv(lev);
        if (s.p[i] + s.Rd[i] / (s.Cp[i] - s.Rd[i]) * d * P.timestep < 0)
            d = -s.p[i] / P.timestep;
        f.dtemp[i] = d;
        f.qheat[i] = d;
        s.Qheat[i] += st.Qheat_scaling * d;
    }
}

// ---- logging of plain-RT columns for training -----------------------------------------------
__global__ void log_reserve_kernel(SurLog lg, const RtStep* st, int N) {
    if (!st->run) {
        *lg.base = -1;
        return;
    }
    *lg.base = *lg.count;
    *lg.count += N;
}

__global__ void log_write_kernel(SurLog lg, SurNet net, Geometry g, State s, RtFields f) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= g.N)
        return;
    const long long base = *lg.base;
    if (base < 0)
        return;
    const long long row = (base + id) % lg.cap;
    float*          x   = lg.X + (size_t)row * net.n_in;
    float*          y   = lg.Y + (size_t)row * net.nv;
    for (int lev = 0; lev < net.nv; lev++) {
        const size_t i  = (size_t)lev * g.Np + id;
        x[lev]          = (float)s.T[i];
        x[net.nv + lev] = (float)log(s.p[i]);
        y[lev]          = (float)(f.dtemp[i] / (s.Rho[i] * (s.Cp[i] - s.Rd[i]))); // K/s
    }
    x[2 * net.nv] = (float)f.cos_zenith[id];
}

// Online logging in surrogate mode: each column the plain RT ran on this step (fallen back, or
// re-checked: the predicate of rt_column_kernel) takes the next row of the ring, with its raw
// heating rate (before the combine's limiter, as the RT computed it).
__global__ void log_used_kernel(SurLog lg, SurNet net, Geometry g, State s, RtFields f) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= g.N)
        return;
    const RtStep st = *f.step;
    if (!st.run || !(f.fallback[id] || recheck_column(id, f.period, st.cur)))
        return;
    const long long n   = (long long)atomicAdd((unsigned long long*)lg.count, 1ull);
    const long long row = n % lg.cap;
    float*          x   = lg.X + (size_t)row * net.n_in;
    float*          y   = lg.Y + (size_t)row * net.nv;
    for (int lev = 0; lev < net.nv; lev++) {
        const size_t i  = (size_t)lev * g.Np + id;
        x[lev]          = (float)s.T[i];
        x[net.nv + lev] = (float)log(s.p[i]);
        y[lev]          = (float)(f.dtemp[i] / (s.Rho[i] * (s.Cp[i] - s.Rd[i]))); // K/s
    }
    x[2 * net.nv] = (float)f.cos_zenith[id];
}

// Mean and standard deviation of column j of a [rows][ld] f32 table (one block per column).
__global__ void stats_kernel(const float* X, long long rows, int ld, float* mean, float* stdv) {
    __shared__ double s1[256], s2[256];
    const int         j = blockIdx.x;
    double            a = 0.0, b = 0.0;
    for (long long r = threadIdx.x; r < rows; r += blockDim.x) {
        const double v = X[(size_t)r * ld + j];
        a += v;
        b += v * v;
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) {
            s1[threadIdx.x] += s1[threadIdx.x + st];
            s2[threadIdx.x] += s2[threadIdx.x + st];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double m  = s1[0] / (double)rows;
        const double sd = sqrt(fmax(s2[0] / (double)rows - m * m, 0.0));
        mean[j]         = (float)m;
        stdv[j]         = (float)(sd > 0.0 ? sd : 1.0);
    }
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

} // namespace

// ---- host side --------------------------------------------------------------------------------
int Surrogate::init(int nv_, int hidden, long long log_capacity, int batch_rows, int ncols,
                    uint64_t seed_) {
    net.nv   = nv_;
    net.n_in = 2 * nv_ + 1;
    net.Kin  = ((net.n_in + 63) / 64) * 64;
    net.H    = hidden;
    net.Nout = ((nv_ + 63) / 64) * 64;
    seed     = seed_;
    Bcap     = ((batch_rows + 127) / 128) * 128;
    const int Ns[4] = {net.H, net.H, net.H, net.Nout}, Ks[4] = {net.Kin, net.H, net.H, net.H};
    const int nvalid[4] = {net.H, net.H, net.H, net.nv}, kvalid[4] = {net.n_in, net.H, net.H, net.H};
    size_t    bytes = 0;
    auto      alloc = [&](void** p, size_t n) -> bool {
        if (cudaMalloc(p, n) != cudaSuccess)
            return false;
        allocs.push_back(*p);
        bytes += n;
        return cudaMemset(*p, 0, n) == cudaSuccess;
    };
    for (int l = 0; l < 4; l++) {
        SurLayer& L = lay[l];
        L.N         = Ns[l];
        L.K         = Ks[l];
        const size_t nw = (size_t)L.N * L.K;
        // the weight-gradient GEMM's M is the layer's N, padded to 128 rows
        const size_t ng = (size_t)std::max(L.N, 128) * L.K;
        if (!alloc((void**)&L.W, nw * 4) || !alloc((void**)&L.b, L.N * 4)
            || !alloc((void**)&L.mW, nw * 4) || !alloc((void**)&L.vW, nw * 4)
            || !alloc((void**)&L.mb, L.N * 4) || !alloc((void**)&L.vb, L.N * 4)
            || !alloc((void**)&L.gW, ng * 4) || !alloc((void**)&L.gb, L.N * 4)
            || !alloc((void**)&L.Wbf, nw * 2) || !alloc((void**)&L.Wt, nw * 2))
            return THORX_E_CUDA;
        init_layer_kernel<<<nblk(nw, 256), 256>>>(L.W, L.b, L.N, L.K, nvalid[l], kvalid[l],
                                                 seed + 7919ull * (l + 1));
    }
    if (!alloc((void**)&net.in_mean, net.Kin * 4) || !alloc((void**)&net.in_std, net.Kin * 4)
        || !alloc((void**)&net.out_mean, net.Nout * 4) || !alloc((void**)&net.out_std, net.Nout * 4))
        return THORX_E_CUDA;
    {
        std::vector<float> one(std::max(net.Kin, net.Nout), 1.0f);
        cudaMemcpy(net.in_std, one.data(), net.Kin * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(net.out_std, one.data(), net.Nout * 4, cudaMemcpyHostToDevice);
    }
    const size_t B = Bcap;
    if (!alloc((void**)&X0, B * net.Kin * 2) || !alloc((void**)&Y, B * net.Nout * 4)
        || !alloc((void**)&Yt, B * net.Nout * 4)
        || !alloc((void**)&tgt, B * net.Nout * 4) || !alloc((void**)&dYf, B * net.Nout * 4)
        || !alloc((void**)&dY, B * net.Nout * 2) || !alloc((void**)&dZ[0], B * net.H * 2)
        || !alloc((void**)&dZ[1], B * net.H * 2)
        || !alloc((void**)&T1, (size_t)std::max(net.H, 128) * B * 2)
        || !alloc((void**)&T2, (size_t)std::max(net.H, net.Kin) * B * 2)
        || !alloc((void**)&lpart, nblk(B * net.Nout, 256) * 8) || !alloc((void**)&err, 4)
        || !alloc((void**)&splitk, (size_t)kMaxSplits * std::max(net.H, 128)
                                       * std::max(net.H, net.Kin) * 4)
        || !alloc((void**)&colpart, (size_t)kColsumChunks * std::max(net.H, net.Nout) * 4)
        || !alloc((void**)&stats, 16))
        return THORX_E_CUDA;
    for (int l = 0; l < 3; l++)
        if (!alloc((void**)&Gd[l], B * net.H * 2) || !alloc((void**)&A[l], B * net.H * 2))
            return THORX_E_CUDA;
    log.cap = log_capacity;
    if (log_capacity > 0)
        if (!alloc((void**)&log.X, (size_t)log_capacity * net.n_in * 4)
            || !alloc((void**)&log.Y, (size_t)log_capacity * net.nv * 4))
            return THORX_E_CUDA;
    if (!alloc((void**)&log.count, 8) || !alloc((void**)&log.base, 8)
        || !alloc((void**)&fallback, (size_t)ncols))
        return THORX_E_CUDA;
    device_bytes = bytes;
    cast_all(0);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : THORX_E_CUDA;
}

void Surrogate::release() {
    for (void* p : allocs)
        cudaFree(p);
    allocs.clear();
}

void Surrogate::cast_all(cudaStream_t st) {
    for (int l = 0; l < 4; l++) {
        SurLayer& L = lay[l];
        cast_layer_kernel<<<nblk((long long)L.N * L.K, 256), 256, 0, st>>>(L.W, L.Wbf, L.Wt, L.N, L.K);
    }
}

// Y = net(X0) for the first B rows (B a multiple of 128). keep_z (training, tests): the GELU
// derivatives the backward pass needs (bf16) and Y row by row; otherwise (inference in the step)
// neither, and the output transposed into Yt.
void Surrogate::forward(int B, cudaStream_t st, bool keep_z) {
    for (int l = 0; l < 3; l++) {
        const bf16*   in = l == 0 ? X0 : A[l - 1];
        umma::EpiArgs e{nullptr, A[l], keep_z ? Gd[l] : nullptr, nullptr, lay[l].b, net.H};
        umma::gemm_tma<256, umma::kEpiBiasGelu>(in, lay[l].Wbf, B, net.H, lay[l].K, e, err, st);
    }
    if (keep_z) {
        umma::EpiArgs e{Y, nullptr, nullptr, nullptr, lay[3].b, net.Nout};
        umma::gemm_tma<64, umma::kEpiBiasF32>(A[2], lay[3].Wbf, B, net.Nout, net.H, e, err, st);
    }
    else { // inference: the output plane by plane (Yt [Nout][Bcap]) for the per-level combine
        umma::EpiArgs e{Yt, nullptr, nullptr, nullptr, lay[3].b, Bcap};
        umma::gemm_tma<64, umma::kEpiBiasF32T>(A[2], lay[3].Wbf, B, net.Nout, net.H, e, err, st);
    }
}

// D[M x N] = A[M x K] . B[N x K]^T into f32, tile width chosen from N.
void Surrogate::gemm_n(const bf16* Am, const bf16* Bm, int M, int N, int K, const umma::EpiArgs& e,
                       cudaStream_t st) {
    if (N % 256 == 0)
        umma::gemm_tma<256, umma::kEpiF32>(Am, Bm, M, N, K, e, err, st);
    else if (N % 128 == 0)
        umma::gemm_tma<128, umma::kEpiF32>(Am, Bm, M, N, K, e, err, st);
    else
        umma::gemm_tma<64, umma::kEpiF32>(Am, Bm, M, N, K, e, err, st);
}
// Weight gradient D[M x N] = A[M x K] . B[N x K]^T with K = the batch, split over CTAs in
// partial products (so that the few 128 x N tiles of a layer fill the GPU) and reduced in order.
void Surrogate::gemm_wgrad(const bf16* Am, const bf16* Bm, int M, int N, int K, float* out,
                           cudaStream_t st) {
    int splits = 1;
    while (splits < kMaxSplits && K % (2 * splits * umma::kKChunk) == 0
           && K / (2 * splits) >= 2 * umma::kKChunk)
        splits *= 2;
    const size_t  stride = (size_t)M * N;
    umma::EpiArgs e{splitk, nullptr, nullptr, nullptr, nullptr, N, stride};
    if (N % 256 == 0)
        umma::gemm_tma<256, umma::kEpiF32>(Am, Bm, M, N, K, e, err, st, splits);
    else if (N % 128 == 0)
        umma::gemm_tma<128, umma::kEpiF32>(Am, Bm, M, N, K, e, err, st, splits);
    else
        umma::gemm_tma<64, umma::kEpiF32>(Am, Bm, M, N, K, e, err, st, splits);
    splitk_reduce_kernel<<<nblk((long long)stride, 256), 256, 0, st>>>(splitk, splits, stride,
                                                                      stride, out);
}

void Surrogate::colsum(const float* G, int B, int N, float* db, cudaStream_t st) {
    colsum_kernel<float><<<dim3(nblk(N, 32), kColsumChunks), dim3(32, 8), 0, st>>>(G, B, N, colpart);
    colsum_final_kernel<<<nblk(N, 128), 128, 0, st>>>(colpart, N, db);
}
void Surrogate::colsum(const bf16* G, int B, int N, float* db, cudaStream_t st) {
    colsum_kernel<bf16><<<dim3(nblk(N, 32), kColsumChunks), dim3(32, 8), 0, st>>>(G, B, N, colpart);
    colsum_final_kernel<<<nblk(N, 128), 128, 0, st>>>(colpart, N, db);
}

void Surrogate::gemm_gelu_bwd(const bf16* Am, const bf16* Bm, int M, int N, int K,
                              const umma::EpiArgs& e, cudaStream_t st) {
    umma::gemm_tma<256, umma::kEpiGeluBwdBf16>(Am, Bm, M, N, K, e, err, st);
}

// Gradients of the MSE loss for the first B rows (targets in tgt): fills gW, gb of every layer.
void Surrogate::backward(int B, cudaStream_t st) {
    const int H = net.H, Nout = net.Nout;
    lpart_n     = nblk((long long)B * Nout, 256);
    loss_grad_kernel<<<lpart_n, 256, 0, st>>>(net, Y, tgt, B, dYf, dY, lpart);
    // output layer: gW4 = dY^T A3, gb4 = colsum dY, dZ3 = (dY W4) * gelu'(Z3) (stored in bf16)
    colsum(dYf, B, Nout, lay[3].gb, st);
    cudaMemsetAsync(T1, 0, (size_t)128 * B * 2, st); // dY^T padded to 128 rows
    transpose_bf16_kernel<<<dim3(Nout / 32, B / 32), dim3(32, 8), 0, st>>>(dY, T1, B, Nout, B);
    transpose_bf16_kernel<<<dim3(H / 32, B / 32), dim3(32, 8), 0, st>>>(A[2], T2, B, H, B);
    {
        gemm_wgrad(T1, T2, 128, H, B, lay[3].gW, st);
    }
    {
        umma::EpiArgs e{nullptr, dZ[0], nullptr, Gd[2], nullptr, H};
        gemm_gelu_bwd(dY, lay[3].Wt, B, H, Nout, e, st);
    }
    // hidden layers 3, 2, 1 (indices 2, 1, 0)
    int cur = 0;
    for (int l = 2; l >= 0; l--) {
        const bf16* dz = dZ[cur];
        colsum(dz, B, H, lay[l].gb, st);
        transpose_bf16_kernel<<<dim3(H / 32, B / 32), dim3(32, 8), 0, st>>>(dz, T1, B, H, B);
        const bf16* in  = l == 0 ? X0 : A[l - 1];
        const int   Kin = lay[l].K;
        transpose_bf16_kernel<<<dim3(Kin / 32, B / 32), dim3(32, 8), 0, st>>>(in, T2, B, Kin, B);
        {
            gemm_wgrad(T1, T2, H, Kin, B, lay[l].gW, st);
        }
        if (l > 0) {
            umma::EpiArgs e{nullptr, dZ[cur ^ 1], nullptr, Gd[l - 1], nullptr, H};
            gemm_gelu_bwd(dz, lay[l].Wt, B, H, H, e, st);
            cur ^= 1;
        }
    }
}

void Surrogate::adam(float lr, cudaStream_t st) {
    adam_t++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.0f - powf(b1, (float)adam_t), c2 = 1.0f - powf(b2, (float)adam_t);
    for (int l = 0; l < 4; l++) {
        SurLayer& L  = lay[l];
        const int nw = L.N * L.K;
        adam_kernel<<<nblk(nw, 256), 256, 0, st>>>(L.W, L.mW, L.vW, L.gW, nw, lr, b1, b2, eps, c1, c2);
        adam_kernel<<<nblk(L.N, 256), 256, 0, st>>>(L.b, L.mb, L.vb, L.gb, L.N, lr, b1, b2, eps, c1, c2);
    }
    cast_all(st);
}

void Surrogate::fit_normalisation(long long rows, cudaStream_t st) {
    stats_kernel<<<net.n_in, 256, 0, st>>>(log.X, rows, net.n_in, net.in_mean, net.in_std);
    stats_kernel<<<net.nv, 256, 0, st>>>(log.Y, rows, net.nv, net.out_mean, net.out_std);
}

void Surrogate::train_batch(long long nlogged, int B, float lr, cudaStream_t st) {
    features_log_kernel<<<nblk(B, 128), 128, 0, st>>>(
        net, log, nlogged, seed ^ (0xD1B54A32D192ED03ull * (uint64_t)(adam_t + 1)), X0, tgt, B);
    forward(B, st);
    backward(B, st);
    adam(lr, st);
}

void Surrogate::load_host_batch(const float* dx, const float* dt, int B, cudaStream_t st) {
    cudaMemsetAsync(X0, 0, (size_t)Bcap * net.Kin * 2, st);
    cudaMemsetAsync(tgt, 0, (size_t)Bcap * net.Nout * 4, st);
    features_host_kernel<<<nblk(B, 128), 128, 0, st>>>(net, dx, dt, B, X0, tgt);
}

void Surrogate::step_features(const Geometry& g, const State& s, const RtFields& f, cudaStream_t st) {
    const int B = ((g.N + 127) / 128) * 128;
    features_state_kernel<<<B / kFeatCols, kFeatCols * kFeatWarps,
                            (size_t)kFeatCols * (net.Kin + 2) * sizeof(bf16), st>>>(
        net, g, s, f.cos_zenith, X0, B);
    forward(B, st, false);
}

void Surrogate::step_combine(const Geometry& g, const Phys& P, const State& s, const RtFields& f,
                             cudaStream_t st) {
    combine_kernel<<<(g.N + 31) / 32, 32 * kCombGroups, 0, st>>>(net, g, P, s, f, Yt, Bcap, fallback,
                                                                 period, tol, stats);
}

void Surrogate::log_used(const Geometry& g, const State& s, const RtFields& f, cudaStream_t st) {
    log_used_kernel<<<nblk(g.N, 128), 128, 0, st>>>(log, net, g, s, f);
}

void Surrogate::log_step(const Geometry& g, const State& s, const RtFields& f, cudaStream_t st) {
    log_reserve_kernel<<<1, 1, 0, st>>>(log, f.step, g.N);
    log_write_kernel<<<nblk(g.N, 128), 128, 0, st>>>(log, net, g, s, f);
}

} // namespace thorx

// ---- context-free entry points -----------------------------------------------------------------
namespace {
thread_local std::string g_sur_err;
int                      sur_fail(int code, const std::string& m) {
    g_sur_err = m;
    return code;
}
} // namespace

extern "C" {

const char* thorx_surrogate_last_error(void) { return g_sur_err.c_str(); }

int thorx_bf16_gemm(const unsigned short* A, const unsigned short* B, int M, int N, int K, float* D) {
    using namespace thorx;
    if (!A || !B || !D || M <= 0 || N <= 0 || K <= 0)
        return sur_fail(THORX_E_ARG, "thorx_bf16_gemm: null pointer or non-positive size");
    if (M % umma::kM || K % umma::kKChunk || N % 64)
        return sur_fail(THORX_E_ARG, "thorx_bf16_gemm: M must be a multiple of 128, N of 64, K of 64");
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float*         dD  = nullptr;
    unsigned int*  err = nullptr;
    cudaError_t    e   = cudaSuccess;
    auto           ck  = [&](cudaError_t x) {
        if (e == cudaSuccess)
            e = x;
    };
    ck(cudaMalloc(&dA, (size_t)M * K * 2));
    ck(cudaMalloc(&dB, (size_t)N * K * 2));
    ck(cudaMalloc(&dD, (size_t)M * N * 4));
    ck(cudaMalloc(&err, sizeof(unsigned int)));
    if (e == cudaSuccess) {
        ck(cudaMemcpy(dA, A, (size_t)M * K * 2, cudaMemcpyHostToDevice));
        ck(cudaMemcpy(dB, B, (size_t)N * K * 2, cudaMemcpyHostToDevice));
        ck(cudaMemset(err, 0, sizeof(unsigned int)));
    }
    if (e == cudaSuccess) {
        umma::EpiArgs ea{dD, nullptr, nullptr, nullptr, nullptr, N};
        if (N % 256 == 0)
            umma::gemm_tma<256, umma::kEpiF32>(dA, dB, M, N, K, ea, err, 0);
        else if (N % 128 == 0)
            umma::gemm_tma<128, umma::kEpiF32>(dA, dB, M, N, K, ea, err, 0);
        else
            umma::gemm_tma<64, umma::kEpiF32>(dA, dB, M, N, K, ea, err, 0);
        ck(cudaGetLastError());
        ck(cudaDeviceSynchronize());
    }
    unsigned int herr = 0;
    if (e == cudaSuccess) {
        ck(cudaMemcpy(D, dD, (size_t)M * N * 4, cudaMemcpyDeviceToHost));
        ck(cudaMemcpy(&herr, err, sizeof(herr), cudaMemcpyDeviceToHost));
    }
    cudaFree(dA), cudaFree(dB), cudaFree(dD), cudaFree(err);
    if (e != cudaSuccess)
        return sur_fail(THORX_E_CUDA, std::string("thorx_bf16_gemm: ") + cudaGetErrorString(e));
    if (herr)
        return sur_fail(THORX_E_CUDA, "thorx_bf16_gemm: tensor-core wait timed out");
    return 0;
}

} // extern "C"
