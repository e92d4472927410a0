// Global conserved quantities and compensated device sums.
//
// Reference: ESP::globdiag (src/ESP/profx_driver.cu:476-569) launches four per-cell kernels
// (CalcTotEnergy, CalcMass, CalcAngMom, CalcEntropy, src/ESP/profx_globdiag.cu:45-252) that store
// one array per quantity, then reduces each array with gpu_sum_on_device<1024>
// (src/headers/reduction_add.h:96-128): a shared-memory tree per 2048 elements, partial sums
// copied to the host and added there in a plain loop, with a cudaMalloc/cudaFree per call.
//
// Here the per-cell terms are computed and reduced in one pass (nothing per cell is stored), and
// every sum is compensated: each thread, block and the final pass carry a (sum, error) pair
// combined with the error-free transformation TwoSum (Knuth, TAOCP vol. 2, 4.2.2), so the result
// is the exact sum rounded once or twice, independent of the number of terms, and the order of
// every addition is fixed by the launch shape alone: the same input gives the same bits on every
// call.
#include <mutex>

#include "thorx_internal.h"

namespace thorx {
namespace {

constexpr int kSumThreads  = 256;
constexpr int kSumPerThread = 8;
constexpr int kSumChunk    = kSumThreads * kSumPerThread; // elements per partial
constexpr int kFinalThreads = 1024;

// s + e == a + b exactly (no multiplication, so no contraction can change it)
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s         = a + b;
    double bp = s - a;
    e         = (a - (s - bp)) + (b - bp);
}
__device__ __forceinline__ double2 cs_add(double2 x, double v) {
    double s, e;
    two_sum(x.x, v, s, e);
    return make_double2(s, x.y + e);
}
__device__ __forceinline__ double2 cs_merge(double2 x, double2 y) {
    double s, e;
    two_sum(x.x, y.x, s, e);
    return make_double2(s, (x.y + y.y) + e);
}

// Fixed-shape tree over the block's threads; returns the block total in thread 0.
template<int NT> __device__ double2 block_reduce(double2 v, double2* sh) {
    const int t = threadIdx.x;
    sh[t]       = v;
    __syncthreads();
#pragma unroll
    for (int stride = NT / 2; stride > 0; stride >>= 1) {
        if (t < stride)
            sh[t] = cs_merge(sh[t], sh[t + stride]);
        __syncthreads();
    }
    double2 r = sh[0];
    __syncthreads();
    return r;
}

// Partial (sum, error) of each chunk of kSumChunk consecutive elements: part[blockIdx.x].
__global__ void __launch_bounds__(kSumThreads) sum_partials_kernel(const double* __restrict__ x,
                                                                   long long n, double2* part) {
    __shared__ double2 sh[kSumThreads];
    const long long    base = (long long)blockIdx.x * kSumChunk + threadIdx.x;
    double2            acc  = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < kSumPerThread; k++) {
        long long i = base + (long long)k * kSumThreads;
        if (i < n)
            acc = cs_add(acc, x[i]);
    }
    double2 r = block_reduce<kSumThreads>(acc, sh);
    if (threadIdx.x == 0)
        part[blockIdx.x] = r;
}

// out[q] = total of part[q * stride + 0 .. nparts-1], one block per q.
__global__ void __launch_bounds__(kFinalThreads) sum_final_kernel(const double2* __restrict__ part,
                                                                  int nparts, int stride,
                                                                  double* out) {
    __shared__ double2 sh[kFinalThreads];
    const double2*     p   = part + (size_t)blockIdx.x * stride;
    double2            acc = make_double2(0.0, 0.0);
    for (int i = threadIdx.x; i < nparts; i += kFinalThreads)
        acc = cs_merge(acc, p[i]);
    double2 r = block_reduce<kFinalThreads>(acc, sh);
    if (threadIdx.x == 0)
        out[blockIdx.x] = r.x + r.y;
}

// Control volume of a cell as the reference computes it (src/ESP/profx_globdiag.cu:82-90).
__device__ __forceinline__ double control_volume(double areasT, double A, double zup,
                                                 double zlow, bool deep) {
    if (deep)
        return areasT / pow(A, 2) * (pow(zup, 3) - pow(zlow, 3)) / 3;
    return areasT * (zup - zlow);
}

// One thread per (column, level); block (bx, lev) writes the partials of its 256 columns for the
// six quantities at part[q * nblk + lev * gridDim.x + bx].
__global__ void __launch_bounds__(kSumThreads)
    globdiag_kernel(Geometry g, Phys P, const double* __restrict__ Rho,
                    const double* __restrict__ Mh, const double* __restrict__ W,
                    const double* __restrict__ T, const double* __restrict__ p,
                    const double* __restrict__ Cp, const double* __restrict__ Rd, double2* part,
                    double* __restrict__ cells) {
    __shared__ double2 sh[kSumThreads];
    const int          col = blockIdx.x * kSumThreads + threadIdx.x, lev = blockIdx.y;
    const int          Np = g.Np, nv = g.nv;
    double             term[6] = {0, 0, 0, 0, 0, 0};
    if (col < g.N) {
        const size_t i   = (size_t)lev * Np + col;
        const double A   = P.A;
        const double Vol = control_volume(g.areasT[col], A, g.Altitudeh[lev + 1] + A,
                                          g.Altitudeh[lev] + A, P.DeepModel);
        const double lon = g.lon[col], lat = g.lat[col];
        const double m0 = Mh[(size_t)(0 * nv + lev) * Np + col],
                     m1 = Mh[(size_t)(1 * nv + lev) * Np + col],
                     m2 = Mh[(size_t)(2 * nv + lev) * Np + col];
        const double rho = Rho[i];
        // CalcTotEnergy (:45-112)
        {
            double Cv   = Cp[i] - Rd[i];
            double wx   = W[i] * cos(lat) * cos(lon);
            double wy   = W[i] * cos(lat) * sin(lon);
            double wz   = W[i] * sin(lat);
            double Ek   = 0.5 * ((m0 + wx) * (m0 + wx) + (m1 + wy) * (m1 + wy) + (m2 + wz) * (m2 + wz))
                        / rho;
            double Eint = Cv * T[i] * rho;
            double Eg   = rho * P.Gravit * g.Altitude[lev];
            term[0]     = (Ek + Eint + Eg) * Vol;
        }
        // CalcMass (:182-212)
        term[1] = rho * Vol;
        // CalcAngMom (:119-180)
        {
            double r   = (A + g.Altitude[lev]);
            double rx  = r * g.func_r[0 * Np + col], ry = r * g.func_r[1 * Np + col],
                   rz  = r * g.func_r[2 * Np + col];
            double AMx = ry * m2 - rz * m1 - rho * P.Omega * r * rz * cos(lat) * cos(lon);
            double AMy = -rx * m2 + rz * m0 - rho * P.Omega * r * rz * cos(lat) * sin(lon);
            double AMz = rx * m1 - ry * m0 + rho * P.Omega * r * r * cos(lat) * cos(lat);
            term[2]    = AMx * Vol;
            term[3]    = AMy * Vol;
            term[4]    = AMz * Vol;
        }
        // CalcEntropy (:214-252)
        {
            double kappa = Rd[i] / Cp[i];
            double potT  = T[i] * pow(P.P_Ref / p[i], kappa);
            double Sdens = Cp[i] * log(potT);
            term[5]      = Sdens * Vol;
        }
    }
    if (cells && col < g.N) // the per-cell terms (the reference's Etotal_d, Mass_d, ... arrays)
#pragma unroll
        for (int q = 0; q < 6; q++)
            cells[((size_t)q * nv + lev) * Np + col] = term[q];
    const int nblk = gridDim.x * gridDim.y, b = lev * gridDim.x + blockIdx.x;
#pragma unroll
    for (int q = 0; q < 6; q++) {
        double2 r = block_reduce<kSumThreads>(make_double2(term[q], 0.0), sh);
        if (threadIdx.x == 0)
            part[(size_t)q * nblk + b] = r;
    }
}

} // namespace

int globdiag_partials(const Geometry& g) { return ((g.N + kSumThreads - 1) / kSumThreads) * g.nv; }

void launch_globdiag(const Geometry& g, const Phys& P, const State& s, double2* part, double* out6,
                     cudaStream_t st, double* cells) {
    dim3 grid((g.N + kSumThreads - 1) / kSumThreads, g.nv);
    globdiag_kernel<<<grid, kSumThreads, 0, st>>>(g, P, s.Rho, s.Mh, s.W, s.T, s.p, s.Cp, s.Rd,
                                                  part, cells);
    const int nblk = (int)(grid.x * grid.y);
    sum_final_kernel<<<6, kFinalThreads, 0, st>>>(part, nblk, nblk, out6);
}

long long device_sum_partials(long long n) { return (n + kSumChunk - 1) / kSumChunk; }

void launch_device_sum(const double* x, long long n, double2* part, double* out, cudaStream_t st) {
    const long long np = device_sum_partials(n);
    if (np > 0)
        sum_partials_kernel<<<(unsigned)np, kSumThreads, 0, st>>>(x, n, part);
    sum_final_kernel<<<1, kFinalThreads, 0, st>>>(part, (int)np, 0, out);
}

} // namespace thorx

// ---------------------------------------------------------------------------------------------
// Allocation-free device sum: the partials of a call live in this fixed array of the library's
// own device memory instead of a cudaMalloc per call. 65536 partials of 2048 elements each cap
// one call at 134,217,728 doubles; the entry after the partials holds the result. Nothing here
// needs to start at zero: a call writes every partial it reads, and the result, before reading.
// ---------------------------------------------------------------------------------------------
namespace thorx {
namespace {

constexpr long long kNoAllocPartials = 65536;
constexpr int       kMaxDevices      = 64;

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocPartials + 1];

} // namespace

long long noalloc_sum_max_n() { return kNoAllocPartials * kSumChunk; }

// Device address of the scratch on the current device, looked up once per device (with that
// device current) and remembered; later calls only read the table.
cudaError_t noalloc_sum_scratch(double2** part, double** result) {
    static std::mutex mu;
    static double2*   addr[kMaxDevices] = {};
    int               dev               = -1;
    cudaError_t       e                 = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    if (dev < 0 || dev >= kMaxDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        e       = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return e;
        addr[dev] = (double2*)p;
    }
    *part   = addr[dev];
    *result = (double*)(addr[dev] + kNoAllocPartials);
    return cudaSuccess;
}

} // namespace thorx
