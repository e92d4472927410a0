// Probe physics module for the module interface of include/thorx.h. TEST INFRASTRUCTURE ONLY:
// loaded by tests/test_modules.py, never by the product.
//
// Hooks (the same as the probe module of oracle/ref_harness.cu, which calls them where the
// reference's ESP calls its module manager):
//   dyn_core_loop_init        tracerk = tracer, tracers = 0
//   dyn_core_loop_fast_modes  tracers += times (a tendency of 1 per second); at the last small
//                             step of the last RK stage, snapshots of Rhos and Whs
//   dyn_core_loop_end         tracer = tracerk
//   phy_loop                  temperature += 0.5 K (before the pressure update)
// The tracer (two components) is registered with thorx_rk_register_array, so the RK stages
// reset and accumulate it as the reference's UpdateRK / UpdateRK2 do. Every hook counts its calls.
#include <cstring>

#include <cuda_runtime.h>

#include "thorx.h"

namespace {

struct Probe {
    thorx_ctx* ctx;
    int        nv, nvi;
    long       plane;
    int        flags;                     // bit 0: phy_loop, bit 1: fast-mode hook
    double *   q, *qk, *qs, *snap_rhos, *snap_whs;
    double *   Rhos, *Whs, *T;
    long long  calls[5] = {0, 0, 0, 0, 0}; // init, slow, fast, end, phy_loop
};

__global__ void add_kernel(double* x, long long n, double v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        x[i] += v;
}

int status() { return cudaGetLastError() == cudaSuccess ? 0 : 1; }

int init_hook(void* u, thorx_ctx*, void* st) {
    Probe*       p = (Probe*)u;
    const size_t n = 2 * (size_t)p->nv * p->plane;
    p->calls[0]++;
    cudaMemcpyAsync(p->qk, p->q, n * sizeof(double), cudaMemcpyDeviceToDevice, (cudaStream_t)st);
    cudaMemsetAsync(p->qs, 0, n * sizeof(double), (cudaStream_t)st);
    return status();
}
int slow_hook(void* u, thorx_ctx*, void*, int, double) {
    ((Probe*)u)->calls[1]++;
    return 0;
}
int fast_hook(void* u, thorx_ctx*, void* st, int rk, int ns, double times) {
    Probe* p = (Probe*)u;
    p->calls[2]++;
    add_kernel<<<256, 256, 0, (cudaStream_t)st>>>(p->qs, 2LL * p->nv * p->plane, times);
    if (rk == 2 && ns == 5) {
        cudaMemcpyAsync(p->snap_rhos, p->Rhos, (size_t)p->nv * p->plane * sizeof(double),
                        cudaMemcpyDeviceToDevice, (cudaStream_t)st);
        cudaMemcpyAsync(p->snap_whs, p->Whs, (size_t)p->nvi * p->plane * sizeof(double),
                        cudaMemcpyDeviceToDevice, (cudaStream_t)st);
    }
    return status();
}
int end_hook(void* u, thorx_ctx*, void* st) {
    Probe* p = (Probe*)u;
    p->calls[3]++;
    cudaMemcpyAsync(p->q, p->qk, 2 * (size_t)p->nv * p->plane * sizeof(double),
                    cudaMemcpyDeviceToDevice, (cudaStream_t)st);
    return status();
}
int phy_hook(void* u, thorx_ctx*, void* st, double) {
    Probe* p = (Probe*)u;
    p->calls[4]++;
    add_kernel<<<256, 256, 0, (cudaStream_t)st>>>(p->T, (long long)p->nv * p->plane, 0.5);
    return status();
}

} // namespace

extern "C" {

// Creates the probe on ctx, registers its tracer and adds it as a module. flags: bit 0 phy_loop,
// bit 1 the fast-mode hook (the tracer needs both bit 1 and the init/end hooks, always on).
int probe_create(thorx_ctx* ctx, int flags, void** out) {
    Probe* p = new Probe;
    p->ctx   = ctx;
    p->flags = flags;
    int comps;
    if (thorx_device_field(ctx, "Rhos", &p->Rhos, &p->nv, &comps, &p->plane)
        || thorx_device_field(ctx, "Whs", &p->Whs, &p->nvi, &comps, nullptr)
        || thorx_device_field(ctx, "temperature", &p->T, nullptr, nullptr, nullptr))
        return -1;
    const size_t n = 2 * (size_t)p->nv * p->plane;
    if (cudaMalloc(&p->q, n * 8) || cudaMalloc(&p->qk, n * 8) || cudaMalloc(&p->qs, n * 8)
        || cudaMalloc(&p->snap_rhos, (size_t)p->nv * p->plane * 8)
        || cudaMalloc(&p->snap_whs, (size_t)p->nvi * p->plane * 8))
        return -2;
    cudaMemset(p->q, 0, n * 8);
    cudaMemset(p->snap_rhos, 0, (size_t)p->nv * p->plane * 8);
    cudaMemset(p->snap_whs, 0, (size_t)p->nvi * p->plane * 8);
    if (thorx_rk_register_array(ctx, p->qs, p->qk, p->q, 2))
        return -3;
    thorx_module m;
    std::memset(&m, 0, sizeof m);
    m.user                     = p;
    m.dyn_core_loop_init       = init_hook;
    m.dyn_core_loop_slow_modes = slow_hook;
    m.dyn_core_loop_fast_modes = (flags & 2) ? fast_hook : nullptr;
    m.dyn_core_loop_end        = end_hook;
    m.phy_loop                 = (flags & 1) ? phy_hook : nullptr;
    if (thorx_module_add(ctx, &m))
        return -4;
    *out = p;
    return 0;
}

// Host copies, without the padding columns: "tracer" [2][nv][N], "snap_Rhos" [nv][N],
// "snap_Whs" [nv+1][N]; "set_tracer" copies host [2][nv][N] in.
int probe_io(void* h, const char* what, int N, double* host) {
    Probe*  p = (Probe*)h;
    double* d;
    int     rows;
    bool    in = false;
    if (!std::strcmp(what, "tracer"))
        d = p->q, rows = 2 * p->nv;
    else if (!std::strcmp(what, "set_tracer"))
        d = p->q, rows = 2 * p->nv, in = true;
    else if (!std::strcmp(what, "snap_Rhos"))
        d = p->snap_rhos, rows = p->nv;
    else if (!std::strcmp(what, "snap_Whs"))
        d = p->snap_whs, rows = p->nvi;
    else
        return -1;
    cudaError_t e;
    if (in)
        e = cudaMemcpy2D(d, p->plane * 8, host, (size_t)N * 8, (size_t)N * 8, rows,
                         cudaMemcpyHostToDevice);
    else
        e = cudaMemcpy2D(host, (size_t)N * 8, d, p->plane * 8, (size_t)N * 8, rows,
                         cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? 0 : -2;
}

long long probe_calls(void* h, int which) { return ((Probe*)h)->calls[which]; }

void probe_destroy(void* h) {
    Probe* p = (Probe*)h;
    cudaFree(p->q);
    cudaFree(p->qk);
    cudaFree(p->qs);
    cudaFree(p->snap_rhos);
    cudaFree(p->snap_whs);
    delete p;
}

} // extern "C"
