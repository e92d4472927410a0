// Probe physics module written against the reference's phy_modules_* interface
// (src/headers/phy_modules.h:57-98), built with the thorx_phy shim (thor_b200/phy/). TEST
// INFRASTRUCTURE ONLY: loaded by tests/test_phy_shim.py, never by the product.
//
// It does what the probe of oracle/ref_harness.cu does at the same hooks, in the reference layouts:
//   init_mem                  tracer, tracerk, tracers [col][lev][2], registered with the RK array
//                             manager (register_array, 2 dimensions)
//   dyn_core_loop_init        tracerk = tracer, tracers = 0
//   dyn_core_loop_fast_modes  tracers += times; at the 10th small step of a large step (the last
//                             small step of the last RK stage) snapshots of Rhos_d and Whs_d
//   dyn_core_loop_end         tracer = tracerk
//   phy_loop                  temperature_d += probe_heating (a configuration key, default 0.5 K)
// Every hook counts its calls.
#include <cstring>

#include "phy_modules.h"

namespace {
double*   tracer = nullptr, *tracerk = nullptr, *tracers = nullptr;
double*   snap_rhos = nullptr, *snap_whs = nullptr;
long long calls[5] = {0, 0, 0, 0, 0}; // init, slow, fast, end, phy_loop
int       fast_in_step = 0;
long      N = 0, nv = 0, nvi = 0;
double    heating = 0.0;

__global__ void add_kernel(double* x, long n, double v) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        x[i] += v;
}
} // namespace

std::string phy_modules_get_name() { return std::string("refapi_probe"); }

void phy_modules_print_config() { log::printf("  probe module, heating %g K per step\n", heating); }

bool phy_modules_generate_config(config_file& config_reader) {
    return config_reader.append_config_var("probe_heating", heating, 0.5);
}

bool phy_modules_init_mem(const ESP& esp, device_RK_array_manager& phy_modules_core_arrays) {
    N   = esp.point_num;
    nv  = esp.nv;
    nvi = esp.nvi;
    const size_t n = 2 * (size_t)N * nv * sizeof(double);
    cudaMalloc((void**)&tracer, n);
    cudaMalloc((void**)&tracerk, n);
    cudaMalloc((void**)&tracers, n);
    cudaMalloc((void**)&snap_rhos, (size_t)N * nv * sizeof(double));
    cudaMalloc((void**)&snap_whs, (size_t)N * nvi * sizeof(double));
    cudaMemset(tracer, 0, n);
    return phy_modules_core_arrays.register_array(tracers, tracerk, tracer, 2);
}

bool phy_modules_init_data(const ESP& esp, const SimulationSetup& sim, storage* s) {
    cudaMemset(snap_rhos, 0, (size_t)N * nv * sizeof(double));
    cudaMemset(snap_whs, 0, (size_t)N * nvi * sizeof(double));
    return true;
}

bool phy_modules_dyn_core_loop_init(const ESP& esp) {
    calls[0]++;
    fast_in_step = 0;
    cudaMemcpy(tracerk, tracer, 2 * (size_t)N * nv * sizeof(double), cudaMemcpyDeviceToDevice);
    cudaMemset(tracers, 0, 2 * (size_t)N * nv * sizeof(double));
    return true;
}

bool phy_modules_dyn_core_loop_slow_modes(const ESP& esp, const SimulationSetup& sim, int nstep,
                                          double times) {
    calls[1]++;
    return true;
}

bool phy_modules_dyn_core_loop_fast_modes(const ESP& esp, const SimulationSetup& sim, int nstep,
                                          double time_step) {
    calls[2]++;
    add_kernel<<<256, 256>>>(tracers, 2 * N * nv, time_step);
    if (++fast_in_step == 10) {
        cudaMemcpy(snap_rhos, esp.Rhos_d, (size_t)N * nv * sizeof(double), cudaMemcpyDeviceToDevice);
        cudaMemcpy(snap_whs, esp.Whs_d, (size_t)N * nvi * sizeof(double), cudaMemcpyDeviceToDevice);
    }
    return true;
}

bool phy_modules_dyn_core_loop_end(const ESP& esp) {
    calls[3]++;
    cudaMemcpy(tracer, tracerk, 2 * (size_t)N * nv * sizeof(double), cudaMemcpyDeviceToDevice);
    return true;
}

bool phy_modules_phy_loop(ESP& esp, const SimulationSetup& sim, kernel_diagnostics& diag, int nstep,
                          double time_step) {
    calls[4]++;
    add_kernel<<<256, 256>>>(esp.temperature_d, N * nv, heating);
    return true;
}

bool phy_modules_store_init(storage& s) { return true; }

bool phy_modules_store(const ESP& esp, storage& s) { return true; }

bool phy_modules_free_mem() {
    cudaFree(tracer);
    cudaFree(tracerk);
    cudaFree(tracers);
    cudaFree(snap_rhos);
    cudaFree(snap_whs);
    tracer = tracerk = tracers = snap_rhos = snap_whs = nullptr;
    return true;
}

// test access, reference layouts: "tracer" [col][lev][2], "set_tracer" (host in), "snap_Rhos"
// [col][lev], "snap_Whs" [col][lev+1]
extern "C" int refprobe_io(const char* what, double* host) {
    cudaError_t e;
    if (!std::strcmp(what, "tracer"))
        e = cudaMemcpy(host, tracer, 2 * (size_t)N * nv * 8, cudaMemcpyDeviceToHost);
    else if (!std::strcmp(what, "set_tracer"))
        e = cudaMemcpy(tracer, host, 2 * (size_t)N * nv * 8, cudaMemcpyHostToDevice);
    else if (!std::strcmp(what, "snap_Rhos"))
        e = cudaMemcpy(host, snap_rhos, (size_t)N * nv * 8, cudaMemcpyDeviceToHost);
    else if (!std::strcmp(what, "snap_Whs"))
        e = cudaMemcpy(host, snap_whs, (size_t)N * nvi * 8, cudaMemcpyDeviceToHost);
    else
        return -1;
    return e == cudaSuccess ? 0 : -2;
}
extern "C" long long refprobe_calls(int which) { return calls[which]; }
