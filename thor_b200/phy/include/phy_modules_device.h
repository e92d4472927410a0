// The RK array registry of the reference (device_RK_array_manager,
// src/headers/dyn/phy_modules_device.h:63-74, src/ESP/phy_modules_device.cu:53-67): arrays of
// point_num * nv * dimensions doubles in the module's own layout that the dynamical core's RK
// stages reset (array = arrayi - arrayk) and accumulate (arrayk += array). The shim passes them on
// to thorx_rk_register_array_n; at most 10.
#pragma once

#define NUM_PHY_MODULES_DYN_CORE_ARRAYS 10

struct thorx_ctx;

class device_RK_array_manager
{
public:
    device_RK_array_manager(thorx_ctx* ctx_, long long cells_) : ctx(ctx_), cells(cells_) {}
    bool register_array(double* array_d, double* arrayk_d, double* arrayi_d, int dimensions);
    void allocate_device_array() {}
    int  registered = 0;

private:
    thorx_ctx* ctx;
    long long  cells; // point_num * nv
};
