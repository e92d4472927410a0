// The ESP object a physics module receives (the reference's class ESP, src/headers/esp.h:72-371),
// as the thorx_phy shim fills it: the grid sizes and, on the device, in the reference layouts
// ([col][lev], [col][lev][xyz], [col][lev+1]), the geometry and the state, stage, deviation and
// coupling arrays below. The shim copies the dynamical core's arrays into these before every hook
// and back after it. Members the shim does not provide are null.
#pragma once

class Insolation;

class ESP
{
public:
    ESP(int point_num_, int nv_, int nl_region_, int nr_, int glevel_) :
        point_num(point_num_), nv(nv_), nvi(nv_ + 1), nl_region(nl_region_), nr(nr_),
        glevel(glevel_) {}

    // general
    const int    point_num;
    const int    nv;
    const int    nvi;
    const int    nl_region;
    const int    nr;
    const int    glevel;
    const bool   spring_dynamics = true;
    const double spring_beta     = 1.15;
    int          current_step    = 0;
    double       simulation_time = 0.0;

    // geometry on the device (reference layouts)
    int*    point_local_d = nullptr;
    int*    maps_d        = nullptr;
    double* Altitude_d    = nullptr;
    double* Altitudeh_d   = nullptr;
    double* nvecoa_d      = nullptr;
    double* nvecti_d      = nullptr;
    double* nvecte_d      = nullptr;
    double* areasT_d      = nullptr;
    double* areasTr_d     = nullptr;
    double* areas_d       = nullptr;
    double* lonlat_d      = nullptr;
    double* div_d         = nullptr;
    double* grad_d        = nullptr;
    double* func_r_d      = nullptr;

    // state
    double* temperature_d = nullptr;
    double* Mh_d          = nullptr;
    double* W_d           = nullptr;
    double* Wh_d          = nullptr;
    double* Rho_d         = nullptr;
    double* pressure_d    = nullptr;
    double* Rd_d          = nullptr;
    double* Cp_d          = nullptr;

    // RK stage and small-step deviation
    double* Rhos_d      = nullptr;
    double* pressures_d = nullptr;
    double* Mhs_d       = nullptr;
    double* Whs_d       = nullptr;
    double* Rhok_d      = nullptr;
    double* pressurek_d = nullptr;
    double* Mhk_d       = nullptr;
    double* Wk_d        = nullptr;
    double* Whk_d       = nullptr;

    // module coupling
    double* profx_Qheat_d = nullptr;
    double* profx_dMh_d   = nullptr;
    double* profx_dWh_d   = nullptr;

    // not provided by the shim
    double* h_d = nullptr;
    double* hh_d = nullptr;
    double* pt_d = nullptr;
    double* pth_d = nullptr;
    double* gtil_d = nullptr;
    double* gtilh_d = nullptr;
    double* Adv_d = nullptr;
    double* SlowMh_d = nullptr;
    double* SlowWh_d = nullptr;
    double* SlowRho_d = nullptr;
    double* Slowpressure_d = nullptr;
    double* Ws_d = nullptr;
    double* profx_dW_d = nullptr;
    double* Tsurface_d = nullptr;
};
