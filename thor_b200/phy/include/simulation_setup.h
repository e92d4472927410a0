// The run parameters a physics module reads (the reference's SimulationSetup,
// src/headers/simulation_setup.h), filled by thorx_phy_attach from thorx_phy_setup.
#pragma once

#define kb_constant 1.38e-23  // Boltzmann constant [J/K]
#define mu_constant 1.660e-27 // Atomic mass unit   [kg]

class SimulationSetup
{
public:
    char   simulation_ID[160] = "thorx";
    double A = 6371000.0, Omega = 7.292e-5, Gravit = 9.8;
    bool   GravHeightVar = false;
    double Rd = 287.0, Cp = 1005.0, Tmean = 300.0, P_Ref = 1e5, Top_altitude = 36000.0;
    double Diffc = 0.0, Diffc_v = 0.0, DivDampc = 0.0;
    bool   DeepModel = true, HyDiff = true;
    int    HyDiffOrder = 4;
    bool   DivDampP = true, VertHyDiff = false;
    int    VertHyDiffOrder = 6;
    bool   NonHydro = true, globdiag = false;
    int    increased_damping_for_n_steps = 0;
    bool   RayleighSponge = false, RayleighSpongeT = false, DiffSponge = false;
    bool   output_mean = false, out_interm_momentum = false, output_diffusion = false;
    bool   conv_adj = false;
    int    conv_adj_iter = 1;
    bool   soft_adjustment = false, gcm_off = false, single_column = false, rest = true;
    int    n_out = 1000;
};
