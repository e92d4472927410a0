/* thorx_phy: the reference's physics-module managers on the thorx dynamical core.
 *
 * A module manager written for the reference (the phy_modules_* functions of
 * src/headers/phy_modules.h:57-98, e.g. src/physics/managers/empty/src/phy_modules.cu) compiles
 * unchanged against the headers in thor_b200/phy/include and links with thor_b200/phy/thorx_phy.cu
 * and libthorx.so into one shared library (thor_b200/phy/Makefile). thorx_phy_attach then plays the
 * part of ESP for it: the manager's hooks run where the reference's ESP calls them (through
 * thorx_module_add), on an ESP object whose device arrays are in the reference layouts, copied
 * from the dynamical core's arrays before every hook and back after it. The manager's kernels run
 * on the legacy default stream and its hooks may synchronise, so the context steps without graph
 * capture (thorx_set_graph_mode(ctx, 0)).
 *
 * Replaces the module-manager calls of src/ESP/esp_initial.cu:1462-1476 (generate_config,
 * print_config, init_mem, init_data) and src/ESP/esp.cu (free_mem at the end of the run).
 */
#ifndef THORX_PHY_H
#define THORX_PHY_H

#include "thorx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The SimulationSetup values a manager may read (src/headers/simulation_setup.h). */
typedef struct {
    double A, Omega, Gravit, Rd, Cp, Tmean, P_Ref, Top_altitude, Diffc, Diffc_v, DivDampc;
    int    GravHeightVar, DeepModel, HyDiff, HyDiffOrder, DivDampP, VertHyDiff, VertHyDiffOrder;
    int    NonHydro, conv_adj, conv_adj_iter, soft_adjustment;
    int    first_step; /* step number of the next physics step (1 for a new run)              */
} thorx_phy_setup;

/* Attaches the manager linked into this library to ctx (which must have been created from `grid`;
 * its arrays are copied to the device once, in the reference layouts): generate_config, the nkeys
 * configuration values (keys the manager registered; an unknown key or a value that does not parse
 * is THORX_E_ARG), print_config, init_mem (its register_array calls go to
 * thorx_rk_register_array_n), init_data, then the dynamical-core and physics hooks. The context
 * stops capturing its step as a graph. *handle is released by thorx_phy_detach, which calls
 * free_mem: call it only after the last step of ctx (or after thorx_destroy). */
int thorx_phy_attach(thorx_ctx* ctx, const thorx_grid* grid, const thorx_phy_setup* sim,
                     const char* const* keys, const char* const* values, int nkeys, void** handle);
int thorx_phy_detach(void* handle);
/* phy_modules_get_name() of the linked manager, into buf (size n). */
int thorx_phy_name(char* buf, int n);

#ifdef __cplusplus
}
#endif
#endif
