// The physics-module interface of the reference (src/headers/phy_modules.h:57-98), for module
// managers compiled against the thorx_phy shim instead of the reference's ESP. Same declarations;
// the types behind them (ESP, SimulationSetup, config_file, storage, device_RK_array_manager,
// kernel_diagnostics) are the shim's own, in this directory. A manager defines the functions it
// needs; the shim supplies weak defaults (return true) for the rest, so both phy_loop forms link:
// the header's (with kernel_diagnostics) and the empty manager's (without,
// src/physics/managers/empty/src/phy_modules.cu:81).
#pragma once

#include <string>

#include "config_file.h"
#include "define.h"
#include "diagnostics.h"
#include "esp.h"
#include "grid.h"
#include "log_writer.h"
#include "phy_modules_device.h"
#include "simulation_setup.h"
#include "storage.h"

std::string phy_modules_get_name();
void        phy_modules_print_config();
bool        phy_modules_generate_config(config_file& config_reader);
bool        phy_modules_init_mem(const ESP& esp, device_RK_array_manager& phy_modules_core_arrays);
bool        phy_modules_free_mem();
bool        phy_modules_init_data(const ESP& esp, const SimulationSetup& sim, storage* s);
bool        phy_modules_dyn_core_loop_init(const ESP& esp);
bool        phy_modules_dyn_core_loop_slow_modes(const ESP& esp, const SimulationSetup& sim,
                                                 int nstep, double times);
bool        phy_modules_dyn_core_loop_fast_modes(const ESP& esp, const SimulationSetup& sim,
                                                 int nstep, double time_step);
bool        phy_modules_dyn_core_loop_end(const ESP& esp);
bool        phy_modules_phy_loop(ESP& esp, const SimulationSetup& sim, kernel_diagnostics& diag,
                                 int nstep, double time_step);
bool        phy_modules_phy_loop(ESP& esp, const SimulationSetup& sim, int nstep, double time_step);
bool        phy_modules_store(const ESP& esp, storage& s);
bool        phy_modules_store_init(storage& s);
