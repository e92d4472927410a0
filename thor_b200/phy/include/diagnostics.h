// The kernel_diagnostics object of the reference's phy_loop (src/headers/diagnostics.h:29): the
// shim passes one with no diagnostics enabled.
#pragma once

class kernel_diagnostics
{
public:
    bool check_flag() { return false; }
    void reset_flag() {}
};
