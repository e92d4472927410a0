// Double-gray radiative transfer (DualbandGray) and the insolation it needs, on the device.
//
// Reference: Insolation::phy_loop (src/ESP/insolation.cu:459-490, orbit update :514-529,
// calc_zenith :128-168) and radiative_transfer::phy_loop (spin-up/down, rtm_dual_band launch,
// annual insolation; src/physics/modules/src/radiative_transfer.cu:769-1105) with the kernel
// rtm_dual_band and its device functions (src/physics/modules/inc/profx_RT.h:30-587). The
// arithmetic of each piece follows the reference operation for operation.
//
// Differences of form: the orbit update, a few scalar lines of host code in the reference, runs
// in a one-thread kernel on a device-resident step counter so that a captured step graph
// advances it by itself; the column kernel works on the column-fastest layout (each level a
// plane, coalesced across a warp, one thread per column for the serial level recurrences).
// GravHeightVar with RT is rejected at enable time: the reference's radcsw then reads
// Altitudeh[nv+1], past the end of the array (profx_RT.h:68).
#include "thorx_internal.h"

namespace thorx {
namespace {

// Kepler's equation by the third-order iteration of insolation.cu:65-88 (which stops as soon as
// the last correction is not above 1e-15, signed); bounded at 100 iterations.
__device__ double solve_kepler(double M, double ecc) {
    double E  = M + (sin(M) < 0.0 ? -1.0 : 1.0) * 0.85 * ecc;
    double d3 = 1.0;
    for (int it = 0; it < 100 && d3 > 1e-15; it++) {
        double fi = E - ecc * sin(E) - M, f1 = 1.0 - ecc * cos(E), f2 = ecc * sin(E),
               f3 = ecc * cos(E);
        double d1 = -fi / f1;
        double d2 = -fi / (f1 + 0.5 * d1 * f2);
        d3        = -fi / (f1 + 0.5 * d2 * f2 + 1. / 6. * d2 * d2 * f3);
        E         = E + d3;
    }
    return E;
}

// Orbit update (when the reference calls it), spin-up/down scaling and the run flag of this step.
__global__ void rt_orbit_kernel(RtConst c, Phys P, RtStep* st) {
    const long long nstep = st->nstep;
    st->cur               = nstep;
    st->nstep             = nstep + 1;
    const double dt       = P.timestep;
    if (!c.sync_rot || c.ecc > 1e-10) {
        const double time = nstep * dt;
        double       M    = fmod((c.mean_motion * time + c.mean_anomaly_i), (2 * M_PI));
        double       E    = fmod(solve_kepler(M, c.ecc), (2 * M_PI));
        st->r_orb         = 1.0 - c.ecc * cos(E);
        double f          = 2.0 * atan(sqrt((1.0 + c.ecc) / (1.0 - c.ecc)) * tan(E / 2.0));
        if (f < 0.0)
            f += 2 * M_PI;
        const double true_long = fmod((f + c.longp), (2 * M_PI));
        st->sin_decl           = sin(c.obliquity) * sin(true_long);
        st->cos_decl           = sqrt(1.0 - st->sin_decl * st->sin_decl);
        st->alpha              = -P.Omega * time + true_long - c.true_long_i + c.alpha_i;
    }
    bool   run = true;
    double Qs  = 1.0;
    if (c.spinup_start > -1 && c.spinup_stop > -1) {
        if (nstep < c.spinup_start) {
            run = false;
            Qs  = 0.0;
        }
        else if (nstep >= c.spinup_start && nstep <= c.spinup_stop) {
            double x = (double)(nstep - c.spinup_start) / (double)(c.spinup_stop - c.spinup_start);
            Qs       = (1 + sin(M_PI * x - M_PI / 2.0)) / 2.0;
            run      = true;
        }
    }
    if (c.spindown_start > -1 && c.spindown_stop > -1) {
        if (nstep >= c.spindown_start && nstep <= c.spindown_stop) {
            double x = (double)(nstep - c.spindown_start) / (double)(c.spindown_stop - c.spindown_start);
            Qs       = 1.0 - (1 + sin(M_PI * x - M_PI / 2.0)) / 2.0;
            run      = true;
        }
        else if (nstep >= c.spindown_stop) {
            run = false;
            Qs  = 0.0;
        }
    }
    st->Qheat_scaling = Qs;
    st->run           = run;
}

__device__ int factorial_num(int n) {
    int t = 1;
    while (n != 0) {
        t = t * n;
        n = n - 1;
    }
    return t;
}

// source_func_lin (profx_RT.h:133-160)
__device__ double source_func_lin(double bb, double bl, double bt, double tau, double diff_ang) {
    double e1 = 0.0, e2 = 0.0;
    if (tau >= 1e-10) {
        e1 = bb - bl + (bl - (diff_ang / (tau / 2.0)) * (bb - bl)) * (1.0 - exp(-(tau / 2.0) / diff_ang));
        e2 = bl - bt + (bt - (diff_ang / (tau / 2.0)) * (bl - bt)) * (1.0 - exp(-(tau / 2.0) / diff_ang));
    }
    else {
        for (int i = 0; i < 5; i++) {
            int fac = factorial_num(i + 2);
            e1 = e1 + (pow(-1.0, i + 2.0)) * ((bl + (i + 1) * bl) / fac) * pow((tau / 2.0) / diff_ang, i + 1.0);
            e2 = e2 + (pow(-1.0, i + 2.0)) * ((bt + (i + 1) * bb) / fac) * pow((tau / 2.0) / diff_ang, i + 1.0);
        }
    }
    return e1 + e2 * exp(-(tau / 2.0) / diff_ang);
}

// One thread per column: calc_zenith, the top-of-atmosphere insolation and annual_insol, then
// rtm_dual_band (profx_RT.h:316-587) with computetau, radcsw (no surface, GravHeightVar
// excluded), radclw (reflecting lower boundary), the cooling limiter and the coupling into
// profx_Qheat. The reference computes the insolation inside radcsw and the annual average after
// the RT; both depend on the zenith angle only, so computing them first changes no value.
__global__ void __launch_bounds__(128) rt_column_kernel(Geometry g, Phys P, RtConst c, RtFields f,
                                                       State s) {
    const int id = g.tile0 * 32 + blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= g.col_end)
        return;
    const RtStep  st = *f.step;
    const int     nv = g.nv, Np = g.Np;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    const double  A = P.A, gravit = P.Gravit, ps0 = P.P_Ref, timestep = P.timestep;
    const double  lat = g.lat[id], lon = g.lon[id];
    // ---- calc_zenith + compute_cos_zenith_angles (insolation.cu:128-207) ----
    {
        const bool obl = !(c.obliquity < 1e-10);
        double     cz;
        if (c.sync_rot && c.ecc < 1e-10)
            cz = obl ? (sin(lat) * st.sin_decl + cos(lat) * st.cos_decl * cos(lon - c.alpha_i))
                     : cos(lat) * cos(lon - c.alpha_i);
        else if (c.sync_rot && !obl)
            cz = cos(lat) * cos(lon - st.alpha);
        else
            cz = (sin(lat) * st.sin_decl + cos(lat) * st.cos_decl * cos(lon - st.alpha));
        f.cos_zenith[id] = cz < 0.0 ? 0.0 : cz;
    }
    if (!st.run)
        return;
    const double coszrs = c.rt1Dmode ? 0.5 : f.cos_zenith[id];
    // insolation at the top (radcsw, profx_RT.h:74; 0 on the night side) and its first-orbit
    // average (annual_insol, profx_RT.h:30-37), for every column in either mode
    f.insol[id]           = coszrs > 0.0 ? c.incflx * pow(st.r_orb, -2) * coszrs : 0.0;
    const long long nstep = st.cur;
    if (nstep * timestep < (2 * M_PI / c.mean_motion))
        f.insol_ann[id] = f.insol_ann[id] * (nstep - 1) / nstep + f.insol[id] / nstep;
    if (f.fallback && !(f.fallback[id] || recheck_column(id, f.period, nstep)))
        return;
    auto P_ = [&](int lev) { return s.p[lev * Np + id]; };
    auto R_ = [&](int lev) { return s.Rho[lev * Np + id]; };
    auto T_ = [&](int lev) { return s.T[lev * Np + id]; };
    auto H  = [&](double* a, int lev) -> double& { return a[lev * Np + id]; };
    auto TAU = [&](int lev, int k) -> double& { return f.tau[(k * nv + lev) * Np + id]; };

    for (int lev = 0; lev < nv; lev++)
        H(f.dtemp, lev) = 0.0;
    // interface pressures and temperatures (profx_RT.h:419-466)
    for (int lev = 0; lev <= nv; lev++) {
        if (lev == 0) {
            const double psm = P_(1) - R_(0) * gravit * (-Alt[0] - Alt[1]);
            const double ps  = 0.5 * (P_(0) + psm);
            H(f.phtemp, 0)   = ps;
            H(f.ttemp, 0)    = T_(0);
            H(f.thtemp, 0)   = H(f.ttemp, 0);
        }
        else if (lev == nv) {
            double pp = P_(nv - 2)
                        + (P_(nv - 1) - P_(nv - 2)) / (Alt[nv - 1] - Alt[nv - 2])
                              * (2 * Alth[nv] - Alt[nv - 1] - Alt[nv - 2]);
            if (pp < 0)
                pp = 0;
            const double ptop = 0.5 * (P_(nv - 1) + pp);
            H(f.phtemp, nv)   = ptop;
            H(f.thtemp, nv)   = T_(nv - 1);
        }
        else {
            H(f.ttemp, lev) = T_(lev);
            const double xi = Alth[lev], xim = Alt[lev - 1], xip = Alt[lev];
            const double a = (xi - xip) / (xim - xip), b = (xi - xim) / (xip - xim);
            H(f.phtemp, lev) = P_(lev - 1) * a + P_(lev) * b;
            H(f.thtemp, lev) = T_(lev - 1) * a + H(f.ttemp, lev) * b;
        }
    }
    const double kappa_lw_lat = c.latf_lw ? c.kappa_lw + (c.kappa_lw_pole - c.kappa_lw) * pow(sin(lat), 2)
                                          : c.kappa_lw;
    // computetau (profx_RT.h:278-314)
    for (int lev = 0; lev < nv; lev++) {
        TAU(lev, 0) = c.n_sw * c.kappa_sw * pow(P_(lev) / ps0, c.n_sw - 1) * R_(lev) * (Alth[lev + 1] - Alth[lev]);
        TAU(lev, 1) = kappa_lw_lat * (1 + c.n_lw * (1 - c.f_lw) / c.f_lw * pow(P_(lev) / ps0, c.n_lw - 1))
                      * R_(lev) * (Alth[lev + 1] - Alth[lev]);
    }
    for (int lev = 0; lev <= nv; lev++)
        H(f.fsw_up, lev) = 0.0;
    for (int lev = 0; lev <= nv; lev++)
        H(f.fsw_dn, lev) = 0.0;
    if (coszrs > 0.0) { // radcsw (profx_RT.h:39-118)
        const double tau      = (c.kappa_sw / gravit) * (H(f.phtemp, nv));
        const double flux_top = f.insol[id] * (1.0 - c.albedo);
        H(f.fsw_dn, nv)       = flux_top * exp(-(1.0 / coszrs) * tau);
        for (int lev = nv; lev >= 1; lev--)
            H(f.fsw_dn, lev - 1) = H(f.fsw_dn, lev) * exp(-(1.0 / coszrs) * TAU(lev - 1, 0));
        for (int lev = 0; lev <= nv; lev++)
            H(f.fsw_up, lev) = 0.0;
        for (int lev = 0; lev < nv; lev++) {
            const double rup = 1.0, rlow = 1.0;
            H(f.dtemp, lev) = -(pow(rlow, 2) * (H(f.fsw_up, lev) - H(f.fsw_dn, lev))
                                - pow(rup, 2) * (H(f.fsw_up, lev + 1) - H(f.fsw_dn, lev + 1)))
                              / ((Alth[lev] - Alth[lev + 1]));
        }
    }
    const double rscale = P.DeepModel ? (A + Alth[nv]) / A : 1.0;
    f.ASR[id]           = H(f.fsw_dn, nv) * g.areasT[id] * pow(rscale, 2);
    for (int lev = 0; lev <= nv; lev++)
        H(f.flw_up, lev) = 0.0;
    for (int lev = 0; lev <= nv; lev++)
        H(f.flw_dn, lev) = 0.0;
    // radclw (profx_RT.h:162-275)
    const double bc = 5.677036E-8;
    H(f.flw_dn, nv) = 0.0;
    for (int lev = nv - 1; lev >= 0; lev--) {
        if (TAU(lev, 1) < 0.0)
            TAU(lev, 1) = 0.0;
        const double tb = H(f.thtemp, lev), tl = H(f.ttemp, lev), tt = H(f.thtemp, lev + 1);
        const double bb = bc * tb * tb * tb * tb, bl = bc * tl * tl * tl * tl, bt = bc * tt * tt * tt * tt;
        const double ed = source_func_lin(bb, bl, bt, TAU(lev, 1), c.diff_ang);
        H(f.flw_dn, lev) = ed + H(f.flw_dn, lev + 1) * exp(-(1. / c.diff_ang) * TAU(lev, 1));
    }
    H(f.flw_up, 0) = bc * c.Tint * c.Tint * c.Tint * c.Tint;
    H(f.flw_up, 0) += H(f.flw_dn, 0);
    for (int lev = 1; lev <= nv; lev++) {
        if (TAU(lev - 1, 1) < 0.0)
            TAU(lev - 1, 1) = 0.0;
        const double tb = H(f.thtemp, lev - 1), tl = H(f.ttemp, lev - 1), tt = H(f.thtemp, lev);
        const double bb = bc * tb * tb * tb * tb, bl = bc * tl * tl * tl * tl, bt = bc * tt * tt * tt * tt;
        const double eu = source_func_lin(bt, bl, bb, TAU(lev - 1, 1), c.diff_ang);
        H(f.flw_up, lev) = eu + H(f.flw_up, lev - 1) * exp(-(1. / c.diff_ang) * TAU(lev - 1, 1));
    }
    for (int lev = 0; lev < nv; lev++) {
        const double rup = 1.0, rlow = 1.0;
        H(f.dtemp, lev) = H(f.dtemp, lev)
                          - (pow(rlow, 2) * (H(f.flw_up, lev) - H(f.flw_dn, lev))
                             - pow(rup, 2) * (H(f.flw_up, lev + 1) - H(f.flw_dn, lev + 1)))
                                / ((Alth[lev] - Alth[lev + 1]));
    }
    f.OLR[id] = H(f.flw_up, nv) * g.areasT[id] * pow(rscale, 2);
    if (f.fallback) // surrogate mode: the combine kernel limits and couples
        return;
    // cooling limiter and coupling to the dynamical core (profx_RT.h:560-584)
    for (int lev = 0; lev < nv; lev++) {
        const int i = lev * Np + id;
        double    d = f.dtemp[i];
        if (s.p[i] + s.Rd[i] / (s.Cp[i] - s.Rd[i]) * d * timestep < 0)
            d = -s.p[i] / timestep;
        f.dtemp[i] = d;
        f.qheat[i] = d;
        s.Qheat[i] += st.Qheat_scaling * d;
    }
}

} // namespace

void launch_rt(const Geometry& g, const Phys& P, const RtConst& c, const RtFields& f,
               const State& s, cudaStream_t st) {
    rt_orbit_kernel<<<1, 1, 0, st>>>(c, P, f.step);
    rt_column_kernel<<<(g.ntile * 32 + 127) / 128, 128, 0, st>>>(g, P, c, f, s);
}

} // namespace thorx
