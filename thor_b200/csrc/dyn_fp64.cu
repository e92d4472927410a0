// thorx dynamical-core kernels, all-FP64 form, for sm_100a.
//
// Each kernel is a fusion of reference kernels (file:line in the comment above it). The
// arithmetic of every fused piece follows the reference operation for operation (same operand
// order and association, same math-library calls), so that the only differences from the
// reference build are the FMA contractions the compiler chooses.
//
// Work decomposition:
//   * column kernels (profx, adv_temp, vertical, update_rk2): one thread per column, looping over
//     the levels, because they carry a vertical recurrence (extrapolations, Thomas solve);
//   * stencil kernels (diffusion, divm0, slow_modes, momentum): one thread per column and a
//     chunk of kLevChunk levels, so that the column's geometry (up to 78 doubles) is loaded once
//     into registers and reused across the chunk.
// Neighbours come from the per-column tables described in thorx_internal.h; a hole (-1) reads 0.

#include "thorx_internal.h"

namespace thorx {
namespace {

constexpr int kColBlock  = 128; // threads per block, column kernels
constexpr int kStenBlock = 64;  // threads per block, stencil kernels
constexpr int kLevChunk  = 4;   // levels per thread, stencil kernels
constexpr int kVertBlock = 64;  // threads per block, vertical implicit kernel

__device__ __forceinline__ double gz(const double* __restrict__ plane, int id) {
    return id >= 0 ? __ldg(plane + id) : 0.0;
}

__device__ __forceinline__ double rscale_of(const Phys& P, const Geometry& g, int lev) {
    return P.DeepModel ? P.A / (g.Altitude[lev] + P.A) : 1.0;
}

// ---------------------------------------------------------------------------------------------
// ProfX: Recompute_W (reference src/headers/phy/profx_auxiliary.h:109-130), Compute_temperature
// (:64-92), held_suarez (src/headers/phy/profx_held_suarez.h:51-117), Compute_pressure (:94-107)
// and the NaN check on temperature (:132-146, src/ESP/profx_driver.cu:389-396,451-458).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kColBlock) profx_kernel(Geometry g, Phys P, State s) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int     Np = g.Np, nv = g.nv;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    for (int lev = 0; lev < nv; lev++) {
        double whl = s.Wh[lev * Np + c], wht = s.Wh[(lev + 1) * Np + c];
        double xi = Alt[lev], xim = Alth[lev], xip = Alth[lev + 1];
        double intt = (xi - xip) / (xim - xip);
        double intl = (xi - xim) / (xip - xim);
        s.W[lev * Np + c] = whl * intt + wht * intl;
    }
    for (int lev = 0; lev < nv; lev++) {
        int i   = lev * Np + c;
        s.T[i]  = s.p[i] / (s.Rd[i] * s.Rho[i]);
    }
    if (P.held_suarez) {
        const double sigmab = 0.7, ka = (1.0 / 40.0) * (1.0 / 86400.0), kf = 1.0 / 86400.0;
        const double ks = (1.0 / 4.0) * (1.0 / 86400.0), kappa = P.Rd / P.Cp, dTy = 60.0,
                     dthetaz = 10.0, p0 = 100000.0;
        const double lat  = g.lat[c];
        const double psm1 = s.p[Np + c] - s.Rho[c] * P.Gravit * (-Alt[0] - Alt[1]);
        const double ps   = 0.5 * (s.p[c] + psm1);
        for (int lev = 0; lev < nv; lev++) {
            int    i      = lev * Np + c;
            double pre    = s.p[i];
            double sigma  = (pre / ps);
            double sigma0 = (pre / p0);
            double Teq    = fmax(200.0, (315.0 - dTy * pow(sin(lat), 2.0)
                                      - dthetaz * log(sigma0) * pow(cos(lat), 2.0))
                                         * pow(sigma0, kappa));
            double kt = ka
                        + (ks - ka) * fmax(0.0, (sigma - sigmab) / (1.0 - sigmab))
                              * pow(cos(lat), 4.0);
            double kv = kf * fmax(0.0, (sigma - sigmab) / (1.0 - sigmab));
            for (int k = 0; k < 3; k++) {
                int j    = (k * nv + lev) * Np + c;
                s.Mh[j] = s.Mh[j] / (1.0 + kv * P.timestep);
            }
            s.T[i] -= kt * P.timestep * (s.T[i] - Teq);
        }
    }
    bool bad = false;
    for (int lev = 0; lev < nv; lev++) {
        int i  = lev * Np + c;
        s.p[i] = s.T[i] * s.Rd[i] * s.Rho[i];
        bad |= isnan(s.T[i]);
    }
    if (bad)
        atomicOr(s.flags, kFlagNaN);
}

// ---------------------------------------------------------------------------------------------
// Advection + Coriolis + thermodynamic diagnostics of one RK stage:
//   Compute_Advec_Cori1 / _Poles (src/headers/dyn/thor_adv_cor.h:51-362),
//   Compute_Advec_Cori2 (:366-536) and Compute_Temperature_H_Pt_Geff
//   (src/headers/dyn/thor_auxiliary.h:55-309, calcT = true).
// The cartesian velocity v of the reference is recomputed where it is used instead of stored.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kColBlock) adv_temp_kernel(Geometry g, Phys P, State s) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int     Np = g.Np, nv = g.nv;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    const double  A = P.A, Omega = P.Omega;

    int nb[7];
    nb[0] = c;
    for (int j = 0; j < 6; j++)
        nb[j + 1] = g.nb[j * Np + c];
    double dv[21];
    for (int q = 0; q < 21; q++)
        dv[q] = g.div[q * Np + c];
    double fr[7][3];
    for (int j = 0; j < 7; j++)
        for (int k = 0; k < 3; k++)
            fr[j][k] = gz(g.func_r + k * Np, nb[j]);

    // own-column velocity at a level: v = M/rho + (w/rho) r
    auto vown = [&](int lev, double* v) {
        double rho = s.Rhok[lev * Np + c], w = s.Wk[lev * Np + c];
        for (int k = 0; k < 3; k++)
            v[k] = s.Mhk[(k * nv + lev) * Np + c] / rho + (w / rho) * fr[0][k];
    };

    double vprev[3] = {0, 0, 0}, vcur[3], vnext[3] = {0, 0, 0};
    vown(0, vcur);
    for (int lev = 0; lev < nv; lev++) {
        const double rscale = rscale_of(P, g, lev);
        // horizontal flux divergence of v (x) M over the 7-point stencil
        double M[7][3], V[7][3];
        for (int j = 0; j < 7; j++) {
            int id = nb[j];
            if (id >= 0) {
                double rho = s.Rhok[lev * Np + id], w = s.Wk[lev * Np + id];
                for (int k = 0; k < 3; k++) {
                    M[j][k] = s.Mhk[(k * nv + lev) * Np + id];
                    V[j][k] = M[j][k] / rho + (w / rho) * fr[j][k];
                }
            }
            else {
                for (int k = 0; k < 3; k++)
                    M[j][k] = V[j][k] = 0.0;
            }
        }
        double nflx[3] = {0.0, 0.0, 0.0};
        for (int kk = 0; kk < 3; kk++)
            for (int cc = 0; cc < 3; cc++) {
                double sum = dv[kk] * V[0][cc] * M[0][kk];
                for (int j = 1; j < 7; j++)
                    sum = sum + dv[j * 3 + kk] * V[j][cc] * M[j][kk];
                nflx[cc] += rscale * sum;
            }
        // vertical flux of v w at the interfaces + Coriolis
        if (lev < nv - 1)
            vown(lev + 1, vnext);
        const double altht = Alth[lev + 1], althl = Alth[lev], alt = Alt[lev];
        double       dvwl[3] = {0, 0, 0}, dvwt[3] = {0, 0, 0};
        if (lev > 0) {
            double xi = althl, xim = Alt[lev - 1], xip = alt;
            double intt = (xi - xip) / (xim - xip), intl = (xi - xim) / (xip - xim);
            double whl = s.Whk[lev * Np + c];
            for (int k = 0; k < 3; k++)
                dvwl[k] = (vprev[k] * intt + vcur[k] * intl) * whl;
        }
        if (lev < nv - 1) {
            double xi = altht, xim = alt, xip = Alt[lev + 1];
            double intt = (xi - xip) / (xim - xip), intl = (xi - xim) / (xip - xim);
            double wht = s.Whk[(lev + 1) * Np + c];
            for (int k = 0; k < 3; k++)
                dvwt[k] = (vcur[k] * intt + vnext[k] * intl) * wht;
        }
        double r2p = 1.0, r2m = 1.0, r2l = 1.0;
        if (P.DeepModel) {
            r2p = pow(altht + A, 2.0);
            r2m = pow(alt + A, 2.0);
            r2l = pow(althl + A, 2.0);
        }
        const double dz  = 1.0 / ((althl - altht) * r2m);
        const double rho = s.Rhok[lev * Np + c];
        double       C[3];
        if (P.DeepModel) {
            C[0] = -2.0 * Omega * vcur[1] * rho;
            C[1] = 2.0 * Omega * vcur[0] * rho;
            C[2] = 0.0;
        }
        else {
            const double* f = fr[0];
            C[0] = 2 * Omega * (vcur[2] * f[2] * f[1] - vcur[1] * pow(f[2], 2)) * rho;
            C[1] = -2 * Omega * (vcur[2] * f[2] * f[0] - vcur[0] * pow(f[2], 2)) * rho;
            C[2] = 2 * Omega * (vcur[1] * f[2] * f[0] - vcur[0] * f[2] * f[1]) * rho;
        }
        for (int k = 0; k < 3; k++) {
            double dav                          = (dvwl[k] * r2l - dvwt[k] * r2p) * dz;
            s.Adv[(k * nv + lev) * Np + c] = nflx[k] + (dav + C[k]);
        }
        for (int k = 0; k < 3; k++) {
            vprev[k] = vcur[k];
            vcur[k]  = vnext[k];
        }
    }

    // ---- Compute_Temperature_H_Pt_Geff: column recurrence over levels 0..nv ----
    const bool   eeq = P.energy, ghv = P.GravHeightVar;
    const double P_Ref = P.P_Ref, Gravit = P.Gravit;
    double       rho = 0, rhoh, rhol = 0, rhop, pressure = 0, h_ = 0, hl = 0, pt_ = 0, ptl = 0,
           pl = 0, pp, dpdz, ep = 0, epl = 0, ek = 0, ekl = 0, gtilh_ = 0, gtilht, dz, dp_dz, Cv,
           CvoCp, xi, xim, xip, intt, intl, extr, alt = 0, altl = 0, alth = 0, altht = 0;
    const double* Pk = s.pk;
    const double* Rk = s.Rhok;
    for (int lev = 0; lev < nv + 1; lev++) {
        if (lev < nv) {
            const int i = lev * Np + c;
            Cv          = s.Cp[i] - s.Rd[i];
            CvoCp       = Cv / s.Cp[i];
            if (lev > 0) {
                pl   = pressure;
                rhol = rho;
                hl   = h_;
                if (eeq) {
                    epl = ep;
                    ekl = ek;
                }
                else
                    ptl = pt_;
                altl = alt;
            }
            pressure           = Pk[i];
            rho                = Rk[i];
            double temperature = pressure / (rho * s.Rd[i]);
            s.T[i]             = temperature;
            alt                = Alt[lev];
            alth               = Alth[lev];
            altht              = Alth[lev + 1];
            h_                 = Cv * temperature + pressure / rho;
            s.h[i]             = h_;
            if (eeq) {
                if (ghv)
                    ep = Gravit * pow(A / (A + Alt[lev]), 2) * Alt[lev];
                else
                    ep = Gravit * Alt[lev];
                s.ep[i] = ep;
                double m0 = s.Mhk[(0 * nv + lev) * Np + c], m1 = s.Mhk[(1 * nv + lev) * Np + c],
                       m2 = s.Mhk[(2 * nv + lev) * Np + c], w = s.Wk[i];
                ek = 0.5 * (m0 * m0 + m1 * m1 + m2 * m2 + w * w) / (Rk[i] * Rk[i]);
                s.ek[i]     = ek;
                s.Etotal[i] = Rk[i] * (ep + ek) + Cv / s.Rd[i] * pressure;
            }
            else {
                pt_     = (P_Ref / (s.Rd[i] * rho)) * pow(pressure / P_Ref, CvoCp);
                s.pt[i] = pt_;
            }
        }
        if (lev == 0) {
            extr     = (-alt - Alt[lev + 1]) / (Alt[lev + 1] - alt);
            s.hh[c]  = h_;
            if (ghv)
                pl = Pk[Np + c] - rho * Gravit * pow(A / (A + Alt[0]), 2) * (-alt - Alt[1]);
            else
                pl = Pk[Np + c] - rho * Gravit * (-alt - Alt[1]);
            rhol       = Rk[Np + c] + (Rk[Np + c] - rho) * extr;
            rhoh       = 0.5 * (rho + rhol);
            dz         = 2.0 * Alt[0];
            dpdz       = (Pk[c] - pl) / dz;
            s.gtilh[c] = -(1.0 / rhoh) * dpdz;
            gtilh_     = 0.0;
        }
        else if (lev == nv) {
            const int top = (nv - 1) * Np + c, top2 = (nv - 2) * Np + c;
            extr  = (2 * Alth[nv] - alt - Alt[nv - 2]) / (Alt[nv - 1] - Alt[nv - 2]);
            Cv    = s.Cp[top] - s.Rd[top];
            CvoCp = Cv / s.Cp[top];
            s.hh[nv * Np + c] = h_;
            if (ghv)
                pp = Pk[top2] - rho * Gravit * pow(A / (A + Alt[lev]), 2)
                                    * (2 * Alth[nv] - alt - Alt[nv - 2]);
            else
                pp = Pk[top2] - rho * Gravit * (2 * Alth[nv] - alt - Alt[nv - 2]);
            if (pp < 0)
                pp = 0;
            rhop = Rk[top2] + (Rk[top] - Rk[top2]) * extr;
            rhoh = 0.5 * (rho + rhop);
            if (eeq) {
                if (ghv) {
                    s.eph[nv * Np + c] = Gravit * pow(A / (A + Alth[nv]), 2) * Alth[nv];
                    s.eph[c]           = Gravit * pow(A / (A + Alth[0]), 2) * Alth[0];
                }
                else {
                    s.eph[nv * Np + c] = Gravit * Alth[nv];
                    s.eph[c]           = Gravit * Alth[0];
                }
                s.ekh[nv * Np + c] = s.ek[top2] + (s.ek[top] - s.ek[top2]) * extr;
                s.ekh[c] = s.ek[Np + c] + (s.ek[Np + c] - s.ek[c]) * (Alth[0] - Alt[1]) / (Alt[1] - Alt[0]);
            }
            else {
                s.pth[nv * Np + c] = s.pt[top2] + (s.pt[top] - s.pt[top2]) * extr;
                s.pth[c] = s.pt[Np + c] + (s.pt[Np + c] - s.pt[c]) * (Alth[0] - Alt[1]) / (Alt[1] - Alt[0]);
            }
            dz = 2.0 * (Alth[nv] - Alt[nv - 1]);
            if (ghv)
                pp = Pk[top2] - Rk[top] * Gravit * pow(A / (A + Alt[nv - 1]), 2)
                                    * (2 * Alth[nv] - Alt[nv - 1] - Alt[nv - 2]);
            else
                pp = Pk[top2] - Rk[top] * Gravit * (2 * Alth[nv] - Alt[nv - 1] - Alt[nv - 2]);
            dpdz                = (pp - Pk[top]) / dz;
            s.gtilh[nv * Np + c] = -(1.0 / rhoh) * dpdz;
            gtilht              = 0.0;
            xi                  = alt;
            xim                 = alth;
            xip                 = altht;
            intt                = (xi - xip) / (xim - xip);
            intl                = (xi - xim) / (xip - xim);
            s.gtil[top]         = gtilh_ * intt + gtilht * intl;
        }
        else {
            dz    = alt - altl;
            dp_dz = (pressure - pl) / dz;
            xi    = alth;
            xim   = altl;
            xip   = alt;
            intt  = (xi - xip) / (xim - xip);
            intl  = (xi - xim) / (xip - xim);
            s.hh[lev * Np + c] = hl * intt + h_ * intl;
            if (eeq) {
                s.eph[lev * Np + c] = epl * intt + ep * intl;
                s.ekh[lev * Np + c] = ekl * intt + ek * intl;
            }
            else
                s.pth[lev * Np + c] = ptl * intt + pt_ * intl;
            rhoh   = rhol * intt + rho * intl;
            gtilht = -(s.Whk[lev * Np + c] / rhoh) * dp_dz;
            xi     = alt;
            xim    = alth;
            xip    = altht;
            intt   = (xi - xip) / (xim - xip);
            intl   = (xi - xim) / (xip - xim);
            s.gtil[(lev - 1) * Np + c] = gtilh_ * intt + gtilht * intl;
            gtilh_                     = gtilht;
            s.gtilh[lev * Np + c]      = -(1.0 / rhoh) * dp_dz;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Geometry of the FV Laplacian / divergence damping of one column, held in registers.
// ---------------------------------------------------------------------------------------------
struct RingGeo {
    double ar[18], at[6], ti[18], te[18], oa[18];
    int    ring[6];
    int    n;
    bool   pole;
};

__device__ __forceinline__ void load_ring_geo(const Geometry& g, int c, RingGeo& r) {
    const int Np = g.Np;
    for (int q = 0; q < 18; q++) {
        r.ar[q] = g.areas[q * Np + c];
        r.ti[q] = g.nvecti[q * Np + c];
        r.te[q] = g.nvecte[q * Np + c];
        r.oa[q] = g.nvecoa[q * Np + c];
    }
    for (int j = 0; j < 6; j++) {
        r.at[j]   = g.areasTr[j * Np + c];
        r.ring[j] = g.ring[j * Np + c];
    }
    uint8_t f = g.cflag[c];
    r.n       = (f & kRing5) ? 5 : 6;
    r.pole    = (f & kPole) != 0;
}

// One FV Laplacian (Diffusion_Op, src/headers/dyn/thor_diff.h:306-451; the pole kernel :735-820
// is the same sequence with a five-entry ring).
__device__ __forceinline__ double laplacian(const RingGeo& r, const double* a, double a0,
                                            double rscale) {
    const int n   = r.n;
    double    lap = 0.0;
    double    lap1 = 0, lap2 = 0, lap3 = 0, lapx1 = 0, lapx2 = 0, lapy1 = 0, lapy2 = 0, lapz1 = 0,
           lapz2 = 0, AT1 = 0;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        if (j >= n)
            break;
        const int    jp1 = (j + 1 == n) ? 0 : j + 1;
        const int    jp2 = (jp1 + 1 == n) ? 0 : jp1 + 1;
        const double p1 = a[j], p2 = a[jp1], p3 = a[jp2];
        const double vdiff = 0.5 * rscale;
        double       astar;
        if (j == 0) {
            AT1   = rscale / r.at[j];
            astar = (r.ar[j * 3 + 0] * a0 + r.ar[j * 3 + 1] * p1 + r.ar[j * 3 + 2] * p2) / r.at[j];
            lap1  = (0.5 * (p1 + a0) - astar);
            lap2  = (0.5 * (p1 + p2) - astar);
            lap3  = (0.5 * (a0 + p2) - astar);
        }
        const double AT2 = rscale / r.at[jp1];
        astar = (r.ar[jp1 * 3 + 0] * a0 + r.ar[jp1 * 3 + 1] * p2 + r.ar[jp1 * 3 + 2] * p3) / r.at[jp1];
        const double lap4 = (0.5 * (a0 + p2) - astar);
        const double lap5 = (0.5 * (p2 + p3) - astar);
        const double lap6 = (0.5 * (a0 + p3) - astar);
        if (j == 0) {
            lapx1 = (-lap1 * r.ti[j * 3 + 0] + lap2 * r.te[j * 3 + 0] + lap3 * r.ti[jp1 * 3 + 0]) * AT1;
            lapy1 = (-lap1 * r.ti[j * 3 + 1] + lap2 * r.te[j * 3 + 1] + lap3 * r.ti[jp1 * 3 + 1]) * AT1;
            lapz1 = (-lap1 * r.ti[j * 3 + 2] + lap2 * r.te[j * 3 + 2] + lap3 * r.ti[jp1 * 3 + 2]) * AT1;
        }
        else {
            lapx1 = lapx2;
            lapy1 = lapy2;
            lapz1 = lapz2;
        }
        lapx2 = (-lap4 * r.ti[jp1 * 3 + 0] + lap5 * r.te[jp1 * 3 + 0] + lap6 * r.ti[jp2 * 3 + 0]) * AT2;
        lapy2 = (-lap4 * r.ti[jp1 * 3 + 1] + lap5 * r.te[jp1 * 3 + 1] + lap6 * r.ti[jp2 * 3 + 1]) * AT2;
        lapz2 = (-lap4 * r.ti[jp1 * 3 + 2] + lap5 * r.te[jp1 * 3 + 2] + lap6 * r.ti[jp2 * 3 + 2]) * AT2;
        lap += ((lapx1 + lapx2) * r.oa[j * 3 + 0] + (lapy1 + lapy2) * r.oa[j * 3 + 1]
                + (lapz1 + lapz2) * r.oa[j * 3 + 2])
               * vdiff;
    }
    return lap;
}

// ---------------------------------------------------------------------------------------------
// Hyperdiffusion pass: Diffusion_Op + Diffusion_Op_Poles (src/headers/dyn/thor_diff.h:54-880)
// on the six variables rho, v(3), w, Rd T (or Cv T), without the diffusive sponge; the final pass
// applies Correct_Horizontal (:882-915) to the momentum result.
//   first pass  (stepnum 0): argument = the fields                     -> diff planes (6)
//   middle pass           : argument = diff of the previous pass       -> diff planes (6)
//   final pass (last)     : argument = diff (rho-weighted for v, w, T), scaled by -Kdh4 (-1)^(o/2)
//                            -> diffrh, diffmh(3), diffw, diffpr
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kStenBlock)
    diffusion_kernel(Geometry g, Phys P, State s, const double* __restrict__ diff_in,
                     double* __restrict__ diff_out, int stepnum, bool last) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int Np = g.Np, nv = g.nv;
    const int lev0 = blockIdx.y * kLevChunk;
    const int lev1 = min(lev0 + kLevChunk, nv);
    RingGeo   r;
    load_ring_geo(g, c, r);
    double fr[3];
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    const bool eeq = P.energy;

    for (int lev = lev0; lev < lev1; lev++) {
        const double rscale = rscale_of(P, g, lev);
        const double sdiff  = -g.Kdh4[lev] * pow(-1.0, P.HyDiffOrder / 2);
        double       rho_r[6], rho0 = s.Rhok[lev * Np + c];
        for (int j = 0; j < r.n; j++)
            rho_r[j] = gz(s.Rhok + lev * Np, r.ring[j]);
        double out[6];
        for (int var = 0; var < 6; var++) {
            // argument of the Laplacian at a column id (hole -> 0) with density rho
            auto arg = [&](int id, double rho) -> double {
                if (id < 0)
                    return 0.0;
                const int i = lev * Np + id;
                double    x;
                if (stepnum == 0) {
                    if (var == 0)
                        x = s.Rhok[i];
                    else if (var <= 3)
                        x = s.Mhk[((var - 1) * nv + lev) * Np + id];
                    else if (var == 4)
                        x = s.Wk[i];
                    else
                        x = eeq ? (s.Cp[i] - s.Rd[i]) * s.T[i] : s.Rd[i] * s.T[i];
                    if (var >= 1 && var <= 4)
                        x = x / rho;
                }
                else if (last)
                    x = (var == 0) ? diff_in[(var * nv + lev) * Np + id]
                                   : diff_in[(var * nv + lev) * Np + id] * rho;
                else
                    x = diff_in[(var * nv + lev) * Np + id];
                return x;
            };
            double a[6];
            for (int j = 0; j < r.n; j++)
                a[j] = arg(r.ring[j], rho_r[j]);
            double lap = laplacian(r, a, arg(c, rho0), rscale);
            if (last)
                lap *= sdiff;
            out[var] = lap;
        }
        const int i = lev * Np + c;
        if (last) {
            s.diffrh[i] = out[0];
            // Correct_Horizontal: remove the radial component of the momentum diffusion
            double dmhr = fr[0] * out[1] + fr[1] * out[2] + fr[2] * out[3];
            for (int k = 0; k < 3; k++)
                s.diffmh[(k * nv + lev) * Np + c] = out[1 + k] + -fr[k] * dmhr;
            s.diffw[i]  = out[4];
            s.diffpr[i] = out[5];
        }
        else {
            for (int var = 0; var < 6; var++)
                diff_out[(var * nv + lev) * Np + c] = out[var];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Divergence damping (DivM_Op / DivM_Op_Poles, src/headers/dyn/thor_div.h:49-535).
// Pass 0: grad of the 3D divergence of (Mh, Wh) -> divg; pass 1 (divm_final): the tangential
// part of grad(div) of divg scaled by -Kdhz. The poles' corner mean of w uses the second
// sub-area in place of the third (thor_div.h:443-454), restated as it is.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void divm_core(const RingGeo& r, const double* a0, const double (*ar)[3],
                                          bool with_w, double wl0, double wt0, const double* wl,
                                          const double* wt, double dz, double rscale,
                                          double* lapo) {
    const int n   = r.n;
    double    AT0 = 0.5 * rscale;
    double    lapx = 0.0, lapy = 0.0, lapz = 0.0;
    double    a01x = 0, a01y = 0, a01z = 0, a12x = 0, a12y = 0, a12z = 0, AT1 = 0, lap1 = 0,
           lap2 = 0;
    const int c2 = r.pole ? 1 : 2;
#pragma unroll
    for (int j = 0; j < 6; j++) {
        if (j >= n)
            break;
        const int     jp1 = (j + 1 == n) ? 0 : j + 1;
        const int     jp2 = (jp1 + 1 == n) ? 0 : jp1 + 1;
        const double *p1 = ar[j], *p2 = ar[jp1], *p3 = ar[jp2];
        double        dwdz = 0.0, dwdz2 = 0.0;
        if (with_w) {
            double meanwl  = (r.ar[j * 3 + 0] * wl0 + r.ar[j * 3 + 1] * wl[j] + r.ar[j * 3 + c2] * wl[jp1]) / r.at[j];
            double meanwt  = (r.ar[j * 3 + 0] * wt0 + r.ar[j * 3 + 1] * wt[j] + r.ar[j * 3 + c2] * wt[jp1]) / r.at[j];
            double meanwl2 = (r.ar[jp1 * 3 + 0] * wl0 + r.ar[jp1 * 3 + 1] * wl[jp1] + r.ar[jp1 * 3 + c2] * wl[jp2]) / r.at[jp1];
            double meanwt2 = (r.ar[jp1 * 3 + 0] * wt0 + r.ar[jp1 * 3 + 1] * wt[jp1] + r.ar[jp1 * 3 + c2] * wt[jp2]) / r.at[jp1];
            dwdz           = (meanwl - meanwt) * dz;
            dwdz2          = (meanwl2 - meanwt2) * dz;
        }
        if (j == 0) {
            a01x = (a0[0] + p1[0]);
            a01y = (a0[1] + p1[1]);
            a01z = (a0[2] + p1[2]);
            a12x = (p1[0] + p2[0]);
            a12y = (p1[1] + p2[1]);
            a12z = (p1[2] + p2[2]);
            AT1  = 0.5 * rscale / r.at[j];
        }
        const double AT2  = 0.5 * rscale / r.at[jp1];
        const double a02x = (a0[0] + p2[0]), a02y = (a0[1] + p2[1]), a02z = (a0[2] + p2[2]);
        const double a23x = (p2[0] + p3[0]), a23y = (p2[1] + p3[1]), a23z = (p2[2] + p3[2]);
        const double a03x = (a0[0] + p3[0]), a03y = (a0[1] + p3[1]), a03z = (a0[2] + p3[2]);
        const double* ti = r.ti;
        const double* te = r.te;
        if (j == 0)
            lap1 = (-a01x * ti[j * 3 + 0] - a01y * ti[j * 3 + 1] - a01z * ti[j * 3 + 2]
                    + a12x * te[j * 3 + 0] + a12y * te[j * 3 + 1] + a12z * te[j * 3 + 2]
                    + a02x * ti[jp1 * 3 + 0] + a02y * ti[jp1 * 3 + 1] + a02z * ti[jp1 * 3 + 2])
                   * AT1;
        else
            lap1 = lap2;
        lap2 = (-a02x * ti[jp1 * 3 + 0] - a02y * ti[jp1 * 3 + 1] - a02z * ti[jp1 * 3 + 2]
                + a23x * te[jp1 * 3 + 0] + a23y * te[jp1 * 3 + 1] + a23z * te[jp1 * 3 + 2]
                + a03x * ti[jp2 * 3 + 0] + a03y * ti[jp2 * 3 + 1] + a03z * ti[jp2 * 3 + 2])
               * AT2;
        lapx += (lap1 + dwdz + lap2 + dwdz2) * r.oa[j * 3 + 0] * AT0;
        lapy += (lap1 + dwdz + lap2 + dwdz2) * r.oa[j * 3 + 1] * AT0;
        lapz += (lap1 + dwdz + lap2 + dwdz2) * r.oa[j * 3 + 2] * AT0;
    }
    lapo[0] = lapx;
    lapo[1] = lapy;
    lapo[2] = lapz;
}

// Pass 0 of the divergence damping on (Mh, Wh) -> divg.
__global__ void __launch_bounds__(kStenBlock)
    divm0_kernel(Geometry g, Phys P, const double* __restrict__ Mh, const double* __restrict__ Wh,
                 double* __restrict__ divg) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int Np = g.Np, nv = g.nv;
    const int lev0 = blockIdx.y * kLevChunk;
    const int lev1 = min(lev0 + kLevChunk, nv);
    RingGeo   r;
    load_ring_geo(g, c, r);
    for (int lev = lev0; lev < lev1; lev++) {
        const double rscale = rscale_of(P, g, lev);
        const double dz     = 1.0 / (g.Altitudeh[lev] - g.Altitudeh[lev + 1]);
        double       a0[3], ar[6][3], wl[6], wt[6];
        for (int k = 0; k < 3; k++)
            a0[k] = Mh[(k * nv + lev) * Np + c];
        for (int j = 0; j < r.n; j++) {
            for (int k = 0; k < 3; k++)
                ar[j][k] = gz(Mh + (k * nv + lev) * Np, r.ring[j]);
            wl[j] = gz(Wh + lev * Np, r.ring[j]);
            wt[j] = gz(Wh + (lev + 1) * Np, r.ring[j]);
        }
        double out[3];
        divm_core(r, a0, ar, true, Wh[lev * Np + c], Wh[(lev + 1) * Np + c], wl, wt, dz, rscale,
                  out);
        for (int k = 0; k < 3; k++)
            divg[(k * nv + lev) * Np + c] = out[k];
    }
}

// Pass 1 of the divergence damping at (column, level): DivM from divg.
__device__ __forceinline__ void divm_final(const Geometry& g, const Phys& P, const RingGeo& r,
                                           const double* __restrict__ divg, int c, int lev,
                                           const double* fr, double* DivM) {
    const int Np = g.Np, nv = g.nv;
    double    a0[3], ar[6][3];
    for (int k = 0; k < 3; k++)
        a0[k] = divg[(k * nv + lev) * Np + c];
    for (int j = 0; j < r.n; j++)
        for (int k = 0; k < 3; k++)
            ar[j][k] = gz(divg + (k * nv + lev) * Np, r.ring[j]);
    double lap[3];
    divm_core(r, a0, ar, false, 0, 0, nullptr, nullptr, 0, rscale_of(P, g, lev), lap);
    const double sdiff = g.Kdhz[lev];
    const double lapr  = fr[0] * lap[0] + fr[1] * lap[1] + fr[2] * lap[2];
    for (int k = 0; k < 3; k++) {
        double l = lap[k] - fr[k] * lapr;
        DivM[k]  = -l * sdiff;
    }
}

// ---------------------------------------------------------------------------------------------
// Slow modes of one RK stage: divergence-damping pass 1 on (Mhk, Whk) + Compute_Slow_Modes /
// _Poles (src/headers/dyn/thor_slowmodes.h:48-683) + UpdateRK
// (src/headers/dyn/thor_auxiliary.h:311-418, without module arrays and without the never-read
// Ws). DivM is consumed where it is produced and not stored.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kStenBlock)
    slow_modes_kernel(Geometry g, Phys P, State s, bool update_rk) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int Np = g.Np, nv = g.nv;
    const int lev0 = blockIdx.y * kLevChunk;
    const int lev1 = min(lev0 + kLevChunk, nv);
    const double A = P.A, Gravit = P.Gravit;
    int          nb[7];
    nb[0] = c;
    for (int j = 0; j < 6; j++)
        nb[j + 1] = g.nb[j * Np + c];
    double dv[21], gr[21], fr[3];
    for (int q = 0; q < 21; q++) {
        dv[q] = g.div[q * Np + c];
        gr[q] = g.grad[q * Np + c];
    }
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    const bool pole = (g.cflag[c] & kPole) != 0;
    RingGeo    r;
    if (P.DivDampP)
        load_ring_geo(g, c, r);

    for (int lev = lev0; lev < lev1; lev++) {
        const int i = lev * Np + c;
        double    DivM[3] = {0.0, 0.0, 0.0};
        if (P.DivDampP)
            divm_final(g, P, r, s.divg, c, lev, fr, DivM);

        const double Cv = s.Cp[i] - s.Rd[i];
        double       adv[3];
        for (int k = 0; k < 3; k++)
            adv[k] = s.Adv[(k * nv + lev) * Np + c];
        const double rho = s.Rhok[i];
        double       rhol = 0, altl = 0, pressurel = 0, advrl = 0;
        if (lev != 0) {
            advrl = s.Adv[(0 * nv + lev - 1) * Np + c] * fr[0] + s.Adv[(1 * nv + lev - 1) * Np + c] * fr[1]
                    + s.Adv[(2 * nv + lev - 1) * Np + c] * fr[2];
            rhol      = s.Rhok[i - Np];
            altl      = g.Altitude[lev - 1];
            pressurel = s.pk[i - Np];
        }
        double advr = adv[0] * fr[0] + adv[1] * fr[1] + adv[2] * fr[2];
        for (int k = 0; k < 3; k++)
            adv[k] += -advr * fr[k];
        const double altht = g.Altitudeh[lev + 1], althl = g.Altitudeh[lev], alt = g.Altitude[lev];
        double       M0[3];
        for (int k = 0; k < 3; k++)
            M0[k] = s.Mhk[(k * nv + lev) * Np + c];
        if (!P.NonHydro) {
            advr = (pow(M0[0], 2) + pow(M0[1], 2) + pow(M0[2], 2)) / (rho * (alt + A));
            if (lev != 0)
                advrl = (pow(s.Mhk[(0 * nv + lev - 1) * Np + c], 2) + pow(s.Mhk[(1 * nv + lev - 1) * Np + c], 2)
                         + pow(s.Mhk[(2 * nv + lev - 1) * Np + c], 2))
                        / (rhol * (altl + A));
        }
        const double dz = altht - althl;
        double       r2p, r2m, r2l, rscale, dr2dz;
        if (P.DeepModel) {
            r2p    = pow(altht + A, 2.0);
            r2m    = pow(alt + A, 2.0);
            r2l    = pow(althl + A, 2.0);
            rscale = A / (alt + A);
            dr2dz  = (pow(altht + A, 3.0) - pow(althl + A, 3.0)) / 3;
        }
        else {
            r2p = r2m = r2l = rscale = 1.0;
            dr2dz                    = r2m * dz;
        }
        // horizontal stencils at this level
        double pv[7], hv[7], Mv[7][3];
        for (int j = 0; j < 7; j++) {
            pv[j] = gz(s.pk + lev * Np, nb[j]);
            hv[j] = gz(s.h + lev * Np, nb[j]);
            for (int k = 0; k < 3; k++)
                Mv[j][k] = gz(s.Mhk + (k * nv + lev) * Np, nb[j]);
        }
        double nflxv[3], nflxr = 0.0, nflxp = 0.0;
        for (int k = 0; k < 3; k++) {
            double sg = gr[k] * pv[0], sd = dv[k] * Mv[0][k], sp = dv[k] * Mv[0][k] * hv[0];
            for (int j = 1; j < 7; j++) {
                sg = sg + gr[j * 3 + k] * pv[j];
                sd = sd + dv[j * 3 + k] * Mv[j][k];
                sp = sp + dv[j * 3 + k] * Mv[j][k] * hv[j];
            }
            nflxv[k] = rscale * sg;
            nflxr += rscale * sd;
            nflxp += rscale * sp;
        }
        double whl, wht, hhl, hht;
        if (lev == 0) {
            whl = 0.0;
            wht = s.Whk[(lev + 1) * Np + c];
            hhl = 0.0;
            hht = s.hh[(lev + 1) * Np + c];
        }
        else {
            whl = s.Whk[lev * Np + c];
            wht = s.Whk[(lev + 1) * Np + c];
            hhl = s.hh[lev * Np + c];
            hht = s.hh[(lev + 1) * Np + c];
        }
        const double dwdz  = pole ? (wht * r2p - whl * r2l) / (dz * r2m) : (wht * r2p - whl * r2l) / (dr2dz);
        const double dwhdz = (wht * r2p * hht - whl * r2l * hhl) / (dz * r2m);
        const double dpr   = nflxv[0] * fr[0] + nflxv[1] * fr[1] + nflxv[2] * fr[2];
        for (int k = 0; k < 3; k++) {
            const int j = (k * nv + lev) * Np + c;
            s.SlowMh[j] = -(nflxv[k] - dpr * fr[k]) - adv[k] + DivM[k] + s.diffmh[j] + s.dMh[j];
        }
        if (lev == 0) {
            s.SlowWh[c]           = 0.0;
            s.SlowWh[nv * Np + c] = 0.0;
        }
        else {
            double xi = althl, xim = altl, xip = alt;
            double intt = (xi - xip) / (xim - xip), intl = (xi - xim) / (xip - xim);
            double swr;
            if (P.DeepModel) {
                if (P.GravHeightVar)
                    swr = (advrl + rhol * Gravit * pow(A / (A + altl), 2)) * intt
                          + (advr + rho * Gravit * pow(A / (A + alt), 2)) * intl;
                else
                    swr = (advrl + rhol * Gravit) * intt + (advr + rho * Gravit) * intl;
            }
            else {
                if (P.GravHeightVar)
                    swr = (rhol * Gravit * pow(A / (A + altl), 2)) * intt
                          + (rho * Gravit * pow(A / (A + alt), 2)) * intl;
                else
                    swr = (rhol * Gravit) * intt + (rho * Gravit) * intl;
            }
            if (P.NonHydro)
                swr += (-s.diffw[i - Np]) * intt + (-s.diffw[i]) * intl;
            const double dz2  = alt - altl;
            const double dpdz = (pv[0] - pressurel) / dz2;
            swr += dpdz;
            swr -= s.dWh[lev * Np + c];
            s.SlowWh[lev * Np + c] = -swr;
        }
        nflxr += dwdz;
        s.SlowRho[i]   = -nflxr + s.diffrh[i];
        const double r_ = 1.0 / rho;
        const double vgp = (nflxv[0] - dpr * fr[0]) * M0[0] * r_ + (nflxv[1] - dpr * fr[1]) * M0[1] * r_
                           + (nflxv[2] - dpr * fr[2]) * M0[2] * r_;
        double sp = (s.Rd[i] / Cv) * (-nflxp - s.gtil[i] - dwhdz + vgp + s.Qheat[i]);
        if (P.energy)
            sp += s.Rd[i] / Cv * (s.diffpr[i]);
        else
            sp += s.diffpr[i];
        s.Slowp[i] = sp;

        if (update_rk) {
            // deviations from the start of the large step
            double Mx = s.Mh[(0 * nv + lev) * Np + c] - M0[0];
            double My = s.Mh[(1 * nv + lev) * Np + c] - M0[1];
            double Mz = s.Mh[(2 * nv + lev) * Np + c] - M0[2];
            double aux = Mx * fr[0] + My * fr[1] + Mz * fr[2];
            s.Mhs[(0 * nv + lev) * Np + c] = Mx - aux * fr[0];
            s.Mhs[(1 * nv + lev) * Np + c] = My - aux * fr[1];
            s.Mhs[(2 * nv + lev) * Np + c] = Mz - aux * fr[2];
            s.Rhos[i]                      = s.Rho[i] - rho;
            s.ps[i]                        = s.p[i] - s.pk[i];
            s.Whs[lev * Np + c] = (lev == 0) ? 0.0 : s.Wh[lev * Np + c] - s.Whk[lev * Np + c];
            if (lev == nv - 1)
                s.Whs[nv * Np + c] = 0.0;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Small step, horizontal momentum: divergence-damping pass 1 on the deviations (Mhs, Whs) +
// Momentum_Eq / _Poles (src/headers/dyn/thor_fastmodes.h:54-253).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kStenBlock)
    momentum_kernel(Geometry g, Phys P, State s, double dt) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int Np = g.Np, nv = g.nv;
    const int lev0 = blockIdx.y * kLevChunk;
    const int lev1 = min(lev0 + kLevChunk, nv);
    int       nb[7];
    nb[0] = c;
    for (int j = 0; j < 6; j++)
        nb[j + 1] = g.nb[j * Np + c];
    double gr[21], fr[3];
    for (int q = 0; q < 21; q++)
        gr[q] = g.grad[q * Np + c];
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    RingGeo r;
    if (P.DivDampP)
        load_ring_geo(g, c, r);
    for (int lev = lev0; lev < lev1; lev++) {
        double DivM[3] = {0.0, 0.0, 0.0};
        if (P.DivDampP)
            divm_final(g, P, r, s.divg, c, lev, fr, DivM);
        const double rscale = rscale_of(P, g, lev);
        double       pv[7];
        for (int j = 0; j < 7; j++)
            pv[j] = gz(s.ps + lev * Np, nb[j]);
        double Mv[3];
        for (int k = 0; k < 3; k++) {
            double sg = gr[k] * pv[0];
            for (int j = 1; j < 7; j++)
                sg = sg + gr[j * 3 + k] * pv[j];
            double nflxv = rscale * sg;
            Mv[k]        = (-nflxv + s.SlowMh[(k * nv + lev) * Np + c] + DivM[k]) * dt;
        }
        const double vr = Mv[0] * fr[0] + Mv[1] * fr[1] + Mv[2] * fr[2];
        for (int k = 0; k < 3; k++) {
            Mv[k] += -vr * fr[k];
            s.Mhs[(k * nv + lev) * Np + c] += Mv[k];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Small step, vertically implicit part, one thread per column:
//   Prepare_Implicit_Vertical / _Poles (src/headers/dyn/thor_vertical_int.h:566-771),
//   Vertical_Eq (:52-563, Thomas forward elimination and back substitution, FP64),
//   Density_Pressure_Eqs / _Poles (src/headers/dyn/thor_fastmodes.h:255-847).
// Sp and Sd are produced level by level inside the forward sweep that consumes them; the
// Thomas coefficients live in shared memory, [interface][thread]; Whs is written once and the
// density / pressure update reads it back from the same shared array.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kVertBlock) vertical_kernel(Geometry g, Phys P, State s, double deltat) {
    extern __shared__ double smem[];
    const int c  = blockIdx.x * blockDim.x + threadIdx.x;
    const int nv = g.nv, nvi = g.nvi, Np = g.Np;
    double*   cc = smem;                      // [nvi][blockDim]
    double*   dd = smem + nvi * blockDim.x;   // [nvi][blockDim]
    const int t  = threadIdx.x;
    const int B  = blockDim.x;
    if (c >= g.N)
        return;
    const double  A = P.A, Gravit = P.Gravit;
    const bool    deep = P.DeepModel, nonh = P.NonHydro, ghv = P.GravHeightVar;
    const double* Alt  = g.Altitude;
    const double* Alth = g.Altitudeh;
    int           nb[7];
    nb[0] = c;
    for (int j = 0; j < 6; j++)
        nb[j + 1] = g.nb[j * Np + c];
    double dv[21];
    for (int q = 0; q < 21; q++)
        dv[q] = g.div[q * Np + c];
    const bool pole = (g.cflag[c] & kPole) != 0;

    // Sp, Sd at one level (Prepare_Implicit_Vertical)
    auto prepare = [&](int lev, double& Sp, double& Sd) {
        const int    i      = lev * Np + c;
        const double RoC    = s.Rd[i] / (s.Cp[i] - s.Rd[i]);
        const double rscale = rscale_of(P, g, lev);
        double       hv[7], Mv[7][3];
        for (int j = 0; j < 7; j++) {
            hv[j] = gz(s.h + lev * Np, nb[j]);
            for (int k = 0; k < 3; k++)
                Mv[j][k] = gz(s.Mhs + (k * nv + lev) * Np, nb[j]);
        }
        double nflxr = 0.0, nflxp = 0.0;
        for (int k = 0; k < 3; k++) {
            double sd = dv[k] * Mv[0][k], sp = dv[k] * Mv[0][k] * hv[0];
            for (int j = 1; j < 7; j++) {
                sd = sd + dv[j * 3 + k] * Mv[j][k];
                sp = sp + dv[j * 3 + k] * Mv[j][k] * hv[j];
            }
            nflxr -= rscale * sd;
            nflxp -= (RoC)*rscale * sp;
        }
        Sp = nflxp + s.Slowp[i];
        Sd = nflxr + s.SlowRho[i];
    };

    double Spl, Sdl, Sp, Sd;
    prepare(0, Spl, Sdl);
    for (int lev = 1; lev < nv; lev++) {
        prepare(lev, Sp, Sd);
        const double altht = Alth[lev + 1], althl = Alth[lev - 1], alth = Alth[lev];
        const double alt = Alt[lev], altl = Alt[lev - 1];
        double       hp = s.hh[(lev + 1) * Np + c], h = s.hh[lev * Np + c], hm = s.hh[(lev - 1) * Np + c];
        const double gp = s.gtilh[(lev + 1) * Np + c], gg = s.gtilh[lev * Np + c], gm = s.gtilh[(lev - 1) * Np + c];
        const int    iu = lev * Np + c, il = (lev - 1) * Np + c;
        const double p = s.ps[iu], pl = s.ps[il], r = s.Rhos[iu], rl = s.Rhos[il];
        const double CRddl = (s.Cp[il] - s.Rd[il]) / (s.Rd[il] * deltat * deltat);
        const double CRddu = (s.Cp[iu] - s.Rd[iu]) / (s.Rd[iu] * deltat * deltat);
        double       GCoRl, GCoRu;
        if (ghv) {
            GCoRl = Gravit * pow(A / (A + altl), 2) * (s.Cp[il] - s.Rd[il]) / s.Rd[il];
            GCoRu = Gravit * pow(A / (A + alt), 2) * (s.Cp[iu] - s.Rd[iu]) / s.Rd[iu];
        }
        else {
            GCoRl = Gravit * (s.Cp[il] - s.Rd[il]) / s.Rd[il];
            GCoRu = Gravit * (s.Cp[iu] - s.Rd[iu]) / s.Rd[iu];
        }
        const double dzp  = 1.0 / (altht - alth);
        const double dzh  = 1.0 / (alt - altl);
        const double dzm  = 1.0 / (alth - althl);
        const double dzph = dzp * dzh;
        const double dzmh = dzm * dzh;
        double       xi, xim, xip, intl, inttm, intt, aa, bb, ccv;
        const double CRdd = (CRddl * (alt - alth) + CRddu * (alth - altl)) / (alt - altl);
        const double GCoR = (GCoRl * (alt - alth) + GCoRu * (alth - altl)) / (alt - altl);
        if (deep) {
            hp                = hp * pow(altht + A, 2);
            h                 = h * pow(alth + A, 2);
            hm                = hm * pow(althl + A, 2);
            const double or2  = 1 / pow(alth + A, 2);
            const double tor3 = 2 / pow(alth + A, 3);
            xi    = alt;
            xim   = alth;
            xip   = altht;
            intl  = (xi - xim) * dzp * dzh;
            xi    = altl;
            xim   = althl;
            xip   = alth;
            inttm = -(xi - xip) * dzm * dzh;
            ccv   = -dzph * or2 * hp - inttm * (gp + GCoR - tor3 * hp);
            if (nonh)
                bb = CRdd + (dzph + dzmh) * or2 * h + (intl - inttm) * (gg + GCoR - tor3 * h);
            else
                bb = (dzph + dzmh) * or2 * h + (intl - inttm) * (gg + GCoR - tor3 * h);
            aa = -dzmh * or2 * hm + intl * (gm + GCoR - tor3 * hm);
        }
        else {
            xi    = alt;
            xim   = alth;
            xip   = altht;
            intl  = (xi - xim) * dzp * dzh;
            xi    = altl;
            xim   = althl;
            xip   = alth;
            inttm = -(xi - xip) * dzm * dzh;
            ccv   = -dzph * hp - inttm * (gp + GCoR);
            if (nonh)
                bb = CRdd + (dzph + dzmh) * h + (intl - inttm) * (gg + GCoR);
            else
                bb = (dzph + dzmh) * h + (intl - inttm) * (gg + GCoR);
            aa = -dzmh * hm + intl * (gm + GCoR);
        }
        const double dSpdz = (Sp - Spl) * dzh;
        const double dPdz  = (p - pl) * dzh;
        xi   = alth;
        xim  = altl;
        xip  = alt;
        intt = (xi - xip) / (xim - xip);
        intl = (xi - xim) / (xip - xim);
        const double rhohs = rl * intt + r * intl;
        const double Sdh   = Sdl * intt + Sd * intl;
        const double Srh   = s.SlowWh[lev * Np + c];
        double       C0;
        if (!nonh) {
            if (ghv)
                C0 = (pow(deltat, 2.0) * dSpdz + pow(deltat, 2.0) * Gravit * pow(A / (A + alt), 2) * Sdh
                      + Gravit * pow(A / (A + alt), 2) * deltat * rhohs + deltat * dPdz - deltat * Srh)
                     * (CRdd);
            else
                C0 = (pow(deltat, 2.0) * dSpdz + pow(deltat, 2.0) * Gravit * Sdh + Gravit * deltat * rhohs
                      + deltat * dPdz - deltat * Srh)
                     * (CRdd);
        }
        else {
            const double whs = s.Whs[lev * Np + c];
            if (ghv)
                C0 = (-whs + pow(deltat, 2.0) * dSpdz + pow(deltat, 2.0) * Gravit * pow(A / (A + alt), 2) * Sdh
                      + Gravit * pow(A / (A + alt), 2) * deltat * rhohs + deltat * dPdz - deltat * Srh)
                     * (CRdd);
            else
                C0 = (-whs + pow(deltat, 2.0) * dSpdz + pow(deltat, 2.0) * Gravit * Sdh
                      + Gravit * deltat * rhohs + deltat * dPdz - deltat * Srh)
                     * (CRdd);
        }
        double ddv = -C0;
        if (lev == 1) {
            ccv = ccv / bb;
            ddv = ddv / bb;
        }
        else {
            const double tt = 1.0 / (bb - cc[(lev - 1) * B + t] * aa);
            ccv *= tt;
            ddv = (ddv - dd[(lev - 1) * B + t] * aa) * tt;
        }
        cc[lev * B + t] = ccv;
        dd[lev * B + t] = ddv;
        Spl             = Sp;
        Sdl             = Sd;
    }
    // back substitution; dd[] is overwritten with Whs
    double wnext = 0.0;
    dd[nv * B + t] = 0.0;
    for (int lev = nv - 1; lev > 0; lev--) {
        double w = (lev == nv - 1) ? dd[lev * B + t] : (-cc[lev * B + t] * wnext + dd[lev * B + t]);
        dd[lev * B + t]     = w;
        s.Whs[lev * Np + c] = w;
        wnext               = w;
    }
    dd[t]                = 0.0;
    s.Whs[c]             = 0.0;
    s.Whs[nv * Np + c]   = 0.0;

    // Density_Pressure_Eqs
    const bool   eeq = P.energy;
    const double P_Ref = P.P_Ref;
    for (int lev = 0; lev < nv; lev++) {
        const int    i     = lev * Np + c;
        const double Cv    = s.Cp[i] - s.Rd[i];
        const double altht = Alth[lev + 1], althl = Alth[lev];
        const double dz    = altht - althl;
        double       r2p, r2m, r2l, rscale, dr2dz;
        if (deep) {
            const double alt = Alt[lev];
            r2p              = pow(altht + A, 2.0);
            r2m              = pow(alt + A, 2.0);
            r2l              = pow(althl + A, 2.0);
            rscale           = A / (alt + A);
            dr2dz            = (pow(altht + A, 3.0) - pow(althl + A, 3.0)) / 3.0;
        }
        else {
            r2p = r2m = r2l = rscale = 1.0;
            dr2dz                    = r2m * dz;
        }
        double vs[7][3], v1[7][3], ptv[7];
        for (int j = 0; j < 7; j++) {
            const int id = nb[j];
            if (id >= 0) {
                for (int k = 0; k < 3; k++) {
                    vs[j][k] = s.Mhs[(k * nv + lev) * Np + id];
                    v1[j][k] = vs[j][k] + s.Mhk[(k * nv + lev) * Np + id];
                }
                const int q = lev * Np + id;
                ptv[j]      = eeq ? (s.h[q] + s.ep[q] + s.ek[q]) : s.pt[q];
            }
            else {
                for (int k = 0; k < 3; k++)
                    vs[j][k] = v1[j][k] = 0.0;
                ptv[j] = 0.0;
            }
        }
        double nflxr = 0.0, nflxpt = 0.0;
        for (int k = 0; k < 3; k++) {
            double sr = dv[k] * vs[0][k], st = dv[k] * v1[0][k] * ptv[0];
            for (int j = 1; j < 7; j++) {
                sr = sr + dv[j * 3 + k] * vs[j][k];
                st = st + dv[j * 3 + k] * v1[j][k] * ptv[j];
            }
            nflxr += rscale * sr;
            nflxpt += rscale * st;
        }
        auto phv = [&](int l) -> double {
            const int q = l * Np + c;
            return eeq ? (s.hh[q] + s.eph[q] + s.ekh[q]) : s.pth[q];
        };
        double whl, wht, whl2, wht2, phl, pht;
        if (lev == 0) {
            whl  = 0.0;
            wht  = dd[(lev + 1) * B + t];
            whl2 = 0.0;
            wht2 = dd[(lev + 1) * B + t] + s.Whk[(lev + 1) * Np + c];
            phl  = 0.0;
            pht  = phv(lev + 1);
        }
        else {
            whl  = dd[lev * B + t];
            wht  = dd[(lev + 1) * B + t];
            whl2 = dd[lev * B + t] + s.Whk[lev * Np + c];
            wht2 = dd[(lev + 1) * B + t] + s.Whk[(lev + 1) * Np + c];
            phl  = phv(lev);
            pht  = phv(lev + 1);
        }
        const double dwdz   = pole ? (wht * r2p - whl * r2l) / (dz * r2m) : (wht * r2p - whl * r2l) / (dr2dz);
        const double dwptdz = (wht2 * pht * r2p - whl2 * phl * r2l) / (dz * r2m);
        double       aux    = -(nflxpt + dwptdz) * deltat;
        const double rk_    = s.Rhok[i];
        const double r      = rk_ + s.Rhos[i];
        nflxr += dwdz;
        const double rhos_new = s.Rhos[i] + (s.SlowRho[i] - nflxr) * deltat;
        s.Rhos[i]             = rhos_new;
        if (eeq) {
            aux += s.Etotal[i] + (s.diffpr[i]) * deltat + s.Qheat[i] * deltat;
            s.Etotal[i] = aux;
            const double w = (whl2 * (Alth[lev + 1] - Alt[lev]) + wht2 * (Alt[lev] - Alth[lev]))
                             / (Alth[lev + 1] - Alth[lev]);
            double Epot_kin;
            if (P.GravHeightVar)
                Epot_kin = (rhos_new + rk_) * Gravit * pow(A / (A + Alt[lev]), 2) * Alt[lev]
                           + 0.5 * (pow(v1[0][0], 2) + pow(v1[0][1], 2) + pow(v1[0][2], 2) + pow(w, 2))
                                 / (rhos_new + rk_);
            else
                Epot_kin = (rhos_new + rk_) * Gravit * Alt[lev]
                           + 0.5 * (pow(v1[0][0], 2) + pow(v1[0][1], 2) + pow(v1[0][2], 2) + pow(w, 2))
                                 / (rhos_new + rk_);
            s.ps[i] = s.Rd[i] / Cv * (aux - Epot_kin) - s.pk[i];
        }
        else {
            const double ptc = (P_Ref / (s.Rd[i] * r)) * pow((s.ps[i] + s.pk[i]) / P_Ref, Cv / s.Cp[i]);
            aux += ptc * r;
            const double pn = P_Ref * pow(s.Rd[i] * aux / P_Ref, s.Cp[i] / Cv);
            s.ps[i] = pn - s.pk[i] + (s.diffpr[i]) * deltat + s.Rd[i] / Cv * s.Qheat[i] * deltat;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// End of an RK stage: UpdateRK2 (src/headers/dyn/thor_auxiliary.h:420-529, no module arrays).
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kColBlock) update_rk2_kernel(Geometry g, Phys P, State s) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.N)
        return;
    const int Np = g.Np, nv = g.nv;
    double    fr[3];
    for (int k = 0; k < 3; k++)
        fr[k] = g.func_r[k * Np + c];
    for (int lev = 0; lev < nv; lev++) {
        double Mx = s.Mhs[(0 * nv + lev) * Np + c] + s.Mhk[(0 * nv + lev) * Np + c];
        double My = s.Mhs[(1 * nv + lev) * Np + c] + s.Mhk[(1 * nv + lev) * Np + c];
        double Mz = s.Mhs[(2 * nv + lev) * Np + c] + s.Mhk[(2 * nv + lev) * Np + c];
        double aux = Mx * fr[0] + My * fr[1] + Mz * fr[2];
        s.Mhk[(0 * nv + lev) * Np + c] = Mx - aux * fr[0];
        s.Mhk[(1 * nv + lev) * Np + c] = My - aux * fr[1];
        s.Mhk[(2 * nv + lev) * Np + c] = Mz - aux * fr[2];
        const int i = lev * Np + c;
        s.Rhok[i] += s.Rhos[i];
        s.pk[i] += s.ps[i];
    }
    for (int lev = 0; lev < nv + 1; lev++) {
        if (lev == 0 || lev == nv)
            s.Whk[lev * Np + c] = 0.0;
        else
            s.Whk[lev * Np + c] += s.Whs[lev * Np + c];
    }
    double althl = 0, altht = g.Altitudeh[1], whl = 0.0, wht = s.Whk[Np + c];
    for (int lev = 0; lev < nv; lev++) {
        double xi = g.Altitude[lev], xim = althl, xip = altht;
        double intt = (xi - xip) / (xim - xip), intl = (xi - xim) / (xip - xim);
        s.Wk[lev * Np + c] = whl * intt + wht * intl;
        if (lev < nv - 1) {
            althl = altht;
            altht = g.Altitudeh[lev + 2];
            whl   = wht;
            wht   = s.Whk[(lev + 2) * Np + c];
        }
    }
}

inline dim3 col_grid(const Geometry& g, int block) { return dim3((g.N + block - 1) / block); }
inline dim3 sten_grid(const Geometry& g) {
    return dim3((g.N + kStenBlock - 1) / kStenBlock, (g.nv + kLevChunk - 1) / kLevChunk);
}

} // namespace

void launch_profx(const Geometry& g, const Phys& P, const State& s, cudaStream_t st) {
    profx_kernel<<<col_grid(g, kColBlock), kColBlock, 0, st>>>(g, P, s);
}
void launch_adv_temp(const Geometry& g, const Phys& P, const State& s, cudaStream_t st) {
    adv_temp_kernel<<<col_grid(g, kColBlock), kColBlock, 0, st>>>(g, P, s);
}
void launch_diffusion(const Geometry& g, const Phys& P, const State& s, int stepnum, bool last,
                      cudaStream_t st) {
    // passes alternate between the two halves of the diff buffer
    const size_t plane6 = (size_t)6 * g.nv * g.Np;
    const double* in    = s.diff + ((stepnum + 1) % 2) * plane6;
    double*       out   = s.diff + (stepnum % 2) * plane6;
    diffusion_kernel<<<sten_grid(g), kStenBlock, 0, st>>>(g, P, s, in, out, stepnum, last);
}
void launch_divm0(const Geometry& g, const Phys& P, const State& s, bool small_step,
                  cudaStream_t st) {
    divm0_kernel<<<sten_grid(g), kStenBlock, 0, st>>>(g, P, small_step ? s.Mhs : s.Mhk,
                                                      small_step ? s.Whs : s.Whk, s.divg);
}
void launch_slow_modes(const Geometry& g, const Phys& P, const State& s, bool update_rk,
                       cudaStream_t st) {
    slow_modes_kernel<<<sten_grid(g), kStenBlock, 0, st>>>(g, P, s, update_rk);
}
void launch_momentum(const Geometry& g, const Phys& P, const State& s, double dt,
                     cudaStream_t st) {
    momentum_kernel<<<sten_grid(g), kStenBlock, 0, st>>>(g, P, s, dt);
}
void launch_vertical(const Geometry& g, const Phys& P, const State& s, double dt,
                     cudaStream_t st) {
    size_t smem = (size_t)2 * g.nvi * kVertBlock * sizeof(double);
    static size_t configured = 0;
    if (smem > configured) {
        cudaFuncSetAttribute(vertical_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        configured = smem;
    }
    vertical_kernel<<<col_grid(g, kVertBlock), kVertBlock, smem, st>>>(g, P, s, dt);
}
void launch_update_rk2(const Geometry& g, const Phys& P, const State& s, cudaStream_t st) {
    update_rk2_kernel<<<col_grid(g, kColBlock), kColBlock, 0, st>>>(g, P, s);
}

} // namespace thorx
