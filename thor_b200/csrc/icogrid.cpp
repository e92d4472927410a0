// Icosahedral grid for thorx, built on the host.
//
// Produces the same grid as THOR's Icogrid (src/ESP/grid.cu:84-302) bit for bit: the same point
// positions and ordering, neighbour lists, rhombus halo maps, spring-dynamics relaxation, control
// volumes and FV operators. The construction steps therefore follow the reference's, in the
// reference's arithmetic order; the data structures and the neighbour search are this file's own:
//   * the recursive bisection works on one (S+1)x(S+1) lattice of positions per rhombic face,
//   * the nearest-neighbour search uses a uniform 3D hash of the unit sphere instead of the
//     reference's all-pairs scan, and applies the reference's selection rule (smallest distance,
//     later index on ties) to the candidates in index order, which returns the same neighbours,
//   * spring dynamics runs its per-point loops in parallel (each point's arithmetic unchanged).
// Host compiler flags: no -ffast-math and no FMA contraction (x86-64 baseline ISA), so that the
// arithmetic is the plain IEEE sequence written here, as in the reference's host build.

#include "icogrid.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
    double x, y, z;
};
inline V3     operator+(const V3& a, const V3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3     operator-(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3     operator*(const V3& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3     operator*(double s, const V3& a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3     operator/(const V3& a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double length(const V3& a) { return std::sqrt(dot(a, a)); }
inline V3     normalize(const V3& a) { return a / length(a); }
inline V3     cross(const V3& a, const V3& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Great-circle arc vector from v2 towards v1 scaled by the arc angle (grid.cu:70-82).
inline V3 arc_vector(const V3& v1, const V3& v2) {
    double l1  = dot(v1, v2);
    V3     vc1 = cross(v1, v2);
    double l2  = length(vc1);
    return vc1 / l2 * std::atan2(l2, l1);
}

// Sum of three triangle vertices in an order fixed by their z (then x) coordinates, so that
// every cell sharing the triangle gets the same rounding (vector_operations.h:242-341).
inline V3 ordered_sum3(const V3& a, const V3& b, const V3& c) {
    V3 w1, w2, w3;
    if (a.z == b.z || a.z == c.z || b.z == c.z) {
        V3 odd, s1, s2;
        if (a.z == b.z) {
            odd = c, s1 = a, s2 = b;
        }
        else if (a.z == c.z) {
            odd = b, s1 = a, s2 = c;
        }
        else {
            odd = a, s1 = b, s2 = c;
        }
        bool s1_first = s1.x < s2.x;
        if (odd.z < s1.z) {
            w1 = odd;
            w2 = s1_first ? s1 : s2;
            w3 = s1_first ? s2 : s1;
        }
        else {
            w1 = s1_first ? s1 : s2;
            w2 = s1_first ? s2 : s1;
            w3 = odd;
        }
    }
    else {
        V3 v[3] = {a, b, c};
        std::sort(v, v + 3, [](const V3& p, const V3& q) { return p.z < q.z; });
        w1 = v[0], w2 = v[1], w3 = v[2];
    }
    return w1 + w2 + w3;
}

// Spherical excess angle at a of triangle (a, b, c) (grid.cu:2176-2198).
inline double corner_angle(const V3& a, const V3& b, const V3& c) {
    V3     v0 = a, v1 = b - a, v2 = c - a;
    double t    = 1.0 / dot(v0, v0);
    double fac1 = dot(v0, v1) * t;
    double fac2 = dot(v0, v2) * t;
    V3     w1   = v1 - fac1 * v0;
    V3     w2   = v2 - fac2 * v0;
    double ang  = dot(w1, w2) / (length(w1) * length(w2));
    if (ang > 1)
        ang = 1;
    if (ang < -1)
        ang = -1;
    return std::acos(ang);
}

inline double tri_area(const V3& a, const V3& b, const V3& c) {
    double s = corner_angle(a, b, c) + corner_angle(b, a, c) + corner_angle(c, a, b);
    double r = length(a);
    return (s - M_PI) * std::pow(r, 2);
}

// Edge vector of arc (v1 -> v2) with length equal to the arc length, normal to the arc plane.
inline V3 arc_normal(const V3& v1, const V3& v2) {
    double vec_l = length(v1);
    double l     = std::acos(dot(v1, v2) / (std::pow(vec_l, 2.0))) * vec_l;
    V3     nv    = cross(v1, v2);
    double fac   = l / length(nv);
    return nv * fac;
}

struct Builder {
    int              glevel, nv, N, nl, nr, nfaces, kxl, S;
    std::vector<V3>  xyz, xyzq;
    std::vector<int> pent, point_local, halo, maps;
    std::vector<char> is_pent;

    // ---- positions: recursive bisection of the 10 rhombic faces (grid.cu:305-661) ----
    void positions() {
        S          = 1 << glevel;
        const int E = S + 1;
        // icosahedron vertices: the poles and two rings of five
        const double w = 2.0 * std::acos(1.0 / (2.0 * std::sin(M_PI / 5.0)));
        V3           ico[12];
        ico[0] = {0.0, 0.0, 1.0};
        ico[1] = {0.0, 0.0, -1.0};
        const double up[5] = {-M_PI / 5.0, M_PI / 5.0, 3.0 * M_PI / 5.0, M_PI, -(3.0 / 5.0) * M_PI};
        for (int i = 0; i < 5; i++)
            ico[2 + i] = {std::cos(up[i]) * std::cos(M_PI / 2.0 - w),
                          std::sin(up[i]) * std::cos(M_PI / 2.0 - w), std::sin(M_PI / 2.0 - w)};
        // (the reference writes the third vertex's z as sin(M_PI / 2 - w): the same value)
        const double dn[5] = {0.0, 2.0 * M_PI / 5.0, 4.0 * M_PI / 5.0, -4.0 * M_PI / 5.0,
                              -2.0 * M_PI / 5.0};
        for (int i = 0; i < 5; i++)
            ico[7 + i] = {std::cos(dn[i]) * std::cos(w - M_PI / 2.0),
                          std::sin(dn[i]) * std::cos(w - M_PI / 2.0), std::sin(w - M_PI / 2.0)};
        // corners (0,0), (S,0), (0,S), (S,S) of each face
        const int corner[10][4] = {{2, 0, 7, 3}, {3, 0, 8, 4},  {4, 0, 9, 5},  {5, 0, 10, 6},
                                   {6, 0, 11, 2}, {7, 3, 1, 8}, {8, 4, 1, 9}, {9, 5, 1, 10},
                                   {10, 6, 1, 11}, {11, 2, 1, 7}};
        std::vector<V3> lat((size_t)10 * E * E);
        auto            P = [&](int fc, int X, int Y) -> V3& { return lat[((size_t)fc * E + X) * E + Y]; };
        auto mid = [&](int fc, int X, int Y, int X1, int Y1, int X2, int Y2) {
            P(fc, X, Y) = normalize((P(fc, X1, Y1) + P(fc, X2, Y2)) * 0.5);
        };
        for (int fc = 0; fc < 10; fc++) {
            P(fc, 0, 0) = ico[corner[fc][0]];
            P(fc, S, 0) = ico[corner[fc][1]];
            P(fc, 0, S) = ico[corner[fc][2]];
            P(fc, S, S) = ico[corner[fc][3]];
            // edges and the (0,0)-(S,S) diagonal, coarse to fine
            for (int grd = 0; grd < glevel; grd++) {
                const int jump = 1 << (glevel - grd - 1);
                for (int it = 0, ind = jump; it < (1 << grd); it++, ind += 2 * jump) {
                    mid(fc, ind, 0, ind + jump, 0, ind - jump, 0);
                    mid(fc, 0, ind, 0, ind + jump, 0, ind - jump);
                    mid(fc, ind, ind, ind + jump, ind + jump, ind - jump, ind - jump);
                    mid(fc, ind, S, ind + jump, S, ind - jump, S);
                    mid(fc, S, ind, S, ind + jump, S, ind - jump);
                }
            }
            // interior of the two triangles either side of the diagonal
            for (int grd = 1; grd < glevel; grd++) {
                const int jump = 1 << (glevel - grd - 1);
                for (int j = 0, indj = jump; j < (1 << grd) - 1; j++, indj += 2 * jump)
                    for (int i = 0, ix = 0, iy = jump; i < j + 1; i++, ix += 2 * jump, iy += 2 * jump) {
                        const int X = S - indj + ix, Y = iy;
                        mid(fc, X, Y, X - jump, Y - jump, X + jump, Y + jump);
                        mid(fc, X - jump, Y, X - jump, Y - jump, X - jump, Y + jump);
                        mid(fc, X, Y + jump, X + jump, Y + jump, X - jump, Y + jump);
                    }
                for (int j = 0, indj = jump; j < (1 << grd) - 1; j++, indj += 2 * jump)
                    for (int i = 0, ix = jump, iy = 0; i < j + 1; i++, ix += 2 * jump, iy += 2 * jump) {
                        const int X = ix, Y = S - indj + iy;
                        mid(fc, X, Y, X - jump, Y - jump, X + jump, Y + jump);
                        mid(fc, X, Y - jump, X - jump, Y - jump, X + jump, Y - jump);
                        mid(fc, X + jump, Y, X + jump, Y + jump, X + jump, Y - jump);
                    }
            }
        }
        // global order: face, sub-rhombus (ky, kx), row j, column i; lattice X = ky*nl + j,
        // Y = kx*nl + i; the two poles last
        const int nl2 = nl * nl;
        xyz.assign(N, V3{0, 0, 0});
        for (int fc = 0; fc < 10; fc++)
            for (int kx = 0; kx < kxl; kx++)
                for (int ky = 0; ky < kxl; ky++)
                    for (int i = 0; i < nl; i++)
                        for (int j = 0; j < nl; j++)
                            xyz[(size_t)fc * nfaces * nl2 + ky * kxl * nl2 + kx * nl2 + j * nl + i] =
                                P(fc, ky * nl + j, kx * nl + i);
        xyz[N - 2] = {0.0, 0.0, 1.0};
        xyz[N - 1] = {0.0, 0.0, -1.0};
        pent.resize(12);
        for (int fc = 0; fc < 10; fc++)
            pent[fc] = fc * nfaces * nl2;
        pent[10] = N - 2;
        pent[11] = N - 1;
        is_pent.assign(N, 0);
        for (int p : pent)
            is_pent[p] = 1;
    }

    // ---- nearest neighbours (result of grid.cu:663-724 / 726-779) ----
    // Candidates within `radius` of each point from a uniform hash; the reference's selection
    // loop is then applied to the candidates in increasing index order.
    void nearest(const std::vector<int>& which, int count, std::vector<int>& out) {
        const double spacing = 2.0 * M_PI / (10.0 * std::pow(2.0, glevel - 1)) * 0.5;
        const double radius  = 3.5 * spacing;
        const int    G       = std::max(1, (int)std::floor(2.0 / radius));
        auto cell = [&](double v) { return std::min(G - 1, std::max(0, (int)((v + 1.0) / 2.0 * G))); };
        std::unordered_map<long, std::vector<int>> hash;
        for (int j = 0; j < N; j++)
            hash[((long)cell(xyz[j].x) * G + cell(xyz[j].y)) * G + cell(xyz[j].z)].push_back(j);
        bool ok = true;
#pragma omp parallel for schedule(dynamic, 64)
        for (size_t w = 0; w < which.size(); w++) {
            const int        i = which[w];
            std::vector<int> cand;
            int cx = cell(xyz[i].x), cy = cell(xyz[i].y), cz = cell(xyz[i].z);
            for (int a = cx - 1; a <= cx + 1; a++)
                for (int b = cy - 1; b <= cy + 1; b++)
                    for (int c = cz - 1; c <= cz + 1; c++) {
                        if (a < 0 || b < 0 || c < 0 || a >= G || b >= G || c >= G)
                            continue;
                        auto it = hash.find(((long)a * G + b) * G + c);
                        if (it != hash.end())
                            cand.insert(cand.end(), it->second.begin(), it->second.end());
                    }
            std::sort(cand.begin(), cand.end());
            std::vector<double> d(cand.size());
            for (size_t q = 0; q < cand.size(); q++) {
                const V3& p = xyz[cand[q]];
                double    dx = p.x - xyz[i].x, dy = p.y - xyz[i].y, dz = p.z - xyz[i].z;
                d[q]         = std::sqrt(dx * dx + dy * dy + dz * dz);
            }
            int* pl = &out[(size_t)i * 6];
            double dmax = 0;
            for (int k = 0; k < count; k++) {
                double small = 2;
                int    pos   = -1;
                for (size_t q = 0; q < cand.size(); q++) {
                    if (small >= d[q] && d[q] > 0) {
                        int j = cand[q];
                        if (k == 0 || (pl[0] != j && pl[1] != j && pl[2] != j && pl[3] != j && pl[4] != j && pl[5] != j)) {
                            small = d[q];
                            pos   = j;
                        }
                    }
                }
                pl[k] = pos;
                dmax  = std::max(dmax, small);
            }
            // every point closer than the farthest selected one must have been a candidate
            if (dmax >= radius * 0.999)
#pragma omp atomic write
                ok = false;
        }
        if (!ok)
            std::fprintf(stderr, "icogrid: neighbour search radius too small\n");
    }

    // ---- clockwise ordering by angle about the mean of the neighbours (grid.cu:781-917) ----
    void order_by_angle(int i, int geo) {
        double ang[6] = {0, 0, 0, 0, 0, 0};
        int*   pl     = &point_local[(size_t)i * 6];
        int    nw[6];
        for (int j = 0; j < 6; j++)
            nw[j] = pl[j];
        double x1 = 0, y1 = 0, z1 = 0;
        for (int j = 0; j < geo; j++) {
            x1 = x1 + xyz[pl[j]].x / geo;
            y1 = y1 + xyz[pl[j]].y / geo;
            z1 = z1 + xyz[pl[j]].z / geo;
        }
        double dx21 = xyz[pl[0]].x - x1, dy21 = xyz[pl[0]].y - y1, dz21 = xyz[pl[0]].z - z1;
        for (int j = 1; j < geo; j++) {
            double dx31 = xyz[pl[j]].x - x1, dy31 = xyz[pl[j]].y - y1, dz31 = xyz[pl[j]].z - z1;
            double n21 = std::sqrt(dx21 * dx21 + dy21 * dy21 + dz21 * dz21);
            double n31 = std::sqrt(dx31 * dx31 + dy31 * dy31 + dz31 * dz31);
            double cx = dy21 * dz31 - dy31 * dz21, cy = dz21 * dx31 - dz31 * dx21, cz = dx21 * dy31 - dx31 * dy21;
            double dn = cx * x1 + cy * y1 + cz * z1;
            double a  = std::acos((dx21 * dx31 + dy21 * dy31 + dz21 * dz31) / (n21 * n31));
            ang[j]    = (dn <= 0) ? a : 2.0 * M_PI - a;
        }
        // the reference's exchange sort (ties keep its exchange pattern)
        for (int j = 0; j < geo; j++)
            for (int k = geo - 1; k >= j; k--)
                if (ang[j] > ang[k]) {
                    std::swap(ang[j], ang[k]);
                    std::swap(nw[j], nw[k]);
                }
        for (int j = 0; j < 6; j++)
            pl[j] = nw[j];
    }

    // ---- halos around each rhombus (grid.cu:1009-1493) ----
    void halos() {
        const int nl2 = nl * nl, nh = 4 * (nl + 2);
        halo.assign((size_t)10 * nfaces * nh, -1);
        int ind_nei = 0; // persists across corners, as in the reference
        for (int fc = 0; fc < 10; fc++)
            for (int kx = 0; kx < kxl; kx++)
                for (int ky = 0; ky < kxl; ky++) {
                    const int base = fc * nfaces * nl2 + ky * kxl * nl2 + kx * nl2;
                    int*      H    = &halo[(size_t)fc * kxl * kxl * nh + ky * kxl * nh + kx * nh];
                    const bool first_is_pent = (kx == 0 && ky == 0);
                    auto inside = [&](int v) { return v >= base && v < base + nl2; };
                    // common neighbour of cells a, b outside the rhombus (last match wins)
                    auto between = [&](int a, int b, int ka, int& slot) {
                        for (int k = 0; k < ka; k++)
                            for (int kk = 0; kk < 6; kk++) {
                                int v1 = point_local[(size_t)a * 6 + k], v2 = point_local[(size_t)b * 6 + kk];
                                if (v1 == v2 && !inside(v1))
                                    slot = v1;
                            }
                    };
                    // neighbour of cell a that precedes `prev` in a's clockwise order
                    auto corner = [&](int a, int prev, int& slot) {
                        for (int k = 0; k < 6; k++)
                            if (point_local[(size_t)a * 6 + k] == prev)
                                ind_nei = k;
                        slot = (ind_nei > 0) ? point_local[(size_t)a * 6 + ind_nei - 1]
                                             : point_local[(size_t)a * 6 + 5];
                    };
                    auto cellid = [&](int j, int i) { return base + j * nl + i; };
                    // side 1 (row j = 0)
                    for (int i = 0; i < nl - 1; i++)
                        between(cellid(0, i), cellid(0, i + 1), (first_is_pent && i == 0) ? 5 : 6, H[i]);
                    corner(cellid(0, nl - 1), H[nl - 2], H[nl - 1]);
                    // side 2 (column i = nl-1)
                    corner(cellid(0, nl - 1), H[nl - 1], H[nl + 2]);
                    for (int j = 0; j < nl - 1; j++)
                        between(cellid(j, nl - 1), cellid(j + 1, nl - 1), 6, H[(nl + 2) + j + 1]);
                    // side 3 (row j = nl-1, walked backwards)
                    corner(cellid(nl - 1, nl - 1), H[nl + 2 + nl - 1], H[2 * (nl + 2)]);
                    for (int i = 0; i < nl - 1; i++)
                        between(cellid(nl - 1, nl - i - 1), cellid(nl - 1, nl - i - 2), 6,
                                H[2 * (nl + 2) + i + 1]);
                    corner(cellid(nl - 1, 0), H[2 * (nl + 2) + nl - 1], H[2 * (nl + 2) + nl]);
                    // side 4 (column i = 0, walked backwards)
                    corner(cellid(nl - 1, 0), H[2 * (nl + 2) + nl], H[3 * (nl + 2)]);
                    for (int j = 0; j < nl - 1; j++)
                        between(cellid(nl - j - 1, 0), cellid(nl - j - 2, 0), 6, H[3 * (nl + 2) + j + 1]);
                    if (!first_is_pent)
                        corner(cellid(0, 0), H[3 * (nl + 2) + nl - 1], H[3 * (nl + 2) + nl]);
                }
    }

    // ---- neighbours in rhombus order (grid.cu:1495-1621) ----
    void rhombus_neighbours() {
        const int nl2 = nl * nl, nlhalo = nl + 2, nh2 = 4 * nlhalo;
        std::fill(point_local.begin(), point_local.end(), -1);
        for (int r = 0; r < nr; r++) {
            const bool pe = is_pent[nl2 * r];
            const int* H  = &halo[(size_t)r * nh2];
            for (int j = 0; j < nl; j++)
                for (int k = 0; k < nl; k++) {
                    const int np = nl2 * r + j * nl + k;
                    int*      pl = &point_local[(size_t)np * 6];
                    const int in = nl2 * r;
                    // along j
                    if (j == 0) {
                        pl[0] = in + (j + 1) * nl + k;
                        pl[3] = H[k];
                    }
                    else if (j == nl - 1) {
                        pl[0] = H[2 * nlhalo + nl - k];
                        pl[3] = in + (j - 1) * nl + k;
                    }
                    else {
                        pl[0] = in + (j + 1) * nl + k;
                        pl[3] = in + (j - 1) * nl + k;
                    }
                    // along k
                    if (k == 0) {
                        pl[2] = in + j * nl + k + 1;
                        pl[5] = (pe && j == 0) ? -1 : H[3 * nlhalo + nl - j - 1];
                    }
                    else if (k == nl - 1) {
                        pl[2] = H[nlhalo + j];
                        pl[5] = in + j * nl + k - 1;
                    }
                    else {
                        pl[2] = in + j * nl + k + 1;
                        pl[5] = in + j * nl + k - 1;
                    }
                    // diagonal
                    if (j == 0) {
                        if (k == 0) {
                            pl[4] = pe ? H[3 * nlhalo + nl - 1] : H[3 * nlhalo + nl];
                            pl[1] = in + nl + k + 1;
                        }
                        else if (k == nl - 1) {
                            pl[4] = H[nl - 2];
                            pl[1] = H[nl + 3];
                        }
                        else {
                            pl[4] = H[k - 1];
                            pl[1] = in + (j + 1) * nl + k + 1;
                        }
                    }
                    else if (j == nl - 1) {
                        if (k == 0) {
                            pl[4] = H[3 * nlhalo + 1];
                            pl[1] = H[2 * nlhalo + nl - 1];
                        }
                        else if (k == nl - 1) {
                            pl[4] = in + (j - 1) * nl + k - 1;
                            pl[1] = H[2 * nlhalo];
                        }
                        else {
                            pl[4] = in + (j - 1) * nl + k - 1;
                            pl[1] = H[2 * nlhalo - k + nl - 1];
                        }
                    }
                    else {
                        if (k == 0) {
                            pl[4] = H[3 * nlhalo - j + nl];
                            pl[1] = in + (j + 1) * nl + k + 1;
                        }
                        else if (k == nl - 1) {
                            pl[4] = in + (j - 1) * nl + k - 1;
                            pl[1] = H[nl + 2 + j + 1];
                        }
                        else {
                            pl[4] = in + (j - 1) * nl + k - 1;
                            pl[1] = in + (j + 1) * nl + k + 1;
                        }
                    }
                }
        }
    }

    // ---- rhombus tiles with a one-cell halo (grid.cu:1624-1668) ----
    void make_maps() {
        const int nl2 = nl + 2, nl22 = nl2 * nl2, nh2 = 4 * (nl + 2), nlr2 = nl * nl;
        maps.assign((size_t)nl22 * nr, 0);
        for (int l = 0; l < nr; l++) {
            int*       M = &maps[(size_t)l * nl22];
            const int* H = &halo[(size_t)l * nh2];
            for (int i = 0; i < nl; i++)
                for (int j = 0; j < nl; j++)
                    M[(j + 1) * nl2 + i + 1] = l * nlr2 + j * nl + i;
            for (int i = 0; i < nl + 1; i++)
                M[i + 1] = H[i];
            for (int i = 0; i < nl + 2; i++)
                M[i * nl2] = H[3 * nl2 + nl - i];
            for (int i = 0; i < nl + 1; i++)
                M[(nl + 1) * nl2 + i + 1] = H[2 * nl2 + nl - i];
            for (int i = 0; i < nl; i++)
                M[(i + 1) * nl2 + nl + 1] = H[nl2 + i];
        }
    }

    // ---- spring dynamics, Tomita et al. 2002 (grid.cu:1670-1815) ----
    int spring_dynamics(double beta) {
        std::vector<V3>     vel(N, V3{0, 0, 0}), F(N), Fnei((size_t)N * 6);
        std::vector<double> Fnet(N, 0.0);
        V3                  fixed[12];
        const double lba   = 2.0 * M_PI / (10.0 * std::pow(2.0, glevel - 1));
        const double dbar  = beta * lba;
        const double drag  = 1;
        const double tstep = 2.0E-2;
        const double cond  = 1.0E-4;
        for (int i = 0; i < 12; i++) {
            fixed[i]                      = xyz[pent[i]];
            point_local[pent[i] * 6 + 5] = point_local[pent[i] * 6];
        }
        std::vector<V3> P(N);
        int             it;
        for (it = 0; it < 100000; it++) {
            P = xyz;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < N; i++)
                for (int j = 0; j < 6; j++) {
                    const V3& q = P[point_local[(size_t)i * 6 + j]];
                    V3        W = cross(P[i], q);
                    V3        V = cross(W, P[i]);
                    double    l = length(V);
                    double    d = std::acos(dot(P[i], q));
                    Fnei[(size_t)i * 6 + j] = ((d - dbar) * V) / l;
                }
            for (int i = 0; i < 12; i++)
                Fnei[(size_t)pent[i] * 6 + 5] = V3{0.0, 0.0, 0.0};
            double max_v = -1E-10;
#pragma omp parallel for schedule(static) reduction(max : max_v)
            for (int i = 0; i < N; i++) {
                const V3* f = &Fnei[(size_t)i * 6];
                V3        net = f[0] + f[1] + f[2] + f[3] + f[4] + f[5];
                Fnet[i]       = length(net) / lba;
                F[i]          = net - drag * vel[i];
                V3 D          = xyz[i] + vel[i] * tstep;
                xyz[i]        = normalize(D);
                V3     vv     = vel[i] + F[i] * tstep;
                double H      = dot(xyz[i], vv);
                vel[i]        = vv - H * xyz[i];
                if (!is_pent[i] && Fnet[i] > max_v)
                    max_v = Fnet[i];
            }
            for (int i = 0; i < 12; i++) {
                vel[pent[i]]  = V3{0.0, 0.0, 0.0};
                Fnet[pent[i]] = 0.0;
                xyz[pent[i]]  = fixed[i];
            }
            if (max_v < 0.0)
                max_v = 0.0; // every point a pentagon: Fnet would all be 0 in the reference
            if (max_v < cond)
                break;
        }
        return it;
    }

    // ---- corners of the control volumes (grid.cu:1817-1870) ----
    void qpoints() {
        xyzq.assign((size_t)N * 6, V3{0, 0, 0});
#pragma omp parallel for schedule(static)
        for (int i = 0; i < N; i++) {
            const int  geo = is_pent[i] ? 5 : 6;
            const int* pl  = &point_local[(size_t)i * 6];
            for (int j = 0; j < geo; j++) {
                const int a = pl[j], b = pl[(j + 1) % geo];
                V3 vc1 = arc_vector(xyz[a], xyz[i]);
                V3 vc2 = arc_vector(xyz[b], xyz[a]);
                V3 vc3 = arc_vector(xyz[i], xyz[b]);
                xyzq[(size_t)i * 6 + j] = normalize(ordered_sum3(vc1, vc2, vc3));
            }
            if (geo == 5)
                xyzq[(size_t)i * 6 + 5] = V3{0.0, 0.0, 0.0};
        }
    }

    // ---- centroids from the corners (grid.cu:1873-1921) ----
    void relocate_centres() {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < N; i++) {
            const int geo = is_pent[i] ? 5 : 6;
            const V3* q   = &xyzq[(size_t)i * 6];
            V3        vgc{0.0, 0.0, 0.0};
            for (int j = 1; j < geo; j++)
                vgc = vgc + arc_vector(q[j], q[j - 1]);
            vgc    = vgc + arc_vector(q[0], q[geo - 1]);
            xyz[i] = normalize(vgc);
        }
    }
};

} // namespace

struct thorx_icogrid {
    int                                glevel, nv, N, nl, nr;
    int                                spring_iterations = 0;
    std::map<std::string, std::vector<double>> f;
    std::vector<int>                   maps, point_local, pent_ind;
};

extern "C" int thorx_grid_build(int glevel, int vlevel, double A, double Top_altitude,
                                int spring, double spring_beta, thorx_icogrid** out) {
    if (!out)
        return -1;
    *out = nullptr;
    if (glevel < 4 || glevel > 7 || vlevel < 3 || A <= 0 || Top_altitude <= 0)
        return -1; // the rhombus split (divide_face) is defined for glevel 4..7 only
    Builder b;
    b.glevel          = glevel;
    b.nv              = vlevel;
    b.N               = 2 + 10 * (1 << (2 * glevel));
    const int divide  = glevel - 4;
    b.nl              = (1 << glevel) >> divide;
    b.nfaces          = 1 << (2 * divide);
    b.kxl             = 1 << divide;
    b.nr              = (b.N - 2) / (b.nl * b.nl);
    const int N       = b.N;
    b.positions();
    // neighbours of every point, clockwise
    b.point_local.assign((size_t)N * 6, -1);
    {
        std::vector<int> all(N);
        for (int i = 0; i < N; i++)
            all[i] = i;
        b.nearest(all, 6, b.point_local);
        for (int p : b.pent)
            b.point_local[(size_t)p * 6 + 5] = -1;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < N; i++)
            b.order_by_angle(i, b.is_pent[i] ? 5 : 6);
    }
    b.halos();
    b.rhombus_neighbours();
    {
        std::vector<int> poles = {N - 2, N - 1};
        b.nearest(poles, 5, b.point_local);
        for (int p : poles)
            b.order_by_angle(p, 5);
    }
    b.make_maps();
    int its = 0;
    if (spring) {
        its = b.spring_dynamics(spring_beta);
        b.qpoints();
        b.relocate_centres();
    }
    else
        b.qpoints();

    // ---- scale to the planet radius (grid.cu:2130-2174) ----
    for (int i = 0; i < N; i++) {
        for (int j = 0; j < (b.is_pent[i] ? 5 : 6); j++)
            b.xyzq[(size_t)i * 6 + j] = b.xyzq[(size_t)i * 6 + j] * A;
        b.xyz[i] = b.xyz[i] * A;
    }

    thorx_icogrid* g = new thorx_icogrid;
    g->glevel = glevel, g->nv = vlevel, g->N = N, g->nl = b.nl, g->nr = b.nr;
    g->spring_iterations = its;
    auto& F = g->f;
    std::vector<double>& func_r = F["func_r"];
    func_r.resize(3 * (size_t)N);
    for (int i = 0; i < N; i++) {
        V3 u = normalize(b.xyz[i]);
        func_r[3 * i] = u.x, func_r[3 * i + 1] = u.y, func_r[3 * i + 2] = u.z;
    }

    // ---- control areas (grid.cu:2200-2420) ----
    std::vector<double>& areas = F["areas"];
    std::vector<double>& areasTr = F["areasTr"];
    std::vector<double>& areasT = F["areasT"];
    areas.assign(18 * (size_t)N, 0.0);
    areasTr.assign(6 * (size_t)N, 0.0);
    areasT.assign(N, 0.0);
    const auto& X = b.xyz;
    const auto& Q = b.xyzq;
    const auto& PL = b.point_local;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        const int geo = b.is_pent[i] ? 5 : 6;
        for (int j = 0; j < geo; j++) {
            const int nj = PL[(size_t)i * 6 + j], nj1 = PL[(size_t)i * 6 + (j + 1) % geo];
            const V3& q  = Q[(size_t)i * 6 + j];
            areas[(size_t)i * 18 + j * 3 + 0] = tri_area(X[nj1], X[nj], q);
            areas[(size_t)i * 18 + j * 3 + 1] = tri_area(X[nj1], X[i], q);
            areas[(size_t)i * 18 + j * 3 + 2] = tri_area(X[i], X[nj], q);
            areasTr[(size_t)i * 6 + j] = areas[(size_t)i * 18 + j * 3 + 0] + areas[(size_t)i * 18 + j * 3 + 1]
                                         + areas[(size_t)i * 18 + j * 3 + 2];
        }
        double sum = 0.0;
        for (int j = 0; j < geo; j++)
            sum += tri_area(X[i], Q[(size_t)i * 6 + j], Q[(size_t)i * 6 + (j + 1) % geo]);
        areasT[i] = sum;
    }
    // normalise to the exact sphere area; sums in the reference's serial order
    {
        double area_tot_exact = 4 * M_PI * std::pow(A, 2.0), tot_T = 0.0, tot_Tr = 0.0, tot_sub = 0.0;
        for (int i = 0; i < N; i++) {
            if (i < N - 2)
                for (int j = 0; j < 2; j++) {
                    tot_Tr += areasTr[(size_t)i * 6 + j];
                    tot_sub += (areas[(size_t)i * 18 + j * 3 + 0] + areas[(size_t)i * 18 + j * 3 + 1]
                                + areas[(size_t)i * 18 + j * 3 + 2]);
                }
        }
        for (int i = 0; i < N; i++)
            tot_T += areasT[i];
        for (int i = 0; i < N; i++) {
            areasT[i] *= area_tot_exact / tot_T;
            for (int j = 0; j < 6; j++) {
                areasTr[(size_t)i * 6 + j] *= area_tot_exact / tot_Tr;
                for (int k = 0; k < 3; k++)
                    areas[(size_t)i * 18 + j * 3 + k] *= area_tot_exact / tot_sub;
            }
        }
    }

    // ---- normal vectors of edges (grid.cu:2423-2630) ----
    std::vector<double>& nvec = F["nvec"];
    std::vector<double>& nvecoa = F["nvecoa"];
    std::vector<double>& nvecti = F["nvecti"];
    std::vector<double>& nvecte = F["nvecte"];
    nvec.assign(18 * (size_t)N, 0.0);
    nvecoa.assign(18 * (size_t)N, 0.0);
    nvecti.assign(18 * (size_t)N, 0.0);
    nvecte.assign(18 * (size_t)N, 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        const int geo = b.is_pent[i] ? 5 : 6;
        for (int j = 0; j < geo; j++) {
            const int jn = (j + 1) % geo;
            V3        n  = arc_normal(Q[(size_t)i * 6 + j], Q[(size_t)i * 6 + jn]);
            V3        oa = n / areasT[i];
            V3        ti = arc_normal(X[PL[(size_t)i * 6 + j]], X[i]);
            V3        te = arc_normal(X[PL[(size_t)i * 6 + j]], X[PL[(size_t)i * 6 + jn]]);
            double*   pn = &nvec[(size_t)i * 18 + j * 3];
            double*   po = &nvecoa[(size_t)i * 18 + j * 3];
            double*   pi = &nvecti[(size_t)i * 18 + j * 3];
            double*   pe = &nvecte[(size_t)i * 18 + j * 3];
            pn[0] = n.x, pn[1] = n.y, pn[2] = n.z;
            po[0] = oa.x, po[1] = oa.y, po[2] = oa.z;
            pi[0] = ti.x, pi[1] = ti.y, pi[2] = ti.z;
            pe[0] = te.x, pe[1] = te.y, pe[2] = te.z;
        }
    }

    // ---- vertical levels, uniform (grid.cu:1923-1948) ----
    std::vector<double>& Alt = F["Altitude"];
    std::vector<double>& Alth = F["Altitudeh"];
    Alt.resize(vlevel);
    Alth.resize(vlevel + 1);
    {
        double res = Top_altitude / vlevel;
        Alth[0]    = 0.0;
        for (int lev = 0; lev < vlevel; lev++)
            Alth[lev + 1] = Alth[lev] + res;
        for (int lev = 0; lev < vlevel; lev++)
            Alt[lev] = (Alth[lev] + Alth[lev + 1]) / 2.0;
    }

    // ---- longitude, latitude (grid.cu:2111-2128) ----
    std::vector<double>& lonlat = F["lonlat"];
    lonlat.resize(2 * (size_t)N);
    for (int i = 0; i < N; i++) {
        lonlat[2 * i]     = std::atan2(X[i].y, X[i].x);
        lonlat[2 * i + 1] = std::atan2(X[i].z, std::sqrt(std::pow(X[i].x, 2) + std::pow(X[i].y, 2)));
    }

    // ---- divergence and gradient operators, Satoh et al. 2008 eqs 15-16 (grid.cu:2656-2831,
    // 3015-3200): one 7-point stencil per column, point 0 the cell, 1..6 its neighbours ----
    std::vector<double>& div = F["div"];
    std::vector<double>& grad = F["grad"];
    div.assign(21 * (size_t)N, 0.0);
    grad.assign(21 * (size_t)N, 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; i++) {
        const bool   p5  = b.is_pent[i];
        const int    geo = p5 ? 5 : 6;
        double       aq[6][3];
        const double* ar = &areas[(size_t)i * 18];
        double        at[6];
        for (int j = 0; j < 6; j++)
            at[j] = (p5 && j == 5) ? 0 : ar[j * 3 + 0] + ar[j * 3 + 1] + ar[j * 3 + 2];
        for (int j = 0; j < 6; j++)
            for (int k = 0; k < 3; k++)
                aq[j][k] = (p5 && j == 5) ? 0 : ar[j * 3 + k] / at[j];
        const double* nv_ = &nvec[(size_t)i * 18];
        for (int k = 0; k < 3; k++) {
            auto n = [&](int j) { return nv_[j * 3 + k]; };
            // point 0: every edge, with the mean of the two sub-areas either side
            double d0 = 0;
            for (int j = 0; j < geo; j++) {
                double t = n(j) * (aq[j][0] + aq[(j + 1) % geo][0]);
                d0       = (j == 0) ? t : d0 + t;
            }
            double s = 0;
            for (int j = 0; j < geo; j++)
                s = (j == 0) ? n(j) : s + n(j);
            double* D = &div[(size_t)i * 21];
            double* G = &grad[(size_t)i * 21];
            D[k]      = d0;
            G[k]      = d0 - 2 * s;
            // neighbour m (1..geo): edges m-2, m-1 of its two triangles
            for (int m = 1; m <= geo; m++) {
                const int a  = m - 1;                    // triangle after neighbour m
                const int bq = (m - 2 + geo) % geo;      // triangle before neighbour m
                double    t  = n(bq) * (aq[a][1] + aq[bq][2]) + n((bq + geo - 1) % geo) * aq[bq][2] + n(a) * aq[a][1];
                D[m * 3 + k] = t;
                G[m * 3 + k] = t;
            }
            if (p5) {
                D[6 * 3 + k] = 0.0;
                G[6 * 3 + k] = 0.0;
            }
        }
        for (int q = 0; q < 21; q++) {
            div[(size_t)i * 21 + q]  = div[(size_t)i * 21 + q] / (2.0 * areasT[i]);
            grad[(size_t)i * 21 + q] = grad[(size_t)i * 21 + q] / (2.0 * areasT[i]);
        }
    }

    std::vector<double>& xyz = F["point_xyz"];
    std::vector<double>& xyzq = F["point_xyzq"];
    xyz.resize(3 * (size_t)N);
    xyzq.resize(18 * (size_t)N);
    for (int i = 0; i < N; i++) {
        xyz[3 * i] = X[i].x, xyz[3 * i + 1] = X[i].y, xyz[3 * i + 2] = X[i].z;
        for (int j = 0; j < 6; j++) {
            xyzq[(size_t)i * 18 + j * 3]     = Q[(size_t)i * 6 + j].x;
            xyzq[(size_t)i * 18 + j * 3 + 1] = Q[(size_t)i * 6 + j].y;
            xyzq[(size_t)i * 18 + j * 3 + 2] = Q[(size_t)i * 6 + j].z;
        }
    }
    g->maps        = b.maps;
    g->point_local = b.point_local;
    g->pent_ind    = b.pent;
    *out           = g;
    return 0;
}

extern "C" void thorx_grid_free(thorx_icogrid* g) { delete g; }

extern "C" int thorx_grid_info(const thorx_icogrid* g, int* point_num, int* nv, int* nl_region,
                               int* nr, int* spring_iterations) {
    if (!g)
        return -1;
    if (point_num)
        *point_num = g->N;
    if (nv)
        *nv = g->nv;
    if (nl_region)
        *nl_region = g->nl;
    if (nr)
        *nr = g->nr;
    if (spring_iterations)
        *spring_iterations = g->spring_iterations;
    return 0;
}

extern "C" long thorx_grid_get(const thorx_icogrid* g, const char* name, void* out) {
    if (!g || !name)
        return -1;
    std::string n(name);
    const std::vector<int>* iv = nullptr;
    if (n == "maps")
        iv = &g->maps;
    else if (n == "point_local")
        iv = &g->point_local;
    else if (n == "pent_ind")
        iv = &g->pent_ind;
    if (iv) {
        if (out)
            std::memcpy(out, iv->data(), iv->size() * sizeof(int));
        return (long)iv->size();
    }
    auto it = g->f.find(n);
    if (it == g->f.end())
        return -1;
    if (out)
        std::memcpy(out, it->second.data(), it->second.size() * sizeof(double));
    return (long)it->second.size();
}

extern "C" int thorx_grid_describe(const thorx_icogrid* g, thorx_grid* d) {
    if (!g || !d)
        return -1;
    auto P = [&](const char* k) { return g->f.at(k).data(); };
    d->point_num   = g->N;
    d->nv          = g->nv;
    d->nl_region   = g->nl;
    d->nr          = g->nr;
    d->glevel      = g->glevel;
    d->maps        = g->maps.data();
    d->point_local = g->point_local.data();
    d->Altitude    = P("Altitude");
    d->Altitudeh   = P("Altitudeh");
    d->lonlat      = P("lonlat");
    d->areas       = P("areas");
    d->areasTr     = P("areasTr");
    d->areasT      = P("areasT");
    d->nvecoa      = P("nvecoa");
    d->nvecti      = P("nvecti");
    d->nvecte      = P("nvecte");
    d->div         = P("div");
    d->grad        = P("grad");
    d->func_r      = P("func_r");
    return 0;
}
