// The immersed body's tables, built on the host when a run is created (ImmersedBoundary's constructor and build_ghosts,
// cpp/src/Physics.cpp:850-866 and 1397-1537, for a static cylinder (2-D, or extruded along z) or sphere with the ghost-cell
// wall, slip or no-slip, without the curvature correction). The arithmetic keeps the reference's expressions, so the
// mask, the image-point weights and the ratios are its bits; the device kernels (ibm.cuh) only apply them.
#pragma once

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/fenice_gpu.h"

namespace fvg {

struct IbmTable {
    std::vector<unsigned char> mask;   // 1 = solid cell
    std::vector<int> ghost;            // ghost cells, in cell order (the solid cells within two cells of a fluid cell)
    std::vector<int> img_cell;         // 8 per ghost: the image point's interpolation cells (the first four in 2-D / extruded bodies)
    std::vector<double> img_w;         // 8 per ghost: their weights (0 for a solid cell; renormalised)
    std::vector<double> ratio, gnx, gny, gnz;   // per ghost: distance ghost-wall / distance image-wall, and the wall normal
    std::vector<double> gwx, gwy, gwz;          // per ghost: its wall point (the wall velocity of a moving body is taken there)
    std::vector<double> span;                   // per ghost: distance ghost-wall + wall-image (the hydrostatic correction's; 0 in a fallback)
    std::vector<int> deep;             // the other solid cells
    int fallback = 0;                  // ghosts with no fluid around any image point (nearest fluid cell, ratio 0)
};

struct IbmGeom {
    bool ball;   // a sphere in 3-D; otherwise a circle (2-D) or a cylinder along z (3-D)
    double cx, cy, cz, r;
    int nx, ny, nz;
    double dx, dy, dz;
    size_t cell(int i, int j, int k) const { return (static_cast<size_t>(k) * ny + j) * nx + i; }
    double xc(int i) const { return (i + 0.5) * dx + 0.0; }
    double yc(int j) const { return (j + 0.5) * dy + 0.0; }
    double zc(int k) const { return (k + 0.5) * dz + 0.0; }
    bool solid_at(double x, double y, double z) const {
        if (ball) {
            const double dxc = x - cx, dyc = y - cy;
            const double r2 = dxc * dxc + dyc * dyc + (z - cz) * (z - cz);
            return std::sqrt(r2) <= r;
        }
        const double dxc = x - cx, dyc = y - cy;
        const double r2 = dxc * dxc + dyc * dyc;
        return std::sqrt(r2) <= r;
    }
};

inline double dmax_(double a, double b) { return (a < b) ? b : a; }
inline double dmin_(double a, double b) { return (b < a) ? b : a; }

// bilinear probe in the four cell centres around (x, y) of layer k; solid cells weigh 0, the rest renormalised (make_probe)
inline bool make_probe(const IbmGeom& m, const std::vector<unsigned char>& mask, double x, double y, int layer, int* cell, double* w) {
    const double fx = (x - 0.0) / m.dx - 0.5, fy = (y - 0.0) / m.dy - 0.5;
    int i0 = static_cast<int>(std::floor(fx)), j0 = static_cast<int>(std::floor(fy));
    i0 = std::min(std::max(i0, 0), m.nx - 2);
    j0 = std::min(std::max(j0, 0), m.ny - 2);
    const double tx = dmin_(1.0, dmax_(0.0, fx - i0)), ty = dmin_(1.0, dmax_(0.0, fy - j0));
    const int ci[4] = {i0, i0 + 1, i0, i0 + 1}, cj[4] = {j0, j0, j0 + 1, j0 + 1};
    const double ww[4] = {(1 - tx) * (1 - ty), tx * (1 - ty), (1 - tx) * ty, tx * ty};
    double sum = 0.0;
    for (int k = 0; k < 8; ++k) {
        cell[k] = 0;
        w[k] = 0.0;
    }
    for (int k = 0; k < 4; ++k) {
        cell[k] = static_cast<int>(m.cell(ci[k], cj[k], layer));
        w[k] = mask[m.cell(ci[k], cj[k], layer)] ? 0.0 : ww[k];
        sum += w[k];
    }
    if (sum < 1e-6) return false;
    for (int k = 0; k < 8; ++k) w[k] /= sum;
    return true;
}

// trilinear probe in the eight cell centres around (x, y, z) (make_probe3)
inline bool make_probe3(const IbmGeom& m, const std::vector<unsigned char>& mask, double x, double y, double z, int* cell, double* w) {
    const double fx = (x - 0.0) / m.dx - 0.5, fy = (y - 0.0) / m.dy - 0.5, fz = (z - 0.0) / m.dz - 0.5;
    int i0 = static_cast<int>(std::floor(fx)), j0 = static_cast<int>(std::floor(fy)), k0 = static_cast<int>(std::floor(fz));
    i0 = std::min(std::max(i0, 0), m.nx - 2);
    j0 = std::min(std::max(j0, 0), m.ny - 2);
    k0 = std::min(std::max(k0, 0), m.nz - 2);
    const double tx = dmin_(1.0, dmax_(0.0, fx - i0)), ty = dmin_(1.0, dmax_(0.0, fy - j0)), tz = dmin_(1.0, dmax_(0.0, fz - k0));
    double sum = 0.0;
    for (int q = 0; q < 8; ++q) {
        const int di = q & 1, dj = (q >> 1) & 1, dk = (q >> 2) & 1;
        const double ww = (di ? tx : 1 - tx) * (dj ? ty : 1 - ty) * (dk ? tz : 1 - tz);
        cell[q] = static_cast<int>(m.cell(i0 + di, j0 + dj, k0 + dk));
        w[q] = mask[m.cell(i0 + di, j0 + dj, k0 + dk)] ? 0.0 : ww;
        sum += w[q];
    }
    if (sum < 1e-6) return false;
    for (int q = 0; q < 8; ++q) w[q] /= sum;
    return true;
}

// The body's geometry on the mesh of a configuration, its centre at (cx, cy, cz) (a moving body: its placement plus the
// displacement of its pose, ImmersedBoundary::place_geometry, cpp/src/Physics.cpp:1162-1194).
inline IbmGeom ibm_geom(const fvg_config& c, double cx, double cy, double cz) {
    IbmGeom m;
    m.ball = c.nz > 1 && c.ibm_shape == 1;
    m.cx = cx;
    m.cy = cy;
    m.cz = cz;
    m.r = c.ibm_radius;
    m.nx = c.nx;
    m.ny = c.ny;
    m.nz = c.nz;
    m.dx = c.Lx / c.nx;
    m.dy = c.Ly / c.ny;
    m.dz = c.Lz / c.nz;
    return m;
}

inline std::string build_ibm_geom(const IbmGeom& m, IbmTable& t);

// The mask and the ghost table of a static body on the whole mesh; returns "" or an error message.
inline std::string build_ibm(const fvg_config& c, IbmTable& t) {
    if (c.ibm_shape != 0 && c.ibm_shape != 1) return "ibm_shape: Cylinder or Sphere only on the device";
    if (c.ibm_curvature) return "ibm_curvature is not supported on the device";
    return build_ibm_geom(ibm_geom(c, c.ibm_cx, c.ibm_cy, c.ibm_cz), t);
}

// The mask and the ghost table of the body of geometry m (ImmersedBoundary::build_ghosts, Physics.cpp:1397-1537).
inline std::string build_ibm_geom(const IbmGeom& m, IbmTable& t) {
    const bool d3 = m.nz > 1;
    if (m.nx < 2 || m.ny < 2 || (m.ball && m.nz < 2)) return "the immersed body needs at least two cells per axis";
    const size_t n = static_cast<size_t>(m.nx) * m.ny * m.nz;
    t = IbmTable();
    t.mask.assign(n, 0);
    for (int k = 0; k < m.nz; ++k)
        for (int j = 0; j < m.ny; ++j)
            for (int i = 0; i < m.nx; ++i) t.mask[m.cell(i, j, k)] = m.solid_at(m.xc(i), m.yc(j), m.zc(k)) ? 1 : 0;
    const double h = m.ball ? std::max({m.dx, m.dy, m.dz}) : std::max(m.dx, m.dy);
    const int dkmax = d3 ? 2 : 0;
    const auto solid = [&](int i, int j, int k) { return t.mask[m.cell(i, j, k)] != 0; };
    std::vector<unsigned char> is_ghost(n, 0);
    for (int k = 0; k < m.nz; ++k)
        for (int j = 0; j < m.ny; ++j)
            for (int i = 0; i < m.nx; ++i) {
                if (!solid(i, j, k)) continue;
                bool near = false;
                for (int dk = -dkmax; dk <= dkmax && !near; ++dk)
                    for (int dj = -2; dj <= 2 && !near; ++dj)
                        for (int di = -2; di <= 2 && !near; ++di) {
                            const int ii = i + di, jj = j + dj, kk = k + dk;
                            if (ii >= 0 && ii < m.nx && jj >= 0 && jj < m.ny && kk >= 0 && kk < m.nz && !solid(ii, jj, kk)) near = true;
                        }
                if (!near) continue;
                double wx, wy, wz = 0.0, gx, gy, gz = 0.0;
                const double x = m.xc(i), y = m.yc(j), z = m.zc(k);
                if (m.ball) {   // closest_wall_point3
                    const double ex = x - m.cx, ey = y - m.cy, ez = z - m.cz, d = std::sqrt(ex * ex + ey * ey + ez * ez);
                    gx = d > 0.0 ? ex / d : 1.0;
                    gy = d > 0.0 ? ey / d : 0.0;
                    gz = d > 0.0 ? ez / d : 0.0;
                    wx = m.cx + m.r * gx;
                    wy = m.cy + m.r * gy;
                    wz = m.cz + m.r * gz;
                } else {        // closest_wall_point
                    const double ex = x - m.cx, ey = y - m.cy, d = std::sqrt(ex * ex + ey * ey);
                    gx = d > 0.0 ? ex / d : 1.0;
                    gy = d > 0.0 ? ey / d : 0.0;
                    wx = m.cx + m.r * gx;
                    wy = m.cy + m.r * gy;
                }
                const double ez = m.ball ? z - wz : 0.0;
                const double dg = std::sqrt((x - wx) * (x - wx) + (y - wy) * (y - wy) + ez * ez);
                int cell[8];
                double w[8];
                bool found = false;
                double di = 0.0;
                for (di = dmax_(dg, 1.5 * h); di <= 4.0 * h + 1e-12; di += 0.5 * h) {
                    found = m.ball ? make_probe3(m, t.mask, wx + di * gx, wy + di * gy, wz + di * gz, cell, w)
                                   : make_probe(m, t.mask, wx + di * gx, wy + di * gy, k, cell, w);
                    if (found) break;
                }
                double ratio;
                if (!found) {
                    double best = 1e300;
                    int cn = -1;
                    for (int dk = -dkmax; dk <= dkmax; ++dk)
                        for (int dj = -2; dj <= 2; ++dj)
                            for (int dii = -2; dii <= 2; ++dii) {
                                const int ii = i + dii, jj = j + dj, kk = k + dk;
                                if (ii < 0 || ii >= m.nx || jj < 0 || jj >= m.ny || kk < 0 || kk >= m.nz || solid(ii, jj, kk)) continue;
                                const double ex2 = dii * m.dx, ey2 = dj * m.dy, ez2 = d3 ? dk * m.dz : 0.0;
                                const double d2 = ex2 * ex2 + ey2 * ey2 + ez2 * ez2;
                                if (d2 < best) {
                                    best = d2;
                                    cn = static_cast<int>(m.cell(ii, jj, kk));
                                }
                            }
                    for (int q = 0; q < 8; ++q) {
                        cell[q] = cn;
                        w[q] = q == 0 ? 1.0 : 0.0;
                    }
                    ratio = 0.0;
                    ++t.fallback;
                } else {
                    ratio = dg / di;
                }
                t.ghost.push_back(static_cast<int>(m.cell(i, j, k)));
                for (int q = 0; q < 8; ++q) {
                    t.img_cell.push_back(cell[q]);
                    t.img_w.push_back(w[q]);
                }
                t.ratio.push_back(ratio);
                t.span.push_back(found ? dg + di : 0.0);
                t.gnx.push_back(gx);
                t.gny.push_back(gy);
                t.gnz.push_back(gz);
                t.gwx.push_back(wx);
                t.gwy.push_back(wy);
                t.gwz.push_back(m.ball ? wz : z);   // (a cylinder's wall point is at the cell's z)
                is_ghost[m.cell(i, j, k)] = 1;
            }
    for (size_t cc = 0; cc < n; ++cc)
        if (t.mask[cc] && !is_ghost[cc]) t.deep.push_back(static_cast<int>(cc));
    return "";
}

// The cells a moving body has left, to be given the state of the wall layer (ImmersedBoundary::build_fresh,
// Physics.cpp:1230-1290): per cell the image probe on the normal through its closest wall point (reading settled fluid
// only: the fresh cells count as solid meanwhile), the ratio of the distances, and the wall velocity at the wall point.
struct FreshTable {
    std::vector<int> cell, img_cell;
    std::vector<double> img_w, ratio, wvel;   // img: 8 per cell; wvel: 3 per cell
};

template <class WallVelocity>
inline void build_fresh(const IbmGeom& m, std::vector<unsigned char>& mask, const std::vector<int>& cells, WallVelocity vel, FreshTable& f) {
    f = FreshTable();
    for (const int c : cells) mask[c] = 1;
    const bool d3 = m.nz > 1;
    const double hh = d3 ? dmax_(dmax_(m.dx, m.dy), m.dz) : dmax_(m.dx, m.dy);
    for (const int c : cells) {
        const int i = c % m.nx, j = (c / m.nx) % m.ny, k = c / (m.nx * m.ny);
        const double x = m.xc(i), y = m.yc(j), z = m.zc(k);
        double wx, wy, wz = 0.0, gx, gy, gz = 0.0, dg;
        if (d3) {   // closest_wall_point3
            if (m.ball) {
                const double ex = x - m.cx, ey = y - m.cy, ez = z - m.cz, d = std::sqrt(ex * ex + ey * ey + ez * ez);
                gx = d > 0.0 ? ex / d : 1.0;
                gy = d > 0.0 ? ey / d : 0.0;
                gz = d > 0.0 ? ez / d : 0.0;
                wx = m.cx + m.r * gx;
                wy = m.cy + m.r * gy;
                wz = m.cz + m.r * gz;
            } else {
                const double ex = x - m.cx, ey = y - m.cy, d = std::sqrt(ex * ex + ey * ey);
                gx = d > 0.0 ? ex / d : 1.0;
                gy = d > 0.0 ? ey / d : 0.0;
                wx = m.cx + m.r * gx;
                wy = m.cy + m.r * gy;
                wz = z;
            }
            dg = std::sqrt((x - wx) * (x - wx) + (y - wy) * (y - wy) + (z - wz) * (z - wz));
        } else {    // closest_wall_point
            const double ex = x - m.cx, ey = y - m.cy, d = std::sqrt(ex * ex + ey * ey);
            gx = d > 0.0 ? ex / d : 1.0;
            gy = d > 0.0 ? ey / d : 0.0;
            wx = m.cx + m.r * gx;
            wy = m.cy + m.r * gy;
            dg = std::hypot(x - wx, y - wy);
        }
        double wv[3];
        vel(wx, wy, wz, wv);
        int cell[8];
        double w[8];
        bool found = false;
        double d = 0.0;
        for (d = dmax_(dg + hh, 1.5 * hh); d <= 4.0 * hh + dg + 1e-12; d += 0.5 * hh) {
            found = d3 ? make_probe3(m, mask, wx + d * gx, wy + d * gy, wz + d * gz, cell, w) : make_probe(m, mask, wx + d * gx, wy + d * gy, k, cell, w);
            if (found) break;
        }
        double ratio;
        if (found) {
            ratio = dg / d;
        } else {   // the nearest settled fluid cell of the two-cell neighbourhood, at the wall velocity
            double best = 1e300;
            int cn = c;
            for (int dk = d3 ? -2 : 0; dk <= (d3 ? 2 : 0); ++dk)
                for (int dj = -2; dj <= 2; ++dj)
                    for (int di = -2; di <= 2; ++di) {
                        const int ii = i + di, jj = j + dj, kk = k + dk;
                        if (ii < 0 || ii >= m.nx || jj < 0 || jj >= m.ny || kk < 0 || kk >= m.nz || mask[m.cell(ii, jj, kk)]) continue;
                        const double d2 = static_cast<double>(di * di + dj * dj + dk * dk);
                        if (d2 < best) {
                            best = d2;
                            cn = static_cast<int>(m.cell(ii, jj, kk));
                        }
                    }
            for (int q = 0; q < 8; ++q) {
                cell[q] = cn;
                w[q] = q == 0 ? 1.0 : 0.0;
            }
            ratio = 0.0;
        }
        f.cell.push_back(c);
        for (int q = 0; q < 8; ++q) {
            f.img_cell.push_back(cell[q]);
            f.img_w.push_back(w[q]);
        }
        f.ratio.push_back(ratio);
        for (int q = 0; q < 3; ++q) f.wvel.push_back(wv[q]);
    }
    for (const int c : cells) mask[c] = 0;
}

}   // namespace fvg
