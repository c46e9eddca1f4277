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

inline double dmax_(double a, double b) { return (a < b) ? b : a; }
inline double dmin_(double a, double b) { return (b < a) ? b : a; }

// Polygon2D::contains (cpp/src/Geometry.cpp:30-38): the even-odd rule
inline bool poly_contains(const std::vector<double>& P, double x, double y) {
    bool in = false;
    const size_t n = P.size() / 2;
    for (size_t i = 0, j = n - 1; i < n; j = i++) {
        const double xi = P[2 * i], yi = P[2 * i + 1], xj = P[2 * j], yj = P[2 * j + 1];
        if ((yi > y) != (yj > y) && x < (xj - xi) * (y - yi) / (yj - yi) + xi) in = !in;
    }
    return in;
}

struct IbmGeom {
    bool ball = false;   // a sphere in 3-D; otherwise a circle (2-D) or a cylinder along z (3-D) ...
    bool poly = false;   // ... or a polygon section (an airfoil; extruded along z in 3-D)
    double cx = 0, cy = 0, cz = 0, r = 0;
    std::vector<double> pts;                    // the polygon's vertices (x, y) where it is placed
    double px0 = 0, px1 = 0, py0 = 0, py1 = 0;  // and its bounding box
    int nx = 0, ny = 0, nz = 0;
    double dx = 0, dy = 0, dz = 0;
    size_t cell(int i, int j, int k) const { return (static_cast<size_t>(k) * ny + j) * nx + i; }
    double xc(int i) const { return (i + 0.5) * dx + 0.0; }
    double yc(int j) const { return (j + 0.5) * dy + 0.0; }
    double zc(int k) const { return (k + 0.5) * dz + 0.0; }
    void set_polygon(std::vector<double> p) {   // the bounding box as ImmersedBoundary's polygon constructor takes it
        pts = std::move(p);
        double x0 = 1e300, x1 = -1e300, y0 = 1e300, y1 = -1e300;
        for (size_t q = 0; q < pts.size() / 2; ++q) {
            x0 = dmin_(x0, pts[2 * q]);
            x1 = dmax_(x1, pts[2 * q]);
            y0 = dmin_(y0, pts[2 * q + 1]);
            y1 = dmax_(y1, pts[2 * q + 1]);
        }
        px0 = x0;
        px1 = x1;
        py0 = y0;
        py1 = y1;
    }
    // ImmersedBoundary::solid_at (cpp/src/Physics.cpp:892-907)
    bool solid_at(double x, double y, double z) const {
        if (poly) return !(x < px0 || x > px1 || y < py0 || y > py1 || !poly_contains(pts, x, y));
        if (ball) {
            const double dxc = x - cx, dyc = y - cy;
            const double r2 = dxc * dxc + dyc * dyc + (z - cz) * (z - cz);
            return std::sqrt(r2) <= r;
        }
        const double dxc = x - cx, dyc = y - cy;
        const double r2 = dxc * dxc + dyc * dyc;
        return std::sqrt(r2) <= r;
    }
    // ImmersedBoundary::closest_wall_point (Physics.cpp:989-1034): the wall point nearest to (x, y) and the outward normal
    void closest_wall_point(double x, double y, double& wx, double& wy, double& gx, double& gy) const {
        if (!poly) {
            const double ex = x - cx, ey = y - cy, d = std::sqrt(ex * ex + ey * ey);
            gx = d > 0.0 ? ex / d : 1.0;
            gy = d > 0.0 ? ey / d : 0.0;
            wx = cx + r * gx;
            wy = cy + r * gy;
            return;
        }
        const size_t n = pts.size() / 2;
        double best = 1e300;
        size_t seg = 0;
        wx = wy = 0.0;
        for (size_t k = 0; k < n; ++k) {
            const double ax = pts[2 * k], ay = pts[2 * k + 1], bx = pts[2 * ((k + 1) % n)], by = pts[2 * ((k + 1) % n) + 1];
            const double ox = dmax_(dmax_(dmin_(ax, bx) - x, x - dmax_(ax, bx)), 0.0);
            const double oy = dmax_(dmax_(dmin_(ay, by) - y, y - dmax_(ay, by)), 0.0);
            if (ox * ox + oy * oy > best * (1.0 + 1e-9)) continue;   // cannot win
            const double ex = bx - ax, ey = by - ay, l2 = ex * ex + ey * ey;
            double t = l2 > 0.0 ? ((x - ax) * ex + (y - ay) * ey) / l2 : 0.0;
            t = dmin_(1.0, dmax_(0.0, t));
            const double qx = ax + t * ex, qy = ay + t * ey, d2 = (x - qx) * (x - qx) + (y - qy) * (y - qy);
            if (d2 < best) {
                best = d2;
                wx = qx;
                wy = qy;
                seg = k;
            }
        }
        const double d = std::sqrt(best);
        const bool inside = poly_contains(pts, x, y);
        if (d > 1e-12) {   // outward: from the point to the wall if it is inside, from the wall to the point if outside
            gx = (inside ? wx - x : x - wx) / d;
            gy = (inside ? wy - y : y - wy) / d;
            return;
        }
        const double ax = pts[2 * seg], ay = pts[2 * seg + 1], bx = pts[2 * ((seg + 1) % n)], by = pts[2 * ((seg + 1) % n) + 1];
        const double ex = bx - ax, ey = by - ay, l = std::sqrt(ex * ex + ey * ey);   // on the wall: the segment normal, pointing out
        gx = ey / l;
        gy = -ex / l;
        if (poly_contains(pts, wx + 1e-6 * l * gx, wy + 1e-6 * l * gy)) {
            gx = -gx;
            gy = -gy;
        }
    }
};

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

// place_airfoil (cpp/src/Geometry.cpp:143-152): the unit section of the configuration (leading edge at the origin, chord 1)
// scaled to ibm_chord, its quarter chord at (ibm_cx, ibm_cy), turned clockwise by ibm_aoa degrees (nose up).
inline std::vector<double> place_section(const fvg_config& c, std::string& err) {
    std::vector<double> out;
    if (!c.ibm_section || c.ibm_section_points < 3) {
        err = "an airfoil section needs at least 3 points (ibm_section)";
        return out;
    }
    if (!(c.ibm_chord > 0.0)) {
        err = "ibm_chord must be > 0";
        return out;
    }
    const double a = c.ibm_aoa * 3.14159265358979323846 / 180.0, ca = std::cos(a), sa = std::sin(a);
    for (int q = 0; q < c.ibm_section_points; ++q) {
        const double x = (c.ibm_section[2 * q] - 0.25) * c.ibm_chord, y = c.ibm_section[2 * q + 1] * c.ibm_chord;
        out.push_back(c.ibm_cx + x * ca + y * sa);
        out.push_back(c.ibm_cy - x * sa + y * ca);
    }
    return out;
}

// The body's geometry on the mesh of a configuration, its centre at (cx, cy, cz) (a moving body: its placement plus the
// displacement of its pose, ImmersedBoundary::place_geometry, cpp/src/Physics.cpp:1162-1194).
inline IbmGeom ibm_geom(const fvg_config& c, double cx, double cy, double cz) {
    IbmGeom m;
    m.ball = c.nz > 1 && c.ibm_shape == 1;
    m.poly = c.ibm_shape == 2;
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
    if (c.ibm_shape < 0 || c.ibm_shape > 2) return "ibm_shape: Cylinder, Sphere or a section (airfoil) on the device";
    if (c.ibm_curvature) return "ibm_curvature is not supported on the device";
    IbmGeom g = ibm_geom(c, c.ibm_cx, c.ibm_cy, c.ibm_cz);
    if (g.poly) {
        std::string err;
        g.set_polygon(place_section(c, err));
        if (!err.empty()) return err;
    }
    return build_ibm_geom(g, t);
}

// The mask and the ghost table of the body of geometry m (ImmersedBoundary::build_ghosts, Physics.cpp:1397-1537).
inline std::string build_ibm_geom(const IbmGeom& m, IbmTable& t) {
    const bool d3 = m.nz > 1;
    if (m.nx < 2 || m.ny < 2 || (m.ball && m.nz < 2)) return "the immersed body needs at least two cells per axis";
    const size_t n = static_cast<size_t>(m.nx) * m.ny * m.nz;
    t = IbmTable();
    t.mask.assign(n, 0);
    if (m.poly) {   // a section: the same in every layer
        for (int j = 0; j < m.ny; ++j)
            for (int i = 0; i < m.nx; ++i) {
                if (!m.solid_at(m.xc(i), m.yc(j), 0.0)) continue;
                for (int k = 0; k < m.nz; ++k) t.mask[m.cell(i, j, k)] = 1;
            }
    } else {
        for (int k = 0; k < m.nz; ++k)
            for (int j = 0; j < m.ny; ++j)
                for (int i = 0; i < m.nx; ++i) t.mask[m.cell(i, j, k)] = m.solid_at(m.xc(i), m.yc(j), m.zc(k)) ? 1 : 0;
    }
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
                } else {
                    m.closest_wall_point(x, y, wx, wy, gx, gy);
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
                t.gwz.push_back(wz);
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
            } else {   // a cylinder or a section extruded along z
                m.closest_wall_point(x, y, wx, wy, gx, gy);
                wz = z;
            }
            dg = std::sqrt((x - wx) * (x - wx) + (y - wy) * (y - wy) + (z - wz) * (z - wz));
        } else {
            m.closest_wall_point(x, y, wx, wy, gx, gy);
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
