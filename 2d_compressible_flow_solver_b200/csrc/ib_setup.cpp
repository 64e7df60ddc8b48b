// Host-side immersed-boundary set-up.  Built with -ffp-contract=off so that
// the classification, image points and donor lists reproduce the reference's
// doubles exactly (Circle.cpp uses only + - * / sqrt, cos and sin).
#include "ib_setup.h"

#include "cfs_layout.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>
#include <utility>

namespace cfs {

namespace {

struct P2 {
    double x, y;
};

// v / sqrt(v.v) when v.v > 0, else v (Eigen's normalized()).
inline P2 normalized(P2 v) {
    const double z = v.x * v.x + v.y * v.y;
    if (z > 0.0) {
        const double n = std::sqrt(z);
        return {v.x / n, v.y / n};
    }
    return v;
}

inline double norm(P2 v) { return std::sqrt(v.x * v.x + v.y * v.y); }

}  // namespace

void circle_polygon(double radius, double cx, double cy, int npoints, std::vector<double>& pts_xy,
                    std::vector<double>& dir_xy) {
    // Circle::Initialize (Circle.cpp:12-41): polygon vertices and unit segment
    // directions (segment k runs from vertex k to vertex k+1).
    pts_xy.assign(2 * static_cast<size_t>(npoints), 0.0);
    dir_xy.assign(2 * static_cast<size_t>(npoints), 0.0);
    for (int k = 0; k < npoints; ++k) {
        const double angle = 2.0 * M_PI * static_cast<double>(k) / static_cast<double>(npoints);
        pts_xy[2 * k] = cx + radius * std::cos(angle);
        pts_xy[2 * k + 1] = cy + radius * std::sin(angle);
    }
    for (int k = 0; k < npoints; ++k) {
        const int k1 = (k + 1) % npoints;
        const P2 d = normalized({pts_xy[2 * k1] - pts_xy[2 * k], pts_xy[2 * k1 + 1] - pts_xy[2 * k + 1]});
        dir_xy[2 * k] = d.x;
        dir_xy[2 * k + 1] = d.y;
    }
}

bool select_donors(const uint8_t* t, int nx, int ny, double dx, double dy, const std::vector<int32_t>& cells,
                   const std::vector<double>& image, std::vector<int32_t>& donor, std::string& err) {
    // FindNearest4FluidCellsIndexed (Circle.cpp:160-215): fluid cells of the
    // 11 x 11 window around the image point's cell, visited i outer / j inner,
    // sorted by squared distance with the same comparator.
    auto centre = [&](int i, int j) { return P2{(i + 0.5) * dx, (j + 0.5) * dy}; };  // CartesianMesh.cpp:92
    const P2 origin = centre(0, 0);
    donor.clear();
    donor.reserve(4 * cells.size());
    std::vector<std::pair<double, int>> cand;
    for (size_t g = 0; g < cells.size(); ++g) {
        const P2 img{image[2 * g], image[2 * g + 1]};
        const int ic = static_cast<int>((img.x - origin.x) / dx);
        const int jc = static_cast<int>((img.y - origin.y) / dy);
        cand.clear();
        for (int a = ic - 5; a <= ic + 5; ++a)
            for (int b = jc - 5; b <= jc + 5; ++b) {
                if (a >= 0 && a < nx && b >= 0 && b < ny && t[static_cast<size_t>(a) * ny + b] == 0) {
                    const P2 c = centre(a, b);
                    const double ddx = c.x - img.x, ddy = c.y - img.y;
                    cand.emplace_back(ddx * ddx + ddy * ddy, a * ny + b);
                }
            }
        std::sort(cand.begin(), cand.end(),
                  [](const std::pair<double, int>& p, const std::pair<double, int>& q) { return p.first < q.first; });
        if (cand.size() < 4) {
            const int i = cells[g] / ny, j = cells[g] % ny;
            err = "immersed-ghost cell (" + std::to_string(i) + ", " + std::to_string(j) + ") has " +
                  std::to_string(cand.size()) + " fluid donors, 4 needed";
            return false;
        }
        for (int k = 0; k < 4; ++k) donor.push_back(cand[k].second);
    }
    return true;
}

void mark_ghosts(std::vector<uint8_t>& t, int nx, int ny) {
    // SetGhostcell(cells, 3) (Circle.cpp:53-103): from every fluid cell, walk
    // each axis direction into solid/ghost cells and mark up to 3 as ghosts.
    const int dirs[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
    auto at = [&](int i, int j) -> uint8_t& { return t[static_cast<size_t>(i) * ny + j]; };
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            if (at(i, j) != 0) continue;
            for (const auto& d : dirs) {
                const int ni = i + d[0], nj = j + d[1];
                if (ni >= 0 && ni < nx && nj >= 0 && nj < ny && at(ni, nj) != 0) {
                    for (int k = 1; k <= 3; ++k) {
                        const int gi = i + k * d[0], gj = j + k * d[1];
                        if (gi >= 0 && gi < nx && gj >= 0 && gj < ny && at(gi, gj) != 0) at(gi, gj) = 2;
                        else break;
                    }
                }
            }
        }
}

bool build_polygon(int nx, int ny, double lx, double ly, const std::vector<double>& xy, IbList& out,
                   std::string& err) {
    const int np = static_cast<int>(xy.size() / 2);
    if (np < 3 || xy.size() != 2 * static_cast<size_t>(np)) {
        err = "a polygon needs at least 3 vertices (x, y pairs)";
        return false;
    }
    for (double v : xy)
        if (!std::isfinite(v)) {
            err = "polygon vertex not finite";
            return false;
        }
    const double dx = lx / nx, dy = ly / ny;
    auto centre = [&](int i, int j) { return P2{(i + 0.5) * dx, (j + 0.5) * dy}; };  // CartesianMesh.cpp:92
    // solid iff the centre is inside (even-odd rule: crossings of a ray to +x)
    std::vector<uint8_t>& t = out.types;
    t.assign(static_cast<size_t>(nx) * ny, 0);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const P2 p = centre(i, j);
            bool inside = false;
            for (int k = 0, m = np - 1; k < np; m = k++) {
                const double xk = xy[2 * k], yk = xy[2 * k + 1], xm = xy[2 * m], ym = xy[2 * m + 1];
                if ((yk > p.y) != (ym > p.y) && p.x < (xm - xk) * (p.y - yk) / (ym - yk) + xk) inside = !inside;
            }
            if (inside) t[static_cast<size_t>(i) * ny + j] = 1;
        }
    mark_ghosts(t, nx, ny);
    // image point: the mirror of the ghost centre in its nearest boundary
    // point (projection onto each segment, clamped to it; the first segment
    // wins ties)
    out.cell.clear();
    out.image.clear();
    out.normal.clear();
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            if (t[static_cast<size_t>(i) * ny + j] != 2) continue;
            const P2 pos = centre(i, j);
            double best = std::numeric_limits<double>::max();
            P2 q{pos.x, pos.y};
            for (int k = 0; k < np; ++k) {
                const int k1 = (k + 1) % np;
                const P2 a{xy[2 * k], xy[2 * k + 1]}, b{xy[2 * k1], xy[2 * k1 + 1]};
                const P2 ab{b.x - a.x, b.y - a.y};
                const double len2 = ab.x * ab.x + ab.y * ab.y;
                double u = len2 > 0.0 ? ((pos.x - a.x) * ab.x + (pos.y - a.y) * ab.y) / len2 : 0.0;
                u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
                const P2 c{a.x + u * ab.x, a.y + u * ab.y};
                const double dist = norm({c.x - pos.x, c.y - pos.y});
                if (dist < best) {
                    best = dist;
                    q = c;
                }
            }
            const P2 n = normalized({q.x - pos.x, q.y - pos.y});
            out.cell.push_back(i * ny + j);
            out.image.push_back(pos.x + 2 * (best * n.x));
            out.image.push_back(pos.y + 2 * (best * n.y));
            out.normal.push_back(n.x);
            out.normal.push_back(n.y);
        }
    return select_donors(t.data(), nx, ny, dx, dy, out.cell, out.image, out.donor, err);
}

bool build_circle(int nx, int ny, double lx, double ly, double radius, double cx, double cy, int npoints,
                  IbList& out, std::string& err) {
    if (npoints < 3) {
        err = "circle needs at least 3 polygon points";
        return false;
    }
    const double dx = lx / nx, dy = ly / ny;  // CartesianMesh::CalCellsize (CartesianMesh.cpp:150-154)
    auto centre = [&](int i, int j) { return P2{(i + 0.5) * dx, (j + 0.5) * dy}; };  // CartesianMesh.cpp:92
    std::vector<double> pts, dir;
    circle_polygon(radius, cx, cy, npoints, pts, dir);

    // DistinguishWallandFluid (Circle.cpp:43-51): solid iff |x_c - c| <= r.
    std::vector<uint8_t>& t = out.types;
    t.assign(static_cast<size_t>(nx) * ny, 0);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const P2 p = centre(i, j);
            if (norm({p.x - cx, p.y - cy}) <= radius) t[static_cast<size_t>(i) * ny + j] = 1;
        }

    mark_ghosts(t, nx, ny);
    auto at = [&](int i, int j) -> uint8_t& { return t[static_cast<size_t>(i) * ny + j]; };

    out.cell.clear();
    out.image.clear();
    out.normal.clear();
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            if (at(i, j) != 2) continue;
            // SetImagepoint (Circle.cpp:105-138): nearest segment line by
            // orthogonal projection (strictly smaller distance wins), mirror.
            const P2 pos = centre(i, j);
            double minDistance = std::numeric_limits<double>::max();
            P2 intercept{0.0, 0.0};
            for (int k = 0; k < npoints; ++k) {
                const P2 s{dir[2 * k], dir[2 * k + 1]}, a{pts[2 * k], pts[2 * k + 1]};
                const double dd = s.x * (pos.x - a.x) + s.y * (pos.y - a.y);
                const P2 proj{dd * s.x + a.x, dd * s.y + a.y};
                const double dist = norm({proj.x - pos.x, proj.y - pos.y});
                if (dist < minDistance) {
                    minDistance = dist;
                    intercept = proj;
                }
            }
            const P2 n = normalized({intercept.x - pos.x, intercept.y - pos.y});
            out.cell.push_back(i * ny + j);
            out.image.push_back(pos.x + 2 * (minDistance * n.x));
            out.image.push_back(pos.y + 2 * (minDistance * n.y));
            out.normal.push_back(n.x);
            out.normal.push_back(n.y);
        }
    return select_donors(t.data(), nx, ny, dx, dy, out.cell, out.image, out.donor, err);
}

// Outer-product LDL^T with symmetric diagonal pivoting (largest remaining
// |diagonal| first; Golub & Van Loan 4.1/4.4, Higham ch. 10-11), reading the
// lower triangle only, as Eigen documents for ldlt().
void ldlt4_lower(const double M[4][4], double fac[10], int perm[4]) {
    double w[4][4], l[4][4], d[4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            w[r][c] = (r >= c) ? M[r][c] : M[c][r];
            l[r][c] = 0.0;
        }
    for (int k = 0; k < 4; ++k) perm[k] = k;
    for (int k = 0; k < 4; ++k) {
        int p = k;
        double best = std::fabs(w[k][k]);
        for (int i = k + 1; i < 4; ++i) {
            const double v = std::fabs(w[i][i]);
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (p != k) {
            for (int c = 0; c < 4; ++c) std::swap(w[k][c], w[p][c]);
            for (int r = 0; r < 4; ++r) std::swap(w[r][k], w[r][p]);
            for (int c = 0; c < k; ++c) std::swap(l[k][c], l[p][c]);
            std::swap(perm[k], perm[p]);
        }
        const double dk = w[k][k];
        d[k] = dk;
        const bool usable = std::fabs(dk) > DBL_MIN;
        for (int i = k + 1; i < 4; ++i) l[i][k] = usable ? w[i][k] / dk : 0.0;
        for (int i = k + 1; i < 4; ++i)
            for (int j = k + 1; j < 4; ++j) w[i][j] = w[i][j] - l[i][k] * dk * l[j][k];
    }
    fac[0] = l[1][0];
    fac[1] = l[2][0];
    fac[2] = l[2][1];
    fac[3] = l[3][0];
    fac[4] = l[3][1];
    fac[5] = l[3][2];
    for (int k = 0; k < 4; ++k) fac[6 + k] = d[k];
}

void slip_donors(const uint8_t* types, int nx, int ny, double dx, double dy, double X, double Y,
                 const int32_t fallback[4], int32_t donor[4], double w[4]) {
    const double fx = (X - 0.5 * dx) / dx, fy = (Y - 0.5 * dy) / dy;
    const int i0 = static_cast<int>(std::floor(fx)), j0 = static_cast<int>(std::floor(fy));
    const double tx = fx - i0, ty = fy - j0;
    const int ci[4] = {i0, i0 + 1, i0, i0 + 1};
    const int cj[4] = {j0, j0, j0 + 1, j0 + 1};
    const double cw[4] = {(1 - tx) * (1 - ty), tx * (1 - ty), (1 - tx) * ty, tx * ty};
    int keep = -1;
    double sum = 0.0;
    for (int k = 0; k < 4; ++k) {
        const bool ok = ci[k] >= 0 && ci[k] < nx && cj[k] >= 0 && cj[k] < ny &&
                        types[static_cast<size_t>(ci[k]) * ny + cj[k]] == 0;
        donor[k] = ok ? ci[k] * ny + cj[k] : -1;
        w[k] = ok ? cw[k] : 0.0;
        if (ok) {
            sum += cw[k];
            if (keep < 0) keep = k;
        }
    }
    if (sum > 1e-3) {
        for (int k = 0; k < 4; ++k) {
            if (donor[k] < 0) donor[k] = donor[keep];
            w[k] = w[k] / sum;
        }
        return;
    }
    double s = 0.0;
    for (int k = 0; k < 4; ++k) {
        const int i = fallback[k] / ny, j = fallback[k] % ny;
        const double ddx = (i + 0.5) * dx - X, ddy = (j + 0.5) * dy - Y;
        w[k] = 1.0 / (ddx * ddx + ddy * ddy + 1e-300);
        donor[k] = fallback[k];
        s += w[k];
    }
    for (int k = 0; k < 4; ++k) w[k] /= s;
}

void ib_factors(int mode, const uint8_t* types, int nx, int ny, double dx, double dy, int n, const int32_t* donor4,
                const double* image, const double* normal, std::vector<int32_t>& dev_donor, std::vector<double>& fac,
                std::vector<int>& perm) {
    fac.assign(16 * static_cast<size_t>(n), 0.0);
    perm.assign(4 * static_cast<size_t>(n), 0);
    dev_donor.assign(donor4, donor4 + 4 * static_cast<size_t>(n));
    for (int g = 0; g < n; ++g) {
        if (mode == 0) {
            double M[4][4];
            for (int k = 0; k < 4; ++k) {
                const int d = donor4[4 * g + k];
                const int i = d / ny, j = d % ny;
                const double x = (i + 0.5) * dx, y = (j + 0.5) * dy;  // CartesianMesh.cpp:92
                M[k][0] = x * y;
                M[k][1] = x;
                M[k][2] = y;
                M[k][3] = 1.0;
            }
            ldlt4_lower(M, &fac[16 * g], &perm[4 * g]);
        } else {
            double w[4];
            slip_donors(types, nx, ny, dx, dy, image[2 * g], image[2 * g + 1], &donor4[4 * g], &dev_donor[4 * g], w);
            for (int k = 0; k < 4; ++k) fac[16 * g + k] = w[k];
            fac[16 * g + 4] = normal[2 * g];
            fac[16 * g + 5] = normal[2 * g + 1];
        }
    }
}

static inline int face_slot(int a, int k, int n, bool lo_rule, bool hi_rule) {
    int i = a - 3 + k;
    if (a == 0 && lo_rule && k >= 3) i = 0;
    if (a == n && hi_rule && k <= 2) i = n - 1;
    return i;
}

std::vector<uint8_t> low_order_faces(const uint8_t* types, int nx, int ny, const int bc[4]) {
    auto rule = [&](int s) { return bc[s] == 0 || bc[s] == 1; };  // Neumann or Dirichlet side
    std::vector<uint8_t> f(static_cast<size_t>(nx + 1) * (ny + 1), 0);
    for (int a = 0; a <= nx; ++a)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < 6; ++k) {
                const int i = face_slot(a, k, nx, rule(0), rule(1));
                if (i >= 0 && i < nx && types[static_cast<size_t>(i) * ny + j]) {
                    f[static_cast<size_t>(a) * (ny + 1) + j] |= 1;
                    break;
                }
            }
    for (int i = 0; i < nx; ++i)
        for (int a = 0; a <= ny; ++a)
            for (int k = 0; k < 6; ++k) {
                const int j = face_slot(a, k, ny, rule(2), rule(3));
                if (j >= 0 && j < ny && types[static_cast<size_t>(i) * ny + j]) {
                    f[static_cast<size_t>(i) * (ny + 1) + a] |= 2;
                    break;
                }
            }
    return f;
}

std::vector<uint8_t> cell_flags(const uint8_t* types, const uint8_t* lowo, int nx, int ny) {
    const int w = ny + 2;
    std::vector<uint8_t> f(static_cast<size_t>(nx + 2) * w, 0);
    auto face = [&](int i, int j) { return lowo[static_cast<size_t>(i) * (ny + 1) + j]; };
    for (int i = -1; i <= nx; ++i)
        for (int j = -1; j <= ny; ++j) {
            const bool in_i = i >= 0 && i < nx, in_j = j >= 0 && j < ny;
            uint8_t b = 0;
            if (in_i && in_j && types[static_cast<size_t>(i) * ny + j]) b |= kCellSolid;
            if (lowo) {
                if (in_j && i >= 0 && i <= nx && (face(i, j) & 1)) b |= kCellLowXlo;
                if (in_j && i + 1 >= 0 && i + 1 <= nx && (face(i + 1, j) & 1)) b |= kCellLowXhi;
                if (in_i && j >= 0 && j <= ny && (face(i, j) & 2)) b |= kCellLowYlo;
                if (in_i && j + 1 >= 0 && j + 1 <= ny && (face(i, j + 1) & 2)) b |= kCellLowYhi;
            }
            f[static_cast<size_t>(i + 1) * w + (j + 1)] = b;
        }
    return f;
}

}  // namespace cfs
