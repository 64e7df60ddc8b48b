// Host-side immersed-boundary set-up (one-time, not per stage).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace cfs {

struct IbList {
    std::vector<uint8_t> types;    // [nx*ny] 0 fluid, 1 solid, 2 immersed ghost
    std::vector<int32_t> cell;     // [n] i*ny + j, i outer / j inner order
    std::vector<int32_t> donor;    // [4n] i*ny + j, nearest first
    std::vector<double> image;     // [2n]
    std::vector<double> normal;    // [2n] unit vector from the ghost centre to its image point
};

// Circle immersed boundary as the reference builds it (Circle.cpp:12-215,
// called from CartesianMesh::setImmersedBoundary, CartesianMesh.cpp:357-374).
// Returns false with a message when an immersed-ghost cell has fewer than 4
// fluid donors in its 11 x 11 window.
bool build_circle(int nx, int ny, double lx, double ly, double radius, double cx, double cy, int npoints,
                  IbList& out, std::string& err);

// Pivoted LDL^T of the symmetric matrix read from the lower triangle of M
// (Eigen's ldlt(), ImagePoint.cpp:44): fac = l10 l20 l21 l30 l31 l32 d0 d1 d2 d3.
void ldlt4_lower(const double M[4][4], double fac[10], int perm[4]);

// Weights w with w . f equal to the bilinear interpolant of the donor values f
// at (X, Y): solves M^T w = (XY, X, Y, 1) with partial pivoting.
// Returns false when M is singular.
bool bilinear_weights(const double M[4][4], double X, double Y, double w[4]);

}  // namespace cfs
