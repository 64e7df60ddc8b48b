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

// The same set-up with the per-cell work on the device (ib_device.cu):
// classification, ghost marking and image points as kernels (bit for bit the
// host doubles: built without FMA contraction), donors on the host from the
// read-back types (the reference's sort order).  Uses the current device and
// `stream` (waits for it).
bool build_circle_device(int nx, int ny, double lx, double ly, double radius, double cx, double cy, int npoints,
                         void* stream, IbList& out, std::string& err);

// A closed polygon body (no counterpart in the reference, whose only
// ImmersedBoundary shape is the circle): vertices xy[2*np] in order; a cell is
// solid when its centre is inside (even-odd rule); ghosts are marked as for the
// circle; a ghost's image point mirrors its centre in the nearest point of the
// boundary (projection clamped to each segment, so non-convex shapes work);
// donors as for the circle.
bool build_polygon(int nx, int ny, double lx, double ly, const std::vector<double>& xy, IbList& out,
                   std::string& err);

// Ghost marking of SetGhostcell(cells, 3) (Circle.cpp:53-103) on types 0/1 in
// place: from every fluid cell, up to 3 consecutive non-fluid cells along each
// axis direction become ghosts (2).
void mark_ghosts(std::vector<uint8_t>& types, int nx, int ny);

// Pieces shared by both: the polygon of Circle::Initialize (Circle.cpp:12-41) as
// vertex and unit-direction arrays [2*npoints]; and the 4 nearest fluid donors
// of each image point (FindNearest4FluidCellsIndexed, Circle.cpp:160-215),
// false when one has fewer than 4.
void circle_polygon(double radius, double cx, double cy, int npoints, std::vector<double>& pts_xy,
                    std::vector<double>& dir_xy);
bool select_donors(const uint8_t* types, int nx, int ny, double dx, double dy, const std::vector<int32_t>& cells,
                   const std::vector<double>& image, std::vector<int32_t>& donor, std::string& err);

// Pivoted LDL^T of the symmetric matrix read from the lower triangle of M
// (Eigen's ldlt(), ImagePoint.cpp:44): fac = l10 l20 l21 l30 l31 l32 d0 d1 d2 d3.
void ldlt4_lower(const double M[4][4], double fac[10], int perm[4]);

// Donors and weights of the slip-wall form for one image point (X, Y): the
// 2 x 2 block of cell centres around the point with tensor-product bilinear
// weights; donors that are not fluid (or off the grid) are dropped and the
// remaining weights renormalised (a dropped slot repeats a kept donor with
// weight 0).  When the kept weight is below 1e-3, inverse-squared-distance
// weights over the `fallback` donors (the reference's 4 nearest fluid cells).
// types: [nx*ny], 0 = fluid.  Donor indices are i*ny + j.
void slip_donors(const uint8_t* types, int nx, int ny, double dx, double dy, double X, double Y,
                 const int32_t fallback[4], int32_t donor[4], double w[4]);

// Device-side fill data of n immersed-ghost cells.  Reference form: the
// pivoted LDL^T factor of each donor matrix (fac[16g..16g+9], perm[4g..]).
// Slip form: slip_donors' donors (dev_donor) and weights (fac[16g..16g+3]) with
// the wall normal (fac[16g+4..5]); donor4 serve as its fallback.
void ib_factors(int mode, const uint8_t* types, int nx, int ny, double dx, double dy, int n, const int32_t* donor4,
                const double* image, const double* normal, std::vector<int32_t>& dev_donor, std::vector<double>& fac,
                std::vector<int>& perm);

// Face flags of the body positivity mode, [nx+1][ny+1] bytes: bit 0 of (i, j)
// for the x-face between cells (i-1, j) and (i, j), bit 1 for the y-face between
// (i, j-1) and (i, j).  A flag is set when a cell of the face's 6-cell stencil
// that lies in the grid is not fluid.  The stencil slots are those the stage
// kernels read, including the reference's boundary-face rule on Neumann and
// Dirichlet sides (CellInterface.cpp:172-178: every interior slot of a
// physical-boundary face is the first interior cell).  bc: cfs_bc per side.
std::vector<uint8_t> low_order_faces(const uint8_t* types, int nx, int ny, const int bc[4]);

// Per-cell flag bytes of the row march (StageArgs::cflags, kCell* bits),
// [nx+2][ny+2] for cells i = -1..nx, j = -1..ny: the cell's own type (solid
// bit) and, with face flags `lowo` (low_order_faces; null = none), the flags of
// its four faces.
std::vector<uint8_t> cell_flags(const uint8_t* types, const uint8_t* lowo, int nx, int ny);

}  // namespace cfs
