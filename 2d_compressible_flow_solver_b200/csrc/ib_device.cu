// Immersed-boundary set-up of a circle with its per-cell work on the device:
// classification (Circle::DistinguishWallandFluid, Circle.cpp:43-51), ghost
// marking (SetGhostcell(cells, 3), :53-103) and image points (SetImagepoint,
// :105-138) as kernels; donor selection (FindNearest4FluidCellsIndexed,
// :160-215) stays on the host, whose sort fixes the reference's tie order.
//
// Built with -fmad=false (no FMA contraction; division and square root
// correctly rounded), so every double is the one the host set-up computes with
// -ffp-contract=off from the same operations in the same order.
#include <cuda_runtime.h>

#include <cfloat>
#include <string>
#include <vector>

#include "ib_setup.h"

namespace cfs {
namespace {

__device__ __forceinline__ double norm2(double x, double y) { return sqrt(x * x + y * y); }

// Solid iff the cell centre lies within the radius.
__global__ void circle_classify_kernel(int nx, int ny, double dx, double dy, double radius, double cx, double cy,
                                       uint8_t* t0) {
    const long long n = static_cast<long long>(nx) * ny;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int i = static_cast<int>(k / ny), j = static_cast<int>(k - static_cast<long long>(k / ny) * ny);
        const double px = (i + 0.5) * dx, py = (j + 0.5) * dy;
        t0[k] = norm2(px - cx, py - cy) <= radius ? 1 : 0;
    }
}

// A non-fluid cell becomes an immersed ghost when, walking from it against
// one axis direction, the first fluid cell lies within 3 steps on the grid:
// the set the host's walk from every fluid cell marks, independent of order.
__global__ void ghost_mark_kernel(int nx, int ny, const uint8_t* t0, uint8_t* t) {
    const long long n = static_cast<long long>(nx) * ny;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        uint8_t v = t0[k];
        if (v != 0) {
            const int i = static_cast<int>(k / ny), j = static_cast<int>(k - static_cast<long long>(k / ny) * ny);
            const int di[4] = {1, -1, 0, 0}, dj[4] = {0, 0, 1, -1};
            for (int d = 0; d < 4 && v == 1; ++d)
                for (int m = 1; m <= 3; ++m) {
                    const int a = i - m * di[d], b = j - m * dj[d];
                    if (a < 0 || a >= nx || b < 0 || b >= ny) break;
                    if (t0[static_cast<long long>(a) * ny + b] == 0) {
                        v = 2;
                        break;
                    }
                }
        }
        t[k] = v;
    }
}

// Nearest polygon-segment line of each ghost centre (strictly smaller distance
// wins, so the first segment on ties), its image point and the unit normal.
__global__ void image_point_kernel(int n, const int32_t* cells, int ny, double dx, double dy, int npoints,
                                   const double* pts, const double* dir, double* image, double* normal) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const int c = cells[g];
    const int i = c / ny, j = c - (c / ny) * ny;
    const double px = (i + 0.5) * dx, py = (j + 0.5) * dy;
    double minDistance = DBL_MAX, ix = 0.0, iy = 0.0;
    for (int k = 0; k < npoints; ++k) {
        const double sx = dir[2 * k], sy = dir[2 * k + 1], ax = pts[2 * k], ay = pts[2 * k + 1];
        const double dd = sx * (px - ax) + sy * (py - ay);
        const double qx = dd * sx + ax, qy = dd * sy + ay;
        const double dist = norm2(qx - px, qy - py);
        if (dist < minDistance) {
            minDistance = dist;
            ix = qx;
            iy = qy;
        }
    }
    double nxv = ix - px, nyv = iy - py;
    const double z = nxv * nxv + nyv * nyv;
    if (z > 0.0) {
        const double nn = sqrt(z);
        nxv = nxv / nn;
        nyv = nyv / nn;
    }
    image[2 * g] = px + 2 * (minDistance * nxv);
    image[2 * g + 1] = py + 2 * (minDistance * nyv);
    normal[2 * g] = nxv;
    normal[2 * g + 1] = nyv;
}

struct DeviceBuffers {
    std::vector<void*> p;
    ~DeviceBuffers() {
        for (void* q : p) cudaFree(q);
    }
    template <class T>
    bool alloc(T** out, size_t count) {
        void* q = nullptr;
        if (count == 0) count = 1;
        if (cudaMalloc(&q, count * sizeof(T)) != cudaSuccess) return false;
        p.push_back(q);
        *out = static_cast<T*>(q);
        return true;
    }
};

int flat_grid(long long work) {
    const long long b = (work + 255) / 256;
    return static_cast<int>(b < 65535 * 16 ? (b > 0 ? b : 1) : 65535 * 16);
}

}  // namespace

bool build_circle_device(int nx, int ny, double lx, double ly, double radius, double cx, double cy, int npoints,
                         void* stream, IbList& out, std::string& err) {
    if (npoints < 3) {
        err = "circle needs at least 3 polygon points";
        return false;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double dx = lx / nx, dy = ly / ny;  // CartesianMesh::CalCellsize (CartesianMesh.cpp:150-154)
    const size_t ncell = static_cast<size_t>(nx) * ny;
    auto cuda_fail = [&](const char* what, cudaError_t e) {
        err = std::string("device circle set-up: ") + what + ": " + cudaGetErrorString(e);
        return false;
    };
    DeviceBuffers buf;
    uint8_t *t0 = nullptr, *t = nullptr;
    if (!buf.alloc(&t0, ncell) || !buf.alloc(&t, ncell)) return cuda_fail("allocation", cudaErrorMemoryAllocation);
    const int grid = flat_grid(static_cast<long long>(ncell));
    circle_classify_kernel<<<grid, 256, 0, s>>>(nx, ny, dx, dy, radius, cx, cy, t0);
    ghost_mark_kernel<<<grid, 256, 0, s>>>(nx, ny, t0, t);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("classification launch", e);
    out.types.assign(ncell, 0);
    e = cudaMemcpyAsync(out.types.data(), t, ncell, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail("classification", e);

    // ghost list in the reference's order (i outer, j inner)
    out.cell.clear();
    for (size_t k = 0; k < ncell; ++k)
        if (out.types[k] == 2) out.cell.push_back(static_cast<int32_t>(k));
    const int n = static_cast<int>(out.cell.size());
    out.image.assign(2 * static_cast<size_t>(n), 0.0);
    out.normal.assign(2 * static_cast<size_t>(n), 0.0);
    if (n > 0) {
        std::vector<double> pts, dir;
        circle_polygon(radius, cx, cy, npoints, pts, dir);
        int32_t* cells = nullptr;
        double *dpts = nullptr, *ddir = nullptr, *img = nullptr, *nrm = nullptr;
        if (!buf.alloc(&cells, n) || !buf.alloc(&dpts, pts.size()) || !buf.alloc(&ddir, dir.size()) ||
            !buf.alloc(&img, 2 * static_cast<size_t>(n)) || !buf.alloc(&nrm, 2 * static_cast<size_t>(n)))
            return cuda_fail("allocation", cudaErrorMemoryAllocation);
        e = cudaMemcpyAsync(cells, out.cell.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dpts, pts.data(), sizeof(double) * pts.size(), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ddir, dir.data(), sizeof(double) * dir.size(), cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return cuda_fail("upload", e);
        image_point_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, cells, ny, dx, dy, npoints, dpts, ddir, img, nrm);
        e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail("image-point launch", e);
        e = cudaMemcpyAsync(out.image.data(), img, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(out.normal.data(), nrm, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail("image points", e);
    }
    return select_donors(out.types.data(), nx, ny, dx, dy, out.cell, out.image, out.donor, err);
}

}  // namespace cfs
