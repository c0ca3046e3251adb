// Coil placement: closest point on the skin surface to each target centre, and the coil frame.
//
// Compiled with -fmad=false so the FP64 frame matches the CPU restatement to the last bit.
// Reference behaviour restated: place.cu:64-230 (closest point on a triangle in Ericson's case
// order; minimum over the total order (d^2, triangle index); frame [x | y | z | c] with z the
// inward smoothed normal, y the tangential handle direction, x = y cross z, c offset distance_mm
// along the outward normal; a handle within sin^2 <= 1e-12 of the normal is degenerate and the
// frame falls back to a canonical in-plane axis).
#include <cfloat>
#include <climits>

#include <algorithm>

#include "internal.hpp"

namespace cunibs {
namespace {

__device__ __forceinline__ double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

__device__ double closest_on_tri(const double* p, const double* a, const double* b, const double* c, double* q) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    for (int i = 0; i < 3; ++i) {
        ab[i] = b[i] - a[i];
        ac[i] = c[i] - a[i];
        ap[i] = p[i] - a[i];
        bp[i] = p[i] - b[i];
        cp[i] = p[i] - c[i];
    }
    const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    const double vc = d1 * d4 - d3 * d2;
    const double vb = d5 * d2 - d1 * d6;
    const double va = d3 * d6 - d5 * d4;
    if (d1 <= 0.0 && d2 <= 0.0) {
        for (int i = 0; i < 3; ++i) q[i] = a[i];
    } else if (d3 >= 0.0 && d4 <= d3) {
        for (int i = 0; i < 3; ++i) q[i] = b[i];
    } else if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
        const double t = d1 / (d1 - d3);
        for (int i = 0; i < 3; ++i) q[i] = a[i] + t * ab[i];
    } else if (d6 >= 0.0 && d5 <= d6) {
        for (int i = 0; i < 3; ++i) q[i] = c[i];
    } else if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double t = d2 / (d2 - d6);
        for (int i = 0; i < 3; ++i) q[i] = a[i] + t * ac[i];
    } else if (va <= 0.0 && (d4 - d3) >= 0.0 && (d5 - d6) >= 0.0) {
        const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        for (int i = 0; i < 3; ++i) q[i] = b[i] + t * (c[i] - b[i]);
    } else {
        const double denom = 1.0 / (va + vb + vc);
        const double v = vb * denom, w = vc * denom;
        for (int i = 0; i < 3; ++i) q[i] = a[i] + v * ab[i] + w * ac[i];
    }
    const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
    return dx * dx + dy * dy + dz * dz;
}

// One block per placement: scan all skin triangles, reduce to the (d2, index) minimum, then
// thread 0 builds the frame.
// (distance^2, triangle) minimum of a block's threads, ties to the lower triangle index: an exact,
// order-free reduction, so any split of the scan finds the same triangle.
__device__ __forceinline__ void block_argmin(double& best, int& bi) {
    __shared__ double sd[kBlock];
    __shared__ int si[kBlock];
    sd[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            const double d = sd[threadIdx.x + off];
            const int i = si[threadIdx.x + off];
            if (d < sd[threadIdx.x] || (d == sd[threadIdx.x] && i < si[threadIdx.x])) {
                sd[threadIdx.x] = d;
                si[threadIdx.x] = i;
            }
        }
        __syncthreads();
    }
    best = sd[0];
    bi = si[0];
}

// Closest skin triangle to each placement's centre: blockIdx.y = placement, blockIdx.x = one of
// gridDim.x segments of the triangle list; each segment's minimum goes to part_d/part_i.
__global__ void nearest_tri_kernel(const double* __restrict__ nodes, const int* __restrict__ tris, int n_tri,
                                   const double* __restrict__ centers, double* __restrict__ part_d,
                                   int* __restrict__ part_i) {
    const int p = blockIdx.y;
    const double center[3] = {centers[3 * p], centers[3 * p + 1], centers[3 * p + 2]};
    double best = DBL_MAX;
    int bi = INT_MAX;
    double q[3];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_tri; t += gridDim.x * blockDim.x) {
        const double d2 = closest_on_tri(center, nodes + 3 * static_cast<long>(tris[3 * t]),
                                         nodes + 3 * static_cast<long>(tris[3 * t + 1]),
                                         nodes + 3 * static_cast<long>(tris[3 * t + 2]), q);
        if (d2 < best) {
            best = d2;
            bi = t;
        }
    }
    block_argmin(best, bi);
    if (threadIdx.x == 0) {
        part_d[p * gridDim.x + blockIdx.x] = best;
        part_i[p * gridDim.x + blockIdx.x] = bi;
    }
}

// One block per placement: the minimum over the segments, then the coil frame.
__global__ void place_kernel(const double* __restrict__ nodes, const int* __restrict__ tris, int n_seg,
                             const double* __restrict__ part_d, const int* __restrict__ part_i,
                             const double* __restrict__ tnorm, const double* __restrict__ centers,
                             const double* __restrict__ handles, const double* __restrict__ dists,
                             double* __restrict__ out, int* __restrict__ degenerate) {
    const int p = blockIdx.x;
    const double center[3] = {centers[3 * p], centers[3 * p + 1], centers[3 * p + 2]};
    double best = DBL_MAX;
    int bi = INT_MAX;
    for (int j = threadIdx.x; j < n_seg; j += blockDim.x) {
        const double d = part_d[p * n_seg + j];
        const int i = part_i[p * n_seg + j];
        if (d < best || (d == best && i < bi)) {
            best = d;
            bi = i;
        }
    }
    block_argmin(best, bi);
    if (threadIdx.x != 0) return;
    const int tri = bi;
    double proj[3];
    closest_on_tri(center, nodes + 3 * static_cast<long>(tris[3 * tri]), nodes + 3 * static_cast<long>(tris[3 * tri + 1]),
                   nodes + 3 * static_cast<long>(tris[3 * tri + 2]), proj);
    const double nrm[3] = {tnorm[3 * tri], tnorm[3 * tri + 1], tnorm[3 * tri + 2]};
    const double z[3] = {-nrm[0], -nrm[1], -nrm[2]};
    double y[3];
    bool from_handle = false;
    if (handles != nullptr) {
        for (int i = 0; i < 3; ++i) y[i] = handles[3 * p + i] - proj[i];
        const double yy = dot3(y, y);
        if (yy > 0.0) {
            const double inv = 1.0 / sqrt(yy);
            for (int i = 0; i < 3; ++i) y[i] = y[i] * inv;
            const double cz = dot3(y, z);
            if ((1.0 - cz * cz) > 1e-12) {
                for (int i = 0; i < 3; ++i) y[i] = y[i] - z[i] * cz;
                const double inv2 = 1.0 / sqrt(dot3(y, y));
                for (int i = 0; i < 3; ++i) y[i] = y[i] * inv2;
                from_handle = true;
            }
        }
    }
    if (!from_handle) {
        int m = 0;
        if (fabs(z[1]) < fabs(z[m])) m = 1;
        if (fabs(z[2]) < fabs(z[m])) m = 2;
        double ref[3] = {0.0, 0.0, 0.0};
        ref[m] = 1.0;
        y[0] = z[1] * ref[2] - z[2] * ref[1];
        y[1] = z[2] * ref[0] - z[0] * ref[2];
        y[2] = z[0] * ref[1] - z[1] * ref[0];
        const double inv = 1.0 / sqrt(dot3(y, y));
        for (int i = 0; i < 3; ++i) y[i] = y[i] * inv;
    }
    if (degenerate) degenerate[p] = from_handle ? 0 : 1;
    const double x[3] = {y[1] * z[2] - y[2] * z[1], y[2] * z[0] - y[0] * z[2], y[0] * z[1] - y[1] * z[0]};
    double* T = out + 16 * static_cast<long>(p);
    for (int i = 0; i < 16; ++i) T[i] = 0.0;
    for (int r = 0; r < 3; ++r) {
        T[4 * r + 0] = x[r];
        T[4 * r + 1] = y[r];
        T[4 * r + 2] = z[r];
        T[4 * r + 3] = proj[r] + dists[p] * nrm[r];
    }
    T[15] = 1.0;
}

}  // namespace

void place_transforms(const Mesh& m, const double* centers, const double* handles, const double* dists, int k,
                      double* transforms_dev, int* degenerate_dev, cudaStream_t s) {
    if (m.n_skin <= 0) fail(kEInval, "the mesh has no skin triangles to place a coil on");
    if (k <= 0) return;
    // Enough segments that the scan fills the GPU: about 2 x 148 blocks over all placements.
    const int n_seg = std::max(1, std::min(static_cast<int>(grid_for(m.n_skin)), (296 + k - 1) / k));
    m.place_d.reserve(static_cast<std::size_t>(n_seg) * k);
    m.place_i.reserve(static_cast<std::size_t>(n_seg) * k);
    nearest_tri_kernel<<<dim3(n_seg, k), kBlock, 0, s>>>(m.nodes.get(), m.skin.get(), m.n_skin, centers,
                                                         m.place_d.get(), m.place_i.get());
    place_kernel<<<k, kBlock, 0, s>>>(m.nodes.get(), m.skin.get(), n_seg, m.place_d.get(), m.place_i.get(),
                                      m.skin_normals.get(), centers, handles, dists, transforms_dev, degenerate_dev);
    count_launch(2);
    CUNIBS_LAUNCH_CHECK("place");
}

}  // namespace cunibs
