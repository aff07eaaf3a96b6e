// rb_sdf.cu -- signed distance grid of a closed triangle mesh (shape set-up).
//
// Replaces the igl.signed_distance call of grid3.py:338 (create_signed_distance).  For every grid node:
//   distance = min over triangles of |p - closest point on the triangle| (Voronoi-region case analysis of
//              Ericson, Real-Time Collision Detection, 2005, section 5.1.5);
//   sign     = negative when the generalized winding number |w| > 1/2, w = sum of the triangles' signed
//              solid angles / 4 pi (Van Oosterom & Strackee, IEEE TBME 1983).
// One thread per node; triangles are streamed through shared memory in tiles.
#include <cuda_runtime.h>

#include <string>

#include "rainbow_b200.h"
#include "rb_device.cuh"
#include "rb_internal.h"

namespace {

using rb::d3;

__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 scale(d3 a, double s) { return d3{a.x * s, a.y * s, a.z * s}; }

__device__ d3 closest_point(d3 p, d3 a, d3 b, d3 c) {
    const d3 ab = rb::sub(b, a), ac = rb::sub(c, a), ap = rb::sub(p, a);
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.0 && d2 <= 0.0) return a;
    const d3 bp = rb::sub(p, b);
    const double d3v = dot(ab, bp), d4 = dot(ac, bp);
    if (d3v >= 0.0 && d4 <= d3v) return b;
    const double vc = d1 * d4 - d3v * d2;
    if (vc <= 0.0 && d1 >= 0.0 && d3v <= 0.0) {
        const double v = d1 / (d1 - d3v);
        return rb::add(a, scale(ab, v));
    }
    const d3 cp = rb::sub(p, c);
    const double d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.0 && d5 <= d6) return c;
    const double vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
        const double w = d2 / (d2 - d6);
        return rb::add(a, scale(ac, w));
    }
    const double va = d3v * d6 - d5 * d4;
    if (va <= 0.0 && (d4 - d3v) >= 0.0 && (d5 - d6) >= 0.0) {
        const double w = (d4 - d3v) / ((d4 - d3v) + (d5 - d6));
        return rb::add(b, scale(rb::sub(c, b), w));
    }
    const double denom = 1.0 / (va + vb + vc);
    const double v = vb * denom, w = vc * denom;
    return rb::add(a, rb::add(scale(ab, v), scale(ac, w)));
}

constexpr int kTile = 128;
constexpr int kSdfBlock = 128;

// distance and sign of node `node` of a grid (meta: min[3], max[3], spacing[3], I, J, K) around the mesh
// (V, T with n_tri triangles); every thread of the block calls it (the triangle tiles go through shared memory)
__device__ __forceinline__ void sdf_node(const double* __restrict__ V, const int32_t* __restrict__ T, int n_tri,
                                         const double* __restrict__ meta, int64_t node, double* __restrict__ values) {
    __shared__ double tri[kTile][9];
    const int I = (int)meta[9], J = (int)meta[10], K = (int)meta[11];
    const int64_t n_nodes = (int64_t)I * J * K;
    d3 p = d3{0.0, 0.0, 0.0};
    if (node < n_nodes) {
        const int i = (int)(node % I), j = (int)((node / I) % J), k = (int)(node / ((int64_t)I * J));
        // grid3.py:88 get_node_coord: min + spacing * (i, j, k)
        p = d3{meta[0] + meta[6] * (double)i, meta[1] + meta[7] * (double)j, meta[2] + meta[8] * (double)k};
    }
    double best = INFINITY, wind = 0.0;
    for (int t0 = 0; t0 < n_tri; t0 += kTile) {
        __syncthreads();
        for (int e = threadIdx.x; e < kTile * 9; e += blockDim.x) {
            const int t = t0 + e / 9, c = (e % 9) / 3, axis = e % 3;
            tri[e / 9][e % 9] = t < n_tri ? V[3 * T[3 * t + c] + axis] : 0.0;
        }
        __syncthreads();
        const int nt = min(kTile, n_tri - t0);
        for (int t = 0; t < nt; ++t) {
            const d3 a = d3{tri[t][0], tri[t][1], tri[t][2]};
            const d3 b = d3{tri[t][3], tri[t][4], tri[t][5]};
            const d3 c = d3{tri[t][6], tri[t][7], tri[t][8]};
            const d3 q = closest_point(p, a, b, c);
            const d3 dq = rb::sub(p, q);
            best = fmin(best, sqrt(dot(dq, dq)));
            const d3 A = rb::sub(a, p), B = rb::sub(b, p), C = rb::sub(c, p);
            const double la = sqrt(dot(A, A)), lb = sqrt(dot(B, B)), lc = sqrt(dot(C, C));
            const double num = dot(A, rb::cross_np(B, C));
            const double den = la * lb * lc + dot(A, B) * lc + dot(B, C) * la + dot(C, A) * lb;
            wind += 2.0 * atan2(num, den);
        }
    }
    if (node < n_nodes) values[node] = (fabs(wind) / (4.0 * M_PI) > 0.5) ? -best : best;
}

__global__ void __launch_bounds__(kSdfBlock) k_sdf(const double* __restrict__ V, const int32_t* __restrict__ T,
                                                   int n_tri, const double* __restrict__ meta,
                                                   double* __restrict__ values) {
    sdf_node(V, T, n_tri, meta, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, values);
}

// many grids in one launch: block b belongs to the shape s with block_off[s] <= b < block_off[s + 1]
__global__ void __launch_bounds__(kSdfBlock) k_sdf_many(int n_shapes, const double* __restrict__ V,
                                                        const int32_t* __restrict__ v_off,
                                                        const int32_t* __restrict__ T,
                                                        const int32_t* __restrict__ t_off,
                                                        const double* __restrict__ meta,
                                                        const int64_t* __restrict__ g_off,
                                                        const int64_t* __restrict__ block_off,
                                                        double* __restrict__ values) {
    const int64_t b = blockIdx.x;
    int lo = 0, hi = n_shapes;   // the last s with block_off[s] <= b
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (block_off[mid] <= b) lo = mid; else hi = mid;
    }
    const int s = lo;
    const int64_t node = (b - block_off[s]) * kSdfBlock + threadIdx.x;
    sdf_node(V + 3 * (size_t)v_off[s], T + 3 * (size_t)t_off[s], t_off[s + 1] - t_off[s], meta + 12 * (size_t)s,
             node, values + g_off[s]);
}

}  // namespace

extern "C" int rb_signed_distance_grid(const double* V, int32_t n_vertices, const int32_t* T, int32_t n_triangles,
                                       const double* grid_meta_dev, double* values, void* stream) {
    if (!V || !T || !grid_meta_dev || !values || n_vertices <= 0 || n_triangles <= 0) {
        rb::g_error = "rb_signed_distance_grid: bad argument";
        return RB_ERR_ARG;
    }
    // the node count is read on the device from grid_meta; the launch covers the largest grid allowed here
    double meta[12];
    cudaError_t e = cudaMemcpyAsync(meta, grid_meta_dev, sizeof(meta), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) {
        rb::g_error = std::string("rb_signed_distance_grid: ") + cudaGetErrorString(e);
        return RB_ERR_CUDA;
    }
    const int64_t n_nodes = (int64_t)meta[9] * (int64_t)meta[10] * (int64_t)meta[11];
    if (meta[9] < 2 || meta[10] < 2 || meta[11] < 2 || n_nodes > (int64_t)1 << 30) {
        rb::g_error = "rb_signed_distance_grid: grid size out of range";
        return RB_ERR_ARG;
    }
    const int block = kSdfBlock;
    k_sdf<<<(unsigned)((n_nodes + block - 1) / block), block, 0, (cudaStream_t)stream>>>(V, T, n_triangles,
                                                                                      grid_meta_dev, values);
    rb::note_launch();
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        rb::g_error = std::string("rb_signed_distance_grid: ") + cudaGetErrorString(e);
        return RB_ERR_CUDA;
    }
    return RB_OK;
}

extern "C" int rb_signed_distance_grids(int32_t n_shapes, const double* V, const int32_t* v_off, const int32_t* T,
                                        const int32_t* t_off, const double* grid_meta, const int64_t* g_off,
                                        const int64_t* block_off, int64_t total_blocks, double* values,
                                        void* stream) {
    if (n_shapes <= 0 || !V || !v_off || !T || !t_off || !grid_meta || !g_off || !block_off || !values ||
        total_blocks <= 0 || total_blocks > INT32_MAX) {
        rb::g_error = "rb_signed_distance_grids: bad argument";
        return RB_ERR_ARG;
    }
    k_sdf_many<<<(unsigned)total_blocks, kSdfBlock, 0, (cudaStream_t)stream>>>(n_shapes, V, v_off, T, t_off,
                                                                             grid_meta, g_off, block_off, values);
    rb::note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        rb::g_error = std::string("rb_signed_distance_grids: ") + cudaGetErrorString(e);
        return RB_ERR_CUDA;
    }
    return RB_OK;
}
