// rb_step.cu -- the prox_rigid_bodies semi-implicit time step on sm_100a.
//
// One rb_step call advances every scene of an rb_bodies batch by one step.  The pipeline (one kernel per
// stage, all on the caller's stream, no host synchronisation, so a sequence of steps can be captured in a
// CUDA graph) follows steppers.py:47 SemiImplicitStepper.step:
//
//   k_bodies          forces, gyroscopic torque, world inverse inertia, W f_ext      state_storage.py:43-185
//   k_world_vertices  rotate_array(q, V) + r for every body vertex                   collision_detection.py:32
//   k_clusters        32-leaf cluster boxes (unions of k-DOP K=3 leaf boxes + envelope) kdop_bvh.py:52, kdop.py:53
//   k_roots           body boxes (the BVH root)                                         kdop_bvh.py:215
//   k_pairs           body pairs in combinations() order whose roots overlap           collision_detection.py:70
//   k_mid             per pair, the triangles of each side whose leaf overlaps a leaf   kdop_bvh.py:127, :234
//                     of the other side (ascending, = np.unique of the traversal)      collision_detection.py:234
//   k_narrow          Frank-Wolfe deepest point on each candidate triangle in the       collision_detection.py:87
//                     other body's SDF, contact emission
//   k_dedup           first-occurrence duplicate removal and compaction                 collision_detection.py:255
//   k_contacts        contact frame, Jacobian, W J^T, b, Delassus diagonal, r, mu        contacts.py:31-55
//   k_solve           proximal solver (one block per scene)                             gauss_seidel_solver.py:14
//   k_integrate       u += dt W f + W J^T sol; r, q update                               state_storage.py:239-302
//   k_post_*          post-stabilisation                                                steppers.py:15
//
// Counts that are only known on the device (pairs, candidates, contacts) are read by the consumers from
// device counters; kernels that depend on them run grid-stride loops over those counters.
#include <cuda_runtime.h>

#include <cstdio>
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "rainbow_b200.h"
#include "rb_device.cuh"
#include "rb_internal.h"
#include "rb_layout.h"

namespace rb {

// kernels launched by this library in this process (rb_launch_count)
std::atomic<int64_t> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

constexpr int kWarpsPerBlock = 4;
constexpr int kBlock = 32 * kWarpsPerBlock;
constexpr int kAbort = 15;   // counters[kAbort]: nonzero once a capacity was exceeded
constexpr int kSolveSmemBodies = 4608;   // 216 KB of body accumulators per solver block

// ---------------------------------------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ int scene_of(const int32_t* scene_start, int n_scenes, int body) {
    int lo = 0, hi = n_scenes;   // find s with scene_start[s] <= body < scene_start[s+1]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(scene_start + mid) <= body) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------------------------------------
// device-wide exclusive scan of int32 counts (three phases; the element count may live on the device)
// data[0..n) -> exclusive prefix sums, data[n] = total, *total_out = total
// ---------------------------------------------------------------------------------------------------------
// with a device count, n_host is the capacity the count is clamped to
__device__ __forceinline__ int scan_n(const int32_t* n_dev, int n_host) { return n_dev ? min(*n_dev, n_host) : n_host; }

__global__ void k_scan_reduce(const int32_t* __restrict__ data, const int32_t* n_dev, int n_host,
                              int32_t* __restrict__ partial) {
    const int n = scan_n(n_dev, n_host);
    const int chunk = (n + gridDim.x - 1) / gridDim.x;
    const int start = blockIdx.x * chunk, end = min(n, start + chunk);
    int s = 0;
    for (int i = start + threadIdx.x; i < end; i += blockDim.x) s += data[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ int ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
        partial[blockIdx.x] = t;
    }
}
__global__ void k_scan_top(int32_t* __restrict__ partial, int nblocks, int32_t* total_out) {
    // single block of 1024 threads, nblocks <= 1024
    __shared__ int s[1024];
    const int t = threadIdx.x;
    int v = t < nblocks ? partial[t] : 0;
    s[t] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int a = t >= o ? s[t - o] : 0;
        __syncthreads();
        s[t] += a;
        __syncthreads();
    }
    if (t < nblocks) partial[t] = s[t] - v;
    if (t == 1023) { partial[nblocks] = s[t]; if (total_out) *total_out = s[t]; }
}
__global__ void k_scan_down(int32_t* __restrict__ data, const int32_t* n_dev, int n_host,
                            const int32_t* __restrict__ partial) {
    const int n = scan_n(n_dev, n_host);
    const int chunk = (n + gridDim.x - 1) / gridDim.x;
    const int start = blockIdx.x * chunk, end = min(n, start + chunk);
    __shared__ int ws[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = partial[blockIdx.x];
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int base = start; base < end; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int v = i < end ? data[i] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            int a = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += a;
        }
        if (lane == 31) ws[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            int wv = lane < nw ? ws[lane] : 0;
            int wi = wv;
            for (int o = 1; o < 32; o <<= 1) {
                int a = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += a;
            }
            if (lane < nw) ws[lane] = wi - wv;
        }
        __syncthreads();
        const int c = carry;
        if (i < end) data[i] = c + ws[wid] + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = c + ws[wid] + incl;
        __syncthreads();
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) data[n] = partial[gridDim.x];
}
void scan(int32_t* data, const int32_t* n_dev, int n_host, int32_t* partial, int32_t* total_out, cudaStream_t st) {
    const int G = kScanGrid;
    k_scan_reduce<<<G, 256, 0, st>>>(data, n_dev, n_host, partial); note_launch();
    k_scan_top<<<1, 1024, 0, st>>>(partial, G, total_out); note_launch();
    k_scan_down<<<G, 256, 0, st>>>(data, n_dev, n_host, partial); note_launch();
}

__global__ void k_zero_i32(int32_t* p, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
}
struct StepArgs;
// capacity check after a scan: a total above the capacity aborts the rest of the step
__global__ void k_check(int32_t* counters, int which, int cap, int bit, int32_t* status) {
    if (counters[kAbort]) return;   // an earlier stage overflowed: this stage's total is not meaningful
    if (counters[which] > cap) {
        atomicOr(counters + kAbort, bit);
        atomicOr(status, bit);
    }
}

// ---------------------------------------------------------------------------------------------------------
// bodies: state_storage.py:108 _compute_total_external_forces, :158 _compute_inverse_mass_matrix, :53
// ---------------------------------------------------------------------------------------------------------
struct StepArgs {
    rb_shapes sh;
    rb_bodies bd;
    rb_caps caps;
    rb_params pr;
    rb_outputs out;
    Workspace ws;
};

__global__ void k_bodies(const StepArgs a) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.bd.n_bodies) return;
    double* d = a.ws.dux + 6 * b;
    double* du = a.ws.du + 6 * b;
    double* Wi = a.ws.Winv + 9 * b;
    if (a.bd.fixed[b]) {
        for (int i = 0; i < 6; ++i) { d[i] = 0.0; du[i] = 0.0; }
        for (int i = 0; i < 9; ++i) Wi[i] = 0.0;
        return;
    }
    const double* q = a.bd.x + 7 * b + 3;
    const d3 v = ld3(a.bd.u + 6 * b), w = ld3(a.bd.u + 6 * b + 3);
    double R[9], Iw[9], Ib[3], Binv[3];
    quat_to_matrix(q, R);
    for (int i = 0; i < 3; ++i) Ib[i] = a.bd.inertia[3 * b + i];
    update_inertia_tensor(R, Ib, Iw);
    const d3 c = cross_np(w, gemv3_np(Iw, w));
    double T[3] = {-c.x, -c.y, -c.z}, F[3] = {0.0, 0.0, 0.0};
    const double mass = a.bd.mass[b];
    for (int e = a.bd.force_ptr[b]; e < a.bd.force_ptr[b + 1]; ++e) {
        const int f = a.bd.force_list[e];
        const double* fp = a.bd.force_params + 4 * f;
        double Fi[3], Ti[3];
        if (a.bd.force_kind[f] == 0) {          // types.py:204 Gravity.compute: F = -m g up
            const double s = -mass * fp[0];
            Fi[0] = s * fp[1]; Fi[1] = s * fp[2]; Fi[2] = s * fp[3];
            Ti[0] = 0.0; Ti[1] = 0.0; Ti[2] = 0.0;
        } else {                                 // types.py:239 Damping.compute: F = -v alpha, T = -w beta
            Fi[0] = -v.x * fp[0]; Fi[1] = -v.y * fp[0]; Fi[2] = -v.z * fp[0];
            Ti[0] = -w.x * fp[1]; Ti[1] = -w.y * fp[1]; Ti[2] = -w.z * fp[1];
        }
        for (int i = 0; i < 3; ++i) { F[i] = F[i] + Fi[i]; T[i] = T[i] + Ti[i]; }
    }
    const double m = 1.0 / mass;
    for (int i = 0; i < 3; ++i) Binv[i] = 1.0 / Ib[i];
    update_inertia_tensor(R, Binv, Wi);
    const double dt = a.pr.dt;
    for (int i = 0; i < 3; ++i) {   // bsr_matvec over the 3x3 blocks of W
        double s = 0.0;
        s += (i == 0 ? m : 0.0) * F[0];
        s += (i == 1 ? m : 0.0) * F[1];
        s += (i == 2 ? m : 0.0) * F[2];
        double t = 0.0;
        t += Wi[3 * i] * T[0];
        t += Wi[3 * i + 1] * T[1];
        t += Wi[3 * i + 2] * T[2];
        d[i] = s; d[3 + i] = t;
        du[i] = dt * s; du[3 + i] = dt * t;   // steppers.py:64 delta_u = dt * delta_u_ext
    }
}

__global__ void k_zero_stats(const StepArgs a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < a.bd.n_scenes) {
        rb_scene_stats* st = a.out.stats + s;
        st->n_grid_lookups = 0; st->n_leaf_overlaps = 0;
        st->n_grid_lookups32 = 0; st->n_search_flips = 0; st->n_accept_flips = 0;
    }
}

// collision_detection.py:32 V_world = rotate_array(q, V) + r
__global__ void k_world_vertices(const StepArgs a, int n_verts) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_verts) return;
    const int b = a.bd.vert_body[g];
    const int local = g - a.bd.body_v0[b];
    const int s = a.bd.shape[b];
    const d3 V = ld3(a.sh.V + 3 * (size_t)(a.sh.v_off[s] + local));
    const double* xb = a.bd.x + 7 * b;
    const d3 p = quat_rotate_row(xb + 3, V);
    st3(a.ws.Vw + 3 * (size_t)g, d3{p.x + xb[0], p.y + xb[1], p.z + xb[2]});
}

// leaf box of triangle t of a body (kdop.py:53 make with K=3: min/max of the triangle's world coordinates
// -/+ envelope), from the body's world vertices Vw and its shape's triangles T; L = (lo[3], hi[3])
__device__ __forceinline__ void leaf_box(const int32_t* T, const double* Vw, int t, double env, double* L) {
    const int32_t* tri = T + 3 * (size_t)t;
    const int v[3] = {tri[0], tri[1], tri[2]};
    for (int axis = 0; axis < 3; ++axis) {
        double l = INFINITY, h = -INFINITY;
        for (int k = 0; k < 3; ++k) {
            const double pr = Vw[3 * v[k] + axis];
            if (pr < l) l = pr;
            if (pr > h) h = pr;
        }
        L[axis] = l - env;
        L[3 + axis] = h + env;
    }
}

// the box of every run of 32 consecutive triangles of a body (the union of their leaf boxes); one warp per
// cluster.  Leaf boxes are not stored: the mid phase recomputes the few it tests from the world vertices.
__global__ void k_clusters(const StepArgs a, int n_clusters) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n_clusters) return;
    const int b = a.bd.clu_body[warp];
    const int c = warp - a.bd.body_c0[b];
    const int s = a.bd.shape[b];
    const int nt = a.sh.t_off[s + 1] - a.sh.t_off[s];
    const int t = 32 * c + lane;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (t < nt) {
        double L[6];
        leaf_box(a.sh.T + 3 * (size_t)a.sh.t_off[s], a.ws.Vw + 3 * (size_t)a.bd.body_v0[b], t, a.pr.envelope, L);
        for (int axis = 0; axis < 3; ++axis) { lo[axis] = L[axis]; hi[axis] = L[3 + axis]; }
    }
    for (int axis = 0; axis < 3; ++axis) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[axis] = fmin(lo[axis], __shfl_xor_sync(0xffffffffu, lo[axis], o));
            hi[axis] = fmax(hi[axis], __shfl_xor_sync(0xffffffffu, hi[axis], o));
        }
    }
    if (lane == 0) {
        double* C = a.ws.clu + 6 * (size_t)warp;
        C[0] = lo[0]; C[1] = lo[1]; C[2] = lo[2]; C[3] = hi[0]; C[4] = hi[1]; C[5] = hi[2];
    }
}

// body box = union of its cluster boxes (kdop_bvh.py:229-231); one warp per body
__global__ void k_roots(const StepArgs a) {
    const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (b >= a.bd.n_bodies) return;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = a.bd.body_c0[b] + lane; c < a.bd.body_c0[b + 1]; c += 32) {
        const double* C = a.ws.clu + 6 * (size_t)c;
        for (int axis = 0; axis < 3; ++axis) { lo[axis] = fmin(lo[axis], C[axis]); hi[axis] = fmax(hi[axis], C[3 + axis]); }
    }
    for (int axis = 0; axis < 3; ++axis)
        for (int o = 16; o > 0; o >>= 1) {
            lo[axis] = fmin(lo[axis], __shfl_xor_sync(0xffffffffu, lo[axis], o));
            hi[axis] = fmax(hi[axis], __shfl_xor_sync(0xffffffffu, hi[axis], o));
        }
    if (lane == 0) {
        double* R = a.ws.root + 6 * b;
        R[0] = lo[0]; R[1] = lo[1]; R[2] = lo[2]; R[3] = hi[0]; R[4] = hi[1]; R[5] = hi[2];
    }
}

// ---------------------------------------------------------------------------------------------------------
// broad phase: body pairs (i < j, same scene) in combinations() order whose boxes overlap; warp per body
// ---------------------------------------------------------------------------------------------------------
template <bool WRITE>
__global__ void k_pairs(const StepArgs a) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= a.bd.n_bodies) return;
    if (WRITE && a.ws.counters[kAbort]) return;
    const int s = scene_of(a.bd.scene_start, a.bd.n_scenes, i);
    const int end = a.bd.scene_start[s + 1];
    double Ri[6];
    for (int k = 0; k < 6; ++k) Ri[k] = a.ws.root[6 * i + k];
    int count = 0;
    const int base = WRITE ? a.ws.pair_cnt[i] : 0;
    for (int j0 = i + 1; j0 < end; j0 += 32) {
        const int j = j0 + lane;
        const bool ov = j < end && overlap(Ri, a.ws.root + 6 * j);
        const unsigned bal = __ballot_sync(0xffffffffu, ov);
        if (WRITE && ov) {
            const int pos = base + count + __popc(bal & lanemask_lt());
            a.ws.pairs[2 * pos] = i;
            a.ws.pairs[2 * pos + 1] = j;
        }
        count += __popc(bal);
    }
    if (!WRITE && lane == 0) a.ws.pair_cnt[i] = count;
}

// ---------------------------------------------------------------------------------------------------------
// mid phase: for body pair (A, B) the A-triangles whose leaf box overlaps some B leaf box and vice versa.
// The reference's tandem traversal (kdop_bvh.py:127-178) reports exactly the overlapping leaf pairs because
// each inner volume is the exact union of its children; np.unique of each column (collision_detection.py:234)
// makes both sets ascending.  Clusters of 32 triangles with exact union boxes prune the same way.
// ---------------------------------------------------------------------------------------------------------
// per-warp shared arrays of k_mid, sized at launch by the largest shape: lists of the clusters of A (of B)
// whose box overlaps B's (A's) body box, and the hit masks of their 32 triangles
__device__ __forceinline__ void mid_arrays(int max_clusters, int warp, int16_t*& listA, int16_t*& listB,
                                           uint32_t*& maskA, uint32_t*& maskB) {
    extern __shared__ uint32_t mid_smem[];
    const int words = 3 * max_clusters;   // 2 lists of int16 + 2 masks of uint32 = 3 words per cluster
    uint32_t* base = mid_smem + (size_t)warp * words;
    maskA = base;
    maskB = base + max_clusters;
    listA = reinterpret_cast<int16_t*>(base + 2 * max_clusters);
    listB = listA + max_clusters;
}

// single pass: warps take pairs from a shared counter, find the pair's candidate triangles, reserve room
// with one atomic and write them in ascending (side, triangle) order; pair_items[p] = first candidate of
// the pair, pair_itemsA[p] = number of candidates
__global__ void __launch_bounds__(kBlock) k_mid(const StepArgs a, int max_clusters) {
    int16_t *listA, *listB;
    uint32_t *maskA, *maskB;
    mid_arrays(max_clusters, threadIdx.x >> 5, listA, listB, maskA, maskB);
    const int lane = threadIdx.x & 31;
    if (a.ws.counters[kAbort]) return;
    const int n_pairs = a.ws.counters[kNPairs];
    for (;;) {
        int p = 0;
        if (lane == 0) p = atomicAdd(a.ws.counters + kMidNext, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= n_pairs) break;
        const int A = a.ws.pairs[2 * p], B = a.ws.pairs[2 * p + 1];
        const int cA0 = a.bd.body_c0[A], ncA = a.bd.body_c0[A + 1] - cA0;
        const int cB0 = a.bd.body_c0[B], ncB = a.bd.body_c0[B + 1] - cB0;
        const int ntA = a.bd.body_t0[A + 1] - a.bd.body_t0[A];
        const int ntB = a.bd.body_t0[B + 1] - a.bd.body_t0[B];
        const int32_t* TA = a.sh.T + 3 * (size_t)a.sh.t_off[a.bd.shape[A]];
        const int32_t* TB = a.sh.T + 3 * (size_t)a.sh.t_off[a.bd.shape[B]];
        const double* VwA = a.ws.Vw + 3 * (size_t)a.bd.body_v0[A];
        const double* VwB = a.ws.Vw + 3 * (size_t)a.bd.body_v0[B];
        const double env = a.pr.envelope;
        const double* rootA = a.ws.root + 6 * A;
        const double* rootB = a.ws.root + 6 * B;
        if (ncA > max_clusters || ncB > max_clusters) {
            if (lane == 0) {
                atomicOr(a.out.status, RB_STATUS_MESH_TOO_LARGE);
                atomicOr(a.ws.counters + kAbort, RB_STATUS_MESH_TOO_LARGE);
                a.ws.pair_items[p] = 0; a.ws.pair_itemsA[p] = 0; a.ws.pair_ovl[p] = 0;
            }
            continue;
        }
        int nA = 0, nB = 0;
        for (int c0 = 0; c0 < ncA; c0 += 32) {
            const int c = c0 + lane;
            const bool ok = c < ncA && overlap(a.ws.clu + 6 * (size_t)(cA0 + c), rootB);
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (ok) listA[nA + __popc(bal & lanemask_lt())] = (int16_t)c;
            nA += __popc(bal);
        }
        for (int c0 = 0; c0 < ncB; c0 += 32) {
            const int c = c0 + lane;
            const bool ok = c < ncB && overlap(a.ws.clu + 6 * (size_t)(cB0 + c), rootA);
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (ok) listB[nB + __popc(bal & lanemask_lt())] = (int16_t)c;
            nB += __popc(bal);
        }
        for (int k = lane; k < nA; k += 32) maskA[k] = 0u;
        for (int k = lane; k < nB; k += 32) maskB[k] = 0u;
        __syncwarp();
        int n_ovl = 0;
        for (int ia = 0; ia < nA; ++ia) {
            const int ca = listA[ia];
            double CA[6];
            for (int k = 0; k < 6; ++k) CA[k] = a.ws.clu[6 * (size_t)(cA0 + ca) + k];
            const int ta = 32 * ca + lane;
            const bool validA = ta < ntA;
            double LA[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            if (validA) leaf_box(TA, VwA, ta, env, LA);
            bool hitA = false;
            for (int ib = 0; ib < nB; ++ib) {
                const int cb = listB[ib];
                const double* CB = a.ws.clu + 6 * (size_t)(cB0 + cb);
                if (!overlap(CA, CB)) continue;
                // a leaf pair can only overlap if each leaf overlaps the other leaf's cluster box
                const unsigned amask = __ballot_sync(0xffffffffu, validA && overlap(LA, CB));
                if (!amask) continue;
                const int tb = 32 * cb + lane;
                const bool validB = tb < ntB;
                double LB[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                if (validB) leaf_box(TB, VwB, tb, env, LB);
                unsigned bmask = __ballot_sync(0xffffffffu, validB && overlap(LB, CA));
                unsigned hitB = 0u;
                // every candidate leaf pair is tested once, broadcasting the leaves of the side with fewer
                if (__popc(bmask) <= __popc(amask)) {   // B leaves to the A lanes
                    const bool mine = (amask >> lane) & 1u;
                    while (bmask) {
                        const int jb = __ffs(bmask) - 1;
                        bmask &= bmask - 1;
                        double Lj[6];
                        for (int k = 0; k < 6; ++k) Lj[k] = __shfl_sync(0xffffffffu, LB[k], jb);
                        if (mine && overlap(LA, Lj)) { hitA = true; hitB |= 1u << jb; }
                    }
                    n_ovl += __popc(hitB);
                    hitB = __reduce_or_sync(0xffffffffu, hitB);
                } else {                                 // A leaves to the B lanes
                    const bool mineB = (bmask >> lane) & 1u;
                    unsigned am = amask, hitAbits = 0u;
                    bool bhit = false;
                    while (am) {
                        const int ja = __ffs(am) - 1;
                        am &= am - 1;
                        double Li[6];
                        for (int k = 0; k < 6; ++k) Li[k] = __shfl_sync(0xffffffffu, LA[k], ja);
                        if (mineB && overlap(Li, LB)) { bhit = true; hitAbits |= 1u << ja; ++n_ovl; }
                    }
                    hitB = __ballot_sync(0xffffffffu, bhit);
                    hitAbits = __reduce_or_sync(0xffffffffu, hitAbits);
                    if ((hitAbits >> lane) & 1u) hitA = true;
                }
                if (lane == 0) maskB[ib] |= hitB;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, hitA);
            if (lane == 0) maskA[ia] = bal;
        }
        __syncwarp();
        int cntA = 0, cntB = 0;
        for (int k = lane; k < nA; k += 32) cntA += __popc(maskA[k]);
        for (int k = lane; k < nB; k += 32) cntB += __popc(maskB[k]);
        cntA = __reduce_add_sync(0xffffffffu, cntA);
        cntB = __reduce_add_sync(0xffffffffu, cntB);
        n_ovl = __reduce_add_sync(0xffffffffu, n_ovl);
        int pos = 0;
        if (lane == 0) pos = atomicAdd(a.ws.counters + kNItems, cntA + cntB);
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if (lane == 0) { a.ws.pair_items[p] = pos; a.ws.pair_itemsA[p] = cntA + cntB; a.ws.pair_ovl[p] = n_ovl; }
        if (pos + cntA + cntB <= a.caps.item_capacity) {   // otherwise k_check aborts the step
            for (int side = 0; side < 2; ++side) {
                const int n = side ? nB : nA;
                const int16_t* list = side ? listB : listA;
                const uint32_t* mask = side ? maskB : maskA;
                for (int k = 0; k < n; ++k) {
                    const uint32_t bits = mask[k];
                    if (bits & (1u << lane)) {
                        const int at = pos + __popc(bits & lanemask_lt());
                        a.ws.item_pair[at] = p;
                        a.ws.item_tri[at] = (side << 31) | (32 * list[k] + lane);
                    }
                    pos += __popc(bits);
                }
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------------------------
// narrow phase (collision_detection.py:87 _compute_contacts): one thread per candidate triangle
// ---------------------------------------------------------------------------------------------------------
// seed and Frank-Wolfe search on one triangle (ps: its corners in the SDF owner's frame) in FP64
// (collision_detection.py:134-165).  Returns the point; n_fw = iterations, trace = the seed (bits 0-1) and
// each iteration's vertex (2 bits each from bit 2)
__device__ __forceinline__ d3 fw_search64(const GridView& g, const d3* ps, int max_it, double tol, int& n_fw,
                                          uint32_t& trace) {
    // seed: corner with the smallest gradient norm (:136-140); norm(list, axis=1) sums squares unfused
    double gn[3];
    for (int c = 0; c < 3; ++c) {
        const d3 gr = grid_gradient(g, ps[c]);
        gn[c] = sqrt((gr.x * gr.x + gr.y * gr.y) + gr.z * gr.z);
    }
    int best = 0;
    if (gn[1] < gn[best]) best = 1;
    if (gn[2] < gn[best]) best = 2;
    trace = (uint32_t)best;
    d3 x = best == 0 ? ps[0] : (best == 1 ? ps[1] : ps[2]);   // selects keep ps in registers
    n_fw = 0;
    for (int i = 0; i < max_it; ++i) {   // Frank-Wolfe (:144-165)
        ++n_fw;
        // the reference evaluates the same gradient once per corner; one evaluation gives identical values
        const d3 gr = grid_gradient(g, x);
        const double o0 = dot3_np(ps[0], gr), o1 = dot3_np(ps[1], gr), o2 = dot3_np(ps[2], gr);
        int v = 0;
        double ov = o0;
        if (o1 < ov) { v = 1; ov = o1; }
        if (o2 < ov) { v = 2; ov = o2; }
        if (i < 15) trace |= (uint32_t)v << (2 + 2 * i);
        const double alpha = 2.0 / (double)(i + 2);
        const d3 s = v == 0 ? ps[0] : (v == 1 ? ps[1] : ps[2]);
        x = d3{x.x + alpha * (s.x - x.x), x.y + alpha * (s.y - x.y), x.z + alpha * (s.z - x.z)};
        if (ov > tol) break;
    }
    return x;
}

// the same search with its lookups on the FP32 copy of the grid (the FP32 precision modes).  The point x and
// the objectives stay FP64; a decision whose margin lies within the FP32 lookups' error bound (an exact tie of
// coplanar corners, a near-tie, an objective next to the tolerance) is taken again on FP64 lookups, so every
// decision, and x, equal fw_search64's.  l64 / l32 count the FP64 and FP32 lookups made.
__device__ __forceinline__ d3 fw_search_f32(const GridView& g, const float* values32, const d3* ps, int max_it,
                                            double tol, int& n_fw, uint32_t& trace, int& l64, int& l32) {
    double scale = 0.0;   // max over corners of |p|_1: an objective's error is at most err x scale
    for (int c = 0; c < 3; ++c) scale = fmax(scale, fabs(ps[c].x) + fabs(ps[c].y) + fabs(ps[c].z));
    double gn[3], err = 0.0;
    for (int c = 0; c < 3; ++c) {
        double e;
        const d3 gr = grid_gradient_f32(g, values32, ps[c], e);
        gn[c] = sqrt((gr.x * gr.x + gr.y * gr.y) + gr.z * gr.z);
        err = fmax(err, e);
    }
    l32 += 3;
    {   // a seed whose gradient norms lie within 2 sqrt(3) err of another's is chosen on FP64 lookups
        const double lo = fmin(gn[0], fmin(gn[1], gn[2]));
        int close = 0;
        for (int c = 0; c < 3; ++c) close += gn[c] - lo <= 4.0 * 1.7320508075688772 * err;
        if (close > 1) {
            for (int c = 0; c < 3; ++c) {
                const d3 gr = grid_gradient(g, ps[c]);
                gn[c] = sqrt((gr.x * gr.x + gr.y * gr.y) + gr.z * gr.z);
            }
            l64 += 3;
        }
    }
    int best = 0;
    if (gn[1] < gn[best]) best = 1;
    if (gn[2] < gn[best]) best = 2;
    trace = (uint32_t)best;
    d3 x = best == 0 ? ps[0] : (best == 1 ? ps[1] : ps[2]);
    n_fw = 0;
    for (int i = 0; i < max_it; ++i) {
        ++n_fw;
        double e;
        d3 gr = grid_gradient_f32(g, values32, x, e);
        ++l32;
        double o0 = dot3_np(ps[0], gr), o1 = dot3_np(ps[1], gr), o2 = dot3_np(ps[2], gr);
        const double margin = 4.0 * e * scale;
        const double lo = fmin(o0, fmin(o1, o2));
        const int close = (o0 - lo <= margin) + (o1 - lo <= margin) + (o2 - lo <= margin);
        if (close > 1 || fabs(lo - tol) <= margin) {   // decide on the FP64 gradient
            gr = grid_gradient(g, x);
            ++l64;
            o0 = dot3_np(ps[0], gr); o1 = dot3_np(ps[1], gr); o2 = dot3_np(ps[2], gr);
        }
        int v = 0;
        double ov = o0;
        if (o1 < ov) { v = 1; ov = o1; }
        if (o2 < ov) { v = 2; ov = o2; }
        if (i < 15) trace |= (uint32_t)v << (2 + 2 * i);
        const double alpha = 2.0 / (double)(i + 2);
        const d3 s = v == 0 ? ps[0] : (v == 1 ? ps[1] : ps[2]);
        x = d3{x.x + alpha * (s.x - x.x), x.y + alpha * (s.y - x.y), x.z + alpha * (s.z - x.z)};
        if (ov > tol) break;
    }
    return x;
}

// the plain FP64 search's trace and acceptance for a profiled step's check of the FP32 search (a call of its
// own, so that it does not raise the registers of the search itself)
__device__ __noinline__ void fw_check64(const GridView& g, const d3* ps, const double* qB, int max_it, double tol,
                                        double envelope, int& n64, uint32_t& trace64, int& accept64) {
    const d3 x64 = fw_search64(g, ps, max_it, tol, n64, trace64);
    accept64 = 0;
    if (grid_is_inside(g, x64, 0.5) && grid_value(g, x64) <= envelope)
        accept64 = norm3_np(quat_rotate(qB, grid_gradient(g, x64))) > 0.0;
}

// kF32: the seed and Frank-Wolfe lookups on the FP32 grid copy (near-ties decided on FP64 lookups); the
// acceptance tests (is_inside, phi <= envelope) and the contact's point, normal and gap in FP64 at the point
// found.  A step profiled with bit 2 set also runs the plain FP64 search and counts, per scene, the candidates
// whose search decisions or acceptance differ (a check of the error bound: zero when it holds).
template <bool kF32>
__global__ void __launch_bounds__(256, 2) k_narrow(const StepArgs a) {
    if (a.ws.counters[kAbort]) return;
    const int n_items = a.ws.counters[kNItems];
    const int max_it = a.pr.contact_optimization_max_iterations;
    const double tol = a.pr.contact_optimization_tolerance;
    const double envelope = a.pr.envelope;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < n_items; it += gridDim.x * blockDim.x) {
        const int p = a.ws.item_pair[it];
        const unsigned st = (unsigned)a.ws.item_tri[it];
        const int side = st >> 31, tri = st & 0x7fffffff;
        const int A = a.ws.pairs[2 * p], B = a.ws.pairs[2 * p + 1];
        const int mesh = side ? B : A, sdf = side ? A : B;
        const int sm = a.bd.shape[mesh], ss = a.bd.shape[sdf];
        const int32_t* T = a.sh.T + 3 * (size_t)(a.sh.t_off[sm] + tri);
        const double* Vw = a.ws.Vw + 3 * (size_t)a.bd.body_v0[mesh];
        const double* xB = a.bd.x + 7 * sdf;
        const double qB[4] = {xB[3], xB[4], xB[5], xB[6]};
        const double cqB[4] = {qB[0], -qB[1], -qB[2], -qB[3]};
        const d3 rB = d3{xB[0], xB[1], xB[2]};
        d3 ps[3];
        for (int c = 0; c < 3; ++c) {
            const d3 pw = ld3(Vw + 3 * T[c]);
            ps[c] = quat_rotate_row(cqB, sub(pw, rB));   // :120-121
        }
        const GridView g = load_grid(a.sh.grid_meta + 12 * ss, a.sh.grid + a.sh.g_off[ss]);
        int n_fw = 0, lookups = 0, lookups32 = 0;
        uint32_t trace = 0u;
        d3 x;
        if (kF32) {
            x = fw_search_f32(g, a.sh.grid32 + a.sh.g_off[ss], ps, max_it, tol, n_fw, trace, lookups, lookups32);
        } else {
            x = fw_search64(g, ps, max_it, tol, n_fw, trace);
            lookups = 3 + n_fw;   // seed gradients + one gradient per Frank-Wolfe iteration
        }
        int flag = 0;
        if (grid_is_inside(g, x, 0.5)) {   // :172 (is_inside default boundary 0.5)
            lookups += 1;
            const double phi = grid_value(g, x);
            if (phi <= envelope) {
                lookups += 1;
                const d3 nb = grid_gradient(g, x);
                const d3 nw = quat_rotate(qB, nb);
                const double ln = norm3_np(nw);
                if (ln > 0.0) {
                    const d3 xr = quat_rotate(qB, x);
                    st3(a.ws.item_p + 3 * (size_t)it, d3{xr.x + rB.x, xr.y + rB.y, xr.z + rB.z});
                    st3(a.ws.item_n + 3 * (size_t)it, d3{nw.x / ln, nw.y / ln, nw.z / ln});
                    a.ws.item_g[it] = phi;
                    flag = 1;
                    if (fabs(1.0 - norm3_np(d3{nw.x / ln, nw.y / ln, nw.z / ln})) > 0.1)   // types.py:293
                        atomicOr(a.out.status, RB_STATUS_NONUNIT_NORMAL);
                }
            }
        }
        a.ws.item_flag[it] = flag;
        if (a.pr.profiling) {   // statistics for the bandwidth accounting (lookups per scene) and decision flips
            const int s = scene_of(a.bd.scene_start, a.bd.n_scenes, A);
            atomicAdd(&a.out.stats[s].n_grid_lookups, lookups);
            if (kF32) atomicAdd(&a.out.stats[s].n_grid_lookups32, lookups32);
            if (kF32 && (a.pr.profiling & 2)) {   // the check against the plain FP64 search, on request
                int n64 = 0, accept64 = 0;
                uint32_t trace64 = 0u;
                fw_check64(g, ps, qB, max_it, tol, envelope, n64, trace64, accept64);
                if (n64 != n_fw || trace64 != trace) atomicAdd(&a.out.stats[s].n_search_flips, 1);
                if (accept64 != flag) atomicAdd(&a.out.stats[s].n_accept_flips, 1);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------------------
// contact reduction (collision_detection.py:255): a contact is dropped when an earlier contact of the same
// unordered body pair has the identical position.  Contacts of one body pair are contiguous (one pair list
// entry), so the test runs per pair.  Pass 1 counts survivors, pass 2 writes them in order.
// ---------------------------------------------------------------------------------------------------------
template <bool WRITE>
__global__ void k_dedup(const StepArgs a) {
    if (a.ws.counters[kAbort]) return;
    const int lane = threadIdx.x & 31;
    const int n_pairs = a.ws.counters[kNPairs];
    for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n_pairs; p += (gridDim.x * blockDim.x) >> 5) {
        const int i0 = a.ws.pair_items[p], i1 = i0 + a.ws.pair_itemsA[p];
        int kept = 0;
        int base = WRITE ? a.ws.pair_cont[p] : 0;
        const int A = a.ws.pairs[2 * p], B = a.ws.pairs[2 * p + 1];
        for (int c0 = i0; c0 < i1; c0 += 32) {
            const int i = c0 + lane;
            bool keep = false;
            if (!WRITE) {
                // candidate i is kept if no earlier accepted candidate of the pair has its position: the
                // earlier accepted ones, 32 at a time, are found by ballot and their positions broadcast
                const bool mine = i < i1 && a.ws.item_flag[i] != 0;
                double px = 0.0, py = 0.0, pz = 0.0;
                if (mine) { const double* pi = a.ws.item_p + 3 * (size_t)i; px = pi[0]; py = pi[1]; pz = pi[2]; }
                keep = mine;
                for (int e0 = i0; e0 <= c0; e0 += 32) {
                    const int j = e0 + lane;
                    const bool fj = j < i1 && (e0 == c0 ? mine : a.ws.item_flag[j] != 0);
                    double qx = 0.0, qy = 0.0, qz = 0.0;
                    if (fj) { const double* pj = a.ws.item_p + 3 * (size_t)j; qx = pj[0]; qy = pj[1]; qz = pj[2]; }
                    unsigned m = __ballot_sync(0xffffffffu, fj);
                    while (m) {   // in the own chunk only lanes below this one count as earlier
                        const int b = __ffs(m) - 1;
                        m &= m - 1;
                        const double bx = __shfl_sync(0xffffffffu, qx, b);
                        const double by = __shfl_sync(0xffffffffu, qy, b);
                        const double bz = __shfl_sync(0xffffffffu, qz, b);
                        const bool earlier = e0 < c0 || b < lane;
                        if (keep && earlier && px == bx && py == by && pz == bz) keep = false;
                    }
                }
            } else {
                keep = i < i1 && a.ws.item_flag[i] == 2;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (!WRITE && i < i1 && keep) a.ws.item_flag[i] = 2;   // the write pass reads flag 2 = kept
            if (WRITE && keep) {
                const int k = base + kept + __popc(bal & lanemask_lt());
                if (k < a.caps.contact_capacity) {
                    const int side = ((unsigned)a.ws.item_tri[i]) >> 31;
                    const int mesh = side ? B : A, sdf = side ? A : B;
                    a.out.contact_ids[2 * k] = sdf;     // ContactPoint(bodyB_sdf_owner, bodyA_mesh_owner, ...)
                    a.out.contact_ids[2 * k + 1] = mesh;
                    for (int c = 0; c < 3; ++c) {
                        a.out.contact_p[3 * k + c] = a.ws.item_p[3 * (size_t)i + c];
                        a.out.contact_n[3 * k + c] = a.ws.item_n[3 * (size_t)i + c];
                    }
                    a.out.contact_g[k] = a.ws.item_g[i];
                    a.ws.c_scene[k] = scene_of(a.bd.scene_start, a.bd.n_scenes, A);
                    // key of the contact for warm starting: contacts come out in ascending key order
                    a.ws.ckey[2 * k] = ((int64_t)A << 31) | (int64_t)B;
                    a.ws.ckey[2 * k + 1] = (int64_t)(((unsigned)a.ws.item_tri[i] >> 31) << 30) |
                                           (int64_t)(a.ws.item_tri[i] & 0x7fffffff);
                }
            }
            kept += __popc(bal);
        }
        if (!WRITE && lane == 0) a.ws.pair_cont[p] = kept;
    }
}

// ---------------------------------------------------------------------------------------------------------
// contact problem (contacts.py:31 initialize): thread per contact
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ double jrow_dot(const double* Jr, const double* wlo, const double* whi) {
    double s = 0.0;
    for (int c = 0; c < 6; ++c) s += Jr[c] * wlo[c];
    for (int c = 0; c < 6; ++c) s += Jr[6 + c] * whi[c];
    return s;
}

__global__ void k_contacts(const StepArgs a) {
    // one thread per (contact, row): row q's J and W J^T blocks, b, Delassus diagonal, r and start impulse;
    // the row-0 thread also writes the contact's body pair and mu
    if (a.ws.counters[kAbort]) return;
    const int K = a.ws.counters[kNContacts];
    const double dt = a.pr.dt;
    double r_scale = a.pr.scheme == RB_SCHEME_RIGID_GS ? 1.0 : 0.1;   // solver_interface.py:48
    if (a.pr.termination == RB_TERMINATE_RESIDUAL_FIXED_R && a.pr.relaxation > 0.0) r_scale *= a.pr.relaxation;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 4 * K; t += gridDim.x * blockDim.x) {
        const int k = t >> 2, row = t & 3;
        const int A = a.out.contact_ids[2 * k], B = a.out.contact_ids[2 * k + 1];
        const d3 p = ld3(a.out.contact_p + 3 * k);
        const d3 rA = sub(p, ld3(a.bd.x + 7 * A)), rB = sub(p, ld3(a.bd.x + 7 * B));
        d3 vs, vt, vn;
        make_orthonormal_vectors(ld3(a.out.contact_n + 3 * k), vs, vt, vn);   // (t, b, n)
        const int lo = min(A, B), hi = max(A, B);
        const int offA = (A == lo) ? 0 : 6, offB = (B == lo) ? 0 : 6;
        double* J = a.ws.J + 48 * (size_t)k + 12 * row;
        double* W = a.ws.WJT + 48 * (size_t)k + 12 * row;
        double* JA = J + offA;
        double* JB = J + offB;
        if (row < 3) {   // contacts.py:140-147
            const d3 d = row == 0 ? vn : (row == 1 ? vs : vt);
            const d3 ca = cross_np(rA, d), cb = cross_np(rB, d);
            JA[0] = -d.x; JA[1] = -d.y; JA[2] = -d.z; JA[3] = -ca.x; JA[4] = -ca.y; JA[5] = -ca.z;
            JB[0] = d.x; JB[1] = d.y; JB[2] = d.z; JB[3] = cb.x; JB[4] = cb.y; JB[5] = cb.z;
        } else {
            JA[0] = -0.0; JA[1] = -0.0; JA[2] = -0.0; JA[3] = -vn.x; JA[4] = -vn.y; JA[5] = -vn.z;
            JB[0] = 0.0; JB[1] = 0.0; JB[2] = 0.0; JB[3] = vn.x; JB[4] = vn.y; JB[5] = vn.z;
        }
        bool hasw[2];
        for (int side = 0; side < 2; ++side) {   // WJT = W J^T (bsr_matmat order)
            const int bb = side ? hi : lo;
            hasw[side] = !a.bd.fixed[bb];
            const double m = hasw[side] ? 1.0 / a.bd.mass[bb] : 0.0;
            const double* Wi = a.ws.Winv + 9 * bb;
            const double* Jr = J + 6 * side;
            double* Wr = W + 6 * side;
            for (int i = 0; i < 3; ++i) {
                double s = 0.0;
                s += (i == 0 ? m : 0.0) * Jr[0];
                s += (i == 1 ? m : 0.0) * Jr[1];
                s += (i == 2 ? m : 0.0) * Jr[2];
                double tt = 0.0;
                tt += Wi[3 * i + 0] * Jr[3];
                tt += Wi[3 * i + 1] * Jr[4];
                tt += Wi[3 * i + 2] * Jr[5];
                Wr[i] = hasw[side] ? s : 0.0;
                Wr[3 + i] = hasw[side] ? tt : 0.0;
            }
        }
        // b = (1 + e) v + J (dt W f_ext) + g   (contacts.py:46)
        const int sc = scene_of(a.bd.scene_start, a.bd.n_scenes, A);
        const int M = a.bd.scene_material_count[sc];
        const int entry = a.bd.scene_material_offset[sc] + a.bd.material[A] * M + a.bd.material[B];
        const double eps = a.pr.use_bounce ? a.bd.material_eps[entry] : 0.0;
        const double* ulo = a.bd.u + 6 * lo;
        const double* uhi = a.bd.u + 6 * hi;
        const double* dlo = a.ws.du + 6 * lo;
        const double* dhi = a.ws.du + 6 * hi;
        const double vrow = jrow_dot(J, ulo, uhi);
        double gk0 = 0.0;
        if (row == 0 && a.pr.use_pre_stabilization) {   // contacts.py:188 _compute_error_vector
            const double gap = a.out.contact_g[k];
            const double rate = a.pr.gap_reduction / dt;
            const double upper = -a.pr.max_gap_value / dt;
            const double lower = -a.pr.min_gap_value;
            if (gap < lower && vrow <= 0.0) {
                const double tg = rate * gap;
                gk0 = upper > tg ? upper : tg;
            }
        }
        const double jd = jrow_dot(J, dlo, dhi);
        const double e = row == 0 ? eps : 0.0;
        a.ws.b[4 * k + row] = ((1.0 + e) * vrow + jd) + gk0;
        // Delassus diagonal: reduceat over the nonzero products J .* WJT^T in column order (contacts.py:49)
        double prods[12];
        int m = 0;
        for (int c = 0; c < 12; ++c) {
            if (!hasw[c / 6]) continue;
            const double pr = J[c] * W[c];
            if (pr != 0.0) prods[m++] = pr;
        }
        double dg = np_reduce_sum(prods, m);
        if (dg == 0.0) dg = 1.0;
        a.ws.diag[4 * k + row] = dg;
        a.ws.r[4 * k + row] = r_scale / dg;
        double x0 = 0.0;
        if (a.pr.warm_start && a.out.cache_count) {   // previous impulse of the same contact (binary search)
            const int64_t k1 = a.ws.ckey[2 * k], k2 = a.ws.ckey[2 * k + 1];
            int lo_i = 0, hi_i = min(*a.out.cache_count, a.caps.contact_capacity);
            while (lo_i < hi_i) {
                const int mid = (lo_i + hi_i) >> 1;
                const int64_t m1 = a.out.cache_key[2 * mid], m2 = a.out.cache_key[2 * mid + 1];
                if (m1 < k1 || (m1 == k1 && m2 < k2)) lo_i = mid + 1; else hi_i = mid;
            }
            if (lo_i < *a.out.cache_count && a.out.cache_key[2 * lo_i] == k1 && a.out.cache_key[2 * lo_i + 1] == k2)
                x0 = a.out.cache_sol[4 * lo_i + row];
        }
        a.ws.x[4 * k + row] = x0;
        a.out.contact_sol[4 * k + row] = x0;
        if (row == 0) {
            a.ws.lohi[2 * k] = lo;
            a.ws.lohi[2 * k + 1] = hi;
            a.ws.mu[k] = a.bd.material_mu[3 * entry];
        }
    }
}

// per-body contact lists, ascending contact index (the column order of the SciPy products)
__global__ void k_body_contacts_count(const StepArgs a) {
    if (a.ws.counters[kAbort]) return;
    const int K = a.ws.counters[kNContacts];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x)
        for (int side = 0; side < 2; ++side) {
            const int b = a.ws.lohi[2 * k + side];
            if (!a.bd.fixed[b]) atomicAdd(a.ws.bc_ptr + b, 1);
        }
}
__global__ void k_body_contacts_fill(const StepArgs a) {
    if (a.ws.counters[kAbort]) return;
    const int K = a.ws.counters[kNContacts];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x)
        for (int side = 0; side < 2; ++side) {
            const int b = a.ws.lohi[2 * k + side];
            if (a.bd.fixed[b]) continue;
            const int at = a.ws.bc_ptr[b] + atomicAdd(a.ws.bc_fill + b, 1);
            a.ws.bc_list[at] = (k << 1) | side;
        }
}
__global__ void k_body_contacts_sort(const StepArgs a) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.bd.n_bodies || a.ws.counters[kAbort]) return;
    int32_t* l = a.ws.bc_list + a.ws.bc_ptr[b];
    const int n = a.ws.bc_ptr[b + 1] - a.ws.bc_ptr[b];
    for (int i = 1; i < n; ++i) {
        const int32_t v = l[i];
        int j = i - 1;
        while (j >= 0 && l[j] > v) { l[j + 1] = l[j]; --j; }
        l[j + 1] = v;
    }
    // predecessor of each contact along this body: the chain the Gauss-Seidel levels follow
    int prev = -1;
    for (int i = 0; i < n; ++i) {
        const int code = l[i];
        a.ws.cpred[code] = prev;   // code = (k << 1) | side
        prev = code >> 1;
    }
}
__global__ void k_preds_init(const StepArgs a) {
    if (a.ws.counters[kAbort]) return;
    const int K = a.ws.counters[kNContacts];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * K; i += gridDim.x * blockDim.x) a.ws.cpred[i] = -1;
}

// w[b] = (WJT x) rows of body b: sequential over its contacts (ascending) and their 4 columns.  The loads of
// four contacts are issued before their products are accumulated (in order) to overlap their latency.
__device__ __forceinline__ void body_wjt_dot(const Workspace& ws, int b, const double* x, double* out6) {
    double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int e0 = ws.bc_ptr[b], e1 = ws.bc_ptr[b + 1];
    int e = e0;
    for (; e + 4 <= e1; e += 4) {
        int code[4];
        for (int j = 0; j < 4; ++j) code[j] = ws.bc_list[e + j];
        double xv[4][4];
        const double* Wk[4];
        for (int j = 0; j < 4; ++j) {
            const int k = code[j] >> 1;
            Wk[j] = ws.WJT + 48 * (size_t)k + 6 * (code[j] & 1);
            for (int i = 0; i < 4; ++i) xv[j][i] = x[4 * k + i];
        }
        for (int d = 0; d < 6; ++d) {
            double t = s[d];
            for (int j = 0; j < 4; ++j) {
                t += Wk[j][d] * xv[j][0];
                t += Wk[j][12 + d] * xv[j][1];
                t += Wk[j][24 + d] * xv[j][2];
                t += Wk[j][36 + d] * xv[j][3];
            }
            s[d] = t;
        }
    }
    for (; e < e1; ++e) {
        const int code = ws.bc_list[e];
        const int k = code >> 1, side = code & 1;
        const double* Wk = ws.WJT + 48 * (size_t)k + 6 * side;
        const double x0 = x[4 * k], x1 = x[4 * k + 1], x2 = x[4 * k + 2], x3 = x[4 * k + 3];
        for (int d = 0; d < 6; ++d) {
            double t = s[d];
            t += Wk[d] * x0;
            t += Wk[12 + d] * x1;
            t += Wk[24 + d] * x2;
            t += Wk[36 + d] * x3;
            s[d] = t;
        }
    }
    for (int d = 0; d < 6; ++d) out6[d] = s[d];
}

// ---------------------------------------------------------------------------------------------------------
// solver: one thread group per scene -- a warp for small scenes (warp-synchronous, many scenes per SM), a
// block for large ones.  Every member of the group evaluates the solver's control logic redundantly from the
// same reduced values, so no broadcast through shared memory is needed.
// ---------------------------------------------------------------------------------------------------------
struct SceneRange { int b0, b1, c0, c1; };
__device__ __forceinline__ SceneRange scene_range(const StepArgs& a, int s) {
    SceneRange R;
    R.b0 = a.bd.scene_start[s];
    R.b1 = a.bd.scene_start[s + 1];
    // contacts follow the pair order, pairs follow the body order
    const int p0 = a.ws.pair_cnt[R.b0], p1 = a.ws.pair_cnt[R.b1];
    R.c0 = a.ws.pair_cont[p0];
    R.c1 = a.ws.pair_cont[p1];
    return R;
}

__device__ __forceinline__ double nanmax(double v, double t) { return (t > v || t != t) ? t : v; }

struct WarpGroup {
    __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
    __device__ __forceinline__ int size() const { return 32; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    __device__ __forceinline__ bool any(bool p) const { __syncwarp(); return __any_sync(0xffffffffu, p); }
    __device__ __forceinline__ double max(double v) const {
        for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        return v;
    }
    __device__ __forceinline__ int imax(int v) const {
        for (int o = 16; o > 0; o >>= 1) v = ::max(v, __shfl_xor_sync(0xffffffffu, v, o));
        return v;
    }
};

struct BlockGroup {
    double* red;   // 33 doubles of shared memory
    int* ired;     // 33 ints of shared memory
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ int size() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ bool any(bool p) const { return __syncthreads_or(p); }
    __device__ double max(double v) const {
        for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        __syncthreads();
        if (lane == 0) red[wid] = v;
        __syncthreads();
        double m = red[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) m = nanmax(m, red[k]);
        __syncthreads();
        return m;
    }
    __device__ int imax(int v) const {
        for (int o = 16; o > 0; o >>= 1) v = ::max(v, __shfl_xor_sync(0xffffffffu, v, o));
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
        __syncthreads();
        if (lane == 0) ired[wid] = v;
        __syncthreads();
        int m = ired[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) m = ::max(m, ired[k]);
        __syncthreads();
        return m;
    }
};

// Body accumulators w = WJT x of one scene: in shared memory when the scene fits, else in global memory.
struct WView {
    double* base;
    int b0;
    __device__ __forceinline__ double* at(int b) const { return base + 6 * (b - b0); }
};

// w for every body of the scene from x (sequential over the body's contacts: the order of WJT.dot(x))
template <class G>
__device__ __forceinline__ void scene_wjt(const StepArgs& a, const G& g, const SceneRange& R, const double* x, WView w) {
    for (int bb = R.b0 + g.rank(); bb < R.b1; bb += g.size()) {
        double* o = w.at(bb);
        if (a.bd.fixed[bb]) { for (int d = 0; d < 6; ++d) o[d] = 0.0; continue; }
        body_wjt_dot(a.ws, bb, x, o);
    }
    g.sync();
}

// One projected Gauss-Seidel update of contact k (contacts.py:78-107): z from the current w, normal impulse
// clamped at zero, friction projected on the ball of radius mu x_n (or zeroed for post-stabilisation),
// then w += WJT[:, block] delta with the reference's term order.
__device__ __forceinline__ void gs_contact(const StepArgs& a, int k, const double* b, const double* r, double* x,
                                           WView w, bool normal_only) {
    const int lo = a.ws.lohi[2 * k], hi = a.ws.lohi[2 * k + 1];
    const double* J = a.ws.J + 48 * (size_t)k;
    const double* Wk = a.ws.WJT + 48 * (size_t)k;
    const double* wlo = w.at(lo);
    const double* whi = w.at(hi);
    double xo[4], z[4];
    for (int row = 0; row < 4; ++row) {
        xo[row] = x[4 * k + row];
        z[row] = xo[row] - r[4 * k + row] * (jrow_dot(J + 12 * row, wlo, whi) + b[4 * k + row]);
    }
    const double xn = z[0] > 0.0 ? z[0] : 0.0;
    double f[3];
    if (normal_only) { f[0] = 0.0; f[1] = 0.0; f[2] = 0.0; }
    else prox_sphere(z[1], z[2], z[3], a.ws.mu[k], xn, f);
    const double d0 = xn - xo[0], d1 = f[0] - xo[1], d2 = f[1] - xo[2], d3v = f[2] - xo[3];
    x[4 * k] = xn; x[4 * k + 1] = f[0]; x[4 * k + 2] = f[1]; x[4 * k + 3] = f[2];
    for (int side = 0; side < 2; ++side) {
        const int bb = side ? hi : lo;
        if (a.bd.fixed[bb]) continue;
        double* wb = w.at(bb);
        const double* Ws = Wk + 6 * side;
        for (int d = 0; d < 6; ++d) {
            double t = 0.0;
            t += Ws[d] * d0;
            t += Ws[12 + d] * d1;
            t += Ws[24 + d] * d2;
            t += Ws[36 + d] * d3v;
            wb[d] = wb[d] + t;
        }
    }
}

// Wavefront levels of the serial Gauss-Seidel order: level(k) = 1 + max level of the earlier contacts on
// k's non-fixed bodies.  Contacts of one level share no non-fixed body and every body sees its contacts in
// ascending order, so sweeping level by level (each level in parallel, any order inside a level) reproduces
// the serial sweep exactly.  The levels are the longest-path depths along the per-body predecessor chains,
// found by parallel relaxation; contacts are then bucketed by level.  Returns the number of levels.
template <class G>
__device__ int bucket_classes(const StepArgs& a, const G& g, const SceneRange& R, int s);

template <class G>
__device__ int scene_levels(const StepArgs& a, const G& g, const SceneRange& R, int s) {
    for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) a.ws.lev_of[k] = 1;
    g.sync();
    for (;;) {
        bool changed = false;
        for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) {
            const int p0 = a.ws.cpred[2 * k], p1 = a.ws.cpred[2 * k + 1];
            const int l0 = p0 >= 0 ? *(volatile int*)(a.ws.lev_of + p0) : 0;
            const int l1 = p1 >= 0 ? *(volatile int*)(a.ws.lev_of + p1) : 0;
            const int l = 1 + max(l0, l1);
            if (l != a.ws.lev_of[k]) { a.ws.lev_of[k] = l; changed = true; }
        }
        if (!g.any(changed)) break;
    }
    return bucket_classes(a, g, R, s);
}

// The same levels with the relaxation and the bucketing in shared memory: scratch (s32_level_scratch bytes)
// holds the two predecessors of each contact (scene-local int16), its level (int16) and one counter per level;
// the levels then go to lev_of and the buckets to lev_ptr / lev_order.  Same fixed point, same order within a
// level up to the order of atomics, which no result depends on.
__host__ __device__ inline size_t s32_level_scratch(int K) { return 6 * (size_t)K + 4 * (size_t)(K + 2) + 16; }
template <class G>
__device__ int scene_levels_smem(const StepArgs& a, const G& g, const SceneRange& R, int s, int16_t* scratch) {
    const int K = R.c1 - R.c0;
    int16_t* pred = scratch;
    volatile int16_t* lev = scratch + 2 * K;
    int* cnt = reinterpret_cast<int*>(reinterpret_cast<char*>(scratch) + ((6 * (size_t)K + 15) & ~size_t(15)));
    for (int k = g.rank(); k < K; k += g.size()) {
        const int p0 = a.ws.cpred[2 * (R.c0 + k)], p1 = a.ws.cpred[2 * (R.c0 + k) + 1];
        pred[2 * k] = (int16_t)(p0 >= 0 ? p0 - R.c0 : -1);
        pred[2 * k + 1] = (int16_t)(p1 >= 0 ? p1 - R.c0 : -1);
        lev[k] = 1;
    }
    g.sync();
    for (;;) {
        bool changed = false;
        for (int k = g.rank(); k < K; k += g.size()) {
            const int p0 = pred[2 * k], p1 = pred[2 * k + 1];
            const int l0 = p0 >= 0 ? lev[p0] : 0;
            const int l1 = p1 >= 0 ? lev[p1] : 0;
            const int l = 1 + max(l0, l1);
            if (l != lev[k]) { lev[k] = (int16_t)l; changed = true; }
        }
        if (!g.any(changed)) break;
    }
    int L = 0;
    for (int k = g.rank(); k < K; k += g.size()) {
        const int l = lev[k];
        a.ws.lev_of[R.c0 + k] = l;
        L = max(L, l);
    }
    L = g.imax(L);
    for (int l = g.rank(); l <= L; l += g.size()) cnt[l] = 0;
    g.sync();
    for (int k = g.rank(); k < K; k += g.size()) atomicAdd(cnt + lev[k] - 1, 1);
    g.sync();
    int* ptr = a.ws.lev_ptr + R.c0 + s;   // ptr[l-1] .. ptr[l]: contacts of level l (1-based), ptr[L] = K
    if (g.rank() == 0) {
        int acc = 0;
        for (int l = 0; l < L; ++l) { const int c = cnt[l]; ptr[l] = acc; cnt[l] = acc; acc += c; }
        ptr[L] = acc;
    }
    g.sync();
    // the order within a level does not change any result (its contacts share no body that is written)
    for (int k = g.rank(); k < K; k += g.size()) a.ws.lev_order[R.c0 + atomicAdd(cnt + lev[k] - 1, 1)] = R.c0 + k;
    g.sync();
    return L;
}

// Groups the scene's contacts by their class lev_of[k] (1-based level or colour): lev_ptr[c-1] .. lev_ptr[c]
// index lev_order, which lists the contacts of class c.  Returns the number of classes.
template <class G>
__device__ int bucket_classes(const StepArgs& a, const G& g, const SceneRange& R, int s) {
    int L = 0;
    for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) L = max(L, a.ws.lev_of[k]);
    L = g.imax(L);
    int* ptr = a.ws.lev_ptr + R.c0 + s;   // ptr[l-1] .. ptr[l]: contacts of level l (1-based), ptr[L] = K
    int* cur = a.ws.lev_cur + R.c0 + s;
    for (int l = g.rank(); l <= L; l += g.size()) cur[l] = 0;
    g.sync();
    for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) atomicAdd(cur + a.ws.lev_of[k] - 1, 1);
    g.sync();
    if (g.rank() == 0) {
        int acc = 0;
        for (int l = 0; l < L; ++l) { const int c = cur[l]; ptr[l] = acc; cur[l] = acc; acc += c; }
        ptr[L] = acc;
    }
    g.sync();
    for (int k = R.c0 + g.rank(); k < R.c1; k += g.size())
        a.ws.lev_order[R.c0 + atomicAdd(cur + a.ws.lev_of[k] - 1, 1)] = k;
    g.sync();
    return L;
}

// Graph colouring of the scene's contacts for RB_ORDER_COLOURED: two contacts are neighbours when they share a
// non-fixed body.  Jones-Plassmann rounds with hashed priorities (higher hash first, then lower scene-local
// index): in each round every uncoloured contact whose uncoloured neighbours all come later in priority takes
// the smallest colour none of its coloured neighbours has.  Deterministic, so every launch shape gives the
// same colours; the oracle's rbo_colour_contacts is the same procedure.
__device__ __forceinline__ uint32_t jp_hash(uint32_t k) {
    k ^= k >> 16; k *= 0x7feb352dU; k ^= k >> 15; k *= 0x846ca68bU; k ^= k >> 16;
    return k;
}
__device__ __forceinline__ bool jp_before(int p, int q) {
    const uint32_t hp = jp_hash((uint32_t)p), hq = jp_hash((uint32_t)q);
    return hp > hq || (hp == hq && p < q);
}
// colour (0-based) contact k takes this round, or -1 while a neighbour of higher priority is uncoloured
__device__ int colour_pick(const StepArgs& a, const SceneRange& R, int k) {
    const int* col = a.ws.lev_of;   // colour + 1; 0 = uncoloured
    uint64_t used = 0;
    for (int side = 0; side < 2; ++side) {
        const int b = a.ws.lohi[2 * k + side];
        if (a.bd.fixed[b]) continue;
        for (int e = a.ws.bc_ptr[b]; e < a.ws.bc_ptr[b + 1]; ++e) {
            const int m = a.ws.bc_list[e] >> 1;
            if (m == k) continue;
            const int c = col[m];
            if (c == 0) {
                if (jp_before(m - R.c0, k - R.c0)) return -1;
            } else if (c <= 64) {
                used |= 1ull << (c - 1);
            }
        }
    }
    for (int c = 0;; ++c) {
        bool taken = false;
        if (c < 64) {
            taken = (used >> c) & 1ull;
        } else {
            for (int side = 0; side < 2 && !taken; ++side) {
                const int b = a.ws.lohi[2 * k + side];
                if (a.bd.fixed[b]) continue;
                for (int e = a.ws.bc_ptr[b]; e < a.ws.bc_ptr[b + 1] && !taken; ++e) {
                    const int m = a.ws.bc_list[e] >> 1;
                    taken = m != k && col[m] == c + 1;
                }
            }
        }
        if (!taken) return c;
    }
}
template <class G>
__device__ int scene_colours(const StepArgs& a, const G& g, const SceneRange& R, int s) {
    int* col = a.ws.lev_of;
    int* pick = a.ws.lev_cur + R.c0 + s;   // this round's choices (the class counters are built afterwards)
    for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) col[k] = 0;
    g.sync();
    const int K = R.c1 - R.c0;
    for (int round = 0; round <= K; ++round) {   // every round colours at least the top-priority contact
        bool left = false;
        for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) {
            int c = -1;
            if (col[k] == 0) { c = colour_pick(a, R, k); left = true; }
            pick[k - R.c0] = c;
        }
        g.sync();
        if (!g.any(left)) break;
        for (int k = R.c0 + g.rank(); k < R.c1; k += g.size())
            if (pick[k - R.c0] >= 0) col[k] = pick[k - R.c0] + 1;
        g.sync();
    }
    return bucket_classes(a, g, R, s);
}

template <class G>
__device__ __forceinline__ void gs_sweep_levels(const StepArgs& a, const G& g, const SceneRange& R, int s, int L,
                                                const double* b, const double* r, double* x, WView w,
                                                bool normal_only) {
    const int* ptr = a.ws.lev_ptr + R.c0 + s;
    for (int l = 1; l <= L; ++l) {
        const int start = ptr[l - 1], end = ptr[l];
        if (l < L) {   // pull the next level's Jacobian blocks into L1 while this level runs
            const int i = end + g.rank();
            if (i < ptr[l + 1]) {
                const int kn = a.ws.lev_order[R.c0 + i];
                const char* pj = reinterpret_cast<const char*>(a.ws.J + 48 * (size_t)kn);
                const char* pw = reinterpret_cast<const char*>(a.ws.WJT + 48 * (size_t)kn);
                for (int off = 0; off < 384; off += 128) {
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(pj + off));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(pw + off));
                }
            }
        }
        for (int i = start + g.rank(); i < end; i += g.size())
            gs_contact(a, a.ws.lev_order[R.c0 + i], b, r, x, w, normal_only);
        g.sync();
    }
}

// complementarity residual ||x - prox(x - D^-1 (A x + b))||_inf / max(1, ||x||_inf), D = diag(A): the
// tolerance the solver modes are compared at.  Every scheme scales the prox argument by a positive multiple of
// D^-1, so they all share this map's zeros as fixed points.  A x = J W J^T x through w = WJT x (the
// accumulators are rebuilt from x at the start of every sweep, so they are free to hold this product here).
template <class G>
__device__ double scene_residual(const StepArgs& a, const G& g, const SceneRange& R, const double* x, WView w) {
    scene_wjt(a, g, R, x, w);
    double m = 0.0, xm = 0.0;
    for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) {
        const int lo = a.ws.lohi[2 * k], hi = a.ws.lohi[2 * k + 1];
        const double* J = a.ws.J + 48 * (size_t)k;
        double z[4];
        for (int row = 0; row < 4; ++row)
            z[row] = x[4 * k + row] -
                     (1.0 / a.ws.diag[4 * k + row]) * (jrow_dot(J + 12 * row, w.at(lo), w.at(hi)) + a.ws.b[4 * k + row]);
        const double pn = z[0] > 0.0 ? z[0] : 0.0;
        double f[3];
        prox_sphere(z[1], z[2], z[3], a.ws.mu[k], pn, f);
        const double d[4] = {x[4 * k] - pn, x[4 * k + 1] - f[0], x[4 * k + 2] - f[1], x[4 * k + 3] - f[2]};
        for (int i = 0; i < 4; ++i) {
            m = nanmax(m, fabs(d[i]));
            xm = fmax(xm, fabs(x[4 * k + i]));
        }
    }
    const double mres = g.max(m);
    const double mx = g.max(xm);
    return mres / (mx > 1.0 ? mx : 1.0);
}

// ---------------------------------------------------------------------------------------------------------
// hinge joints (constraints/hinges.py): 5 rows per hinge between a parent and a child body
// ---------------------------------------------------------------------------------------------------------
// per-body hinge lists of each scene (thread per scene): entries (hinge << 1 | side), hinges ascending; every
// hinge gives both of its bodies an entry, so scene s's entries fill [2 h0, 2 h1) exactly
__global__ void k_hinge_lists(const StepArgs a) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.bd.n_scenes || a.ws.counters[kAbort]) return;
    const int b0 = a.bd.scene_start[s], b1 = a.bd.scene_start[s + 1];
    const int h0 = a.bd.scene_hinge_start[s], h1 = a.bd.scene_hinge_start[s + 1];
    int32_t* cnt = a.ws.hlast;
    for (int b = b0; b < b1; ++b) cnt[b] = 0;
    for (int k = h0; k < h1; ++k) { cnt[a.bd.hinge_bodies[2 * k]]++; cnt[a.bd.hinge_bodies[2 * k + 1]]++; }
    int pos = 2 * h0;
    for (int b = b0; b < b1; ++b) { a.ws.hbody_ptr[b] = pos; pos += cnt[b]; cnt[b] = 0; }
    if (s == a.bd.n_scenes - 1) a.ws.hbody_ptr[a.bd.n_bodies] = pos;
    for (int k = h0; k < h1; ++k)
        for (int side = 0; side < 2; ++side) {
            const int P = a.bd.hinge_bodies[2 * k], C = a.bd.hinge_bodies[2 * k + 1];
            const int b = side ? max(P, C) : min(P, C);
            a.ws.hbody_list[a.ws.hbody_ptr[b] + cnt[b]++] = (k << 1) | side;
        }
}

// hinges.py:28-50 Hinges.initialize with _compute_jacobian_matrix (:95-180) and _compute_error_vector
// (:188-218): J, W J^T (bsr_matmat order), b = (J u + J dt du_ext) + g, diag = sum(J .* WJT^T) (zeros -> 1),
// r = 1/diag, x = sol = 0.  Thread per hinge.
__global__ void k_hinges(const StepArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.bd.n_hinges || a.ws.counters[kAbort]) return;
    const int A = a.bd.hinge_bodies[2 * k], B = a.bd.hinge_bodies[2 * k + 1];
    const double* f = a.bd.hinge_frames + 12 * (size_t)k;
    const double* qA = a.bd.x + 7 * A + 3;
    const double* qB = a.bd.x + 7 * B + 3;
    const d3 ap = quat_rotate(qA, ld3(f)), ac = quat_rotate(qB, ld3(f + 3)), np_ = quat_rotate(qA, ld3(f + 6));
    d3 t, bb, nn;
    make_orthonormal_vectors(np_, t, bb, nn);
    // JA_v[0:3] = I, JA_w[0:3] = -star(arm_p), JA_w[3] = t, JA_w[4] = b; JB_v[0:3] = -I, JB_w[0:3] = star(arm_c),
    // JB_w[3] = -t, JB_w[4] = -b; star(v) = [[0, -v2, v1], [v2, 0, -v0], [-v1, v0, 0]]
    const double sp[3][3] = {{0.0, -ap.z, ap.y}, {ap.z, 0.0, -ap.x}, {-ap.y, ap.x, 0.0}};
    const double sc[3][3] = {{0.0, -ac.z, ac.y}, {ac.z, 0.0, -ac.x}, {-ac.y, ac.x, 0.0}};
    double JA[5][6], JB[5][6];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 6; ++j) { JA[i][j] = 0.0; JB[i][j] = 0.0; }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            JA[i][j] = i == j ? 1.0 : 0.0;
            JA[i][3 + j] = -sp[i][j];
            JB[i][j] = -(i == j ? 1.0 : 0.0);
            JB[i][3 + j] = sc[i][j];
        }
    const double tv[3] = {t.x, t.y, t.z}, bv[3] = {bb.x, bb.y, bb.z};
    for (int j = 0; j < 3; ++j) {
        JA[3][3 + j] = tv[j]; JA[4][3 + j] = bv[j];
        JB[3][3 + j] = -tv[j]; JB[4][3 + j] = -bv[j];
    }
    const int lo = min(A, B), hi = max(A, B);
    a.ws.hlohi[2 * k] = lo;
    a.ws.hlohi[2 * k + 1] = hi;
    double* J = a.ws.hJ + 60 * (size_t)k;
    double* W = a.ws.hWJT + 60 * (size_t)k;
    for (int row = 0; row < 5; ++row)
        for (int j = 0; j < 6; ++j) {
            J[12 * row + (A == lo ? 0 : 6) + j] = JA[row][j];
            J[12 * row + (B == lo ? 0 : 6) + j] = JB[row][j];
        }
    bool hasw[2];
    for (int side = 0; side < 2; ++side) {
        const int bd = side ? hi : lo;
        hasw[side] = !a.bd.fixed[bd];
        const double m = hasw[side] ? 1.0 / a.bd.mass[bd] : 0.0;
        const double* Wi = a.ws.Winv + 9 * (size_t)bd;
        for (int row = 0; row < 5; ++row) {
            const double* Jr = J + 12 * row + 6 * side;
            double* Wr = W + 12 * row + 6 * side;
            for (int i = 0; i < 3; ++i) {
                double s = 0.0;
                s += (i == 0 ? m : 0.0) * Jr[0];
                s += (i == 1 ? m : 0.0) * Jr[1];
                s += (i == 2 ? m : 0.0) * Jr[2];
                double u = 0.0;
                u += Wi[3 * i + 0] * Jr[3];
                u += Wi[3 * i + 1] * Jr[4];
                u += Wi[3 * i + 2] * Jr[5];
                Wr[i] = hasw[side] ? s : 0.0;
                Wr[3 + i] = hasw[side] ? u : 0.0;
            }
        }
    }
    double g[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (a.pr.use_pre_stabilization) {
        const d3 rp = add(ap, ld3(a.bd.x + 7 * A)), rc = add(ac, ld3(a.bd.x + 7 * B));
        const d3 ncv = quat_rotate(qB, ld3(f + 9));
        const d3 u = cross_np(nn, ncv);
        const double rate = a.pr.gap_reduction / a.pr.dt;
        g[0] = (rc.x - rp.x) * rate;
        g[1] = (rc.y - rp.y) * rate;
        g[2] = (rc.z - rp.z) * rate;
        g[3] = dot3_np(t, u) * rate;
        g[4] = dot3_np(bb, u) * rate;
    }
    const double* ulo = a.bd.u + 6 * lo;
    const double* uhi = a.bd.u + 6 * hi;
    const double* dlo = a.ws.du + 6 * lo;
    const double* dhi = a.ws.du + 6 * hi;
    for (int row = 0; row < 5; ++row) {
        const double* Jr = J + 12 * row;
        const double* Wr = W + 12 * row;
        a.ws.hb[5 * (size_t)k + row] = (jrow_dot(Jr, ulo, uhi) + jrow_dot(Jr, dlo, dhi)) + g[row];
        double prods[12];
        int m = 0;
        for (int c = 0; c < 12; ++c) {
            if (!hasw[c / 6]) continue;
            const double prod = Jr[c] * Wr[c];
            if (prod != 0.0) prods[m++] = prod;
        }
        const double d = np_reduce_sum(prods, m);
        const double diag = d == 0.0 ? 1.0 : d;
        a.ws.hdiag[5 * (size_t)k + row] = diag;
        a.ws.hr[5 * (size_t)k + row] = 1.0 / diag;
        a.ws.hx[5 * (size_t)k + row] = 0.0;
        a.ws.hsol[5 * (size_t)k + row] = 0.0;
    }
}

// w = W J^T x of the hinge problem for every body of the scene (hinges ascending, 5 rows each)
template <class G>
__device__ void hinge_wjt(const StepArgs& a, const G& g, const SceneRange& R) {
    for (int b = R.b0 + g.rank(); b < R.b1; b += g.size()) {
        double s6[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (!a.bd.fixed[b])
            for (int e = a.ws.hbody_ptr[b]; e < a.ws.hbody_ptr[b + 1]; ++e) {
                const int code = a.ws.hbody_list[e];
                const int k = code >> 1, side = code & 1;
                const double* Wk = a.ws.hWJT + 60 * (size_t)k + 6 * side;
                for (int d = 0; d < 6; ++d) {
                    double t = s6[d];
                    for (int row = 0; row < 5; ++row) t += Wk[12 * row + d] * a.ws.hx[5 * (size_t)k + row];
                    s6[d] = t;
                }
            }
        for (int d = 0; d < 6; ++d) a.ws.hw[6 * (size_t)b + d] = s6[d];
    }
    g.sync();
}

// hinges.py:62-90: x_b -= r_b (J w + b)_b from the w before this hinge, then w += WJT[:, b] dx
__device__ __forceinline__ void hinge_update(const StepArgs& a, int k) {
    const int lo = a.ws.hlohi[2 * k], hi = a.ws.hlohi[2 * k + 1];
    const double* J = a.ws.hJ + 60 * (size_t)k;
    double* wlo = a.ws.hw + 6 * (size_t)lo;
    double* whi = a.ws.hw + 6 * (size_t)hi;
    double jw[5], delta[5];
    for (int row = 0; row < 5; ++row) jw[row] = jrow_dot(J + 12 * row, wlo, whi);
    for (int row = 0; row < 5; ++row) {
        const size_t i = 5 * (size_t)k + row;
        const double xo = a.ws.hx[i];
        const double xn = xo - a.ws.hr[i] * (jw[row] + a.ws.hb[i]);
        a.ws.hx[i] = xn;
        delta[row] = xn - xo;
    }
    for (int side = 0; side < 2; ++side) {
        const int bd = side ? hi : lo;
        if (a.bd.fixed[bd]) continue;
        double* wb = side ? whi : wlo;
        const double* Ws = a.ws.hWJT + 60 * (size_t)k + 6 * side;
        for (int d = 0; d < 6; ++d) {
            double t = 0.0;
            for (int row = 0; row < 5; ++row) t += Ws[12 * row + d] * delta[row];
            wb[d] = wb[d] + t;
        }
    }
}

// levels of the scene's hinges in their serial order (a hinge follows the earlier hinges on its non-fixed
// bodies), by one thread: hlev_order[h0 ..] lists the hinges level by level, ascending inside a level, and
// hlev_ptr[h0 + s + l - 1] .. hlev_ptr[h0 + s + l] index the hinges of level l.  Returns the number of levels.
template <class G>
__device__ int hinge_levels(const StepArgs& a, const G& g, const SceneRange& R, int s, int h0, int h1) {
    int L = 0;
    if (g.rank() == 0) {
        int32_t* last = a.ws.hlast;
        for (int b = R.b0; b < R.b1; ++b) last[b] = 0;
        int32_t* lev = a.ws.hlev;
        for (int k = h0; k < h1; ++k) {
            const int lo = a.ws.hlohi[2 * k], hi = a.ws.hlohi[2 * k + 1];
            const int l0 = a.bd.fixed[lo] ? 0 : last[lo], l1 = a.bd.fixed[hi] ? 0 : last[hi];
            const int l = 1 + max(l0, l1);
            if (!a.bd.fixed[lo]) last[lo] = l;
            if (!a.bd.fixed[hi]) last[hi] = l;
            lev[k] = l;
            L = max(L, l);
        }
        int32_t* ptr = a.ws.hlev_ptr + h0 + s;
        for (int l = 0; l <= L; ++l) ptr[l] = 0;
        for (int k = h0; k < h1; ++k) ptr[lev[k]]++;
        for (int l = 1; l <= L; ++l) ptr[l] += ptr[l - 1];          // ptr[l] = end of level l
        for (int l = L; l >= 1; --l) ptr[l] = ptr[l - 1];          // ptr[l] = start of level l, used as
        ptr[0] = 0;                                                  // the level's cursor: after the fill
        for (int k = h0; k < h1; ++k) a.ws.hlev_order[h0 + ptr[lev[k]]++] = k;   // it is the level's end
    }
    g.sync();
    return g.imax(L);
}

// The reference stepper's Gauss-Seidel loop over [contacts (when any), hinges] (gauss_seidel_solver.py:14-101):
// every iteration sweeps each problem in turn (each with its own accumulators w, built from its own x at the
// start of its sweep), accepts or rolls back its iterate against that problem's own last merit and adapts its
// r-factors; the convergence tests use the largest merit of the iteration.  FP64, serial order, merit rule.
template <class G>
__device__ void solve_scene_hinges(const StepArgs& a, const G& g, int s, double* w_smem, int smem_bodies) {
    const int max_it = a.pr.max_iterations;
    double* x = a.ws.x;
    double* sol = a.out.contact_sol;
    const double* b = a.ws.b;
    double* r = a.ws.r;
    const SceneRange R = scene_range(a, s);
    const int K = R.c1 - R.c0, nb = R.b1 - R.b0;
    const int h0 = a.bd.scene_hinge_start[s], h1 = a.bd.scene_hinge_start[s + 1];
    rb_scene_stats* st = a.out.stats + s;
    double* hist = (a.out.residuals && a.pr.profiling) ? a.out.residuals + (size_t)s * a.caps.max_iterations : nullptr;
    if (g.rank() == 0) {
        st->n_contacts = K; st->contact_start = R.c0; st->iterations = -1; st->exitcode = -1;
        st->merit = 0.0; st->residual = 0.0; st->post_iterations = -1; st->post_exitcode = -1;
        st->n_levels = 0; st->fp32_sweeps = 0;
    }
    if (hist) for (int i = g.rank(); i < max_it; i += g.size()) hist[i] = INFINITY;
    const bool on_chip = w_smem != nullptr && nb <= smem_bodies;
    const WView w = {on_chip ? w_smem : a.ws.w + 6 * R.b0, R.b0};
    const int L = K > 0 ? scene_levels(a, g, R, s) : 0;
    const int HL = hinge_levels(a, g, R, s, h0, h1);
    if (g.rank() == 0) st->n_levels = L;
    const int* hptr = a.ws.hlev_ptr + h0 + s;
    double last_c = INFINITY, last_h = INFINITY, global_last = INFINITY, shown = 0.0;
    int iterations = max_it, exitcode = 0;
    for (int it = 0; it < max_it; ++it) {
        double gm = 0.0;
        if (K > 0) {   // Contacts.sweep, then the accept / roll-back rule
            scene_wjt(a, g, R, x, w);
            gs_sweep_levels(a, g, R, s, L, b, r, x, w, false);
            double m = 0.0;
            for (int i = 4 * R.c0 + g.rank(); i < 4 * R.c1; i += g.size()) m = nanmax(m, fabs(x[i] - sol[i]));
            const double merit = g.max(m);
            const bool reject = merit > last_c;
            const bool inc = !reject && last_c - merit < a.pr.too_small_merit_change;
            for (int i = 4 * R.c0 + g.rank(); i < 4 * R.c1; i += g.size()) {
                if (reject) { r[i] = a.pr.nu_reduce * r[i]; x[i] = sol[i]; }
                else { sol[i] = x[i]; if (inc) r[i] = a.pr.nu_increase * r[i]; }
            }
            if (reject) gm = gm > last_c ? gm : last_c;
            else { last_c = merit; gm = gm > merit ? gm : merit; }
            g.sync();
        }
        {              // Hinges.sweep, then the same rule with the hinge problem's own merit and r-factors
            hinge_wjt(a, g, R);
            for (int l = 1; l <= HL; ++l) {
                for (int i = hptr[l - 1] + g.rank(); i < hptr[l]; i += g.size()) hinge_update(a, a.ws.hlev_order[h0 + i]);
                g.sync();
            }
            double m = 0.0;
            for (int i = 5 * h0 + g.rank(); i < 5 * h1; i += g.size()) m = nanmax(m, fabs(a.ws.hx[i] - a.ws.hsol[i]));
            const double merit = g.max(m);
            const bool reject = merit > last_h;
            const bool inc = !reject && last_h - merit < a.pr.too_small_merit_change;
            for (int i = 5 * h0 + g.rank(); i < 5 * h1; i += g.size()) {
                if (reject) { a.ws.hr[i] = a.pr.nu_reduce * a.ws.hr[i]; a.ws.hx[i] = a.ws.hsol[i]; }
                else { a.ws.hsol[i] = a.ws.hx[i]; if (inc) a.ws.hr[i] = a.pr.nu_increase * a.ws.hr[i]; }
            }
            if (reject) gm = gm > last_h ? gm : last_h;
            else { last_h = merit; gm = gm > merit ? gm : merit; }
            g.sync();
        }
        if (hist && g.rank() == 0) hist[it] = gm;
        shown = gm;
        bool stop = false;
        if (gm < a.pr.absolute_tolerance) { stop = true; exitcode = 1; }
        else if (fabs(gm - global_last) < a.pr.relative_tolerance * global_last) { stop = true; exitcode = 2; }
        global_last = gm;
        if (stop) { iterations = it; break; }
    }
    if (a.out.hinge_sol)
        for (int i = 5 * h0 + g.rank(); i < 5 * h1; i += g.size()) a.out.hinge_sol[i] = a.ws.hsol[i];
    if (g.rank() == 0) { st->iterations = iterations; st->exitcode = exitcode; st->merit = shown; }
    g.sync();
}

// device clock in microseconds (the global nanosecond timer)
__device__ __forceinline__ double device_us() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return 1e-3 * (double)t;
}

template <class G>
__device__ void solve_scene_body(const StepArgs& a, const G& g, int s, int post, double* w_smem, int smem_bodies);

// The proximal solve of one scene (gauss_seidel_solver.py:14 / solver_interface.py:123); with profiling on,
// its device time goes to the scene's statistics (added to the FP32 phase's time when one ran).
template <class G>
__device__ void solve_scene(const StepArgs& a, const G& g, int s, int post, double* w_smem, int smem_bodies) {
    if (!post && a.ws.fin32[s]) return;   // finished by the FP32 phase
    const bool timed = !post && a.pr.profiling;
    const double t0 = timed ? device_us() : 0.0;
    solve_scene_body(a, g, s, post, w_smem, smem_bodies);
    if (!post && g.rank() == 0) {
        rb_scene_stats* st = a.out.stats + s;
        const bool fp32_phase = a.pr.precision != RB_PRECISION_FP64 && a.ws.sweeps32[s] >= 0;
        if (!timed) { st->solve_start_us = 0.0; st->solve_us = 0.0; }
        else if (fp32_phase) st->solve_us += device_us() - t0;
        else { st->solve_start_us = t0; st->solve_us = device_us() - t0; }
    }
}

template <class G>
__device__ void solve_scene_body(const StepArgs& a, const G& g, int s, int post, double* w_smem, int smem_bodies) {
    if (!post && a.bd.n_hinges > 0 && a.bd.scene_hinge_start[s + 1] > a.bd.scene_hinge_start[s]) {
        solve_scene_hinges(a, g, s, w_smem, smem_bodies);
        return;
    }
    const int scheme = post ? RB_SCHEME_RIGID_GS : a.pr.scheme;
    const bool rigid = scheme == RB_SCHEME_RIGID_GS;
    const bool jacobi = scheme == RB_SCHEME_JACOBI || scheme == RB_SCHEME_JACOBI_HYBRID;
    const int max_it = a.pr.max_iterations;
    double* x = a.ws.x;
    double* sol = post ? a.ws.xold : a.out.contact_sol;
    const double* b = a.ws.b;
    double* r = a.ws.r;
    const SceneRange R = scene_range(a, s);
    const int K = R.c1 - R.c0;
    const int nb = R.b1 - R.b0;
    rb_scene_stats* st = a.out.stats + s;
    double* hist = (!post && a.out.residuals && a.pr.profiling) ? a.out.residuals + (size_t)s * a.caps.max_iterations
                                                                : nullptr;
    if (g.rank() == 0) {
        if (!post) {
            st->n_contacts = K; st->contact_start = R.c0; st->iterations = -1; st->exitcode = -1;
            st->merit = 0.0; st->residual = 0.0; st->post_iterations = -1; st->post_exitcode = -1;
            st->n_levels = 0; st->fp32_sweeps = 0;
        } else {
            st->post_iterations = -1; st->post_exitcode = -1;
        }
    }
    if (hist) for (int i = g.rank(); i < max_it; i += g.size()) hist[i] = INFINITY;
    if (K == 0) { g.sync(); return; }
    if (post) {   // steppers.py:32: no solve when no contact is deeper than min_gap
        bool any = false;
        for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) any |= (b[4 * k] != 0.0);
        if (!g.any(any)) return;
    }
    const bool on_chip = w_smem != nullptr && nb <= smem_bodies;
    const WView w = {on_chip ? w_smem : a.ws.w + 6 * R.b0, R.b0};
    const bool coloured = !post && !jacobi &&
                          (scheme == RB_SCHEME_COLOURED_GS || a.pr.ordering == RB_ORDER_COLOURED);
    // FP32 modes: the scene's FP32 phase left its iterate in x and its level order in lev_order / lev_ptr
    const int sweeps32 = (!post && a.pr.precision != RB_PRECISION_FP64) ? a.ws.sweeps32[s] : -1;
    const int L = jacobi ? 0 : sweeps32 >= 0 ? a.ws.nlev[s]
                : (coloured ? scene_colours(a, g, R, s) : scene_levels(a, g, R, s));
    if (!post && g.rank() == 0) st->n_levels = L;
    const bool by_residual = !post && a.pr.termination != RB_TERMINATE_MERIT;
    const bool fixed_r = !post && a.pr.termination == RB_TERMINATE_RESIDUAL_FIXED_R;
    const int interval = a.pr.residual_interval > 1 ? a.pr.residual_interval : 1;
    double last = INFINITY, global_last = INFINITY, shown = 0.0;
    int iterations = max_it, exitcode = 0;
    bool w_is_wjt_x = false;   // w already holds WJT x for the current x (left by the residual pass)
    // FP32 modes: test the FP32 iterate in FP64, then refine it in FP64 with the sweeps left
    int loop_max = max_it;
    if (sweeps32 >= 0) {
        const double res0 = scene_residual(a, g, R, x, w);
        w_is_wjt_x = true;
        shown = res0;
        if (g.rank() == 0) st->fp32_sweeps = sweeps32;
        if (res0 <= a.pr.residual_tolerance || a.pr.precision == RB_PRECISION_FP32 || sweeps32 >= max_it) {
            for (int i = 4 * R.c0 + g.rank(); i < 4 * R.c1; i += g.size()) sol[i] = x[i];
            g.sync();
            const bool ok = res0 <= a.pr.residual_tolerance;
            if (g.rank() == 0) {
                st->iterations = ok ? max(sweeps32 - 1, 0) : max_it;
                st->exitcode = ok ? 3 : 0;
                st->merit = res0;
                st->residual = res0;
            }
            g.sync();
            return;
        }
        loop_max = max_it - sweeps32;   // the sweeps the FP32 phase left over
    }
    for (int it = 0; it < loop_max; ++it) {
        if (!w_is_wjt_x) scene_wjt(a, g, R, x, w);   // every sweep starts from w = WJT x (contacts.py:72)
        if (jacobi) {               // proximal_contact/jacobi_solver.py:41-79
            const bool hybrid = scheme == RB_SCHEME_JACOBI_HYBRID;
            for (int k = R.c0 + g.rank(); k < R.c1; k += g.size()) {
                const int lo = a.ws.lohi[2 * k], hi = a.ws.lohi[2 * k + 1];
                const double* J = a.ws.J + 48 * (size_t)k;
                double z[4];
                for (int row = 0; row < 4; ++row)
                    z[row] = x[4 * k + row] - r[4 * k + row] * (jrow_dot(J + 12 * row, w.at(lo), w.at(hi)) + b[4 * k + row]);
                const double xn = z[0] > 0.0 ? z[0] : 0.0;
                double f[3];
                prox_sphere(z[1], z[2], z[3], a.ws.mu[k], hybrid ? xn : x[4 * k], f);
                x[4 * k] = xn; x[4 * k + 1] = f[0]; x[4 * k + 2] = f[1]; x[4 * k + 3] = f[2];
            }
            g.sync();
        } else {
            gs_sweep_levels(a, g, R, s, L, b, r, x, w, post != 0);
        }
        // merit = ||x - sol||_inf (problem.py:53); the fixed-r rule never looks at it
        double merit = 0.0;
        if (!fixed_r) {
            double m = 0.0;
            for (int i = 4 * R.c0 + g.rank(); i < 4 * R.c1; i += g.size()) m = nanmax(m, fabs(x[i] - sol[i]));
            merit = g.max(m);
        }
        const bool check = by_residual && (!fixed_r || (it + 1) % interval == 0 || it + 1 == loop_max);
        const double res = check ? scene_residual(a, g, R, x, w) : 0.0;
        int decision = 0;   // 0 accept, 1 reject, 2 keep sol, 3 take x
        bool stop = false, inc = false;
        if (rigid) {        // gauss_seidel_solver.py:439-482
            double gm;
            if (merit > last) { decision = 1; gm = last > 0.0 ? last : 0.0; }
            else {
                inc = last - merit < a.pr.too_small_merit_change;
                last = merit;
                gm = merit > 0.0 ? merit : 0.0;
            }
            if (gm < a.pr.absolute_tolerance) { stop = true; exitcode = 1; }
            else if (fabs(gm - global_last) < a.pr.relative_tolerance * global_last) { stop = true; exitcode = 2; }
            global_last = gm;
            shown = gm;
        } else {            // solver_interface.py:88-113 then :50-69
            if (merit < a.pr.absolute_tolerance) { stop = true; exitcode = 1; }
            else if (fabs(merit - last) < a.pr.relative_tolerance * last) { stop = true; exitcode = 2; }
            if (!stop) {
                if (merit > last) decision = 1;
                else { inc = last - merit < a.pr.too_small_merit_change; last = merit; }
            } else decision = 2;
            shown = merit;
        }
        if (by_residual && !check) {   // fixed r between residual tests: accept the sweep
            stop = false; exitcode = 0; decision = 0; inc = false;
        } else if (by_residual) {      // stop only on the complementarity residual
            shown = res;
            if (res <= a.pr.residual_tolerance) { stop = true; exitcode = 3; decision = 3; }
            else if (fixed_r) { stop = false; exitcode = 0; decision = 0; inc = false; }
            else {
                stop = false;
                exitcode = 0;
                if (decision == 2) {   // a merit test would have stopped: apply the accept/reject rule
                    if (merit > last) decision = 1;
                    else { inc = last - merit < a.pr.too_small_merit_change; last = merit; decision = 0; }
                }
            }
        }
        if (hist && g.rank() == 0) hist[it] = shown;
        if (decision == 1) {
            for (int i = 4 * R.c0 + g.rank(); i < 4 * R.c1; i += g.size()) {
                r[i] = a.pr.nu_reduce * r[i];
                x[i] = sol[i];
            }
        } else if (decision == 0) {
            for (int i = 4 * R.c0 + g.rank(); i < 4 * R.c1; i += g.size()) {
                sol[i] = x[i];
                if (inc) r[i] = a.pr.nu_increase * r[i];
            }
        } else if (decision == 3) {   // converged by residual: the current iterate is the solution
            for (int i = 4 * R.c0 + g.rank(); i < 4 * R.c1; i += g.size()) sol[i] = x[i];
        }
        // the residual pass computed w = WJT x; unless x was rolled back that is the next sweep's start
        w_is_wjt_x = check && decision != 1;
        g.sync();
        if (stop) { iterations = it; break; }
    }
    if (sweeps32 >= 0) iterations = exitcode == 3 ? sweeps32 + iterations : max_it;
    if (by_residual && exitcode != 3) shown = scene_residual(a, g, R, sol, w);   // residual of what is returned
    if (g.rank() == 0) {
        if (!post) {
            st->iterations = iterations; st->exitcode = exitcode; st->merit = shown;
            if (by_residual) st->residual = shown;
        } else {
            st->post_iterations = iterations; st->post_exitcode = exitcode;
        }
    }
    g.sync();
}

// ---------------------------------------------------------------------------------------------------------
// FP32 phase of the FP32 precision modes.  A scene's whole contact problem is copied into shared memory as
// FP32 in a compact form and swept there, level by level (or colour by colour), with the fixed-r rule until
// the FP32 residual meets the tolerance, stalls near FP32 rounding, or the sweep budget is spent; the iterate
// is then tested in FP64 and, if it misses the tolerance, refined by the same team with FP64 sweeps (the
// budget left).
//
// Compact form.  A contact's Jacobian rows are [lin_lo | ang_lo | lin_hi | ang_hi] with lin_hi = -lin_lo
// (the frame direction, zero on the torsion row) and W J^T = (m^-1 lin, I_w^-1 ang) per body, so a contact
// stores per row q: lin_lo (3), ang_lo (3), ang_hi (3), b, 1/diag and x -- 12 floats, 48 per contact (the
// torsion row's unused lin slot holds mu), in a record of kS32Floats -- and a body stores its accumulator
// w (6), m^-1, a fixed flag and the world inverse inertia (6, symmetric), in a record of kS32BodyFloats
// (m^-1 = I^-1 = 0 for a fixed body).  The update of w after a contact changes by dx is m^-1 sum_q lin_q dx_q
// (negated on the hi side) and I^-1 sum_q ang_q dx_q.
//
// Execution.  A team -- one warp for scenes of up to the mid slab, a 128-thread block above, a 512-thread
// block for the scenes whose rows stay in L2 -- takes scenes from its size class's queue; the slab scenes are
// swept one lane per contact (s32_sweep_lane, by warp 0 in a block team), the L2 scenes four lanes per
// contact (s32_sweep).  The four classes' launches run concurrently on separate streams.
// ---------------------------------------------------------------------------------------------------------
constexpr int kQueueFp32 = 5;                        // counters[5..8]: scene queues of the four size classes
constexpr int kClassEnd32 = 9;                       // counters[9..12]: end of each class's range in list32
constexpr int kFp32Block = 128;                      // threads per block of the FP32 launches
constexpr int kFp32BlockMax = 256;                   // ... at most, in the launches for slab scenes
constexpr int kFp32L2Block = 512;                    // threads of the launch for the scenes beyond any slab
constexpr int kFp32LargeSmem = 224 * 1024;           // slab of a block team (one scene per SM)
constexpr int kS32SmallSlab = 28 * 1024;             // slab of a warp team, small class (8 scenes per SM)
constexpr int kS32MidSlab = 56 * 1024;               // slab of a warp team, mid class (4 scenes per SM)
// relative residual below which a stalled FP32 iteration may have met FP32 rounding
constexpr float kFp32Floor = 1e-5f;
// residual tests without a 5 % improvement after which an FP32 round ends in a defect correction (with the
// test every 4 sweeps: 64 sweeps; Gauss-Seidel often progresses by less than 5 % in 12 sweeps near 1e-6).
// A round that did not lower the FP64 residual by kS32RoundGain doubles the next round's window (up to
// kS32StallTestsMax): a scene whose Gauss-Seidel iteration itself has stalled keeps sweeping in FP32 with
// rare corrections, as FP64 sweeps would stall on it just the same
constexpr float kS32FarFactor = 100.0f;   // residual / tolerance above which tests are spaced twice as far
constexpr int kS32StallTests = 16;
constexpr int kS32StallTestsMax = 512;
constexpr double kS32RoundGain = 0.9;

struct S32Scene {
    float* c;          // kS32Floats per contact, in level order; row q at 12 q as three float4 groups
                       // (lin[3], b | ang_lo[3], 1/diag | ang_hi[3], x); the torsion row's lin is (mu, 0, 0)
    float* body;       // kS32BodyFloats per body: w[6], m^-1, fixed, I^-1 (xx, xy, xz, yy, yz, zz), padding
    uint32_t* lohi;    // per contact in level order: scene-local lo | hi << 16
    uint16_t* pos;     // level-order position of each contact (scene-local contact index -> position)
    uint16_t* lptr;    // level starts (L + 1)
    uint16_t* bptr;    // per body: start of its contact list in blist (nb + 1)
    uint32_t* blist;   // per body, its contacts in ascending order: level-order position << 1 | side (2K)
};
__host__ __device__ inline size_t s32_align(size_t v) { return (v + 15) & ~size_t(15); }
// shared memory of a scene's FP32 copy; with in_l2 the contact rows, the level-order positions and the
// per-body contact lists live in global memory (L2) and only the bodies, body indices and level and list
// starts stay on chip
__host__ __device__ inline size_t s32_bytes(int K, int nb, bool in_l2 = false, bool bodies_global = false) {
    return (in_l2 ? 0 : s32_align(sizeof(float) * (size_t)K * kS32Floats) + s32_align(sizeof(uint16_t) * (size_t)K) +
                        s32_align(sizeof(uint32_t) * 2 * (size_t)K)) +
           (bodies_global ? 0 : s32_align(sizeof(float) * (size_t)nb * kS32BodyFloats)) +
           s32_align(sizeof(uint32_t) * (size_t)K) +
           s32_align(sizeof(uint16_t) * (size_t)(K + 1)) + s32_align(sizeof(uint16_t) * (size_t)(nb + 1));
}
// with l2, the contact rows, positions and body lists go to the workspace; with bodies_global the body
// records too (the scene's team is the only reader and writer, so block barriers keep them consistent)
__device__ __forceinline__ S32Scene s32_carve(char* base, int K, int nb, const StepArgs* l2 = nullptr, int c0 = 0,
                                              bool bodies_global = false, int b0 = 0) {
    S32Scene f;
    size_t o = 0;
    auto take = [&](size_t bytes) { char* p = base + o; o += s32_align(bytes); return p; };
    f.c = l2 ? l2->ws.c32 + kS32Floats * (size_t)c0 : (float*)take(sizeof(float) * (size_t)K * kS32Floats);
    f.body = (l2 && bodies_global) ? l2->ws.body32 + kS32BodyFloats * (size_t)b0
                                   : (float*)take(sizeof(float) * (size_t)nb * kS32BodyFloats);
    f.lohi = (uint32_t*)take(sizeof(uint32_t) * (size_t)K);
    f.pos = l2 ? l2->ws.pos32 + c0 : (uint16_t*)take(sizeof(uint16_t) * (size_t)K);
    f.lptr = (uint16_t*)take(sizeof(uint16_t) * (size_t)(K + 1));
    f.bptr = (uint16_t*)take(sizeof(uint16_t) * (size_t)(nb + 1));
    f.blist = l2 ? l2->ws.blist32 + 2 * (size_t)c0 : (uint32_t*)take(sizeof(uint32_t) * 2 * (size_t)K);
    return f;
}

__device__ __forceinline__ void f32_prox(float zs, float zt, float ztau, float mu, float xn, float* o) {
    if (xn <= 0.0f) { o[0] = 0.0f; o[1] = 0.0f; o[2] = 0.0f; return; }
    const float radius = mu * xn;
    const float sqr = fmaf(zs, zs, fmaf(zt, zt, ztau * ztau));
    if (sqr <= radius * radius) { o[0] = zs; o[1] = zt; o[2] = ztau; return; }
    const float scale = radius * rsqrtf(sqr);
    o[0] = zs * scale; o[1] = zt * scale; o[2] = ztau * scale;
}

// y = I^-1 t with I^-1 stored symmetric (xx, xy, xz, yy, yz, zz)
__device__ __forceinline__ void s32_sym3(const float* I, const float* t, float* y) {
    y[0] = fmaf(I[0], t[0], fmaf(I[1], t[1], I[2] * t[2]));
    y[1] = fmaf(I[1], t[0], fmaf(I[3], t[1], I[4] * t[2]));
    y[2] = fmaf(I[2], t[0], fmaf(I[4], t[1], I[5] * t[2]));
}

// J_q . [w_lo; w_hi] of row q (the torsion row has no linear part): three partial sums, then their total
__device__ __forceinline__ float s32_jw(const float* row, int q, const float* wl, const float* wh) {
    float lin = 0.0f;
    if (q < 3) lin = fmaf(row[0], wl[0] - wh[0], fmaf(row[1], wl[1] - wh[1], row[2] * (wl[2] - wh[2])));
    const float alo = fmaf(row[4], wl[3], fmaf(row[5], wl[4], row[6] * wl[5]));
    const float ahi = fmaf(row[8], wh[3], fmaf(row[9], wh[4], row[10] * wh[5]));
    return (lin + alo) + ahi;
}

// copy scene R into the team's slab as FP32, contacts in level order; returns the number of levels
template <class G>
__device__ __forceinline__ int s32_load(const StepArgs& a, const G& g, const SceneRange& R, int s, const S32Scene& f,
                                        bool coloured, int16_t* scratch) {
    const int K = R.c1 - R.c0, nb = R.b1 - R.b0;
    // levels by relaxation in shared memory when a scratch is given (the rows' room, not yet filled)
    const int L = coloured ? scene_colours(a, g, R, s)
                : scratch ? scene_levels_smem(a, g, R, s, scratch) : scene_levels(a, g, R, s);
    const int* order = a.ws.lev_order + R.c0;
    for (int t = g.rank(); t < 16 * K; t += g.size()) {   // (position, row, float4 group; part 3 idle)
        const int i = t >> 4, q = (t >> 2) & 3, part = t & 3;
        const size_t k = (size_t)order[i];
        float* row = f.c + kS32Floats * i + 12 * q;
        const double* J = a.ws.J + 48 * k + 12 * q;
        if (part == 0) {
            row[0] = q < 3 ? (float)J[0] : (float)a.ws.mu[k];
            row[1] = q < 3 ? (float)J[1] : 0.0f;
            row[2] = q < 3 ? (float)J[2] : 0.0f;
            row[3] = (float)a.ws.b[4 * k + q];
        } else if (part == 1) {
            row[4] = (float)J[3]; row[5] = (float)J[4]; row[6] = (float)J[5];
            row[7] = (float)(1.0 / a.ws.diag[4 * k + q]);
        } else if (part == 2) {
            row[8] = (float)J[9]; row[9] = (float)J[10]; row[10] = (float)J[11];
            row[11] = (float)a.ws.x[4 * k + q];
        }
    }
    for (int i = g.rank(); i < K; i += g.size()) {
        const int k = order[i];
        f.pos[k - R.c0] = (uint16_t)i;
        f.lohi[i] = (uint32_t)(a.ws.lohi[2 * k] - R.b0) | ((uint32_t)(a.ws.lohi[2 * k + 1] - R.b0) << 16);
    }
    for (int l = g.rank(); l <= L; l += g.size()) f.lptr[l] = (uint16_t)a.ws.lev_ptr[R.c0 + s + l];
    g.sync();   // pos complete
    // per-body contact lists (the residual's w = W J^T x), positions in level order
    const int e0 = a.ws.bc_ptr[R.b0];
    for (int bl = g.rank(); bl <= nb; bl += g.size()) f.bptr[bl] = (uint16_t)(a.ws.bc_ptr[R.b0 + bl] - e0);
    for (int e = g.rank(); e < a.ws.bc_ptr[R.b1] - e0; e += g.size()) {
        const int code = a.ws.bc_list[e0 + e];
        f.blist[e] = ((uint32_t)f.pos[(code >> 1) - R.c0] << 1) | (uint32_t)(code & 1);
    }
    for (int bl = g.rank(); bl < nb; bl += g.size()) {
        const int b = R.b0 + bl;
        float* B = f.body + kS32BodyFloats * bl;
        const bool fx = a.bd.fixed[b] != 0;
        const double* Wi = a.ws.Winv + 9 * (size_t)b;
        B[6] = fx ? 0.0f : (float)(1.0 / a.bd.mass[b]);
        B[7] = fx ? 1.0f : 0.0f;
        // a fixed body's update is zero (m^-1 = I^-1 = 0); the sweeps still only store to free bodies
        B[8] = fx ? 0.0f : (float)Wi[0]; B[9] = fx ? 0.0f : (float)Wi[1]; B[10] = fx ? 0.0f : (float)Wi[2];
        B[11] = fx ? 0.0f : (float)Wi[4]; B[12] = fx ? 0.0f : (float)Wi[5]; B[13] = fx ? 0.0f : (float)Wi[8];
    }
    g.sync();
    return L;
}

// w = W J^T x (each body sums its contacts in ascending order)
template <class G>
__device__ __forceinline__ void s32_rebuild_w(const G& g, const SceneRange& R, const S32Scene& f) {
    const int nb = R.b1 - R.b0;
    for (int bl = g.rank(); bl < nb; bl += g.size()) {
        float* B = f.body + kS32BodyFloats * bl;
        float P[3] = {0.f, 0.f, 0.f}, T[3] = {0.f, 0.f, 0.f};
        if (B[7] == 0.0f) {   // rows read as float4 groups (lin, b | ang_lo, 1/diag | ang_hi, x)
            for (int e = f.bptr[bl]; e < f.bptr[bl + 1]; ++e) {
                const uint32_t code = f.blist[e];
                const int side = code & 1;
                const float4* C4 = reinterpret_cast<const float4*>(f.c + kS32Floats * (code >> 1));
                for (int q = 0; q < 4; ++q) {
                    const float4 lin = C4[3 * q], alo = C4[3 * q + 1], ahi = C4[3 * q + 2];
                    const float xq = ahi.w;
                    if (q < 3) {
                        const float sx = side ? -xq : xq;
                        P[0] = fmaf(lin.x, sx, P[0]); P[1] = fmaf(lin.y, sx, P[1]); P[2] = fmaf(lin.z, sx, P[2]);
                    }
                    const float4 ang = side ? ahi : alo;
                    T[0] = fmaf(ang.x, xq, T[0]); T[1] = fmaf(ang.y, xq, T[1]); T[2] = fmaf(ang.z, xq, T[2]);
                }
            }
        }
        float om[3];
        s32_sym3(B + 8, T, om);
        B[0] = B[6] * P[0]; B[1] = B[6] * P[1]; B[2] = B[6] * P[2];
        B[3] = om[0]; B[4] = om[1]; B[5] = om[2];
    }
    g.sync();
}

// w = W J^T x, then the FP32 residual ||x - prox(x - D^-1 (A x + b))||_inf / max(1, ||x||_inf)
template <class G>
__device__ __forceinline__ float s32_residual(const StepArgs& a, const G& g, const SceneRange& R, const S32Scene& f) {
    const int K = R.c1 - R.c0;
    s32_rebuild_w(g, R, f);
    float m = 0.0f, xm = 0.0f;
    for (int i = g.rank(); i < K; i += g.size()) {
        const float4* C4 = reinterpret_cast<const float4*>(f.c + kS32Floats * i);
        const uint32_t lh = f.lohi[i];
        const float* Bl = f.body + kS32BodyFloats * (int)(lh & 0xffffu);
        const float* Bh = f.body + kS32BodyFloats * (int)(lh >> 16);
        const float4 l0 = *reinterpret_cast<const float4*>(Bl), l1 = *reinterpret_cast<const float4*>(Bl + 4);
        const float4 h0 = *reinterpret_cast<const float4*>(Bh), h1 = *reinterpret_cast<const float4*>(Bh + 4);
        float z[4], x[4];
        float mu = 0.0f;
        for (int q = 0; q < 4; ++q) {   // the expressions of s32_jw, on float4 loads
            const float4 r0 = C4[3 * q], r1 = C4[3 * q + 1], r2 = C4[3 * q + 2];
            float lin = 0.0f;
            if (q < 3) lin = fmaf(r0.x, l0.x - h0.x, fmaf(r0.y, l0.y - h0.y, r0.z * (l0.z - h0.z)));
            else mu = r0.x;
            const float alo = fmaf(r1.x, l0.w, fmaf(r1.y, l1.x, r1.z * l1.y));
            const float ahi = fmaf(r2.x, h0.w, fmaf(r2.y, h1.x, r2.z * h1.y));
            x[q] = r2.w;
            z[q] = x[q] - r1.w * (((lin + alo) + ahi) + r0.w);
        }
        const float pn = fmaxf(z[0], 0.0f);
        float fr[3];
        f32_prox(z[1], z[2], z[3], mu, pn, fr);
        const float d[4] = {x[0] - pn, x[1] - fr[0], x[2] - fr[1], x[3] - fr[2]};
        for (int t = 0; t < 4; ++t) {
            m = fmaxf(m, fabsf(d[t]));
            if (d[t] != d[t]) m = d[t];
            xm = fmaxf(xm, fabsf(x[t]));
        }
    }
    const double mres = g.max((double)m);
    const double mx = g.max((double)xm);
    return (float)(mres / (mx > 1.0 ? mx : 1.0));
}

// One Gauss-Seidel sweep over the levels, four lanes per contact.  Lane q computes row q of J w; the z of
// the four rows meet by shuffles and every lane applies the prox; lane q then forms one 3-vector of the
// update from the four rows' float4 group it owns (lin for q = 0, 1; ang_lo for 2; ang_hi for 3) and applies
// +m^-1, -m^-1, I_lo^-1 or I_hi^-1 to it.  Every lane runs the same instructions (lane-dependent offsets);
// all shared-memory reads are float4 / float2.
template <class G, bool kL2>
__device__ __forceinline__ void s32_sweep(const G& g, const S32Scene& f, int L, float rscale, bool bodies_global) {
    const int q = g.rank() & 3, slot = g.rank() >> 2, nslot = g.size() >> 2;
    const int base = (threadIdx.x & 31) & ~3;
    const unsigned qm = 0xfu << base;
    const int grp = q < 2 ? 0 : q - 1;          // the float4 group of the update columns this lane sums
    const bool on_hi = (q & 1) != 0;            // lanes 1 and 3 update the hi body
    const bool linear = q < 2;
    int start = f.lptr[0], end = f.lptr[1];
    for (int l = 1; l <= L; ++l) {
        const int next_end = l < L ? f.lptr[l + 1] : end;
        if (kL2) {   // rows in L2: pull the next level's rows (contiguous in level order) into L1 meanwhile
            const char* p0 = reinterpret_cast<const char*>(f.c + kS32Floats * (size_t)end);
            const int lines = (int)(((size_t)(next_end - end) * kS32Floats * sizeof(float) + 127) / 128);
            for (int t = g.rank(); t < lines; t += g.size())
                asm volatile("prefetch.global.L1 [%0];" ::"l"(p0 + 128 * (size_t)t));
            if (bodies_global)   // and the body records those rows touch
                for (int i = end + g.rank(); i < next_end; i += g.size()) {
                    const uint32_t lh = f.lohi[i];
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(f.body + kS32BodyFloats * (size_t)(lh & 0xffffu)));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(f.body + kS32BodyFloats * (size_t)(lh >> 16)));
                }
        }
        // one contact update; every lane of a quad takes the same contacts, so its shuffles see all four lanes
        auto update = [&](int i) {
                const float4* C4 = reinterpret_cast<const float4*>(f.c + kS32Floats * i);
                const uint32_t lh = f.lohi[i];
                float* Bl = f.body + kS32BodyFloats * (int)(lh & 0xffffu);
                float* Bh = f.body + kS32BodyFloats * (int)(lh >> 16);
                const float4 r0 = C4[3 * q], r1 = C4[3 * q + 1], r2 = C4[3 * q + 2];   // own row
                float4 v[4];                                                         // update columns
                for (int j = 0; j < 4; ++j) v[j] = C4[3 * j + grp];
                float xo[4];
                for (int j = 0; j < 4; ++j) xo[j] = f.c[kS32Floats * i + 12 * j + 11];
                const float4 l0 = *reinterpret_cast<const float4*>(Bl);
                const float4 l1 = *reinterpret_cast<const float4*>(Bl + 4);
                const float4 h0 = *reinterpret_cast<const float4*>(Bh);
                const float4 h1 = *reinterpret_cast<const float4*>(Bh + 4);
                float* B = on_hi ? Bh : Bl;
                const float4 I0 = *reinterpret_cast<const float4*>(B + 8);
                const float2 I1 = *reinterpret_cast<const float2*>(B + 12);
                // J_q w: linear part (rows 0-2), angular parts of both bodies
                float lin = fmaf(r0.x, l0.x - h0.x, fmaf(r0.y, l0.y - h0.y, r0.z * (l0.z - h0.z)));
                if (q == 3) lin = 0.0f;
                const float alo = fmaf(r1.x, l0.w, fmaf(r1.y, l1.x, r1.z * l1.y));
                const float ahi = fmaf(r2.x, h0.w, fmaf(r2.y, h1.x, r2.z * h1.y));
                const float z = r2.w - rscale * r1.w * (((lin + alo) + ahi) + r0.w);
                float zz[4];
                for (int j = 0; j < 4; ++j) zz[j] = __shfl_sync(qm, z, base | j);
                const float mu = __shfl_sync(qm, r0.x, base | 3);
                const float xn = fmaxf(zz[0], 0.0f);
                // prox onto the friction ball of radius mu xn, without branches
                const float radius = mu * xn;
                const float sqr = fmaf(zz[1], zz[1], fmaf(zz[2], zz[2], zz[3] * zz[3]));
                float scale = sqr > radius * radius ? radius * rsqrtf(sqr) : 1.0f;
                if (xn <= 0.0f) scale = 0.0f;
                const float f1 = zz[1] * scale, f2 = zz[2] * scale, f3 = zz[3] * scale;
                const float d0 = xn - xo[0], d1 = f1 - xo[1], d2 = f2 - xo[2];
                const float d3 = linear ? 0.0f : f3 - xo[3];   // the torsion row has no linear columns
                const float xq = q == 0 ? xn : (q == 1 ? f1 : (q == 2 ? f2 : f3));
                f.c[kS32Floats * i + 12 * q + 11] = xq;
                const float T0 = fmaf(v[2].x, d2, fmaf(v[1].x, d1, v[0].x * d0));
                const float T1 = fmaf(v[2].y, d2, fmaf(v[1].y, d1, v[0].y * d0));
                const float T2 = fmaf(v[2].z, d2, fmaf(v[1].z, d1, v[0].z * d0));
                // the torsion row has no linear columns: linear lanes sum three rows
                const float S0 = linear ? T0 : fmaf(v[3].x, d3, T0);
                const float S1 = linear ? T1 : fmaf(v[3].y, d3, T1);
                const float S2 = linear ? T2 : fmaf(v[3].z, d3, T2);
                // the lane's body: w, m^-1 and fixed flag were loaded above
                const float4 w0 = on_hi ? h0 : l0;
                const float4 w1 = on_hi ? h1 : l1;
                const float m = on_hi ? -w1.z : w1.z;
                const float dw0 = linear ? m * S0 : fmaf(I0.x, S0, fmaf(I0.y, S1, I0.z * S2));
                const float dw1 = linear ? m * S1 : fmaf(I0.y, S0, fmaf(I0.w, S1, I1.x * S2));
                const float dw2 = linear ? m * S2 : fmaf(I0.z, S0, fmaf(I1.x, S1, I1.y * S2));
                // the lane's three components of w: linear (0-2) or angular (3-5), without a branch
                const int off = linear ? 0 : 3;
                const float o0 = linear ? w0.x : w0.w, o1 = linear ? w0.y : w1.x, o2 = linear ? w0.z : w1.y;
                if (w1.w == 0.0f) {   // not a fixed body
                    B[off] = o0 + dw0; B[off + 1] = o1 + dw1; B[off + 2] = o2 + dw2;
                }
        };
        // the first pass outside the loop: most levels hold no more contacts than a team has quads
        int i = start + slot;
        if (i < end) {
            update(i);
            for (i += nslot; i < end; i += nslot) update(i);
        }
        g.sync();
        start = end;
        end = next_end;
    }
}

// The same Gauss-Seidel sweep with one lane per contact: the lane loads the contact's twelve row groups,
// computes the four rows' J w as independent chains, applies the prox and updates both bodies.  A warp takes
// 32 contacts of a level per pass instead of 8, and no shuffle lies on the chain.  Every expression is the
// four-lane sweep's (the same operands, the same fmaf order), so both give the same bits.
template <class G, bool kL2>
__device__ __forceinline__ void s32_sweep_lane(const G& g, const S32Scene& f, int L, float rscale, bool bodies_global) {
    int start = f.lptr[0], end = f.lptr[1];
    for (int l = 1; l <= L; ++l) {
        const int next_end = l < L ? f.lptr[l + 1] : end;
        if (kL2) {   // rows in L2: pull the next level's rows (contiguous in level order) into L1 meanwhile
            const char* p0 = reinterpret_cast<const char*>(f.c + kS32Floats * (size_t)end);
            const int lines = (int)(((size_t)(next_end - end) * kS32Floats * sizeof(float) + 127) / 128);
            for (int t = g.rank(); t < lines; t += g.size())
                asm volatile("prefetch.global.L1 [%0];" ::"l"(p0 + 128 * (size_t)t));
            if (bodies_global)
                for (int i = end + g.rank(); i < next_end; i += g.size()) {
                    const uint32_t lh = f.lohi[i];
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(f.body + kS32BodyFloats * (size_t)(lh & 0xffffu)));
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(f.body + kS32BodyFloats * (size_t)(lh >> 16)));
                }
        }
        for (int i = start + g.rank(); i < end; i += g.size()) {
            const float4* C4 = reinterpret_cast<const float4*>(f.c + kS32Floats * i);
            const uint32_t lh = f.lohi[i];
            float* Bl = f.body + kS32BodyFloats * (int)(lh & 0xffffu);
            float* Bh = f.body + kS32BodyFloats * (int)(lh >> 16);
            float4 R[12];
            for (int k = 0; k < 12; ++k) R[k] = C4[k];
            const float4 l0 = *reinterpret_cast<const float4*>(Bl), l1 = *reinterpret_cast<const float4*>(Bl + 4);
            const float4 h0 = *reinterpret_cast<const float4*>(Bh), h1 = *reinterpret_cast<const float4*>(Bh + 4);
            float z[4];
            for (int q = 0; q < 4; ++q) {
                const float4 r0 = R[3 * q], r1 = R[3 * q + 1], r2 = R[3 * q + 2];
                float lin = fmaf(r0.x, l0.x - h0.x, fmaf(r0.y, l0.y - h0.y, r0.z * (l0.z - h0.z)));
                if (q == 3) lin = 0.0f;
                const float alo = fmaf(r1.x, l0.w, fmaf(r1.y, l1.x, r1.z * l1.y));
                const float ahi = fmaf(r2.x, h0.w, fmaf(r2.y, h1.x, r2.z * h1.y));
                z[q] = r2.w - rscale * r1.w * (((lin + alo) + ahi) + r0.w);
            }
            const float mu = R[9].x;
            const float xn = fmaxf(z[0], 0.0f);
            const float radius = mu * xn;
            const float sqr = fmaf(z[1], z[1], fmaf(z[2], z[2], z[3] * z[3]));
            float scale = sqr > radius * radius ? radius * rsqrtf(sqr) : 1.0f;
            if (xn <= 0.0f) scale = 0.0f;
            const float f1 = z[1] * scale, f2 = z[2] * scale, f3 = z[3] * scale;
            const float d0 = xn - R[2].w, d1 = f1 - R[5].w, d2 = f2 - R[8].w, d3 = f3 - R[11].w;
            f.c[kS32Floats * i + 11] = xn;
            f.c[kS32Floats * i + 23] = f1;
            f.c[kS32Floats * i + 35] = f2;
            f.c[kS32Floats * i + 47] = f3;
            // the three sums of the update (the torsion row has no linear columns)
            const float L0 = fmaf(R[6].x, d2, fmaf(R[3].x, d1, R[0].x * d0));
            const float L1 = fmaf(R[6].y, d2, fmaf(R[3].y, d1, R[0].y * d0));
            const float L2 = fmaf(R[6].z, d2, fmaf(R[3].z, d1, R[0].z * d0));
            const float A0 = fmaf(R[10].x, d3, fmaf(R[7].x, d2, fmaf(R[4].x, d1, R[1].x * d0)));
            const float A1 = fmaf(R[10].y, d3, fmaf(R[7].y, d2, fmaf(R[4].y, d1, R[1].y * d0)));
            const float A2 = fmaf(R[10].z, d3, fmaf(R[7].z, d2, fmaf(R[4].z, d1, R[1].z * d0)));
            const float H0 = fmaf(R[11].x, d3, fmaf(R[8].x, d2, fmaf(R[5].x, d1, R[2].x * d0)));
            const float H1 = fmaf(R[11].y, d3, fmaf(R[8].y, d2, fmaf(R[5].y, d1, R[2].y * d0)));
            const float H2 = fmaf(R[11].z, d3, fmaf(R[8].z, d2, fmaf(R[5].z, d1, R[2].z * d0)));
            // lo body: +m^-1 on the linear sums, I_lo^-1 on the angular ones; hi body: -m^-1 and I_hi^-1.
            // Both are computed without a branch; only free bodies are written (a fixed body's is zero).
            const float4 Il0 = *reinterpret_cast<const float4*>(Bl + 8);
            const float2 Il1 = *reinterpret_cast<const float2*>(Bl + 12);
            const float4 Ih0 = *reinterpret_cast<const float4*>(Bh + 8);
            const float2 Ih1 = *reinterpret_cast<const float2*>(Bh + 12);
            const float ml = l1.z, mh = -h1.z;
            const float nl0 = l0.x + ml * L0, nl1 = l0.y + ml * L1, nl2 = l0.z + ml * L2;
            const float nl3 = l0.w + fmaf(Il0.x, A0, fmaf(Il0.y, A1, Il0.z * A2));
            const float nl4 = l1.x + fmaf(Il0.y, A0, fmaf(Il0.w, A1, Il1.x * A2));
            const float nl5 = l1.y + fmaf(Il0.z, A0, fmaf(Il1.x, A1, Il1.y * A2));
            const float nh0 = h0.x + mh * L0, nh1 = h0.y + mh * L1, nh2 = h0.z + mh * L2;
            const float nh3 = h0.w + fmaf(Ih0.x, H0, fmaf(Ih0.y, H1, Ih0.z * H2));
            const float nh4 = h1.x + fmaf(Ih0.y, H0, fmaf(Ih0.w, H1, Ih1.x * H2));
            const float nh5 = h1.y + fmaf(Ih0.z, H0, fmaf(Ih1.x, H1, Ih1.y * H2));
            if (l1.w == 0.0f) { Bl[0] = nl0; Bl[1] = nl1; Bl[2] = nl2; Bl[3] = nl3; Bl[4] = nl4; Bl[5] = nl5; }
            if (h1.w == 0.0f) { Bh[0] = nh0; Bh[1] = nh1; Bh[2] = nh2; Bh[3] = nh3; Bh[4] = nh4; Bh[5] = nh5; }
        }
        g.sync();
        start = end;
        end = next_end;
    }
}

// One proximal Jacobi sweep (proximal_contact/jacobi_solver.py:41-57) on the FP32 copy: every contact's new
// impulse from the accumulators w = W J^T x of the previous iterate, four lanes per contact as in the
// Gauss-Seidel sweep (any order: no contact reads another's new impulse), then w rebuilt from the new
// impulses.  hybrid (jacobi_solver.py:60-79): the friction ball's radius uses the new normal impulse instead
// of the previous one.
template <class G>
__device__ __forceinline__ void s32_sweep_jacobi(const G& g, const SceneRange& R, const S32Scene& f, float rscale,
                                                 bool hybrid) {
    const int K = R.c1 - R.c0;
    const int q = g.rank() & 3, slot = g.rank() >> 2, nslot = g.size() >> 2;
    const int base = (threadIdx.x & 31) & ~3;
    const unsigned qm = 0xfu << base;
    for (int i = slot; i < K; i += nslot) {   // the four lanes of a quad take the same contacts
        const float4* C4 = reinterpret_cast<const float4*>(f.c + kS32Floats * i);
        const uint32_t lh = f.lohi[i];
        const float* Bl = f.body + kS32BodyFloats * (int)(lh & 0xffffu);
        const float* Bh = f.body + kS32BodyFloats * (int)(lh >> 16);
        const float4 r0 = C4[3 * q], r1 = C4[3 * q + 1], r2 = C4[3 * q + 2];   // own row
        const float4 l0 = *reinterpret_cast<const float4*>(Bl), l1 = *reinterpret_cast<const float4*>(Bl + 4);
        const float4 h0 = *reinterpret_cast<const float4*>(Bh), h1 = *reinterpret_cast<const float4*>(Bh + 4);
        float lin = fmaf(r0.x, l0.x - h0.x, fmaf(r0.y, l0.y - h0.y, r0.z * (l0.z - h0.z)));
        if (q == 3) lin = 0.0f;
        const float alo = fmaf(r1.x, l0.w, fmaf(r1.y, l1.x, r1.z * l1.y));
        const float ahi = fmaf(r2.x, h0.w, fmaf(r2.y, h1.x, r2.z * h1.y));
        const float z = r2.w - rscale * r1.w * (((lin + alo) + ahi) + r0.w);
        float zz[4];
        for (int j = 0; j < 4; ++j) zz[j] = __shfl_sync(qm, z, base | j);
        const float mu = __shfl_sync(qm, r0.x, base | 3);
        const float xn_old = __shfl_sync(qm, r2.w, base);   // every read of the old impulses is done here
        const float xn = fmaxf(zz[0], 0.0f);
        float fr[3];
        f32_prox(zz[1], zz[2], zz[3], mu, hybrid ? xn : xn_old, fr);
        f.c[kS32Floats * i + 12 * q + 11] = q == 0 ? xn : fr[q - 1];
    }
    g.sync();
    s32_rebuild_w(g, R, f);
}

// FP64 check of the FP32 iterate and defect correction of the FP32 problem.  With x the current FP32 iterate,
// evaluates A x + b in FP64 (J, W J^T and b of the FP64 problem, w in the scene's global FP64 accumulators)
// and in FP32 (the shared copy), adds the difference to the FP32 b, and returns the FP64 residual
// ||x - prox(x - D^-1 (A x + b))||_inf / max(1, ||x||_inf).  The FP32 sweeps that follow then converge to the
// FP64 problem's solution: at the current x the corrected FP32 problem has the FP64 problem's residual.  The
// FP32 w must hold W J^T x for this x (the residual test just before rebuilt it).
template <class G>
__device__ __forceinline__ double s32_correct(const StepArgs& a, const G& g, const SceneRange& R, const S32Scene& f,
                                              bool correct = true) {
    const int K = R.c1 - R.c0, nb = R.b1 - R.b0;
    const int* order = a.ws.lev_order + R.c0;
    double* w64 = a.ws.w + 6 * (size_t)R.b0;   // the scene's FP64 accumulators, unused until the FP64 solve
    for (int bl = g.rank(); bl < nb; bl += g.size()) {
        double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (f.body[kS32BodyFloats * bl + 7] == 0.0f) {
            for (int e = f.bptr[bl]; e < f.bptr[bl + 1]; ++e) {
                const uint32_t code = f.blist[e];
                const int i = (int)(code >> 1), side = (int)(code & 1);
                const double* Wk = a.ws.WJT + 48 * (size_t)order[i] + 6 * side;
                for (int q = 0; q < 4; ++q) {
                    const double xq = (double)f.c[kS32Floats * i + 12 * q + 11];
                    for (int d = 0; d < 6; ++d) acc[d] = fma(Wk[12 * q + d], xq, acc[d]);
                }
            }
        }
        for (int d = 0; d < 6; ++d) w64[6 * bl + d] = acc[d];
    }
    g.sync();
    double m = 0.0, xm = 0.0;
    for (int i = g.rank(); i < K; i += g.size()) {
        const size_t k = (size_t)order[i];
        const uint32_t lh = f.lohi[i];
        const int lo = (int)(lh & 0xffffu), hi = (int)(lh >> 16);
        const double* wl = w64 + 6 * lo;
        const double* wh = w64 + 6 * hi;
        const float* wl32 = f.body + kS32BodyFloats * lo;
        const float* wh32 = f.body + kS32BodyFloats * hi;
        double z[4], x[4];
        for (int q = 0; q < 4; ++q) {
            const double* J = a.ws.J + 48 * k + 12 * q;
            double v64 = a.ws.b[4 * k + q];
            for (int c = 0; c < 6; ++c) v64 = fma(J[c], wl[c], v64);
            for (int c = 0; c < 6; ++c) v64 = fma(J[6 + c], wh[c], v64);
            float* row = f.c + kS32Floats * i + 12 * q;
            if (correct) {
                const float v32 = s32_jw(row, q, wl32, wh32) + row[3];
                row[3] += (float)(v64 - (double)v32);
            }
            x[q] = (double)row[11];
            z[q] = x[q] - v64 / a.ws.diag[4 * k + q];
        }
        const double pn = z[0] > 0.0 ? z[0] : 0.0;
        double fr[3];
        prox_sphere(z[1], z[2], z[3], a.ws.mu[k], pn, fr);
        const double d[4] = {x[0] - pn, x[1] - fr[0], x[2] - fr[1], x[3] - fr[2]};
        for (int t = 0; t < 4; ++t) {
            m = fmax(m, fabs(d[t]));
            if (d[t] != d[t]) m = d[t];
            xm = fmax(xm, fabs(x[t]));
        }
    }
    const double mres = g.max(m);
    const double mx = g.max(xm);
    g.sync();
    return mres / (mx > 1.0 ? mx : 1.0);
}

// size class of a scene's FP32 copy: 0 and 1 warp teams with small and mid slabs, 2 block teams with the
// large slab, 3 block teams with the contact rows in L2; -1 for a scene the FP32 phase leaves to FP64
__host__ __device__ inline int s32_class(int K, int nb, size_t small_slab, size_t mid_slab) {
    if (K == 0 || K > 32767 || nb > 32767) return -1;   // 16-bit positions and list offsets
    const size_t bytes = s32_bytes(K, nb);
    if (bytes <= small_slab) return 0;
    if (bytes <= mid_slab) return 1;
    if (bytes <= (size_t)kFp32LargeSmem) return 2;
    const bool bodies_global = s32_bytes(K, nb, true) > (size_t)kFp32LargeSmem;
    return s32_bytes(K, nb, true, bodies_global) <= (size_t)kFp32LargeSmem ? 3 : -1;
}

// Per-scene FP32 bookkeeping of the step, and the scene list of each size class, longest expected chain
// first, so that every team's next scene is one of its class and the scenes that bound the step start first.
// The expected chain of a scene is its previous step's levels x sweeps (the solve length in level steps,
// the sweeps floored at half the cap), read before this step resets them; without a plausible history (first
// step, a scene new to its slot) it is estimated from the contact count.  The order decides only which team takes which scene and when, never a
// result.  One block.
constexpr int kClassBuckets = 64;
__global__ void __launch_bounds__(1024) k_fp32_classes(const StepArgs a, size_t small_slab, size_t mid_slab) {
    __shared__ int cnt[4 * kClassBuckets];
    const int S = a.bd.n_scenes;
    // no lists after an overflow: the contact ranges are not valid then, and the solvers do not run
    const bool fp32 = a.pr.precision != RB_PRECISION_FP64 && !a.ws.counters[kAbort];
    const int max_it = a.pr.max_iterations;
    for (int t = threadIdx.x; t < 4 * kClassBuckets; t += blockDim.x) cnt[t] = 0;
    __syncthreads();
    auto slot = [&](int s) -> int {   // class x buckets + expected-chain bucket (descending), or -1
        const SceneRange R = scene_range(a, s);
        const int K = R.c1 - R.c0;
        const int c = s32_class(K, R.b1 - R.b0, small_slab, mid_slab);
        if (c < 0) return -1;
        // previous levels x sweeps, the sweeps floored at half the cap: whether a scene converges early varies
        // from step to step, and one that converged last step may run to the cap in this one
        const int Lp = a.ws.nlev[s], Sp = a.ws.sweeps32[s];
        const bool known = Lp > 0 && Lp <= K && Sp > 0 && Sp <= max_it;
        const float w = known ? (float)Lp * (float)max(Sp, max_it / 2) : 0.25f * (float)K * (float)max_it;
        const int lg = (int)(2.0f * log2f(w + 1.0f));   // buckets of a factor 2^(1/2)
        return kClassBuckets * c + kClassBuckets - 1 - min(lg, kClassBuckets - 1);
    };
    if (fp32)
        for (int s = threadIdx.x; s < S; s += blockDim.x) {
            const int t = slot(s);
            if (t >= 0) atomicAdd(&cnt[t], 1);
        }
    __syncthreads();
    if (fp32 && threadIdx.x == 0) {   // counts -> starts; class ends to the counters
        int run = 0;
        for (int t = 0; t < 4 * kClassBuckets; ++t) {
            const int n = cnt[t];
            cnt[t] = run;
            run += n;
            if ((t % kClassBuckets) == kClassBuckets - 1) a.ws.counters[kClassEnd32 + t / kClassBuckets] = run;
        }
    }
    __syncthreads();
    for (int s = threadIdx.x; s < S; s += blockDim.x) {   // the thread that keyed scene s places and resets it
        if (fp32) {
            const int t = slot(s);
            if (t >= 0) a.ws.list32[atomicAdd(&cnt[t], 1)] = s;
        }
        a.ws.sweeps32[s] = -1;
        a.ws.fin32[s] = 0;
    }
}

template <class G>
__device__ __forceinline__ int team_next(const G& g, int* counter, int* slot) {
    int s = 0;
    if (g.rank() == 0) s = atomicAdd(counter, 1);
    if (g.size() == 32) return __shfl_sync(0xffffffffu, s, 0);
    if (g.rank() == 0) *slot = s;
    __syncthreads();
    s = *slot;
    __syncthreads();
    return s;
}

// the FP64 solve of a scene as a call of its own, so that it does not raise the FP32 kernel's registers
template <class G>
__device__ __noinline__ void solve_scene_call(const StepArgs& a, const G& g, int s) {
    solve_scene(a, g, s, 0, nullptr, 0);
}

// FP32 phase for the scenes whose compact copy takes lo_bytes < bytes <= slab bytes; G = WarpGroup gives
// every warp of the block its own slab and scene, G = BlockGroup one slab and scene per block.  kL2: the
// scenes too large for any slab, with their contact rows in global memory (L2-resident) and the rest of
// the copy in the slab.
template <class G, bool kL2>
__global__ void __launch_bounds__(kL2 ? kFp32L2Block : kFp32BlockMax, 1) k_solve_fp32(const StepArgs a, int queue, size_t lo_bytes, size_t slab) {
    extern __shared__ __align__(16) char f32_smem[];
    __shared__ double red[33];
    __shared__ int ired[33];
    __shared__ int next_slot;
    if (a.ws.counters[kAbort]) return;
    G g;
    constexpr bool block_team = std::is_same_v<G, BlockGroup>;
    if constexpr (block_team) { g.red = red; g.ired = ired; }
    const int team = block_team ? 0 : (int)(threadIdx.x >> 5);
    char* my_slab = f32_smem + (size_t)team * slab;
    const int max_it = a.pr.max_iterations;
    const int interval = a.pr.residual_interval > 1 ? a.pr.residual_interval : 1;
    // the FP32 sweeps aim a little below the tolerance when an FP64 test follows, so that the FP32 problem
    // rarely meets it while the FP64 one misses it
    const float tol = (float)(a.pr.precision == RB_PRECISION_FP32_REFINE ? 0.5 * a.pr.residual_tolerance
                                                                        : a.pr.residual_tolerance);
    // sweeps reserved for the FP64 refinement
    const int reserve = a.pr.precision == RB_PRECISION_FP32_REFINE ? min(max(a.pr.refine_iterations, 0), max_it) : 0;
    const int budget = max_it - reserve;
    double rs = a.pr.scheme == RB_SCHEME_RIGID_GS ? 1.0 : 0.1;   // the r of the scheme: r = rs / diag
    if (a.pr.relaxation > 0.0) rs *= a.pr.relaxation;
    const float rscale = (float)rs;
    const bool coloured = a.pr.scheme == RB_SCHEME_COLOURED_GS || a.pr.ordering == RB_ORDER_COLOURED;
    const bool jacobi = a.pr.scheme == RB_SCHEME_JACOBI || a.pr.scheme == RB_SCHEME_JACOBI_HYBRID;
    const bool hybrid = a.pr.scheme == RB_SCHEME_JACOBI_HYBRID;
    const int cls = queue - kQueueFp32;
    const int list0 = cls == 0 ? 0 : a.ws.counters[kClassEnd32 + cls - 1];
    const int list1 = a.ws.counters[kClassEnd32 + cls];
    for (;;) {
        const int idx = list0 + team_next(g, a.ws.counters + queue, &next_slot);
        if (idx >= list1) break;
        const int s = a.ws.list32[idx];
        const SceneRange R = scene_range(a, s);
        const int K = R.c1 - R.c0, nb = R.b1 - R.b0;
        if (K == 0 || K > 32767 || nb > 32767) continue;   // 16-bit positions and list offsets
        bool bodies_global = false;
        if (kL2) {   // the scenes no slab holds whole: contact rows in L2, and the bodies too if they do not fit
            if (s32_bytes(K, nb) <= lo_bytes) continue;
            bodies_global = s32_bytes(K, nb, true) > slab;
            if (s32_bytes(K, nb, true, bodies_global) > slab) continue;
        } else {
            const size_t bytes = s32_bytes(K, nb);
            if (bytes <= lo_bytes || bytes > slab) continue;
        }
        const double t0 = a.pr.profiling ? device_us() : 0.0;
        const S32Scene f = s32_carve(my_slab, K, nb, kL2 ? &a : nullptr, R.c0, bodies_global, R.b0);
        // scratch for the level relaxation: the rows' room of the slab, or with rows in L2 what the slab has left
        int16_t* scratch = nullptr;
        if (!kL2) {   // a contact record's bytes per contact there, more than s32_level_scratch needs
            scratch = reinterpret_cast<int16_t*>(f.c);
        } else {
            const size_t off = (s32_bytes(K, nb, true, bodies_global) + 15) & ~size_t(15);
            if (off + s32_level_scratch(K) <= slab) scratch = reinterpret_cast<int16_t*>(my_slab + off);
        }
        const int L = s32_load(a, g, R, s, f, coloured, scratch);
        if (g.rank() == 0) a.ws.nlev[s] = L;
        float res = s32_residual(a, g, R, f);   // the warm-started iterate may already be good enough
        float best = res;
        int sweeps = 0, stalls = 0, window = kS32StallTests;
        // far above the tolerance (and the stall floor) the residual is tested half as often: no stop and no
        // stall can be decided there, and each test rebuilds w
        auto gap = [&](float r) { return r > kS32FarFactor * tol ? 2 * interval : interval; };
        int next_test = gap(res);
        double r64 = -1.0;            // FP64 residual of the current iterate, once evaluated
        double r64_round = INFINITY;  // FP64 residual after the previous correction round
        for (;;) {
            const int round_start = sweeps;
            while (res > tol && sweeps < budget) {
                if (jacobi) {
                    s32_sweep_jacobi(g, R, f, rscale, hybrid);
                } else if (!block_team) {
                    s32_sweep_lane<G, kL2>(g, f, L, rscale, bodies_global);
                } else if (!kL2) {
                    // a block team's slab scene: its levels rarely hold more contacts than a warp has lanes,
                    // so warp 0 sweeps it one lane per contact (the same bits as four lanes per contact) with
                    // warp barriers between levels, and the block meets once per sweep
                    if (threadIdx.x < 32) s32_sweep_lane<WarpGroup, false>(WarpGroup{}, f, L, rscale, false);
                    g.sync();
                } else {
                    s32_sweep<G, kL2>(g, f, L, rscale, bodies_global);
                }
                ++sweeps;
                if (--next_test == 0 || sweeps == budget) {
                    res = s32_residual(a, g, R, f);
                    next_test = gap(res);
                    // a round ends once the residual, already small, stops improving for a while (the FP32
                    // problem's own rounding, or slow progress a defect correction may speed up).  Above the
                    // floor a pause is the Gauss-Seidel iteration itself (it is not monotone), so go on.
                    if (res < 0.95f * best) { best = res; stalls = 0; }
                    else if (best < kFp32Floor && ++stalls >= window) break;
                }
            }
            // FP32 + refinement: test in FP64; if the FP32 answer misses the tolerance in FP64, correct the FP32
            // problem's b by the FP64 defect and sweep on in FP32.  FP64 sweeps take over only when the FP32
            // problem meets the tolerance and the FP64 one does not (the FP32 sweeps can do no more).
            if (a.pr.precision != RB_PRECISION_FP32_REFINE || sweeps >= budget) break;
            r64 = s32_correct(a, g, R, f);
            if (r64 <= a.pr.residual_tolerance) break;
            if (sweeps == round_start) break;   // r64 stays valid for x
            if (r64 > kS32RoundGain * r64_round) window = min(2 * window, kS32StallTestsMax);
            r64_round = fmin(r64_round, r64);
            r64 = -1.0;   // the sweeps that follow change the iterate
            res = s32_residual(a, g, R, f);
            next_test = gap(res);
            best = res;
            stalls = 0;
        }
        // the FP64 residual of the iterate decides whether FP64 sweeps follow; when none do, this kernel
        // finishes the scene (solution, statistics), and when some do, this team runs them right away, so
        // the FP64 solver launched after the FP32 phase skips the scene either way
        if (r64 < 0.0) r64 = s32_correct(a, g, R, f, false);
        const bool finished = r64 <= a.pr.residual_tolerance || sweeps >= max_it ||
                              a.pr.precision == RB_PRECISION_FP32;
        for (int t = g.rank(); t < 4 * K; t += g.size()) {   // back to contact order
            const int i = t >> 2, q = t & 3;
            const size_t k4 = 4 * (size_t)a.ws.lev_order[R.c0 + i] + q;
            const double xv = (double)f.c[kS32Floats * i + 12 * q + 11];
            a.ws.x[k4] = xv;
            if (finished) a.out.contact_sol[k4] = xv;
        }
        if (finished && a.out.residuals && a.pr.profiling)
            for (int i = g.rank(); i < max_it; i += g.size()) a.out.residuals[(size_t)s * a.caps.max_iterations + i] = INFINITY;
        if (g.rank() == 0) {
            a.ws.sweeps32[s] = sweeps;
            a.ws.fin32[s] = finished ? 1 : 0;
            rb_scene_stats* st = a.out.stats + s;
            st->solve_start_us = t0;
            st->solve_us = a.pr.profiling ? device_us() - t0 : 0.0;
            if (finished) {
                const bool ok = r64 <= a.pr.residual_tolerance;
                st->n_contacts = K; st->contact_start = R.c0;
                st->iterations = ok ? max(sweeps - 1, 0) : max_it;
                st->exitcode = ok ? 3 : 0;
                st->merit = r64; st->residual = r64;
                st->post_iterations = -1; st->post_exitcode = -1;
                st->n_levels = L; st->fp32_sweeps = sweeps;
            }
        }
        g.sync();
        if (!kL2 && !finished) {   // FP64 sweeps with the budget left, by this team at once (w in global memory)
            solve_scene_call(a, g, s);
            if (g.rank() == 0) a.ws.fin32[s] = 1;
            g.sync();
        }
    }
}

constexpr int kSolveBlock = 128;   // threads per scene in the block solver (levels rarely hold more contacts)
constexpr int kWarpSceneMaxContacts = 2048;
constexpr int kWarpSceneMaxBodies = 384;
constexpr int kSolveWarpsPerBlock = 4;

__device__ __forceinline__ int scene_contacts(const StepArgs& a, int s) {
    const SceneRange R = scene_range(a, s);
    return R.c1 - R.c0;
}

// scenes with at most kWarpSceneMaxContacts contacts and warp_bodies bodies: one warp each
__global__ void __launch_bounds__(32 * kSolveWarpsPerBlock) k_solve_warps(const StepArgs a, int post, int warp_bodies) {
    extern __shared__ double wsm[];
    if (a.ws.counters[kAbort]) return;
    const WarpGroup g;
    const int wib = threadIdx.x >> 5;
    double* w_smem = warp_bodies > 0 ? wsm + (size_t)wib * 6 * warp_bodies : nullptr;
    for (int s = blockIdx.x * kSolveWarpsPerBlock + wib; s < a.bd.n_scenes; s += gridDim.x * kSolveWarpsPerBlock) {
        const int nb = a.bd.scene_start[s + 1] - a.bd.scene_start[s];
        if (scene_contacts(a, s) > kWarpSceneMaxContacts || nb > warp_bodies) continue;
        solve_scene(a, g, s, post, w_smem, warp_bodies);
    }
}

// the other scenes: one block each; the body accumulators are on chip up to smem_bodies bodies
__global__ void __launch_bounds__(kSolveBlock) k_solve_blocks(const StepArgs a, int post, int warp_bodies, int smem_bodies) {
    extern __shared__ double wsm[];
    __shared__ double red[33];
    __shared__ int ired[33];
    if (a.ws.counters[kAbort]) return;
    const BlockGroup g = {red, ired};
    for (int s = blockIdx.x; s < a.bd.n_scenes; s += gridDim.x) {
        const int nb = a.bd.scene_start[s + 1] - a.bd.scene_start[s];
        if (scene_contacts(a, s) <= kWarpSceneMaxContacts && nb <= warp_bodies) continue;
        solve_scene(a, g, s, post, smem_bodies > 0 ? wsm : nullptr, smem_bodies);
    }
}

// ---------------------------------------------------------------------------------------------------------
// integration (state_storage.py:239 velocity_update, :251 position_update): thread per body
// ---------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void position_update(double* xb, const double* ub, double dt) {
    for (int i = 0; i < 3; ++i) xb[i] = xb[i] + ub[i] * dt;
    const double qw[4] = {0.0, ub[3], ub[4], ub[5]};
    double q[4] = {xb[3], xb[4], xb[5], xb[6]}, dq[4], qn[4];
    quat_prod(qw, q, dq);
    for (int i = 0; i < 4; ++i) qn[i] = q[i] + (dq[i] * dt) * 0.5;
    quat_unit(qn, xb + 3);
}

__global__ void k_integrate(const StepArgs a) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.bd.n_bodies || a.ws.counters[kAbort]) return;
    double* ub = a.bd.u + 6 * b;
    double du[6];
    for (int d = 0; d < 6; ++d) du[d] = a.ws.du[6 * b + d];
    if (!a.bd.fixed[b] && a.ws.bc_ptr[b + 1] > a.ws.bc_ptr[b]) {   // delta_u += WJT sol (steppers.py:84-85)
        double dc[6];
        body_wjt_dot(a.ws, b, a.out.contact_sol, dc);
        for (int d = 0; d < 6; ++d) du[d] = du[d] + dc[d];
    }
    if (a.bd.n_hinges > 0 && !a.bd.fixed[b] && a.ws.hbody_ptr[b + 1] > a.ws.hbody_ptr[b]) {
        // then the hinge problem's WJT sol (hinges.py:52), hinges ascending, 5 rows each
        for (int d = 0; d < 6; ++d) {
            double t = 0.0;
            for (int e = a.ws.hbody_ptr[b]; e < a.ws.hbody_ptr[b + 1]; ++e) {
                const int code = a.ws.hbody_list[e];
                const int k = code >> 1, side = code & 1;
                const double* Wk = a.ws.hWJT + 60 * (size_t)k + 6 * side;
                for (int row = 0; row < 5; ++row) t += Wk[12 * row + d] * a.ws.hsol[5 * (size_t)k + row];
            }
            du[d] = du[d] + t;
        }
    }
    for (int d = 0; d < 6; ++d) ub[d] = ub[d] + du[d];
    if (a.bd.fixed[b]) return;
    position_update(a.bd.x + 7 * b, ub, a.pr.dt);
    bool finite = true;
    for (int d = 0; d < 7; ++d) finite &= isfinite(a.bd.x[7 * b + d]);
    for (int d = 0; d < 6; ++d) finite &= isfinite(ub[d]);
    if (!finite) atomicOr(a.out.status, RB_STATUS_NONFINITE);
}

// post-stabilisation problem (post_stabilization.py:30-104): b = gap on deep normal rows, r = 1/diag
__global__ void k_post_setup(const StepArgs a) {
    if (a.ws.counters[kAbort]) return;
    const int K = a.ws.counters[kNContacts];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        const double g = a.out.contact_g[k];
        for (int row = 0; row < 4; ++row) {
            a.ws.b[4 * k + row] = (row == 0 && g < -a.pr.min_gap_value) ? g : 0.0;
            a.ws.r[4 * k + row] = 1.0 / a.ws.diag[4 * k + row];
            a.ws.x[4 * k + row] = 0.0;
            a.ws.xold[4 * k + row] = 0.0;
        }
    }
}
__global__ void k_post_apply(const StepArgs a) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.bd.n_bodies || a.ws.counters[kAbort] || a.bd.fixed[b]) return;
    // every non-fixed body of a corrected scene is updated (and its quaternion renormalised), contacts or not
    const int s = scene_of(a.bd.scene_start, a.bd.n_scenes, b);
    if (a.out.stats[s].post_iterations < 0) return;   // this scene had nothing to correct
    double dr[6];
    body_wjt_dot(a.ws, b, a.ws.xold, dr);
    position_update(a.bd.x + 7 * b, dr, 1.0);
}

// energies and largest penetration (state_storage.py:188, contacts.py:222): thread per scene, body order
// one warp per scene: the deepest gap and the pair / candidate counts by warp reductions (order-free), the
// energy sums by lane 0 in body order (their rounding follows state_storage.py:188-237)
__global__ void k_scene_summary(const StepArgs a) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= a.bd.n_scenes || a.ws.counters[kAbort]) return;
    rb_scene_stats* st = a.out.stats + s;
    const SceneRange R = scene_range(a, s);
    double gap = 0.0;
    for (int k = R.c0 + lane; k < R.c1; k += 32) gap = fmin(gap, a.out.contact_g[k]);
    for (int o = 16; o > 0; o >>= 1) gap = fmin(gap, __shfl_xor_sync(0xffffffffu, gap, o));
    const int p0 = a.ws.pair_cnt[R.b0], p1 = a.ws.pair_cnt[R.b1];
    int ovl = 0, cand = 0;
    if (a.pr.profiling)
        for (int p = p0 + lane; p < p1; p += 32) { ovl += a.ws.pair_ovl[p]; cand += a.ws.pair_itemsA[p]; }
    for (int o = 16; o > 0; o >>= 1) {
        ovl += __shfl_xor_sync(0xffffffffu, ovl, o);
        cand += __shfl_xor_sync(0xffffffffu, cand, o);
    }
    if (lane != 0) return;
    st->max_penetration = -gap;
    st->n_pairs = p1 - p0;
    st->n_candidates = cand;
    st->n_leaf_overlaps = ovl;
    if (!a.pr.profiling) return;
    int has_gravity = 0;
    for (int f = a.bd.scene_force_start[s]; f < a.bd.scene_force_start[s + 1]; ++f)
        if (a.bd.force_kind[f] == 0) has_gravity = 1;
    // the per-body terms come from k_body_energy
    double kinetic = 0.0, potential = 0.0;
#pragma unroll 8
    for (int b = R.b0; b < R.b1; ++b) {
        if (a.bd.fixed[b]) continue;
        if (has_gravity) potential += a.ws.eterm[2 * (size_t)b + 1];
        kinetic += a.ws.eterm[2 * (size_t)b];
    }
    st->kinetic_energy = kinetic;
    st->potential_energy = potential;
}

// per-body energy terms of a profiled step (StateStorage.compute_total_energy, state_storage.py:188-237):
// 0.5 (m v.v + w.(I_w w)) and m g (up . r) with the scene's summed gravity
__global__ void k_body_energy(const StepArgs a) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.bd.n_bodies || a.ws.counters[kAbort]) return;
    double* out = a.ws.eterm + 2 * (size_t)b;
    if (a.bd.fixed[b]) { out[0] = 0.0; out[1] = 0.0; return; }
    const int s = scene_of(a.bd.scene_start, a.bd.n_scenes, b);
    double G[3] = {0.0, 0.0, 0.0};
    int has_gravity = 0;
    for (int f = a.bd.scene_force_start[s]; f < a.bd.scene_force_start[s + 1]; ++f)
        if (a.bd.force_kind[f] == 0) {
            const double* fp = a.bd.force_params + 4 * f;
            for (int i = 0; i < 3; ++i) G[i] = G[i] + fp[1 + i] * fp[0];
            has_gravity = 1;
        }
    const double* xb = a.bd.x + 7 * b;
    double Rm[9], Iw[9], Ib[3] = {a.bd.inertia[3 * b], a.bd.inertia[3 * b + 1], a.bd.inertia[3 * b + 2]};
    quat_to_matrix(xb + 3, Rm);
    update_inertia_tensor(Rm, Ib, Iw);
    const double m = a.bd.mass[b];
    double pot = 0.0;
    if (has_gravity) {
        const d3 Gv = d3{G[0], G[1], G[2]};
        const double ln = norm3_np(Gv);
        const d3 up = d3{G[0] / ln, G[1] / ln, G[2] / ln};
        const double g = norm3_np(Gv);
        const double h = dot3_np(up, ld3(xb));
        pot = m * g * h;
    }
    const d3 v = ld3(a.bd.u + 6 * b), w = ld3(a.bd.u + 6 * b + 3);
    const double wIw = dot3_np(w, gemv3_np(Iw, w));
    out[0] = 0.5 * (m * dot3_np(v, v) + wIw);
    out[1] = pot;
}

// keep this step's contact keys and impulses for the next step's warm start
__global__ void k_cache_store(const StepArgs a) {
    if (!a.out.cache_key || !a.out.cache_sol || !a.out.cache_count) return;
    if (a.ws.counters[kAbort]) return;
    const int K = min(a.ws.counters[kNContacts], a.caps.contact_capacity);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < K; k += gridDim.x * blockDim.x) {
        a.out.cache_key[2 * k] = a.ws.ckey[2 * k];
        a.out.cache_key[2 * k + 1] = a.ws.ckey[2 * k + 1];
        for (int row = 0; row < 4; ++row) a.out.cache_sol[4 * k + row] = a.out.contact_sol[4 * k + row];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.out.cache_count = K;
}

__global__ void k_finish(const StepArgs a) {
    if (a.out.n_contacts_total) *a.out.n_contacts_total = a.ws.counters[kNContacts];
    if (a.out.needed) {   // a stage after an overflow did not run: its total is reported as 0
        const int ab = a.ws.counters[kAbort];
        a.out.needed[0] = a.ws.counters[kNPairs];
        a.out.needed[1] = (ab & RB_STATUS_PAIR_OVERFLOW) ? 0 : a.ws.counters[kNItems];
        a.out.needed[2] = (ab & (RB_STATUS_PAIR_OVERFLOW | RB_STATUS_ITEM_OVERFLOW)) ? 0 : a.ws.counters[kNContacts];
    }
}

// ---------------------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------------------
thread_local std::string g_error;

// phase events of the last profiled step (host-side CUDA events; no device memory)
struct ProfileEvents {
    cudaEvent_t ev[8];
    bool created = false;
    bool recorded = false;
};
thread_local ProfileEvents g_prof;

static void prof_mark(bool on, int i, cudaStream_t st) {
    if (!on) return;
    if (!g_prof.created) {
        for (int k = 0; k < 8; ++k) cudaEventCreate(&g_prof.ev[k]);
        g_prof.created = true;
    }
    cudaEventRecord(g_prof.ev[i], st);
    if (i == 6) g_prof.recorded = true;
}

static int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

static inline int blocks_for(int64_t n, int block) { return (int)((n + block - 1) / block > 0 ? (n + block - 1) / block : 1); }

}  // namespace rb

using namespace rb;

extern "C" {

int rb_abi_version(void) { return RB_ABI_VERSION; }

const char* rb_last_error(void) { return rb::g_error.c_str(); }

int rb_topology_sizes(int32_t n_bodies, const int32_t* body_shape, int32_t n_shapes, const int32_t* v_off,
                      const int32_t* t_off, int64_t* out) {
    if (n_bodies < 0 || n_shapes <= 0 || !body_shape || !v_off || !t_off || !out)
        return fail(RB_ERR_ARG, "rb_topology_sizes: bad argument");
    int64_t nv = 0, nt = 0, nc = 0;
    for (int b = 0; b < n_bodies; ++b) {
        const int s = body_shape[b];
        if (s < 0 || s >= n_shapes) return fail(RB_ERR_ARG, "rb_topology_sizes: shape index out of range");
        nv += v_off[s + 1] - v_off[s];
        const int t = t_off[s + 1] - t_off[s];
        nt += t;
        nc += (t + 31) / 32;
    }
    out[0] = nv; out[1] = nt; out[2] = nc;
    return RB_OK;
}

int rb_workspace_bytes(const rb_bodies* bd, const rb_caps* caps, size_t* bytes) {
    if (!bd || !caps || !bytes) return fail(RB_ERR_ARG, "rb_workspace_bytes: null argument");
    if (bd->n_bodies < 0 || bd->n_body_vertices < 0 || bd->n_body_triangles < 0 || bd->n_clusters < 0 ||
        caps->pair_capacity < 0 || caps->item_capacity < 0 || caps->contact_capacity < 0)
        return fail(RB_ERR_ARG, "rb_workspace_bytes: negative size");
    if (bd->n_hinges < 0) return fail(RB_ERR_ARG, "rb_workspace_bytes: negative hinge count");
    *bytes = rb::layout(nullptr, nullptr, bd->n_bodies, bd->n_body_vertices, bd->n_body_triangles, bd->n_clusters,
                        caps->pair_capacity, caps->item_capacity, caps->contact_capacity, bd->n_scenes,
                        bd->n_hinges);
    return RB_OK;
}

}  // extern "C"

namespace {
// Largest dynamic shared memory of each solver kernel, granted once per device.  Done outside the launch
// sequence so that a step can be captured into a CUDA graph once the device has seen one uncaptured step.
std::mutex g_attr_mutex;
bool g_attr_done[64] = {false};
int ensure_kernel_attributes() {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return fail(RB_ERR_CUDA, "rb_step: no current device");
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    if (g_attr_done[dev]) return RB_OK;
    const int warp_max = kSolveWarpsPerBlock * 6 * (int)sizeof(double) * kWarpSceneMaxBodies;
    const int block_max = 6 * (int)sizeof(double) * kSolveSmemBodies;
    e = cudaFuncSetAttribute(k_solve_warps, cudaFuncAttributeMaxDynamicSharedMemorySize, warp_max);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_solve_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, block_max);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_solve_fp32<WarpGroup, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFp32LargeSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_solve_fp32<BlockGroup, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFp32LargeSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_solve_fp32<BlockGroup, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFp32LargeSmem);
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, std::string("rb_step: cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    g_attr_done[dev] = true;
    return RB_OK;
}

// Side streams of the FP32 size classes, per host thread and device: kSideSets sets, all made on the thread's
// first step on the device (an uncaptured call).  Each caller stream gets a set of its own (round robin over
// the sets, so steps on different streams run their solves concurrently); a step forks its set from its
// stream with an event and joins it back, which a stream capture records as parallel branches.
constexpr int kSideStreams = 4;
constexpr int kSideSets = 4;
struct SideStreams {
    cudaStream_t s[kSideStreams] = {};
    cudaEvent_t fork = nullptr, join[kSideStreams] = {};
};
struct SideSets {
    SideStreams set[kSideSets];
    const void* key[kSideSets] = {};
    int next = 0;
    bool made = false;
};
thread_local SideSets g_side[64];
int side_streams(cudaStream_t caller, SideStreams** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return fail(RB_ERR_CUDA, "rb_step: no current device");
    SideSets& ss = g_side[dev];
    if (!ss.made) {
        cudaError_t e = cudaSuccess;
        for (int k = 0; k < kSideSets && e == cudaSuccess; ++k) {
            SideStreams& t = ss.set[k];
            e = cudaEventCreateWithFlags(&t.fork, cudaEventDisableTiming);
            for (int c = 0; c < kSideStreams && e == cudaSuccess; ++c) {
                e = cudaStreamCreateWithFlags(&t.s[c], cudaStreamNonBlocking);
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t.join[c], cudaEventDisableTiming);
            }
        }
        if (e != cudaSuccess) return fail(RB_ERR_CUDA, std::string("rb_step: side streams: ") + cudaGetErrorString(e));
        ss.made = true;
    }
    int k = 0;
    while (k < kSideSets && ss.key[k] != (const void*)caller) ++k;
    if (k == kSideSets) {   // a caller stream not seen before takes the next set
        k = ss.next;
        ss.next = (ss.next + 1) % kSideSets;
        ss.key[k] = (const void*)caller;
    }
    *out = &ss.set[k];
    return RB_OK;
}
}  // namespace

extern "C" {

int rb_step(const rb_shapes* sh, const rb_bodies* bd, const rb_caps* caps, const rb_params* pr,
            const rb_outputs* out, void* workspace, size_t workspace_bytes, void* stream_ptr) {
    if (!sh || !bd || !caps || !pr || !out || !workspace) return fail(RB_ERR_ARG, "rb_step: null argument");
    if (bd->n_bodies <= 0 || bd->n_scenes <= 0) return fail(RB_ERR_ARG, "rb_step: empty scene batch");
    if (!bd->x || !bd->u || !out->contact_ids || !out->stats || !out->status)
        return fail(RB_ERR_ARG, "rb_step: null state or output buffer");
    if (pr->scheme < 0 || pr->scheme > RB_SCHEME_COLOURED_GS)
        return fail(RB_ERR_UNSUPPORTED, "rb_step: unknown solver scheme");
    if (pr->ordering != RB_ORDER_SERIAL && pr->ordering != RB_ORDER_COLOURED)
        return fail(RB_ERR_ARG, "rb_step: unknown contact ordering");
    if (bd->n_hinges < 0 || (bd->n_hinges > 0 && (!bd->scene_hinge_start || !bd->hinge_bodies || !bd->hinge_frames)))
        return fail(RB_ERR_ARG, "rb_step: hinge arrays missing");
    if (bd->n_hinges > 0 && (pr->scheme != RB_SCHEME_RIGID_GS || pr->termination != RB_TERMINATE_MERIT ||
                             pr->ordering != RB_ORDER_SERIAL || pr->precision != RB_PRECISION_FP64))
        return fail(RB_ERR_UNSUPPORTED, "rb_step: hinge joints are solved with the reference stepper's rule only "
                                        "(rigid Gauss-Seidel, merit termination, serial order, FP64)");
    // launch shapes
    const int small_slab = pr->fp32_small_slab > 0 ? pr->fp32_small_slab : kS32SmallSlab;
    const int mid_slab = pr->fp32_mid_slab > 0 ? pr->fp32_mid_slab : kS32MidSlab;
    const int mid_blocks = pr->mid_blocks > 0 ? pr->mid_blocks : 148 * 16;
    const int narrow_blocks = pr->narrow_blocks > 0 ? pr->narrow_blocks : 148 * 8;
    const int narrow_threads = pr->narrow_threads > 0 ? pr->narrow_threads : 256;
    if (small_slab % 16 || mid_slab % 16 || small_slab < 4096 || small_slab >= mid_slab || mid_slab > kS32MidSlab)
        return fail(RB_ERR_ARG, "rb_step: FP32 slabs must be multiples of 16 with 4096 <= small < mid <= 57344");
    if (mid_blocks > 65535 || narrow_blocks > 65535 ||
        (narrow_threads != 64 && narrow_threads != 128 && narrow_threads != 256))
        return fail(RB_ERR_ARG, "rb_step: launch shape out of range");
    if (pr->max_iterations < 0 || pr->max_iterations > caps->max_iterations)
        return fail(RB_ERR_ARG, "rb_step: max_iterations exceeds rb_caps.max_iterations");
    if (!(pr->dt > 0.0)) return fail(RB_ERR_ARG, "rb_step: dt must be positive");
    if (pr->precision != RB_PRECISION_FP64 && pr->termination != RB_TERMINATE_RESIDUAL_FIXED_R)
        return fail(RB_ERR_UNSUPPORTED, "rb_step: FP32 precision needs the fixed-r residual rule");
    if (pr->precision < RB_PRECISION_FP64 || pr->precision > RB_PRECISION_FP32)
        return fail(RB_ERR_ARG, "rb_step: unknown precision");
    if (sh->max_shape_triangles <= 0 || sh->max_shape_triangles > 32 * kMaxClustersPerShape)
        return fail(RB_ERR_ARG, "rb_step: max_shape_triangles must be in 1..16384");
    size_t need = 0;
    int rc = rb_workspace_bytes(bd, caps, &need);
    if (rc != RB_OK) return rc;
    if (workspace_bytes < need) return fail(RB_ERR_WORKSPACE, "rb_step: workspace too small");
    rc = ensure_kernel_attributes();
    if (rc != RB_OK) return rc;
    const int64_t n_body_vertices = bd->n_body_vertices, n_body_triangles = bd->n_body_triangles,
                  n_clusters = bd->n_clusters;
    cudaStream_t st = (cudaStream_t)stream_ptr;
    StepArgs a;
    a.sh = *sh; a.bd = *bd; a.caps = *caps; a.pr = *pr; a.out = *out;
    rb::layout(&a.ws, (char*)workspace, bd->n_bodies, n_body_vertices, n_body_triangles, n_clusters,
               caps->pair_capacity, caps->item_capacity, caps->contact_capacity, bd->n_scenes, bd->n_hinges);
    if (n_body_vertices <= 0 || n_body_triangles <= 0 || n_clusters <= 0)
        return fail(RB_ERR_ARG, "rb_step: bodies without geometry");
    const int N = bd->n_bodies;
    const int G = 148 * 8;
    const bool prof = pr->profiling != 0;
    prof_mark(prof, 0, st);
    k_zero_i32<<<1, 32, 0, st>>>(a.ws.counters, 16); note_launch();
    k_zero_stats<<<blocks_for(bd->n_scenes, 128), 128, 0, st>>>(a); note_launch();
    k_zero_i32<<<blocks_for(N + 1, 256), 256, 0, st>>>(a.ws.bc_ptr, N + 1); note_launch();
    k_zero_i32<<<blocks_for(N, 256), 256, 0, st>>>(a.ws.bc_fill, N); note_launch();
    k_bodies<<<blocks_for(N, 128), 128, 0, st>>>(a); note_launch();
    k_world_vertices<<<blocks_for(n_body_vertices, 256), 256, 0, st>>>(a, (int)n_body_vertices); note_launch();
    k_clusters<<<blocks_for(32 * n_clusters, kBlock), kBlock, 0, st>>>(a, (int)n_clusters); note_launch();
    k_roots<<<blocks_for(32 * (int64_t)N, kBlock), kBlock, 0, st>>>(a); note_launch();
    prof_mark(prof, 1, st);
    // broad phase
    k_pairs<false><<<blocks_for(32 * (int64_t)N, kBlock), kBlock, 0, st>>>(a); note_launch();
    scan(a.ws.pair_cnt, nullptr, N, a.ws.scan_tmp, a.ws.counters + kNPairs, st);
    k_check<<<1, 1, 0, st>>>(a.ws.counters, kNPairs, caps->pair_capacity, RB_STATUS_PAIR_OVERFLOW, out->status); note_launch();
    k_pairs<true><<<blocks_for(32 * (int64_t)N, kBlock), kBlock, 0, st>>>(a); note_launch();
    // mid phase
    {
        const int max_clusters = (sh->max_shape_triangles + 31) / 32;
        const size_t mid_smem = (size_t)kWarpsPerBlock * 3 * sizeof(uint32_t) * (max_clusters > 0 ? max_clusters : 1);
        k_mid<<<mid_blocks, kBlock, mid_smem, st>>>(a, max_clusters > 0 ? max_clusters : 1); note_launch();
    }
    k_check<<<1, 1, 0, st>>>(a.ws.counters, kNItems, caps->item_capacity, RB_STATUS_ITEM_OVERFLOW, out->status); note_launch();
    prof_mark(prof, 2, st);
    // narrow phase
    if (pr->precision != RB_PRECISION_FP64 && sh->grid32) {
        k_narrow<true><<<narrow_blocks, narrow_threads, 0, st>>>(a); note_launch();
    } else {
        k_narrow<false><<<narrow_blocks, narrow_threads, 0, st>>>(a); note_launch();
    }
    prof_mark(prof, 3, st);
    // reduction and compaction
    k_dedup<false><<<G, kBlock, 0, st>>>(a); note_launch();
    scan(a.ws.pair_cont, a.ws.counters + kNPairs, caps->pair_capacity, a.ws.scan_tmp, a.ws.counters + kNContacts, st);
    k_check<<<1, 1, 0, st>>>(a.ws.counters, kNContacts, caps->contact_capacity, RB_STATUS_CONTACT_OVERFLOW, out->status); note_launch();
    k_dedup<true><<<G, kBlock, 0, st>>>(a); note_launch();
    prof_mark(prof, 4, st);
    // contact problem
    k_contacts<<<2 * G, 128, 0, st>>>(a); note_launch();   // a thread per contact row
    if (bd->n_hinges > 0) {   // the hinge problem of every scene that has hinges
        k_hinge_lists<<<blocks_for(bd->n_scenes, 64), 64, 0, st>>>(a); note_launch();
        k_hinges<<<blocks_for(bd->n_hinges, 128), 128, 0, st>>>(a); note_launch();
    }
    k_body_contacts_count<<<G, 256, 0, st>>>(a); note_launch();
    scan(a.ws.bc_ptr, nullptr, N, a.ws.scan_tmp, nullptr, st);
    k_body_contacts_fill<<<G, 256, 0, st>>>(a); note_launch();
    k_preds_init<<<G, 256, 0, st>>>(a); note_launch();
    k_body_contacts_sort<<<blocks_for(N, 128), 128, 0, st>>>(a); note_launch();
    // solve, integrate, post-stabilise
    // small scenes: one warp each with its body accumulators in shared memory; large scenes: one block each
    // a warp per scene only pays off once the scenes alone fill the GPU (>= 32 per SM); otherwise blocks
    const int warp_bodies = bd->n_scenes < 148 * 32 ? 0
                          : (bd->max_scene_bodies < kWarpSceneMaxBodies ? bd->max_scene_bodies : kWarpSceneMaxBodies);
    const size_t warp_smem = (size_t)kSolveWarpsPerBlock * 6 * sizeof(double) * (warp_bodies > 0 ? warp_bodies : 1);
    const int wg = (bd->n_scenes + kSolveWarpsPerBlock - 1) / kSolveWarpsPerBlock;
    const int smem_bodies = bd->max_scene_bodies <= kSolveSmemBodies ? bd->max_scene_bodies : 0;
    const size_t block_smem = (size_t)6 * sizeof(double) * (smem_bodies > 0 ? smem_bodies : 1);
    const int bg = bd->n_scenes < 148 * 16 ? bd->n_scenes : 148 * 16;
    k_fp32_classes<<<1, 1024, 0, st>>>(a, small_slab, mid_slab); note_launch();
    if (pr->precision != RB_PRECISION_FP64) {
        // FP32 phase, four size classes side by side: warp teams with small slabs (28 KB unless tuned), warp
        // teams with mid slabs (56 KB), block teams with 224 KB (1 per SM), and 512-thread block teams for the
        // scenes beyond that, whose contact rows stay in L2
        SideStreams* ss = nullptr;
        rc = side_streams(st, &ss);
        if (rc != RB_OK) return rc;
        cudaEventRecord(ss->fork, st);
        for (int c = 0; c < kSideStreams; ++c) cudaStreamWaitEvent(ss->s[c], ss->fork, 0);
        k_solve_fp32<BlockGroup, true><<<148, kFp32L2Block, (size_t)kFp32LargeSmem, ss->s[3]>>>(
            a, kQueueFp32 + 3, kFp32LargeSmem, kFp32LargeSmem); note_launch();
        k_solve_fp32<BlockGroup, false><<<148, kFp32Block, (size_t)kFp32LargeSmem, ss->s[2]>>>(
            a, kQueueFp32 + 2, mid_slab, kFp32LargeSmem); note_launch();
        // warp teams as one-warp blocks: a team's slab is released as soon as the team finds its queue empty
        // (in blocks of four teams the slowest held all four slabs), so the small class fills the room the mid
        // class leaves; as many blocks per SM as the shared memory (227 KB) allows, up to 32
        const int small_per_sm = std::min(32, (227 * 1024) / small_slab);
        const int mid_per_sm = std::max(1, std::min(32, (227 * 1024) / mid_slab));
        k_solve_fp32<WarpGroup, false><<<148 * mid_per_sm, 32, (size_t)mid_slab, ss->s[1]>>>(
            a, kQueueFp32 + 1, small_slab, mid_slab); note_launch();
        k_solve_fp32<WarpGroup, false><<<148 * small_per_sm, 32, (size_t)small_slab, ss->s[0]>>>(
            a, kQueueFp32, 0, small_slab); note_launch();
        for (int c = 0; c < kSideStreams; ++c) {
            cudaEventRecord(ss->join[c], ss->s[c]);
            cudaStreamWaitEvent(st, ss->join[c], 0);
        }
    }
    if (warp_bodies > 0) { k_solve_warps<<<wg, 32 * kSolveWarpsPerBlock, warp_smem, st>>>(a, 0, warp_bodies); note_launch(); }
    k_solve_blocks<<<bg, kSolveBlock, block_smem, st>>>(a, 0, warp_bodies, smem_bodies); note_launch();
    prof_mark(prof, 5, st);
    k_integrate<<<blocks_for(N, 128), 128, 0, st>>>(a); note_launch();
    if (pr->use_post_stabilization) {
        k_post_setup<<<G, 128, 0, st>>>(a); note_launch();
        if (warp_bodies > 0) { k_solve_warps<<<wg, 32 * kSolveWarpsPerBlock, warp_smem, st>>>(a, 1, warp_bodies); note_launch(); }
        k_solve_blocks<<<bg, kSolveBlock, block_smem, st>>>(a, 1, warp_bodies, smem_bodies); note_launch();
        k_post_apply<<<blocks_for(N, 128), 128, 0, st>>>(a); note_launch();
    }
    if (prof) { k_body_energy<<<blocks_for(N, 128), 128, 0, st>>>(a); note_launch(); }
    k_scene_summary<<<blocks_for(32 * (int64_t)bd->n_scenes, 128), 128, 0, st>>>(a); note_launch();
    k_cache_store<<<G, 256, 0, st>>>(a); note_launch();
    k_finish<<<1, 1, 0, st>>>(a); note_launch();
    prof_mark(prof, 6, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, std::string("rb_step: ") + cudaGetErrorString(e));
    return RB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------
// rb_step_noalloc: the same step with its temporaries in a fixed scratch array of this library
// ---------------------------------------------------------------------------------------------------------
namespace {

// Scratch of rb_step_noalloc.  In host code this name only stands for the array: the kernels receive the
// device address looked up with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[RB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

// device address of the scratch array on the current device, looked up once per device
int noalloc_scratch(void** ptr) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, std::string("rb_step_noalloc: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(RB_ERR_UNSUPPORTED, "rb_step_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(RB_ERR_CUDA, std::string("rb_step_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *ptr = g_noalloc_ptr[dev];
    return RB_OK;
}

}  // namespace

extern "C" {

int rb_step_noalloc(const rb_shapes* sh, const rb_bodies* bd, const rb_caps* caps, const rb_params* pr,
                    const rb_outputs* out, void* stream) {
    if (!sh || !bd || !caps || !pr || !out) return fail(RB_ERR_ARG, "rb_step_noalloc: null argument");
    size_t need = 0;
    int rc = rb_workspace_bytes(bd, caps, &need);
    if (rc != RB_OK) return rc;
    if (need > (size_t)RB_NOALLOC_SCRATCH_BYTES)
        return fail(RB_ERR_WORKSPACE, "rb_step_noalloc: this batch needs " + std::to_string(need) +
                                          " bytes of scratch, more than the " +
                                          std::to_string((size_t)RB_NOALLOC_SCRATCH_BYTES) +
                                          " bytes available; use rb_step with a workspace");
    void* scratch = nullptr;
    rc = noalloc_scratch(&scratch);
    if (rc != RB_OK) return rc;
    // rb_step clears the counters and per-body tallies it needs at the start of every step, so the
    // previous call's contents of the shared array do no harm
    return rb_step(sh, bd, caps, pr, out, scratch, (size_t)RB_NOALLOC_SCRATCH_BYTES, stream);
}

int64_t rb_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int rb_profile_times(float* out, int32_t n) {
    if (!out || n < 7) return fail(RB_ERR_ARG, "rb_profile_times: need room for 7 values");
    if (!g_prof.recorded) return fail(RB_ERR_ARG, "rb_profile_times: no profiled step on this thread");
    cudaError_t e = cudaEventSynchronize(g_prof.ev[6]);
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, std::string("rb_profile_times: ") + cudaGetErrorString(e));
    for (int i = 0; i < 6; ++i) cudaEventElapsedTime(out + i, g_prof.ev[i], g_prof.ev[i + 1]);
    cudaEventElapsedTime(out + 6, g_prof.ev[0], g_prof.ev[6]);
    return RB_OK;
}

}  // extern "C"
