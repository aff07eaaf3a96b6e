// rb_batch.cu -- changing the membership of a resident scene batch (continuous batching).
//
// A serving loop keeps one batch of scenes resident and steps it with rb_step.  Between steps scenes finish
// and new ones are admitted, so the batch is re-laid out: the bodies that stay keep their relative order and
// the new scenes' bodies are appended.  Two entry points do the device side of that:
//   rb_build_topology  derives the per-body topology arrays (vertex / triangle / cluster prefix sums and the
//                      owner of every body-vertex, body-triangle and cluster) from the body-to-shape map, so
//                      the host never materialises per-vertex arrays;
//   rb_repack          moves the state (x, u) of the staying bodies to their new rows and filters and
//                      re-keys the warm-start contact cache, whose keys hold global body indices.
// Neither has a counterpart in the reference, which steps one engine at a time.
#include <cuda_runtime.h>

#include <string>

#include "rainbow_b200.h"
#include "rb_internal.h"

namespace {

inline int fail(int code, const std::string& msg) {
    rb::g_error = msg;
    return code;
}
inline int blocks_for(int64_t n, int block, int cap = 148 * 16) {
    const int64_t b = (n + block - 1) / block;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

// per-body counts of vertices, triangles and 32-triangle clusters (the scans turn them into prefix sums)
__global__ void k_topology_counts(const rb_shapes sh, const rb_bodies bd, int32_t* v0, int32_t* t0, int32_t* c0) {
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < bd.n_bodies; b += gridDim.x * blockDim.x) {
        const int s = bd.shape[b];
        const int nv = sh.v_off[s + 1] - sh.v_off[s];
        const int nt = sh.t_off[s + 1] - sh.t_off[s];
        v0[b] = nv;
        t0[b] = nt;
        c0[b] = (nt + 31) / 32;
    }
}

// owner of every body-vertex, body-triangle and cluster: one warp per body; writes stay inside the totals
// the caller declared, whatever the prefix sums say
__global__ void k_topology_owners(const rb_bodies bd, int32_t* vert_body, int32_t* tri_body, int32_t* clu_body) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < bd.n_bodies; b += warps) {
        const int v1 = min(bd.body_v0[b + 1], bd.n_body_vertices);
        const int t1 = min(bd.body_t0[b + 1], bd.n_body_triangles);
        const int c1 = min(bd.body_c0[b + 1], bd.n_clusters);
        for (int i = bd.body_v0[b] + lane; i < v1; i += 32) vert_body[i] = b;
        for (int i = bd.body_t0[b] + lane; i < t1; i += 32) tri_body[i] = b;
        for (int i = bd.body_c0[b] + lane; i < c1; i += 32) clu_body[i] = b;
    }
}

// state rows of the staying bodies move to their new index
__global__ void k_repack_state(const int32_t* map, int n_old, const double* x_old, const double* u_old,
                               double* x_new, double* u_new) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_old; i += gridDim.x * blockDim.x) {
        const int m = map[i];
        if (m < 0) continue;
        for (int d = 0; d < 7; ++d) x_new[7 * (size_t)m + d] = x_old[7 * (size_t)i + d];
        for (int d = 0; d < 6; ++d) u_new[6 * (size_t)m + d] = u_old[6 * (size_t)i + d];
    }
}

// cache entry i stays when both its bodies stay (they belong to one scene, so they stay or go together)
__global__ void k_cache_keep(const int32_t* map, int n_old, const int64_t* key, const int32_t* count, int capacity,
                             int32_t* keep) {
    const int n = min(*count, capacity);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int64_t k0 = key[2 * (size_t)i];
        const int a = (int)(k0 >> 31), b = (int)(k0 & 0x7fffffff);
        keep[i] = (a < n_old && b < n_old && map[a] >= 0 && map[b] >= 0) ? 1 : 0;
    }
}

// kept entries, re-keyed, to their compacted position (the staying bodies keep their order, so the keys stay
// ascending); entries past the new capacity are dropped
__global__ void k_cache_move(const int32_t* map, const int64_t* key_old, const double* sol_old, const int32_t* count,
                             int capacity_old, const int32_t* pos, int64_t* key_new, double* sol_new,
                             int32_t* count_new, int capacity_new) {
    const int n = min(*count, capacity_old);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = pos[i];
        if (pos[i + 1] == p || p >= capacity_new) continue;   // not kept, or beyond the new capacity
        const int64_t k0 = key_old[2 * (size_t)i];
        const int a = map[(int)(k0 >> 31)], b = map[(int)(k0 & 0x7fffffff)];
        key_new[2 * (size_t)p] = ((int64_t)a << 31) | (int64_t)b;
        key_new[2 * (size_t)p + 1] = key_old[2 * (size_t)i + 1];
        for (int d = 0; d < 4; ++d) sol_new[4 * (size_t)p + d] = sol_old[4 * (size_t)i + d];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *count_new = min(pos[n], capacity_new);
}

}  // namespace

extern "C" {

int rb_build_topology(const rb_shapes* sh, const rb_bodies* bd, void* scratch, size_t scratch_bytes, void* stream) {
    if (!sh || !bd || !scratch) return fail(RB_ERR_ARG, "rb_build_topology: null argument");
    if (scratch_bytes < (size_t)RB_TOPOLOGY_SCRATCH_BYTES)
        return fail(RB_ERR_WORKSPACE, "rb_build_topology: scratch smaller than RB_TOPOLOGY_SCRATCH_BYTES");
    if (bd->n_bodies <= 0 || !bd->shape || !bd->body_v0 || !bd->body_t0 || !bd->body_c0 || !bd->vert_body ||
        !bd->tri_body || !bd->clu_body)
        return fail(RB_ERR_ARG, "rb_build_topology: missing body arrays");
    cudaStream_t st = (cudaStream_t)stream;
    int32_t* v0 = const_cast<int32_t*>(bd->body_v0);
    int32_t* t0 = const_cast<int32_t*>(bd->body_t0);
    int32_t* c0 = const_cast<int32_t*>(bd->body_c0);
    int32_t* partial = static_cast<int32_t*>(scratch);
    const int N = bd->n_bodies;
    k_topology_counts<<<blocks_for(N, 256), 256, 0, st>>>(*sh, *bd, v0, t0, c0);
    rb::note_launch();
    rb::scan(v0, nullptr, N, partial, nullptr, st);
    rb::scan(t0, nullptr, N, partial, nullptr, st);
    rb::scan(c0, nullptr, N, partial, nullptr, st);
    k_topology_owners<<<blocks_for(32 * (int64_t)N, 256), 256, 0, st>>>(*bd, const_cast<int32_t*>(bd->vert_body),
                                                                       const_cast<int32_t*>(bd->tri_body),
                                                                       const_cast<int32_t*>(bd->clu_body));
    rb::note_launch();
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, std::string("rb_build_topology: ") + cudaGetErrorString(e));
    return RB_OK;
}

int rb_repack_workspace_bytes(int32_t cache_capacity_old, size_t* bytes) {
    if (!bytes || cache_capacity_old < 0) return fail(RB_ERR_ARG, "rb_repack_workspace_bytes: bad argument");
    *bytes = sizeof(int32_t) * ((size_t)cache_capacity_old + 1 + rb::kScanPartials);
    return RB_OK;
}

int rb_repack(const int32_t* body_map, int32_t n_old_bodies, const double* x_old, const double* u_old, double* x_new,
              double* u_new, const int64_t* cache_key_old, const double* cache_sol_old,
              const int32_t* cache_count_old, int32_t cache_capacity_old, int64_t* cache_key_new,
              double* cache_sol_new, int32_t* cache_count_new, int32_t cache_capacity_new, void* workspace,
              size_t workspace_bytes, void* stream) {
    if (!body_map || n_old_bodies < 0 || !x_old || !u_old || !x_new || !u_new)
        return fail(RB_ERR_ARG, "rb_repack: null state argument");
    const bool cache = cache_key_old != nullptr;
    if (cache && (!cache_sol_old || !cache_count_old || !cache_key_new || !cache_sol_new || !cache_count_new ||
                  cache_capacity_old < 0 || cache_capacity_new < 0))
        return fail(RB_ERR_ARG, "rb_repack: incomplete cache arguments");
    cudaStream_t st = (cudaStream_t)stream;
    if (n_old_bodies > 0) {
        k_repack_state<<<blocks_for(n_old_bodies, 256), 256, 0, st>>>(body_map, n_old_bodies, x_old, u_old, x_new,
                                                                      u_new);
        rb::note_launch();
    }
    if (cache) {
        size_t need = 0;
        rb_repack_workspace_bytes(cache_capacity_old, &need);
        if (!workspace || workspace_bytes < need) return fail(RB_ERR_WORKSPACE, "rb_repack: workspace too small");
        int32_t* keep = static_cast<int32_t*>(workspace);
        int32_t* partial = keep + cache_capacity_old + 1;
        const int G = blocks_for(cache_capacity_old, 256);
        k_cache_keep<<<G, 256, 0, st>>>(body_map, n_old_bodies, cache_key_old, cache_count_old, cache_capacity_old,
                                         keep);
        rb::note_launch();
        rb::scan(keep, cache_count_old, cache_capacity_old, partial, nullptr, st);
        k_cache_move<<<G, 256, 0, st>>>(body_map, cache_key_old, cache_sol_old, cache_count_old, cache_capacity_old,
                                         keep, cache_key_new, cache_sol_new, cache_count_new, cache_capacity_new);
        rb::note_launch();
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(RB_ERR_CUDA, std::string("rb_repack: ") + cudaGetErrorString(e));
    return RB_OK;
}

}  // extern "C"
