// rb_layout.h -- carving of the caller-provided workspace into the per-step arrays.
#pragma once
#include <cstddef>
#include <cstdint>
#include <type_traits>

#include "rainbow_b200.h"

namespace rb {

constexpr int kMaxClustersPerShape = 512;   // 16384 triangles per shape (mid-phase cluster masks in shared memory)
constexpr int kScanBlocks = 1024;           // partial sums of the device-wide scans
// Strides of the compact FP32 records.  A contact record (12 floats per row, 4 rows) is padded to an odd
// number of float4s (13), so the 128-bit row loads of eight lanes reading eight different contacts fall on
// eight different groups of four shared-memory banks (with 12 float4s every other contact shared its banks:
// 4-way conflicts once a level holds several contacts).  Body records (w, m^-1, fixed, I^-1) are read two
// per contact and often the same body by several lanes; padding them did not pay.
constexpr int kS32Floats = 52;               // floats per contact record (48 used)
constexpr int kS32BodyFloats = 16;           // floats per body record

struct Workspace {
    // per body
    double* Winv;        // 9N world-frame inverse inertia
    double* dux;         // 6N  W f_ext
    double* du;          // 6N  velocity change of the step
    double* root;        // 6N  body bounding box (lo, hi)
    double* w;           // 6N  WJT x accumulator of the solver
    double* w2;          // 6N  second accumulator (Jacobi / residual)
    int32_t* pair_cnt;   // N+1 overlapping pairs per body -> offsets
    int32_t* bc_ptr;     // N+1 contacts per body -> offsets
    int32_t* bc_fill;    // N
    // per body-vertex / triangle / cluster
    double* Vw;          // 3 NV world vertices
    double* clu;         // 6 NC cluster boxes
    // pairs
    int32_t* pairs;      // 2P
    int32_t* pair_items; // P+1 candidate triangles per pair -> offsets
    int32_t* pair_itemsA;// P   of which from side A
    int32_t* pair_cont;  // P+1 contacts per pair -> offsets
    int32_t* pair_ovl;   // P   overlapping leaf pairs per pair (profiling statistic)
    // items
    int32_t* item_pair;  // C
    int32_t* item_tri;   // C  side << 31 | triangle
    int32_t* item_flag;  // C
    double* item_p;      // 3C
    double* item_n;      // 3C
    double* item_g;      // C
    // contacts
    int32_t* lohi;       // 2K
    int32_t* c_scene;    // K
    int32_t* bc_list;    // 2K
    double* J;           // 48K
    double* WJT;         // 48K
    float* c32;          // 52K   compact FP32 contacts of the scenes whose copy does not fit in shared memory
    uint32_t* blist32;   // 2K    ... their per-body contact lists
    uint16_t* pos32;     // K     ... and level-order positions
    float* body32;       // 16N   ... and, for scenes with too many bodies for the slab, their body records
    double* b;           // 4K
    double* diag;        // 4K
    double* r;           // 4K
    double* x;           // 4K
    double* xold;        // 4K
    double* mu;          // K
    int64_t* ckey;       // 2K  contact keys (pair, side << 30 | triangle)
    int32_t* lev_of;     // K   Gauss-Seidel level of each contact
    int32_t* lev_order;  // K   contacts sorted by level (per scene)
    int32_t* lev_ptr;    // K + S + 1 level boundaries (per scene)
    int32_t* lev_cur;    // K + S + 1 scatter cursors
    int32_t* cpred;      // 2K  previous contact on the same (non-fixed) body, per side, or -1
    int32_t* sweeps32;   // S   FP32 sweeps done per scene (-1: the scene is solved in FP64 only)
    int32_t* nlev;       // S   levels (or colours) the FP32 phase found for the scene
    int32_t* fin32;      // S   1 when the FP32 phase finished the scene (no FP64 sweeps needed)
    int32_t* list32;     // S   the FP32 phase's scenes by size class, larger contact counts first
    double* eterm;       // 2N  kinetic and potential energy of each body (profiled steps)
    // hinge joints (H of them): J and W J^T blocks (5 rows x 12), b, diag, r, x, sol, body pairs (ascending),
    // level order and starts per scene, per-body hinge lists, the hinge problem's own accumulators w
    double *hJ, *hWJT, *hb, *hdiag, *hr, *hx, *hsol, *hw;
    int32_t *hlohi, *hlev, *hlev_order, *hlev_ptr, *hbody_ptr, *hbody_list, *hlast;
    // scans and counters
    int32_t* scan_tmp;   // kScanBlocks + 1
    int32_t* counters;   // 16
};

enum Counter { kNPairs = 0, kNItems = 1, kNRaw = 2, kNContacts = 3, kMidNext = 4 };

inline size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

// Computes (and, when base != nullptr, assigns) every array; returns the total bytes.
inline size_t layout(Workspace* ws, char* base, int64_t N, int64_t NV, int64_t NT, int64_t NC, int64_t P,
                     int64_t C, int64_t K, int64_t S, int64_t H) {
    size_t off = 0;
    auto take = [&](auto*& ptr, int64_t count) {
        using T = std::remove_reference_t<decltype(*ptr)>;
        size_t bytes = align_up(sizeof(T) * (size_t)(count > 0 ? count : 1));
        if (base) ptr = reinterpret_cast<T*>(base + off);
        off += bytes;
    };
    Workspace dummy;
    Workspace* w = ws ? ws : &dummy;
    take(w->Winv, 9 * N); take(w->dux, 6 * N); take(w->du, 6 * N); take(w->root, 6 * N);
    take(w->w, 6 * N); take(w->w2, 6 * N);
    take(w->pair_cnt, N + 1); take(w->bc_ptr, N + 1); take(w->bc_fill, N);
    take(w->Vw, 3 * NV); take(w->clu, 6 * NC);
    take(w->pairs, 2 * P); take(w->pair_items, P + 1); take(w->pair_itemsA, P); take(w->pair_cont, P + 1); take(w->pair_ovl, P);
    take(w->item_pair, C); take(w->item_tri, C); take(w->item_flag, C);
    take(w->item_p, 3 * C); take(w->item_n, 3 * C); take(w->item_g, C);
    take(w->lohi, 2 * K); take(w->c_scene, K); take(w->bc_list, 2 * K);
    take(w->J, 48 * K); take(w->WJT, 48 * K); take(w->c32, (size_t)kS32Floats * K); take(w->blist32, 2 * K); take(w->pos32, K);
    take(w->body32, (size_t)kS32BodyFloats * N);
    take(w->b, 4 * K); take(w->diag, 4 * K); take(w->r, 4 * K); take(w->x, 4 * K); take(w->xold, 4 * K);
    take(w->mu, K);
    take(w->ckey, 2 * K);
    take(w->lev_of, K); take(w->lev_order, K); take(w->lev_ptr, K + S + 1); take(w->lev_cur, K + S + 1);
    take(w->cpred, 2 * K);
    take(w->sweeps32, S); take(w->nlev, S); take(w->fin32, S); take(w->list32, S); take(w->eterm, 2 * N);
    take(w->hJ, 60 * H); take(w->hWJT, 60 * H); take(w->hb, 5 * H); take(w->hdiag, 5 * H); take(w->hr, 5 * H);
    take(w->hx, 5 * H); take(w->hsol, 5 * H); take(w->hlohi, 2 * H); take(w->hlev_order, H);
    take(w->hlev_ptr, H + S + 1); take(w->hbody_ptr, N + 1); take(w->hbody_list, 2 * H); take(w->hw, 6 * N);
    take(w->hlast, N); take(w->hlev, H);
    take(w->scan_tmp, kScanBlocks + 1); take(w->counters, 16);
    return off;
}

}  // namespace rb
