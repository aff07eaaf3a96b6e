/*
 * rainbow_b200.h -- C ABI of the B200 (sm_100a) implementation of RAINBOW's prox_rigid_bodies time step.
 *
 * The reference step is the Python call chain
 *     rainbow/simulators/prox_rigid_bodies/api.py:676 simulate(engine, T)
 *       -> steppers.py:47 SemiImplicitStepper.step(dt, engine, profiling_on)
 * A Python engine drives this library through ctypes (rainbow_b200/stepper.py, GpuStepper).  Every pointer
 * inside the structs below is a DEVICE pointer owned by the caller (torch tensors in the Python host); the
 * structs themselves live in host memory and are read during the call.  No entry point allocates device
 * memory: per-step temporaries live in a caller-provided workspace of rb_workspace_bytes() bytes.
 *
 * All entry points return RB_OK (0) or a positive RB_ERR_* code; rb_last_error() describes the last failure
 * of the calling thread.  Launch-time failures are reported synchronously; conditions only known on the
 * device (capacity overflow, non-finite state, a solver that gave up) are written to rb_outputs.status and
 * to the per-scene statistics, which the caller reads after synchronising the stream.
 */
#ifndef RAINBOW_B200_H
#define RAINBOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RB_ABI_VERSION 2

/* return codes */
#define RB_OK 0
#define RB_ERR_ARG 1          /* a null pointer, a negative size or an inconsistent descriptor */
#define RB_ERR_CUDA 2         /* a CUDA launch or API call failed */
#define RB_ERR_WORKSPACE 3    /* workspace too small for the requested capacities */
#define RB_ERR_UNSUPPORTED 4  /* a parameter combination this build does not implement */

/* device status bits (rb_outputs.status[0]) */
#define RB_STATUS_PAIR_OVERFLOW 1
#define RB_STATUS_ITEM_OVERFLOW 2
#define RB_STATUS_CONTACT_OVERFLOW 4
#define RB_STATUS_NONFINITE 8
#define RB_STATUS_NONUNIT_NORMAL 16
#define RB_STATUS_MESH_TOO_LARGE 32   /* a shape has more than 16384 triangles */

/* solver schemes (engine.params.proximal_solver) */
#define RB_SCHEME_RIGID_GS 0          /* gauss_seidel_solver.py:14 + contacts.py:66 (the reference stepper) */
#define RB_SCHEME_GS 1                /* proximal_contact/gauss_seidel_solver.py:8 GaussSeidelSolver */
#define RB_SCHEME_JACOBI 2            /* proximal_contact/jacobi_solver.py:41 ParallelJacobiSolver */
#define RB_SCHEME_JACOBI_HYBRID 3     /* proximal_contact/jacobi_solver.py:60 ParallelJacobiHybridSolver */
#define RB_SCHEME_COLOURED_GS 4       /* graph-coloured Gauss-Seidel (proximal_contact/gauss_seidel_solver.py:89
                                         ParallelGaussSeidelSolver): the RB_SCHEME_GS rules swept in RB_ORDER_COLOURED */

/* termination rules */
#define RB_TERMINATE_MERIT 0          /* the reference's iterate-change merit (problem.py:53) */
/* complementarity residual: ||x - prox(x - D^-1 (A x + b))||_inf / max(1, ||x||_inf), D = diag(A), A = J W J^T */
#define RB_TERMINATE_RESIDUAL 1       /* complementarity residual <= residual_tolerance; the reference's merit
                                         rule still rejects iterates and adapts r */
#define RB_TERMINATE_RESIDUAL_FIXED_R 2 /* complementarity residual <= residual_tolerance; every sweep is
                                         accepted and r stays at its initial value */

/* solver precision */
#define RB_ORDER_SERIAL 0             /* ascending contact order, as the reference sweeps (contacts.py:74) */
#define RB_ORDER_COLOURED 1           /* colour by colour: contacts that share no non-fixed body form a colour
                                         (deterministic Jones-Plassmann colouring with hashed priorities); the
                                         order RB_SCHEME_COLOURED_GS always uses */

#define RB_PRECISION_FP64 0           /* every sweep in FP64 (bit-exact with the reference's NumPy step) */
#define RB_PRECISION_FP32_REFINE 1    /* sweeps in FP32 on chip until the residual tolerance, then FP64 sweeps until
                                         the FP64 residual meets it */
#define RB_PRECISION_FP32 2           /* FP32 sweeps only; the FP64 residual of the result is reported */

/* Shapes (rainbow/simulators/prox_rigid_bodies/types.py:82 Shape): body-frame mesh and signed distance grid. */
typedef struct rb_shapes {
    int32_t n_shapes;
    const double* V;            /* 3 doubles per vertex, body frame (api.py:228-230) */
    const int32_t* v_off;       /* n_shapes+1 vertex offsets */
    const int32_t* T;           /* 3 shape-local vertex indices per triangle */
    const int32_t* t_off;       /* n_shapes+1 triangle offsets */
    const double* grid;         /* SDF node values, index i + I*(j + J*k) (grid3.py:71) */
    const int64_t* g_off;       /* n_shapes+1 value offsets */
    const double* grid_meta;    /* 12 doubles per shape: min[3], max[3], spacing[3], I, J, K (grid3.py:16) */
    int32_t max_shape_triangles; /* triangles of the largest shape (at most 16384) */
    const float* grid32;        /* optional FP32 copy of grid (same offsets), or NULL.  With it, the FP32
                                   precision modes run the contact search's signed distance lookups (the seed
                                   and Frank-Wolfe iterations, collision_detection.py:134-165) in FP32; the
                                   acceptance tests and the contact's point, normal and gap (:172-188) stay
                                   FP64, evaluated at the point the FP32 search found */
} rb_shapes;

/* Bodies of one or more independent scenes; scene s owns bodies scene_start[s] .. scene_start[s+1]-1 in the
   reference's body order (engine.bodies insertion order = RigidBody.idx, api.py:67). */
typedef struct rb_bodies {
    int32_t n_bodies;
    int32_t n_scenes;
    const int32_t* scene_start;   /* n_scenes+1 */
    const int32_t* shape;         /* shape index per body */
    const double* mass;           /* types.py:111 RigidBody.mass */
    const double* inertia;        /* 3 per body: body-frame principal inertia */
    const uint8_t* fixed;         /* RigidBody.is_fixed */
    const int32_t* material;      /* material index per body */
    const int32_t* force_ptr;     /* n_bodies+1: connected forces per body (api.py:331 connect_force order) */
    const int32_t* force_list;    /* global force indices */
    int32_t n_forces;
    const int32_t* scene_force_start; /* n_scenes+1: scene s owns forces scene_force_start[s].. (engine.forces) */
    const int32_t* force_kind;    /* 0 = Gravity (types.py:189), 1 = Damping (types.py:224) */
    const double* force_params;   /* 4 per force: gravity (g, up[3]); damping (alpha, beta, 0, 0) */
    /* materials: body material indices are local to the scene; scene s owns an M_s x M_s interaction table
       starting at entry scene_material_offset[s] (SurfacesInteractionLibrary.get_interaction, types.py:42) */
    const int32_t* scene_material_offset;
    const int32_t* scene_material_count;
    const double* material_mu;    /* 3 per table entry: SurfacesInteraction.mu */
    const double* material_eps;   /* 1 per table entry: SurfacesInteraction.epsilon */
    /* topology derived from the shapes, fixed for the life of the scene (see rb_topology_sizes) */
    int32_t n_body_vertices;      /* sum over bodies of their shape's vertex count */
    int32_t n_body_triangles;     /* sum over bodies of their shape's triangle count */
    int32_t n_clusters;           /* sum over bodies of ceil(triangles / 32) */
    int32_t max_scene_bodies;     /* bodies of the largest scene (sizes the solver's on-chip body arrays) */
    const int32_t* body_v0;       /* n_bodies+1 prefix sums of per-body vertex counts */
    const int32_t* body_t0;       /* n_bodies+1 prefix sums of per-body triangle counts */
    const int32_t* body_c0;       /* n_bodies+1 prefix sums of per-body 32-triangle cluster counts */
    const int32_t* vert_body;     /* owning body of each body-vertex */
    const int32_t* tri_body;      /* owning body of each body-triangle */
    const int32_t* clu_body;      /* owning body of each cluster */
    /* state, read at the start and written at the end of a step (state_storage.py:43-68 layout) */
    double* x;                    /* 7 per body: r[3], q[4] */
    double* u;                    /* 6 per body: v[3], w[3] */
    /* hinge joints (types.py:304 Hinge, constraints/hinges.py); scene s owns hinges scene_hinge_start[s] ..
       scene_hinge_start[s+1]-1 in Hinge.idx order.  They are solved with the reference stepper's rule only
       (RB_SCHEME_RIGID_GS, RB_TERMINATE_MERIT, RB_ORDER_SERIAL, RB_PRECISION_FP64); other settings are
       rejected with RB_ERR_UNSUPPORTED for batches that hold hinges */
    int32_t n_hinges;
    const int32_t* scene_hinge_start; /* n_scenes+1 (may be NULL when n_hinges == 0) */
    const int32_t* hinge_bodies;  /* 2 per hinge: parent, child (global body indices) */
    const double* hinge_frames;   /* 12 per hinge: arm_p[3], arm_c[3], axis_p[3], axis_c[3] in the parent's and
                                     the child's body frames (Hinge.arm_p, .arm_c, .axis_p, .axis_c) */
} rb_bodies;

/* Capacities of the per-step work lists.  Exceeding one sets a status bit; the step then leaves x and u
   untouched so the caller can grow the workspace and repeat it. */
typedef struct rb_caps {
    int32_t pair_capacity;        /* body pairs whose bounding boxes overlap */
    int32_t item_capacity;        /* candidate triangles sent to the Frank-Wolfe search */
    int32_t contact_capacity;     /* contacts before duplicate removal */
    int32_t max_iterations;       /* solver iteration cap (length of each scene's residual history) */
} rb_caps;

/* Parameters (types.py:356 Parameters) plus the solver options of this implementation. */
typedef struct rb_params {
    double dt;
    int32_t max_iterations;
    int32_t use_bounce;
    int32_t use_pre_stabilization;
    int32_t use_post_stabilization;
    double gap_reduction;
    double min_gap_value;
    double max_gap_value;
    double absolute_tolerance;
    double relative_tolerance;
    double nu_reduce;
    double nu_increase;
    double too_small_merit_change;
    int32_t contact_optimization_max_iterations;
    double contact_optimization_tolerance;
    double envelope;
    int32_t scheme;               /* RB_SCHEME_* */
    int32_t termination;          /* RB_TERMINATE_* */
    double residual_tolerance;    /* used by RB_TERMINATE_RESIDUAL */
    int32_t profiling;            /* nonzero: phase times, energies and residual histories; bit 2 (value 2) also
                                     checks the FP32 modes' contact search against the plain FP64 search
                                     (rb_scene_stats.n_search_flips / n_accept_flips) */
    double relaxation;            /* RB_TERMINATE_RESIDUAL_FIXED_R: r = relaxation / diag (over-relaxation of the
                                     projected Gauss-Seidel update; values <= 0 mean 1) */
    int32_t residual_interval;    /* RB_TERMINATE_RESIDUAL_FIXED_R: test the residual every this many sweeps
                                     (values below 1 mean every sweep); the other rules test every sweep */
    int32_t precision;            /* RB_PRECISION_*; the FP32 modes need RB_TERMINATE_RESIDUAL_FIXED_R and a
                                     Gauss-Seidel scheme */
    int32_t refine_iterations;    /* RB_PRECISION_FP32_REFINE: FP64 sweeps reserved after the FP32 phase (0 to
                                     max_iterations).  The FP32 phase sweeps until its residual meets the
                                     tolerance, stalls below 1e-5, or max_iterations - refine_iterations sweeps
                                     are done; the FP64 refinement then gets the sweeps left of max_iterations.
                                     The residual of the result is always evaluated in FP64 */
    int32_t warm_start;           /* nonzero: start each contact's impulse from the previous step's solution for
                                     the same (body pair, side, triangle) found in rb_outputs.cache_*; the
                                     reference always starts from zero (contacts.py:53), so this is off for
                                     parity runs */
    int32_t ordering;             /* RB_ORDER_*: contact visiting order of the Gauss-Seidel schemes */
    /* launch shapes (0 = built-in value); they change speed only, never results */
    int32_t fp32_small_slab;      /* bytes of a warp team's slab in the FP32 solve's small class (28672);
                                     multiple of 16, 4096 .. fp32_mid_slab - 16 */
    int32_t fp32_mid_slab;        /* bytes of a warp team's slab in the mid class (57344), at most 57344 */
    int32_t mid_blocks;           /* blocks of the triangle-candidate search (2368) */
    int32_t narrow_blocks;        /* blocks of the Frank-Wolfe contact search (1184) */
    int32_t narrow_threads;       /* threads per contact-search block: 64, 128 or 256 (256) */
} rb_params;

/* Per-scene results of one step. */
typedef struct rb_scene_stats {
    int32_t n_contacts;           /* after duplicate removal (collision_detection.py:255) */
    int32_t contact_start;        /* first contact of this scene in the contact outputs */
    int32_t iterations;           /* gauss_seidel_solver.py:471-489 'iterations' */
    int32_t exitcode;             /* 0 not converged, 1 absolute, 2 relative, 3 residual */
    int32_t post_iterations;
    int32_t post_exitcode;
    int32_t n_pairs;              /* body pairs with overlapping bounding boxes */
    int32_t n_candidates;         /* triangles searched (profiling only) */
    int32_t n_leaf_overlaps;      /* overlapping leaf (triangle) pairs: profile key number_of_overlaps (profiling only) */
    int32_t n_grid_lookups;       /* signed distance lookups of the contact search (profiling only) */
    int32_t n_levels;             /* Gauss-Seidel wavefront levels of the scene's contact order */
    int32_t fp32_sweeps;          /* sweeps done in FP32 (FP32 precision modes; included in iterations) */
    double merit;                 /* last global merit */
    double residual;              /* complementarity residual of the returned solution (when computed) */
    double kinetic_energy;        /* state_storage.py:188 (profiling only) */
    double potential_energy;
    double max_penetration;       /* contacts.py:222 */
    double solve_start_us;        /* device clock (%globaltimer, microseconds) when the scene's solve started (profiling only) */
    double solve_us;              /* device time of the scene's contact solve, FP32 and FP64 phases (profiling only) */
    int32_t n_search_flips;       /* FP32 contact search (profiling bit 2): candidates whose seed, Frank-Wolfe vertex
                                     choices or iteration count differ from the FP64 search's */
    int32_t n_accept_flips;       /* ... candidates the FP32 search accepts as a contact and the FP64 search does
                                     not, or the other way round */
    int32_t n_grid_lookups32;     /* signed distance lookups of the contact search made on grid32 (profiling only;
                                     n_grid_lookups counts the FP64 ones) */
} rb_scene_stats;

/* Outputs: device buffers sized by rb_caps.contact_capacity / n_scenes / max_iterations. */
typedef struct rb_outputs {
    int32_t* contact_ids;         /* 2 per contact: bodyA (SDF owner), bodyB (mesh owner), global body indices */
    double* contact_p;            /* 3 per contact, world frame */
    double* contact_n;            /* 3 per contact, unit normal */
    double* contact_g;            /* gap (SDF value) */
    double* contact_sol;          /* 4 per contact: solver result (n, s, t, tau impulses) */
    rb_scene_stats* stats;        /* n_scenes */
    double* residuals;            /* n_scenes * max_iterations (profiling), may be NULL */
    int32_t* status;              /* 1 int32: RB_STATUS_* bits, OR-ed by the step (caller zeroes it) */
    int32_t* n_contacts_total;    /* 1 int32 */
    int32_t* needed;              /* 3 int32: body pairs, candidates and contacts the step produced (a stage
                                     after an overflow reports 0); used to size the capacities */
    /* contact cache carried from step to step for warm starting (capacity rb_caps.contact_capacity): keys
       (lower body index << 31 | higher body index, side << 30 | triangle) in ascending order and the 4
       impulses per contact.  Read when params->warm_start is set, always rewritten at the end of a step.
       Set *cache_count = 0 when the scene batch changes. */
    int64_t* cache_key;           /* 2 per contact */
    double* cache_sol;            /* 4 per contact */
    int32_t* cache_count;         /* 1 int32 */
    double* hinge_sol;            /* 5 per hinge: the hinge problem's solution (hinges.py:52), or NULL */
} rb_outputs;

/* Library ABI version (RB_ABI_VERSION). */
int rb_abi_version(void);

/* Description of the last error on the calling thread. */
const char* rb_last_error(void);

/* Sizes of the derived topology arrays of rb_bodies for the given per-body shape assignment (host arrays):
   out[0] = total body-vertices, out[1] = total body-triangles, out[2] = total clusters. */
int rb_topology_sizes(int32_t n_bodies, const int32_t* body_shape_host, int32_t n_shapes,
                      const int32_t* v_off_host, const int32_t* t_off_host, int64_t* out);

/* Workspace bytes needed by rb_step for these bodies and capacities.
   Replaces the host-side temporaries the reference builds each step (state_storage.py:43, contacts.py:31). */
int rb_workspace_bytes(const rb_bodies* bodies, const rb_caps* caps, size_t* bytes);

/* One semi-implicit time step of every scene in `bodies` on `stream` (a cudaStream_t, NULL = default).
   Replaces steppers.py:47 SemiImplicitStepper.step: forces and inverse mass (state_storage.py:43), collision
   detection (collision_detection.py:293), contact problem (contacts.py:31), proximal solve
   (gauss_seidel_solver.py:14 or the proximal_contact scheme in params->scheme), velocity and position update
   (state_storage.py:239-302) and optional post-stabilisation (steppers.py:15).  Asynchronous. */
int rb_step(const rb_shapes* shapes, const rb_bodies* bodies, const rb_caps* caps, const rb_params* params,
            const rb_outputs* out, void* workspace, size_t workspace_bytes, void* stream);

/* Phase times (milliseconds) of the last rb_step issued with params->profiling on this thread, after waiting
   for it: out[0] bounding volumes (steppers.py 'update_bvh'), out[1] body pairs and triangle candidates
   ('narrow_phase'), out[2] Frank-Wolfe contact search ('contact_determination'), out[3] duplicate removal
   ('contact_point_reduction'), out[4] contact problem set-up and solve ('solver_time'), out[5] integration and
   post-stabilisation, out[6] the whole step.  Returns RB_ERR_ARG if no profiled step was issued. */
int rb_profile_times(float* out, int32_t n);

/* Number of kernels this library has launched in this process so far (every entry point, all threads and
   devices).  Callers take the difference around a region to count the device work it issued.  It has no
   counterpart in the reference. */
int64_t rb_launch_count(void);

/* rb_step without a workspace argument, for callers that cannot allocate device memory themselves -- for
   example a host application that owns every device allocation through its own fixed pool, or a real-time
   loop that must not call into an allocator once it runs.  The per-step temporaries live in a scratch array
   that this library keeps in device global memory, RB_NOALLOC_SCRATCH_BYTES (16 MiB) on every device that
   loads the library, held until the process exits.  Batches whose rb_workspace_bytes() exceeds that size are
   rejected with RB_ERR_WORKSPACE.  The first call on a device looks up the array's device address (with that
   device current) and, like the first rb_step on that device, grants the solver kernels their shared memory;
   the first FP32-precision step on each host thread and device also creates that thread's side streams and
   events.  Make those first calls during warm-up, outside any stream capture.  The address is kept for the
   life of the process: after a cudaDeviceReset the array may move, so do not use this entry point across a
   device reset.  All calls share the one array: calls that may overlap on the GPU (different streams, or
   different host threads) race and must be serialised by the caller.  This entry point calls no allocator.
   It has no counterpart in the reference. */
#define RB_NOALLOC_SCRATCH_BYTES (16u << 20)
int rb_step_noalloc(const rb_shapes* shapes, const rb_bodies* bodies, const rb_caps* caps, const rb_params* params,
                    const rb_outputs* out, void* stream);

/* ---- continuous batching: re-laying out a resident batch between steps (no reference counterpart; the
   reference steps one engine at a time) ---- */

/* Derived topology arrays of `bodies` (body_v0, body_t0, body_c0, vert_body, tri_body, clu_body, written
   through the struct's pointers) from bodies->shape and the shape table, on the device and on `stream`.
   bodies->n_body_vertices / n_body_triangles / n_clusters must hold the totals (rb_topology_sizes) and the
   arrays must have room for them; no owner entry is written past a declared total.  `scratch` is device
   memory of at least RB_TOPOLOGY_SCRATCH_BYTES. */
#define RB_TOPOLOGY_SCRATCH_BYTES 4096u
int rb_build_topology(const rb_shapes* shapes, const rb_bodies* bodies, void* scratch, size_t scratch_bytes,
                      void* stream);

/* Device workspace bytes rb_repack needs for a warm-start cache of the given capacity. */
int rb_repack_workspace_bytes(int32_t cache_capacity_old, size_t* bytes);

/* Carries a batch's state into its next layout, on `stream`.  body_map[i] (device, n_old_bodies entries) is
   the new index of old body i, or -1 when its scene leaves; the bodies that stay must keep their relative
   order (new scenes are appended after them).  Rows x[7], u[6] of the staying bodies are copied from
   x_old/u_old to x_new/u_new (distinct buffers); rows of new bodies are left for the caller to fill.  When
   cache_key_old is not NULL the warm-start cache (rb_outputs.cache_*) is filtered to the staying scenes and
   re-keyed with the new body indices into cache_*_new, keeping ascending key order; entries past
   cache_capacity_new are dropped.  `workspace`: rb_repack_workspace_bytes(cache_capacity_old) bytes. */
int rb_repack(const int32_t* body_map, int32_t n_old_bodies, const double* x_old, const double* u_old, double* x_new,
              double* u_new, const int64_t* cache_key_old, const double* cache_sol_old,
              const int32_t* cache_count_old, int32_t cache_capacity_old, int64_t* cache_key_new,
              double* cache_sol_new, int32_t* cache_count_new, int32_t cache_capacity_new, void* workspace,
              size_t workspace_bytes, void* stream);

/* Signed distance grid of a closed triangle mesh (replaces grid3.py:320 create_signed_distance's call to
   igl.signed_distance at grid3.py:338): values[i + I*(j + J*k)] for nodes min + spacing*(i,j,k).
   Unsigned distance by closest point on each triangle, sign by the generalized winding number. */
int rb_signed_distance_grid(const double* V, int32_t n_vertices, const int32_t* T, int32_t n_triangles,
                            const double* grid_meta, double* values, void* stream);

/* The grids of many shapes in one launch (grid3.py:320 create_signed_distance once per shape, for batches that
   give every body a shape of its own).  Shape s: vertices V[3 v_off[s] ..], triangles T[3 t_off[s] ..] with
   shape-local vertex indices, grid_meta[12 s ..] as above, values[g_off[s] ..].  block_off (n_shapes + 1) holds
   the prefix sums of ceil(I J K / 128) over the shapes, block_off[0] = 0, and total_blocks = block_off[n_shapes].
   Every pointer is a device pointer; the values equal rb_signed_distance_grid's, shape by shape.  Asynchronous. */
int rb_signed_distance_grids(int32_t n_shapes, const double* V, const int32_t* v_off, const int32_t* T,
                             const int32_t* t_off, const double* grid_meta, const int64_t* g_off,
                             const int64_t* block_off, int64_t total_blocks, double* values, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* RAINBOW_B200_H */
