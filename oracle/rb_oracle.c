/*
 * rb_oracle.c -- CPU restatement of RAINBOW's prox_rigid_bodies semi-implicit time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle for the CUDA implementation in
 * rainbow_b200/csrc.  Only the tests, the smoke check and the CPU-baseline leg of bench.py load it; the
 * product path never links or calls it.
 *
 * Every function restates the reference file:line it cites (paths relative to the RAINBOW checkout).
 * Floating-point operation order follows what NumPy / SciPy execute for the reference's Python:
 *   - np.dot / np.linalg.norm on 3- and 4-vectors go through OpenBLAS ddot, which evaluates a chain of
 *     fused multiply-adds: fma(a2,b2, fma(a1,b1, a0*b0))  (measured against NumPy 2.3.5 / OpenBLAS 0.3.30);
 *   - np.dot(3x3 matrix, 3-vector) goes through OpenBLAS dgemv: row i = fma(m_i2,v2, fma(m_i0,v0, m_i1*v1));
 *   - elementwise ufunc arithmetic and Python float arithmetic round after every operation (no fusion);
 *   - SciPy sparse mat-vec / mat-mat products accumulate sequentially in ascending column order starting
 *     from 0.0 (sparsetools csr_matvec, bsr_matvec, bsr_matmat).
 * Build with -ffp-contract=off so that the compiler fuses nothing beyond the explicit fma() calls.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------------------ */
/* NumPy-faithful small-vector helpers                                                                     */
/* ------------------------------------------------------------------------------------------------------ */
static inline double dot3_np(const double* a, const double* b) { return fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0])); }
static inline double dot4_np(const double* a, const double* b) {
    return fma(a[3], b[3], fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0])));
}
static inline double norm3_np(const double* a) { return sqrt(dot3_np(a, a)); }
static inline double norm4_np(const double* a) { return sqrt(dot4_np(a, a)); }
/* np.cross for 3-vectors (numpy/_core/numeric.py cross: cp0 = a1*b2 - a2*b1, ...) */
static inline void cross_np(const double* a, const double* b, double* c) {
    double c0 = a[1] * b[2] - a[2] * b[1];
    double c1 = a[2] * b[0] - a[0] * b[2];
    double c2 = a[0] * b[1] - a[1] * b[0];
    c[0] = c0; c[1] = c1; c[2] = c2;
}
/* np.dot(M, v) with M a C-ordered 3x3 (OpenBLAS dgemv, row-major no-trans) */
static inline void gemv3_np(const double* M, const double* v, double* y) {
    double t[3];
    for (int i = 0; i < 3; ++i) t[i] = fma(M[3 * i + 2], v[2], fma(M[3 * i + 0], v[0], M[3 * i + 1] * v[1]));
    y[0] = t[0]; y[1] = t[1]; y[2] = t[2];
}

/* rainbow/math/quaternion.py:76 unit */
static void quat_unit(const double* q, double* out) {
    double l = norm4_np(q);
    if (l > 0.0) {
        double t0 = q[0] / l, t1 = q[1] / l, t2 = q[2] / l, t3 = q[3] / l;
        out[0] = t0; out[1] = t1; out[2] = t2; out[3] = t3;
    } else {
        out[0] = 1.0; out[1] = 0.0; out[2] = 0.0; out[3] = 0.0;
    }
}
/* rainbow/math/quaternion.py:186 prod */
static void quat_prod(const double* qa, const double* qb, double* out) {
    double a = qa[0], b = qb[0];
    const double* A = qa + 1;
    const double* B = qb + 1;
    double qs = a * b - dot3_np(A, B);
    double cr[3];
    cross_np(A, B, cr);
    double v0 = (a * B[0] + A[0] * b) + cr[0];
    double v1 = (a * B[1] + A[1] * b) + cr[1];
    double v2 = (a * B[2] + A[2] * b) + cr[2];
    out[0] = qs; out[1] = v0; out[2] = v1; out[3] = v2;
}
/* rainbow/math/quaternion.py:196 rotate */
static void quat_rotate(const double* q, const double* r, double* out) {
    double qr[4] = {0.0, r[0], r[1], r[2]};
    double cq[4] = {q[0], -q[1], -q[2], -q[3]};
    double t[4], u[4];
    quat_prod(q, qr, t);
    quat_prod(t, cq, u);
    out[0] = u[1]; out[1] = u[2]; out[2] = u[3];
}
/* rainbow/math/quaternion.py:244 rotate_array for one row, via prod_array (:201-241) */
static void quat_rotate_row(const double* q, const double* p, double* out) {
    const double x = p[0], y = p[1], z = p[2];
    /* inner = prod_array(q, [0, x, y, z]) (1-D times 2-D branch, :206-220) */
    double a0 = ((q[0] * 0.0 - q[1] * x) - q[2] * y) - q[3] * z;
    double a1 = ((q[0] * x + q[1] * 0.0) + q[2] * z) - q[3] * y;
    double a2 = ((q[0] * y - q[1] * z) + q[2] * 0.0) + q[3] * x;
    double a3 = ((q[0] * z + q[1] * y) - q[2] * x) + q[3] * 0.0;
    /* outer = prod_array(inner, conjugate(q)) (2-D times 1-D branch, :221-235); keep the vector part */
    const double c0 = q[0], c1 = -q[1], c2 = -q[2], c3 = -q[3];
    double o1 = ((a0 * c1 + a1 * c0) + a2 * c3) - a3 * c2;
    double o2 = ((a0 * c2 - a1 * c3) + a2 * c0) + a3 * c1;
    double o3 = ((a0 * c3 + a1 * c2) - a2 * c1) + a3 * c0;
    out[0] = o1; out[1] = o2; out[2] = o3;
}
/* rainbow/math/quaternion.py:108 to_matrix */
static void quat_to_matrix(const double* Q, double* R) {
    double q[4];
    quat_unit(Q, q);
    double qs = q[0], qx = q[1], qy = q[2], qz = q[3];
    R[0] = 1.0 - 2.0 * (qy * qy + qz * qz);
    R[4] = 1.0 - 2.0 * (qx * qx + qz * qz);
    R[8] = 1.0 - 2.0 * (qy * qy + qx * qx);
    R[3] = 2.0 * (qx * qy + qs * qz);
    R[1] = 2.0 * (qx * qy - qs * qz);
    R[6] = 2.0 * (-qs * qy + qx * qz);
    R[2] = 2.0 * (qs * qy + qx * qz);
    R[7] = 2.0 * (qz * qy + qs * qx);
    R[5] = 2.0 * (qz * qy - qs * qx);
}
/* rainbow/simulators/prox_rigid_bodies/mass.py:395 update_inertia_tensor (W = R diag(Bv) R^T) */
static void update_inertia_tensor(const double* R, const double* Bv, double* W) {
    double w00 = (R[0] * R[0] * Bv[0] + R[1] * R[1] * Bv[1]) + R[2] * R[2] * Bv[2];
    double w11 = (R[3] * R[3] * Bv[0] + R[4] * R[4] * Bv[1]) + R[5] * R[5] * Bv[2];
    double w22 = (R[6] * R[6] * Bv[0] + R[7] * R[7] * Bv[1]) + R[8] * R[8] * Bv[2];
    double w10 = (R[3] * R[0] * Bv[0] + R[4] * R[1] * Bv[1]) + R[5] * R[2] * Bv[2];
    double w20 = (R[6] * R[0] * Bv[0] + R[7] * R[1] * Bv[1]) + R[8] * R[2] * Bv[2];
    double w21 = (R[3] * R[6] * Bv[0] + R[4] * R[7] * Bv[1]) + R[5] * R[8] * Bv[2];
    W[0] = w00; W[4] = w11; W[8] = w22;
    W[3] = W[1] = w10;
    W[6] = W[2] = w20;
    W[7] = W[5] = w21;
}
/* rainbow/math/vector3.py:75 make_orthonormal_vectors -> (t, b, n) */
static void make_orthonormal_vectors(const double* nin, double* t, double* b, double* n) {
    double l = norm3_np(nin);
    n[0] = nin[0] / l; n[1] = nin[1] / l; n[2] = nin[2] / l;
    double nx = fabs(n[0]), ny = fabs(n[1]), nz = fabs(n[2]);
    double tg[3] = {0.0, 0.0, 0.0};
    if (nx <= ny && nx <= nz) { tg[0] = 1.0; tg[1] = 0.0; tg[2] = 0.0; }
    if (ny <= nx && ny <= nz) { tg[0] = 0.0; tg[1] = 1.0; tg[2] = 0.0; }
    if (nz <= nx && nz <= ny) { tg[0] = 0.0; tg[1] = 0.0; tg[2] = 1.0; }
    cross_np(n, tg, b);
    double lb = norm3_np(b);
    b[0] /= lb; b[1] /= lb; b[2] /= lb;
    cross_np(b, n, t);
}
/* rainbow/simulators/prox_rigid_bodies/prox_operators.py:14 prox_sphere */
static void prox_sphere(double zs, double zt, double ztau, double mu, double xn, double* out) {
    if (xn <= 0.0) { out[0] = 0.0; out[1] = 0.0; out[2] = 0.0; return; }
    double radius = mu * xn;
    double sqr = zs * zs + zt * zt + ztau * ztau;
    if (sqr <= radius * radius) { out[0] = zs; out[1] = zt; out[2] = ztau; return; }
    double scale = radius / sqrt(sqr);
    out[0] = zs * scale; out[1] = zt * scale; out[2] = ztau * scale;
}

/* ------------------------------------------------------------------------------------------------------ */
/* Signed distance grid lookups: rainbow/geometry/grid3.py                                                 */
/* meta layout per shape: min[3], max[3], spacing[3], I, J, K                                             */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct {
    const double* values;
    double mn[3], mx[3], sp[3];
    long I, J, K;
} Grid;

/* grid3.py:107 get_enclosing_cell_idx */
static void grid_cell(const Grid* g, const double* p, long* ijk) {
    const long lim[3] = {g->I - 2, g->J - 2, g->K - 2};
    for (int a = 0; a < 3; ++a) {
        double f = floor((p[a] - g->mn[a]) / g->sp[a]);
        long c;
        if (!(f >= 0.0)) c = 0;                       /* negative (or NaN) clips to 0 */
        else if (f > (double)lim[a]) c = lim[a];
        else c = (long)f;
        if (c > lim[a]) c = lim[a];
        ijk[a] = c;
    }
}
static inline double node(const Grid* g, long i, long j, long k) { return g->values[i + g->I * (j + g->J * k)]; }

/* grid3.py:126 get_value */
static double grid_value(const Grid* g, const double* p) {
    long c[3];
    grid_cell(g, p, c);
    long i = c[0], j = c[1], k = c[2];
    double d000 = node(g, i, j, k), d001 = node(g, i, j, k + 1), d010 = node(g, i, j + 1, k),
           d011 = node(g, i, j + 1, k + 1), d100 = node(g, i + 1, j, k), d101 = node(g, i + 1, j, k + 1),
           d110 = node(g, i + 1, j + 1, k), d111 = node(g, i + 1, j + 1, k + 1);
    double s = (p[0] - (((double)i * g->sp[0]) + g->mn[0])) / g->sp[0];
    double t = (p[1] - (((double)j * g->sp[1]) + g->mn[1])) / g->sp[1];
    double u = (p[2] - (((double)k * g->sp[2]) + g->mn[2])) / g->sp[2];
    double x00 = (d100 - d000) * s + d000;
    double x01 = (d101 - d001) * s + d001;
    double x10 = (d110 - d010) * s + d010;
    double x11 = (d111 - d011) * s + d011;
    double y0 = (x10 - x00) * t + x00;
    double y1 = (x11 - x01) * t + x01;
    return (y1 - y0) * u + y0;
}
/* grid3.py:180 get_gradient -- including the reference's division by min_coord in s, t, u (:209-211) */
static void grid_gradient(const Grid* g, const double* p, double* grad) {
    long c[3];
    grid_cell(g, p, c);
    long i = c[0], j = c[1], k = c[2];
    double d000 = node(g, i, j, k), d001 = node(g, i, j, k + 1), d010 = node(g, i, j + 1, k),
           d011 = node(g, i, j + 1, k + 1), d100 = node(g, i + 1, j, k), d101 = node(g, i + 1, j, k + 1),
           d110 = node(g, i + 1, j + 1, k), d111 = node(g, i + 1, j + 1, k + 1);
    double s = (p[0] - ((double)i * g->sp[0] + g->mn[0])) / g->mn[0];
    double t = (p[1] - ((double)j * g->sp[1] + g->mn[1])) / g->mn[1];
    double u = (p[2] - ((double)k * g->sp[2] + g->mn[2])) / g->mn[2];
    double x00 = (d100 - d000) * s + d000;
    double x01 = (d101 - d001) * s + d001;
    double x10 = (d110 - d010) * s + d010;
    double x11 = (d111 - d011) * s + d011;
    double y0 = (x10 - x00) * t + x00;
    double y1 = (x11 - x01) * t + x01;
    double dx00 = d100 - d000, dx01 = d101 - d001, dx10 = d110 - d010, dx11 = d111 - d011;
    double dy0_ds = (dx10 - dx00) * t + dx00;
    double dy1_ds = (dx11 - dx01) * t + dx01;
    double dy0_dt = x10 - x00;
    double dy1_dt = x11 - x01;
    double dp_ds = (dy1_ds - dy0_ds) * u + dy0_ds;
    double dp_dt = (dy1_dt - dy0_dt) * u + dy0_dt;
    double dp_du = y1 - y0;
    grad[0] = dp_ds * (1.0 / g->sp[0]);
    grad[1] = dp_dt * (1.0 / g->sp[1]);
    grad[2] = dp_du * (1.0 / g->sp[2]);
}
/* grid3.py:275 is_inside */
static int grid_is_inside(const Grid* g, const double* p, double boundary) {
    if (p[0] > (g->mx[0] - boundary)) return 0;
    if (p[1] > (g->mx[1] - boundary)) return 0;
    if (p[2] > (g->mx[2] - boundary)) return 0;
    if (p[0] < (g->mn[0] + boundary)) return 0;
    if (p[1] < (g->mn[1] + boundary)) return 0;
    if (p[2] < (g->mn[2] + boundary)) return 0;
    return 1;
}

/* ------------------------------------------------------------------------------------------------------ */
/* Scene description (flat arrays, owned by the caller)                                                    */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct {
    int32_t n_shapes;
    const double* V; const int64_t* v_off;        /* body-frame vertices, shape s: rows v_off[s]..v_off[s+1] */
    const int32_t* T; const int64_t* t_off;       /* triangles (vertex indices local to the shape) */
    const double* grid; const int64_t* g_off;     /* SDF node values */
    const double* grid_meta;                      /* 12 doubles per shape */
    int32_t n_bodies;
    const int32_t* body_shape;
    const double* mass; const double* inertia;    /* inertia: 3 per body (body frame diagonal) */
    const uint8_t* fixed;
    const int32_t* material;
    int32_t n_forces;
    const int32_t* force_kind;                    /* 0 gravity, 1 damping */
    const double* force_params;                   /* gravity: g, up[3]; damping: alpha, beta */
    const int32_t* body_force_order;              /* n_bodies x n_forces, connection order, -1 padded */
    int32_t n_materials;
    const double* material_mu;                    /* M x M x 3 */
    const double* material_eps;                   /* M x M */
    int32_t n_hinges;                             /* engine.hinges in Hinge.idx order */
    const int32_t* hinge_bodies;                  /* 2 per hinge: parent, child */
    const double* hinge_frames;                   /* 12 per hinge: arm_p, arm_c, axis_p, axis_c (body frames) */
} OScene;

/* Parameter vector order (Parameters fields, types.py:356-418) */
enum {
    P_TIME_STEP = 0, P_MAX_ITER, P_USE_BOUNCE, P_USE_PRE, P_USE_POST, P_GAP_REDUCTION, P_MIN_GAP, P_MAX_GAP,
    P_ABS_TOL, P_REL_TOL, P_NU_REDUCE, P_NU_INCREASE, P_TOO_SMALL, P_FW_MAX_ITER, P_FW_TOL, P_CHUNK, P_K,
    P_ENVELOPE, P_RESOLUTION, P_COUNT
};

/* solver schemes */
enum { S_RIGID_GS = 0, S_IFACE_GS = 1, S_JACOBI = 2, S_JACOBI_HYBRID = 3, S_COLOURED_GS = 4 };

typedef struct {
    /* inputs */
    int32_t scheme;
    int32_t capacity;            /* contact capacity of the arrays below */
    /* outputs */
    int32_t n_contacts;
    int32_t iterations, exitcode;
    int32_t post_iterations, post_exitcode;
    int32_t overflow;
    int32_t n_overlap_pairs;     /* body pairs with at least one overlapping leaf pair */
    int64_t n_leaf_overlaps;     /* number of overlapping leaf pairs (profile key number_of_overlaps) */
    int64_t n_candidates;        /* triangles sent to the Frank-Wolfe search */
    int32_t n_colours;
    int32_t* ids;                /* 2 per contact: bodyA (SDF owner), bodyB (mesh owner) */
    double* p; double* n; double* g;
    double* b; double* diag; double* sol;   /* 4 per contact */
    double* residuals;           /* max_iterations */
    double* delta_u_ext;         /* 6 per body */
    double kinetic, potential, max_penetration;
    double* hinge_b; double* hinge_diag; double* hinge_sol;   /* 5 per hinge (NULL: not recorded) */
    /* warm start (an option of the GPU step, not of the reference, which starts from zero, contacts.py:53):
       contact k starts from the impulses of the cache entry with its key, when there is one.  Key of a
       contact = (lower body << 31 | higher body, side << 30 | triangle), side 1 when the mesh owner is the
       higher body; the contacts of a step come out in ascending key order. */
    int32_t warm_count;          /* entries of warm_key / warm_sol (0: every contact starts from zero) */
    const int64_t* warm_key;     /* 2 per entry, ascending */
    const double* warm_sol;      /* 4 per entry */
    int64_t* keys;               /* out: 2 per contact (NULL: not recorded) */
} OStepOut;

typedef struct { double lo[3], hi[3]; } AABB;

static inline int aabb_overlap(const AABB* a, const AABB* b) {
    for (int k = 0; k < 3; ++k)
        if (a->hi[k] < b->lo[k] || b->hi[k] < a->lo[k]) return 0;
    return 1;
}

static void load_grid(const OScene* sc, int s, Grid* g) {
    const double* m = sc->grid_meta + 12 * s;
    g->values = sc->grid + sc->g_off[s];
    for (int a = 0; a < 3; ++a) { g->mn[a] = m[a]; g->mx[a] = m[3 + a]; g->sp[a] = m[6 + a]; }
    g->I = (long)m[9]; g->J = (long)m[10]; g->K = (long)m[11];
}

/* ------------------------------------------------------------------------------------------------------ */
/* Collision detection: rainbow/simulators/prox_rigid_bodies/collision_detection.py                       */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct {
    int n;
    int cap;
    int32_t* ids; double* p; double* n_; double* g;
    int64_t* key;   /* 2 per contact: warm-start key (see OStepOut.warm_key) */
} ContactList;

static void contacts_push(ContactList* cl, int a, int b, const double* p, const double* n, double g, int tri) {
    if (cl->n == cl->cap) {
        cl->cap = cl->cap ? 2 * cl->cap : 64;
        cl->ids = (int32_t*)realloc(cl->ids, sizeof(int32_t) * 2 * cl->cap);
        cl->p = (double*)realloc(cl->p, sizeof(double) * 3 * cl->cap);
        cl->n_ = (double*)realloc(cl->n_, sizeof(double) * 3 * cl->cap);
        cl->g = (double*)realloc(cl->g, sizeof(double) * cl->cap);
        cl->key = (int64_t*)realloc(cl->key, sizeof(int64_t) * 2 * cl->cap);
    }
    int k = cl->n++;
    cl->ids[2 * k] = a; cl->ids[2 * k + 1] = b;
    memcpy(cl->p + 3 * k, p, 3 * sizeof(double));
    memcpy(cl->n_ + 3 * k, n, 3 * sizeof(double));
    cl->g[k] = g;
    /* a = SDF owner, b = mesh owner */
    const int lo = a < b ? a : b, hi = a < b ? b : a;
    cl->key[2 * k] = ((int64_t)lo << 31) | (int64_t)hi;
    cl->key[2 * k + 1] = ((int64_t)(b == hi) << 30) | (int64_t)tri;
}

/* collision_detection.py:87 _compute_contacts: triangles of body A (mesh) against the SDF of body B */
static void compute_contacts(const OScene* sc, const double* params, const double* Vw_all, const int64_t* body_v0,
                             const double* r, const double* q, int A, int B, const int32_t* tris, int ntris,
                             ContactList* out) {
    const int sa = sc->body_shape[A], sb = sc->body_shape[B];
    const int64_t v0 = sc->v_off[sa], nv = sc->v_off[sa + 1] - v0;
    const int32_t* T = sc->T + 3 * sc->t_off[sa];
    Grid grid;
    load_grid(sc, sb, &grid);
    const double* qB = q + 4 * B;
    const double* rB = r + 3 * B;
    const double cqB[4] = {qB[0], -qB[1], -qB[2], -qB[3]};
    /* V_b = rotate_array(conjugate(qB), V_w - rB)  (:120-121) */
    double* Vb = (double*)malloc(sizeof(double) * 3 * (size_t)nv);
    for (int64_t v = 0; v < nv; ++v) {
        const double* pw = Vw_all + 3 * (body_v0[A] + v);
        double d[3] = {pw[0] - rB[0], pw[1] - rB[1], pw[2] - rB[2]};
        quat_rotate_row(cqB, d, Vb + 3 * v);
    }
    const int max_it = (int)params[P_FW_MAX_ITER];
    const double tol = params[P_FW_TOL];
    const double envelope = params[P_ENVELOPE];
    for (int ti = 0; ti < ntris; ++ti) {
        const int32_t* tri = T + 3 * tris[ti];
        const double* ps[3] = {Vb + 3 * tri[0], Vb + 3 * tri[1], Vb + 3 * tri[2]};
        /* seed: corner with the smallest gradient norm (:136-140) */
        double gn[3];
        for (int c = 0; c < 3; ++c) {
            double gr[3];
            grid_gradient(&grid, ps[c], gr);
            /* np.linalg.norm(list, axis=1) squares elementwise and add.reduce's along rows: no fusion */
            gn[c] = sqrt((gr[0] * gr[0] + gr[1] * gr[1]) + gr[2] * gr[2]);
        }
        int best = 0;
        for (int c = 1; c < 3; ++c) if (gn[c] < gn[best]) best = c;
        double x[3] = {ps[best][0], ps[best][1], ps[best][2]};
        /* Frank-Wolfe iterations (:144-165) */
        for (int it = 0; it < max_it; ++it) {
            double obj[3];
            for (int c = 0; c < 3; ++c) {
                double gr[3];
                grid_gradient(&grid, x, gr);
                obj[c] = dot3_np(ps[c], gr);
            }
            int v = 0;
            for (int c = 1; c < 3; ++c) if (obj[c] < obj[v]) v = c;
            const double alpha = 2.0 / (double)(it + 2);
            double nx[3];
            for (int a = 0; a < 3; ++a) nx[a] = x[a] + alpha * (ps[v][a] - x[a]);
            x[0] = nx[0]; x[1] = nx[1]; x[2] = nx[2];
            if (obj[v] > tol) break;
        }
        /* contact generation (:172-188) */
        if (grid_is_inside(&grid, x, 0.5)) {
            double phi = grid_value(&grid, x);
            if (phi <= envelope) {
                double nb[3], nw[3];
                grid_gradient(&grid, x, nb);
                quat_rotate(qB, nb, nw);
                double ln = norm3_np(nw);
                if (ln > 0.0) {
                    double pw[3], xr[3];
                    quat_rotate(qB, x, xr);
                    pw[0] = xr[0] + rB[0]; pw[1] = xr[1] + rB[1]; pw[2] = xr[2] + rB[2];
                    double un[3] = {nw[0] / ln, nw[1] / ln, nw[2] / ln};
                    contacts_push(out, B, A, pw, un, phi, tris[ti]);
                }
            }
        }
    }
    free(Vb);
}

/* collision_detection.py:293 run_collision_detection (BVH refit + traversal + determination + reduction) */
static void run_collision_detection(const OScene* sc, const double* params, const double* r, const double* q,
                                    ContactList* cl, OStepOut* out) {
    const int N = sc->n_bodies;
    const double env = params[P_ENVELOPE];
    /* world-space vertices (:32) and leaf volumes (kdop_bvh.py:52-73, kdop.py:53-75 with K=3: axis slabs) */
    int64_t* body_v0 = (int64_t*)malloc(sizeof(int64_t) * (N + 1));
    int64_t* body_t0 = (int64_t*)malloc(sizeof(int64_t) * (N + 1));
    body_v0[0] = 0; body_t0[0] = 0;
    for (int b = 0; b < N; ++b) {
        int s = sc->body_shape[b];
        body_v0[b + 1] = body_v0[b] + (sc->v_off[s + 1] - sc->v_off[s]);
        body_t0[b + 1] = body_t0[b] + (sc->t_off[s + 1] - sc->t_off[s]);
    }
    double* Vw = (double*)malloc(sizeof(double) * 3 * (size_t)(body_v0[N] ? body_v0[N] : 1));
    AABB* leaf = (AABB*)malloc(sizeof(AABB) * (size_t)(body_t0[N] ? body_t0[N] : 1));
    AABB* root = (AABB*)malloc(sizeof(AABB) * N);
    for (int b = 0; b < N; ++b) {
        int s = sc->body_shape[b];
        const double* V = sc->V + 3 * sc->v_off[s];
        int64_t nv = sc->v_off[s + 1] - sc->v_off[s];
        for (int64_t v = 0; v < nv; ++v) {
            double* o = Vw + 3 * (body_v0[b] + v);
            quat_rotate_row(q + 4 * b, V + 3 * v, o);
            o[0] = o[0] + r[3 * b + 0]; o[1] = o[1] + r[3 * b + 1]; o[2] = o[2] + r[3 * b + 2];
        }
        const int32_t* T = sc->T + 3 * sc->t_off[s];
        int64_t nt = sc->t_off[s + 1] - sc->t_off[s];
        for (int a = 0; a < 3; ++a) { root[b].lo[a] = INFINITY; root[b].hi[a] = -INFINITY; }
        for (int64_t t = 0; t < nt; ++t) {
            AABB* L = leaf + body_t0[b] + t;
            for (int a = 0; a < 3; ++a) {
                double lo = INFINITY, hi = -INFINITY;
                for (int c = 0; c < 3; ++c) {
                    double pr = Vw[3 * (body_v0[b] + T[3 * t + c]) + a];
                    if (pr < lo) lo = pr;
                    if (pr > hi) hi = pr;
                }
                L->lo[a] = lo - env;
                L->hi[a] = hi + env;
                if (L->lo[a] < root[b].lo[a]) root[b].lo[a] = L->lo[a];
                if (L->hi[a] > root[b].hi[a]) root[b].hi[a] = L->hi[a];
            }
        }
    }
    /* narrow phase over combinations(bodies, 2) (:70-77) and contact determination (:221-249) */
    int32_t* candA = NULL; int32_t* candB = NULL; size_t cap_cand = 0;
    for (int A = 0; A < N; ++A) {
        for (int B = A + 1; B < N; ++B) {
            if (!aabb_overlap(root + A, root + B)) continue;     /* kdop_bvh.py:246 */
            int sa = sc->body_shape[A], sb = sc->body_shape[B];
            int64_t ta = sc->t_off[sa + 1] - sc->t_off[sa], tb = sc->t_off[sb + 1] - sc->t_off[sb];
            size_t need = (size_t)(ta > tb ? ta : tb);
            if (need > cap_cand) {
                cap_cand = need;
                candA = (int32_t*)realloc(candA, sizeof(int32_t) * cap_cand);
                candB = (int32_t*)realloc(candB, sizeof(int32_t) * cap_cand);
            }
            /* The tandem traversal reports exactly the overlapping leaf pairs, because every inner volume is the
               exact union of its children.  np.unique of each column gives the ascending triangle sets. */
            uint8_t* hitB = (uint8_t*)calloc((size_t)tb + 1, 1);
            /* only leaves that overlap the other body's root can overlap one of its leaves */
            int nbr = 0;
            for (int64_t j = 0; j < tb; ++j)
                if (aabb_overlap(leaf + body_t0[B] + j, root + A)) candB[nbr++] = (int32_t)j;
            int na = 0;
            int64_t overlaps = 0;
            for (int64_t i = 0; i < ta; ++i) {
                const AABB* la = leaf + body_t0[A] + i;
                if (!aabb_overlap(la, root + B)) continue;
                int hit = 0;
                for (int e = 0; e < nbr; ++e) {
                    const int64_t j = candB[e];
                    if (aabb_overlap(la, leaf + body_t0[B] + j)) { hit = 1; hitB[j] = 1; ++overlaps; }
                }
                if (hit) candA[na++] = (int32_t)i;
            }
            if (overlaps == 0) { free(hitB); continue; }
            int nb = 0;
            for (int64_t j = 0; j < tb; ++j) if (hitB[j]) candB[nb++] = (int32_t)j;
            free(hitB);
            out->n_overlap_pairs += 1;
            out->n_leaf_overlaps += overlaps;
            out->n_candidates += na + nb;
            compute_contacts(sc, params, Vw, body_v0, r, q, A, B, candA, na, cl);
            compute_contacts(sc, params, Vw, body_v0, r, q, B, A, candB, nb, cl);
        }
    }
    free(candA); free(candB);
    /* contact reduction (:255-290): drop a contact whose unordered body pair and position equal an earlier one */
    int kept = 0;
    for (int k = 0; k < cl->n; ++k) {
        int a = cl->ids[2 * k], b = cl->ids[2 * k + 1];
        const double* pk = cl->p + 3 * k;
        int unique = 1;
        for (int m = 0; m < kept; ++m) {
            int c = cl->ids[2 * m], d = cl->ids[2 * m + 1];
            int same_pair = (a == c && b == d) || (a == d && b == c);
            const double* pm = cl->p + 3 * m;
            if (same_pair && pk[0] == pm[0] && pk[1] == pm[1] && pk[2] == pm[2]) { unique = 0; break; }
        }
        if (unique) {
            if (kept != k) {
                cl->ids[2 * kept] = a; cl->ids[2 * kept + 1] = b;
                cl->key[2 * kept] = cl->key[2 * k]; cl->key[2 * kept + 1] = cl->key[2 * k + 1];
                memmove(cl->p + 3 * kept, pk, 3 * sizeof(double));
                memmove(cl->n_ + 3 * kept, cl->n_ + 3 * k, 3 * sizeof(double));
                cl->g[kept] = cl->g[k];
            }
            ++kept;
        }
    }
    cl->n = kept;
    free(body_v0); free(body_t0); free(Vw); free(leaf); free(root);
}

/* ------------------------------------------------------------------------------------------------------ */
/* Contact problem: rainbow/simulators/prox_rigid_bodies/constraints/contacts.py                          */
/* Each contact k owns J rows 4k..4k+3 with 12 nonzeros per row (6 per body).  WJT columns 4k..4k+3 hold  */
/* the same pattern transposed.  Per-body contact lists (ascending k) give the sequential column order    */
/* of the SciPy products.                                                                                   */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct {
    int K, N;
    const int32_t* ids;
    double* J;      /* K x 4 x 12: [body lo: v(3) w(3) | body hi: v(3) w(3)], lo/hi = ascending body index */
    int32_t* lohi;  /* K x 2 body indices in ascending order */
    double* WJT;    /* K x 4 x 12 transposed values: WJT[dof, row] stored at [k][row][slot] */
    uint8_t* has_w; /* K x 2: whether the body side has a W block (non-fixed) */
    int32_t* body_ptr; int32_t* body_list; /* CSR: contacts touching each body, ascending */
} Problem;

/* row dot product J_row . w with columns ascending (csr_matvec) */
static inline double jrow_dot(const Problem* P, int k, int row, const double* w) {
    const double* Jr = P->J + 48 * k + 12 * row;
    const int lo = P->lohi[2 * k], hi = P->lohi[2 * k + 1];
    double s = 0.0;
    for (int c = 0; c < 6; ++c) s += Jr[c] * w[6 * lo + c];
    for (int c = 0; c < 6; ++c) s += Jr[6 + c] * w[6 * hi + c];
    return s;
}

/* y = WJT . x  (6N), accumulated per dof over contacts ascending, 4 columns each (bsr/csr matvec order) */
static void wjt_dot(const Problem* P, const double* x, double* y) {
    for (int b = 0; b < P->N; ++b) {
        for (int d = 0; d < 6; ++d) {
            double s = 0.0;
            for (int e = P->body_ptr[b]; e < P->body_ptr[b + 1]; ++e) {
                int k = P->body_list[e];
                int side = (P->lohi[2 * k] == b) ? 0 : 1;
                if (!P->has_w[2 * k + side]) continue;
                for (int row = 0; row < 4; ++row) s += P->WJT[48 * k + 12 * row + 6 * side + d] * x[4 * k + row];
            }
            y[6 * b + d] = s;
        }
    }
}

static void problem_build(Problem* P, const OScene* sc, const ContactList* cl, const double* r,
                          const double* Winv /* N x 9 world inverse inertia */) {
    const int K = cl->n, N = sc->n_bodies;
    P->K = K; P->N = N; P->ids = cl->ids;
    P->J = (double*)calloc((size_t)48 * (K ? K : 1), sizeof(double));
    P->WJT = (double*)calloc((size_t)48 * (K ? K : 1), sizeof(double));
    P->lohi = (int32_t*)malloc(sizeof(int32_t) * 2 * (K ? K : 1));
    P->has_w = (uint8_t*)malloc(2 * (K ? K : 1));
    P->body_ptr = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
    P->body_list = (int32_t*)malloc(sizeof(int32_t) * 2 * (K ? K : 1));
    for (int k = 0; k < K; ++k) {
        const int A = cl->ids[2 * k], B = cl->ids[2 * k + 1];
        const double* p = cl->p + 3 * k;
        double rA[3] = {p[0] - r[3 * A], p[1] - r[3 * A + 1], p[2] - r[3 * A + 2]};
        double rB[3] = {p[0] - r[3 * B], p[1] - r[3 * B + 1], p[2] - r[3 * B + 2]};
        double vs[3], vt[3], vn[3];
        make_orthonormal_vectors(cl->n_ + 3 * k, vs, vt, vn);   /* (t, b, n) */
        double JAv[4][3], JAw[4][3], JBv[4][3], JBw[4][3];
        const double* dirs[3] = {vn, vs, vt};
        for (int i = 0; i < 3; ++i) {
            double ca[3], cb[3];
            cross_np(rA, dirs[i], ca);
            cross_np(rB, dirs[i], cb);
            for (int a = 0; a < 3; ++a) {
                JAv[i][a] = -dirs[i][a]; JAw[i][a] = -ca[a];
                JBv[i][a] = dirs[i][a];  JBw[i][a] = cb[a];
            }
        }
        for (int a = 0; a < 3; ++a) { JAv[3][a] = -0.0; JAw[3][a] = -vn[a]; JBv[3][a] = 0.0; JBw[3][a] = vn[a]; }
        const int lo = A < B ? A : B, hi = A < B ? B : A;
        P->lohi[2 * k] = lo; P->lohi[2 * k + 1] = hi;
        for (int row = 0; row < 4; ++row) {
            double* Jr = P->J + 48 * k + 12 * row;
            double* sideA = Jr + (A == lo ? 0 : 6);
            double* sideB = Jr + (B == lo ? 0 : 6);
            for (int a = 0; a < 3; ++a) {
                sideA[a] = JAv[row][a]; sideA[3 + a] = JAw[row][a];
                sideB[a] = JBv[row][a]; sideB[3 + a] = JBw[row][a];
            }
        }
        for (int side = 0; side < 2; ++side) {
            const int b = P->lohi[2 * k + side];
            P->has_w[2 * k + side] = sc->fixed[b] ? 0 : 1;
            P->body_ptr[b + 1] += 1;
            if (sc->fixed[b]) continue;
            /* WJT = W J^T through bsr_matmat: per entry ((0 + W_i0 J_0) + W_i1 J_1) + W_i2 J_2 */
            const double m = 1.0 / sc->mass[b];
            const double* Wi = Winv + 9 * b;
            for (int row = 0; row < 4; ++row) {
                const double* Jr = P->J + 48 * k + 12 * row + 6 * side;
                double* Wr = P->WJT + 48 * k + 12 * row + 6 * side;
                for (int i = 0; i < 3; ++i) {
                    double s = 0.0;
                    s += (i == 0 ? m : 0.0) * Jr[0];
                    s += (i == 1 ? m : 0.0) * Jr[1];
                    s += (i == 2 ? m : 0.0) * Jr[2];
                    Wr[i] = s;
                    double u = 0.0;
                    u += Wi[3 * i + 0] * Jr[3];
                    u += Wi[3 * i + 1] * Jr[4];
                    u += Wi[3 * i + 2] * Jr[5];
                    Wr[3 + i] = u;
                }
            }
        }
    }
    for (int b = 0; b < N; ++b) P->body_ptr[b + 1] += P->body_ptr[b];
    int32_t* fill = (int32_t*)calloc((size_t)N, sizeof(int32_t));
    for (int k = 0; k < K; ++k)
        for (int side = 0; side < 2; ++side) {
            int b = P->lohi[2 * k + side];
            P->body_list[P->body_ptr[b] + fill[b]++] = k;
        }
    free(fill);
}

static void problem_free(Problem* P) {
    free(P->J); free(P->WJT); free(P->lohi); free(P->has_w); free(P->body_ptr); free(P->body_list);
}

/* np.add.reduceat over one segment: out = a[0] + pairwise_sum(a[1:]), NumPy's pairwise summation adding
   8 interleaved partial sums once the remainder has at least 8 elements (numpy/_core/src/umath/loops_utils) */
static double np_reduce_sum(const double* a, int m) {
    if (m <= 0) return 0.0;
    const double* rest = a + 1;
    const int n = m - 1;
    double res;
    if (n < 8) {
        res = 0.0;
        for (int i = 0; i < n; ++i) res += rest[i];
    } else {
        double r[8];
        for (int j = 0; j < 8; ++j) r[j] = rest[j];
        int i = 8;
        for (; i + 8 <= n; i += 8)
            for (int j = 0; j < 8; ++j) r[j] += rest[i + j];
        res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res += rest[i];
    }
    return a[0] + res;
}

/* diag = sum(J .* WJT^T, axis=1) (contacts.py:49-50): the elementwise product keeps nonzero products in
   column order and the row sum is a reduceat over them */
static void problem_diag(const Problem* P, double* diag) {
    for (int k = 0; k < P->K; ++k)
        for (int row = 0; row < 4; ++row) {
            const double* Jr = P->J + 48 * k + 12 * row;
            const double* Wr = P->WJT + 48 * k + 12 * row;
            double prods[12];
            int m = 0;
            for (int c = 0; c < 12; ++c) {
                int side = c / 6;
                if (!P->has_w[2 * k + side]) continue;
                double prod = Jr[c] * Wr[c];
                if (prod != 0.0) prods[m++] = prod;
            }
            double s = np_reduce_sum(prods, m);
            diag[4 * k + row] = (s == 0.0) ? 1.0 : s;
        }
}

/* ------------------------------------------------------------------------------------------------------ */
/* Sweeps                                                                                                   */
/* ------------------------------------------------------------------------------------------------------ */
/* constraints/contacts.py:66 Contacts.sweep (serial Gauss-Seidel with incremental w) */
/* order: contact visiting order (NULL = ascending, the reference's serial sweep).  A colour-grouped order
   gives the graph-coloured Gauss-Seidel sweep: contacts of one colour share no non-fixed body, so visiting them
   one after the other equals updating them together from the w left by the earlier colours. */
static void sweep_gs(const Problem* P, const double* r, const double* b, const double* mu, double* x, double* w,
                     int normal_only, const int32_t* order) {
    wjt_dot(P, x, w);
    for (int e = 0; e < P->K; ++e) {
        const int k = order ? order[e] : e;
        double xb[4], delta[4], z[4];
        for (int i = 0; i < 4; ++i) { xb[i] = x[4 * k + i]; delta[i] = xb[i]; }
        for (int i = 0; i < 4; ++i) z[i] = xb[i] - r[4 * k + i] * (jrow_dot(P, k, i, w) + b[4 * k + i]);
        xb[0] = z[0] > 0.0 ? z[0] : 0.0;
        if (normal_only) {
            xb[1] = 0.0; xb[2] = 0.0; xb[3] = 0.0;
        } else {
            double f[3];
            prox_sphere(z[1], z[2], z[3], mu[k], xb[0], f);
            xb[1] = f[0]; xb[2] = f[1]; xb[3] = f[2];
        }
        for (int i = 0; i < 4; ++i) { x[4 * k + i] = xb[i]; delta[i] = xb[i] - delta[i]; }
        for (int side = 0; side < 2; ++side) {
            if (!P->has_w[2 * k + side]) continue;
            const int bb = P->lohi[2 * k + side];
            for (int d = 0; d < 6; ++d) {
                double s = 0.0;
                for (int row = 0; row < 4; ++row) s += P->WJT[48 * k + 12 * row + 6 * side + d] * delta[row];
                w[6 * bb + d] = w[6 * bb + d] + s;
            }
        }
    }
}

/* proximal_contact/jacobi_solver.py:6-57 (hybrid: the friction radius uses the new x_n) */
static void sweep_jacobi(const Problem* P, const double* r, const double* b, const double* mu, double* x, double* w,
                         double* xold, int hybrid) {
    wjt_dot(P, x, w);
    memcpy(xold, x, sizeof(double) * 4 * P->K);
    for (int k = 0; k < P->K; ++k) {
        double z[4];
        for (int i = 0; i < 4; ++i) z[i] = xold[4 * k + i] - r[4 * k + i] * (jrow_dot(P, k, i, w) + b[4 * k + i]);
        double xn = z[0] > 0.0 ? z[0] : 0.0;
        double f[3];
        prox_sphere(z[1], z[2], z[3], mu[k], hybrid ? xn : xold[4 * k], f);
        x[4 * k] = xn; x[4 * k + 1] = f[0]; x[4 * k + 2] = f[1]; x[4 * k + 3] = f[2];
    }
}

/* Deterministic parallel colouring (Jones-Plassmann with hashed priorities; ties broken by index).
   A contact takes the smallest colour unused by its already-coloured neighbours once every neighbour of
   higher priority is coloured.  Neighbours: contacts sharing a non-fixed body.  Returns number of colours. */
static inline uint32_t jp_hash(uint32_t k) {
    k ^= k >> 16; k *= 0x7feb352dU; k ^= k >> 15; k *= 0x846ca68bU; k ^= k >> 16;
    return k;
}
static inline int jp_before(int a, int b) {  /* priority order: higher hash first, then lower index */
    uint32_t ha = jp_hash((uint32_t)a), hb = jp_hash((uint32_t)b);
    return ha > hb || (ha == hb && a < b);
}
int rbo_colour_contacts(int K, int N, const int32_t* ids, const uint8_t* fixed, int32_t* colour) {
    int32_t* ptr = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
    int32_t* lst = (int32_t*)malloc(sizeof(int32_t) * 2 * (K ? K : 1));
    for (int k = 0; k < K; ++k)
        for (int s = 0; s < 2; ++s) if (!fixed[ids[2 * k + s]]) ptr[ids[2 * k + s] + 1]++;
    for (int b = 0; b < N; ++b) ptr[b + 1] += ptr[b];
    int32_t* fill = (int32_t*)calloc((size_t)N, sizeof(int32_t));
    for (int k = 0; k < K; ++k)
        for (int s = 0; s < 2; ++s) {
            int b = ids[2 * k + s];
            if (!fixed[b]) lst[ptr[b] + fill[b]++] = k;
        }
    for (int k = 0; k < K; ++k) colour[k] = -1;
    int remaining = K, n_colours = 0, round = 0;
    int32_t* newc = (int32_t*)malloc(sizeof(int32_t) * (size_t)(K > 0 ? K : 1));
    while (remaining > 0) {
        /* one synchronous round: every uncoloured contact whose uncoloured neighbours all have lower priority */
        for (int k = 0; k < K; ++k) {
            newc[k] = -1;
            if (colour[k] >= 0) continue;
            int ready = 1;
            uint64_t used = 0;            /* colours < 64 tracked in a mask, larger ones by scan */
            int maxc = -1;
            for (int s = 0; s < 2 && ready; ++s) {
                int b = ids[2 * k + s];
                if (fixed[b]) continue;
                for (int e = ptr[b]; e < ptr[b + 1]; ++e) {
                    int m = lst[e];
                    if (m == k) continue;
                    if (colour[m] < 0) { if (jp_before(m, k)) { ready = 0; break; } }
                    else { if (colour[m] < 64) used |= (1ULL << colour[m]); if (colour[m] > maxc) maxc = colour[m]; }
                }
            }
            if (!ready) continue;
            int c = 0;
            for (;;) {
                int taken = 0;
                if (c < 64) taken = (int)((used >> c) & 1ULL);
                else {
                    for (int s = 0; s < 2 && !taken; ++s) {
                        int b = ids[2 * k + s];
                        if (fixed[b]) continue;
                        for (int e = ptr[b]; e < ptr[b + 1]; ++e) if (lst[e] != k && colour[lst[e]] == c) { taken = 1; break; }
                    }
                }
                if (!taken) break;
                ++c;
            }
            newc[k] = c;
        }
        for (int k = 0; k < K; ++k) if (newc[k] >= 0) { colour[k] = newc[k]; --remaining; if (newc[k] + 1 > n_colours) n_colours = newc[k] + 1; }
        ++round;
    }
    free(ptr); free(lst); free(fill); free(newc);
    (void)round;
    return n_colours;
}

/* complementarity residual: max | x - prox(x - D^-1 (A x + b)) |_inf / max(1, |x|_inf) with D = diag(A).
   Every solver of the reference scales the prox argument by a positive multiple of D^-1 (r = 1/diag,
   0.1/diag, and uniform factors of them), so all of them share this map's zeros as their fixed points. */
/* ------------------------------------------------------------------------------------------------------ */
/* Hinge joints (constraints/hinges.py): 5 rows per hinge, solved in the same Gauss-Seidel loop as the      */
/* contacts (gauss_seidel_solver.py:14), each problem with its own w, r-factors and merit                  */
/* ------------------------------------------------------------------------------------------------------ */
typedef struct {
    int H, N;
    double* J;      /* H x 5 x 12: [body lo: v(3) w(3) | body hi: v(3) w(3)] */
    int32_t* lohi;  /* H x 2 body indices in ascending order */
    double* WJT;    /* H x 5 x 12 */
    uint8_t* has_w; /* H x 2 */
    int32_t* body_ptr; int32_t* body_list;
} HProblem;

/* hinges.py:95-180 _compute_jacobian_matrix and the W J^T product of hinges.py:37 */
static void hinge_build(HProblem* P, const OScene* sc, const double* q, const double* Winv) {
    const int H = sc->n_hinges, N = sc->n_bodies;
    P->H = H; P->N = N;
    P->J = (double*)calloc((size_t)60 * (H ? H : 1), sizeof(double));
    P->WJT = (double*)calloc((size_t)60 * (H ? H : 1), sizeof(double));
    P->lohi = (int32_t*)malloc(sizeof(int32_t) * 2 * (H ? H : 1));
    P->has_w = (uint8_t*)malloc(2 * (H ? H : 1));
    P->body_ptr = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
    P->body_list = (int32_t*)malloc(sizeof(int32_t) * 2 * (H ? H : 1));
    /* the reference fills preallocated 5x3 blocks; rows 3-4 of the linear blocks stay 0 */
    double JAv[5][3] = {{0}}, JAw[5][3] = {{0}}, JBv[5][3] = {{0}}, JBw[5][3] = {{0}};
    for (int k = 0; k < H; ++k) {
        const int A = sc->hinge_bodies[2 * k], B = sc->hinge_bodies[2 * k + 1];
        const double* f = sc->hinge_frames + 12 * k;
        double ap[3], ac[3], np_[3], t[3], bb[3], nn[3];
        quat_rotate(q + 4 * A, f, ap);
        quat_rotate(q + 4 * B, f + 3, ac);
        quat_rotate(q + 4 * A, f + 6, np_);
        make_orthonormal_vectors(np_, t, bb, nn);
        /* JA_v[0:3] = I, JA_w[0:3] = -star(arm_p), JA_w[3] = t, JA_w[4] = b; JB_v[0:3] = -I,
           JB_w[0:3] = star(arm_c), JB_w[3] = -t, JB_w[4] = -b  (star(v) = [[0,-v2,v1],[v2,0,-v0],[-v1,v0,0]]) */
        const double sp[3][3] = {{0.0, -ap[2], ap[1]}, {ap[2], 0.0, -ap[0]}, {-ap[1], ap[0], 0.0}};
        const double sc3[3][3] = {{0.0, -ac[2], ac[1]}, {ac[2], 0.0, -ac[0]}, {-ac[1], ac[0], 0.0}};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                JAv[i][j] = i == j ? 1.0 : 0.0;
                JAw[i][j] = -sp[i][j];
                JBv[i][j] = -(i == j ? 1.0 : 0.0);
                JBw[i][j] = sc3[i][j];
            }
        for (int j = 0; j < 3; ++j) {
            JAw[3][j] = t[j]; JAw[4][j] = bb[j];
            JBw[3][j] = -t[j]; JBw[4][j] = -bb[j];
        }
        const int lo = A < B ? A : B, hi = A < B ? B : A;
        P->lohi[2 * k] = lo; P->lohi[2 * k + 1] = hi;
        for (int row = 0; row < 5; ++row) {
            double* Jr = P->J + 60 * k + 12 * row;
            double* sideA = Jr + (A == lo ? 0 : 6);
            double* sideB = Jr + (B == lo ? 0 : 6);
            for (int a = 0; a < 3; ++a) {
                sideA[a] = JAv[row][a]; sideA[3 + a] = JAw[row][a];
                sideB[a] = JBv[row][a]; sideB[3 + a] = JBw[row][a];
            }
        }
        for (int side = 0; side < 2; ++side) {
            const int b = P->lohi[2 * k + side];
            P->has_w[2 * k + side] = sc->fixed[b] ? 0 : 1;
            P->body_ptr[b + 1] += 1;
            if (sc->fixed[b]) continue;
            const double m = 1.0 / sc->mass[b];
            const double* Wi = Winv + 9 * b;
            for (int row = 0; row < 5; ++row) {
                const double* Jr = P->J + 60 * k + 12 * row + 6 * side;
                double* Wr = P->WJT + 60 * k + 12 * row + 6 * side;
                for (int i = 0; i < 3; ++i) {
                    double s2 = 0.0;
                    s2 += (i == 0 ? m : 0.0) * Jr[0];
                    s2 += (i == 1 ? m : 0.0) * Jr[1];
                    s2 += (i == 2 ? m : 0.0) * Jr[2];
                    Wr[i] = s2;
                    double u = 0.0;
                    u += Wi[3 * i + 0] * Jr[3];
                    u += Wi[3 * i + 1] * Jr[4];
                    u += Wi[3 * i + 2] * Jr[5];
                    Wr[3 + i] = u;
                }
            }
        }
    }
    for (int b = 0; b < N; ++b) P->body_ptr[b + 1] += P->body_ptr[b];
    int32_t* fill = (int32_t*)calloc((size_t)N, sizeof(int32_t));
    for (int k = 0; k < H; ++k)
        for (int side = 0; side < 2; ++side) {
            int b = P->lohi[2 * k + side];
            P->body_list[P->body_ptr[b] + fill[b]++] = k;
        }
    free(fill);
}

static void hinge_free(HProblem* P) {
    free(P->J); free(P->WJT); free(P->lohi); free(P->has_w); free(P->body_ptr); free(P->body_list);
}

static inline double hrow_dot(const HProblem* P, int k, int row, const double* w) {
    const double* Jr = P->J + 60 * k + 12 * row;
    const int lo = P->lohi[2 * k], hi = P->lohi[2 * k + 1];
    double s = 0.0;
    for (int c = 0; c < 6; ++c) s += Jr[c] * w[6 * lo + c];
    for (int c = 0; c < 6; ++c) s += Jr[6 + c] * w[6 * hi + c];
    return s;
}

static void hinge_wjt_dot(const HProblem* P, const double* x, double* y) {
    for (int b = 0; b < P->N; ++b)
        for (int d = 0; d < 6; ++d) {
            double s = 0.0;
            for (int e = P->body_ptr[b]; e < P->body_ptr[b + 1]; ++e) {
                int k = P->body_list[e];
                int side = (P->lohi[2 * k] == b) ? 0 : 1;
                if (!P->has_w[2 * k + side]) continue;
                for (int row = 0; row < 5; ++row) s += P->WJT[60 * k + 12 * row + 6 * side + d] * x[5 * k + row];
            }
            y[6 * b + d] = s;
        }
}

/* hinges.py:188-218 _compute_error_vector (pre-stabilisation only) */
static void hinge_error(const OScene* sc, const double* params, double dt, const double* r, const double* q,
                        double* g) {
    const int H = sc->n_hinges;
    for (int i = 0; i < 5 * H; ++i) g[i] = 0.0;
    if (params[P_USE_PRE] == 0.0) return;
    for (int k = 0; k < H; ++k) {
        const int A = sc->hinge_bodies[2 * k], B = sc->hinge_bodies[2 * k + 1];
        const double* f = sc->hinge_frames + 12 * k;
        double rp[3], rc[3], np_[3], t[3], bb[3], nn[3], nc[3], u[3];
        quat_rotate(q + 4 * A, f, rp);
        quat_rotate(q + 4 * B, f + 3, rc);
        for (int i = 0; i < 3; ++i) { rp[i] = rp[i] + r[3 * A + i]; rc[i] = rc[i] + r[3 * B + i]; }
        quat_rotate(q + 4 * A, f + 6, np_);
        make_orthonormal_vectors(np_, t, bb, nn);
        quat_rotate(q + 4 * B, f + 9, nc);
        cross_np(nn, nc, u);
        for (int i = 0; i < 3; ++i) g[5 * k + i] = rc[i] - rp[i];
        g[5 * k + 3] = dot3_np(t, u);
        g[5 * k + 4] = dot3_np(bb, u);
    }
    const double rate = params[P_GAP_REDUCTION] / dt;
    for (int i = 0; i < 5 * H; ++i) g[i] = g[i] * rate;
}

/* hinges.py:57-90 Hinges.sweep: x_b -= r_b (J w + b)_b, then w += WJT[:, b] dx */
static void hinge_sweep(const HProblem* P, const double* r, const double* b, double* x, double* w) {
    hinge_wjt_dot(P, x, w);
    for (int k = 0; k < P->H; ++k) {
        double xb[5], delta[5], jw[5];
        for (int i = 0; i < 5; ++i) jw[i] = hrow_dot(P, k, i, w);
        for (int i = 0; i < 5; ++i) {
            xb[i] = x[5 * k + i];
            delta[i] = xb[i];
            xb[i] = xb[i] - r[5 * k + i] * (jw[i] + b[5 * k + i]);
            x[5 * k + i] = xb[i];
            delta[i] = xb[i] - delta[i];
        }
        for (int side = 0; side < 2; ++side) {
            if (!P->has_w[2 * k + side]) continue;
            const int bb = P->lohi[2 * k + side];
            for (int d = 0; d < 6; ++d) {
                double s = 0.0;
                for (int row = 0; row < 5; ++row) s += P->WJT[60 * k + 12 * row + 6 * side + d] * delta[row];
                w[6 * bb + d] = w[6 * bb + d] + s;
            }
        }
    }
}

static const double* g_residual_diag = NULL;
static int g_residual_interval = 1;   /* tol_mode 2: residual tested every this many sweeps */
static double g_relaxation = 1.0;     /* tol_mode 2: r = relaxation / diag */
void rbo_set_relaxation(double w) { g_relaxation = w; }
void rbo_set_residual_interval(int n) { g_residual_interval = n > 1 ? n : 1; }
static int g_ordering = 0;             /* 1: Gauss-Seidel schemes visit contacts in graph-coloured order */
void rbo_set_ordering(int o) { g_ordering = o; }
static double complementarity_residual(const Problem* P, const double* b, const double* mu, const double* x,
                                       double* w) {
    wjt_dot(P, x, w);
    double res = 0.0, xm = 0.0;
    for (int k = 0; k < P->K; ++k) {
        double z[4];
        for (int i = 0; i < 4; ++i)
            z[i] = x[4 * k + i] - (1.0 / g_residual_diag[4 * k + i]) * (jrow_dot(P, k, i, w) + b[4 * k + i]);
        double pn = z[0] > 0.0 ? z[0] : 0.0;
        double f[3];
        prox_sphere(z[1], z[2], z[3], mu[k], pn, f);
        double d[4] = {x[4 * k] - pn, x[4 * k + 1] - f[0], x[4 * k + 2] - f[1], x[4 * k + 3] - f[2]};
        for (int i = 0; i < 4; ++i) {
            double a = fabs(d[i]);
            if (a > res) res = a;
            double ax = fabs(x[4 * k + i]);
            if (ax > xm) xm = ax;
        }
    }
    return res / (xm > 1.0 ? xm : 1.0);
}
double rbo_problem_residual(void* P, const double* b, const double* mu, const double* x);

/* ------------------------------------------------------------------------------------------------------ */
/* Solvers                                                                                                  */
/* ------------------------------------------------------------------------------------------------------ */
static inline double merit_inf(const double* x, const double* sol, int n) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) {
        double e = fabs(x[i] - sol[i]);
        if (e > m || isnan(e)) m = e;
    }
    return m;
}

/* gauss_seidel_solver.py:14 solve, for a single problem (contacts or post-stabilisation) */
static void solve_rigid(const Problem* P, const double* params, double* r, const double* b, const double* mu,
                        double* x, double* sol, double* residuals, int* iterations, int* exitcode, int normal_only,
                        int tol_mode, double tol, const int32_t* order) {
    const int n = 4 * P->K, max_it = (int)params[P_MAX_ITER];
    double* w = (double*)malloc(sizeof(double) * 6 * (P->N ? P->N : 1));
    double last_merit = INFINITY, global_last = INFINITY;
    *iterations = max_it; *exitcode = 0;
    for (int it = 0; it < max_it; ++it) {
        double global_merit = 0.0;
        sweep_gs(P, r, b, mu, x, w, normal_only, order);
        double merit = merit_inf(x, sol, n);
        if (tol_mode == 2 && g_residual_interval > 1 && (it + 1) % g_residual_interval != 0 && it + 1 != max_it) {
            memcpy(sol, x, sizeof(double) * n);   /* fixed r between residual tests: accept */
            continue;
        }
        if (tol_mode >= 1) {   /* stop on the complementarity residual only; merit still adapts r (mode 1) */
            double res = complementarity_residual(P, b, mu, x, w);
            if (residuals) residuals[it] = res;
            if (res <= tol) { memcpy(sol, x, sizeof(double) * n); *iterations = it; *exitcode = 3; break; }
            if (tol_mode == 2) {   /* fixed r, every sweep accepted */
                memcpy(sol, x, sizeof(double) * n);
                continue;
            }
            if (merit > last_merit) {
                for (int i = 0; i < n; ++i) r[i] = params[P_NU_REDUCE] * r[i];
                memcpy(x, sol, sizeof(double) * n);
            } else {
                memcpy(sol, x, sizeof(double) * n);
                if (last_merit - merit < params[P_TOO_SMALL])
                    for (int i = 0; i < n; ++i) r[i] = params[P_NU_INCREASE] * r[i];
                last_merit = merit;
            }
            continue;
        }
        if (merit > last_merit) {
            for (int i = 0; i < n; ++i) r[i] = params[P_NU_REDUCE] * r[i];
            memcpy(x, sol, sizeof(double) * n);
            global_merit = global_merit > last_merit ? global_merit : last_merit;
        } else {
            memcpy(sol, x, sizeof(double) * n);
            if (last_merit - merit < params[P_TOO_SMALL])
                for (int i = 0; i < n; ++i) r[i] = params[P_NU_INCREASE] * r[i];
            last_merit = merit;
            global_merit = global_merit > merit ? global_merit : merit;
        }
        if (residuals) residuals[it] = global_merit;
        if (global_merit < params[P_ABS_TOL]) { *iterations = it; *exitcode = 1; break; }
        if (fabs(global_merit - global_last) < params[P_REL_TOL] * global_last) { *iterations = it; *exitcode = 2; break; }
        global_last = global_merit;
    }
    free(w);
}

/* gauss_seidel_solver.py:14 solve over the problem list [contacts (when any), hinges]: every iteration
   sweeps each problem in turn and accepts or rolls back its iterate against that problem's own last merit;
   the convergence tests use the largest merit of the iteration */
static void solve_problems(const Problem* P, double* r, const double* b, const double* mu, double* x, double* sol,
                           const HProblem* HP, double* hr, const double* hb, double* hx, double* hsol,
                           const double* params, double* residuals, int* iterations, int* exitcode) {
    const int max_it = (int)params[P_MAX_ITER];
    const int N = HP->N;
    double* w = (double*)malloc(sizeof(double) * 6 * (N ? N : 1));
    double last[2] = {INFINITY, INFINITY}, global_last = INFINITY;
    *iterations = max_it; *exitcode = 0;
    for (int it = 0; it < max_it; ++it) {
        double global_merit = 0.0;
        for (int prob = (P ? 0 : 1); prob < 2; ++prob) {
            double* xx = prob ? hx : x;
            double* ss = prob ? hsol : sol;
            double* rr = prob ? hr : r;
            const int n = prob ? 5 * HP->H : 4 * P->K;
            if (prob) hinge_sweep(HP, hr, hb, hx, w);
            else sweep_gs(P, r, b, mu, x, w, 0, NULL);
            const double merit = merit_inf(xx, ss, n);
            if (merit > last[prob]) {
                for (int i = 0; i < n; ++i) rr[i] = params[P_NU_REDUCE] * rr[i];
                memcpy(xx, ss, sizeof(double) * n);
                global_merit = global_merit > last[prob] ? global_merit : last[prob];
            } else {
                memcpy(ss, xx, sizeof(double) * n);
                if (last[prob] - merit < params[P_TOO_SMALL])
                    for (int i = 0; i < n; ++i) rr[i] = params[P_NU_INCREASE] * rr[i];
                last[prob] = merit;
                global_merit = global_merit > merit ? global_merit : merit;
            }
        }
        if (residuals) residuals[it] = global_merit;
        if (global_merit < params[P_ABS_TOL]) { *iterations = it; *exitcode = 1; break; }
        if (fabs(global_merit - global_last) < params[P_REL_TOL] * global_last) { *iterations = it; *exitcode = 2; break; }
        global_last = global_merit;
    }
    free(w);
}

/* proximal_contact/solver_interface.py:123 SolverInterface.solve: r = 0.1/diag, convergence test before
   accepting the iterate.  tol_mode 1 replaces the merit tests by the complementarity residual. */
static void solve_interface(const Problem* P, const double* params, int scheme, const double* diag, const double* b,
                            const double* mu, double* x, double* sol, double* residuals, int* iterations,
                            int* exitcode, const int32_t* order, int tol_mode, double tol) {
    const int n = 4 * P->K, max_it = (int)params[P_MAX_ITER];
    double* w = (double*)malloc(sizeof(double) * 6 * (P->N ? P->N : 1));
    double* xold = (double*)malloc(sizeof(double) * (n ? n : 1));
    double* r = (double*)malloc(sizeof(double) * (n ? n : 1));
    for (int i = 0; i < n; ++i) r[i] = (tol_mode == 2 && g_relaxation > 0.0 ? 0.1 * g_relaxation : 0.1) / diag[i];
    double last_merit = INFINITY;
    *iterations = max_it; *exitcode = 0;
    for (int it = 0; it < max_it; ++it) {
        if (scheme == S_JACOBI) sweep_jacobi(P, r, b, mu, x, w, xold, 0);
        else if (scheme == S_JACOBI_HYBRID) sweep_jacobi(P, r, b, mu, x, w, xold, 1);
        else sweep_gs(P, r, b, mu, x, w, 0, order);   /* S_IFACE_GS, S_COLOURED_GS */
        double merit = merit_inf(x, sol, n);
        if (residuals) residuals[it] = merit;
        if (tol_mode == 2 && g_residual_interval > 1 && (it + 1) % g_residual_interval != 0 && it + 1 != max_it) {
            memcpy(sol, x, sizeof(double) * n);
            continue;
        }
        if (tol_mode == 0) {
            if (merit < params[P_ABS_TOL]) { *iterations = it; *exitcode = 1; break; }
            if (fabs(merit - last_merit) < params[P_REL_TOL] * last_merit) { *iterations = it; *exitcode = 2; break; }
        } else {
            double res = complementarity_residual(P, b, mu, x, w);
            if (residuals) residuals[it] = res;
            if (res <= tol) { memcpy(sol, x, sizeof(double) * n); *iterations = it; *exitcode = 3; break; }
            if (tol_mode == 2) { memcpy(sol, x, sizeof(double) * n); continue; }   /* fixed r, always accept */
        }
        if (merit > last_merit) {
            for (int i = 0; i < n; ++i) r[i] = params[P_NU_REDUCE] * r[i];
            memcpy(x, sol, sizeof(double) * n);
        } else {
            if (last_merit - merit < params[P_TOO_SMALL])
                for (int i = 0; i < n; ++i) r[i] = params[P_NU_INCREASE] * r[i];
            last_merit = merit;
            memcpy(sol, x, sizeof(double) * n);
        }
    }
    free(w); free(xold); free(r);
}

/* ------------------------------------------------------------------------------------------------------ */
/* State: rainbow/simulators/prox_rigid_bodies/state_storage.py                                            */
/* ------------------------------------------------------------------------------------------------------ */
/* state_storage.py:108 _compute_total_external_forces and :158 _compute_inverse_mass_matrix, then
   delta_u_ext = W f_ext through bsr_matvec (:53) */
static void external_forces(const OScene* sc, const double* r, const double* q, const double* v, const double* w,
                            double* dux, double* Winv) {
    for (int b = 0; b < sc->n_bodies; ++b) {
        double* d = dux + 6 * b;
        double* Wi = Winv + 9 * b;
        if (sc->fixed[b]) {
            for (int i = 0; i < 6; ++i) d[i] = 0.0;
            for (int i = 0; i < 9; ++i) Wi[i] = 0.0;
            continue;
        }
        double R[9], Iw[9], Iw_w[3], T[3], F[3] = {0.0, 0.0, 0.0};
        quat_to_matrix(q + 4 * b, R);
        update_inertia_tensor(R, sc->inertia + 3 * b, Iw);
        gemv3_np(Iw, w + 3 * b, Iw_w);
        double c[3];
        cross_np(w + 3 * b, Iw_w, c);
        T[0] = -c[0]; T[1] = -c[1]; T[2] = -c[2];
        for (int f = 0; f < sc->n_forces; ++f) {
            int fi = sc->body_force_order[b * sc->n_forces + f];
            if (fi < 0) break;
            const double* fp = sc->force_params + 4 * fi;
            double Fi[3], Ti[3];
            if (sc->force_kind[fi] == 0) {           /* types.py:204 Gravity.compute */
                double s = -sc->mass[b] * fp[0];
                Fi[0] = s * fp[1]; Fi[1] = s * fp[2]; Fi[2] = s * fp[3];
                Ti[0] = 0.0; Ti[1] = 0.0; Ti[2] = 0.0;
            } else {                                  /* types.py:239 Damping.compute */
                for (int a = 0; a < 3; ++a) { Fi[a] = -v[3 * b + a] * fp[0]; Ti[a] = -w[3 * b + a] * fp[1]; }
            }
            for (int a = 0; a < 3; ++a) { F[a] = F[a] + Fi[a]; T[a] = T[a] + Ti[a]; }
        }
        if (sc->mass[b] == 0.0) { /* state_storage.py:170 raises; reported by the caller */ }
        const double m = 1.0 / sc->mass[b];
        double Binv[3] = {1.0 / sc->inertia[3 * b], 1.0 / sc->inertia[3 * b + 1], 1.0 / sc->inertia[3 * b + 2]};
        update_inertia_tensor(R, Binv, Wi);
        /* bsr_matvec gemv on 3x3 blocks: y_i = ((0 + A_i0 x0) + A_i1 x1) + A_i2 x2 */
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            s += (i == 0 ? m : 0.0) * F[0];
            s += (i == 1 ? m : 0.0) * F[1];
            s += (i == 2 ? m : 0.0) * F[2];
            d[i] = s;
            double t = 0.0;
            t += Wi[3 * i] * T[0];
            t += Wi[3 * i + 1] * T[1];
            t += Wi[3 * i + 2] * T[2];
            d[3 + i] = t;
        }
    }
}

/* state_storage.py:251 position_update */
static void position_update(const OScene* sc, double* r, double* q, const double* u, double dt) {
    for (int b = 0; b < sc->n_bodies; ++b) {
        if (sc->fixed[b]) continue;
        const double* vb = u + 6 * b;
        const double* wb = u + 6 * b + 3;
        for (int a = 0; a < 3; ++a) r[3 * b + a] = r[3 * b + a] + vb[a] * dt;
        double qw[4] = {0.0, wb[0], wb[1], wb[2]};
        double dq[4], qn[4];
        quat_prod(qw, q + 4 * b, dq);
        for (int a = 0; a < 4; ++a) qn[a] = q[4 * b + a] + (dq[a] * dt) * 0.5;
        quat_unit(qn, q + 4 * b);
    }
}

/* state_storage.py:188 compute_total_energy and contacts.py:222 get_largest_penetration */
static void energies(const OScene* sc, const double* r, const double* q, const double* v, const double* w,
                     double* kin, double* pot) {
    double G[3] = {0.0, 0.0, 0.0};
    int has_gravity = 0;
    for (int f = 0; f < sc->n_forces; ++f)
        if (sc->force_kind[f] == 0) {
            const double* fp = sc->force_params + 4 * f;
            for (int a = 0; a < 3; ++a) G[a] = G[a] + fp[1 + a] * fp[0];
            has_gravity = 1;
        }
    double kinetic = 0.0, potential = 0.0;
    for (int b = 0; b < sc->n_bodies; ++b) {
        if (sc->fixed[b]) continue;
        double R[9], Iw[9], Iw_w[3];
        quat_to_matrix(q + 4 * b, R);
        update_inertia_tensor(R, sc->inertia + 3 * b, Iw);
        if (has_gravity) {
            double ln = norm3_np(G);
            double up[3] = {G[0] / ln, G[1] / ln, G[2] / ln};
            double g = norm3_np(G);
            double h = dot3_np(up, r + 3 * b);
            potential += sc->mass[b] * g * h;
        }
        gemv3_np(Iw, w + 3 * b, Iw_w);
        double wIw = dot3_np(w + 3 * b, Iw_w);
        kinetic += 0.5 * (sc->mass[b] * dot3_np(v + 3 * b, v + 3 * b) + wIw);
    }
    *kin = kinetic; *pot = potential;
}

/* ------------------------------------------------------------------------------------------------------ */
/* One time step: rainbow/simulators/prox_rigid_bodies/steppers.py:47 SemiImplicitStepper.step            */
/* State arrays r (3N), q (4N), v (3N), w (3N) are updated in place.                                       */
/* Returns 0 on success, 1 on contact capacity overflow (outputs truncated; state still advanced),        */
/* 2 if a non-fixed body has zero mass (state_storage.py:170-171), 3 on a non-unit normal (types.py:293).  */
/* ------------------------------------------------------------------------------------------------------ */
int rbo_step(const OScene* sc, const double* params, double dt, double* r, double* q, double* v, double* w,
             OStepOut* out, int tol_mode, double tol) {
    const int N = sc->n_bodies;
    for (int b = 0; b < N; ++b) if (!sc->fixed[b] && sc->mass[b] == 0.0) return 2;
    out->n_contacts = 0; out->iterations = -1; out->exitcode = -1; out->post_iterations = -1;
    out->post_exitcode = -1; out->overflow = 0; out->n_overlap_pairs = 0; out->n_leaf_overlaps = 0;
    out->n_candidates = 0; out->n_colours = 0;
    double* dux = (double*)malloc(sizeof(double) * 6 * N);
    double* Winv = (double*)malloc(sizeof(double) * 9 * N);
    double* u = (double*)malloc(sizeof(double) * 6 * N);
    double* du = (double*)malloc(sizeof(double) * 6 * N);
    for (int b = 0; b < N; ++b)
        for (int a = 0; a < 3; ++a) { u[6 * b + a] = v[3 * b + a]; u[6 * b + 3 + a] = w[3 * b + a]; }
    external_forces(sc, r, q, v, w, dux, Winv);
    if (out->delta_u_ext) memcpy(out->delta_u_ext, dux, sizeof(double) * 6 * N);
    for (int i = 0; i < 6 * N; ++i) du[i] = dt * dux[i];

    const int H = sc->n_hinges;
    /* hinges are solved by the reference stepper's own Gauss-Seidel rule only */
    if (H > 0 && (out->scheme != S_RIGID_GS || tol_mode != 0 || g_ordering != 0)) {
        free(dux); free(Winv); free(u); free(du);
        return 4;
    }
    ContactList cl = {0, 0, NULL, NULL, NULL, NULL, NULL};
    run_collision_detection(sc, params, r, q, &cl, out);
    const int K = cl.n;
    for (int k = 0; k < K; ++k) {
        double ln = norm3_np(cl.n_ + 3 * k);
        if (fabs(1.0 - ln) > 0.1) {
            free(cl.ids); free(cl.p); free(cl.n_); free(cl.g); free(cl.key);
            free(dux); free(Winv); free(u); free(du);
            return 3;
        }
    }
    Problem P;
    memset(&P, 0, sizeof(P));
    double *b = NULL, *diag = NULL, *rr = NULL, *x = NULL, *sol = NULL, *mu = NULL;
    /* hinges.py:28-50 Hinges.initialize */
    HProblem HP;
    memset(&HP, 0, sizeof(HP));
    double *hb = NULL, *hdiag = NULL, *hr = NULL, *hx = NULL, *hsol = NULL;
    if (H > 0) {
        hinge_build(&HP, sc, q, Winv);
        hb = (double*)malloc(sizeof(double) * 5 * H);
        hdiag = (double*)malloc(sizeof(double) * 5 * H);
        hr = (double*)malloc(sizeof(double) * 5 * H);
        hx = (double*)calloc((size_t)5 * H, sizeof(double));
        hsol = (double*)calloc((size_t)5 * H, sizeof(double));
        double* g = (double*)malloc(sizeof(double) * 5 * H);
        double* dtd = (double*)malloc(sizeof(double) * 6 * N);
        for (int i = 0; i < 6 * N; ++i) dtd[i] = dt * dux[i];
        hinge_error(sc, params, dt, r, q, g);
        for (int k = 0; k < H; ++k)
            for (int i = 0; i < 5; ++i)
                hb[5 * k + i] = (hrow_dot(&HP, k, i, u) + hrow_dot(&HP, k, i, dtd)) + g[5 * k + i];
        /* diag = sum(J .* WJT^T, axis=1), zero entries replaced by 1; r = 1 / diag */
        for (int k = 0; k < H; ++k)
            for (int row = 0; row < 5; ++row) {
                const double* Jr = HP.J + 60 * k + 12 * row;
                const double* Wr = HP.WJT + 60 * k + 12 * row;
                double prods[12];
                int m = 0;
                for (int c = 0; c < 12; ++c) {
                    if (!HP.has_w[2 * k + c / 6]) continue;
                    const double prod = Jr[c] * Wr[c];
                    if (prod != 0.0) prods[m++] = prod;
                }
                const double sd = np_reduce_sum(prods, m);
                hdiag[5 * k + row] = sd == 0.0 ? 1.0 : sd;
            }
        for (int i = 0; i < 5 * H; ++i) hr[i] = 1.0 / hdiag[i];
        free(g); free(dtd);
    }
    if (K > 0) {
        problem_build(&P, sc, &cl, r, Winv);
        b = (double*)malloc(sizeof(double) * 4 * K);
        diag = (double*)malloc(sizeof(double) * 4 * K);
        rr = (double*)malloc(sizeof(double) * 4 * K);
        x = (double*)calloc((size_t)4 * K, sizeof(double));
        sol = (double*)calloc((size_t)4 * K, sizeof(double));
        mu = (double*)malloc(sizeof(double) * K);
        if (out->warm_count > 0 && out->warm_key && out->warm_sol) {
            /* warm start: x = sol = the cached impulses of the contact with the same key (binary search) */
            for (int k = 0; k < K; ++k) {
                const int64_t k1 = cl.key[2 * k], k2 = cl.key[2 * k + 1];
                int lo_i = 0, hi_i = out->warm_count;
                while (lo_i < hi_i) {
                    const int mid = (lo_i + hi_i) >> 1;
                    const int64_t m1 = out->warm_key[2 * mid], m2 = out->warm_key[2 * mid + 1];
                    if (m1 < k1 || (m1 == k1 && m2 < k2)) lo_i = mid + 1; else hi_i = mid;
                }
                if (lo_i < out->warm_count && out->warm_key[2 * lo_i] == k1 && out->warm_key[2 * lo_i + 1] == k2)
                    for (int i = 0; i < 4; ++i) x[4 * k + i] = sol[4 * k + i] = out->warm_sol[4 * lo_i + i];
            }
        }
        double* vv = (double*)malloc(sizeof(double) * 4 * K);
        double* jd = (double*)malloc(sizeof(double) * 4 * K);
        double* dtd = (double*)malloc(sizeof(double) * 6 * N);
        for (int i = 0; i < 6 * N; ++i) dtd[i] = dt * dux[i];
        const int M = sc->n_materials;
        for (int k = 0; k < K; ++k) {
            const int A = cl.ids[2 * k], B = cl.ids[2 * k + 1];
            const int ma = sc->material[A], mb = sc->material[B];
            mu[k] = sc->material_mu[3 * (ma * M + mb)];
            const double eps = params[P_USE_BOUNCE] != 0.0 ? sc->material_eps[ma * M + mb] : 0.0;
            for (int i = 0; i < 4; ++i) {
                vv[4 * k + i] = jrow_dot(&P, k, i, u);
                jd[4 * k + i] = jrow_dot(&P, k, i, dtd);
            }
            /* contacts.py:188 pre-stabilisation error vector */
            double gk[4] = {0.0, 0.0, 0.0, 0.0};
            if (params[P_USE_PRE] != 0.0) {
                const double rate = params[P_GAP_REDUCTION] / dt;
                const double upper = -params[P_MAX_GAP] / dt;
                const double lower = -params[P_MIN_GAP];
                if (cl.g[k] < lower && vv[4 * k] <= 0.0) {
                    double t = rate * cl.g[k];
                    gk[0] = upper > t ? upper : t;
                }
            }
            const double e4[4] = {eps, 0.0, 0.0, 0.0};
            for (int i = 0; i < 4; ++i) b[4 * k + i] = ((1.0 + e4[i]) * vv[4 * k + i] + jd[4 * k + i]) + gk[i];
        }
        free(vv); free(jd); free(dtd);
        problem_diag(&P, diag);
        {
            /* fixed-r rule: r = relaxation / diag (1/diag without relaxation) */
            const double om = (tol_mode == 2 && g_relaxation > 0.0) ? g_relaxation : 1.0;
            for (int i = 0; i < 4 * K; ++i) rr[i] = om / diag[i];
        }
        g_residual_diag = diag;

        int iters = 0, exitc = 0;
        /* graph-coloured visiting order: always for S_COLOURED_GS, on request for the other Gauss-Seidel schemes */
        int32_t* clist = NULL;
        const int coloured = out->scheme == S_COLOURED_GS ||
                             (g_ordering == 1 && (out->scheme == S_RIGID_GS || out->scheme == S_IFACE_GS));
        if (coloured && K > 0) {
            int32_t* colour = (int32_t*)malloc(sizeof(int32_t) * K);
            const int nc = rbo_colour_contacts(K, N, cl.ids, sc->fixed, colour);
            int32_t* cptr = (int32_t*)calloc((size_t)nc + 1, sizeof(int32_t));
            clist = (int32_t*)malloc(sizeof(int32_t) * K);
            for (int k = 0; k < K; ++k) cptr[colour[k] + 1]++;
            for (int c = 0; c < nc; ++c) cptr[c + 1] += cptr[c];
            for (int k = 0; k < K; ++k) clist[cptr[colour[k]]++] = k;   /* ascending within a colour */
            free(colour); free(cptr);
            out->n_colours = nc;
        }
        if (H > 0)
            solve_problems(&P, rr, b, mu, x, sol, &HP, hr, hb, hx, hsol, params, out->residuals, &iters, &exitc);
        else if (out->scheme == S_RIGID_GS)
            solve_rigid(&P, params, rr, b, mu, x, sol, out->residuals, &iters, &exitc, 0, tol_mode, tol, clist);
        else
            solve_interface(&P, params, out->scheme, diag, b, mu, x, sol, out->residuals, &iters, &exitc, clist,
                            tol_mode, tol);
        free(clist);
        out->iterations = iters; out->exitcode = exitc;
        /* finalize (contacts.py:57) and delta_u += WJT sol (steppers.py:84-85) */
        double* dc = (double*)malloc(sizeof(double) * 6 * N);
        wjt_dot(&P, sol, dc);
        for (int i = 0; i < 6 * N; ++i) du[i] = du[i] + dc[i];
        free(dc);
    } else if (H > 0) {
        int iters = 0, exitc = 0;
        solve_problems(NULL, NULL, NULL, NULL, NULL, NULL, &HP, hr, hb, hx, hsol, params, out->residuals, &iters,
                       &exitc);
        out->iterations = iters; out->exitcode = exitc;
    }
    if (H > 0) {   /* hinges.py:52 finalize_solution, added after the contacts' (steppers.py:84-85) */
        double* dh = (double*)malloc(sizeof(double) * 6 * N);
        hinge_wjt_dot(&HP, hsol, dh);
        for (int i = 0; i < 6 * N; ++i) du[i] = du[i] + dh[i];
        free(dh);
        if (out->hinge_b) memcpy(out->hinge_b, hb, sizeof(double) * 5 * H);
        if (out->hinge_diag) memcpy(out->hinge_diag, hdiag, sizeof(double) * 5 * H);
        if (out->hinge_sol) memcpy(out->hinge_sol, hsol, sizeof(double) * 5 * H);
        hinge_free(&HP);
        free(hb); free(hdiag); free(hr); free(hx); free(hsol);
    }
    /* state_storage.py:239 velocity_update, :251 position_update */
    for (int i = 0; i < 6 * N; ++i) u[i] = u[i] + du[i];
    position_update(sc, r, q, u, dt);
    /* steppers.py:15 post-stabilisation */
    if (K > 0 && params[P_USE_POST] != 0.0) {
        double* g = (double*)calloc((size_t)4 * K, sizeof(double));
        int any = 0;
        for (int k = 0; k < K; ++k) if (cl.g[k] < -params[P_MIN_GAP]) { g[4 * k] = cl.g[k]; any = 1; }
        if (any) {
            double* pr = (double*)malloc(sizeof(double) * 4 * K);
            double* px = (double*)calloc((size_t)4 * K, sizeof(double));
            double* ps = (double*)calloc((size_t)4 * K, sizeof(double));
            for (int i = 0; i < 4 * K; ++i) pr[i] = 1.0 / diag[i];
            int it2 = 0, ex2 = 0;
            solve_rigid(&P, params, pr, g, mu, px, ps, NULL, &it2, &ex2, 1, 0, 0.0, NULL);
            out->post_iterations = it2; out->post_exitcode = ex2;
            double* dr = (double*)malloc(sizeof(double) * 6 * N);
            wjt_dot(&P, ps, dr);
            position_update(sc, r, q, dr, 1.0);
            free(pr); free(px); free(ps); free(dr);
        }
        free(g);
    }
    for (int b2 = 0; b2 < N; ++b2)
        for (int a = 0; a < 3; ++a) { v[3 * b2 + a] = u[6 * b2 + a]; w[3 * b2 + a] = u[6 * b2 + 3 + a]; }
    /* outputs */
    out->n_contacts = K;
    if (K > out->capacity) out->overflow = 1;
    const int Kc = K < out->capacity ? K : out->capacity;
    if (Kc > 0) {
        if (out->ids) memcpy(out->ids, cl.ids, sizeof(int32_t) * 2 * Kc);
        if (out->p) memcpy(out->p, cl.p, sizeof(double) * 3 * Kc);
        if (out->n) memcpy(out->n, cl.n_, sizeof(double) * 3 * Kc);
        if (out->g) memcpy(out->g, cl.g, sizeof(double) * Kc);
        if (out->b) memcpy(out->b, b, sizeof(double) * 4 * Kc);
        if (out->diag) memcpy(out->diag, diag, sizeof(double) * 4 * Kc);
        if (out->sol) memcpy(out->sol, sol, sizeof(double) * 4 * Kc);
        if (out->keys) memcpy(out->keys, cl.key, sizeof(int64_t) * 2 * Kc);
    }
    double gap = 0.0;
    for (int k = 0; k < K; ++k) if (cl.g[k] < gap) gap = cl.g[k];
    out->max_penetration = -gap;
    energies(sc, r, q, v, w, &out->kinetic, &out->potential);
    if (K > 0) problem_free(&P);
    free(b); free(diag); free(rr); free(x); free(sol); free(mu);
    free(cl.ids); free(cl.p); free(cl.n_); free(cl.g); free(cl.key);
    free(dux); free(Winv); free(u); free(du);
    return out->overflow ? 1 : 0;
}

/* ------------------------------------------------------------------------------------------------------ */
/* Primitive entry points, used to pin the restatement against the reference's own unit-test answers     */
/* ------------------------------------------------------------------------------------------------------ */
void rbo_quat_prod(const double* a, const double* b, double* out) { quat_prod(a, b, out); }
void rbo_quat_rotate(const double* q, const double* r, double* out) { quat_rotate(q, r, out); }
void rbo_quat_rotate_array(const double* q, const double* V, int n, double* out) {
    for (int i = 0; i < n; ++i) quat_rotate_row(q, V + 3 * i, out + 3 * i);
}
void rbo_quat_to_matrix(const double* q, double* R) { quat_to_matrix(q, R); }
void rbo_quat_unit(const double* q, double* out) { quat_unit(q, out); }
void rbo_make_orthonormal_vectors(const double* n, double* t, double* b, double* nn) {
    make_orthonormal_vectors(n, t, b, nn);
}
void rbo_prox_sphere(double zs, double zt, double ztau, double mu, double xn, double* out) {
    prox_sphere(zs, zt, ztau, mu, xn, out);
}
void rbo_update_inertia_tensor(const double* R, const double* Bv, double* W) { update_inertia_tensor(R, Bv, W); }
static void grid_from_meta(Grid* g, const double* values, const double* meta) {
    g->values = values;
    for (int a = 0; a < 3; ++a) { g->mn[a] = meta[a]; g->mx[a] = meta[3 + a]; g->sp[a] = meta[6 + a]; }
    g->I = (long)meta[9]; g->J = (long)meta[10]; g->K = (long)meta[11];
}
double rbo_grid_value(const double* values, const double* meta, const double* p) {
    Grid g; grid_from_meta(&g, values, meta); return grid_value(&g, p);
}
void rbo_grid_gradient(const double* values, const double* meta, const double* p, double* grad) {
    Grid g; grid_from_meta(&g, values, meta); grid_gradient(&g, p, grad);
}
int rbo_grid_is_inside(const double* meta, const double* p, double boundary) {
    Grid g; grid_from_meta(&g, NULL, meta); return grid_is_inside(&g, p, boundary);
}
void rbo_grid_cell(const double* meta, const double* p, int64_t* ijk) {
    Grid g; grid_from_meta(&g, NULL, meta);
    long c[3]; grid_cell(&g, p, c);
    ijk[0] = c[0]; ijk[1] = c[1]; ijk[2] = c[2];
}
