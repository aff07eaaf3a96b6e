// rb_device.cuh -- device arithmetic for the prox_rigid_bodies step.
//
// FP64 parity rule: every expression reproduces the rounding sequence NumPy / SciPy execute for the
// reference's Python.  The library is compiled with -fmad=false so that nvcc fuses nothing on its own; the
// fma() calls below are the fusions OpenBLAS performs inside np.dot / np.linalg.norm on 3- and 4-vectors
// (ddot: fma(a2,b2, fma(a1,b1, a0*b0))) and inside np.dot(3x3, 3) (dgemv: fma(m2,v2, fma(m0,v0, m1*v1))).
// Double division and sqrt are IEEE round-to-nearest in CUDA, like the host.
#pragma once
#include <cstdint>

namespace rb {

struct d3 { double x, y, z; };

__device__ __forceinline__ d3 mk(double x, double y, double z) { return d3{x, y, z}; }
__device__ __forceinline__ d3 ld3(const double* p) { return d3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(double* p, d3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
__device__ __forceinline__ d3 sub(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 add(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }

// np.dot(a, b) on 3-vectors (OpenBLAS ddot)
__device__ __forceinline__ double dot3_np(d3 a, d3 b) { return fma(a.z, b.z, fma(a.y, b.y, a.x * b.x)); }
__device__ __forceinline__ double norm3_np(d3 a) { return sqrt(dot3_np(a, a)); }
__device__ __forceinline__ double dot4_np(const double* a, const double* b) {
    return fma(a[3], b[3], fma(a[2], b[2], fma(a[1], b[1], a[0] * b[0])));
}
// np.cross (numpy/_core/numeric.py: cp0 = a1*b2 - a2*b1, ...)
__device__ __forceinline__ d3 cross_np(d3 a, d3 b) {
    return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// np.dot(M, v), M C-ordered 3x3 (OpenBLAS dgemv)
__device__ __forceinline__ d3 gemv3_np(const double* M, d3 v) {
    return d3{fma(M[2], v.z, fma(M[0], v.x, M[1] * v.y)), fma(M[5], v.z, fma(M[3], v.x, M[4] * v.y)),
              fma(M[8], v.z, fma(M[6], v.x, M[7] * v.y))};
}

// quaternion.py:76 unit
__device__ __forceinline__ void quat_unit(const double* q, double* o) {
    double l = sqrt(dot4_np(q, q));
    if (l > 0.0) {
        double a = q[0] / l, b = q[1] / l, c = q[2] / l, d = q[3] / l;
        o[0] = a; o[1] = b; o[2] = c; o[3] = d;
    } else {
        o[0] = 1.0; o[1] = 0.0; o[2] = 0.0; o[3] = 0.0;
    }
}
// quaternion.py:186 prod: qs = a*b - dot(A,B); qv = (a*B + A*b) + cross(A,B)
__device__ __forceinline__ void quat_prod(const double* qa, const double* qb, double* o) {
    const double a = qa[0], b = qb[0];
    const d3 A = d3{qa[1], qa[2], qa[3]}, B = d3{qb[1], qb[2], qb[3]};
    const double qs = a * b - dot3_np(A, B);
    const d3 c = cross_np(A, B);
    const double v0 = (a * B.x + A.x * b) + c.x;
    const double v1 = (a * B.y + A.y * b) + c.y;
    const double v2 = (a * B.z + A.z * b) + c.z;
    o[0] = qs; o[1] = v0; o[2] = v1; o[3] = v2;
}
// quaternion.py:196 rotate = vector part of prod(prod(q, [0, r]), conjugate(q))
__device__ __forceinline__ d3 quat_rotate(const double* q, d3 r) {
    const double qr[4] = {0.0, r.x, r.y, r.z};
    const double cq[4] = {q[0], -q[1], -q[2], -q[3]};
    double t[4], u[4];
    quat_prod(q, qr, t);
    quat_prod(t, cq, u);
    return d3{u[1], u[2], u[3]};
}
// quaternion.py:244 rotate_array, one row, via prod_array (:201-241)
__device__ __forceinline__ d3 quat_rotate_row(const double* q, d3 p) {
    const double x = p.x, y = p.y, z = p.z;
    const double a0 = ((q[0] * 0.0 - q[1] * x) - q[2] * y) - q[3] * z;
    const double a1 = ((q[0] * x + q[1] * 0.0) + q[2] * z) - q[3] * y;
    const double a2 = ((q[0] * y - q[1] * z) + q[2] * 0.0) + q[3] * x;
    const double a3 = ((q[0] * z + q[1] * y) - q[2] * x) + q[3] * 0.0;
    const double c0 = q[0], c1 = -q[1], c2 = -q[2], c3 = -q[3];
    return d3{((a0 * c1 + a1 * c0) + a2 * c3) - a3 * c2, ((a0 * c2 - a1 * c3) + a2 * c0) + a3 * c1,
              ((a0 * c3 + a1 * c2) - a2 * c1) + a3 * c0};
}
// quaternion.py:108 to_matrix (row-major 3x3)
__device__ __forceinline__ void quat_to_matrix(const double* Q, double* R) {
    double q[4];
    quat_unit(Q, q);
    const double qs = q[0], qx = q[1], qy = q[2], qz = q[3];
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
// mass.py:395 update_inertia_tensor: W = R diag(Bv) R^T with the reference's term order
__device__ __forceinline__ void update_inertia_tensor(const double* R, const double* Bv, double* W) {
    const double w00 = (R[0] * R[0] * Bv[0] + R[1] * R[1] * Bv[1]) + R[2] * R[2] * Bv[2];
    const double w11 = (R[3] * R[3] * Bv[0] + R[4] * R[4] * Bv[1]) + R[5] * R[5] * Bv[2];
    const double w22 = (R[6] * R[6] * Bv[0] + R[7] * R[7] * Bv[1]) + R[8] * R[8] * Bv[2];
    const double w10 = (R[3] * R[0] * Bv[0] + R[4] * R[1] * Bv[1]) + R[5] * R[2] * Bv[2];
    const double w20 = (R[6] * R[0] * Bv[0] + R[7] * R[1] * Bv[1]) + R[8] * R[2] * Bv[2];
    const double w21 = (R[3] * R[6] * Bv[0] + R[4] * R[7] * Bv[1]) + R[5] * R[8] * Bv[2];
    W[0] = w00; W[4] = w11; W[8] = w22;
    W[1] = w10; W[3] = w10;
    W[2] = w20; W[6] = w20;
    W[5] = w21; W[7] = w21;
}
// vector3.py:75 make_orthonormal_vectors -> (t, b, n)
__device__ __forceinline__ void make_orthonormal_vectors(d3 nin, d3& t, d3& b, d3& n) {
    const double l = norm3_np(nin);
    n = d3{nin.x / l, nin.y / l, nin.z / l};
    const double nx = fabs(n.x), ny = fabs(n.y), nz = fabs(n.z);
    d3 tg = d3{0.0, 0.0, 0.0};
    if (nx <= ny && nx <= nz) tg = d3{1.0, 0.0, 0.0};
    if (ny <= nx && ny <= nz) tg = d3{0.0, 1.0, 0.0};
    if (nz <= nx && nz <= ny) tg = d3{0.0, 0.0, 1.0};
    d3 bb = cross_np(n, tg);
    const double lb = norm3_np(bb);
    b = d3{bb.x / lb, bb.y / lb, bb.z / lb};
    t = cross_np(b, n);
}
// prox_operators.py:14 prox_sphere
__device__ __forceinline__ void prox_sphere(double zs, double zt, double ztau, double mu, double xn, double* o) {
    if (xn <= 0.0) { o[0] = 0.0; o[1] = 0.0; o[2] = 0.0; return; }
    const double radius = mu * xn;
    const double sqr = zs * zs + zt * zt + ztau * ztau;
    if (sqr <= radius * radius) { o[0] = zs; o[1] = zt; o[2] = ztau; return; }
    const double scale = radius / sqrt(sqr);
    o[0] = zs * scale; o[1] = zt * scale; o[2] = ztau * scale;
}

// ---------------------------------------------------------------------------------------------------------
// Signed distance grid (grid3.py)
// ---------------------------------------------------------------------------------------------------------
struct GridView {
    const double* values;
    double mn[3], mx[3], sp[3];
    int I, J, K;
};
__device__ __forceinline__ GridView load_grid(const double* meta, const double* values) {
    GridView g;
    g.values = values;
#pragma unroll
    for (int a = 0; a < 3; ++a) { g.mn[a] = meta[a]; g.mx[a] = meta[3 + a]; g.sp[a] = meta[6 + a]; }
    g.I = (int)meta[9]; g.J = (int)meta[10]; g.K = (int)meta[11];
    return g;
}
// grid3.py:107 get_enclosing_cell_idx (floor, then clip to [0, n-2])
__device__ __forceinline__ int cell_index(double p, double mn, double sp, int n) {
    const double f = floor((p - mn) / sp);
    const int lim = n - 2;
    if (!(f >= 0.0)) return 0;
    if (f > (double)lim) return lim;
    return (int)f;
}
struct Corners { double d000, d001, d010, d011, d100, d101, d110, d111; int i, j, k; };
__device__ __forceinline__ Corners load_corners(const GridView& g, d3 p) {
    Corners c;
    c.i = cell_index(p.x, g.mn[0], g.sp[0], g.I);
    c.j = cell_index(p.y, g.mn[1], g.sp[1], g.J);
    c.k = cell_index(p.z, g.mn[2], g.sp[2], g.K);
    const int64_t I = g.I, IJ = (int64_t)g.I * g.J;
    const double* v = g.values + c.i + I * c.j + IJ * c.k;
    c.d000 = __ldg(v);
    c.d100 = __ldg(v + 1);
    c.d010 = __ldg(v + I);
    c.d110 = __ldg(v + I + 1);
    c.d001 = __ldg(v + IJ);
    c.d101 = __ldg(v + IJ + 1);
    c.d011 = __ldg(v + IJ + I);
    c.d111 = __ldg(v + IJ + I + 1);
    return c;
}
// grid3.py:126 get_value
__device__ __forceinline__ double grid_value(const GridView& g, d3 p) {
    const Corners c = load_corners(g, p);
    const double s = (p.x - (((double)c.i * g.sp[0]) + g.mn[0])) / g.sp[0];
    const double t = (p.y - (((double)c.j * g.sp[1]) + g.mn[1])) / g.sp[1];
    const double u = (p.z - (((double)c.k * g.sp[2]) + g.mn[2])) / g.sp[2];
    const double x00 = (c.d100 - c.d000) * s + c.d000;
    const double x01 = (c.d101 - c.d001) * s + c.d001;
    const double x10 = (c.d110 - c.d010) * s + c.d010;
    const double x11 = (c.d111 - c.d011) * s + c.d011;
    const double y0 = (x10 - x00) * t + x00;
    const double y1 = (x11 - x01) * t + x01;
    return (y1 - y0) * u + y0;
}
// grid3.py:180 get_gradient, including the reference's division of s, t, u by min_coord (:209-211)
__device__ __forceinline__ d3 grid_gradient(const GridView& g, d3 p) {
    const Corners c = load_corners(g, p);
    const double s = (p.x - ((double)c.i * g.sp[0] + g.mn[0])) / g.mn[0];
    const double t = (p.y - ((double)c.j * g.sp[1] + g.mn[1])) / g.mn[1];
    const double u = (p.z - ((double)c.k * g.sp[2] + g.mn[2])) / g.mn[2];
    const double x00 = (c.d100 - c.d000) * s + c.d000;
    const double x01 = (c.d101 - c.d001) * s + c.d001;
    const double x10 = (c.d110 - c.d010) * s + c.d010;
    const double x11 = (c.d111 - c.d011) * s + c.d011;
    const double y0 = (x10 - x00) * t + x00;
    const double y1 = (x11 - x01) * t + x01;
    const double dx00 = c.d100 - c.d000, dx01 = c.d101 - c.d001, dx10 = c.d110 - c.d010, dx11 = c.d111 - c.d011;
    const double dy0_ds = (dx10 - dx00) * t + dx00;
    const double dy1_ds = (dx11 - dx01) * t + dx01;
    const double dy0_dt = x10 - x00;
    const double dy1_dt = x11 - x01;
    const double dp_ds = (dy1_ds - dy0_ds) * u + dy0_ds;
    const double dp_dt = (dy1_dt - dy0_dt) * u + dy0_dt;
    const double dp_du = y1 - y0;
    return d3{dp_ds * (1.0 / g.sp[0]), dp_dt * (1.0 / g.sp[1]), dp_du * (1.0 / g.sp[2])};
}
// grid3.py:275 is_inside
__device__ __forceinline__ bool grid_is_inside(const GridView& g, d3 p, double boundary) {
    if (p.x > (g.mx[0] - boundary)) return false;
    if (p.y > (g.mx[1] - boundary)) return false;
    if (p.z > (g.mx[2] - boundary)) return false;
    if (p.x < (g.mn[0] + boundary)) return false;
    if (p.y < (g.mn[1] + boundary)) return false;
    if (p.z < (g.mn[2] + boundary)) return false;
    return true;
}

// Gradient from the FP32 copy of a grid (the contact search of the FP32 precision modes): the cell and the
// fractions s, t, u in FP64 exactly as grid_gradient computes them (so the cell is always the FP64 lookup's,
// grid3.py:107, and the min_coord divisor of :209-211 is kept), the eight corner values and their trilinear
// combination in FP32.  err bounds the absolute difference of each component from grid_gradient's: the FP32
// rounding of the values (at most 2^-24 |v|) and of the combination, amplified by the weights (1 - s, s) ...,
// which the min_coord divisor can take outside [0, 1].
__device__ __forceinline__ d3 grid_gradient_f32(const GridView& g, const float* values32, d3 p, double& err) {
    const int i = cell_index(p.x, g.mn[0], g.sp[0], g.I);
    const int j = cell_index(p.y, g.mn[1], g.sp[1], g.J);
    const int k = cell_index(p.z, g.mn[2], g.sp[2], g.K);
    const int64_t I = g.I, IJ = (int64_t)g.I * g.J;
    const float* v = values32 + i + I * j + IJ * k;
    const float d000 = __ldg(v), d100 = __ldg(v + 1), d010 = __ldg(v + I), d110 = __ldg(v + I + 1);
    const float d001 = __ldg(v + IJ), d101 = __ldg(v + IJ + 1), d011 = __ldg(v + IJ + I), d111 = __ldg(v + IJ + I + 1);
    const double sd = (p.x - ((double)i * g.sp[0] + g.mn[0])) / g.mn[0];
    const double td = (p.y - ((double)j * g.sp[1] + g.mn[1])) / g.mn[1];
    const double ud = (p.z - ((double)k * g.sp[2] + g.mn[2])) / g.mn[2];
    const float s = (float)sd, t = (float)td, u = (float)ud;
    const float x00 = (d100 - d000) * s + d000, x01 = (d101 - d001) * s + d001;
    const float x10 = (d110 - d010) * s + d010, x11 = (d111 - d011) * s + d011;
    const float y0 = (x10 - x00) * t + x00, y1 = (x11 - x01) * t + x01;
    const float dx00 = d100 - d000, dx01 = d101 - d001, dx10 = d110 - d010, dx11 = d111 - d011;
    const float dy0_ds = (dx10 - dx00) * t + dx00, dy1_ds = (dx11 - dx01) * t + dx01;
    const float dy0_dt = x10 - x00, dy1_dt = x11 - x01;
    const float dp_ds = (dy1_ds - dy0_ds) * u + dy0_ds;
    const float dp_dt = (dy1_dt - dy0_dt) * u + dy0_dt;
    const float dp_du = y1 - y0;
    float vmax = fmaxf(fmaxf(fmaxf(fabsf(d000), fabsf(d100)), fmaxf(fabsf(d010), fabsf(d110))),
                       fmaxf(fmaxf(fabsf(d001), fabsf(d101)), fmaxf(fabsf(d011), fabsf(d111))));
    const double amp = (1.0 + 2.0 * fabs(sd)) * (1.0 + 2.0 * fabs(td)) * (1.0 + 2.0 * fabs(ud));
    const double sp_min = fmin(g.sp[0], fmin(g.sp[1], g.sp[2]));
    err = 64.0 * 5.9604644775390625e-8 * (double)vmax * amp / sp_min;   // 64 x 2^-24 x ...
    return d3{(double)dp_ds * (1.0 / g.sp[0]), (double)dp_dt * (1.0 / g.sp[1]), (double)dp_du * (1.0 / g.sp[2])};
}

// NumPy np.add.reduceat over one segment: a[0] + pairwise_sum(a[1:]) (8 interleaved partial sums once the
// remainder holds at least 8 values).  Used for the Delassus diagonal (contacts.py:49).
__device__ __forceinline__ double np_reduce_sum(const double* a, int m) {
    if (m <= 0) return 0.0;
    const int n = m - 1;
    const double* rest = a + 1;
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

struct AABB { double lo[3], hi[3]; };
__device__ __forceinline__ bool overlap(const double* a, const double* b) {
    // kdop.py:21 overlap on axis slabs (K = 3); a, b = lo[3], hi[3]
    return !(a[3] < b[0] || b[3] < a[0] || a[4] < b[1] || b[4] < a[1] || a[5] < b[2] || b[5] < a[2]);
}

}  // namespace rb
