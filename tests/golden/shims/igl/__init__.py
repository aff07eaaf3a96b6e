"""Stand-in for ``igl.signed_distance`` used only when generating golden fixtures.

The reference builds each shape's signed-distance grid with libigl (``rainbow/geometry/grid3.py:338``), which is
not installed here.  This module restates the computation from its mathematics:

* unsigned distance: brute force over all triangles of the closest point on a triangle, following the Voronoi
  region case analysis of Ericson, *Real-Time Collision Detection* (2005), section 5.1.5;
* sign: the generalized winding number, summing each triangle's signed solid angle by the formula of
  Van Oosterom & Strackee (1983); points with |winding number| > 1/2 are inside and get a negative distance.

The grid values are an input of the time step (the oracle and the GPU read the same stored values), so this
stand-in changes which grid a scene uses, not how the step is computed.
"""
import numpy as np


def _closest_points(P, a, b, c):
    ab = b - a
    ac = c - a
    ap = P - a
    d1 = ap @ ab
    d2 = ap @ ac
    bp = P - b
    d3 = bp @ ab
    d4 = bp @ ac
    cp = P - c
    d5 = cp @ ab
    d6 = cp @ ac
    va = d3 * d6 - d5 * d4
    vb = d5 * d2 - d1 * d6
    vc = d1 * d4 - d3 * d2

    def safe(num, den):
        return num / np.where(den == 0.0, 1.0, den)

    # interior of the face
    denom = va + vb + vc
    v = safe(vb, denom)
    w = safe(vc, denom)
    Q = a + v[:, None] * ab + w[:, None] * ac
    # edge regions
    m = (vc <= 0) & (d1 >= 0) & (d3 <= 0)
    t = safe(d1, d1 - d3)
    Q = np.where(m[:, None], a + t[:, None] * ab, Q)
    m = (vb <= 0) & (d2 >= 0) & (d6 <= 0)
    t = safe(d2, d2 - d6)
    Q = np.where(m[:, None], a + t[:, None] * ac, Q)
    m = (va <= 0) & ((d4 - d3) >= 0) & ((d5 - d6) >= 0)
    t = safe(d4 - d3, (d4 - d3) + (d5 - d6))
    Q = np.where(m[:, None], b + t[:, None] * (c - b), Q)
    # vertex regions take precedence
    Q = np.where(((d1 <= 0) & (d2 <= 0))[:, None], a, Q)
    Q = np.where(((d3 >= 0) & (d4 <= d3))[:, None], b, Q)
    Q = np.where(((d6 >= 0) & (d5 <= d6))[:, None], c, Q)
    return Q


def signed_distance(P, V, F, *args, **kwargs):
    P = np.asarray(P, dtype=np.float64)
    V = np.asarray(V, dtype=np.float64)
    best = np.full(len(P), np.inf)
    closest_face = np.zeros(len(P), dtype=np.int64)
    closest_point = np.zeros_like(P)
    winding = np.zeros(len(P))
    for f, tri in enumerate(np.asarray(F)):
        a, b, c = V[tri[0]], V[tri[1]], V[tri[2]]
        Q = _closest_points(P, a, b, c)
        d = np.linalg.norm(P - Q, axis=1)
        better = d < best
        best = np.where(better, d, best)
        closest_face = np.where(better, f, closest_face)
        closest_point = np.where(better[:, None], Q, closest_point)
        A = a - P
        B = b - P
        C = c - P
        la = np.linalg.norm(A, axis=1)
        lb = np.linalg.norm(B, axis=1)
        lc = np.linalg.norm(C, axis=1)
        num = np.einsum("ij,ij->i", A, np.cross(B, C))
        den = (la * lb * lc + np.einsum("ij,ij->i", A, B) * lc + np.einsum("ij,ij->i", B, C) * la
               + np.einsum("ij,ij->i", C, A) * lb)
        winding += 2.0 * np.arctan2(num, den)
    sign = np.where(np.abs(winding) / (4.0 * np.pi) > 0.5, -1.0, 1.0)
    return sign * best, closest_face, closest_point
