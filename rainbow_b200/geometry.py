"""Scene set-up geometry: mesh generators, PCA vertex ordering, mass properties, signed distance grids.

These run once per shape, before any time step, and restate the set-up side of the reference:
``rainbow/geometry/surface_mesh.py`` (create_box :286, create_sphere :211, profile_sweep :85, axis_sort :56),
``rainbow/math/functions.py`` (direction_of_most_variance), ``rainbow/simulators/prox_rigid_bodies/mass.py``
(compute_mass_properties :138, xform_model_2_body_space :366) and ``rainbow/geometry/grid3.py:320``
(create_signed_distance, whose distance field is computed here by the CUDA kernel rb_signed_distance_grid).
"""
import ctypes
from math import cos, sin, sqrt

import numpy as np

from .types import Grid, Mesh


# ------------------------------------------------------------------------------------------------------------
# quaternions used by set-up (Hamilton product, [s, x, y, z])
# ------------------------------------------------------------------------------------------------------------
def quat_prod(a, b):
    s = a[0] * b[0] - np.dot(a[1:], b[1:])
    v = a[0] * b[1:] + a[1:] * b[0] + np.cross(a[1:], b[1:])
    return np.array([s, v[0], v[1], v[2]], dtype=np.float64)


def quat_conj(q):
    return np.array([q[0], -q[1], -q[2], -q[3]], dtype=np.float64)


def quat_rotate(q, r):
    return quat_prod(quat_prod(q, np.array([0.0, r[0], r[1], r[2]])), quat_conj(q))[1:]


def quat_rotate_array(q, V):
    """Rotate every row of V by q (quaternion.py:244 rotate_array, same per-component evaluation order)."""
    V = np.asarray(V, dtype=np.float64)
    x, y, z = V[:, 0], V[:, 1], V[:, 2]
    a0 = q[0] * 0.0 - q[1] * x - q[2] * y - q[3] * z
    a1 = q[0] * x + q[1] * 0.0 + q[2] * z - q[3] * y
    a2 = q[0] * y - q[1] * z + q[2] * 0.0 + q[3] * x
    a3 = q[0] * z + q[1] * y - q[2] * x + q[3] * 0.0
    c = quat_conj(q)
    return np.stack([a0 * c[1] + a1 * c[0] + a2 * c[3] - a3 * c[2],
                     a0 * c[2] - a1 * c[3] + a2 * c[0] + a3 * c[1],
                     a0 * c[3] + a1 * c[2] - a2 * c[1] + a3 * c[0]], axis=1)


def quat_unit(q):
    q = np.asarray(q, dtype=np.float64)
    n = np.linalg.norm(q)
    return q / n if n > 0.0 else np.array([1.0, 0.0, 0.0, 0.0])


def quat_axis_angle(radians, axis):
    c, s = cos(radians / 2.0), sin(radians / 2.0)
    n = np.asarray(axis, dtype=np.float64) / np.linalg.norm(axis)
    return np.array([c, s * n[0], s * n[1], s * n[2]], dtype=np.float64)


def orthonormal_frame(n):
    """(t, b, n) completing the direction n (vector3.py:75 make_orthonormal_vectors): the tangent guess is the
    coordinate axis along the smallest |n_i| (a later tie wins), b = unit(n x t), t = b x n."""
    n = np.asarray(n, dtype=np.float64) / np.linalg.norm(n)
    a = np.fabs(n)
    t = np.zeros(3)
    if a[0] <= a[1] and a[0] <= a[2]:
        t = np.array([1.0, 0.0, 0.0])
    if a[1] <= a[0] and a[1] <= a[2]:
        t = np.array([0.0, 1.0, 0.0])
    if a[2] <= a[0] and a[2] <= a[1]:
        t = np.array([0.0, 0.0, 1.0])
    b = np.cross(n, t)
    b = b / np.linalg.norm(b)
    return np.cross(b, n), b, n


def quat_from_matrix(M):
    """Rotation matrix to quaternion (the trace / largest-diagonal method of quaternion.py:132)."""
    tr = M[0, 0] + M[1, 1] + M[2, 2]
    if tr < 0.0:
        i = 0
        if M[1, 1] > M[0, 0]:
            i = 1
        if M[2, 2] > M[i, i]:
            i = 2
        j, k = (i + 1) % 3, (i + 2) % 3
        r = sqrt((M[i, i] - (M[j, j] + M[k, k])) + 1.0)
        q = np.zeros(4)
        q[1 + i] = 0.5 * r
        r = 0.5 / r
        q[1 + j] = (M[i, j] + M[j, i]) * r
        q[1 + k] = (M[k, i] + M[i, k]) * r
        q[0] = (M[k, j] - M[j, k]) * r
        return q
    r = sqrt(tr + 1.0)
    s = 0.5 / r
    return np.array([0.5 * r, (M[2, 1] - M[1, 2]) * s, (M[0, 2] - M[2, 0]) * s, (M[1, 0] - M[0, 1]) * s])


# ------------------------------------------------------------------------------------------------------------
# mesh generators
# ------------------------------------------------------------------------------------------------------------
def create_box(width, height, depth):
    """Axis-aligned box centred at the origin: 8 vertices, 12 outward triangles (surface_mesh.py:286)."""
    hx, hy, hz = 0.5 * width, 0.5 * height, 0.5 * depth
    V = np.array([[-hx, -hy, -hz], [hx, -hy, -hz], [-hx, hy, -hz], [hx, hy, -hz],
                  [-hx, -hy, hz], [hx, -hy, hz], [-hx, hy, hz], [hx, hy, hz]], dtype=np.float64)
    T = np.array([[0, 2, 3], [0, 3, 1], [4, 5, 7], [4, 7, 6], [1, 3, 7], [1, 7, 5],
                  [0, 4, 6], [0, 6, 2], [0, 1, 5], [0, 5, 4], [3, 2, 6], [3, 6, 7]], dtype=np.int64)
    return V, T


def profile_sweep(profile, slices):
    """Surface of revolution of a profile curve about the y-axis (surface_mesh.py:85)."""
    n = len(profile)
    if n <= 2:
        raise RuntimeError("profile_sweep(): Profile must have at least 3 points")
    if slices <= 2:
        raise RuntimeError("profile_sweep(): Sweep must have at least 3 slices to be a proper volume.")
    rings = n - 2
    nv = rings * slices + 2
    top, bottom = nv - 2, nv - 1
    V = np.zeros((nv, 3))
    rows = []
    for j in range(slices):
        R = quat_axis_angle(j * 2.0 * np.pi / slices, [0.0, 1.0, 0.0])
        for i in range(rings):
            rows.append(quat_rotate(R, profile[i + 1]))
    V[:rings * slices] = np.array(rows)
    V[top] = profile[n - 1]
    V[bottom] = profile[0]
    T = []
    for j in range(slices):
        T.append((bottom, rings * ((j + 1) % slices), rings * j))
    for i in range(rings - 1):
        for j in range(slices):
            l, r = j, (j + 1) % slices
            T.append((l * rings + i, r * rings + i, r * rings + i + 1))
            T.append((l * rings + i, r * rings + i + 1, l * rings + i + 1))
    for j in range(slices):
        T.append((top, j * rings + (n - 3), ((j + 1) % slices) * rings + (n - 3)))
    return V, np.array(T, dtype=np.int32)


def create_sphere(radius, slices=12, segments=12):
    """Sphere as a swept half circle (surface_mesh.py:211)."""
    profile = []
    for i in range(segments):
        R = quat_axis_angle(np.pi / (segments - 1) * i, [0.0, 0.0, 1.0])
        profile.append(quat_rotate(R, np.array([0.0, -radius, 0.0])))
    return profile_sweep(profile, slices)


# ------------------------------------------------------------------------------------------------------------
# PCA ordering (api.py:159 create_mesh)
# ------------------------------------------------------------------------------------------------------------
def direction_of_most_variance(P):
    """Row of the eigenvector matrix of the covariance at the largest eigenvalue (functions.py)."""
    C = P - np.mean(P.T, axis=1)
    values, vectors = np.linalg.eig(np.cov(C.T))
    return np.real(vectors[np.argmax(np.real(values))])


def axis_sort(mesh, axis):
    """Order vertices by their projection on axis, then triangles by mean vertex index (surface_mesh.py:56)."""
    n = np.asarray(axis, dtype=np.float64) / np.linalg.norm(axis)
    d = np.array([np.dot(v, n) for v in mesh.V])
    new2old = sorted(range(len(mesh.V)), key=lambda k: d[k])
    mesh.V = mesh.V[new2old]
    old2new = np.empty(len(new2old), dtype=np.int64)
    old2new[np.array(new2old)] = np.arange(len(new2old))
    mesh.T = old2new[mesh.T].astype(mesh.T.dtype)
    mean = np.mean(mesh.T, axis=1)
    mesh.T = mesh.T[sorted(range(len(mesh.T)), key=lambda k: mean[k])]
    return mesh


def create_mesh(V, T):
    mesh = Mesh(V, T)
    axis_sort(mesh, direction_of_most_variance(mesh.V))
    return mesh


# ------------------------------------------------------------------------------------------------------------
# mass properties of a closed triangle mesh: Mirtich, "Fast and accurate computation of polyhedral mass
# properties", J. Graphics Tools 1(2), 1996 (the algorithm of mass.py:56-256)
# ------------------------------------------------------------------------------------------------------------
def _projected_face_integrals(a, b):
    """Integrals over the face's projection; a, b: the 3 corner coordinates in the projection plane."""
    P = np.zeros(10)   # P1, Pa, Paa, Paaa, Pb, Pbb, Pbbb, Pab, Paab, Pabb
    for e in range(3):
        a0, b0, a1, b1 = a[e], b[e], a[(e + 1) % 3], b[(e + 1) % 3]
        da, db = a1 - a0, b1 - b0
        a0_2, b0_2, a1_2, b1_2 = a0 * a0, b0 * b0, a1 * a1, b1 * b1
        a0_3, b0_3, a1_3, b1_3 = a0_2 * a0, b0_2 * b0, a1_2 * a1, b1_2 * b1
        C1 = a1 + a0
        Ca = a1 * C1 + a0_2
        Caa = a1 * Ca + a0_3
        Caaa = a1 * Caa + a0_3 * a0
        Cb = b1 * (b1 + b0) + b0_2
        Cbb = b1 * Cb + b0_3
        Cbbb = b1 * Cbb + b0_3 * b0
        Cab = 3.0 * a1_2 + 2.0 * a1 * a0 + a0_2
        Kab = a1_2 + 2.0 * a1 * a0 + 3.0 * a0_2
        Caab = a0 * Cab + 4.0 * a1_3
        Kaab = a1 * Kab + 4.0 * a0_3
        Cabb = 4.0 * b1_3 + 3.0 * b1_2 * b0 + 2.0 * b1 * b0_2 + b0_3
        Kabb = b1_3 + 2.0 * b1_2 * b0 + 3.0 * b1 * b0_2 + 4.0 * b0_3
        P += [db * C1, db * Ca, db * Caa, db * Caaa, da * Cb, da * Cbb, da * Cbbb,
              db * (b1 * Cab + b0 * Kab), db * (b1 * Caab + b0 * Kaab), da * (a1 * Cabb + a0 * Kabb)]
    return P / np.array([2.0, 6.0, 12.0, 20.0, -6.0, -12.0, -20.0, 24.0, 60.0, -60.0])


def compute_mass_properties(V, T, density):
    """Mass, centre of mass and inertia tensor (about the model origin) of a closed mesh."""
    T0, T1, T2, TP = 0.0, np.zeros(3), np.zeros(3), np.zeros(3)
    for tri in np.asarray(T):
        p = V[tri]
        n = np.cross(p[1] - p[0], p[2] - p[0])
        n = n / np.linalg.norm(n)
        w = -np.dot(n, (p[0] + p[1] + p[2]) / 3.0)
        an = np.fabs(n)
        Z = 0 if (an[0] > an[1] and an[0] > an[2]) else (1 if an[1] > an[2] else 2)
        X, Y = (Z + 1) % 3, (Z + 2) % 3
        nA, nB, nC = n[X], n[Y], n[Z]
        P1, Pa, Paa, Paaa, Pb, Pbb, Pbbb, Pab, Paab, Pabb = _projected_face_integrals(p[:, X], p[:, Y])
        k1 = 1.0 / nC
        k2, k3, k4 = k1 * k1, k1 * k1 * k1, k1 * k1 * k1 * k1
        Fa, Fb = k1 * Pa, k1 * Pb
        Fc = -k2 * (nA * Pa + nB * Pb + w * P1)
        Faa, Fbb = k1 * Paa, k1 * Pbb
        Fcc = k3 * (nA * nA * Paa + 2.0 * nA * nB * Pab + nB * nB * Pbb + w * (2.0 * (nA * Pa + nB * Pb) + w * P1))
        Faaa, Fbbb = k1 * Paaa, k1 * Pbbb
        Fccc = -k4 * (nA ** 3 * Paaa + 3.0 * nA * nA * nB * Paab + 3.0 * nA * nB * nB * Pabb + nB ** 3 * Pbbb
                      + 3.0 * w * (nA * nA * Paa + 2.0 * nA * nB * Pab + nB * nB * Pbb)
                      + w * w * (3.0 * (nA * Pa + nB * Pb) + w * P1))
        Faab = k1 * Paab
        Fbbc = -k2 * (nA * Pabb + nB * Pbbb + w * Pbb)
        Fcca = k3 * (nA * nA * Paaa + 2.0 * nA * nB * Paab + nB * nB * Pabb + w * (2.0 * (nA * Paa + nB * Pab) + w * Pa))
        T0 += n[0] * (Fa if X == 0 else (Fb if Y == 0 else Fc))
        T1[X] += nA * Faa
        T1[Y] += nB * Fbb
        T1[Z] += nC * Fcc
        T2[X] += nA * Faaa
        T2[Y] += nB * Fbbb
        T2[Z] += nC * Fccc
        TP[X] += nA * Faab
        TP[Y] += nB * Fbbc
        TP[Z] += nC * Fcca
    T1, T2, TP = T1 / 2.0, T2 / 3.0, TP / 2.0
    if not T0 > 0.0:
        raise RuntimeError("compute_mass_properties(): internal error, bad mesh encountered")
    mass = density * T0
    com = T1 / T0
    I = np.array([[density * (T2[1] + T2[2]), -density * TP[0], -density * TP[2]],
                  [-density * TP[0], density * (T2[2] + T2[0]), -density * TP[1]],
                  [-density * TP[2], -density * TP[1], density * (T2[0] + T2[1])]])
    tiny = 1.0e-10
    mass = mass if mass > tiny else 0.0
    com = np.where(np.abs(com) > tiny, com, 0.0)
    for i in range(3):
        I[i, i] = I[i, i] if I[i, i] > tiny else 0.0
    for i, j in ((0, 1), (0, 2), (1, 2)):
        v = I[i, j] if abs(I[i, j]) > tiny else 0.0
        I[i, j] = I[j, i] = v
    return mass, com, I


def xform_model_2_body_space(mass, com, I):
    """Body frame at the centre of mass along the principal axes (mass.py:306-392).

    Returns (r, q, I_body): translation and rotation from body to model frame and the principal inertia."""
    x, y, z = -com
    Ib = I.copy()
    Ib[0, 0] = I[0, 0] - mass * (y * y + z * z)
    Ib[1, 1] = I[1, 1] - mass * (x * x + z * z)
    Ib[2, 2] = I[2, 2] - mass * (x * x + y * y)
    tiny = 1.0e-10
    for (i, j), s in (((0, 1), x * y), ((0, 2), x * z), ((1, 2), y * z)):
        v = I[i, j] + mass * s
        Ib[i, j] = Ib[j, i] = v if abs(v) > tiny else 0.0
    d, R = np.linalg.eig(Ib)
    order = [0, 0, 0]
    for p in ([0, 1, 2], [0, 2, 1], [1, 0, 2], [2, 0, 1], [1, 2, 0], [2, 1, 0]):
        if d[p[0]] >= d[p[1]] >= d[p[2]]:
            order = p
            break
    R = R[:, order]
    if np.linalg.det(R) < 0.0:
        R[:, 0] = -R[:, 0]
    return com.copy(), quat_from_matrix(R), d[order]


# ------------------------------------------------------------------------------------------------------------
# signed distance grid (grid3.py:320 create_signed_distance)
# ------------------------------------------------------------------------------------------------------------
def create_signed_distance(V, T, I, J, K, boundary=0.5, device="cuda"):
    """Grid around the mesh (bounding box grown by boundary) holding signed distances, computed on the GPU."""
    import torch
    from . import _native as N
    if boundary < 0:
        raise ValueError()
    V = np.asarray(V, dtype=np.float64)
    grid = Grid(V.min(axis=0) - boundary, V.max(axis=0) + boundary, I, J, K)
    lib = N.load()
    dev = torch.device(device)
    tV = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
    tT = torch.from_numpy(np.ascontiguousarray(T, dtype=np.int32)).to(dev)
    tM = torch.from_numpy(grid.meta()).to(dev)
    out = torch.empty(I * J * K, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev)
    N.check(lib.rb_signed_distance_grid(tV.data_ptr(), len(V), tT.data_ptr(), len(T), tM.data_ptr(), out.data_ptr(),
                                        ctypes.c_void_p(st.cuda_stream)), "rb_signed_distance_grid")
    grid.values = out.cpu().numpy()
    return grid


def signed_distance_grids(V_list, T_list, metas, device="cuda"):
    """Signed distance grids of many meshes in one launch (rb_signed_distance_grids): mesh i has body-frame
    vertices V_list[i], triangles T_list[i] and grid meta metas[i] (min[3], max[3], spacing[3], I, J, K).
    Returns (values, g_off): one float64 device tensor holding every grid, grid i at g_off[i] .. g_off[i + 1]."""
    import torch
    from . import _native as N
    dev = torch.device(device)
    n = len(V_list)
    nv = np.array([len(v) for v in V_list], np.int64)
    nt = np.array([len(t) for t in T_list], np.int64)
    metas = np.asarray(metas, np.float64).reshape(n, 12)
    nodes = (metas[:, 9] * metas[:, 10] * metas[:, 11]).astype(np.int64)
    g_off = np.concatenate([[0], np.cumsum(nodes)]).astype(np.int64)
    blocks = (nodes + 127) // 128
    block_off = np.concatenate([[0], np.cumsum(blocks)]).astype(np.int64)
    tV = torch.from_numpy(np.ascontiguousarray(np.concatenate(V_list), np.float64).reshape(-1)).to(dev)
    tT = torch.from_numpy(np.ascontiguousarray(np.concatenate(T_list), np.int32).reshape(-1)).to(dev)
    tvo = torch.from_numpy(np.concatenate([[0], np.cumsum(nv)]).astype(np.int32)).to(dev)
    tto = torch.from_numpy(np.concatenate([[0], np.cumsum(nt)]).astype(np.int32)).to(dev)
    tM = torch.from_numpy(np.ascontiguousarray(metas).reshape(-1)).to(dev)
    tg = torch.from_numpy(g_off).to(dev)
    tb = torch.from_numpy(block_off).to(dev)
    out = torch.empty(int(g_off[-1]), dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev)
    N.check(N.load().rb_signed_distance_grids(n, tV.data_ptr(), tvo.data_ptr(), tT.data_ptr(), tto.data_ptr(),
                                              tM.data_ptr(), tg.data_ptr(), tb.data_ptr(), int(block_off[-1]),
                                              out.data_ptr(), ctypes.c_void_p(st.cuda_stream)),
            "rb_signed_distance_grids")
    return out, g_off
