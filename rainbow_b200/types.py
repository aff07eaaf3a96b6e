"""Engine data model with the attribute names of ``rainbow/simulators/prox_rigid_bodies/types.py``.

The GPU stepper reads engines by attribute (duck typing), so it accepts these objects and the reference's own
``Engine`` alike.  This module lets scenes be built where the reference package is not installed.
"""
from typing import Optional

import numpy as np


def _unit(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


class Mesh:
    """Triangle mesh (rainbow/geometry/surface_mesh.py:6 Mesh)."""

    def __init__(self, V, T):
        self.V = np.copy(V)
        self.T = np.copy(T)


class Grid:
    """Regular 3D grid of node values (rainbow/geometry/grid3.py:5 Grid); i runs fastest."""

    def __init__(self, min_coord, max_coord, I, J, K):
        if np.any(np.asarray(min_coord) > np.asarray(max_coord)):
            raise ValueError()
        if I < 2 or J < 2 or K < 2:
            raise ValueError()
        self.min_coord = np.array(min_coord, dtype=np.float64).ravel()
        self.max_coord = np.array(max_coord, dtype=np.float64).ravel()
        self.I, self.J, self.K = int(I), int(J), int(K)
        self.spacing = np.divide(self.max_coord - self.min_coord, np.array([I - 1, J - 1, K - 1], dtype=np.float64))
        self.values = None

    def meta(self):
        return np.concatenate([self.min_coord, self.max_coord, self.spacing, [self.I, self.J, self.K]]).astype(np.float64)


class SurfacesInteraction:
    """types.py:19 SurfacesInteraction: friction coefficients and restitution of a material pair."""

    def __init__(self):
        self.mu = np.ones(3, dtype=np.float64)
        self.epsilon = 0.0


class SurfacesInteractionLibrary:
    """types.py:33: material-pair interactions keyed by the sorted pair of names, with a default."""

    def __init__(self):
        self.storage = {("default", "default"): SurfacesInteraction()}

    def get_interaction(self, A, B):
        key = (A, B) if A < B else (B, A)
        return self.storage.get(key, self.storage[("default", "default")])

    def exist_interaction(self, A, B):
        key = (A, B) if A < B else (B, A)
        return key in self.storage

    def exist_material(self, name):
        return any(name in key for key in self.storage)


class Shape:
    """types.py:82 Shape: body-frame mesh, signed distance grid and unit-density mass properties."""

    def __init__(self, name):
        self.name = name
        self.mesh: Optional[Mesh] = None
        self.grid: Optional[Grid] = None
        self.mass = 0.0
        self.inertia = np.zeros(3, dtype=np.float64)
        self.r = np.zeros(3, dtype=np.float64)
        self.q = np.array([1.0, 0.0, 0.0, 0.0])


class RigidBody:
    """types.py:111 RigidBody."""

    def __init__(self, name):
        self.name = name
        self.idx: Optional[int] = None
        self.q = np.array([1.0, 0.0, 0.0, 0.0])
        self.r = np.zeros(3, dtype=np.float64)
        self.v = np.zeros(3, dtype=np.float64)
        self.w = np.zeros(3, dtype=np.float64)
        self.mass = 0.0
        self.inertia = np.zeros(3, dtype=np.float64)
        self.shape: Optional[Shape] = None
        self.is_fixed = False
        self.forces = []
        self.material = "default"
        self.bvh = None   # the GPU step builds its bounding volumes each step; no per-body tree is kept


class Gravity:
    """types.py:189 Gravity: F = -m g up."""

    def __init__(self, name):
        self.force_type = "Gravity"
        self.name = name
        self.g = 9.81
        self.up = np.array([0.0, 1.0, 0.0])

    def compute(self, body, r, q, v, w):
        return -body.mass * self.g * self.up, np.zeros(3, dtype=np.float64)


class Damping:
    """types.py:224 Damping: F = -alpha v, T = -beta w."""

    def __init__(self, name):
        self.force_type = "Damping"
        self.name = name
        self.alpha = 0.001
        self.beta = 0.001

    def compute(self, body, r, q, v, w):
        return -v * self.alpha, -w * self.beta


class ContactPoint:
    """types.py:259 ContactPoint (bodyA = owner of the signed distance field, bodyB = owner of the mesh)."""

    def __init__(self, bodyA, bodyB, position=None, normal=None, gap=0.0):
        normal = np.array([0.0, 0.0, 1.0]) if normal is None else normal
        if abs(1.0 - np.linalg.norm(normal)) > 0.1:
            raise RuntimeError("ContactPoint.init() was called with non-unit size normal")
        self.bodyA = bodyA
        self.bodyB = bodyB
        self.p = np.zeros(3) if position is None else position
        self.n = normal
        self.g = gap


class Hinge:
    """types.py:304 Hinge: a revolute joint between a parent and a child body; arm_* and axis_* are the joint
    origin and axis in each body's own frame (set by api.set_hinge)."""

    def __init__(self, name):
        self.name = name
        self.idx = None
        self.parent = None
        self.child = None
        self.arm_p = None
        self.arm_c = None
        self.axis_p = None
        self.axis_c = None


class Parameters:
    """types.py:356 Parameters, plus the solver options of the GPU stepper.

    proximal_solver: None (the reference stepper's Gauss-Seidel, gauss_seidel_solver.py:14) or one of the
    proximal_contact scheme names 'gauss_seidel', 'parallel_jacobi', 'parallel_jacboi_hybrid'
    (prox_soft_bodies/types.py:256 spelling; 'parallel_jacobi_hybrid' is accepted too).
    """

    def __init__(self):
        self.time_step = 0.01
        self.max_iterations = 200
        self.use_bounce = False
        self.use_pre_stabilization = False
        self.use_post_stabilization = False
        self.gap_reduction = 0.5
        self.min_gap_value = 0.001
        self.max_gap_value = 0.01
        self.absolute_tolerance = 0.001
        self.relative_tolerance = 0.0001
        self.ellipsoid_max_iterations = 100
        self.ellipsoid_expansion = 1.5
        self.ellipsoid_tolerance = 10e-10
        self.nu_reduce = 0.7
        self.nu_increase = 1.3
        self.too_small_merit_change = 0.01
        self.contact_optimization_max_iterations = 8
        self.contact_optimization_tolerance = 0
        self.bvh_chunk_size = 255
        self.K = 3
        self.envelope = 0.1
        self.resolution = 64
        self.proximal_solver = None
        self.warm_start = False   # start each solve from the previous step's impulses (the reference starts at 0)


class Engine:
    """types.py:421 Engine."""

    def __init__(self):
        self.simulator_type = "rigid_body"
        self.bodies = dict()
        self.forces = dict()
        self.shapes = dict()
        self.hinges = dict()
        self.contact_points = []
        self.surfaces_interactions = SurfacesInteractionLibrary()
        self.params = Parameters()
        self.stepper = None
