"""Rigid-body API with the names, arguments and errors of ``rainbow/simulators/prox_rigid_bodies/api.py``.

``create_engine`` installs :class:`rainbow_b200.stepper.GpuStepper`; everything else builds the scene on the
host exactly as the reference API does, so scripts written against the reference run unchanged::

    import rainbow_b200.api as API
    engine = API.create_engine()
    V, T = API.create_box(1, 1, 1)
    API.create_shape(engine, "box", API.create_mesh(V, T))
    ...
    API.simulate(engine, 1.0)
"""
import numpy as np

from . import geometry as GEO
from .stepper import BatchStepper, GpuStepper   # noqa: F401 (BatchStepper drives simulate_batch)
from .types import Damping, Engine, Gravity, Hinge, RigidBody, Shape, SurfacesInteraction

create_box = GEO.create_box
create_sphere = GEO.create_sphere
create_mesh = GEO.create_mesh


def create_engine(device="cuda"):
    """api.py:42: a new engine whose stepper runs on the GPU."""
    engine = Engine()
    engine.stepper = GpuStepper(device=device)
    return engine


def create_rigid_body(engine, body_name):
    """api.py:56"""
    if body_name in engine.bodies:
        raise RuntimeError("create_rigid_body() rigid body already exist with that name")
    body = RigidBody(body_name)
    body.idx = len(engine.bodies)
    engine.bodies[body_name] = body


def create_hinge(engine, hinge_name):
    """api.py:71"""
    if hinge_name in engine.hinges:
        raise RuntimeError("create_hinge() hinge already exist with that name")
    hinge = Hinge(hinge_name)
    hinge.idx = len(engine.hinges)
    engine.hinges[hinge_name] = hinge


def set_hinge(engine, hinge_name, parent_name, child_name, origin, axis, mode="world"):
    """api.py:86: joint origin and axis given in world coordinates, in the parent's body frame ("body") or in
    the parent's model frame ("model"); stored as each body's arm (origin in its body frame) and axis (the
    joint frame's z axis in its body frame), as Hinge.set_parent_socket / set_child_socket do (types.py:330)."""
    if hinge_name not in engine.hinges:
        raise RuntimeError("set_hinge() no such rigid body exist with that name")
    hinge = engine.hinges[hinge_name]
    if parent_name not in engine.bodies or child_name not in engine.bodies:
        raise RuntimeError("set_hinge() no such rigid body exist with that name")
    parent, child = engine.bodies[parent_name], engine.bodies[child_name]
    origin = np.asarray(origin, dtype=np.float64)
    axis = np.asarray(axis, dtype=np.float64)
    if mode == "world":
        o_world, s_world = origin.copy(), axis.copy()
    elif mode == "body":
        o_world = GEO.quat_rotate(parent.q, origin) + parent.r
        s_world = GEO.quat_rotate(parent.q, axis)
    elif mode == "model":
        o_body = GEO.quat_rotate(GEO.quat_conj(parent.shape.q), origin - parent.shape.r)
        s_body = GEO.quat_rotate(GEO.quat_conj(parent.shape.q), axis)
        o_world = GEO.quat_rotate(parent.q, o_body) + parent.r
        s_world = GEO.quat_rotate(parent.q, s_body)
    else:
        raise ValueError(f"set_hinge() no such mode {mode} is supported")
    t, b, n = GEO.orthonormal_frame(s_world)   # the joint axis is the joint frame's local z axis
    q_world = GEO.quat_from_matrix(np.column_stack([t, b, n]))
    k = np.array([0.0, 0.0, 1.0])
    hinge.parent, hinge.child = parent, child
    hinge.arm_p = GEO.quat_rotate(GEO.quat_conj(parent.q), o_world - parent.r)
    hinge.arm_c = GEO.quat_rotate(GEO.quat_conj(child.q), o_world - child.r)
    hinge.axis_p = GEO.quat_rotate(GEO.quat_prod(GEO.quat_conj(parent.q), q_world), k)
    hinge.axis_c = GEO.quat_rotate(GEO.quat_prod(GEO.quat_conj(child.q), q_world), k)


def create_shape(engine, shape_name, mesh, transform_to_body_frame=True):
    """api.py:176: mass properties, body frame and signed distance grid of a mesh."""
    if shape_name in engine.shapes:
        raise RuntimeError("create_shape(): shape with that name already exist: " + shape_name)
    shape = Shape(shape_name)
    shape.mesh = mesh
    mass, com, I = GEO.compute_mass_properties(mesh.V, mesh.T, 1.0)
    shape.r, shape.q, shape.inertia = GEO.xform_model_2_body_space(mass, com, I)
    shape.mass = mass
    if transform_to_body_frame:
        mesh.V = mesh.V - shape.r
        mesh.V = GEO.quat_rotate_array(GEO.quat_conj(shape.q), mesh.V)
    max_length = (mesh.V.max(axis=0) - mesh.V.min(axis=0)).max()
    boundary = max(max_length * 0.1, engine.params.envelope * 2)
    res = engine.params.resolution
    device = getattr(engine.stepper, "device", "cuda")
    shape.grid = GEO.create_signed_distance(mesh.V, mesh.T, res, res, res, boundary, device=device)
    engine.shapes[shape_name] = shape


def connect_shape(engine, body_name, shape_name):
    """api.py:245 (the GPU step rebuilds its bounding volumes every step, so no per-body tree is made)."""
    if body_name not in engine.bodies:
        raise RuntimeError("connect() no such rigid body exist with that name")
    if shape_name not in engine.shapes:
        raise RuntimeError("connect() no such shape exist with that name")
    engine.bodies[body_name].shape = engine.shapes[shape_name]


def create_gravity_force(engine, force_name, g, up):
    """api.py:284"""
    if force_name in engine.forces:
        raise RuntimeError("create_gravity(): Force already exist with that name")
    if g <= 0.0:
        raise RuntimeError("create_gravity(): Illegal value for gravitational acceleration")
    f = Gravity(force_name)
    f.up = np.asarray(up, dtype=np.float64) / np.linalg.norm(up)
    f.g = g
    engine.forces[force_name] = f


def create_damping_force(engine, force_name, alpha, beta):
    """api.py:310"""
    if force_name in engine.forces:
        raise RuntimeError("create_damping(): Force already exist with that name")
    if alpha <= 0:
        raise RuntimeError("create_damping(): Illegal value for alpha")
    if beta <= 0:
        raise RuntimeError("create_damping(): Illegal value for beta")
    f = Damping(force_name)
    f.alpha, f.beta = alpha, beta
    engine.forces[force_name] = f


def connect_force(engine, body_name, force_name):
    """api.py:335"""
    if body_name not in engine.bodies:
        raise RuntimeError("connect_force() no such rigid body exist with that name")
    if force_name not in engine.forces:
        raise RuntimeError("connect_force() no such force exist with that name")
    body, force = engine.bodies[body_name], engine.forces[force_name]
    if force in body.forces:
        raise RuntimeError("connect_force() force was already connected to body")
    body.forces.append(force)


def _body(engine, name, fn):
    if name not in engine.bodies:
        raise RuntimeError("%s() no such rigid body exist with that name" % fn)
    return engine.bodies[name]


def set_position(engine, body_name, r, use_model_frame=False):
    """api.py:358: position of the body frame, or of the model frame when use_model_frame."""
    body = _body(engine, body_name, "set_position")
    if use_model_frame:
        q_mf2wcs = GEO.quat_prod(np.copy(body.q), GEO.quat_conj(body.shape.q))
        body.r = GEO.quat_rotate(q_mf2wcs, body.shape.r) + np.asarray(r, dtype=np.float64)
    else:
        body.r = np.array(r, dtype=np.float64)


def get_position(engine, body_name):
    return np.copy(_body(engine, body_name, "get_position").r)


def set_orientation(engine, body_name, q, use_model_frame=False):
    """api.py:433"""
    body = _body(engine, body_name, "set_position")
    if use_model_frame:
        q_mf2wcs = GEO.quat_prod(np.copy(body.q), GEO.quat_conj(body.shape.q))
        r_mf2wcs = np.copy(body.r) - GEO.quat_rotate(q_mf2wcs, body.shape.r)
        q_mf2wcs = GEO.quat_unit(q)
        body.q = GEO.quat_prod(q_mf2wcs, body.shape.q)
        body.r = GEO.quat_rotate(q_mf2wcs, body.shape.r) + r_mf2wcs
    else:
        body.q = GEO.quat_unit(q)


def get_orientation(engine, body_name):
    return np.copy(_body(engine, body_name, "get_orientation").q)


def set_velocity(engine, body_name, v):
    _body(engine, body_name, "set_velocity").v = np.array(v, dtype=np.float64)


def get_velocity(engine, body_name):
    return np.copy(_body(engine, body_name, "get_velocity").v)


def set_spin(engine, body_name, w):
    _body(engine, body_name, "set_spin").w = np.array(w, dtype=np.float64)


def get_spin(engine, body_name):
    return np.copy(_body(engine, body_name, "get_spin").w)


def set_mass_properties(engine, body_name, density):
    """api.py:569"""
    body = _body(engine, body_name, "set_mass_properties")
    if body.shape is None:
        raise RuntimeError("set_mass_properties() rigid body did not have a shape")
    body.mass = body.shape.mass * density
    body.inertia = body.shape.inertia * density


def set_body_type(engine, body_name, body_type):
    """api.py:591"""
    body = _body(engine, body_name, "set_body_type")
    if body_type in ["fixed", "Fixed", "FIXED"]:
        body.is_fixed = True
    elif body_type in ["free", "Free", "FREE"]:
        body.is_fixed = False
    else:
        raise RuntimeError("set_body_type(): Unsupported body type found")


def is_fixed_body(engine, body_name):
    return _body(engine, body_name, "is_fixed_body").is_fixed


def set_body_material(engine, body_name, material_name):
    """api.py:626"""
    body = _body(engine, body_name, "set_body_material")
    if not engine.surfaces_interactions.exist_material(material_name):
        raise RuntimeError("set_body_material() no such material exist")
    body.material = material_name


def create_surfaces_interaction(engine, A, B, epsilon, mu):
    """api.py:646"""
    if engine.surfaces_interactions.exist_interaction(A, B):
        raise RuntimeError("create_surfaces_interaction() behaviour already exist")
    if epsilon < 0.0:
        raise RuntimeError("create_surfaces_interaction() illegal epsilon value")
    for k, axis in enumerate("xyz"):
        if mu[k] < 0.0:
            raise RuntimeError("create_surfaces_interaction() illegal mu_%s value" % axis)
    it = SurfacesInteraction()
    it.epsilon = epsilon
    it.mu = np.asarray(mu, dtype=np.float64)
    engine.surfaces_interactions.storage[tuple(sorted([A, B]))] = it


def simulate(engine, T, profiling_on=False):
    """api.py:676: advance by T in steps of at most params.time_step."""
    if T <= 0:
        raise ValueError("Time must be positive")
    if engine.stepper is None:
        raise ValueError("A time-stepper must be initialized")
    T_left = T
    while T_left:
        dt = min(T_left, engine.params.time_step)
        engine.stepper.step(dt, engine, profiling_on)
        T_left -= dt


def simulate_batch(engines, T, stepper, profiling_on=False):
    """Advance every engine by T, all of them in one batch per time step (the many-scene form of
    :func:`simulate`, api.py:676): ``stepper`` is a :class:`rainbow_b200.stepper.BatchStepper`, and the
    engines share ``params.time_step`` and the other step parameters."""
    if T <= 0:
        raise ValueError("Time must be positive")
    engines = list(engines)
    if not engines:
        return
    time_step = engines[0].params.time_step
    T_left = T
    while T_left:
        dt = min(T_left, time_step)
        stepper.step(dt, engines, profiling_on)
        T_left -= dt


def get_log(engine):
    """api.py:696"""
    return engine.stepper.log
