"""Conversion between an engine object and the flat scene arrays consumed by :class:`DeviceWorld`.

Engines are read by attribute only, following ``rainbow/simulators/prox_rigid_bodies/types.py``; both the
reference's ``Engine`` and :class:`rainbow_b200.types.Engine` work.  The array layout is the one of the
``StateStorage`` vectors (``state_storage.py:71-105``: bodies in ``engine.bodies`` insertion order).
"""
import numpy as np

from .world import PARAM_FIELDS


def _force_kind(force):
    kind = getattr(force, "force_type", type(force).__name__)
    if kind == "Gravity":
        return 0
    if kind == "Damping":
        return 1
    raise NotImplementedError("force type %r is not supported by the GPU stepper" % (kind,))


def _is_device_tensor(a):
    return type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False)


def scene_arrays(engine):
    """Flat arrays of one scene.  Grids held as CUDA tensors stay on the device (``shape_grid`` is then a
    device tensor); everything else is a host array."""
    out = {}
    shapes = list(engine.shapes.values())
    shape_index = {id(s): i for i, s in enumerate(shapes)}
    Vs, Ts, Gs, meta = [], [], [], []
    v_off, t_off, g_off = [0], [0], [0]
    on_device = False
    for s in shapes:
        V = np.ascontiguousarray(s.mesh.V, dtype=np.float64)
        T = np.ascontiguousarray(s.mesh.T, dtype=np.int32)
        vals = s.grid.values
        if _is_device_tensor(vals):   # a grid built on (or kept on) the device stays there
            vals = vals.reshape(-1)
            on_device = True
        else:
            vals = np.ascontiguousarray(vals, dtype=np.float64).ravel()
        Vs.append(V)
        Ts.append(T)
        Gs.append(vals)
        v_off.append(v_off[-1] + len(V))
        t_off.append(t_off[-1] + len(T))
        g_off.append(g_off[-1] + len(vals))
        g = s.grid
        meta.append(np.concatenate([np.ravel(g.min_coord), np.ravel(g.max_coord), np.ravel(g.spacing),
                                    [g.I, g.J, g.K]]).astype(np.float64))
    out["shape_V"] = np.concatenate(Vs) if Vs else np.zeros((0, 3))
    out["shape_T"] = np.concatenate(Ts) if Ts else np.zeros((0, 3), np.int32)
    if on_device:
        import torch
        dev = next(g.device for g in Gs if _is_device_tensor(g))
        out["shape_grid"] = torch.cat([g.to(torch.float64) if _is_device_tensor(g) else
                                       torch.from_numpy(g).to(dev) for g in Gs])
    else:
        out["shape_grid"] = np.concatenate(Gs) if Gs else np.zeros(0)
    out["shape_v_off"] = np.array(v_off, dtype=np.int64)
    out["shape_t_off"] = np.array(t_off, dtype=np.int64)
    out["shape_g_off"] = np.array(g_off, dtype=np.int64)
    out["shape_grid_meta"] = np.array(meta, dtype=np.float64).reshape(-1, 12)

    bodies = list(engine.bodies.values())
    for k, b in enumerate(bodies):
        if b.idx != k:
            raise RuntimeError("body %r has idx %r but is stored at position %d" % (b.name, b.idx, k))
        if b.shape is None:
            raise RuntimeError("body %r has no shape" % (b.name,))
        if not b.is_fixed and b.mass == 0:
            raise ValueError("Body {} has no mass.".format(b.name))   # state_storage.py:170-171
    forces = list(engine.forces.values())
    force_index = {id(f): i for i, f in enumerate(forces)}
    lib = engine.surfaces_interactions
    materials = sorted({b.material for b in bodies} | {m for key in lib.storage for m in key})
    mat_index = {m: i for i, m in enumerate(materials)}
    nb, nf = len(bodies), len(forces)
    out["body_shape"] = np.array([shape_index[id(b.shape)] for b in bodies], dtype=np.int32)
    out["body_r"] = np.array([np.asarray(b.r, dtype=np.float64) for b in bodies]).reshape(nb, 3)
    out["body_q"] = np.array([np.asarray(b.q, dtype=np.float64) for b in bodies]).reshape(nb, 4)
    out["body_v"] = np.array([np.asarray(b.v, dtype=np.float64) for b in bodies]).reshape(nb, 3)
    out["body_w"] = np.array([np.asarray(b.w, dtype=np.float64) for b in bodies]).reshape(nb, 3)
    out["body_mass"] = np.array([b.mass for b in bodies], dtype=np.float64)
    out["body_inertia"] = np.array([np.asarray(b.inertia, dtype=np.float64) for b in bodies]).reshape(nb, 3)
    out["body_fixed"] = np.array([bool(b.is_fixed) for b in bodies], dtype=np.uint8)
    out["body_material"] = np.array([mat_index[b.material] for b in bodies], dtype=np.int32)
    order = np.full((nb, max(nf, 1)), -1, dtype=np.int32)
    for k, b in enumerate(bodies):
        for j, f in enumerate(b.forces):
            order[k, j] = force_index[id(f)]
    out["body_force_order"] = order[:, :nf] if nf else np.zeros((nb, 0), np.int32)
    kinds, fparams = [], []
    for f in forces:
        kind = _force_kind(f)
        kinds.append(kind)
        if kind == 0:
            up = np.asarray(f.up, dtype=np.float64)
            fparams.append([float(f.g), up[0], up[1], up[2]])
        else:
            fparams.append([float(f.alpha), float(f.beta), 0.0, 0.0])
    out["force_kind"] = np.array(kinds, dtype=np.int32)
    out["force_params"] = np.array(fparams, dtype=np.float64).reshape(nf, 4)
    M = len(materials)
    mu = np.zeros((M, M, 3))
    eps = np.zeros((M, M))
    for a in range(M):
        for b in range(M):
            it = lib.get_interaction(materials[a], materials[b])
            mu[a, b] = np.asarray(it.mu, dtype=np.float64)[:3]
            eps[a, b] = it.epsilon
    out["material_mu"] = mu
    out["material_epsilon"] = eps
    out["params"] = np.array([float(getattr(engine.params, f)) for f in PARAM_FIELDS])
    # hinge joints (types.py:304), Hinge.idx order: parent/child body indices, body-frame arms and axes
    hinges = sorted(getattr(engine, "hinges", {}).values(), key=lambda h: h.idx)
    if [h.idx for h in hinges] != list(range(len(hinges))):
        raise RuntimeError("hinge indices are not 0 .. n-1")
    out["hinge_bodies"] = np.array([[h.parent.idx, h.child.idx] for h in hinges], dtype=np.int32).reshape(-1, 2)
    out["hinge_frames"] = np.array([np.concatenate([np.asarray(h.arm_p, np.float64), np.asarray(h.arm_c, np.float64),
                                                    np.asarray(h.axis_p, np.float64), np.asarray(h.axis_c, np.float64)])
                                    for h in hinges], dtype=np.float64).reshape(-1, 12)
    return out


def static_signature(engine):
    """Identity of everything the device copy of a scene depends on except the body state."""
    bodies = list(engine.bodies.values())
    sig = [len(bodies), len(engine.shapes), len(engine.forces)]
    for b in bodies:
        sig.append((id(b), id(b.shape), bool(b.is_fixed), float(b.mass), tuple(np.asarray(b.inertia, dtype=np.float64)),
                    b.material, tuple(id(f) for f in b.forces)))
    for s in engine.shapes.values():
        sig.append((id(s), id(s.mesh.V), id(s.mesh.T), id(s.grid), id(s.grid.values)))
    for h in sorted(getattr(engine, "hinges", {}).values(), key=lambda h: h.idx):
        sig.append((id(h), h.parent.idx, h.child.idx,
                    tuple(np.concatenate([np.ravel(h.arm_p), np.ravel(h.arm_c), np.ravel(h.axis_p), np.ravel(h.axis_c)]))))
    for f in engine.forces.values():
        sig.append((id(f), tuple(np.ravel(getattr(f, "up", [0.0]))), float(getattr(f, "g", 0.0)),
                    float(getattr(f, "alpha", 0.0)), float(getattr(f, "beta", 0.0))))
    for key, it in sorted(engine.surfaces_interactions.storage.items()):
        sig.append((key, tuple(np.asarray(it.mu, dtype=np.float64)), float(it.epsilon)))
    return tuple(sig)


def body_state(engine):
    bodies = list(engine.bodies.values())
    x = np.empty((len(bodies), 7))
    u = np.empty((len(bodies), 6))
    for k, b in enumerate(bodies):
        x[k, :3] = b.r
        x[k, 3:] = b.q
        u[k, :3] = b.v
        u[k, 3:] = b.w
    return x, u


def write_back(engine, x, u):
    """state_storage.py:55 copy_to_engine."""
    for k, b in enumerate(engine.bodies.values()):
        b.r = x[k, :3].copy()
        b.q = x[k, 3:].copy()
        b.v = u[k, :3].copy()
        b.w = u[k, 3:].copy()


def engine_from_arrays(arrays, names=None):
    """A :class:`rainbow_b200.types.Engine` holding the scene described by flat arrays (inverse of scene_arrays)."""
    from . import types as TY
    a = arrays
    engine = TY.Engine()
    shape_objs = []
    sv, st, sg = np.asarray(a["shape_v_off"]), np.asarray(a["shape_t_off"]), np.asarray(a["shape_g_off"])
    meta = np.asarray(a["shape_grid_meta"]).reshape(-1, 12)
    shape_names = list(a["shape_names"]) if "shape_names" in a else ["shape%d" % k for k in range(len(sv) - 1)]
    for k in range(len(sv) - 1):
        s = TY.Shape(str(shape_names[k]))
        s.mesh = TY.Mesh(np.asarray(a["shape_V"])[sv[k]:sv[k + 1]], np.asarray(a["shape_T"])[st[k]:st[k + 1]])
        m = meta[k]
        g = TY.Grid(m[0:3], m[3:6], int(m[9]), int(m[10]), int(m[11]))
        g.spacing = m[6:9].copy()
        if _is_device_tensor(a["shape_grid"]):   # grids built on the device: views of the one tensor
            g.values = a["shape_grid"].reshape(-1)[sg[k]:sg[k + 1]]
        else:
            g.values = np.asarray(a["shape_grid"]).ravel()[sg[k]:sg[k + 1]].copy()
        s.grid = g
        engine.shapes[s.name] = s
        shape_objs.append(s)
    forces = []
    fnames = list(a["force_names"]) if "force_names" in a else ["force%d" % k for k in range(len(a["force_kind"]))]
    for k, kind in enumerate(np.asarray(a["force_kind"])):
        fp = np.asarray(a["force_params"]).reshape(-1, 4)[k]
        if kind == 0:
            f = TY.Gravity(str(fnames[k]))
            f.g, f.up = float(fp[0]), fp[1:4].copy()
        else:
            f = TY.Damping(str(fnames[k]))
            f.alpha, f.beta = float(fp[0]), float(fp[1])
        engine.forces[f.name] = f
        forces.append(f)
    mats = [str(m) for m in a["material_names"]] if "material_names" in a else \
        ["m%d" % k for k in range(len(a["material_epsilon"]))]
    lib = engine.surfaces_interactions
    lib.storage = {}
    M = len(mats)
    for i in range(M):
        for j in range(i, M):
            it = TY.SurfacesInteraction()
            it.mu = np.asarray(a["material_mu"])[i, j].copy()
            it.epsilon = float(np.asarray(a["material_epsilon"])[i, j])
            lib.storage[(mats[i], mats[j])] = it
    if ("default", "default") not in lib.storage:
        lib.storage[("default", "default")] = TY.SurfacesInteraction()
    body_names = list(a["body_names"]) if "body_names" in a else ["b%d" % k for k in range(len(a["body_mass"]))]
    order = np.asarray(a["body_force_order"]).reshape(len(body_names), -1)
    for k, nm in enumerate(body_names):
        b = TY.RigidBody(str(nm))
        b.idx = k
        b.shape = shape_objs[int(a["body_shape"][k])]
        b.r, b.q = np.array(a["body_r"][k], dtype=np.float64), np.array(a["body_q"][k], dtype=np.float64)
        b.v, b.w = np.array(a["body_v"][k], dtype=np.float64), np.array(a["body_w"][k], dtype=np.float64)
        b.mass = float(a["body_mass"][k])
        b.inertia = np.array(a["body_inertia"][k], dtype=np.float64)
        b.is_fixed = bool(a["body_fixed"][k])
        b.material = mats[int(a["body_material"][k])]
        b.forces = [forces[f] for f in order[k] if f >= 0]
        engine.bodies[b.name] = b
    p = np.asarray(a["params"], dtype=np.float64)
    for name, v in zip(PARAM_FIELDS, p):
        cur = getattr(engine.params, name)
        setattr(engine.params, name, type(cur)(v) if not isinstance(cur, bool) else bool(v))
    bodies = list(engine.bodies.values())
    hb = np.asarray(a.get("hinge_bodies", np.zeros((0, 2))), np.int64).reshape(-1, 2)
    hf = np.asarray(a.get("hinge_frames", np.zeros((0, 12))), np.float64).reshape(-1, 12)
    for k in range(len(hb)):
        h = TY.Hinge("hinge%d" % k)
        h.idx = k
        h.parent, h.child = bodies[int(hb[k, 0])], bodies[int(hb[k, 1])]
        h.arm_p, h.arm_c, h.axis_p, h.axis_c = hf[k, 0:3].copy(), hf[k, 3:6].copy(), hf[k, 6:9].copy(), hf[k, 9:12].copy()
        engine.hinges[h.name] = h
    return engine
