"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the C++17 restatement of the reference explicit MPM step in
``mpm_oracle.cpp``.  It is the checker for the CUDA path: only the test suite,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
this module.  The product package never imports it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpm_oracle.so")
SOURCES = [os.path.join(HERE, "mpm_oracle.cpp")]


def build(force=False):
    """Compile the oracle with g++ (no Eigen, no fused multiply-add)."""
    import subprocess
    if not force and os.path.exists(LIB_PATH) and all(
            os.path.getmtime(LIB_PATH) >= os.path.getmtime(s) for s in SOURCES):
        return LIB_PATH
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
           "-fopenmp", "-o", LIB_PATH] + SOURCES
    subprocess.check_call(cmd)
    return LIB_PATH


class Config(C.Structure):
    _fields_ = [("dim", C.c_int32), ("scheme", C.c_int32),
                ("velocity_update", C.c_int32), ("locate_particles", C.c_int32),
                ("blending_ratio", C.c_double), ("dt", C.c_double),
                ("damping_factor", C.c_double), ("gravity", C.c_double * 3),
                ("gravity_ramping_time", C.c_double), ("nthreads", C.c_int32),
                ("isoparametric", C.c_int32)]


# velocity_update names -> the reference's VelocityUpdate order (data_types.h:50)
VELOCITY_UPDATES = {"flip": 0, "pic": 1, "asflip": 2, "tpic": 3, "apic": 4}


class Particles(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in (
        "x", "u", "v", "a", "stress", "strain", "dstrain", "strain_rate", "F",
        "volume", "mass", "density", "xi")] + [
        ("cell", C.POINTER(C.c_int64)), ("material", C.POINTER(C.c_int32)),
        ("svars", C.POINTER(C.c_double)), ("status", C.POINTER(C.c_int32)),
        ("mapping", C.POINTER(C.c_double))]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int32, C.c_double
        pd, pi64, pi32 = C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        L.mpmo_create.restype = vp
        L.mpmo_create.argtypes = [C.POINTER(Config)]
        L.mpmo_destroy.argtypes = [vp]
        L.mpmo_last_error.restype = C.c_char_p
        L.mpmo_last_error.argtypes = [vp]
        L.mpmo_set_mesh.argtypes = [vp, i64, pd, i64, i32, pi64]
        L.mpmo_add_material.argtypes = [vp, i32, i32, pd, i32]
        for f in (L.mpmo_add_velocity_constraints, L.mpmo_add_acceleration_constraints):
            f.argtypes = [vp, i64, pi64, pi32, pd]
        L.mpmo_add_friction_constraints.argtypes = [vp, i64, pi64, pi32, pi32, pd]
        L.mpmo_add_particle_velocity_constraint.argtypes = [vp, i64, pi64, i32, dbl]
        L.mpmo_set_nodal_euler_angles.argtypes = [vp, i64, pi64, pd]
        L.mpmo_add_particles.argtypes = [vp, i64, pd, i32]
        L.mpmo_initialise.argtypes = [vp]
        L.mpmo_set_particles.argtypes = [vp, C.POINTER(Particles)]
        L.mpmo_nparticles.restype = i64
        L.mpmo_nparticles.argtypes = [vp]
        L.mpmo_get_particles.argtypes = [vp, C.POINTER(Particles)]
        L.mpmo_step.argtypes = [vp, i64]
        L.mpmo_get_nodes.argtypes = [vp, pd]
        L.mpmo_set_nodes.argtypes = [vp, pd]
        L.mpmo_phase.argtypes = [vp, i32, dbl, pd]
        L.mpmo_element_dn_dx.argtypes = [i32, pd, pd, pd, pd, pd]
        L.mpmo_material_stress.argtypes = [i32, i32, pd, i32, pd, pd, dbl, pd, pd]
        L.mpmo_mc_diagnostics.argtypes = [i32, pd, i32, pd, pd, pd]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _i32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


MATERIAL_TYPES = {"LinearElastic": 0, "MohrCoulomb": 1}


def material_params(mtype, props):
    """Numeric parameter vector from a reference material JSON object
    (linear_elastic.tcc:20-24, mohr_coulomb.tcc:9-71)."""
    if mtype == "LinearElastic":
        return [props["density"], props["youngs_modulus"], props["poisson_ratio"]]
    packing = 1.0
    if "packing_fraction" in props:
        packing = props["packing_fraction"]
    elif "porosity" in props:
        packing = 1.0 - props["porosity"]
    is_wet = "porosity" in props and any(k in props for k in ("k_x", "k_y", "k_z"))
    return [props["density"], props["youngs_modulus"], props["poisson_ratio"],
            props["friction"], props["dilation"], props["cohesion"],
            props["residual_friction"], props["residual_dilation"],
            props["residual_cohesion"], props["peak_pdstrain"],
            props["residual_pdstrain"], props["tension_cutoff"],
            1.0 if props["softening"] else 0.0, packing,
            props.get("packing_fraction_minimum", 0.0), 1.0 if is_wet else 0.0]


MC_STATE = ["yield_state", "phi", "psi", "cohesion", "tension_cutoff",
            "epsilon", "rho", "theta", "pdstrain"]


def mc_initial_state(params):
    """MohrCoulomb::initialise_state_variables (mohr_coulomb.tcc:85-111)."""
    import math
    phi = params[3] * math.pi / 180.
    psi = params[4] * math.pi / 180.
    c = params[5]
    tc = params[11]
    apex = c / math.tan(phi) if math.tan(phi) != 0 else float("inf")
    v = tc if tc < apex else apex
    v = v if v > 1e-15 else 1e-15
    return [0.0, phi, psi, c, v, 0.0, 0.0, 0.0, 0.0]


def material_stress(dim, mtype, props, stress, dstrain, density, state=None):
    """One Material<Tdim>::compute_stress call; returns (stress, state)."""
    p = np.asarray(material_params(mtype, props), dtype=np.float64)
    s = np.asarray(stress, dtype=np.float64)
    d = np.asarray(dstrain, dtype=np.float64)
    st = np.zeros(9) if state is None else np.asarray(state, dtype=np.float64).copy()
    out = np.zeros(6)
    rc = lib().mpmo_material_stress(dim, MATERIAL_TYPES[mtype], _dp(p), len(p), _dp(s),
                                    _dp(d), float(density), _dp(st), _dp(out))
    assert rc == 0
    return out, st


def mc_diagnostics(dim, props, stress, state):
    p = np.asarray(material_params("MohrCoulomb", props), dtype=np.float64)
    s = np.asarray(stress, dtype=np.float64)
    st = np.asarray(state, dtype=np.float64).copy()
    out = np.zeros(20)
    rc = lib().mpmo_mc_diagnostics(dim, _dp(p), len(p), _dp(s), _dp(st), _dp(out))
    assert rc == 0
    return {"epsilon": out[0], "rho": out[1], "theta": out[2], "f0": out[3],
            "f1": out[4], "yield_type": int(out[5]), "df_dsigma": out[6:12],
            "dp_dsigma": out[12:18], "dp_dq": out[18], "softening": out[19]}


def element_dn_dx(dim, xi, X):
    nv = 4 if dim == 2 else 8
    xi = np.asarray(xi, dtype=np.float64)
    X = np.ascontiguousarray(X, dtype=np.float64)
    N = np.zeros(nv)
    G = np.zeros((nv, dim))
    D = np.zeros((nv, dim))
    assert lib().mpmo_element_dn_dx(dim, _dp(xi), _dp(X), _dp(N), _dp(G), _dp(D)) == 0
    return N, G, D


FIELDS3 = ("x", "u", "v", "a", "xi")
FIELDS6 = ("stress", "strain", "dstrain", "strain_rate")


class Oracle:
    """A complete oracle solver instance: mesh, materials, constraints, particles."""

    def __init__(self, dim, scheme="usf", velocity_update="flip", dt=1e-3,
                 gravity=(0, 0, 0), damping_factor=0.0, blending_ratio=1.0,
                 gravity_ramping_time=0.0, locate_particles=True, nthreads=1,
                 isoparametric=False):
        cfg = Config()
        cfg.dim = dim
        cfg.scheme = {"usf": 0, "usl": 1, "musl": 2}[scheme]
        cfg.velocity_update = VELOCITY_UPDATES[velocity_update]
        cfg.locate_particles = 1 if locate_particles else 0
        cfg.isoparametric = 1 if isoparametric else 0
        cfg.blending_ratio = blending_ratio
        cfg.dt = dt
        cfg.damping_factor = damping_factor
        g = list(gravity) + [0.0] * (3 - len(gravity))
        for i in range(3):
            cfg.gravity[i] = g[i]
        cfg.gravity_ramping_time = gravity_ramping_time
        cfg.nthreads = nthreads
        self.dim = dim
        self.h = lib().mpmo_create(C.byref(cfg))
        if not self.h:
            raise ValueError("oracle create failed")

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().mpmo_destroy(h)
            self.h = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(lib().mpmo_last_error(self.h).decode())

    def set_mesh(self, coords, cells):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        self._check(lib().mpmo_set_mesh(self.h, coords.shape[0], _dp(coords), cells.shape[0],
                                        cells.shape[1], _i64p(cells)))

    def add_material(self, mid, mtype, props):
        base = mtype[:-2] if mtype.endswith(("2D", "3D")) else mtype
        p = np.asarray(material_params(base, props), dtype=np.float64)
        self._check(lib().mpmo_add_material(self.h, mid, MATERIAL_TYPES[base], _dp(p), len(p)))

    def add_velocity_constraints(self, nid, direction, value):
        nid = np.ascontiguousarray(nid, dtype=np.int64)
        d = np.ascontiguousarray(direction, dtype=np.int32)
        v = np.ascontiguousarray(value, dtype=np.float64)
        self._check(lib().mpmo_add_velocity_constraints(self.h, len(nid), _i64p(nid), _i32p(d), _dp(v)))

    def add_acceleration_constraints(self, nid, direction, value):
        nid = np.ascontiguousarray(nid, dtype=np.int64)
        d = np.ascontiguousarray(direction, dtype=np.int32)
        v = np.ascontiguousarray(value, dtype=np.float64)
        self._check(lib().mpmo_add_acceleration_constraints(self.h, len(nid), _i64p(nid), _i32p(d), _dp(v)))

    def add_friction_constraints(self, nid, direction, sign_n, mu):
        nid = np.ascontiguousarray(nid, dtype=np.int64)
        d = np.ascontiguousarray(direction, dtype=np.int32)
        s = np.ascontiguousarray(sign_n, dtype=np.int32)
        m = np.ascontiguousarray(mu, dtype=np.float64)
        self._check(lib().mpmo_add_friction_constraints(self.h, len(nid), _i64p(nid), _i32p(d),
                                                        _i32p(s), _dp(m)))

    def set_nodal_euler_angles(self, nid, angles):
        nid = np.ascontiguousarray(nid, dtype=np.int64)
        a = np.ascontiguousarray(angles, dtype=np.float64)
        self._check(lib().mpmo_set_nodal_euler_angles(self.h, len(nid), _i64p(nid), _dp(a)))

    def add_particle_velocity_constraint(self, pids, direction, value):
        if pids is None:
            self._check(lib().mpmo_add_particle_velocity_constraint(self.h, -1, None, direction, value))
            return
        p = np.ascontiguousarray(pids, dtype=np.int64)
        self._check(lib().mpmo_add_particle_velocity_constraint(self.h, len(p), _i64p(p), direction, value))

    def add_particles(self, coords, material_id):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        self._check(lib().mpmo_add_particles(self.h, coords.shape[0], _dp(coords), material_id))

    def initialise(self):
        self._check(lib().mpmo_initialise(self.h))

    def assign_particle_stresses(self, stress):
        """Mesh::assign_particles_stresses (mesh.tcc:1502-1524)."""
        stress = np.ascontiguousarray(stress, dtype=np.float64).reshape(-1, 6)
        self.set({"stress": stress})

    @property
    def nparticles(self):
        return lib().mpmo_nparticles(self.h)

    def step(self, n=1):
        self._check(lib().mpmo_step(self.h, n))

    def get(self):
        n = self.nparticles
        arrs = {}
        P = Particles()
        for f in FIELDS3:
            arrs[f] = np.zeros((n, 3))
            setattr(P, f, _dp(arrs[f]))
        for f in FIELDS6:
            arrs[f] = np.zeros((n, 6))
            setattr(P, f, _dp(arrs[f]))
        arrs["F"] = np.zeros((n, 9))
        P.F = _dp(arrs["F"])
        for f in ("volume", "mass", "density"):
            arrs[f] = np.zeros(n)
            setattr(P, f, _dp(arrs[f]))
        arrs["cell"] = np.zeros(n, dtype=np.int64)
        P.cell = _i64p(arrs["cell"])
        arrs["material"] = np.zeros(n, dtype=np.int32)
        P.material = _i32p(arrs["material"])
        arrs["svars"] = np.zeros((n, 9))
        P.svars = _dp(arrs["svars"])
        arrs["status"] = np.zeros(n, dtype=np.int32)
        P.status = _i32p(arrs["status"])
        arrs["mapping"] = np.zeros((n, 9))
        P.mapping = _dp(arrs["mapping"])
        self._check(lib().mpmo_get_particles(self.h, C.byref(P)))
        for f in FIELDS3:
            arrs[f] = arrs[f][:, :self.dim]
        return arrs

    def set(self, arrs):
        n = self.nparticles
        P = Particles()
        keep = []
        for f in FIELDS3:
            if f in arrs:
                a = np.zeros((n, 3))
                a[:, :self.dim] = np.asarray(arrs[f])[:, :self.dim]
                keep.append(a)
                setattr(P, f, _dp(a))
        for f in ("stress", "strain", "F", "volume", "mass", "density", "svars", "mapping"):
            if f in arrs:
                a = np.ascontiguousarray(arrs[f], dtype=np.float64)
                keep.append(a)
                setattr(P, f, _dp(a))
        if "cell" in arrs:
            a = np.ascontiguousarray(arrs["cell"], dtype=np.int64)
            keep.append(a)
            P.cell = _i64p(a)
        self._check(lib().mpmo_set_particles(self.h, C.byref(P)))

    NODE_COLS = {"mass": 0, "momentum": slice(1, 4), "external_force": slice(4, 7),
                 "internal_force": slice(7, 10), "velocity": slice(10, 13),
                 "acceleration": slice(13, 16), "status": 16}

    def nodes(self, nnodes):
        """nnodes x 17: mass, momentum[3], fext[3], fint[3], vel[3], acc[3], status."""
        out = np.zeros((nnodes, 17))
        self._check(lib().mpmo_get_nodes(self.h, _dp(out)))
        return out

    def set_nodes(self, table):
        table = np.ascontiguousarray(table, dtype=np.float64)
        self._check(lib().mpmo_set_nodes(self.h, _dp(table)))

    PHASES = {"initialise": 0, "p2g_mass_momentum": 1, "compute_velocity": 2,
              "stress_strain": 3, "body_force": 4, "internal_force": 5, "node_update": 6,
              "g2p": 7, "locate": 8}

    def phase(self, name, dt=0.0, gravity=(0.0, 0.0, 0.0)):
        g = np.zeros(3)
        g[:len(gravity)] = gravity
        self._check(lib().mpmo_phase(self.h, self.PHASES[name], dt, _dp(g)))


def build_oracle(prob, nthreads=1, **overrides):
    """Oracle instance for a mpm_b200.problems.Problem (same set-up calls)."""
    from mpm_b200.problems import apply_problem
    a = dict(prob.analysis)
    a.update(overrides)
    o = Oracle(prob.dim, scheme=a.get("scheme", "usf"),
               velocity_update=a.get("velocity_update", "flip"), dt=a["dt"],
               gravity=a.get("gravity", (0, 0, 0)), damping_factor=a.get("damping_factor", 0.0),
               blending_ratio=a.get("blending_ratio", 1.0),
               gravity_ramping_time=a.get("gravity_ramping_time", 0.0),
               locate_particles=a.get("locate_particles", True), nthreads=nthreads,
               isoparametric=a.get("isoparametric", False))
    return apply_problem(prob, o)
