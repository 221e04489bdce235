"""Python host side of the explicit MPM step on the B200.

``MPMExplicit`` mirrors the reference's solver surface (mpm::MPMExplicit,
include/solvers/mpm_explicit.tcc): it is built from a ``Problem`` (mesh,
materials, constraints, particles, analysis settings) or from the reference's
own JSON input (``MPMExplicit.from_input``), and advances with ``solve()`` or
``step(n)``.  All arithmetic runs in libmpm_b200.so through its C ABI.
"""
import ctypes as C
import json

import numpy as np

from . import _native
from ._native import MPMError

SCHEMES = {"usf": 0, "usl": 1, "musl": 2}
# the reference's VelocityUpdate order (data_types.h:50); asflip, tpic and apic
# carry a mapping matrix per particle (``read()["mapping"]``)
VELOCITY_UPDATES = {"flip": 0, "pic": 1, "asflip": 2, "tpic": 3, "apic": 4}
PRECISIONS = {"fp64": 0, "mixed": 1}


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i64p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def _i32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def pinned_empty(shape, dtype=np.float64):
    """An uninitialised numpy array in page-locked host memory
    (mpm_gpu_host_alloc), freed when the array and its views are gone.
    Solver.load and Solver.read copy such arrays by DMA directly."""
    import weakref
    L = _native.lib()
    nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
    ptr = C.c_void_p()
    rc = L.mpm_gpu_host_alloc(max(nbytes, 1), C.byref(ptr))
    if rc != 0:
        raise MPMError(rc, "mpm_gpu_host_alloc: cannot pin %d bytes" % nbytes)
    buf = (C.c_char * max(nbytes, 1)).from_address(ptr.value)
    weakref.finalize(buf, L.mpm_gpu_host_free, C.c_void_p(ptr.value))
    return np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)


class Solver:
    """Thin owner of one ``mpm_gpu_t`` handle."""

    def __init__(self, dim, scheme="usf", velocity_update="flip", dt=1e-5, gravity=(0, 0, 0),
                 damping_factor=0.0, blending_ratio=1.0, gravity_ramping_time=0.0,
                 locate_particles=True, precision="fp64", device=0):
        L = _native.lib()
        cfg = _native.Config()
        cfg.dim = dim
        cfg.scheme = SCHEMES[scheme]
        cfg.velocity_update = VELOCITY_UPDATES[velocity_update]
        self.mapped = cfg.velocity_update >= VELOCITY_UPDATES["asflip"]
        cfg.precision = PRECISIONS[precision]
        cfg.blending_ratio = blending_ratio
        cfg.dt = dt
        cfg.damping_factor = damping_factor
        g = list(gravity) + [0.0] * (3 - len(gravity))
        for i in range(3):
            cfg.gravity[i] = g[i]
        cfg.gravity_ramping_time = gravity_ramping_time
        cfg.locate_particles = 1 if locate_particles else 0
        cfg.device = device
        h = C.c_void_p()
        rc = L.mpm_gpu_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise MPMError(rc, "mpm_gpu_create failed")
        self.h = h
        self.dim = dim
        self.L = L

    def close(self):
        if getattr(self, "h", None):
            self.L.mpm_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        if rc != 0:
            raise MPMError(rc, self.L.mpm_gpu_last_error(self.h).decode())

    def set_mesh(self, coords, cells):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        self._ck(self.L.mpm_gpu_set_mesh(self.h, coords.shape[0], _dp(coords), cells.shape[0],
                                         cells.shape[1], _i64p(cells)))

    def add_material(self, mid, mtype, props):
        self._ck(self.L.mpm_gpu_add_material(self.h, mid, mtype.encode(),
                                             json.dumps(props).encode()))

    def _nodal(self, fn, nid, direction, value):
        nid = np.ascontiguousarray(nid, dtype=np.int64)
        d = np.ascontiguousarray(direction, dtype=np.int32)
        v = np.ascontiguousarray(value, dtype=np.float64)
        self._ck(fn(self.h, len(nid), _i64p(nid), _i32p(d), _dp(v)))

    def add_velocity_constraints(self, nid, direction, value):
        self._nodal(self.L.mpm_gpu_add_velocity_constraints, nid, direction, value)

    def add_acceleration_constraints(self, nid, direction, value):
        self._nodal(self.L.mpm_gpu_add_acceleration_constraints, nid, direction, value)

    def add_friction_constraints(self, nid, direction, sign_n, mu):
        nid = np.ascontiguousarray(nid, dtype=np.int64)
        d = np.ascontiguousarray(direction, dtype=np.int32)
        s = np.ascontiguousarray(sign_n, dtype=np.int32)
        m = np.ascontiguousarray(mu, dtype=np.float64)
        self._ck(self.L.mpm_gpu_add_friction_constraints(self.h, len(nid), _i64p(nid), _i32p(d),
                                                         _i32p(s), _dp(m)))

    def set_nodal_euler_angles(self, nid, angles):
        """Rotated frames (dim Euler angles per node, radians) for the nodes'
        velocity, acceleration and friction constraints."""
        nid = np.ascontiguousarray(nid, dtype=np.int64)
        a = np.ascontiguousarray(angles, dtype=np.float64)
        self._ck(self.L.mpm_gpu_set_nodal_euler_angles(self.h, len(nid), _i64p(nid), _dp(a)))

    def add_particles(self, coords, material_id):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        self._ck(self.L.mpm_gpu_add_particles(self.h, coords.shape[0], _dp(coords), material_id))

    def assign_particle_materials(self, pids, material_id):
        """Material set: the particles with these ids take ``material_id``
        (before ``initialise``; ids without a particle are skipped)."""
        p = np.ascontiguousarray(pids, dtype=np.int64)
        self._ck(self.L.mpm_gpu_assign_particle_materials(self.h, len(p), _i64p(p), material_id))

    def initialise(self):
        self._ck(self.L.mpm_gpu_initialise(self.h))

    def assign_particle_stresses(self, stress):
        stress = np.ascontiguousarray(stress, dtype=np.float64).reshape(-1, 6)
        self._ck(self.L.mpm_gpu_assign_particle_stresses(self.h, stress.shape[0], _dp(stress)))

    def add_particle_velocity_constraint(self, pids, direction, value):
        if pids is None:
            self._ck(self.L.mpm_gpu_add_particle_velocity_constraint(self.h, -1, None, direction,
                                                                     value))
            return
        p = np.ascontiguousarray(pids, dtype=np.int64)
        self._ck(self.L.mpm_gpu_add_particle_velocity_constraint(self.h, len(p), _i64p(p),
                                                                 direction, value))

    def step(self, n=1):
        self._ck(self.L.mpm_gpu_step(self.h, n))

    def step_timed(self, n=1):
        """Advance n steps; return their device time in ms (CUDA events)."""
        ms = C.c_double()
        self._ck(self.L.mpm_gpu_step_timed(self.h, n, C.byref(ms)))
        return ms.value

    def set_launch_shape(self, p2g_tile=0, node_threads=0, return_blocks_per_sm=0):
        """Launch shape of the steps (0: the built-in default); results do
        not depend on it."""
        self._ck(self.L.mpm_gpu_set_launch_shape(self.h, int(p2g_tile), int(node_threads),
                                                 int(return_blocks_per_sm)))

    def set_persistent(self, steps_per_launch):
        """Advance up to ``steps_per_launch`` whole steps per persistent
        (cooperative) kernel launch; 0 returns to one launch per pass,
        replayed from a CUDA graph.  Bit for bit the same results."""
        self._ck(self.L.mpm_gpu_set_persistent(self.h, int(steps_per_launch)))

    def persistent(self):
        """(steps per persistent launch, 0 when off; whether those launches
        replay a captured CUDA graph)."""
        n, g = C.c_int32(), C.c_int32()
        self._ck(self.L.mpm_gpu_get_persistent(self.h, C.byref(n), C.byref(g)))
        return n.value, bool(g.value)

    def launch_shape(self):
        """(p2g_tile, node_threads, return_blocks_per_sm) in use."""
        out = (C.c_int32 * 3)()
        self._ck(self.L.mpm_gpu_get_launch_shape(self.h, out))
        return tuple(int(v) for v in out)

    def autotune(self, steps=5):
        """Time the launch-shape candidates on this solver's state and keep
        the fastest; the state and step counter are restored, so the run
        continues as without it.  Returns the report (ms per step per
        candidate, the chosen shape)."""
        buf = C.create_string_buffer(4096)
        self._ck(self.L.mpm_gpu_autotune(self.h, int(steps), buf, len(buf)))
        return json.loads(buf.value.decode())

    def set_profiling(self, enable=True):
        self._ck(self.L.mpm_gpu_set_profiling(self.h, 1 if enable else 0))

    def kernel_profile(self):
        """{kernel name: (total ms, launches)} since profiling was enabled."""
        out = {}
        k = 0
        while True:
            name = C.c_char_p()
            ms = C.c_double()
            n = C.c_int64()
            if self.L.mpm_gpu_kernel_profile(self.h, k, C.byref(name), C.byref(ms),
                                             C.byref(n)) != 0:
                break
            out[name.value.decode()] = (ms.value, n.value)
            k += 1
        return out

    @property
    def launch_count(self):
        return self.L.mpm_gpu_launch_count(self.h)

    @property
    def nparticles(self):
        return self.L.mpm_gpu_nparticles(self.h)

    @property
    def current_step(self):
        return self.L.mpm_gpu_current_step(self.h)

    def set_isoparametric(self, on=True):
        """Isoparametric local coordinates on a general mesh (the mesh's
        "isoparametric" flag; before the particles are added)."""
        self._ck(self.L.mpm_gpu_set_isoparametric(self.h, 1 if on else 0))

    def state_buffers(self, pinned=False):
        """Empty arrays for ``read(out=...)`` and ``load``: x, u, v as (n, 3)
        rows, in page-locked memory with ``pinned`` (see pinned_empty)."""
        n = self.nparticles
        new = pinned_empty if pinned else (lambda shape, dtype=np.float64: np.zeros(shape, dtype))
        return {"x": new((n, 3)), "u": new((n, 3)), "v": new((n, 3)), "stress": new((n, 6)),
                "strain": new((n, 6)), "F": new((n, 9)), "volume": new((n,)), "mass": new((n,)),
                "density": new((n,)), "cell": new((n,), np.int64), "material": new((n,), np.int32),
                "svars": new((n, 9))}

    def read(self, out=None):
        """Particle state as numpy arrays (rows = particles); with ``out`` (the
        arrays of ``state_buffers``) the state is written into them."""
        n = self.nparticles
        if out is None:
            out = self.state_buffers()
        else:
            out = dict(out)
        P = _native.Particles()
        for k, w in (("stress", 6), ("strain", 6), ("F", 9), ("volume", 0), ("mass", 0),
                     ("density", 0), ("svars", 9), ("x", 3), ("u", 3), ("v", 3)):
            a = out[k]
            if a.shape != ((n, w) if w else (n,)) or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("read: %s must be a C-contiguous float64 array of %s rows" % (k, w or 1))
            setattr(P, k, _dp(a))
        for k, t in (("cell", np.int64), ("material", np.int32)):
            if out[k].shape != (n,) or out[k].dtype != t or not out[k].flags.c_contiguous:
                raise ValueError("read: %s must be a C-contiguous %s array" % (k, np.dtype(t).name))
        P.cell = _i64p(out["cell"])
        P.material = _i32p(out["material"])
        self._ck(self.L.mpm_gpu_read_particles(self.h, C.byref(P)))
        for k in ("x", "u", "v"):
            out[k] = out[k][:, :self.dim]
        if self.mapped:
            out["mapping"] = np.zeros((n, 9))
            self._ck(self.L.mpm_gpu_read_mapping_matrix(self.h, _dp(out["mapping"])))
        return out

    def load(self, state):
        """Replace the particle state (arrays as returned by ``read``)."""
        n = len(state["x"])
        keep = {}
        P = _native.Particles()
        for k in ("x", "u", "v"):
            if k in state:
                a = np.asarray(state[k])
                if a.shape == (n, 3) and self.dim == 3:
                    a = np.ascontiguousarray(a, dtype=np.float64)
                else:  # rows of 3 components, zero beyond the solver's dimension
                    b = np.zeros((n, 3))
                    b[:, :self.dim] = a[:, :self.dim]
                    a = b
                keep[k] = a
                setattr(P, k, _dp(a))
        for k in ("stress", "strain", "F", "volume", "mass", "density", "svars"):
            if k in state:
                keep[k] = np.ascontiguousarray(state[k], dtype=np.float64)
                setattr(P, k, _dp(keep[k]))
        keep["cell"] = np.ascontiguousarray(state["cell"], dtype=np.int64)
        P.cell = _i64p(keep["cell"])
        keep["material"] = np.ascontiguousarray(state["material"], dtype=np.int32)
        P.material = _i32p(keep["material"])
        self._ck(self.L.mpm_gpu_load_particles(self.h, n, C.byref(P)))
        if self.mapped and "mapping" in state:
            keep["mapping"] = np.ascontiguousarray(state["mapping"], dtype=np.float64)
            self._ck(self.L.mpm_gpu_load_mapping_matrix(self.h, _dp(keep["mapping"])))

    def write_pod(self, dtype=None):
        """PODParticle records of the particles in the mesh (particle.tcc:180-306),
        packed on the device, as a numpy structured array."""
        from . import pod
        dtype = pod.POD_DTYPE if dtype is None else dtype
        size, offs, sizes = pod.layout(dtype)
        cap = self.nparticles
        out = np.zeros(cap, dtype=dtype)
        n = C.c_int64()
        psz = C.POINTER(C.c_size_t)
        self._ck(self.L.mpm_gpu_write_pod(self.h, out.ctypes.data_as(C.c_void_p), cap, C.byref(n),
                                          size, offs.ctypes.data_as(psz),
                                          sizes.ctypes.data_as(psz), 74))
        return out[:n.value]

    def load_pod(self, records):
        """Checkpoint resume from PODParticle records (mesh.tcc:1663-1720)."""
        from . import pod
        records = np.ascontiguousarray(records)
        size, offs, sizes = pod.layout(records.dtype)
        psz = C.POINTER(C.c_size_t)
        self._ck(self.L.mpm_gpu_load_pod(self.h, records.ctypes.data_as(C.c_void_p), len(records),
                                         size, offs.ctypes.data_as(psz),
                                         sizes.ctypes.data_as(psz), 74))

    # ---- slab decomposition (mpm_b200.slab): a USL step in two halves with the
    # halo partials of one x-column of cells moved between them
    def step_begin(self):
        self._ck(self.L.mpm_gpu_step_begin(self.h))

    def step_end(self):
        self._ck(self.L.mpm_gpu_step_end(self.h))

    def halo_bytes(self):
        n = C.c_int64()
        self._ck(self.L.mpm_gpu_halo_bytes(self.h, C.byref(n)))
        return n.value

    def halo_pack(self, layer, dst_ptr):
        self._ck(self.L.mpm_gpu_halo_pack(self.h, int(layer), C.c_void_p(dst_ptr)))

    def halo_unpack(self, layer, src_ptr):
        self._ck(self.L.mpm_gpu_halo_unpack(self.h, int(layer), C.c_void_p(src_ptr)))

    def layer_count(self, x_lo, x_hi):
        """Particles whose cell's x index is below x_lo, and at or above x_hi."""
        a, b = C.c_int64(), C.c_int64()
        self._ck(self.L.mpm_gpu_layer_count(self.h, int(x_lo), int(x_hi), C.byref(a), C.byref(b)))
        return a.value, b.value

    def write_hdf5(self, path):
        """The reference's HDF5 particle table (Mesh::write_particles_hdf5)."""
        self._ck(self.L.mpm_gpu_write_hdf5(self.h, str(path).encode()))

    def load_hdf5(self, path):
        """Checkpoint resume from an HDF5 particle table (Mesh::read_particles_hdf5)."""
        self._ck(self.L.mpm_gpu_load_hdf5(self.h, str(path).encode()))

    SENSITIVITY_KINDS = {"youngs_modulus": 0, "friction": 1, "cohesion": 2, "dilation": 3}
    SENSITIVITY_FIELDS = {"x": 0, "u": 1, "v": 2, "stress": 3}

    def set_sensitivities(self, params):
        """Carry derivatives with respect to up to two material parameters,
        given as [(material_id, "youngs_modulus" | "friction" | "cohesion" |
        "dilation"), ...]; an empty list turns them off."""
        n = len(params)
        mids = np.array([m for m, _ in params], dtype=np.int32)
        kinds = np.array([self.SENSITIVITY_KINDS[k] for _, k in params], dtype=np.int32)
        self._ck(self.L.mpm_gpu_set_sensitivities(self.h, n, _i32p(mids), _i32p(kinds)))
        self._nsens = n

    def read_sensitivities(self, field="x"):
        """d(field)/d(parameter): array (n_parameters, n_particles, dim) for x,
        u, v; (n_parameters, n_particles, 6) for stress."""
        n = getattr(self, "_nsens", 0)
        width = 6 if field == "stress" else 3
        out = np.zeros((max(n, 1), self.nparticles, width))
        self._ck(self.L.mpm_gpu_read_sensitivities(self.h, self.SENSITIVITY_FIELDS[field],
                                                   _dp(out)))
        return out if field == "stress" else out[:, :, :self.dim]

    def adjoint_record(self, nsteps, params=(), checkpoint_every=0):
        """Advance ``nsteps`` keeping checkpoints for the reverse sweep;
        ``params`` as for ``set_sensitivities``."""
        n = len(params)
        mids = np.array([m for m, _ in params], dtype=np.int32)
        kinds = np.array([self.SENSITIVITY_KINDS[k] for _, k in params], dtype=np.int32)
        self._ck(self.L.mpm_gpu_adjoint_record(self.h, int(nsteps), int(checkpoint_every), n,
                                               _i32p(mids), _i32p(kinds)))
        self._nadj = n

    def adjoint_reverse(self, dL_dx=None, dL_dv=None):
        """Reverse sweep of the recorded run for terminal cotangents dL/dx,
        dL/dv (particle rows, dim or 3 columns): a dict with dL/dparameter
        ("params") and the cotangents of the recorded run's initial state
        ("x0", "v0": n x dim, "stress0": n x 6)."""
        n = self.nparticles

        def rows(a):
            if a is None:
                return None
            a = np.asarray(a, dtype=np.float64)
            b = np.zeros((n, 3))
            b[:, :a.shape[1]] = a
            return b
        gx, gv = rows(dL_dx), rows(dL_dv)
        out = {"params": np.zeros(max(getattr(self, "_nadj", 0), 1)), "x0": np.zeros((n, 3)),
               "v0": np.zeros((n, 3)), "stress0": np.zeros((n, 6))}
        self._ck(self.L.mpm_gpu_adjoint_reverse(
            self.h, _dp(gx) if gx is not None else None, _dp(gv) if gv is not None else None,
            _dp(out["params"]), _dp(out["x0"]), _dp(out["v0"]), _dp(out["stress0"])))
        out["params"] = out["params"][:getattr(self, "_nadj", 0)]
        out["x0"] = out["x0"][:, :self.dim]
        out["v0"] = out["v0"][:, :self.dim]
        return out

    def adjoint_run(self, nsteps, params, x_target, checkpoint_every=0):
        """(loss, dL/dparameter) of L = sum |x_final - x_target|^2."""
        n = self.nparticles
        t = np.zeros((n, 3))
        t[:, :self.dim] = np.asarray(x_target)[:, :self.dim]
        mids = np.array([m for m, _ in params], dtype=np.int32)
        kinds = np.array([self.SENSITIVITY_KINDS[k] for _, k in params], dtype=np.int32)
        loss = C.c_double()
        grad = np.zeros(max(len(params), 1))
        self._ck(self.L.mpm_gpu_adjoint_run(self.h, int(nsteps), int(checkpoint_every),
                                            len(params), _i32p(mids), _i32p(kinds), _dp(t),
                                            C.byref(loss), _dp(grad)))
        self._nadj = len(params)
        return loss.value, grad[:len(params)]

    def set_current_step(self, step):
        self._ck(self.L.mpm_gpu_set_current_step(self.h, int(step)))

    def device_field(self, field):
        """(address, stride, ncomp) of a device-resident particle field."""
        names = {"x": 0, "u": 1, "v": 2, "stress": 3, "strain": 4, "F": 5, "volume": 6,
                 "density": 7, "mass": 8}
        base = C.c_void_p()
        stride = C.c_int64()
        nc = C.c_int32()
        self._ck(self.L.mpm_gpu_device_field(self.h, names[field], C.byref(base), C.byref(stride),
                                             C.byref(nc)))
        return base.value, stride.value, nc.value


def material_stress_batch(dim, mtype, props, stress, dstrain, density, state=None, device=0):
    """Material<Tdim>::compute_stress on the device for a batch of points."""
    L = _native.lib()
    stress = np.ascontiguousarray(stress, dtype=np.float64).reshape(-1, 6)
    n = stress.shape[0]
    dstrain = np.ascontiguousarray(dstrain, dtype=np.float64).reshape(n, 6)
    density = np.ascontiguousarray(np.broadcast_to(np.asarray(density, dtype=np.float64), (n,)))
    st = np.zeros((n, 9)) if state is None else np.array(state, dtype=np.float64).reshape(n, 9)
    out = np.zeros((n, 6))
    rc = L.mpm_gpu_material_stress_batch(device, dim, mtype.encode(), json.dumps(props).encode(),
                                         n, _dp(stress), _dp(dstrain), _dp(density), _dp(st),
                                         _dp(out))
    if rc != 0:
        raise MPMError(rc, "material_stress_batch failed")
    return out, st
