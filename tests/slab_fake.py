"""A CPU stand-in for the solver in slab-decomposition tests (test helper).

It has the solver methods the slab orchestration calls and a toy step whose
outcome depends on every piece of the decomposition: "P2G" sums the mass and
x-momentum of each cell's particles; the "node update" gives each cell the
velocity (M[i-1] + M[i] + M[i+1]) / (m[i-1] + m[i] + m[i+1]) over its x
neighbours -- at a slab edge one of them is a ghost column, so a missing or
misplaced halo changes it -- plus a drift; particles move with their cell's
velocity (at least 0.2 and below 2.2 times a cell per 0.01 s, so at most
half a cell per step) and are relocated, so they cross slab edges.  Masses are 1 and
momenta multiples of 1/2: every sum is exact whatever the particle order.
"""
import ctypes

import numpy as np

NVALS = 2  # per cell: mass, x-momentum


class FakeSolver:
    def __init__(self, prob, dt=2e-3, drift=1.2):
        self.dim = prob.dim
        self.shape = tuple(prob.shape)
        self.dx = prob.dx
        self.x0 = float(np.min(prob.coords[:, 0]))
        self.dt, self.drift = dt, drift
        self.ncells = int(np.prod(self.shape))
        self.partials = np.zeros((self.ncells, NVALS))
        self.cnt = np.zeros(self.ncells, dtype=np.int32)
        self.state = None
        self.current_step = 0

    # state
    def load(self, st):
        self.state = {k: np.array(v, copy=True) for k, v in st.items()}

    def read(self):
        return {k: np.array(v, copy=True) for k, v in self.state.items()}

    def set_current_step(self, s):
        self.current_step = s

    def close(self):
        pass

    @property
    def nparticles(self):
        return len(self.state["x"])

    # halo layers: [ncols][NVALS] float64 then [ncols] int32, as the library packs them
    def _cols(self):
        return int(np.prod(self.shape[1:]))

    def _column_cells(self, layer):
        return layer + self.shape[0] * np.arange(self._cols())

    def halo_bytes(self):
        return self._cols() * NVALS * 8 + self._cols() * 4

    def halo_pack(self, layer, ptr):
        c = self._column_cells(layer)
        v = np.ascontiguousarray(self.partials[c]).tobytes() + self.cnt[c].astype(np.int32).tobytes()
        ctypes.memmove(ptr, v, len(v))

    def halo_unpack(self, layer, ptr):
        c = self._column_cells(layer)
        n = self._cols()
        raw = ctypes.string_at(ptr, n * NVALS * 8 + n * 4)
        self.partials[c] = np.frombuffer(raw[:n * NVALS * 8], dtype=np.float64).reshape(n, NVALS)
        self.cnt[c] = np.frombuffer(raw[n * NVALS * 8:], dtype=np.int32)

    # the toy step
    def step_begin(self):
        self.partials[:] = 0.0
        self.cnt[:] = 0
        c = self.state["cell"]
        live = c >= 0
        np.add.at(self.partials[:, 0], c[live], self.state["mass"][live])
        np.add.at(self.partials[:, 1], c[live], self.state["mass"][live] * self.state["v"][live, 0])
        np.add.at(self.cnt, c[live], 1)

    def step_end(self):
        nx = self.shape[0]
        P = self.partials.reshape(-1, nx, NVALS)  # [rest][i][value]
        m = P[:, :, 0]
        M = P[:, :, 1]
        ms = m.copy()
        Ms = M.copy()
        ms[:, 1:] += m[:, :-1]
        ms[:, :-1] += m[:, 1:]
        Ms[:, 1:] += M[:, :-1]
        Ms[:, :-1] += M[:, 1:]
        vel = np.where(ms > 0, Ms / np.where(ms > 0, ms, 1.0), 0.0).reshape(-1) + self.drift
        c = self.state["cell"]
        live = c >= 0
        self.state["x"][live, 0] += vel[c[live]] * self.dt
        i = np.floor((self.state["x"][live, 0] - self.x0) / self.dx).astype(np.int64)
        if np.any(i < 0) or np.any(i >= nx):
            raise RuntimeError("particle left the local grid")
        rest = c[live] // nx
        self.state["cell"][live] = i + nx * rest
        self.current_step += 1

    def layer_count(self, x_lo, x_hi):
        c = self.state["cell"]
        i = c[c >= 0] % self.shape[0]
        return int(np.sum(i < x_lo)), int(np.sum(i >= x_hi))


def initial_state(prob, seed=4):
    """Particles at the problem's positions with unit mass and x-velocities in
    {-1, -1/2, 0, 1/2, 1}; cells of the global grid."""
    pts = np.concatenate([p for p, _ in prob.particles])
    n = len(pts)
    rng = np.random.default_rng(seed)
    nx = prob.shape[0]
    ijk = np.floor(pts / prob.dx).astype(np.int64)
    cell = ijk[:, 0] + nx * ijk[:, 1]
    if prob.dim == 3:
        cell = ijk[:, 0] + nx * (ijk[:, 1] + prob.shape[1] * ijk[:, 2])
    v = np.zeros((n, prob.dim))
    v[:, 0] = rng.integers(-2, 3, n) * 0.5
    return {"x": pts.copy(), "v": v, "mass": np.ones(n), "cell": cell,
            "material": np.zeros(n, dtype=np.int32)}
