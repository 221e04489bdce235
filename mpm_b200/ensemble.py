"""Batched ensembles: many independent 2D slope simulations in one solver.

The runs are packed side by side, each in its own rectangle of one structured
quad4 grid, with one empty cell column and row between rectangles: no node is
shared by two runs, so the runs do not interact, and every kernel of a step
processes all runs at once (one launch per step phase for the whole
ensemble).  Each run has its own material slot (its friction angle and
cohesion) and its own walls, so the walls of one run never constrain the
nodes of another.  The per-step launches are replayed from a CUDA graph by the
library (see ``mpm_gpu_step``), so small runs do not pay launch latency.

Slope geometry (one run): a rectangle of ``width`` x ``height`` cells with a
45 degree face on its right, i.e. layer k (from the floor) spans the x cells
[0, width + height - k); 2x2 particles per cell; the run's rectangle adds
``margin`` empty cells to the right and above.  Walls: slip on the left, right
and top of the rectangle, frictional floor.
"""
from dataclasses import dataclass

import numpy as np

from . import problems as P


@dataclass
class SlopeRun:
    height: int           # slope height in cells
    width: int            # width of the rectangular base in cells
    phi: float            # friction angle (degrees)
    cohesion: float       # Pa
    margin: int = 20
    seed: int = P.SEED_BASE

    @property
    def cells(self):
        return (self.width + self.height + self.margin, self.height + self.margin)

    @property
    def nparticles(self):
        h, w = self.height, self.width
        return 4 * (h * w + h * (h + 1) // 2)


def random_runs(nruns, n_min=2000, n_max=40000, seed=P.SEED_BASE + 2):
    """Seeded ensemble: particle counts ~ U[n_min, n_max], phi ~ U[20, 40] deg,
    c ~ U[0, 5] kPa; the slope height follows from the count (base width =
    height)."""
    rng = np.random.default_rng(seed)
    runs = []
    for r in range(nruns):
        n = rng.uniform(n_min, n_max)
        cells = n / 4.0
        h = max(2, int(round((-0.5 + np.sqrt(0.25 + 6.0 * cells)) / 3.0)))
        runs.append(SlopeRun(height=h, width=h, phi=float(rng.uniform(20.0, 40.0)),
                             cohesion=float(rng.uniform(0.0, 5000.0)),
                             seed=P.SEED_BASE + 1000 * (r + 1)))
    return runs


def _pack(runs, gap=1):
    """Shelf packing of the runs' rectangles: origins (in cells) and the grid."""
    sizes = [(r.cells[0] + gap, r.cells[1] + gap) for r in runs]
    area = sum(a * b for a, b in sizes)
    row_width = max(max(a for a, _ in sizes), int(np.sqrt(area) * 1.3))
    origins, x, y, row_h, width = [], 0, 0, 0, 0
    for a, b in sizes:
        if x + a > row_width and x > 0:
            y += row_h
            x, row_h = 0, 0
        origins.append((x, y))
        x += a
        row_h = max(row_h, b)
        width = max(width, x)
    return origins, (width, y + row_h)


def ensemble_problem(runs, dx=0.01, dt=1e-5, nsteps=2000, mu=0.4, E=5e6, nu=0.3, rho=1800.0,
                     scheme="usl", velocity_update="flip"):
    """One Problem holding every run; returns (problem, info) where info lists
    each run's origin (m) and particle range in the solver's particle order."""
    origins, shape = _pack(runs)
    coords, cells = P.structured_mesh(2, shape, dx)
    nx1 = shape[0] + 1
    mats, parts, stresses, vnid, vdir, fnid, ranges = [], [], [], [], [], [], []
    first = 0
    for r, (run, (ox, oy)) in enumerate(zip(runs, origins)):
        h, w = run.height, run.width
        layers = [P.quarter_point_particles(2, [(ox, ox + w + h - k), (oy + k, oy + k + 1)], dx,
                                            seed=run.seed + k)
                  for k in range(h)]
        pts = np.concatenate(layers)
        ix = np.floor(pts[:, 0] / dx) - ox
        top = (oy + np.clip(w + h - ix, 0, h)) * dx
        stresses.append(P.geostatic_stress(pts, 2, rho, nu, top))
        mats.append((r, "MohrCoulomb2D", P.mohr_coulomb(E, nu, rho, run.phi, run.cohesion, 0.0)))
        parts.append((pts, r))
        ranges.append((first, first + len(pts)))
        first += len(pts)
        nx, ny = run.cells
        ii = np.arange(ox, ox + nx + 1)
        jj = np.arange(oy, oy + ny + 1)
        left, right = ox + nx1 * jj, (ox + nx) + nx1 * jj
        floor, roof = ii + nx1 * oy, ii + nx1 * (oy + ny)
        vnid += [left, right, floor, roof]
        vdir += [np.zeros(len(jj), int), np.zeros(len(jj), int), np.ones(len(ii), int),
                 np.ones(len(ii), int)]
        fnid.append(floor)
    vnid = np.concatenate(vnid)
    vdir = np.concatenate(vdir)
    fnid = np.concatenate(fnid)
    prob = P.Problem(dim=2, shape=shape, dx=dx, coords=coords, cells=cells, materials=mats,
                     particles=parts, velocity_constraints=(vnid, vdir, np.zeros(len(vnid))),
                     friction_constraints=(fnid, np.ones(len(fnid), int),
                                           np.full(len(fnid), -1), np.full(len(fnid), mu)),
                     initial_stress=np.concatenate(stresses),
                     analysis=dict(scheme=scheme, velocity_update=velocity_update, dt=dt,
                                   nsteps=nsteps, gravity=(0.0, -9.81), damping_factor=0.0),
                     name="slope_ensemble")
    info = {"origins": [(ox * dx, oy * dx) for ox, oy in origins], "ranges": ranges,
            "shape": shape}
    return prob, info


def standalone_problem(run, **kw):
    """The same run alone in its own grid (for checks against the ensemble)."""
    prob, info = ensemble_problem([run], **kw)
    return prob


class Ensemble:
    """A solver over all runs, with per-run views of the particle state."""

    def __init__(self, runs, precision="mixed", device=0, **kw):
        self.runs = list(runs)
        self.problem, self.info = ensemble_problem(self.runs, **kw)
        self.solver = P.build_solver(self.problem, precision=precision, device=device)

    @property
    def nparticles(self):
        return self.solver.nparticles

    def step(self, n=1):
        self.solver.step(n)

    def step_timed(self, n=1):
        return self.solver.step_timed(n)

    def run_states(self):
        """Per-run dicts of the particle fields, positions relative to the
        run's origin."""
        st = self.solver.read()
        out = []
        for (a, b), o in zip(self.info["ranges"], self.info["origins"]):
            d = {k: v[a:b] for k, v in st.items()}
            d["x"] = d["x"] - np.asarray(o)
            out.append(d)
        return out

    def runout(self):
        """Per-run runout: the largest x of the run's particles (m, from the
        run's left wall)."""
        return np.array([s["x"][:, 0].max() for s in self.run_states()])
