"""Seeded synthetic inputs with the shapes of the benchmark configurations.

A ``Problem`` holds everything the reference reads from its JSON and ASCII
input (mpm_base.tcc:3-207, io_mesh_ascii.tcc): a structured quad4/hex8 mesh
(node ids lexicographic with x fastest, cell node order of
quadrilateral_element.tcc:1-7 and hexahedron_element.tcc:1-13), materials,
nodal velocity/friction constraints, particles and analysis settings.
``write_reference_input`` writes the same problem as the reference's own
input files.

Particles sit at the 2x2(x2) quarter points (0.25, 0.75)*dx of each filled
cell, each coordinate jittered by U(-1e-4, 1e-4) m from a splitmix64 stream
(seed = 20261203 + config index).
"""
import json
import os
from dataclasses import dataclass, field

import numpy as np

SEED_BASE = 20261203


def splitmix64_uniform(seed, n):
    """n doubles in [0, 1) from a splitmix64 stream."""
    M = np.uint64(0xFFFFFFFFFFFFFFFF)
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = (np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)) & M
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@dataclass
class Problem:
    dim: int
    shape: tuple            # cells per axis
    dx: float
    coords: np.ndarray      # nnodes x dim
    cells: np.ndarray       # ncells x nv
    materials: list         # [(id, type, props)]
    particles: list         # [(coords n x dim, material id)]
    velocity_constraints: tuple = None   # (nid, dir, value)
    friction_constraints: tuple = None   # (nid, dir, sign, mu)
    particle_velocity_constraints: list = field(default_factory=list)  # [(pids|None, dir, v)]
    nodal_euler_angles: tuple = None     # (nid, angles n x dim, radians): rotated boundaries
    initial_stress: np.ndarray = None    # nparticles x 6, creation order
    analysis: dict = field(default_factory=dict)
    name: str = ""

    @property
    def nparticles(self):
        return sum(len(c) for c, _ in self.particles)

    @property
    def nnodes(self):
        return len(self.coords)

    @property
    def ncells(self):
        return len(self.cells)


def structured_mesh(dim, shape, dx, origin=None):
    """Node coordinates i*dx (x fastest) and cell connectivity."""
    origin = np.zeros(dim) if origin is None else np.asarray(origin, dtype=np.float64)
    n = [s + 1 for s in shape]
    axes = [origin[d] + np.arange(n[d], dtype=np.float64) * dx for d in range(dim)]
    if dim == 2:
        Y, X = np.meshgrid(axes[1], axes[0], indexing="ij")
        coords = np.stack([X.ravel(), Y.ravel()], axis=1)
        j, i = np.meshgrid(np.arange(shape[1]), np.arange(shape[0]), indexing="ij")
        i, j = i.ravel(), j.ravel()
        nid = lambda a, b: a + n[0] * b
        cells = np.stack([nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)], axis=1)
    else:
        Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
        coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
        k, j, i = np.meshgrid(np.arange(shape[2]), np.arange(shape[1]), np.arange(shape[0]),
                              indexing="ij")
        i, j, k = i.ravel(), j.ravel(), k.ravel()
        nid = lambda a, b, c: a + n[0] * (b + n[1] * c)
        cells = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                          nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1),
                          nid(i, j + 1, k + 1)], axis=1)
    return coords, cells.astype(np.int64)


def quarter_point_particles(dim, cell_range, dx, ppc_dir=2, seed=SEED_BASE, jitter=1e-4,
                            origin=None):
    """Particles at the ppc_dir^dim interior points of every cell in the
    inclusive-exclusive index box cell_range = [(lo, hi)] * dim."""
    origin = np.zeros(dim) if origin is None else np.asarray(origin, dtype=np.float64)
    sub = (np.arange(ppc_dir, dtype=np.float64) + 0.5) / ppc_dir
    idx = [np.arange(lo, hi) for lo, hi in cell_range]
    if dim == 2:
        j, i, sj, si = np.meshgrid(idx[1], idx[0], sub, sub, indexing="ij")
        pts = np.stack([(i + si).ravel(), (j + sj).ravel()], axis=1) * dx
    else:
        k, j, i, sk, sj, si = np.meshgrid(idx[2], idx[1], idx[0], sub, sub, sub, indexing="ij")
        pts = np.stack([(i + si).ravel(), (j + sj).ravel(), (k + sk).ravel()], axis=1) * dx
    pts = pts + origin
    if jitter:
        u = splitmix64_uniform(seed, pts.size).reshape(pts.shape)
        pts = pts + (2.0 * u - 1.0) * jitter
    return pts


def boundary_nodes(coords, d, value, tol=1e-12):
    return np.nonzero(np.abs(coords[:, d] - value) < tol)[0]


def slip_box(coords, dim, faces=None):
    """Normal velocity 0 on the faces of the bounding box."""
    lo, hi = coords.min(axis=0), coords.max(axis=0)
    nid, dirs = [], []
    for d in range(dim):
        for side, val in (("lo", lo[d]), ("hi", hi[d])):
            if faces is not None and (d, side) not in faces:
                continue
            ids = boundary_nodes(coords, d, val)
            nid.append(ids)
            dirs.append(np.full(len(ids), d))
    nid = np.concatenate(nid)
    dirs = np.concatenate(dirs)
    return nid, dirs, np.zeros(len(nid))


def geostatic_stress(pts, dim, rho, nu, top, g=9.81):
    """K0 at-rest stress: vertical -rho g (top - height), horizontal K0 times
    it with K0 = nu / (1 - nu); no shear (compression negative)."""
    h = pts[:, dim - 1]
    sv = -rho * g * (top - h)
    k0 = nu / (1.0 - nu)
    st = np.zeros((len(pts), 6))
    if dim == 2:
        st[:, 0] = k0 * sv
        st[:, 1] = sv
        st[:, 2] = k0 * sv
    else:
        st[:, 0] = k0 * sv
        st[:, 1] = k0 * sv
        st[:, 2] = sv
    return st


def linear_elastic(E, nu, rho):
    return {"density": rho, "youngs_modulus": E, "poisson_ratio": nu}


def mohr_coulomb(E, nu, rho, phi, c, psi, tension_cutoff=0.0, softening=False,
                 residual=None):
    r = residual or {}
    return {"density": rho, "youngs_modulus": E, "poisson_ratio": nu, "softening": softening,
            "friction": phi, "dilation": psi, "cohesion": c,
            "residual_friction": r.get("friction", phi), "residual_dilation": r.get("dilation", psi),
            "residual_cohesion": r.get("cohesion", c), "peak_pdstrain": r.get("peak_pdstrain", 0.0),
            "residual_pdstrain": r.get("residual_pdstrain", 0.0), "tension_cutoff": tension_cutoff}


def column_2d(shape=(100, 50), block=(20, 40), dx=0.01, E=1e6, nu=0.3, rho=1800., dt=1e-5,
              nsteps=10000, scheme="usf", seed=SEED_BASE + 0, material="LinearElastic",
              velocity_update="flip"):
    """2D column collapse: walls x=0, x=max and floor y=0 slip; gravity -y."""
    coords, cells = structured_mesh(2, shape, dx)
    pts = quarter_point_particles(2, [(0, block[0]), (0, block[1])], dx, seed=seed)
    if material == "LinearElastic":
        mat = (0, "LinearElastic2D", linear_elastic(E, nu, rho))
    else:
        mat = (0, "MohrCoulomb2D", mohr_coulomb(E, nu, rho, 30., 0., 0.))
    vc = slip_box(coords, 2, faces={(0, "lo"), (0, "hi"), (1, "lo")})
    # a cohesionless MohrCoulomb material must not start at zero stress: at
    # the apex its plastic corrector is 0/0 (see geostatic_stress)
    st0 = geostatic_stress(pts, 2, rho, nu, block[1] * dx) if material != "LinearElastic" else None
    return Problem(dim=2, shape=shape, dx=dx, coords=coords, cells=cells, materials=[mat],
                   particles=[(pts, 0)], velocity_constraints=vc, initial_stress=st0,
                   analysis=dict(scheme=scheme, velocity_update=velocity_update, dt=dt,
                                 nsteps=nsteps, gravity=(0.0, -9.81), damping_factor=0.0),
                   name="column2d")


def column_3d(shape=(200, 100, 50), block=(100, 100, 50), dx=0.01, E=1e7, nu=0.3, rho=1800.,
              phi=30., c=0., psi=0., mu=0.4, dt=2e-6, nsteps=5000, scheme="usl",
              seed=SEED_BASE + 1, velocity_update="flip", material="MohrCoulomb",
              geostatic=True):
    """3D granular column: floor z=0 frictional (mu), other faces slip.

    The particles start from a K0 geostatic stress.  The benchmark text gives
    no initial stress, but a cohesionless (c = 0, psi = 0) MohrCoulomb point
    at zero stress makes the reference corrector divide 0 by 0
    (mohr_coulomb.tcc:453-455: dP/dsigma vanishes at the apex), so every
    particle would turn NaN on the first step; the reference reads initial
    stresses through particles_stresses (mpm_base.tcc:1591-1625)."""
    coords, cells = structured_mesh(3, shape, dx)
    pts = quarter_point_particles(3, [(0, block[0]), (0, block[1]), (0, block[2])], dx, seed=seed)
    if material == "MohrCoulomb":
        mat = (0, "MohrCoulomb3D", mohr_coulomb(E, nu, rho, phi, c, psi))
    else:
        mat = (0, "LinearElastic3D", linear_elastic(E, nu, rho))
    vc = slip_box(coords, 3)
    floor = boundary_nodes(coords, 2, coords[:, 2].min())
    fc = (floor, np.full(len(floor), 2), np.full(len(floor), -1), np.full(len(floor), mu))
    st0 = geostatic_stress(pts, 3, rho, nu, block[2] * dx) if geostatic else None
    return Problem(dim=3, shape=shape, dx=dx, coords=coords, cells=cells, materials=[mat],
                   particles=[(pts, 0)], velocity_constraints=vc, friction_constraints=fc,
                   initial_stress=st0,
                   analysis=dict(scheme=scheme, velocity_update=velocity_update, dt=dt,
                                 nsteps=nsteps, gravity=(0.0, 0.0, -9.81), damping_factor=0.0),
                   name="column3d")


def footing_slope(shape=(400, 200, 100), dx=0.005, foundation=20, slope_height=40, slope_top=30,
                  footing=(5, 25), dt=1e-6, nsteps=1000, mu=0.4, scheme="usl",
                  velocity_update="flip", footing_velocity=-0.05, seed=SEED_BASE + 4):
    """3D slope on a foundation under a rigid footing (16M particles by default).

    LinearElastic foundation (E=5e7, nu=0.3, rho=1800) filling the lowest
    ``foundation`` cell layers of the whole x-y plane; MohrCoulomb slope (phi=35,
    c=2 kPa, psi=0, rho=1800) on top: ``slope_height`` layers, the layer k above
    the foundation spanning x cells [0, slope_top + slope_height - k) (a 45 deg
    face); 2x2x2 particles per filled cell.  The footing is the set of slope
    particles in the top layer with x cells in [footing[0], footing[1]),
    driven down at ``footing_velocity`` m/s by a particle velocity constraint
    (mesh.tcc:1454-1467).  Slip walls, frictional floor, gravity -z, K0
    geostatic initial stress under the local surface."""
    coords, cells = structured_mesh(3, shape, dx)
    nx, ny = shape[0], shape[1]
    found = quarter_point_particles(3, [(0, nx), (0, ny), (0, foundation)], dx, seed=seed)
    layers = []
    for k in range(slope_height):
        w = min(slope_top + slope_height - k, nx)
        layers.append(quarter_point_particles(
            3, [(0, w), (0, ny), (foundation + k, foundation + k + 1)], dx, seed=seed + 1 + k))
    slope = np.concatenate(layers)

    def surface(x):  # top of the material above x
        cells_x = np.floor(x / dx)
        k_top = np.clip(slope_top + slope_height - cells_x, 0, slope_height)
        return (foundation + k_top) * dx

    rho, nu = 1800.0, 0.3
    st_f = geostatic_stress(found, 3, rho, nu, surface(found[:, 0]))
    st_s = geostatic_stress(slope, 3, rho, nu, surface(slope[:, 0]))
    top_z = (foundation + slope_height - 1) * dx
    on_footing = ((slope[:, 2] > top_z) & (slope[:, 0] >= footing[0] * dx) &
                  (slope[:, 0] < footing[1] * dx))
    pids = len(found) + np.nonzero(on_footing)[0]
    vc = slip_box(coords, 3)
    floor = boundary_nodes(coords, 2, coords[:, 2].min())
    fc = (floor, np.full(len(floor), 2), np.full(len(floor), -1), np.full(len(floor), mu))
    mats = [(0, "LinearElastic3D", linear_elastic(5e7, nu, rho)),
            (1, "MohrCoulomb3D", mohr_coulomb(1e7, nu, rho, 35.0, 2000.0, 0.0))]
    return Problem(dim=3, shape=shape, dx=dx, coords=coords, cells=cells, materials=mats,
                   particles=[(found, 0), (slope, 1)], velocity_constraints=vc,
                   friction_constraints=fc,
                   particle_velocity_constraints=[(pids, 2, footing_velocity)],
                   initial_stress=np.concatenate([st_f, st_s]),
                   analysis=dict(scheme=scheme, velocity_update=velocity_update, dt=dt,
                                 nsteps=nsteps, gravity=(0.0, 0.0, -9.81), damping_factor=0.0),
                   name="footing_slope")


def config_e():
    """3D footing on a MohrCoulomb slope over a LinearElastic foundation,
    400x200x100 hex8 cells of 5 mm, 16,032,000 particles."""
    return footing_slope()


def calibration_column(phi=30.0, E=1e7, shape=(80, 40, 30), block=(40, 40, 20), dx=0.02,
                       dt=1e-5, c=1000.0, tension_cutoff=0.0, nsteps=2000):
    """Config D: the 3D MohrCoulomb column (phi, E) whose final positions a
    calibration matches, 40x40x20 filled cells of 2 cm in an 80x40x30 mesh
    (256,000 particles), USL, dt 1e-5, K0 geostatic start.  Cohesion (1 kPa)
    and tension cutoff (0, the reference's default) are not calibrated."""
    p = column_3d(shape=shape, block=block, dx=dx, E=E, phi=phi, c=c, psi=0.0, dt=dt,
                  nsteps=nsteps, scheme="usl")
    mid, mt, props = p.materials[0]
    props = dict(props)
    props["tension_cutoff"] = tension_cutoff
    p.materials[0] = (mid, mt, props)
    return p


def config_d(phi=30.0, E=1e7):
    return calibration_column(phi=phi, E=E)


def config_a():
    """2D explicit USF column collapse, LinearElastic, 3,200 particles."""
    return column_2d()


def config_b(block=(100, 100, 50)):
    """3D granular column collapse, MohrCoulomb, USL; the 4M-particle block
    [0,1]x[0,1]x[0,0.5] by default ((100, 50, 50) gives the 2M block)."""
    return column_3d(block=block)


def build_solver(prob, solver_cls=None, with_particles=True, **overrides):
    """Create and initialise a GPU solver for ``prob`` (mesh, materials and
    constraints only with ``with_particles=False``, e.g. before a resume)."""
    from .solver import Solver
    a = dict(prob.analysis)
    a.update(overrides)
    s = (solver_cls or Solver)(prob.dim, scheme=a.get("scheme", "usf"),
                               velocity_update=a.get("velocity_update", "flip"), dt=a["dt"],
                               gravity=a.get("gravity", (0, 0, 0)),
                               damping_factor=a.get("damping_factor", 0.0),
                               blending_ratio=a.get("blending_ratio", 1.0),
                               gravity_ramping_time=a.get("gravity_ramping_time", 0.0),
                               locate_particles=a.get("locate_particles", True),
                               precision=a.get("precision", "fp64"),
                               device=a.get("device", 0))
    if a.get("isoparametric", False):
        s.set_isoparametric(True)
    apply_problem(prob, s, with_particles=with_particles)
    return s


def apply_problem(prob, s, with_particles=True):
    """Feed a problem into any object with the solver's set-up methods (the GPU
    solver or the CPU oracle)."""
    s.set_mesh(prob.coords, prob.cells)
    for mid, mtype, props in prob.materials:
        s.add_material(mid, mtype, props)
    if prob.velocity_constraints is not None:
        s.add_velocity_constraints(*prob.velocity_constraints)
    if prob.friction_constraints is not None:
        s.add_friction_constraints(*prob.friction_constraints)
    if prob.nodal_euler_angles is not None:
        s.set_nodal_euler_angles(*prob.nodal_euler_angles)
    if not with_particles:
        return s
    for pts, mid in prob.particles:
        s.add_particles(pts, mid)
    s.initialise()
    if prob.initial_stress is not None:
        s.assign_particle_stresses(prob.initial_stress)
    for pids, d, v in prob.particle_velocity_constraints:
        s.add_particle_velocity_constraint(pids, d, v)
    return s


def write_reference_input(prob, outdir, nsteps=None, output_steps=None):
    """Write the problem as the reference's input: mpm.json, mesh.txt,
    particles-<k>.txt, velocity-constraints.txt, friction-constraints.txt,
    particles-stresses.txt and entity_sets.json (formats of io_mesh_ascii.tcc,
    tests/io/write_mesh_particles.cc, mpm_base.tcc:1550-1625, io.cc:159-194)."""
    os.makedirs(outdir, exist_ok=True)
    dim = prob.dim
    with open(os.path.join(outdir, "mesh.txt"), "w") as f:
        f.write("! elementShape {}\n! elementNumPoints {}\n".format(
            "quadrilateral" if dim == 2 else "hexahedron", 4 if dim == 2 else 8))
        f.write(f"{prob.nnodes}\t{prob.ncells}\n")
        for c in prob.coords:
            f.write("\t".join(repr(float(v)) for v in c) + "\n")
        for c in prob.cells:
            f.write("\t".join(str(int(v)) for v in c) + "\n")
    pfiles = []
    for k, (pts, mid) in enumerate(prob.particles):
        name = f"particles-{k}.txt"
        with open(os.path.join(outdir, name), "w") as f:
            f.write(f"{len(pts)}\n")
            for p in pts:
                f.write("\t".join(repr(float(v)) for v in p) + "\n")
        pfiles.append((name, mid))
    bcs = {}
    if prob.velocity_constraints is not None:
        with open(os.path.join(outdir, "velocity-constraints.txt"), "w") as f:
            for n, d, v in zip(*prob.velocity_constraints):
                f.write(f"{int(n)}\t{int(d)}\t{repr(float(v))}\n")
        bcs["velocity_constraints"] = [{"file": "velocity-constraints.txt"}]
    if prob.friction_constraints is not None:
        with open(os.path.join(outdir, "friction-constraints.txt"), "w") as f:
            for n, d, s, m in zip(*prob.friction_constraints):
                f.write(f"{int(n)}\t{int(d)}\t{int(s)}\t{repr(float(m))}\n")
        bcs["friction_constraints"] = [{"file": "friction-constraints.txt"}]
    psets, pvcs = [], []
    for k, (pids, d, v) in enumerate(prob.particle_velocity_constraints):
        ids = np.arange(prob.nparticles) if pids is None else np.asarray(pids)
        psets.append({"id": k, "set": [int(i) for i in ids]})
        pvcs.append({"pset_id": k, "dir": int(d), "velocity": float(v)})
    if pvcs:
        bcs["particles_velocity_constraints"] = pvcs
    a = prob.analysis
    nsteps = nsteps if nsteps is not None else a.get("nsteps", 1)
    cfg = {
        "title": prob.name,
        "mesh": {"mesh": "mesh.txt", "entity_sets": "entity_sets.json", "io_type": f"Ascii{dim}D",
                 "check_duplicates": True, "isoparametric": False, "node_type": f"N{dim}D",
                 "cell_type": "ED2Q4" if dim == 2 else "ED3H8", "boundary_conditions": bcs},
        "particles": [{"generator": {"check_duplicates": True, "location": name, "io_type":
                                     f"Ascii{dim}D", "pset_id": k, "particle_type": f"P{dim}D",
                                     "material_id": mid, "type": "file"}}
                      for k, (name, mid) in enumerate(pfiles)],
        "materials": [dict(props, id=mid, type=mtype) for mid, mtype, props in prob.materials],
        "external_loading_conditions": (
            {"gravity": {"gravity": list(a.get("gravity", [0.0] * dim)),
                         "ramping_time": a["gravity_ramping_time"]}}
            if a.get("gravity_ramping_time", 0.0) > 0 else
            {"gravity": list(a.get("gravity", [0.0] * dim))}),
        "analysis": {"type": f"MPMExplicit{dim}D", "mpm_scheme": a.get("scheme", "usf"),
                     "velocity_update": a.get("velocity_update", "flip"),
                     "locate_particles": a.get("locate_particles", True), "dt": a["dt"],
                     "uuid": prob.name, "nsteps": nsteps,
                     "velocity_update_settings": {"blending_ratio": a.get("blending_ratio", 1.0)},
                     "damping": {"type": "Cundall", "damping_factor": a.get("damping_factor", 0.0)}},
        "post_processing": {"path": "results/", "output_steps": output_steps or nsteps},
    }
    if prob.initial_stress is not None:
        with open(os.path.join(outdir, "particles-stresses.txt"), "w") as f:
            f.write(f"{len(prob.initial_stress)}\n")
            for row in prob.initial_stress:
                f.write("\t".join(repr(float(v)) for v in row) + "\n")
        cfg["mesh"]["particles_stresses"] = {"type": "file", "location": "particles-stresses.txt"}
    with open(os.path.join(outdir, "mpm.json"), "w") as f:
        json.dump(cfg, f, indent=2)
    with open(os.path.join(outdir, "entity_sets.json"), "w") as f:
        json.dump({"node_sets": [], "particle_sets": psets}, f)
    return os.path.join(outdir, "mpm.json")
