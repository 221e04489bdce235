"""The host driver on input laid out as the reference's own test fixtures write
it (tests/io/write_mesh_particles.cc: write_json :6-118, write_entity_set
:1584-1623, write_mesh_2d :1663-1737, write_particles_2d :1740-1791,
write_mesh_3d :1859-1959, write_particles_3d :1962-2036).

The fixture's JSON is reproduced with nlohmann's structure: objects where the
C++ initialiser lists make objects (so ``boundary_conditions.velocity_constraints``
is an object, which the reference's reader iterates, fails on inside its try
block and applies nothing, mpm_base.tcc:1128-1170), keys sorted as
``Json::dump`` writes them.  Its tractions, nodal forces and rotation forces
are outside the explicit path built here: ``--parse-only`` lists them and a
run refuses them.  With those three entries removed the driver's run equals
the Python API's run of the same analysis bit for bit, and the oracle's
within 1e-10 (material set 2 moves every particle to material 1).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from mpm_b200 import build as B
from mpm_b200 import pod

MESH = {
    2: ([(0., 0.), (0.5, 0.), (0.5, 0.5), (0., 0.5), (1.0, 0.), (1.0, 0.5)],
        [(0, 1, 2, 3), (1, 4, 5, 2)], [(0, 1, 0), (1, 1, 0), (4, 1, 0)]),
    3: ([(0., 0., 0.), (0.5, 0., 0.), (0.5, 0.5, 0.), (0., 0.5, 0.), (0., 0., 0.5), (0.5, 0., 0.5),
         (0.5, 0.5, 0.5), (0., 0.5, 0.5), (1.0, 0., 0.), (1.0, 0.5, 0.), (1.0, 0., 0.5),
         (1.0, 0.5, 0.5)],
        [(0, 1, 2, 3, 4, 5, 6, 7), (1, 8, 9, 2, 5, 10, 11, 6)],
        [(n, 2, 0) for n in (0, 1, 2, 3, 8, 9)]),
}
PARTICLES = {
    2: [(0.125, 0.125), (0.375, 0.125), (0.375, 0.375), (0.125, 0.375),
        (0.625, 0.125), (0.875, 0.125), (0.875, 0.375), (0.625, 0.375)],
    3: [(0.125, 0.125, 0.125), (0.375, 0.125, 0.125), (0.375, 0.375, 0.125), (0.125, 0.375, 0.125),
        (0.125, 0.125, 0.375), (0.375, 0.125, 0.375), (0.375, 0.375, 0.375), (0.125, 0.375, 0.375),
        (0.625, 0.125, 0.125), (0.875, 0.125, 0.125), (0.875, 0.375, 0.125), (0.625, 0.375, 0.125),
        (0.675, 0.125, 0.375), (0.875, 0.125, 0.375), (0.875, 0.375, 0.375), (0.675, 0.375, 0.375)],
}
MATERIALS = [(0, 1000., 1.0E+8, 0.495), (1, 2300., 1.5E+6, 0.25)]


def _cxx(v):
    """A double as std::ostream << writes it (6 significant digits)."""
    return f"{v:g}"


def write_fixture(d, dim, scheme, name="mpm-explicit"):
    """Files of write_json(dim, false, "MPMExplicit<dim>D", scheme, name),
    write_entity_set(), write_mesh_<dim>d() and write_particles_<dim>d()."""
    dimension = f"{dim}d"
    io_type = f"Ascii{dim}D"
    material = f"LinearElastic{dim}D"
    gravity = [0., -9.81] if dim == 2 else [0., 0., -9.81]
    js = {
        "title": "Example JSON Input for MPM",
        "mesh": {"mesh": f"mesh-{dimension}.txt", "entity_sets": "entity_sets_0.json",
                 "io_type": io_type, "check_duplicates": True, "isoparametric": False,
                 "node_type": f"N{dim}D",
                 "boundary_conditions": {"velocity_constraints": {"file": "velocity-constraints.txt"}},
                 "cell_type": "ED2Q4" if dim == 2 else "ED3H8"},
        "particles": [{"generator": {"type": "file", "material_id": 0, "pset_id": 0,
                                     "io_type": io_type, "particle_type": f"P{dim}D",
                                     "check_duplicates": True,
                                     "location": f"particles-{dimension}.txt"}}],
        "materials": [{"id": i, "type": material, "density": r, "youngs_modulus": E,
                       "poisson_ratio": nu} for i, r, E, nu in MATERIALS],
        "material_sets": [{"material_id": 1, "phase_id": 0, "pset_id": 2}],
        "external_loading_conditions": {
            "gravity": gravity,
            "particle_surface_traction": [{"math_function_id": 0, "pset_id": -1, "dir": 1,
                                           "traction": 10.5}],
            "concentrated_nodal_forces": [{"math_function_id": 0, "nset_id": -1, "dir": 1,
                                           "force": 10.5}],
            "rotation_forces": {"origin": [0.0] * dim, "omega": 10.0, "clockwise": False}},
        "math_functions": [{"id": 0, "type": "Linear", "xvalues": [0.0, 0.5, 1.0],
                            "fxvalues": [0.0, 1.0, 1.0]}],
        "analysis": {"type": f"MPMExplicit{dim}D", "mpm_scheme": scheme, "locate_particles": True,
                     "velocity_update": True, "dt": 0.001, "uuid": f"{name}-{dimension}",
                     "nsteps": 10,
                     "resume": {"resume": False, "uuid": f"{name}-{dimension}", "step": 5},
                     "damping": {"type": "Cundall", "damping_factor": 0.02},
                     "newmark": {"beta": 0.25, "gamma": 0.5}},
        "post_processing": {"path": "results/", "vtk": ["stresses", "strains", "velocities"],
                            "vtk_statevars": [{"phase_id": 0, "statevars": ["pdstrain"]}],
                            "output_steps": 5},
    }
    fname = f"{name}-{dimension}.json"
    with open(os.path.join(d, fname), "w") as f:
        f.write(json.dumps(js, indent=2, sort_keys=True))
    sets = {2: {"particle_sets": [{"id": 2, "set": list(range(16))}],
                "node_sets": [{"id": 1, "set": [4, 5]}]}}
    with open(os.path.join(d, "entity_sets_0.json"), "w") as f:
        f.write(json.dumps(sets[2], indent=2, sort_keys=True))
    coords, cells, vcons = MESH[dim]
    with open(os.path.join(d, f"mesh-{dimension}.txt"), "w") as f:
        f.write("! elementShape hexahedron\n! elementNumPoints 8\n")
        f.write(f"{len(coords)}\t{len(cells)}\n")
        for c in coords:
            f.write("".join(_cxx(v) + "\t" for v in c) + "\n")
        for c in cells:
            f.write("".join(f"{n}\t" for n in c) + "\n")
    with open(os.path.join(d, "velocity-constraints.txt"), "w") as f:
        for n, di, v in vcons:
            f.write(f"{n}\t{di}\t{v}\n")
    pts = PARTICLES[dim]
    with open(os.path.join(d, f"particles-{dimension}.txt"), "w") as f:
        f.write(f"{len(pts)}\n")
        for p in pts:
            f.write("".join(_cxx(v) + "\t" for v in p) + "\n")
    return fname, js


def _driver(d, fname, *args):
    return subprocess.run([B.RUNNER, "-f", d, "-i", fname, *args], capture_output=True,
                          text=True, timeout=600)


def _strip_unsupported(d, fname, js):
    el = js["external_loading_conditions"]
    for k in ("particle_surface_traction", "concentrated_nodal_forces", "rotation_forces"):
        del el[k]
    with open(os.path.join(d, fname), "w") as f:
        f.write(json.dumps(js, indent=2, sort_keys=True))


@pytest.mark.parametrize("dim", [2, 3])
def test_reference_fixture_parses_and_lists_what_is_outside_the_path(tmp_path, dim):
    d = str(tmp_path)
    fname, js = write_fixture(d, dim, "usf")
    r = _driver(d, fname, "--parse-only")
    assert r.returncode == 0, r.stderr
    out = r.stdout
    summary = out.splitlines()[0] + " "
    nn, nc = len(MESH[dim][0]), len(MESH[dim][1])
    for key, val in (("dim", dim), ("nodes", nn), ("cells", nc), ("particles", len(PARTICLES[dim])),
                     ("materials", 2), ("nsteps", 10), ("velocity_constraints", 0),
                     ("material_sets", 1)):
        assert f"{key} {val} " in summary, (key, out)
    assert "scheme usf" in out and "velocity_update pic" in out
    for k in ("particle_surface_traction", "concentrated_nodal_forces", "rotation_forces"):
        assert f"unsupported external_loading_conditions.{k}" in out
    assert "velocity_constraints is not a list" in r.stderr
    r = _driver(d, fname)
    assert r.returncode != 0 and "unsupported input" in r.stderr
    _strip_unsupported(d, fname, js)
    r = _driver(d, fname, "--parse-only")
    assert r.returncode == 0 and "unsupported" not in r.stdout


def _api_run(dim, scheme):
    from mpm_b200.solver import Solver
    coords, cells, _ = MESH[dim]
    s = Solver(dim, scheme=scheme, velocity_update="pic", dt=0.001,
               gravity=(0., -9.81) if dim == 2 else (0., 0., -9.81), damping_factor=0.02)
    s.set_mesh(np.array(coords), np.array(cells))
    for i, r, E, nu in MATERIALS:
        s.add_material(i, f"LinearElastic{dim}D", {"density": r, "youngs_modulus": E,
                                                   "poisson_ratio": nu})
    pts = np.array([[float(_cxx(v)) for v in p] for p in PARTICLES[dim]])
    s.add_particles(pts, 0)
    s.assign_particle_materials(np.arange(16), 1)
    s.initialise()
    return s, pts


def _oracle_run(dim, scheme, pts):
    from oracle.oracle import Oracle
    coords, cells, _ = MESH[dim]
    o = Oracle(dim, scheme=scheme, velocity_update="pic", dt=0.001,
               gravity=(0., -9.81) if dim == 2 else (0., 0., -9.81), damping_factor=0.02)
    o.set_mesh(np.array(coords), np.array(cells))
    for i, r, E, nu in MATERIALS:
        o.add_material(i, f"LinearElastic{dim}D", {"density": r, "youngs_modulus": E,
                                                   "poisson_ratio": nu})
    o.add_particles(pts, 1)  # material set 2 holds every particle
    o.initialise()
    return o


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("scheme", ["usf", "usl"])
def test_reference_fixture_runs_as_the_api_and_the_oracle(tmp_path, dim, scheme):
    from tests.parity import assert_parity
    d = str(tmp_path)
    fname, js = write_fixture(d, dim, scheme)
    _strip_unsupported(d, fname, js)
    r = _driver(d, fname)
    assert r.returncode == 0, r.stderr
    from mpm_b200 import h5
    # post_processing.path + analysis.uuid, the step padded to the digits of nsteps
    rec = h5.read_table(os.path.join(d, "results", js["analysis"]["uuid"], "particles10.h5"))
    s, pts = _api_run(dim, scheme)
    s.step(10)
    ref = s.write_pod()
    assert len(rec) == len(ref) == len(PARTICLES[dim])
    for name in pod.NAMES:
        assert np.array_equal(rec[name].astype(ref[name].dtype), ref[name]), name
    assert np.all(rec["material_id"] == 1)
    o = _oracle_run(dim, scheme, pts)
    o.step(10)
    assert_parity(s.read(), o.get(), label=f"fixture {dim}D {scheme}")
