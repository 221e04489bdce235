"""Host-side checks of the batched ensemble's packing (no GPU): the runs'
rectangles share no node, every particle lies inside its run's rectangle and
every run's wall constraints sit on its own nodes."""
import numpy as np

from mpm_b200 import ensemble as E


def _run_nodes(prob, info, runs):
    dx = prob.dx
    nx1 = info["shape"][0] + 1
    out = []
    for run, (ox, oy) in zip(runs, info["origins"]):
        i0, j0 = int(round(ox / dx)), int(round(oy / dx))
        nx, ny = run.cells
        ii, jj = np.meshgrid(np.arange(i0, i0 + nx + 1), np.arange(j0, j0 + ny + 1))
        out.append(set((ii + nx1 * jj).ravel().tolist()))
    return out


def test_runs_share_no_node_and_stay_in_their_rectangles():
    runs = E.random_runs(24, n_min=200, n_max=3000, seed=7)
    prob, info = E.ensemble_problem(runs)
    nodes = _run_nodes(prob, info, runs)
    for a in range(len(runs)):
        for b in range(a + 1, len(runs)):
            assert not (nodes[a] & nodes[b]), (a, b)
    for run, (lo, hi), (ox, oy) in zip(runs, info["ranges"], info["origins"]):
        pts, mid = prob.particles[runs.index(run)]
        assert len(pts) == hi - lo == run.nparticles
        nx, ny = run.cells
        assert np.all(pts[:, 0] > ox) and np.all(pts[:, 0] < ox + nx * prob.dx)
        assert np.all(pts[:, 1] > oy) and np.all(pts[:, 1] < oy + ny * prob.dx)
    vnid = prob.velocity_constraints[0]
    all_nodes = set().union(*nodes)
    assert set(vnid.tolist()) <= all_nodes
    # each run: its material slot, its own walls on all four sides
    assert [m[0] for m in prob.materials] == list(range(len(runs)))
    for r, ns in enumerate(nodes):
        assert len(ns & set(vnid.tolist())) == 2 * (runs[r].cells[0] + 1) + 2 * (runs[r].cells[1] + 1) - 4


def test_random_runs_follow_the_requested_distribution():
    runs = E.random_runs(512)
    n = np.array([r.nparticles for r in runs])
    assert 1800 <= n.min() and n.max() <= 41000
    phi = np.array([r.phi for r in runs])
    c = np.array([r.cohesion for r in runs])
    assert 20 <= phi.min() and phi.max() <= 40 and 0 <= c.min() and c.max() <= 5000
    # seeded: the same ensemble every time
    again = E.random_runs(512)
    assert [r.nparticles for r in again] == n.tolist()
