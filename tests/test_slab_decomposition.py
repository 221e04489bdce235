"""Slab decomposition along x (the reference's MPI halo sum and particle
migration, mesh.tcc:187-205, 737-1040; repartitioning, graph.tcc:120-136).

CPU: the prefix-sum partition; the slab geometry (global and local cells and
nodes, the local problem's coordinates and constraints); and two ranks over
torch.distributed with gloo driving the slab orchestration (halo exchange
between P2G and the node update, migration of particles entering a ghost
column) with a CPU stand-in solver, against one undecomposed run.
GPU: two and three slabs in one process on one GPU, against one solver:
bitwise until the first particle changes slab, within the FP64 parity
tolerance after migrations and a re-slab.
"""
import os
import pickle
import socket

import numpy as np
import pytest

from mpm_b200 import problems as P
from mpm_b200 import slab as S
from tests.slab_fake import FakeSolver, initial_state


def test_partition_balances_particles():
    counts = np.zeros(40, dtype=np.int64)
    counts[:10] = 100  # a column on the left third of the grid
    cuts = S.partition(counts, 4)
    assert cuts[0] == 0 and cuts[-1] == 40 and cuts == sorted(cuts)
    per = [counts[a:b].sum() for a, b in zip(cuts[:-1], cuts[1:])]
    assert max(per[:-1]) - min(per[:-1]) <= 100, per
    assert all(b - a >= 2 for a, b in zip(cuts[:-1], cuts[1:]))
    with pytest.raises(ValueError):
        S.partition(counts, 21)


@pytest.mark.parametrize("dim", [2, 3])
def test_geometry_maps_cells_nodes_and_constraints(dim):
    prob = (P.column_2d(shape=(20, 8), block=(6, 6)) if dim == 2 else
            P.column_3d(shape=(12, 4, 5), block=(6, 4, 4), material="LinearElastic"))
    cuts = [0, 5, prob.shape[0]]
    for r in range(2):
        g = S.SlabGeometry(prob, cuts, r)
        local = S.local_problem(prob, g)
        nodes = g.local_nodes()
        assert np.array_equal(local.coords, prob.coords[nodes])
        gcells = np.arange(prob.ncells)
        mine = (gcells % prob.shape[0] >= g.glo) & (gcells % prob.shape[0] < g.ghi)
        lc = g.to_local_cells(gcells[mine])
        assert np.array_equal(np.sort(lc), np.arange(local.ncells))
        assert np.array_equal(g.to_global_cells(lc), gcells[mine])
        # each local cell's nodes are the global cell's nodes
        assert np.array_equal(nodes[local.cells[lc]], prob.cells[gcells[mine]])
        # constraints: exactly the global ones on local nodes
        vn, vd, _ = prob.velocity_constraints
        on = np.isin(vn, nodes)
        ln, ld, _ = local.velocity_constraints
        assert sorted(zip(nodes[ln].tolist(), ld.tolist())) == sorted(zip(vn[on].tolist(),
                                                                           vd[on].tolist()))


def _fake_problem():
    return P.column_2d(shape=(24, 4), block=(8, 3), dx=0.01)


def _single_domain(prob, state, nsteps):
    s = FakeSolver(prob)
    s.load(state)
    for _ in range(nsteps):
        s.step_begin()
        s.step_end()
    return s.read()


def _rank_main(rank, world, port, nsteps, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob = _fake_problem()
        comm = S.DistComm()
        rows, gid = S.run_distributed(prob, nsteps, comm, state=initial_state(prob),
                                      make_solver=lambda local: FakeSolver(local),
                                      alloc=lambda nb: torch.empty(nb, dtype=torch.uint8))
        with open(out % rank, "wb") as f:
            pickle.dump((rows, gid), f)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_match_one_domain(tmp_path):
    import torch.multiprocessing as mp
    nsteps = 30
    out = str(tmp_path / "rank%d.pkl")
    mp.spawn(_rank_main, args=(2, _free_port(), nsteps, out), nprocs=2, join=True)
    parts = [pickle.load(open(out % r, "rb")) for r in range(2)]
    prob = _fake_problem()
    state = initial_state(prob)
    ref = _single_domain(prob, state, nsteps)
    merged = S.merge_states(parts, len(state["x"]))
    assert sorted(np.concatenate([g for _, g in parts]).tolist()) == list(range(len(state["x"])))
    # particles changed rank during the run: the gids each rank ends with are
    # not the ones it started with
    cuts = S.partition(S._column_counts(prob, state), 2)
    start = S.split_state(prob, state, cuts)
    assert set(parts[0][1].tolist()) != set(start[0][1].tolist())
    assert np.array_equal(merged["x"], ref["x"])
    assert np.array_equal(merged["cell"], ref["cell"])


# ---------------------------------------------------------------- GPU
def _le_column(**kw):
    base = dict(shape=(24, 6, 8), block=(16, 6, 6), material="LinearElastic", E=1e6,
                scheme="usl", dt=1e-5, geostatic=False)
    base.update(kw)
    return P.column_3d(**base)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_slabs_on_one_gpu_are_bitwise_before_any_migration(precision):
    prob = _le_column()
    ref = P.build_solver(prob, precision=precision)
    ref.step(10)
    R = ref.read()
    merged, cuts = S.run_in_process(prob, 2, 10, precision=precision)
    assert 0 < cuts[1] < prob.shape[0]
    for k in ("x", "u", "v", "stress", "strain", "F", "volume", "cell"):
        assert np.array_equal(merged[k], R[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("nranks,reslab", [(2, 0), (3, 40)])
def test_slabs_with_migration_match_one_gpu(nranks, reslab):
    """A block sliding along the floor, away from the walls, whose particles
    cross the slab edges (and, with a re-slab, the recomputed cuts): within
    the FP64 parity tolerance."""
    import dataclasses
    from tests.parity import FP64_RTOL, assert_parity
    prob = P.column_2d(shape=(40, 16), block=(10, 14), E=1e6, scheme="usl", dt=1e-4)
    pts, mid = prob.particles[0]
    prob = dataclasses.replace(prob, particles=[(pts + np.array([10 * prob.dx, 0.0]), mid)])
    steps = 120
    ref = P.build_solver(prob)
    st0 = ref.read()
    st0["v"][:, 0] = 1.5  # the block slides right through the slab edges
    ref.load(st0)
    ref.step(steps)
    R = ref.read()
    merged, cuts = S.run_in_process(prob, nranks, steps, reslab_every=reslab, state=st0)
    xcol0 = st0["cell"] % prob.shape[0]
    xcol1 = R["cell"] % prob.shape[0]
    moved = np.count_nonzero(np.searchsorted(cuts, xcol0, side="right") !=
                             np.searchsorted(cuts, xcol1, side="right"))
    assert moved > 0, "no particle crossed a slab edge"
    assert_parity(merged, R, rtol=FP64_RTOL, label=f"{nranks} slabs")
