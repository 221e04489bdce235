"""Slab decomposition of one run across ranks (one GPU each), along x.

The reference decomposes the mesh with MPI (KaHIP graph partitions,
graph.tcc:120-136), sums the nodal mass, momentum and forces of nodes shared
between ranks after P2G (mesh.tcc:187-205, MPI_Allreduce at :198) and moves
particles that leave a rank's cells to the rank that owns them
(mesh.tcc:737-1040).  Here the tensor-product grid is cut into slabs of whole
x-columns of cells, sized by prefix sums of the particles per column:

* rank r owns the cell columns [lo, hi) and keeps one ghost column on each
  side ([lo - 1, hi + 1) clipped to the grid), with the global mesh's own node
  coordinates, so its solver's local cells and nodes are the global ones;
* after P2G it sends the cell-slot partial sums (and particle counts) of its
  first owned column to the left neighbour and of its last to the right one,
  and writes what it receives into its ghost columns: the node update then
  gathers, for every node of its owned cells, the same partial sums in the same
  order (ascending cell id) as a single-GPU run does;
* after the step, particles whose new cell lies in a ghost column go to the
  neighbour that owns it;
* every ``reslab_every`` steps the cuts are recomputed from the particle
  counts and the particles redistributed (the counterpart of the reference's
  repartitioning).

While no particle has changed rank the slab run's sums are bitwise those of the
single-GPU run; a migrated particle is appended to its new rank's particle
array, so it is summed in a different position within its cell and the results
then agree to rounding.

The transport of halos and migrants is pluggable: ``DistComm`` over
``torch.distributed`` (NCCL with device buffers, or gloo with host buffers),
or ``run_in_process`` for several slabs in one process (on one GPU).
Only the USL FLIP/PIC step on tensor-product grids is decomposed.
"""
import numpy as np

from .problems import Problem, build_solver


def partition(column_counts, nranks, min_columns=2):
    """x-cuts [c_0 = 0, c_1, ..., c_n = nx] giving each rank about the same
    number of particles (prefix sums of the per-column counts), each slab at
    least ``min_columns`` wide."""
    counts = np.asarray(column_counts, dtype=np.float64)
    nx = len(counts)
    if nranks * min_columns > nx:
        raise ValueError(f"{nranks} slabs of at least {min_columns} columns do not fit {nx} columns")
    csum = np.concatenate([[0.0], np.cumsum(counts)])
    total = csum[-1]
    cuts = [0]
    for r in range(1, nranks):
        target = total * r / nranks
        c = int(np.searchsorted(csum, target, side="left"))
        lo = cuts[-1] + min_columns
        hi = nx - (nranks - r) * min_columns
        cuts.append(int(min(max(c, lo), hi)))
    cuts.append(nx)
    return cuts


class SlabGeometry:
    """Global grid, cuts, and one rank's owned and local (with ghosts) columns."""

    def __init__(self, prob, cuts, rank):
        if not isinstance(prob, Problem) or prob.shape is None:
            raise ValueError("a structured problem is decomposed")
        self.dim = prob.dim
        self.shape = tuple(prob.shape)
        self.cuts = list(cuts)
        self.rank = rank
        self.nranks = len(cuts) - 1
        nx = self.shape[0]
        self.lo, self.hi = cuts[rank], cuts[rank + 1]
        self.glo, self.ghi = max(self.lo - 1, 0), min(self.hi + 1, nx)
        self.left = rank - 1 if self.lo > 0 else None
        self.right = rank + 1 if self.hi < nx else None

    @property
    def local_shape(self):
        return (self.ghi - self.glo,) + self.shape[1:]

    # global <-> local indices
    def cell_x(self, cells):
        return np.asarray(cells) % self.shape[0]

    def to_local_cells(self, cells):
        cells = np.asarray(cells, dtype=np.int64)
        nx = self.shape[0]
        i = cells % nx
        rest = cells // nx
        return (i - self.glo) + (self.ghi - self.glo) * rest

    def to_global_cells(self, cells):
        cells = np.asarray(cells, dtype=np.int64)
        nl = self.ghi - self.glo
        i = cells % nl
        rest = cells // nl
        out = (i + self.glo) + self.shape[0] * rest
        return np.where(cells < 0, -1, out)

    def local_nodes(self):
        """Global ids of the local nodes, in local id order (x fastest)."""
        nxn = self.shape[0] + 1
        ids = np.arange(self.glo, self.ghi + 1)
        if self.dim == 2:
            j = np.arange(self.shape[1] + 1)
            J, I = np.meshgrid(j, ids, indexing="ij")
            return (I + nxn * J).ravel()
        nyn = self.shape[1] + 1
        k = np.arange(self.shape[2] + 1)
        j = np.arange(nyn)
        K, J, I = np.meshgrid(k, j, ids, indexing="ij")
        return (I + nxn * (J + nyn * K)).ravel()

    # local column indices of the halo layers
    @property
    def first_owned(self):
        return self.lo - self.glo

    @property
    def last_owned(self):
        return self.hi - 1 - self.glo

    @property
    def left_ghost(self):
        return 0

    @property
    def right_ghost(self):
        return self.ghi - 1 - self.glo


def local_problem(prob, geom):
    """The rank's problem without particles: the local grid (global node
    coordinates), materials and the nodal constraints of its nodes."""
    from .problems import structured_mesh
    g_nodes = geom.local_nodes()
    coords = np.ascontiguousarray(prob.coords[g_nodes])
    _, cells = structured_mesh(geom.dim, geom.local_shape, prob.dx)
    lookup = -np.ones(len(prob.coords), dtype=np.int64)
    lookup[g_nodes] = np.arange(len(g_nodes))

    def restrict(cons):
        if cons is None:
            return None
        nid = np.asarray(cons[0])
        keep = lookup[nid] >= 0
        return tuple([lookup[nid[keep]]] + [np.asarray(c)[keep] for c in cons[1:]])

    if prob.particle_velocity_constraints:
        raise ValueError("particle velocity constraints are not decomposed")
    if prob.nodal_euler_angles is not None:
        raise ValueError("rotated boundaries are not decomposed")
    return Problem(dim=prob.dim, shape=geom.local_shape, dx=prob.dx, coords=coords, cells=cells,
                   materials=prob.materials, particles=[],
                   velocity_constraints=restrict(prob.velocity_constraints),
                   friction_constraints=restrict(prob.friction_constraints),
                   analysis=dict(prob.analysis), name=f"{prob.name}-slab{geom.rank}")


class SlabRank:
    """One rank's part of a slab run: its geometry, solver and the global ids
    of its particles (rows of the solver's state, in order)."""

    def __init__(self, prob, cuts, rank, state, gid, step=0, make_solver=None, **solver_kw):
        self.prob = prob
        self.geom = SlabGeometry(prob, cuts, rank)
        self.solver_kw = solver_kw
        local = local_problem(prob, self.geom)
        self.solver = (make_solver(local) if make_solver else
                       build_solver(local, with_particles=False, **solver_kw))
        st = dict(state)
        st["cell"] = self.geom.to_local_cells(state["cell"])
        self.gid = np.asarray(gid, dtype=np.int64)
        self.solver.load(st)  # a slab may hold no particle
        self.solver.set_current_step(step)
        self.halo_bytes = self.solver.halo_bytes()

    # ---- one step in phases (the caller moves the halos and the migrants)
    def begin(self):
        self.solver.step_begin()

    def halo_out(self, alloc):
        """{neighbour rank: packed layer} for the neighbours; ``alloc(nbytes)``
        returns a device buffer with a ``data_ptr()``."""
        out = {}
        if self.geom.left is not None:
            b = alloc(self.halo_bytes)
            self.solver.halo_pack(self.geom.first_owned, b.data_ptr())
            out[self.geom.left] = b
        if self.geom.right is not None:
            b = alloc(self.halo_bytes)
            self.solver.halo_pack(self.geom.last_owned, b.data_ptr())
            out[self.geom.right] = b
        return out

    def halo_in(self, bufs):
        for peer, b in bufs.items():
            layer = self.geom.left_ghost if peer == self.geom.left else self.geom.right_ghost
            self.solver.halo_unpack(layer, b.data_ptr())

    def end(self):
        self.solver.step_end()

    def migrants_out(self):
        """Remove the particles now in a ghost column; {neighbour: (rows, gids)}."""
        g = self.geom
        below, above = self.solver.layer_count(g.first_owned, g.last_owned + 1)
        if below == 0 and above == 0:
            return {}
        st = self.solver.read()
        xcol = st["cell"] % (g.ghi - g.glo)
        go_left = st["cell"] >= 0
        go_left &= xcol < g.first_owned
        go_right = (st["cell"] >= 0) & (xcol > g.last_owned)
        stay = ~(go_left | go_right)
        out = {}
        for peer, sel in ((g.left, go_left), (g.right, go_right)):
            if peer is not None and np.any(sel):
                rows = {k: np.asarray(v)[sel] for k, v in st.items()}
                rows["cell"] = g.to_global_cells(rows["cell"])
                out[peer] = (rows, self.gid[sel])
        self._pending = ({k: np.asarray(v)[stay] for k, v in st.items()}, self.gid[stay])
        return out

    def migrants_in(self, received):
        """Append the particles received ({peer: (rows, gids)}) after the ones
        that stayed."""
        if not hasattr(self, "_pending") and not received:
            return
        if hasattr(self, "_pending"):
            st, gid = self._pending
            del self._pending
        else:
            st, gid = self.solver.read(), self.gid
        parts, gids = [st], [gid]
        for peer in sorted(received):
            rows, g = received[peer]
            rows = dict(rows)
            rows["cell"] = self.geom.to_local_cells(rows["cell"])
            parts.append(rows)
            gids.append(g)
        merged = {k: np.concatenate([p[k] for p in parts]) for k in st}
        self.gid = np.concatenate(gids)
        step = self.solver.current_step
        self.solver.load(merged)
        self.solver.set_current_step(step)

    def state(self):
        """(global rows of this rank's particles, their global ids)."""
        st = self.solver.read()
        st["cell"] = self.geom.to_global_cells(st["cell"])
        return st, self.gid

    def column_counts(self):
        st = self.solver.read()
        counts = np.zeros(self.geom.shape[0], dtype=np.int64)
        gc = self.geom.to_global_cells(st["cell"])
        gc = gc[gc >= 0]
        np.add.at(counts, gc % self.geom.shape[0], 1)
        return counts


def split_state(prob, state, cuts):
    """The particles of a global state (rows in global id order) by owning rank."""
    nx = prob.shape[0]
    xcol = np.asarray(state["cell"]) % nx
    out = []
    for r in range(len(cuts) - 1):
        sel = (np.asarray(state["cell"]) >= 0) & (xcol >= cuts[r]) & (xcol < cuts[r + 1])
        out.append(({k: np.asarray(v)[sel] for k, v in state.items()}, np.nonzero(sel)[0]))
    return out


def merge_states(parts, n):
    """Global state (rows in global id order) from every rank's (rows, gids)."""
    first = parts[0][0]
    out = {k: np.zeros((n,) + np.asarray(v).shape[1:], dtype=np.asarray(v).dtype)
           for k, v in first.items()}
    out["cell"][:] = -1
    for rows, gid in parts:
        for k in out:
            out[k][gid] = rows[k]
    return out


# ------------------------------------------------------------------ drivers
def run_in_process(prob, nranks, nsteps, reslab_every=0, state=None, **solver_kw):
    """Every slab in this process (on one device): the halos and migrants move
    by device copies and host arrays.  ``state``: the initial global particle
    state (default: the problem's initialised particles).  Returns the merged
    global state and the last cuts."""
    import torch
    dev = torch.device("cuda", solver_kw.get("device", 0))
    if state is None:
        full = build_solver(prob, **solver_kw)
        state = full.read()
        full.close()
    n = len(state["x"])
    cuts = partition(_column_counts(prob, state), nranks)
    ranks = [SlabRank(prob, cuts, r, *split_state(prob, state, cuts)[r], **solver_kw)
             for r in range(nranks)]
    alloc = lambda nb: torch.empty(nb, dtype=torch.uint8, device=dev)  # noqa: E731
    for step in range(nsteps):
        for rk in ranks:
            rk.begin()
        outs = [rk.halo_out(alloc) for rk in ranks]
        for r, rk in enumerate(ranks):
            rk.halo_in({src: o[r] for src, o in enumerate(outs) if r in o})
        for rk in ranks:
            rk.end()
        mig = [rk.migrants_out() for rk in ranks]
        for r, rk in enumerate(ranks):
            rk.migrants_in({src: m[r] for src, m in enumerate(mig) if r in m})
        if reslab_every and (step + 1) % reslab_every == 0 and step + 1 < nsteps:
            ranks, cuts = _reslab(prob, ranks, n, solver_kw)
    merged = merge_states([rk.state() for rk in ranks], n)
    return merged, cuts


def _column_counts(prob, state):
    counts = np.zeros(prob.shape[0], dtype=np.int64)
    c = np.asarray(state["cell"])
    c = c[c >= 0]
    np.add.at(counts, c % prob.shape[0], 1)
    return counts


def _reslab(prob, ranks, n, solver_kw):
    state = merge_states([rk.state() for rk in ranks], n)
    step = ranks[0].solver.current_step
    for rk in ranks:
        rk.solver.close()
    cuts = partition(_column_counts(prob, state), len(ranks))
    parts = split_state(prob, state, cuts)
    return [SlabRank(prob, cuts, r, parts[r][0], parts[r][1], step=step, **solver_kw)
            for r in range(len(ranks))], cuts


class DistComm:
    """Halo and migrant transport over torch.distributed between neighbour
    ranks: device buffers with NCCL, host copies with gloo."""

    def __init__(self, device=None):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        self.nccl = dist.get_backend() == "nccl"
        self.device = device

    def exchange_buffers(self, out, peers, nbytes, alloc):
        """Send out[peer] to each peer, receive one buffer from each peer."""
        import torch
        reqs, recv = [], {}
        for p in peers:
            recv[p] = alloc(nbytes) if self.nccl else torch.empty(nbytes, dtype=torch.uint8)
            src = out[p] if self.nccl else out[p].cpu()
            reqs.append(self.dist.isend(src, p))
            reqs.append(self.dist.irecv(recv[p], p))
        for q in reqs:
            q.wait()
        if not self.nccl:
            recv = {p: b.to(out[p].device) for p, b in recv.items()}
        return recv

    def exchange_objects(self, out, peers):
        """Pickled objects to and from each peer (counts first, then bytes)."""
        import pickle

        import torch
        payload = {p: pickle.dumps(out.get(p)) for p in peers}
        dev = torch.device("cuda", self.device) if self.nccl else torch.device("cpu")
        sizes = {}
        reqs = []
        for p in peers:
            sizes[p] = torch.zeros(1, dtype=torch.int64, device=dev)
            reqs.append(self.dist.isend(torch.tensor([len(payload[p])], dtype=torch.int64,
                                                     device=dev), p))
            reqs.append(self.dist.irecv(sizes[p], p))
        for q in reqs:
            q.wait()
        reqs, bufs = [], {}
        for p in peers:
            data = torch.frombuffer(bytearray(payload[p]), dtype=torch.uint8).to(dev)
            bufs[p] = torch.empty(int(sizes[p].item()), dtype=torch.uint8, device=dev)
            reqs.append(self.dist.isend(data, p))
            reqs.append(self.dist.irecv(bufs[p], p))
        for q in reqs:
            q.wait()
        return {p: pickle.loads(bufs[p].cpu().numpy().tobytes()) for p in peers}


def run_distributed(prob, nsteps, comm, state=None, make_solver=None, alloc=None, **solver_kw):
    """This rank's slab of a run over torch.distributed (every rank calls it
    with the same problem); returns (this rank's rows, their global ids).
    ``state``: the initial global particle state (default: every rank
    initialises the problem's particles itself); ``alloc(nbytes)``: a halo
    buffer (default: a device buffer)."""
    import torch
    world, rank = comm.world, comm.rank
    if state is None:
        full = build_solver(prob, **solver_kw)  # every rank initialises the same particles
        state = full.read()
        full.close()
    cuts = partition(_column_counts(prob, state), world)
    rows, gid = split_state(prob, state, cuts)[rank]
    rk = SlabRank(prob, cuts, rank, rows, gid, make_solver=make_solver, **solver_kw)
    if alloc is None:
        dev = torch.device("cuda", solver_kw.get("device", 0))
        alloc = lambda nb: torch.empty(nb, dtype=torch.uint8, device=dev)  # noqa: E731
    peers = [p for p in (rk.geom.left, rk.geom.right) if p is not None]
    for _ in range(nsteps):
        rk.begin()
        out = rk.halo_out(alloc)
        rk.halo_in(comm.exchange_buffers(out, peers, rk.halo_bytes, alloc))
        rk.end()
        mig = rk.migrants_out()
        rk.migrants_in({p: m for p, m in comm.exchange_objects(mig, peers).items() if m})
    return rk.state()
