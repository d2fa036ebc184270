"""Z-slab decomposition of the LBM step over ranks, one GPU each, with one
halo exchange per step (no counterpart in the reference, which runs on one
node with OpenMP).

The lattice (periodic in z) is cut into equal slabs of whole 4x4x4 tile
layers.  Each rank holds its slab with one tile layer of halo on either side
(HALO planes).  A step of the interior pulls across a z face only the
populations of the 5 directions with e_z pointing into the slab, from the
halo plane next to the face; so after every step each rank sends the
e_z = -1 populations of its first interior plane to the rank below (its top
halo plane) and the e_z = +1 populations of its last interior plane to the
rank above (its bottom halo plane), and the interior evolves exactly as in
the unsplit lattice.  The halo planes' other populations and the rest of the
halo layer are never read by the interior.  SlabLBM is the LBM step alone;
SlabCoupled (below) splits the whole coupled step.
"""
import numpy as np

from . import Context, default_params

HALO = 4  # one tile layer


def slab_bounds(nz, world, rank):
    """Interior z planes [z0, z1) of `rank`: nz splits into `world` equal
    slabs of whole tile layers."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    if nz % (4 * world):
        raise ValueError(f"nz = {nz} does not split into {world} slabs of whole 4-plane tile layers")
    n = nz // world
    return rank * n, (rank + 1) * n


def slab_lattice(b_index, world, rank, halo=HALO):
    """The rank's lattice: its interior planes with `halo` planes on either
    side, taken from the z-periodic lattice b_index [nx][ny][nz]."""
    nz = b_index.shape[2]
    z0, z1 = slab_bounds(nz, world, rank)
    return np.ascontiguousarray(b_index[:, :, np.arange(z0 - halo, z1 + halo) % nz])


def plane_counts(b_index):
    """Listed points of every global z plane."""
    return (b_index >= 0).sum(axis=(0, 1))


def _staged(t, group):
    """Whether a device tensor goes through host memory for this group's
    backend (gloo moves host tensors)."""
    import torch.distributed as dist
    return t.is_cuda and dist.get_backend(group) == "gloo"


def exchange_dist(send_dn, send_up, recv_dn, recv_up, rank, world, group=None):
    """The halo exchange between ranks in a ring: send_dn goes to the rank
    below (rank - 1), whose recv_up takes it; send_up to the rank above, whose
    recv_dn takes it.  Device tensors with NCCL; with gloo they are staged
    through host memory."""
    import torch.distributed as dist
    if _staged(send_dn, group):
        h = [t.cpu() for t in (send_dn, send_up)] + [torch_empty_host(t) for t in (recv_dn, recv_up)]
        exchange_dist(h[0], h[1], h[2], h[3], rank, world, group)
        recv_dn.copy_(h[2])
        recv_up.copy_(h[3])
        return
    below, above = (rank - 1) % world, (rank + 1) % world
    ops = [dist.P2POp(dist.isend, send_dn, below, group, tag=1),
           dist.P2POp(dist.isend, send_up, above, group, tag=2),
           dist.P2POp(dist.irecv, recv_up, above, group, tag=1),
           dist.P2POp(dist.irecv, recv_dn, below, group, tag=2)]
    for req in dist.batch_isend_irecv(ops):
        req.wait()


def torch_empty_host(t):
    import torch
    return torch.empty(t.shape, dtype=t.dtype, device="cpu")


def all_reduce_sum(t, group=None):
    """Sum of t over the group's ranks, in place (staged through host memory
    for gloo)."""
    import torch.distributed as dist
    if _staged(t, group):
        h = t.cpu()
        dist.all_reduce(h, group=group)
        t.copy_(h)
    else:
        dist.all_reduce(t, group=group)


class SlabLBM:
    """One rank's slab of a z-periodic lattice.

    b_index: the whole lattice [nx][ny][nz] (reference codes); params: keyword
    arguments of default_params for the whole lattice (nz and the z
    periodicity are set here).  world == 1 exchanges with itself.  Several
    slabs of one process (for instance on one GPU) are advanced together with
    exchange_local."""

    def __init__(self, b_index, world=1, rank=0, device=0, stream=None, group=None, halo=HALO, **params):
        import torch
        nx, ny, nz = b_index.shape
        if halo < HALO or halo % HALO:
            raise ValueError("the halo is whole tile layers")
        self.world, self.rank, self.group, self.halo = world, rank, group, halo
        self.z0, self.z1 = slab_bounds(nz, world, rank)
        self.nzs = self.z1 - self.z0 + 2 * halo
        per = list(params.pop("periodic", (0, 0, 1)))
        per[2] = 0
        self.ctx = Context(default_params(nx=nx, ny=ny, nz=self.nzs, periodic=tuple(per), **params), device)
        self.ctx.set_lattice(slab_lattice(b_index, world, rank, halo))
        # inner tile layers and the two face layers are stepped apart; the
        # halo layers are not stepped
        self.ctx.set_slab(halo, self.nzs - halo)
        self.stream = stream if stream is not None else torch.cuda.Stream(device=device)
        self.comm = torch.cuda.Stream(device=device) if world > 1 else None
        self.ctx.set_stream(self.stream.cuda_stream)
        # planes (local z): bottom halo / first interior / last interior / top halo
        self.kb_halo, self.kb, self.kt, self.kt_halo = halo - 1, halo, self.nzs - halo - 1, self.nzs - halo
        counts = plane_counts(b_index)
        for k in (self.kb_halo, self.kb, self.kt, self.kt_halo):
            if self.ctx.plane_count(k) != counts[(self.z0 - halo + k) % nz]:
                raise RuntimeError(f"slab plane {k}: listed points differ from the lattice's")
        half = params.get("storage", 0) in (1, 2)
        dt = torch.int16 if half else torch.int32
        mk = lambda k: torch.empty(5 * self.ctx.plane_count(k), dtype=dt, device=f"cuda:{device}")
        self.send_dn, self.send_up = mk(self.kb), mk(self.kt)
        if world == 1:  # the slab is its own neighbour: unpack straight from the packed planes
            self.recv_up, self.recv_dn = self.send_dn, self.send_up
        else:
            self.recv_up, self.recv_dn = mk(self.kt_halo), mk(self.kb_halo)

    def pack(self):
        self.ctx.plane_pack(self.kb, -1, self.send_dn.data_ptr())
        self.ctx.plane_pack(self.kt, +1, self.send_up.data_ptr())

    def unpack(self):
        self.ctx.plane_unpack(self.kt_halo, -1, self.recv_up.data_ptr())
        self.ctx.plane_unpack(self.kb_halo, +1, self.recv_dn.data_ptr())

    def exchange(self):
        """Halo exchange of this rank (all ranks call it together)."""
        import torch
        self.pack()
        if self.world > 1:
            with torch.cuda.stream(self.stream):
                exchange_dist(self.send_dn, self.send_up, self.recv_dn, self.recv_up, self.rank, self.world,
                              self.group)
        self.unpack()

    def step(self, n=1):
        """n LBM steps of the slab.  Each step packs the faces of the current
        state and exchanges them while the inner tile layers are stepped (they
        read no halo plane), then unpacks the halos and steps the two face
        layers.  The halos of the final state are not filled."""
        for _ in range(n):
            self._lbm_step(False)

    def _lbm_step(self, membrane):
        import torch
        self.pack()
        if self.world > 1:
            self.comm.wait_stream(self.stream)
            with torch.cuda.stream(self.comm):
                exchange_dist(self.send_dn, self.send_up, self.recv_dn, self.recv_up, self.rank,
                              self.world, self.group)
        self.ctx.lbm_step_part(0, False, membrane, membrane)
        if self.world > 1:
            self.stream.wait_stream(self.comm)
        self.unpack()
        self.ctx.lbm_step_part(1, True, membrane, membrane)

    def interior(self, dom=None):
        """Mask of the slab's listed points that are interior, and their
        global z plane."""
        dom = self.ctx.domlist() if dom is None else dom
        k = dom[:, 2]
        return (k >= self.halo) & (k < self.nzs - self.halo), self.z0 + k - self.halo

    def close(self):
        self.ctx.close()


def exchange_local(slabs):
    """The halo exchange among the slabs of one process, in ring order (slab
    r's neighbours are r - 1 and r + 1); they must share one stream."""
    import torch
    n = len(slabs)
    for s in slabs:
        s.pack()
    with torch.cuda.stream(slabs[0].stream):
        for r, s in enumerate(slabs):
            s.recv_up.copy_(slabs[(r + 1) % n].send_dn)
            s.recv_dn.copy_(slabs[(r - 1) % n].send_up)
    for s in slabs:
        s.unpack()


# ---- the coupled step over slabs -------------------------------------------------
#
# Fluid sharded, cells replicated.  Every rank holds all cells (their state is
# small beside the fluid's: 2000 cells of 804 nodes are 39 MB of fp64 positions
# against 0.56 GB of populations on the C1 workload) and runs the membrane forces
# for all of them, so cell ownership, migration and ghost cells do not arise.
# The IB coupling is split by lattice plane (zf_set_ib_slab): a rank
# interpolates over its own planes only, pushes (wall, nucleus-membrane,
# RBC-RBC) only the nodes whose lattice point it owns, and spreads only into its
# own planes.  One all-reduce of the node and repulsion velocities per membrane
# iteration (2 x 3 x nodes + 3 x nucleus nodes fp64 values) then gives every
# rank the unsplit velocities, and every rank moves all cells identically.
# IB_HALO planes of halo (two tile layers) keep the +-4 point windows of the
# repulsion searches of owned nodes inside the slab's lattice.

IB_HALO = 8


class SlabCoupled(SlabLBM):
    """One rank's slab of the coupled step (zf_step split over z slabs).

    wall = (xyz [3][nw], tri1 [3][mt], nrm [3][mt]) in the global frame; mesh =
    the zf_set_mesh arguments; cells = (x, xn) of all cells in the global frame;
    params: default_params keywords for the whole lattice (z periodic)."""

    def __init__(self, b_index, wall, mesh, cells, world=1, rank=0, device=0, stream=None, group=None,
                 **params):
        import torch
        nz = b_index.shape[2]
        base = default_params()
        dx = params.get("dx", base.dx)
        origin = tuple(params.pop("origin", tuple(base.origin)))
        z0, _ = slab_bounds(nz, world, rank)
        oz = origin[2] + (z0 - IB_HALO) * dx  # z of the slab lattice's plane 0
        super().__init__(b_index, world, rank, device, stream, group, halo=IB_HALO,
                         origin=(origin[0], origin[1], oz), **params)
        self.lz = nz * dx
        self.stagger = params.get("stagger", base.stagger)
        self.nuc_period = params.get("nuc_list_period", base.nuc_list_period)
        self.ctx.set_ib_slab(IB_HALO, self.nzs - IB_HALO, self.lz)
        xyz, tri, nrm = wall
        xyz = np.array(xyz, np.float32)
        xyz[2] = oz + np.mod(xyz[2] - oz, self.lz)  # folded into the slab's frame
        self.ctx.set_wall(xyz, tri, nrm)
        self.ctx.set_mesh(*mesh)
        self.ctx.set_cells(*cells)
        self.kin = torch.empty(self.ctx.cells_reduce_size(), dtype=torch.float64, device=f"cuda:{device}")

    def membrane_before_reduce(self):
        """The membrane iteration up to the velocities' reduction: forces, the
        LBM step (moments, body force cleared), interpolation and repulsions of
        this slab; the partial velocities are left in self.kin."""
        it = self.ctx.iteration() + 1
        self.ctx.cgsm_forces()
        self._lbm_step(True)
        self.ctx.ibm_interp()
        self.ctx.nuc_memb_repulsion(it % self.nuc_period == 0)
        self.ctx.rbc_rbc_repulsion()
        self.ctx.cells_reduce_buffer(0, self.kin.data_ptr())

    def membrane_after_reduce(self):
        """Back from the reduction: spreading into this slab's planes, update."""
        self.ctx.cells_reduce_buffer(1, self.kin.data_ptr())
        self.ctx.ibm_spread()
        self.ctx.update_positions()

    def step(self, n=1):
        """n iterations of the reference loop (all ranks call it together)."""
        import torch
        for _ in range(n):
            if (self.ctx.iteration() + 1) % self.stagger:
                self._lbm_step(False)
                continue
            self.membrane_before_reduce()
            if self.world > 1:
                with torch.cuda.stream(self.stream):
                    all_reduce_sum(self.kin, self.group)
            self.membrane_after_reduce()


def coupled_step_local(slabs, n=1):
    """n iterations of the coupled step over the slabs of one process (one
    stream): the halo exchange of exchange_local and the velocities' sum in
    place of the collectives."""
    import torch
    for _ in range(n):
        membrane = (slabs[0].ctx.iteration() + 1) % slabs[0].stagger == 0
        it = slabs[0].ctx.iteration() + 1
        if membrane:
            for s in slabs:
                s.ctx.cgsm_forces()
        for s in slabs:
            s.pack()
        with torch.cuda.stream(slabs[0].stream):
            m = len(slabs)
            for r, s in enumerate(slabs):
                s.recv_up.copy_(slabs[(r + 1) % m].send_dn)
                s.recv_dn.copy_(slabs[(r - 1) % m].send_up)
        for s in slabs:
            s.unpack()
            s.ctx.lbm_step_part(0, False, membrane, membrane)
            s.ctx.lbm_step_part(1, True, membrane, membrane)
        if not membrane:
            continue
        for s in slabs:
            s.ctx.ibm_interp()
            s.ctx.nuc_memb_repulsion(it % s.nuc_period == 0)
            s.ctx.rbc_rbc_repulsion()
            s.ctx.cells_reduce_buffer(0, s.kin.data_ptr())
        with torch.cuda.stream(slabs[0].stream):
            total = torch.stack([s.kin for s in slabs]).sum(dim=0)
            for s in slabs:
                s.kin.copy_(total)
        for s in slabs:
            s.membrane_after_reduce()
