"""One lattice split along z over several GPUs: one z-slab per process.

The reference decomposes a lattice into N_GPUS slabs of NZ planes, each with a
ghost plane, and moves the populations that cross a slab face between
neighbouring GPUs in a ring after every step (gpuPopulationsTransfer,
src/CUDA/lbm.cu:601-657, called from main.cu:336-350).  Here:

* A slab of n planes is a simulation of n + 2 planes (vlbm_config.slab_*).
  Local planes 0 and n + 1 mirror global planes z0 - 1 and z0 + n (periodic in
  z, as the whole lattice is) and are marked unused in the node map.
* The in-place step's even phase reads and writes only each node's own slots,
  so it needs no exchange.  Its odd phase reads and writes, for every node x,
  the slots (x + c_i, i); at a slab face half of those belong to the nodes of
  the neighbouring slab.  Around each odd step every slab therefore trades two
  messages per face with its neighbours:

      before the odd step:  plane 1,     c_z = +1  ->  the slab below's plane n + 1
                            plane n,     c_z = -1  ->  the slab above's plane 0
      after it:             plane 0,     c_z = -1  ->  the slab below's plane n
                            plane n + 1, c_z = +1  ->  the slab above's plane 1

  A message is the 5 (D3Q19) or 9 (D3Q27) populations with that c_z of one
  plane, in the storage type (vlbm_halo_pack / vlbm_halo_unpack).  The ghost
  nodes themselves run as unused nodes and write only slots that an exchange
  overwrites before they are read, or that no node of the slab reads.
* Between an even and an odd step a node's populations sit at its neighbours,
  so reading the state (macroscopics, populations, sums) first runs the
  exchange that the next odd step starts with (`refresh`).

The slabs' results equal the whole lattice's: every node of a slab sees the
same populations in the same order as in the unsharded run.  Boundary rules
that read another node's post-collision values across a slab face (free-slip
walls normal to x or y) and spheres are refused on slabs.

Transport: `RingExchange` over a torch.distributed group (NCCL between GPUs,
gloo for host tensors) with one process per slab; `LocalRing` for several
slabs held by one process (on one device, ordered on one stream).
"""
import numpy as np
import torch
import torch.distributed as dist

import vlbm

PRE, POST = 0, 1


def sends(n, phase):
    """(plane, dz) packed for the slab below and for the slab above."""
    return ((1, +1), (n, -1)) if phase == PRE else ((0, -1), (n + 1, +1))


def recvs(n, phase):
    """(plane, dz) receiving the message of the slab above and of the slab below."""
    return ((n + 1, +1), (0, -1)) if phase == PRE else ((n, -1), (1, +1))


def split(nz_total, world, rank):
    """First global plane and plane count of rank's slab."""
    z0 = rank * nz_total // world
    return z0, (rank + 1) * nz_total // world - z0


class SlabHalo:
    """Message buffers of one slab: send[0] goes down, send[1] up; recv[0]
    comes from the slab above, recv[1] from the slab below.  Each exchange is
    one packing launch for both sends and one unpacking launch for both
    receives (vlbm_halo_pack2 / vlbm_halo_unpack2)."""

    def __init__(self, sim, n_planes, device):
        nb = sim.halo_bytes()
        self.sim, self.n = sim, n_planes
        self.send = [torch.empty(nb, dtype=torch.uint8, device=device) for _ in range(2)]
        self.recv = [torch.empty(nb, dtype=torch.uint8, device=device) for _ in range(2)]

    def pack(self, phase):
        (z0, d0), (z1, d1) = sends(self.n, phase)
        self.sim.halo_pack2((z0, d0, self.send[0]), (z1, d1, self.send[1]))

    def unpack(self, phase):
        (z0, d0), (z1, d1) = recvs(self.n, phase)
        self.sim.halo_unpack2((z0, d0, self.recv[0]), (z1, d1, self.recv[1]))


class LocalRing:
    """Slabs held by one process, in ring order: each slab packs straight into
    its neighbours' receive buffers, so the exchange itself moves nothing."""

    def __init__(self, halos):
        r_n = len(halos)
        for r, h in enumerate(halos):
            h.send = [halos[(r - 1) % r_n].recv[0], halos[(r + 1) % r_n].recv[1]]

    def exchange(self, halos):
        pass


class RingExchange:
    """One slab per rank of a torch.distributed group, slab r between ranks r - 1
    and r + 1 (mod world).  Point-to-point messages in one batch: the two sends
    (down, then up) and the two receives (from above, then from below), so that
    with two ranks, where both neighbours are the same peer, the n-th send to a
    peer meets that peer's n-th receive; tags tell them apart on gloo."""

    def __init__(self, group=None):
        self.group = group
        ready = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if ready else 0
        self.world = dist.get_world_size(group) if ready else 1

        def glob(r):
            return dist.get_global_rank(group, r) if group is not None else r

        self.below = glob((self.rank - 1) % self.world)
        self.above = glob((self.rank + 1) % self.world)

    def bind(self, halo):
        """A single slab is its own neighbour: it packs into its receive buffers."""
        if self.world == 1:
            halo.send = [halo.recv[0], halo.recv[1]]

    def exchange(self, halos):
        if self.world == 1:
            return
        (h,) = halos
        ops = [dist.P2POp(dist.isend, h.send[0], self.below, self.group, 0),
               dist.P2POp(dist.isend, h.send[1], self.above, self.group, 1),
               dist.P2POp(dist.irecv, h.recv[0], self.above, self.group, 0),
               dist.P2POp(dist.irecv, h.recv[1], self.below, self.group, 1)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()


def advance(halos, transport, steps):
    """Advance every slab of `halos` by `steps` steps, trading halos around
    each odd step.  The slabs must be in step (same counter and parity)."""
    odd = steps > 0 and halos[0].sim.aa_parity() == 1
    for _ in range(steps):
        if odd:
            for h in halos:
                h.pack(PRE)
            transport.exchange(halos)
            for h in halos:
                h.unpack(PRE)
        for h in halos:
            h.sim.step(1)
        if odd:
            for h in halos:
                h.pack(POST)
            transport.exchange(halos)
            for h in halos:
                h.unpack(POST)
        odd = not odd


def refresh(halos, transport):
    """Fill the ghost planes for reading the state.  Between an even and an odd
    step a node's populations f_i(x) sit at its neighbours (x - c_i), so
    macroscopics, populations and sums read the ghost planes; this is the
    exchange the next odd step starts with (running it twice changes nothing)."""
    if halos[0].sim.aa_parity() == 1:
        for h in halos:
            h.pack(PRE)
        transport.exchange(halos)
        for h in halos:
            h.unpack(PRE)


def slab_config(cfg, z0, n, nz_total):
    """Copy of a whole-lattice configuration for the slab [z0, z0 + n)."""
    c = vlbm.Config()
    C_ = type(cfg)
    for name, _ in C_._fields_:
        setattr(c, name, getattr(cfg, name))
    c.nz = n + 2
    c.slab_z_offset = (z0 - 1) % nz_total
    c.slab_nz_total = nz_total
    return c


def slab_node_map(builder, cfg, z0, n, nz_total):
    """The builder's words of planes z0 - 1 .. z0 + n, ghost planes unused."""
    m = vlbm.build_node_map_planes(builder, cfg.nx, cfg.ny, nz_total, z0 - 1, n + 2)
    m = m.reshape(n + 2, cfg.ny, cfg.nx)
    m[0] = 0
    m[-1] = 0
    return m.ravel()


class ZSlab:
    """This rank's slab of a lattice of cfg.nz planes, sharded over the ranks of
    a torch.distributed group (one process, one GPU per slab).

    cfg describes the whole lattice; builder is a VLBM_BUILDER_* id.  The
    simulation, the packing kernels and the NCCL exchange share one stream
    (`self.stream`), so they are ordered without host synchronisation."""

    def __init__(self, cfg, builder, group=None, autotune=False):
        self.transport = RingExchange(group)
        self.nz_total = cfg.nz
        self.z0, self.n = split(cfg.nz, self.transport.world, self.transport.rank)
        if self.n < 1:
            raise ValueError("fewer planes than ranks")
        self.cfg = slab_config(cfg, self.z0, self.n, cfg.nz)
        self.device = torch.device("cuda", self.cfg.device)
        self.stream = torch.cuda.Stream(self.device)
        self.sim = vlbm.Simulation(self.cfg, node_map=slab_node_map(builder, cfg, self.z0, self.n, cfg.nz))
        self.sim.set_stream(self.stream.cuda_stream)
        if autotune:
            self.sim.autotune()
        self.halo = SlabHalo(self.sim, self.n, self.device)
        self.transport.bind(self.halo)

    def step(self, steps=1):
        with torch.cuda.stream(self.stream):
            advance([self.halo], self.transport, steps)

    def refresh(self):
        with torch.cuda.stream(self.stream):
            refresh([self.halo], self.transport)

    def macroscopics(self):
        """rho, u, omega of this slab's own planes (host arrays, [n][ny][nx])."""
        self.refresh()
        return {k: v[1:-1] for k, v in self.sim.macroscopics().items()}

    def moments_sum(self):
        """FP64 sums of the whole lattice (ghost nodes are unused and not
        counted), all-reduced over the group."""
        self.refresh()
        t = torch.tensor(self.sim.moments_sum(), dtype=torch.float64, device=self.device)
        if self.transport.world > 1:
            dist.all_reduce(t, group=self.transport.group)
        return t.cpu().numpy()

    def close(self):
        self.sim.close()


class LocalSlabs:
    """The same decomposition with every slab in this process, on one device:
    the exchange is a device copy between message buffers, ordered with the
    steps on one stream (`self.stream`)."""

    def __init__(self, cfg, builder, n_slabs, layout=None):
        self.nz_total = cfg.nz
        self.device = torch.device("cuda", cfg.device)
        self.stream = torch.cuda.Stream(self.device)
        self.slabs, self.halos = [], []
        for r in range(n_slabs):
            z0, n = split(cfg.nz, n_slabs, r)
            c = slab_config(cfg, z0, n, cfg.nz)
            if layout is not None:
                c.layout = layout
            sim = vlbm.Simulation(c, node_map=slab_node_map(builder, cfg, z0, n, cfg.nz))
            sim.set_stream(self.stream.cuda_stream)
            self.slabs.append((z0, n, sim))
            self.halos.append(SlabHalo(sim, n, self.device))
        self.transport = LocalRing(self.halos)

    def step(self, steps=1):
        with torch.cuda.stream(self.stream):
            advance(self.halos, self.transport, steps)

    def refresh(self):
        with torch.cuda.stream(self.stream):
            refresh(self.halos, self.transport)

    def macroscopics(self):
        """Macroscopics of the whole lattice, [nz][ny][nx] per field."""
        self.refresh()
        parts = [sim.macroscopics() for _, _, sim in self.slabs]
        return {k: np.concatenate([p[k][1:-1] for p in parts]) for k in parts[0]}

    def populations(self):
        """f_i of the whole lattice, [Q][nz][ny][nx]."""
        self.refresh()
        return np.concatenate([sim.populations()[:, 1:-1] for _, _, sim in self.slabs], axis=1)

    def close(self):
        for _, _, sim in self.slabs:
            sim.close()
