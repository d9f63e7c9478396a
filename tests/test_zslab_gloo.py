"""z-slab decomposition: the exchange schedule of viscoplastic-lbm_b200/zslab.py
run on the host.

The library's slabs trade halos around the odd step of the in-place (AA)
scheme (zslab.py; the reference moves a ghost plane per step,
src/CUDA/lbm.cu:601-657).  Here the device simulation is replaced by a numpy
restatement of the same in-place step (D3Q19 BGK in float64, unused nodes
writing zeros as the library's unused nodes do), so the orchestration --
which planes and populations each phase packs, ring neighbours, message
order and tags, uneven splits, two ranks whose both neighbours are one peer
-- runs as world_size 2 and 3 gloo process groups on CPU and is compared with
the unsharded run bit for bit.
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import zslab

# D3Q19 in the reference's population order (velocitySets/D3Q19.h)
C19 = np.array([(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
                (1, 1, 0), (-1, -1, 0), (1, 0, 1), (-1, 0, -1), (0, 1, 1), (0, -1, -1),
                (1, -1, 0), (-1, 1, 0), (1, 0, -1), (-1, 0, 1), (0, 1, -1), (0, -1, 1)])
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
OPP = np.array([int(np.where((C19 == -c).all(axis=1))[0][0]) for c in C19])
TAU = 0.8


def equilibrium(rho, u):
    cu = np.einsum("qa,a...->q...", C19.astype(float), u)
    uu = (u * u).sum(axis=0)
    return W19[:, None, None, None] * rho * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * uu)


class FakeSlab:
    """In-place D3Q19 BGK on [Q][z][y][x] float64 planes, periodic in every axis.

    Even phase: f_i = A[i](x), A[opp i](x) <- f*_i.  Odd phase: f_i =
    A[opp i](x - c_i), A[i](x + c_i) <- f*_i.  Unused nodes write zeros."""

    def __init__(self, f, unused_planes=()):
        self.A = np.array(f, dtype=np.float64)
        self.parity = 0
        self.unused = np.zeros(self.A.shape[1:], dtype=bool)
        for z in unused_planes:
            self.unused[z] = True
        self.ny, self.nx = self.A.shape[2:]

    def aa_parity(self):
        return self.parity

    def halo_bytes(self):
        return 5 * self.ny * self.nx * 8

    @staticmethod
    def _pops(dz):
        return [i for i in range(19) if C19[i][2] == dz]

    def halo_pack(self, z, dz, dst):
        dst.numpy().view(np.float64)[:] = self.A[self._pops(dz), z].ravel()

    def halo_unpack(self, z, dz, src):
        self.A[self._pops(dz), z] = src.numpy().view(np.float64).reshape(5, self.ny, self.nx)

    def halo_pack2(self, m0, m1):
        for z, dz, buf in (m0, m1):
            self.halo_pack(z, dz, buf)

    def halo_unpack2(self, m0, m1):
        for z, dz, buf in (m0, m1):
            self.halo_unpack(z, dz, buf)

    def _collide(self, f):
        rho = f.sum(axis=0)
        rho = np.where(self.unused, 1.0, rho)
        u = np.einsum("qa,q...->a...", C19.astype(float), f) / rho
        fs = f - (f - equilibrium(rho, u)) / TAU
        fs[:, self.unused] = 0.0
        return fs

    def step(self, n=1):
        for _ in range(n):
            if self.parity == 0:
                self.A = self._collide(self.A)[OPP]
            else:
                f = np.stack([np.roll(self.A[OPP[i]], tuple(C19[i][::-1]), axis=(0, 1, 2)) for i in range(19)])
                fs = self._collide(f)
                self.A = np.stack([np.roll(fs[i], tuple(C19[i][::-1]), axis=(0, 1, 2)) for i in range(19)])
            self.parity ^= 1


def initial_state(nx, ny, nz, seed=7):
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.02 * rng.standard_normal((nz, ny, nx))
    u = 0.04 * rng.standard_normal((3, nz, ny, nx))
    return equilibrium(rho, u)


def slab_of(f, z0, n):
    nz = f.shape[1]
    planes = [(z0 - 1 + k) % nz for k in range(n + 2)]
    return FakeSlab(f[:, planes], unused_planes=(0, n + 1))


def whole(f, steps):
    ref = FakeSlab(f)
    ref.step(steps)
    return ref.A


@pytest.mark.parametrize("n_slabs", [1, 2, 3, 4])
def test_local_ring_equals_the_whole_lattice(n_slabs):
    f = initial_state(6, 5, 11)
    for steps in (5, 6):
        halos = []
        for r in range(n_slabs):
            z0, n = zslab.split(11, n_slabs, r)
            halos.append(zslab.SlabHalo(slab_of(f, z0, n), n, "cpu"))
        zslab.advance(halos, zslab.LocalRing(halos), steps)
        got = np.concatenate([h.sim.A[:, 1:-1] for h in halos], axis=1)
        assert np.array_equal(got, whole(f, steps))


def test_a_slab_that_skips_the_exchange_differs():
    """The comparison can fail: slabs stepped without halos drift from the whole
    lattice after the first odd step."""
    f = initial_state(6, 5, 8)
    halos = [zslab.SlabHalo(slab_of(f, *zslab.split(8, 2, r)), 4, "cpu") for r in range(2)]

    class NoExchange:
        def exchange(self, halos):
            pass

    zslab.advance(halos, NoExchange(), 4)
    got = np.concatenate([h.sim.A[:, 1:-1] for h in halos], axis=1)
    assert not np.allclose(got, whole(f, 4))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nz, steps, out_dir):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        f = initial_state(5, 4, nz)
        z0, n = zslab.split(nz, world, rank)
        halo = zslab.SlabHalo(slab_of(f, z0, n), n, "cpu")
        ring = zslab.RingExchange()
        ring.bind(halo)
        zslab.advance([halo], ring, steps)
        parts = [None] * world
        dist.all_gather_object(parts, halo.sim.A[:, 1:-1])
        if rank == 0:
            np.save(os.path.join(out_dir, "slabs.npy"), np.concatenate(parts, axis=1))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(240)
@pytest.mark.parametrize("world,nz,steps", [(2, 8, 7), (3, 10, 6)])
def test_gloo_ring_equals_the_whole_lattice(tmp_path, world, nz, steps):
    mp.spawn(_worker, args=(world, _free_port(), nz, steps, str(tmp_path)), nprocs=world, join=True)
    got = np.load(os.path.join(tmp_path, "slabs.npy"))
    assert np.array_equal(got, whole(initial_state(5, 4, nz), steps))


def test_schedule_sends_meet_receives():
    """Each message lands where the sender's plane sits in the receiver's
    numbering: the slab below's plane n_b + 1 is this slab's plane 1, and
    the slab above's plane 0 is this slab's plane n."""
    n, n_b, n_a = 4, 3, 5
    for phase in (zslab.PRE, zslab.POST):
        down, up = zslab.sends(n, phase)
        from_above_of_below, _ = zslab.recvs(n_b, phase)
        _, from_below_of_above = zslab.recvs(n_a, phase)
        # the slab below numbers this slab's plane p as n_b + p; the slab above as p - n
        assert from_above_of_below == (n_b + down[0], down[1])
        assert from_below_of_above == (up[0] - n, up[1])


def test_ring_without_a_process_group_is_one_slab_around_itself():
    """RingExchange outside torch.distributed: one rank, periodic onto itself."""
    assert not dist.is_initialized()
    f = initial_state(4, 3, 6)
    halo = zslab.SlabHalo(slab_of(f, 0, 6), 6, "cpu")
    ring = zslab.RingExchange()
    assert (ring.rank, ring.world, ring.below, ring.above) == (0, 1, 0, 0)
    ring.bind(halo)
    zslab.advance([halo], ring, 5)
    assert np.array_equal(halo.sim.A[:, 1:-1], whole(f, 5))
