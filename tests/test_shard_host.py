"""Host logic of the multi-GPU step (simson_b200/shard.py) on the CPU: the
shard ranges, and the two block all-to-alls of a substep run by two and
three gloo ranks over a numpy stand-in for a context's state (the same
[slot][y][kz][kx] blocks, packed and unpacked exactly as sgpu_copy_block
does on the device)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from simson_b200 import shard

NY, NZ, NX2 = 9, 8, 3


class NumpyState:
    """A context's state as numpy: slots x y x kz x kx complex128."""

    def __init__(self, fill):
        self.a = np.full((7, NY, NZ, NX2), fill, np.complex128)

    def copy_block(self, slot0, nslots, ylo, yhi, zlo, zhi, buf_ptr=None, to_state=False):
        n = nslots * (yhi - ylo) * (zhi - zlo) * NX2 * 16
        if buf_ptr is None:
            return n
        buf = np.ctypeslib.as_array((np.ctypeslib.ctypes.c_uint8 * n).from_address(buf_ptr))
        view = buf.view(np.complex128).reshape(nslots, yhi - ylo, zhi - zlo, NX2)
        if to_state:
            self.a[slot0:slot0 + nslots, ylo:yhi, zlo:zhi] = view
        else:
            view[...] = self.a[slot0:slot0 + nslots, ylo:yhi, zlo:zhi]
        return n


def truth(k):
    s, y, z, x = np.meshgrid(np.arange(7), np.arange(NY), np.arange(NZ), np.arange(NX2), indexing="ij")
    return (1000 * s + 100 * y + 10 * z + x + 0.5j * k).astype(np.complex128)


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ranges = shard.shard_ranges(NY, NZ, world)
        ylo, yhi, zlo, zhi = ranges[rank]
        alloc = shard.torch_alloc("cpu")
        a2a = shard.torch_alltoall()
        # A: this rank holds slots 0-4 of its kz planes (all y); afterwards it
        # must hold its planes of every kz plane
        st = NumpyState(-1.0)
        t = truth(1)
        st.a[:, :, zlo:zhi] = t[:, :, zlo:zhi]
        shard.exchange(st, ranges, rank, shard.block_a, a2a, alloc)
        ok_a = np.array_equal(st.a[0:5, ylo:yhi], t[0:5, ylo:yhi])
        # B: this rank holds slots 0-2 of its planes (all kz); afterwards it
        # must hold its kz planes of every plane
        st = NumpyState(-2.0)
        t = truth(2)
        st.a[:, ylo:yhi] = t[:, ylo:yhi]
        shard.exchange(st, ranges, rank, shard.block_b, a2a, alloc)
        ok_b = np.array_equal(st.a[0:3, :, zlo:zhi], t[0:3, :, zlo:zhi])
        out[rank] = int(ok_a) + 2 * int(ok_b)
    finally:
        dist.destroy_process_group()


class CflState:
    """A shard's CFL bookkeeping as the library keeps it (sgpu_cfl_partial,
    sgpu_cfl_set_global): a local partial maximum, the stop test on the
    global one (bla/wcflbl.f:87-93, rot = 0)."""

    def __init__(self, partial, dt, pending=True):
        self.partial, self.dt, self.pending, self.cfl = partial, dt, pending, None

    def cfl_partial(self):
        return self.partial, self.pending

    def cfl_set_global(self, g):
        self.pending = False
        self.cfl = g * np.pi * self.dt
        if not self.cfl <= 10.0:
            raise RuntimeError("CFL*dt above 10")


def _cfl_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        allreduce_max = shard.torch_allreduce_max("cpu")
        # every shard below the limit: the stop test passes everywhere with
        # the largest partial maximum
        st = CflState(10.0 + rank, 0.01)
        g = shard.reduce_cfl(st, allreduce_max)
        ok_max = g == 10.0 + world - 1 and abs(st.cfl - g * np.pi * 0.01) < 1e-15
        # nothing evaluated this substep: no collective, no test
        ok_none = shard.reduce_cfl(CflState(1e9, 0.01, pending=False), allreduce_max) is None
        # only rank 0's planes exceed the limit: every shard stops
        st = CflState(1e6 if rank == 0 else 1.0, 0.01)
        try:
            shard.reduce_cfl(st, allreduce_max)
            stopped = False
        except RuntimeError:
            stopped = True
        # the ranks are still in step afterwards (the same collectives ran)
        dist.barrier()
        out[rank] = int(ok_max) + 2 * int(ok_none) + 4 * int(stopped)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges_cover_the_domain():
    for nr in (1, 2, 3, 4, 8):
        rg = shard.shard_ranges(193, 384, nr)
        assert rg[0][0] == 0 and rg[-1][1] == 193 and rg[0][2] == 0 and rg[-1][3] == 384
        for a, b in zip(rg, rg[1:]):
            assert a[1] == b[0] and a[3] == b[2]
        assert max(r[1] - r[0] for r in rg) - min(r[1] - r[0] for r in rg) <= 1
    with pytest.raises(ValueError):
        shard.shard_ranges(4, 8, 5)


@pytest.mark.parametrize("world", [2, 3])
def test_block_all_to_alls_gloo(world):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert all(out[r] == 3 for r in range(world)), dict(out)


@pytest.mark.parametrize("world", [2, 3])
def test_cfl_all_reduce_gloo(world):
    """The sharded stop test: the shards' partial CFL maxima are all-reduced
    before the test, so one shard over the limit stops every shard (the
    reference all-reduces before wcflbl.f:93)."""
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = free_port()
    procs = [ctx.Process(target=_cfl_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert all(out[r] == 7 for r in range(world)), dict(out)
