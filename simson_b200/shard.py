"""Multi-GPU channel step: the reference's z-slab decomposition (bla/par.f:102,
memnz = nz/nproc) with its two plane transposes per substep (bla/getpxz.f,
bla/putpxz.f) as block all-to-alls between one whole-state context per GPU.

Shard r of P computes step 2 on the xz-planes ylo_r <= y < yhi_r and step 3
on the stored kz planes zlo_r <= iz < zhi_r (all kx); its context holds
whole-size arrays of which it keeps those parts current.  Per substep:

  A. before step 2, slots 0-4 (u, v, w, omega_x, omega_z) of shard s's
     planes and shard r's kz planes go from r to s;
  B. after step 2, slots 0-2 (H) of shard r's planes and shard s's kz
     planes go from r to s;

so each shard moves 8 fields x (1/P of the planes) x (1/P of the pencils)
to each other shard per substep.  The mean flow (kx = kz = 0) and the
constant-flux pressure gradient stay on the shard that owns iz = 0; prhs runs
on the whole uploaded state in every context.

The transport is a function alltoall(send, send_sizes, recv, recv_sizes) on
byte buffers: torch.distributed.all_to_all_single (NCCL between GPUs, gloo in
the CPU tests) or, for P shards emulated in one process on one device, plain
device copies (LocalShards).
"""
from __future__ import annotations

A_SLOTS = (0, 5)  # (first slot, slot count) moved before step 2
B_SLOTS = (0, 3)  # moved after step 2


def split(n, parts):
    """Balanced contiguous ranges [lo, hi) covering 0..n-1."""
    base, extra = divmod(n, parts)
    out, lo = [], 0
    for i in range(parts):
        hi = lo + base + (1 if i < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def shard_ranges(ny, nz, nranks):
    """(ylo, yhi, zlo, zhi) of every shard: xz-planes for step 2, kz planes
    for step 3."""
    if nranks > min(ny, nz):
        raise ValueError(f"{nranks} shards for {ny} planes and {nz} kz planes")
    ys, zs = split(ny, nranks), split(nz, nranks)
    return [(ys[r][0], ys[r][1], zs[r][0], zs[r][1]) for r in range(nranks)]


def block_a(ranges, r, s):
    """Block that shard r sends to shard s before step 2 (slot0, nslots,
    ylo, yhi, zlo, zhi): shard s's planes of shard r's kz planes."""
    return A_SLOTS + (ranges[s][0], ranges[s][1], ranges[r][2], ranges[r][3])


def block_b(ranges, r, s):
    """Block that shard r sends to shard s after step 2: shard r's planes of
    shard s's kz planes."""
    return B_SLOTS + (ranges[r][0], ranges[r][1], ranges[s][2], ranges[s][3])


def exchange(state, ranges, rank, block, alltoall, alloc, nosync=False):
    """One block all-to-all seen from shard `rank`: pack block(rank, s) for
    every other shard s, exchange, unpack block(s, rank) from every s.

    state.copy_block(slot0, nslots, ylo, yhi, zlo, zhi, buf_ptr=None,
    to_state=False) packs/unpacks a block and returns its bytes; alloc(n)
    returns (buffer, address) of n bytes; alltoall moves the buffers.
    nosync: the copies are only enqueued on the state's stream (the
    transport then runs on the same stream)."""
    nr = len(ranges)
    kw = {"nosync": True} if nosync else {}
    send_sizes = [0 if s == rank else state.copy_block(*block(ranges, rank, s)) for s in range(nr)]
    recv_sizes = [0 if s == rank else state.copy_block(*block(ranges, s, rank)) for s in range(nr)]
    send, sp = alloc(sum(send_sizes))
    recv, rp = alloc(sum(recv_sizes))
    off = 0
    for s in range(nr):
        if send_sizes[s]:
            state.copy_block(*block(ranges, rank, s), buf_ptr=sp + off, to_state=False, **kw)
        off += send_sizes[s]
    if nr > 1:
        alltoall(send, send_sizes, recv, recv_sizes)
    off = 0
    for s in range(nr):
        if recv_sizes[s]:
            state.copy_block(*block(ranges, s, rank), buf_ptr=rp + off, to_state=True, **kw)
        off += recv_sizes[s]
    return sum(send_sizes), sum(recv_sizes)


def reduce_cfl(state, allreduce_max):
    """The CFL stop test of a sharded substep (bla/wcflbl.f:82-98): the
    shards' partial maxima all-reduced (MAX), then the test on every shard
    with the global value, so that every shard stops together.  Returns the
    global partial maximum, or None when this substep evaluated no CFL number
    (every shard is at the same substep, so all take the same branch)."""
    m, pending = state.cfl_partial()
    if not pending:
        return None
    g = allreduce_max(m)
    state.cfl_set_global(g)  # raises the library's CFL / non-finite error
    return g


def torch_alloc(device):
    import torch

    def alloc(n):
        t = torch.empty(max(n, 1), dtype=torch.uint8, device=device)
        return t, t.data_ptr()
    return alloc


class PersistentBuffers:
    """Send and receive buffers kept for the life of a sharded run (the
    exchanges reuse them every substep on the library's stream, so no buffer
    is freed while a copy on that stream may still use it).  alloc(tag)
    returns an allocator for one exchange: its first call gives the send
    buffer, its second the receive buffer."""

    def __init__(self, device, sync):
        self.device, self.sync, self.bufs = device, sync, {}

    def alloc(self, tag):
        import torch
        calls = [0]

        def _alloc(n):
            key = (tag, calls[0])
            calls[0] += 1
            t = self.bufs.get(key)
            if t is None or t.numel() < n:
                if t is not None:
                    self.sync()  # a larger block: the old buffer may still be in use
                t = torch.empty(max(n, 1), dtype=torch.uint8, device=self.device)
                self.bufs[key] = t
            return t, t.data_ptr()
        return _alloc


def torch_alltoall(group=None, stream=None):
    """all_to_all_single over the group.  stream: a CUDA stream address (the
    library's) on which the transfer is ordered, with no host
    synchronisation; None: the current stream, completed before returning."""
    import torch.distributed as dist

    def alltoall(send, send_sizes, recv, recv_sizes):
        import torch
        if stream is not None and recv.is_cuda:
            with torch.cuda.stream(torch.cuda.ExternalStream(stream, device=recv.device)):
                dist.all_to_all_single(recv[:sum(recv_sizes)], send[:sum(send_sizes)],
                                       output_split_sizes=recv_sizes, input_split_sizes=send_sizes, group=group)
            return
        dist.all_to_all_single(recv[:sum(recv_sizes)], send[:sum(send_sizes)], output_split_sizes=recv_sizes,
                               input_split_sizes=send_sizes, group=group)
        if recv.is_cuda:
            torch.cuda.current_stream(recv.device).synchronize()
    return alltoall


def torch_allreduce_max(device, group=None):
    import torch
    import torch.distributed as dist

    def allreduce_max(x):
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        return float(t.item())
    return allreduce_max


class ShardedChannel:
    """This rank's shard of a channel spread over the ranks of a
    torch.distributed group (one GPU each).  `channel` holds the whole
    problem (simson_b200.bla.Channel on this rank's device) with the same
    state uploaded and prhs done in every rank.

    Per substep the packs, the NCCL all-to-all and the unpacks are ordered on
    the library's stream, with no host synchronisation between them; the
    host waits only for the CFL partial maximum on the substeps that
    evaluate it (every icfl substeps, as the reference)."""

    def __init__(self, channel, rank, nranks, device, group=None):
        self.ch = channel
        self.nst = getattr(channel, "nst", 3)
        self.rank, self.nranks = rank, nranks
        self.ranges = shard_ranges(channel.ny, channel.nz, nranks)
        channel.set_shard(*self.ranges[rank])
        self._bufs = PersistentBuffers(device, channel.sync)
        self._alltoall = torch_alltoall(group, stream=channel.stream_ptr())
        self._allreduce_max = torch_allreduce_max(device, group)
        self.bytes_moved = 0

    def substep(self):
        s1, _ = exchange(self.ch, self.ranges, self.rank, block_a, self._alltoall, self._bufs.alloc("a"),
                         nosync=True)
        self.ch.nonlinbl()
        reduce_cfl(self.ch, self._allreduce_max)
        s2, _ = exchange(self.ch, self.ranges, self.rank, block_b, self._alltoall, self._bufs.alloc("b"),
                         nosync=True)
        self.ch.linearbl()
        self.bytes_moved += s1 + s2

    def step(self, n=1):
        for _ in range(self.nst * n):
            self.substep()


class LocalShards:
    """P shards of one channel emulated in one process on one device: one
    context each, the all-to-alls as device copies between them (the same
    blocks a multi-GPU run moves).  make_channel() returns a Channel with the
    state uploaded and prhs done."""

    def __init__(self, make_channel, nranks, device):
        self.chs = [make_channel() for _ in range(nranks)]
        self.nst = getattr(self.chs[0], "nst", 3)
        self.ranges = shard_ranges(self.chs[0].ny, self.chs[0].nz, nranks)
        for ch, rg in zip(self.chs, self.ranges):
            ch.set_shard(*rg)
        self._alloc = torch_alloc(device)

    def _exchange(self, block):
        nr = len(self.chs)
        for r in range(nr):
            for s in range(nr):
                if r == s:
                    continue
                b = block(self.ranges, r, s)
                buf, ptr = self._alloc(self.chs[r].copy_block(*b))
                self.chs[r].copy_block(*b, buf_ptr=ptr, to_state=False)
                self.chs[s].copy_block(*b, buf_ptr=ptr, to_state=True)

    def substep(self):
        self._exchange(block_a)
        for ch in self.chs:
            ch.nonlinbl()
        # the CFL stop test on the maximum over the shards
        parts = [ch.cfl_partial() for ch in self.chs]
        if parts[0][1]:
            g = max(m for m, _ in parts)
            for ch in self.chs:
                ch.cfl_set_global(g)
        self._exchange(block_b)
        for ch in self.chs:
            ch.linearbl()

    def step(self, n=1):
        for _ in range(self.nst * n):
            self.substep()

    def state(self, nslots=7):
        """The whole state assembled from the shards' kz planes."""
        import numpy as np
        parts = [ch.state(nslots) for ch in self.chs]
        out = [np.array(p) for p in parts[0]]
        for (ylo, yhi, zlo, zhi), p in zip(self.ranges, parts):
            for k in range(nslots):
                out[k][zlo:zhi] = p[k][zlo:zhi]
        return out

    def close(self):
        for ch in self.chs:
            ch.close()
