"""Column sharding of the answer path across GPUs, one process per GPU.

A response is the concatenation of `outputs = cols / n` parts of part_len bytes, and part o depends only on the
database columns [o n, (o + 1) n), the packing-matrix rows of those columns, bold_t_hat_o and prefix_o: the scan and
the pack work column by column and the tail output by output (src/amx_kernels.cpp:564-615).  So the outputs split
into contiguous ranges, one per rank; each rank holds only its columns (a database larger than one GPU fits across
several), answers every request for its parts, and the parts are gathered in output order.  No reduction is needed;
the only exchanges are the broadcast of the frames and the gather of the parts.

A shard's engine is the ordinary engine over a column slice of the state: every buffer of the state is ordered by
column (or by output), so a slice is a view, and the frames are the same for every shard (the request length depends
on the record count and the key count only).
"""
import dataclasses

import numpy as np

from .engine import Engine, TiledDb
from .service import Params, Q


def output_ranges(outputs, world):
    """Contiguous output ranges [o0, o1), one per rank, sizes differing by at most one (lower ranks take the extra)."""
    if world < 1 or outputs < world:
        raise ValueError(f"cannot split {outputs} outputs over {world} ranks")
    base, extra = divmod(outputs, world)
    ranges, o = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        ranges.append((o, o + k))
        o += k
    return ranges


def slice_state(st, o0, o1):
    """The engine state of outputs [o0, o1) (database columns [o0 n, o1 n)) as views of `st`, a
    service.SyntheticState or any object with its fields."""
    p, n = st.p, st.p.n
    c0, c1 = o0 * n, o1 * n
    count = p.count
    return dataclasses.replace(
        st, p=Params(p.rows, c1 - c0), db_col=st.db_col[c0:c1],
        U=None if st.U is None else st.U[c0:c1],
        ub=st.ub[c0 * 4 * count:c1 * 4 * count],
        that=list(st.that[o0:o1]), prefixes=list(st.prefixes[o0:o1]))


def shard_engine(st, o0, o1, threads=1):
    """An engine over outputs [o0, o1) of the state (its column slice); its responses are those parts."""
    sl = slice_state(st, o0, o1)
    p = sl.p
    tiled = TiledDb.__new__(TiledDb)  # this engine reads the column-order database only
    tiled.rows, tiled.cols, tiled.buf = p.rows, p.record_bytes, np.zeros(64, dtype=np.uint8)
    return Engine(sl.db_col, tiled, st.db_col.shape[1], sl.ub, p.n, p.tg, sl.prefixes, p.row1_off, 1 << p.q1_bits,
                  p.q1_bits, sl.that, sl.inv_table, Q, threads)


def assemble(parts, ranges, part_len, out=None):
    """Full responses from each rank's parts: out[:, o0 * part_len:o1 * part_len] = parts[r][:, :(o1 - o0) * part_len].
    Works on numpy arrays and torch tensors alike (parts may be padded on the right)."""
    b = parts[0].shape[0]
    if out is None:
        like = parts[0]
        total = ranges[-1][1] * part_len
        out = np.empty((b, total), dtype=np.uint8) if isinstance(like, np.ndarray) else like.new_empty((b, total))
    for (o0, o1), part in zip(ranges, parts):
        w = (o1 - o0) * part_len
        out[:, o0 * part_len:o0 * part_len + w] = part[:, :w]
    return out


class ShardedAnswerer:
    """Answers batches on every rank of a torch.distributed group, each rank for its output range.

    `local(slots, stride, b)` answers the batch on this rank and returns (statuses as a numpy int32 array, this rank's
    parts as a tensor of b rows on `device`, at least (o1 - o0) * part_len bytes wide); the engine-backed default is
    `engine_local(engine)`.  `answer` broadcasts the frames from `src`, answers, checks that every rank reached the same
    statuses, and gathers the parts (all_gather over NCCL, or gloo on the CPU) into full responses on every rank.
    """

    def __init__(self, local, ranges, part_len, device, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.local = local
        self.ranges = ranges
        self.part_len = part_len
        self.device = device
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        assert len(ranges) == self.world
        self.width = max(o1 - o0 for o0, o1 in ranges) * part_len

    def answer(self, slots, stride, b, src=0):
        import torch
        dist = self.dist
        dist.broadcast(slots, src=src, group=self.group)
        status, parts = self.local(slots, stride, b)
        if parts.shape[1] < self.width:  # pad to a common width for all_gather
            parts = torch.nn.functional.pad(parts, (0, self.width - parts.shape[1]))
        st_t = torch.as_tensor(np.asarray(status, dtype=np.int32), device=self.device)
        all_status = [torch.empty_like(st_t) for _ in range(self.world)]
        dist.all_gather(all_status, st_t, group=self.group)
        if any(not torch.equal(s, all_status[0]) for s in all_status[1:]):
            raise RuntimeError("ranks reached different statuses for the same frames")
        gathered = [torch.empty_like(parts) for _ in range(self.world)]
        dist.all_gather(gathered, parts.contiguous(), group=self.group)
        return status, assemble(gathered, self.ranges, self.part_len)


def engine_local(engine):
    """The `local` answerer of ShardedAnswerer for an engine on the current CUDA device: frames already in device
    memory (`slots`, frame c at byte c * stride + 7), parts written to a device tensor."""
    import torch

    def local(slots, stride, b):
        parts = torch.zeros((b, engine.response_len()), dtype=torch.uint8, device=slots.device)
        # the frames (the broadcast) and the zeroed parts come through torch's current stream, on which the engine's
        # own stream does not wait
        torch.cuda.current_stream(slots.device).synchronize()
        status = np.full(b, -1, dtype=np.int32)
        r = engine.answer_device(slots.data_ptr(), stride, b, parts.data_ptr(), engine.response_len(), status)
        if r < 0:
            raise RuntimeError(f"engine error {r}")
        return status, parts

    return local


class PeerGather:
    """Column shards whose tails do the all-gather: every rank's tail kernel writes its response parts straight into
    every rank's full-width response buffer -- its own, and the other ranks' through CUDA IPC mappings (NVLink
    stores between GPUs) -- so that after each call and one barrier every rank holds the full responses, and no
    collective moves response bytes (alto_answer_device_parts).

    `engine` is this rank's shard engine over outputs ranges[rank]; `buffer` is this rank's (b_max, full width)
    device tensor of responses, overwritten by every call.  The IPC handles are exchanged once, here, with
    all_gather_object over the process group (any backend).  Call close() on every rank before the group ends."""

    def __init__(self, engine, ranges, part_len, b_max, group=None):
        import ctypes
        import torch
        import torch.distributed as dist
        from . import lib, last_error
        self.dist, self.group, self.engine = dist, group, engine
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        assert len(ranges) == self.world
        self.offset = ranges[self.rank][0]
        self.buffer = torch.zeros((b_max, ranges[-1][1] * part_len), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        # the buffer may sit inside a larger allocation of torch's caching allocator: the handle names that
        # allocation, and the buffer's offset in it travels with the handle
        h, off = (ctypes.c_uint8 * 64)(), ctypes.c_size_t(0)
        if lib().alto_ipc_export(self.buffer.data_ptr(), h, ctypes.byref(off)) != 0:
            raise RuntimeError(f"alto_ipc_export: {last_error()}")
        handles = [None] * self.world
        self.export_offset = off.value
        dist.all_gather_object(handles, (bytes(h), off.value), group=group)
        self.mapped, self.dsts = [], []
        for r, (hb, offset) in enumerate(handles):
            if r == self.rank:
                self.dsts.append(self.buffer.data_ptr())
                continue
            base = lib().alto_ipc_import((ctypes.c_uint8 * 64).from_buffer_copy(hb))
            if not base:
                raise RuntimeError(f"alto_ipc_import of rank {r}: {last_error()}")
            self.mapped.append(base)
            self.dsts.append(base + offset)

    def answer(self, slots, stride, b, src=None):
        """Answers frames resident in device memory (frame c at slots + c * stride + 7), the same frames on every
        rank (broadcast from rank `src` first when given).  Returns (statuses, this rank's full responses, rows
        :b), complete on every rank when the call returns on any and valid until the next call (which first waits
        for every rank to arrive, so no rank overwrites responses another is still reading)."""
        import torch
        self.dist.barrier(group=self.group)  # every rank is done with the previous call's responses
        if src is not None:
            self.dist.broadcast(slots, src=src, group=self.group)
        torch.cuda.current_stream().synchronize()  # the engine's stream does not wait on torch's
        status = np.full(b, -1, dtype=np.int32)
        r = self.engine.answer_device_parts(slots.data_ptr(), stride, b, self.dsts, self.buffer.shape[1],
                                            self.offset, status)
        if r < 0:
            from . import last_error
            raise RuntimeError(f"engine error {r}: {last_error()}")
        self.dist.barrier(group=self.group)  # every shard's parts are in every buffer
        return status, self.buffer[:b]

    def close(self):
        from . import lib
        self.dist.barrier(group=self.group)  # no rank writes into a mapping after this
        for p in self.mapped:
            lib().alto_ipc_release(p)
        self.mapped = []
