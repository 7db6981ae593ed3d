"""Partitioned single-root BFS over several ranks (a 1-D vertex partition).

The reference runs one BFS over a 2-D partition of MPI ranks and exchanges
the frontier every level (mpi/bfs.hpp:521-572 expand, :962-1137 top-down
fold packets, bottom_up_comm.hpp:172-280 the bottom-up bitmap ring; layout
graph_constructor.hpp:18-22).  Here rank r owns a contiguous range of
reordered vertex ids and the rows of those vertices (g500_part_* in
libg500.so does each rank's device work); this module runs the level loop and
the collectives:

  top-down   each rank expands its frontier rows, claims its own targets and
             sends (target, parent) pairs to the owners of the others (one
             all-to-all), which claim them;
  bottom-up  each rank's unvisited vertices look for a parent among the
             vertices visited before the level (the full bitmap);
  every level: the level counters summed over the ranks (every rank takes the
             reference's direction decision, bfs.hpp:2799-2829, from the same
             sums) and the ranks' bitmap slices all-gathered.

At the end the ranks' pred arrays (their own vertices' entries, -1 elsewhere)
combine by an element-wise max into pred (parent | level << 48, root = root).

Two ways to run the ranks:
  TorchComm   one process per GPU over torch.distributed (NCCL; gloo on CPU);
  LocalComm   every rank in one process on one device, the collectives as
              copies between the ranks' buffers (no kernel waits for another).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import G500Error, G500_E_INVAL, _device_u8, check, lib

MAX_LEVELS = 0xFFFE


# ----------------------------------------------------------------------------- engines
class CudaRank:
    """One rank's device work (g500_part_*), on the rank's graph replica."""

    def __init__(self, graph, rank: int, nranks: int):
        import torch
        self.graph, self.rank, self.nranks = graph, rank, nranks
        h = C.c_void_p()
        check(lib().g500_part_create(graph.h, rank, nranks, C.byref(h)))
        self.h = h
        S, lo, hi = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().g500_part_info(self.h, C.byref(S), C.byref(lo), C.byref(hi)))
        self.S, self.lo, self.hi = S.value, lo.value, hi.value
        vf, own, st = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().g500_part_buffers(self.h, C.byref(vf), C.byref(own), C.byref(st)))
        self.vis_full = _device_u8(vf.value, 4 * self.S * nranks).view(torch.int32)
        self.own = _device_u8(own.value, 4 * self.S).view(torch.int32)
        self.device = self.own.device

    def begin(self, root: int):
        out = (C.c_int64 * 3)()
        check(lib().g500_part_begin(self.h, int(root), out))
        return list(out)

    def top_down(self, frontier_edges: int):
        counts = (C.c_int64 * self.nranks)()
        check(lib().g500_part_top_down(self.h, int(frontier_edges), counts))
        return list(counts)

    def send_pairs(self, total: int):
        import torch
        if total == 0:
            return torch.empty(0, dtype=torch.int64, device=self.device)
        p = C.c_void_p()
        check(lib().g500_part_send_buffer(self.h, C.byref(p)))
        return _device_u8(p.value, 8 * total).view(torch.int64)

    def apply(self, recv):
        out = (C.c_int64 * 4)()
        n = int(recv.numel())
        check(lib().g500_part_apply(self.h, C.c_void_p(recv.data_ptr() if n else 0), n, out))
        return list(out)

    def bottom_up(self):
        out = (C.c_int64 * 4)()
        check(lib().g500_part_bottom_up(self.h, out))
        return list(out)

    def compact(self):
        n = C.c_int64()
        check(lib().g500_part_compact(self.h, C.byref(n)))
        return n.value

    def write_pred(self, pred):
        check(lib().g500_part_write_pred(self.h, C.c_void_p(pred.data_ptr())))

    def new_pred(self):
        import torch
        return torch.empty(self.graph.pred_size(), dtype=torch.int64, device=self.device)

    def close(self):
        if self.h is not None:
            check(lib().g500_part_destroy(self.h))
            self.h = None


# ----------------------------------------------------------------------------- collectives
class LocalComm:
    """Every rank in this process: the collectives are copies between the
    ranks' buffers, made between the ranks' steps (each step has finished on
    the device when it returns)."""

    def __init__(self, nranks: int):
        self.nranks = nranks
        self.local_ranks = list(range(nranks))

    def allreduce_sum(self, rows):
        tot = np.sum(np.asarray(rows, dtype=np.int64), axis=0)
        return [tot.copy() for _ in rows]

    def allgather_slices(self, ranks):
        S = ranks[0].S
        for dst in ranks:
            for src in ranks:
                dst.vis_full[src.rank * S:(src.rank + 1) * S].copy_(src.own)
        _sync(ranks[0].device)

    def all_to_all(self, ranks, counts, sends):
        import torch
        out = []
        for j in range(self.nranks):
            parts = []
            for i in range(self.nranks):
                off = sum(counts[i][:j])
                parts.append(sends[i][off:off + counts[i][j]])
            out.append(torch.cat(parts) if parts else sends[j][:0])
        _sync(ranks[0].device)
        return out

    def allreduce_max(self, preds):
        import torch
        m = preds[0]
        for p in preds[1:]:
            m = torch.maximum(m, p)
        _sync(m.device)
        return [m for _ in preds]


class TorchComm:
    """One rank per process over torch.distributed (NCCL between GPUs, gloo on CPU)."""

    def __init__(self, dist, device):
        self.dist, self.device = dist, device
        self.nranks = dist.get_world_size()
        self.local_ranks = [dist.get_rank()]

    def allreduce_sum(self, rows):
        import torch
        t = torch.tensor(np.asarray(rows[0], dtype=np.int64), device=self.device)
        self.dist.all_reduce(t)
        return [t.cpu().numpy()]

    def allgather_slices(self, ranks):
        r = ranks[0]
        self.dist.all_gather_into_tensor(r.vis_full, r.own)
        _sync(r.device)

    def all_to_all(self, ranks, counts, sends):
        import torch
        r = ranks[0]
        send_counts = torch.tensor(counts[0], dtype=torch.int64, device=r.device)
        recv_counts = torch.empty_like(send_counts)
        self.dist.all_to_all_single(recv_counts, send_counts)
        rc = [int(x) for x in recv_counts.cpu().tolist()]
        recv = torch.empty(sum(rc), dtype=torch.int64, device=r.device)
        self.dist.all_to_all_single(recv, sends[0].contiguous(), output_split_sizes=rc, input_split_sizes=counts[0])
        _sync(r.device)
        return [recv]

    def allreduce_max(self, preds):
        self.dist.all_reduce(preds[0], op=self.dist.ReduceOp.MAX)
        _sync(preds[0].device)
        return preds


def _sync(device):
    import torch
    if getattr(device, "type", "cpu") == "cuda":
        torch.cuda.synchronize(device)


# ----------------------------------------------------------------------------- the level loop
class PartitionedBFS:
    """run_bfs(root) over the ranks of `comm`; `ranks` are this process's rank
    engines (one per local rank of comm, e.g. CudaRank)."""

    def __init__(self, comm, ranks, num_global_verts: int, alpha: float = 2000.0, beta: float = 8.0):
        if [r.rank for r in ranks] != list(comm.local_ranks):
            raise G500Error(G500_E_INVAL, "the rank engines do not match the communicator's local ranks")
        self.comm, self.ranks = comm, ranks
        self.ngv, self.alpha, self.beta = num_global_verts, alpha, beta
        self.levels = []  # per level of the last run: (top_down, found)

    def run_bfs(self, root: int):
        """The run's pred (combined over the ranks) on every local rank's device."""
        comm, ranks = self.comm, self.ranks
        begun = [r.begin(root) for r in ranks]
        has_edges = begun[0][0]
        comm.allgather_slices(ranks)
        self.levels = []
        if not has_edges:  # the root alone
            preds = [r.new_pred() for r in ranks]
            for p in preds:
                p.fill_(-1)
                p[int(root)] = int(root)
            return preds[0]
        front_edges = [b[2] for b in begun]
        forward, growing = True, True
        prev_nq, visited, level = 0, 1, 0
        while True:
            level += 1
            if level >= MAX_LEVELS:
                raise G500Error(G500_E_INVAL, "BFS deeper than the level field allows")
            if forward:
                counts = [r.top_down(fe) for r, fe in zip(ranks, front_edges)]
                sends = [r.send_pairs(sum(c)) for r, c in zip(ranks, counts)]
                recvs = comm.all_to_all(ranks, counts, sends)
                outs = [r.apply(rv) for r, rv in zip(ranks, recvs)]
            else:
                outs = [r.bottom_up() for r in ranks]
            tot = comm.allreduce_sum([o[:4] for o in outs])[0]
            nq = int(tot[0])
            self.levels.append((forward, nq))
            was_forward = forward
            if nq > 0:
                visited += nq
                unvisited = self.ngv - visited
                # the reference's switch (bfs.hpp:2799-2829)
                if growing and nq > prev_nq:
                    if forward and nq > self.ngv / self.alpha:
                        forward = False
                elif not forward and unvisited < int(self.ngv / self.beta):
                    forward = True
                    growing = False
                prev_nq = nq
                if forward and not was_forward:  # the new frontier lists, before the gather
                    for r in ranks:
                        r.compact()
            comm.allgather_slices(ranks)
            front_edges = [o[1] for o in outs]
            if nq == 0:
                break
        preds = [r.new_pred() for r in ranks]
        for r, p in zip(ranks, preds):
            r.write_pred(p)
        return comm.allreduce_max(preds)[0]

    def close(self):
        for r in self.ranks:
            r.close()
