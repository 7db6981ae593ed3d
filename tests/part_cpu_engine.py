"""A CPU stand-in for one rank's device work of the partitioned BFS (the
g500_part_* steps of graph500_b200/csrc/part.cu), on the oracle's CSR.

TEST INFRASTRUCTURE: it lets the level loop and the collectives of
graph500_b200.partitioned run on CPU ranks (gloo, or in one process) without
a GPU.  Same partition (S bitmap words per rank, the last range padded), same
pair format (target << 32 | parent original id), same counters."""
from __future__ import annotations

import numpy as np
import torch


class CpuRank:
    def __init__(self, og, rank: int, nranks: int):
        self.rank, self.nranks = rank, nranks
        self.off = og.offsets.astype(np.int64)
        self.col = og.cols
        self.invert = og.invert_map
        self.reorder = og.reorder_map
        self.nlv = og.info["num_local_verts"]
        self.nolv = og.info["pred_size"]
        self.nwords = self.nlv // 32
        self.S = -(-self.nwords // nranks)
        self.lo_w = rank * self.S
        deg = self.off[1:] - self.off[:-1]
        has = np.zeros(self.nranks * self.S * 32, bool)
        has[:self.nlv] = deg > 0
        self.vis_init = np.packbits(~has, bitorder="little").view(np.uint32)  # vertices without edges visited
        self.deg = deg
        self.vis_full = torch.zeros(self.nranks * self.S, dtype=torch.int32)
        self.own = torch.zeros(self.S, dtype=torch.int32)
        self.pred_r = np.full(32 * self.S, -1, np.int64)
        self.front = np.zeros(0, np.int64)
        self.next = []
        self.device = torch.device("cpu")
        self.level = 0

    # bit helpers over the int32 tensors' uint32 views
    def _full(self, t):
        return (int(self.vis_full.numpy().view(np.uint32)[t >> 5]) >> (t & 31)) & 1

    def _own_words(self):
        return self.own.numpy().view(np.uint32)

    def _mine(self, t):
        return self.lo_w <= (t >> 5) < self.lo_w + self.S

    def _claim(self, t, parent, lvl, c):
        w = self._own_words()
        lw, bit = (t >> 5) - self.lo_w, np.uint32(1 << (t & 31))
        if w[lw] & bit:
            return
        w[lw] |= bit
        self.pred_r[t - self.lo_w * 32] = parent | lvl
        self.next.append(t)
        c[0] += 1
        c[1] += int(self.deg[t])
        c[2] += 1

    def begin(self, root):
        r = int(self.reorder[root])
        has = r < self.nlv and self.deg[r] > 0
        w = self._own_words()
        for i in range(self.S):
            gw = self.lo_w + i
            w[i] = self.vis_init[gw] if gw < self.nwords else np.uint32(0xFFFFFFFF)
        self.level = 0
        self.front = np.zeros(0, np.int64)
        mf = 0
        if has and self._mine(r):
            w[(r >> 5) - self.lo_w] |= np.uint32(1 << (r & 31))
            self.pred_r[r - self.lo_w * 32] = int(root)
            self.front = np.array([r], np.int64)
            mf = int(self.deg[r])
        return [1 if has else 0, len(self.front), mf]

    def top_down(self, frontier_edges):
        self.level += 1
        lvl = self.level << 48
        self.next, self.c = [], [0, 0, 0, 0]
        buckets = [[] for _ in range(self.nranks)]
        for u in self.front.tolist():
            parent = int(self.invert[u])
            for t in self.col[self.off[u]:self.off[u + 1]].tolist():
                if self._mine(t):
                    self._claim(t, parent, lvl, self.c)
                elif not self._full(t):
                    buckets[(t >> 5) // self.S].append((t << 32) | parent)
        self.send = torch.tensor(sum(buckets, []), dtype=torch.int64)
        return [len(b) for b in buckets]

    def send_pairs(self, total):
        return self.send

    def apply(self, recv):
        lvl = self.level << 48
        for x in recv.tolist():
            x &= (1 << 64) - 1
            self._claim(x >> 32, x & 0xFFFFFFFF, lvl, self.c)
        self.front = np.array(self.next, np.int64)
        return list(self.c)

    def bottom_up(self):
        self.level += 1
        lvl = self.level << 48
        c = [0, 0, 0, 0]
        full = self.vis_full.numpy().view(np.uint32)
        own = self._own_words()
        for i in range(self.S):
            gw = self.lo_w + i
            if gw >= self.nwords:
                break
            vw = int(full[gw])
            for b in range(32):
                if (vw >> b) & 1:
                    continue
                v = gw * 32 + b
                c[3] += 1
                for n in self.col[self.off[v]:self.off[v + 1]].tolist():
                    if (int(full[n >> 5]) >> (n & 31)) & 1:
                        own[i] |= np.uint32(1 << b)
                        self.pred_r[v - self.lo_w * 32] = int(self.invert[n]) | lvl
                        c[0] += 1
                        c[1] += int(self.deg[v])
                        break
        self.front = np.zeros(0, np.int64)
        return c

    def compact(self):
        full = self.vis_full.numpy().view(np.uint32)
        own = self._own_words()
        fr = []
        for i in range(self.S):
            gw = self.lo_w + i
            if gw >= self.nwords:
                continue
            f = int(own[i]) & ~int(full[gw])
            fr += [gw * 32 + b for b in range(32) if (f >> b) & 1]
        self.front = np.array(fr, np.int64)
        return len(fr)

    def new_pred(self):
        return torch.empty(self.nolv, dtype=torch.int64)

    def write_pred(self, pred):
        full = self.vis_full.numpy().view(np.uint32)
        out = pred.numpy()
        out[:] = -1
        for u in range(self.nolv):
            r = int(self.reorder[u])
            if r < self.nlv and self._mine(r):
                reached = ((int(full[r >> 5]) & ~int(self.vis_init[r >> 5])) >> (r & 31)) & 1
                if reached:
                    out[u] = self.pred_r[r - self.lo_w * 32]

    def close(self):
        pass
