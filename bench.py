#!/usr/bin/env python
"""Graph500 plain direction-optimizing BFS on B200: harmonic-mean GTEPS.

One step = BFS from every one of the NROOTS find_roots roots (default 64,
REAL_BENCHMARK) of a Kronecker SCALE 22 / edgefactor 16 graph built on the GPU
with VERTEX_REORDERING 2.  Each BFS is timed on the device with CUDA events on
the library's stream, with L2 flushed before every root (outside the event
pair).  value = traversed edges (validate.hpp edge_visit_count) / BFS time,
which for this graph equals the Graph500 harmonic mean (every root reaches the
same component).  e2e = the same through the reference-facing call
run_bfs(root, pred) with pred in pinned HOST memory, the device-to-host copy of
pred inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun) runs N independent replicas (one per GPU); value is the sum
of their edges over the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS (harmonic mean, 1×B200) plain vs batched MS-BFS; serving p50/p99 latency"
UNIT = "GTEPS"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edgefactor", type=int, default=16)
    ap.add_argument("--roots", type=int, default=64)
    ap.add_argument("--reorder", type=int, default=2)
    ap.add_argument("--alpha", type=float, default=None, help="fix alpha (disables the autotuner)")
    ap.add_argument("--beta", type=float, default=None, help="fix beta (disables the autotuner)")
    ap.add_argument("--policy", type=int, default=0, help="direction policy with fixed alpha/beta: 0 reference, 1 edges")
    ap.add_argument("--tune-roots", type=int, default=8, help="roots the autotuner samples (untimed)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-samples", default="22:16:4,24:8:4,26:4:2",
                    help="CPU baselines of the reference beside the GPU sections, SCALE:ROOTS:PASSES each "
                         "(ROOTS validated find_roots roots, timed PASSES times)")
    ap.add_argument("--ref-roots-per-step", type=int, default=None,
                    help="reference arm: roots per step (default: --roots, the GPU arm's step)")
    ap.add_argument("--extra-scales", default="24,26",
                    help="graph sizes measured beside the main one (plain + batched), comma-separated; '' for none")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--partitioned-roots", type=int, default=8,
                    help="N > 1: roots of the partitioned single-root BFS over all ranks (0: none)")
    ap.add_argument("--serve-scales", default="18,20,22,24")
    ap.add_argument("--serve-rates", default="1000,3000,10000,30000,100000")
    ap.add_argument("--serve-queries", type=int, default=10000)
    ap.add_argument("--serve-warmup", type=int, default=1000)
    ap.add_argument("--serve-plain-queries", type=int, default=2000)
    ap.add_argument("--serve-workers", type=int, default=2)
    return ap.parse_args()


def workload(a) -> dict:
    return {"workload": f"plain direction-optimizing BFS, Kronecker SCALE {a.scale} edgefactor {a.edgefactor}, "
                        f"VERTEX_REORDERING {a.reorder}, {a.roots} roots per step",
            "scale": a.scale, "edgefactor": a.edgefactor, "roots_per_step": a.roots,
            "vertex_reordering": a.reorder,
            "l2": "flushed (256 MiB write) before every root, outside the timed events",
            "parallelism": f"replicas x{a.gpus}"}


# --------------------------------------------------------------------------- replicas
class Replicas:
    """The multi-GPU plumbing: one process per GPU, each with its own graph
    and roots (replicas; no collective on the data path).  Only the merge of
    the measurements crosses ranks: times as the max over ranks, edge counts
    as sums, so value = all ranks' edges / the slowest rank's time."""

    def __init__(self, dist=None, device: str = "cuda"):
        self.dist, self.device = dist, device

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if not self.dist:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)

    def gteps(self, edges_rank: float, seconds_rank: float) -> float:
        return self.sum(edges_rank) / self.max(seconds_rank) / 1e9


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None
        self.first = 0

    def _lines(self) -> list:
        with open(self.path) as f:
            return [ln for ln in f.read().split("\n")[:-1] if ln.strip()]  # complete lines only

    def start(self):
        """Start sampling every 50 ms and return once the first sample is in,
        so that the timed region that follows is covered from its start."""
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "50"],
                                     stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        t_end = time.time() + 10.0
        while time.time() < t_end and not self._lines() and self.proc.poll() is None:
            time.sleep(0.01)
        self.first = len(self._lines())

    def stop(self) -> dict | None:
        """The samples taken during the timed region; a region shorter than
        the sampling interval gets the first sample after it instead."""
        if not self.proc:
            return None
        last = len(self._lines())
        t_end = time.time() + 1.0
        while last == self.first and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.01)
            last = len(self._lines())
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in self._lines()[self.first:max(last, self.first + 1)]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "max": float(parts[2]), "active": parts[4],
                             "hw": parts[5], "hwt": parts[6], "swt": parts[7], "pcap": parts[8]})
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for k, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"), ("swt", "sw_thermal_slowdown"),
                            ("pcap", "sw_power_cap")):
                if r[k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in rows), "sm_max_mhz": max(r["max"] for r in rows),
                "samples": len(rows), "sampled": "during the timed region" if last > self.first else
                "first sample after the timed region (shorter than the 50 ms interval)",
                "reasons": sorted(reasons)}


# --------------------------------------------------------------------------- CPU baseline
def ref_exe(reorder: int) -> str:
    return os.path.join(ROOT, "oracle", "_ref", f"ref_bench_vr{reorder}")


def run_ref_bench(scale, ef, nroots, warmup, steps, per_step, reorder):
    exe = ref_exe(reorder)
    if not os.path.exists(exe):
        return None, f"{exe} not built"
    cores = os.cpu_count() or 1
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    env.pop("NO_AFFINITY", None)
    r = subprocess.run([exe, str(scale), str(ef), str(nroots), str(warmup), str(steps), str(per_step)],
                       capture_output=True, text=True, env=env)
    if r.returncode != 0:
        return None, f"ref_bench exit {r.returncode}: {r.stderr.strip().splitlines()[-1:]}"
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    rec["cores"] = cores
    return rec, None


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_ram_gb() -> float:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) / (1 << 20)
    except OSError:
        pass
    return 0.0


class RefBaselines:
    """The reference's own run_bfs (oracle/_ref/ref_bench_vr<N>, OpenMP on all
    host cores) at several graph sizes, for the cpu_baseline of each section.

    Generation, construction and validation take minutes at SCALE 26, so the
    processes start with the bench, one after another at the lowest CPU
    priority, overlapping the GPU work; each stops at its gate once its graph is
    built and its sample roots validated.  The timed runs of each sample happen
    one process at a time after the GPU timing, while nothing else runs."""

    RAM_GB = {22: 8, 24: 24, 26: 80}  # host memory a reference process needs (generation + construction)

    def __init__(self, plan, ef: int, reorder: int):
        self.plan, self.ef, self.reorder = plan, ef, reorder  # [(scale, roots, passes)]
        self.ready, self.err = {}, {}
        self.cores = os.cpu_count() or 1
        self.thread = threading.Thread(target=self._build_all, daemon=True)
        self.thread.start()

    def _build_all(self):
        exe = ref_exe(self.reorder)
        env = dict(os.environ, OMP_NUM_THREADS=str(self.cores))
        env.pop("NO_AFFINITY", None)
        for scale, roots, passes in self.plan:
            if not os.path.exists(exe):
                self.err[scale] = f"{exe} not built"
                continue
            # BfsBase::allocate_memory sizes its comm buffer pool as num_local_verts * 4 * 50 bytes and
            # passes it as an int (mpi/bfs.hpp:173, :283); on one process that overflows from SCALE 25 on
            # (num_local_verts is about half of 2^SCALE), and the allocation fails (utils.hpp:351)
            if (1 << scale) * 0.53 * 200 >= 2 ** 31:
                self.err[scale] = (f"the reference cannot run SCALE {scale} in one process: its comm buffer pool "
                                   f"size, num_local_verts*4*50 bytes (about {(1 << scale) * 0.49 * 200 / 1e9:.1f} "
                                   f"GB), is passed as an int (mpi/bfs.hpp:173, :283) and overflows, so its "
                                   f"allocation fails ('Out of memory trying to allocate', mpi/utils.hpp:351)")
                continue
            need = self.RAM_GB.get(scale, 4 << max(0, scale - 22))
            have = host_ram_gb()
            if have < need:
                self.err[scale] = f"host has {have:.0f} GB available, the reference needs about {need} GB at SCALE {scale}"
                continue
            log = tempfile.TemporaryFile(mode="w+")
            p = subprocess.Popen([exe, str(scale), str(self.ef), str(roots), "0", str(passes), str(roots), "gate"],
                                 stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=log, text=True, env=env,
                                 preexec_fn=lambda: os.nice(19))
            line = p.stdout.readline()
            if line.strip() != "ready":
                p.wait()
                log.seek(0)
                tail = log.read().strip().splitlines()[-3:]
                self.err[scale] = f"ref_bench exit {p.returncode}: {tail}"
                continue
            self.ready[scale] = (p, log, roots, passes)

    def time_all(self) -> dict:
        """Time every built sample in turn; {scale: cpu_baseline dict}."""
        self.thread.join()
        out = {}
        for scale, roots, passes in self.plan:
            if scale not in self.ready:
                out[scale] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                              "sample": f"unavailable: {self.err.get(scale, 'not built')}"}
                continue
            p, log, roots, passes = self.ready.pop(scale)
            stdout, _ = p.communicate("go\n")
            log.close()
            if p.returncode != 0:
                out[scale] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                              "sample": f"unavailable: ref_bench exit {p.returncode}"}
                continue
            rec = json.loads(stdout.strip().splitlines()[-1])
            runs = rec["runs"]
            value = sum(x[3] for x in runs) / sum(x[2] for x in runs) / 1e9
            out[scale] = {"value": value, "unit": UNIT, "cores": self.cores, "kind": "reference",
                          "sample": f"{len(runs)} timed runs ({passes} passes over the first {roots} find_roots "
                                    f"roots, each validated) of the reference run_bfs at SCALE {scale} "
                                    f"(edgefactor {self.ef}, VERTEX_REORDERING {self.reorder}), OMP {self.cores} "
                                    f"threads, {cpu_model()}",
                          "construction_s": rec["construction_s"], "generation_s": rec["generation_s"]}
        return out

    def close(self):
        for p, log, _, _ in self.ready.values():
            p.kill()
            p.wait()
            log.close()
        self.ready.clear()


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    per_step = a.ref_roots_per_step or a.roots
    rec, err = run_ref_bench(a.scale, a.edgefactor, min(a.roots, 64), a.warmup, a.steps, per_step, a.reorder)
    if rec is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return
    runs = rec["runs"]
    t = sum(x[2] for x in runs)
    e = sum(x[3] for x in runs)
    hm = 1.0 / (sum(x[2] / x[3] for x in runs) / len(runs))
    value = e / t / 1e9
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000.0 * t / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int64", "data": "synthetic (Graph500 Kronecker generator, seeds 2/3)",
            "impl": "reference", "config": dict(workload(a), roots_per_step=per_step,
                                                 parallelism="1 process, OpenMP",
                                                 l2="not applicable: the reference runs on the host cores"),
            "harmonic_mean_gteps": hm / 1e9,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": rec["cores"], "kind": "reference",
                             "sample": f"{len(runs)} BFS runs ({per_step} roots/step) of the "
                                       f"reference run_bfs at SCALE {a.scale}, {cpu_model()}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "generation_s": rec["generation_s"], "construction_s": rec["construction_s"]}
    print(json.dumps(line))


# --------------------------------------------------------------------------- our arm
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch(kernel: str, scale: int):
    """DRAM bytes (read + write) of one launch of `kernel` at SCALE `scale`, as
    one ncu capture measured them (profiles/dram_traffic.json, a data file
    written from the capture, with the command that made it), and that
    record's source; (None, None) without a capture of this size."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        d = json.load(open(p))
        rec = d["kernels"][kernel][str(scale)]
        return float(rec["bytes_per_launch"]), rec.get("source", "ncu")
    except (OSError, KeyError, ValueError, TypeError):
        return None, None


def bytes_model(levels, pred_size, nlv):
    """Algorithmic bytes of one BFS: 8 B per pred entry, and per level
    TD: 32 B per frontier vertex (offsets) + 32 B per adjacency sector + 32 B per discovered vertex;
    BU: the visited bitmap (nlv/8 B) + 8 B per scanned vertex + 32 B per adjacency sector."""
    td = bu = 0
    for l in levels:
        if l["direction"] == 1:
            td += 32 * l["frontier"] + 32 * l["edge_sectors"] + 32 * l["discovered"]
        else:
            bu += nlv // 8 + 8 * l["scanned"] + 32 * l["edge_sectors"]
    return 8 * pred_size, td, bu


def batched_arm(a, g5, torch, bfs, roots, nedge, pred_dev, local, reduce_max, reduce_sum, barrier) -> dict:
    peak, peak_kind = load_peaks()
    """MS-BFS over the same roots: autotune (untimed), check every root's levels
    against the plain BFS (untimed), then time K launches of all roots."""
    ms = g5.MultiSourceBFS(bfs.graph_, 64, 15.0, True)
    r = np.asarray(roots, dtype=np.int64)
    tune = ms.autotune(r, reps=1)
    out = torch.empty((len(r), bfs.graph_.pred_size()), dtype=torch.uint8, device="cuda")
    ms.run(r, out)
    for i, root in enumerate(r):
        bfs.run_bfs(int(root), pred_dev)
        lv = ((pred_dev >> 48) & 0xFFFF)
        lv = torch.where(pred_dev == -1, torch.full_like(lv, 255), lv).to(torch.uint8)
        if not torch.equal(lv, out[i]):
            raise SystemExit(f"batched levels differ from the plain BFS for root {root}")
    # bytes model of one launch (untimed counting run, same levels): per level
    # the three mask passes, 8 B per row offset read and 32 B per adjacency
    # sector examined; plus the uint8 level rows written
    info = bfs.graph_.info
    lanes = tune["lane_width"]
    ms.set_count(True)
    ms.run(r[:lanes])
    counted = ms.level_info(0)
    ms.set_count(False)
    mask_bytes = 3 * (lanes // 8) * info.num_local_verts
    level_bytes = [mask_bytes + 8 * l["rows_read"] + 32 * l["sectors"] for l in counted]
    bytes_per_launch = sum(level_bytes) + min(len(r), lanes) * info.pred_size
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(a.warmup):
        ms.run(r)
    t = 0.0
    levels = pulls = 0
    barrier()
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize()
        st = ms.run(r)
        t += st.device_ms
        levels, pulls = st.num_levels, st.pull_levels
    barrier()
    t_max = reduce_max(t / 1000.0)
    e_all = reduce_sum(float(a.steps * sum(nedge)))
    launches = a.steps * ((len(r) + lanes - 1) // lanes)
    ms_per_launch = t / launches
    achieved = bytes_per_launch / (ms_per_launch / 1000.0) / 1e9
    ms.close()
    return {"metric": "aggregate GTEPS of batched multi-source BFS (same graph, same roots)",
            "value": e_all / t_max / 1e9, "unit": UNIT, "roots_per_launch": int(min(len(r), lanes)),
            "roots": int(len(r)), "lane_width": lanes, "alpha": tune["alpha"],
            "ms_per_step": 1000.0 * t_max / a.steps, "levels": levels, "pull_levels": pulls,
            "roofline": {"bound": "hbm", "kernel": "msbfs_kernel", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "bytes_per_launch": bytes_per_launch, "ms_per_launch": ms_per_launch,
                         "bytes_model": "sum over levels of 3 mask passes (lane_width/8 B per vertex each) + "
                                        "8 B per row offset read + 32 B per adjacency sector examined, "
                                        "+ roots x pred_size B of uint8 levels (counted on the device)",
                         "level_bytes": level_bytes,
                         "level_pull": [l["pull"] for l in counted]},
            "output": "uint8 level array per root in original-id order, on the device",
            "parity": "levels of every root equal the plain BFS's (pred >> 48)"}


def scale_section(a, g5, torch, scale, reduce_max, reduce_sum, barrier, peak) -> dict:
    """Plain BFS and batched MS-BFS on another graph size (SCALE 24 is the
    batched configuration, SCALE 26 the plain-at-scale one): 64 roots, every
    root validated on the device (untimed), autotuned plain BFS timed with L2
    flushed before each root, then the MS-BFS launch over the same roots with
    each root's levels checked against the plain run."""
    g = g5.Graph2DCSR.generate(scale, a.edgefactor, a.reorder)
    gen_s, build_s = g.timings()
    info = g.info
    bfs = g5.BfsOnGPU(reorder_mode=a.reorder)
    bfs.graph_ = g
    bfs.prepare_bfs()
    roots = g5.find_roots(g, a.roots)
    tune = bfs.autotune(roots[:a.tune_roots], reps=2)
    pred = torch.empty(info.pred_size, dtype=torch.int64, device="cuda")
    nedge, model = [], []
    bfs.set_params(tune["alpha"], tune["beta"], count_edges=True, policy=tune["policy"])
    for r in roots:
        bfs.run_bfs(int(r), pred)
        ok, evc, rep = g5.validate_bfs_result(g, int(r), pred)
        if not ok:
            raise SystemExit(f"SCALE {scale}: validation failed for root {r}: {rep}")
        nedge.append(evc)
        model.append(sum(bytes_model(bfs.level_stats(), info.pred_size, info.num_local_verts)))
    bfs.set_params(tune["alpha"], tune["beta"], count_edges=False, policy=tune["policy"])
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for r in roots[:8]:
        bfs.run_bfs(int(r), pred)
    barrier()
    ts = []
    for r in roots:
        flush.zero_()
        torch.cuda.synchronize()
        ts.append(bfs.run_bfs(int(r), pred).device_ms)
    barrier()
    t_max = reduce_max(sum(ts) / 1000.0)
    e_all = reduce_sum(float(sum(nedge)))
    plain = e_all / t_max / 1e9
    hm = 1.0 / (sum(t / 1000.0 / e for t, e in zip(ts, nedge)) / len(ts)) / 1e9
    achieved = sum(model) / (sum(ts) / 1000.0) / 1e9
    out = {"workload": f"Kronecker SCALE {scale} edgefactor {a.edgefactor}, VERTEX_REORDERING {a.reorder}, "
                       f"{len(roots)} roots, all validated",
           "plain_gteps": plain, "plain_harmonic_mean_gteps": hm, "plain_ms_per_root": sum(ts) / len(ts),
           "plain_tuning": {k: tune[k] for k in ("policy", "alpha", "beta")},
           "plain_roofline": {"bound": "hbm", "kernel": "bfs_persistent_kernel", "achieved": achieved, "peak": peak,
                              "unit": "GB/s", "frac": achieved / peak,
                              "traffic": traffic_per_launch("bfs_persistent_kernel", scale)[0],
                              "traffic_source": traffic_per_launch("bfs_persistent_kernel", scale)[1],
                              "bytes_per_launch": sum(model) / len(model)},
           "graph": {"num_global_verts": info.num_global_verts, "num_global_edges": info.num_global_edges,
                     "generation_s": gen_s, "construction_s": build_s}}
    bat = batched_arm(a, g5, torch, bfs, roots, nedge, pred, 0, reduce_max, reduce_sum, barrier)
    out["batched"] = {k: bat[k] for k in ("value", "unit", "lane_width", "alpha", "ms_per_step", "levels",
                                          "pull_levels", "roofline", "parity")}
    out["batched"]["speedup_vs_plain"] = bat["value"] / plain if plain else None
    bfs.close()
    del pred, flush
    torch.cuda.empty_cache()
    return out


def partitioned_arm(a, g5, torch, dist, graph, roots, nedge, rank, world) -> dict:
    """One BFS over all ranks (1-D partition, NCCL collectives every level):
    each root validated, then timed by host wall clock between barriers, max
    over ranks."""
    from graph500_b200.partitioned import CudaRank, PartitionedBFS, TorchComm
    dev = torch.device("cuda", torch.cuda.current_device())
    bfs = PartitionedBFS(TorchComm(dist, dev), [CudaRank(graph, rank, world)], graph.info.num_global_verts,
                         2000.0, 8.0)
    rs = [int(r) for r in roots[:a.partitioned_roots]]
    for i, r in enumerate(rs):
        pred = bfs.run_bfs(r)
        ok, evc, rep = g5.validate_bfs_result(graph, r, pred)
        if not ok or evc != nedge[i]:
            raise SystemExit(f"partitioned BFS: root {r} not valid ({rep}, {evc} vs {nedge[i]})")
    ts = []
    for r in rs:
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bfs.run_bfs(r)
        torch.cuda.synchronize()
        t = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ts.append(float(t.item()))
    levels = len(bfs.levels)
    bfs.close()
    return {"workload": f"one BFS per root over {world} ranks (1-D vertex partition, NCCL all-to-all of top-down "
                        f"pairs and all-gather of the bitmap every level), SCALE {a.scale}",
            "value": sum(nedge[:len(rs)]) / sum(ts) / 1e9, "unit": UNIT, "roots": len(rs),
            "ms_per_root": 1000.0 * sum(ts) / len(rs), "levels_last_root": levels,
            "timing": "host wall clock between barriers, max over ranks", "parity": "every root validated"}


def serving_arm(a, g5, torch, reduce_sum, barrier) -> dict:
    """Resident graphs at SCALE 18/20/22/24, open-loop Poisson queries (uniform
    graph, uniform degree>=1 root, splitmix64 seed 2026) at each rate; p50/p99
    of completion - arrival after warm-up, aggregate GTEPS = sum of nedge /
    wall.  Beside it, the same stream through plain per-query BFS."""
    scales = [int(x) for x in a.serve_scales.split(",")]
    graphs = [g5.Graph2DCSR.generate(sc, a.edgefactor, 2) for sc in scales]
    out = {"workload": f"{len(graphs)} resident Kronecker graphs SCALE {'/'.join(map(str, scales))} "
                       f"(edgefactor {a.edgefactor}, VERTEX_REORDERING 2), Poisson arrivals, up to 128 queries "
                       f"per multi-source launch",
           "queries_per_rate": a.serve_queries, "warmup_queries": a.serve_warmup}
    srv = g5.Server(graphs, max_batch=128, max_workers_per_graph=a.serve_workers)
    srv.run_poisson(1000.0, 400, seed=7)  # warm-up: captures the CUDA graphs of every lane width in use
    rates = [float(x) for x in a.serve_rates.split(",")]
    # "rates": each query's levels delivered to a device buffer of its own before it completes;
    # "rates_no_delivery": completion only (levels left in the launch workspace);
    # "rates_host_delivery": levels copied to pinned host memory (PCIe-bound), at the rates PCIe can carry
    out["delivery"] = "device: each query's uint8 level array (pred_size bytes) copied to its own device buffer"
    for key, mode, rs in (("rates", g5.DELIVER_DEVICE, rates), ("rates_no_delivery", g5.DELIVER_NONE, rates),
                          ("rates_host_delivery", g5.DELIVER_HOST, [r for r in rates if r <= 3000])):
        srv.set_delivery(mode)
        out[key] = []
        for rate in rs:
            barrier()
            rep = srv.run_poisson(rate, a.serve_queries + a.serve_warmup, seed=2026, warmup=a.serve_warmup)
            rep["gteps_all_ranks"] = reduce_sum(rep["gteps"])
            out[key].append(rep)
    srv.set_delivery(g5.DELIVER_NONE)
    out["server"] = srv.info()
    srv.close()
    plain = g5.Server(graphs, mode=g5.SERVE_PLAIN)
    plain.run_poisson(1000.0, 200, seed=7)
    out["plain_per_query"] = []
    for rate in [float(x) for x in a.serve_rates.split(",")]:
        barrier()
        rep = plain.run_poisson(rate, a.serve_plain_queries + 100, seed=2026, warmup=100)
        out["plain_per_query"].append(rep)
    plain.close()
    for g in graphs:
        g.close()
    return out


def our_arm(a):
    import torch

    import graph500_b200 as g5

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    rep = Replicas(dist, "cuda")
    barrier, reduce_max, reduce_sum = rep.barrier, rep.max, rep.sum
    # the reference's CPU samples build in the background while the GPU works (rank 0 of one process only)
    ref_base = None
    if world == 1 and not a.no_cpu_baseline:
        sizes = {a.scale} | {int(x) for x in a.extra_scales.split(",") if x}
        plan = []
        for item in a.cpu_samples.split(","):
            if item:
                sc, nr, ps = (int(x) for x in item.split(":"))
                if sc in sizes:
                    plan.append((sc, nr, ps))
        ref_base = RefBaselines(plan, a.edgefactor, a.reorder)

    bfs = g5.BfsOnGPU(device=local, reorder_mode=a.reorder)
    t0 = time.time()
    bfs.construct(g5.EdgeList(None, a.scale, a.edgefactor))
    gen_s, build_s = bfs.graph_.timings()
    info = bfs.graph_.info
    bfs.prepare_bfs()
    roots = g5.find_roots(bfs.graph_, a.roots)
    pred_dev = torch.empty(info.pred_size, dtype=torch.int64, device="cuda")
    if a.alpha is None and a.beta is None:
        tune = bfs.autotune(roots[:a.tune_roots], reps=2)  # untimed; picks policy/alpha/beta
        policy, alpha, beta = tune["policy"], tune["alpha"], tune["beta"]
        tuning = {"autotuned_on_roots": int(min(a.tune_roots, len(roots))), "configs_tried": tune["configs_tried"],
                  "tuned_ms": tune["best_ms"], "reference_setting_ms": tune["reference_ms"]}
    else:
        policy = a.policy
        alpha = 2000.0 if a.alpha is None else a.alpha
        beta = 8.0 if a.beta is None else a.beta
        tuning = {"autotuned_on_roots": 0}
    bfs.set_params(alpha, beta, count_edges=True, policy=policy)

    # untimed: validate every root, record the per-level counts of the bytes model
    nedge, model = [], []
    for r in roots:
        bfs.run_bfs(int(r), pred_dev)
        ok, evc, rep = g5.validate_bfs_result(bfs.graph_, int(r), pred_dev)
        if not ok:
            raise SystemExit(f"validation failed for root {r}: {rep}")
        nedge.append(evc)
        model.append(bytes_model(bfs.level_stats(), info.pred_size, info.num_local_verts))
    bfs.set_params(alpha, beta, count_edges=False, policy=policy)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step(record: dict | None):
        for i, r in enumerate(roots):
            flush.zero_()
            torch.cuda.synchronize()
            st = bfs.run_bfs(int(r), pred_dev)
            if record is not None:
                record["t"].append(st.device_ms)
                record["e"].append(nedge[i])
                record["launches"] += st.kernel_launches
                for l in bfs.level_stats():
                    key = "td" if l["direction"] == 1 else "bu"
                    record[key + "_ms"] += l["device_ms"]
                    record[key + "_launches"] += 1
                pb, tdb, bub = model[i]
                record["td_bytes"] += tdb
                record["bu_bytes"] += bub
                record["pred_bytes"] += pb

    for _ in range(a.warmup):
        step(None)
    rec = {"t": [], "e": [], "launches": 0, "td_ms": 0.0, "bu_ms": 0.0, "td_launches": 0, "bu_launches": 0,
           "td_bytes": 0, "bu_bytes": 0, "pred_bytes": 0}
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    for _ in range(a.steps):
        step(rec)
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    t_rank = sum(rec["t"]) / 1000.0
    t_max = reduce_max(t_rank)
    e_all = reduce_sum(float(sum(rec["e"])))
    value = e_all / t_max / 1e9
    hm = 1.0 / (sum(t / 1000.0 / e for t, e in zip(rec["t"], rec["e"])) / len(rec["t"])) / 1e9

    # e2e: run_bfs into pinned host memory, the D2H copy of pred inside the wall-clock time
    hp = __import__("ctypes").c_void_p()
    g5.check(g5.lib().g500_host_alloc(8 * info.pred_size, __import__("ctypes").byref(hp)))
    host_pred = np.ctypeslib.as_array((__import__("ctypes").c_int64 * info.pred_size).from_address(hp.value))
    for r in roots[:4]:
        bfs.run_bfs(int(r), host_pred)
    barrier()
    e2e_t = e2e_dev = 0.0
    for _ in range(a.steps):
        for r in roots:
            flush.zero_()
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            st = bfs.run_bfs(int(r), host_pred)
            e2e_t += time.perf_counter() - w0
            e2e_dev += st.device_ms / 1000.0
    barrier()
    e2e_max = reduce_max(e2e_t)
    e2e_value = e_all / e2e_max / 1e9
    pred_bytes = 8  # a pinned pred: one DMA copy of the int64 entries
    g5.check(g5.lib().g500_host_free(hp))

    # batched multi-source BFS on the same graph and roots (one launch per 64 roots)
    batched = batched_arm(a, g5, torch, bfs, roots, nedge, pred_dev, local, reduce_max, reduce_sum, barrier)
    partitioned = None
    if world > 1 and a.partitioned_roots > 0:
        partitioned = partitioned_arm(a, g5, torch, dist, bfs.graph_, roots, nedge, rank, world)
    peak, peak_kind = load_peaks()
    sections = {}
    for sc in [int(x) for x in a.extra_scales.split(",") if x]:
        sections[f"scale{sc}"] = scale_section(a, g5, torch, sc, reduce_max, reduce_sum, barrier, peak)
    cpu = ref_base.time_all() if ref_base else {}
    for sc, sec in sections.items():
        if int(sc[5:]) in cpu:
            sec["cpu_baseline"] = cpu[int(sc[5:])]
    serving = None if a.no_serving else serving_arm(a, g5, torch, reduce_sum, barrier)

    if rank != 0:
        bfs.close()
        if dist:
            dist.destroy_process_group()
        return

    # One persistent kernel runs a whole BFS, so it is the dominant kernel:
    # algorithmic bytes of one BFS / its mean device time.
    runs = len(rec["t"])
    bytes_per_bfs = (rec["td_bytes"] + rec["bu_bytes"] + rec["pred_bytes"]) / runs
    ms_per_bfs = sum(rec["t"]) / runs
    achieved = bytes_per_bfs / (ms_per_bfs / 1000.0) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1000.0 * t_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (Graph500 Kronecker generator, seeds 2/3, generated on the GPU)",
        "config": dict(workload(a), direction_policy=["reference", "edges"][policy], alpha=alpha, beta=beta,
                       **tuning),
        "harmonic_mean_gteps": hm,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * len(roots),
                "d2h_bytes_per_step": pred_bytes * info.pred_size * len(roots),
                "path": "g500_bfs_run into a pinned host int64 pred (one DMA copy per root)",
                "ms_per_root": 1000.0 * e2e_t / (a.steps * len(roots)),
                "split_ms_per_root": {"bfs_device": 1000.0 * e2e_dev / (a.steps * len(roots)),
                                      "pred_copy_and_host": 1000.0 * (e2e_t - e2e_dev) / (a.steps * len(roots))},
                "pcie_gbs": pred_bytes * info.pred_size * a.steps * len(roots) / max(e2e_t - e2e_dev, 1e-9) / 1e9},
        "gpu_launches": rec["launches"],
        "roofline": {"bound": "hbm", "kernel": "bfs_persistent_kernel", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic_per_launch("bfs_persistent_kernel", a.scale)[0],
                     "traffic_source": traffic_per_launch("bfs_persistent_kernel", a.scale)[1],
                     "bytes_per_launch": bytes_per_bfs, "ms_per_launch": ms_per_bfs,
                     "bytes_split": {"pred": rec["pred_bytes"] / runs, "top_down": rec["td_bytes"] / runs,
                                     "bottom_up": rec["bu_bytes"] / runs},
                     "level_ms": {"top_down": rec["td_ms"] / runs, "bottom_up": rec["bu_ms"] / runs}},
        "clocks": clocks,
        "graph": {"num_global_verts": info.num_global_verts, "num_global_edges": info.num_global_edges,
                  "pred_size": info.pred_size, "nedge_per_root": int(statistics.median(nedge)),
                  "generation_s": gen_s, "construction_s": build_s, "setup_wall_s": time.time() - t0},
    }
    line["batched"] = batched
    line["batched"]["speedup_vs_plain"] = batched["value"] / value if value else None
    line.update(sections)
    if partitioned is not None:
        line["partitioned"] = partitioned
    if serving is not None:
        line["serving"] = serving
    if a.scale in cpu:
        line["cpu_baseline"] = cpu[a.scale]
    print(json.dumps(line))
    bfs.close()
    if dist:
        dist.destroy_process_group()


def main():
    a = parse_args()
    if a.impl == "reference":
        reference_arm(a)
    else:
        our_arm(a)


if __name__ == "__main__":
    main()
