#!/usr/bin/env python
"""Throughput of GASAL2's batched alignment path on B200 (aligned pairs/s).

Default workload (w4, the full mixed production batch): 10,000,000 pairs,
query lengths log-normal (median 250 bp, sigma 0.8, clipped to 50-5000),
60% short-read-like, 30% long-read-like (5-12% errors, indel-dominated), 10%
unrelated; four launches on four streams -- LOCAL WITH_START 30%, LOCAL
WITH_TB 20%, SEMI_GLOBAL (TARGET, TARGET) WITH_START 25%, ksw z-drop 100 25%
-- scores 1/4/6/1.  Seeded synthetic data (per-pair xoshiro256** streams,
seed 20261203+4); the inputs (~7 GB) exceed the 126 MB L2, so no flush is
needed between steps.  Other workloads: --workload w0..w3.

One step = every launch of the workload, each on its own stream.  Reported:
  value      pairs/s with the batch already in HBM (pack -> reverse/complement
             -> length-binned order -> DP -> start pass / traceback), CUDA
             events on the timing stream, max over ranks
  e2e        pairs/s through the GASAL2 storage API (gasal_c_aln_async +
             gasal_c_is_aln_async_done, one storage per launch): host->device
             copy of the pinned batch, kernels, device->host copy of every
             result array
  plain      the plain full-DP form (every pair one per thread, in input
             order, no band) against the batched form on the same stratified
             sample, outputs compared bit for bit
  band       the ksw launch's computed cells; with --band compare (default)
             the same step timed again with the learned band installed
             (band.learned_leg: pairs/s, ratio to the unbanded step, ksw
             outputs compared bit for bit, certificate acceptance,
             recomputations, computed cells); --band learned makes the
             banded step the headline
  roofline   algorithmic integer ops of every alignment kernel of a step /
             the step's wall clock, against this GPU's measured integer-add
             issue rate; pack and reverse/complement in GB/s against the
             measured HBM copy bandwidth
  cpu_baseline  the scalar C oracle, OpenMP on all host cores, on a
             stratified subsample; its outputs are also compared with the GPU
             run's outputs for those pairs (oracle_check)

--impl reference times the reference GASAL2 kernels compiled for the host
(OpenMP over pairs) on a bounded stratified sample per step; the reference
has no CPU aligner of its own and cannot run on this GPU's box as a library
install (it has no packaging).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from gasal_b200 import workloads as W  # noqa: E402
from gasal_b200.capi import LOCAL, GLOBAL, SEMI_GLOBAL, KSW, WITH_TB, Params, has_cigar  # noqa: E402

UNIT = "pairs/s"
# integer ops per computed cell, per algorithm (+4 with traceback)
OPS_PER_CELL = {LOCAL: 11, GLOBAL: 9, SEMI_GLOBAL: 10, KSW: 13}
TB_OPS = 4
HEADLINE_METRIC = "aligned pairs/s + GCUPS, 1 B200: learned-band vs plain full DP, bit-exact"

# name -> (metric, config description, default pairs, generator id, launch params, launch shares)
WORKLOADS = {
    "w4": (HEADLINE_METRIC,
           "w4 full mixed production batch: 10M pairs/GPU, query lengths log-normal (median 250, sigma 0.8, "
           "clipped 50-5000), 60% short-read-like (1-2% subs, 0.2% indels), 30% long-read-like (5-12% errors, "
           "75% indels of 1-5 bp), 10% unrelated; LOCAL WITH_START 30%, LOCAL WITH_TB 20%, "
           "SEMI_GLOBAL(TARGET,TARGET) WITH_START 25%, ksw (h0 20-60, z-drop 100) 25%; four launches on four "
           "streams; scores 1/4/6/1", 10_000_000, 4, W.WORKLOAD4_PARAMS, W.WORKLOAD4_SHARES),
    "w1": ("aligned pairs/s (1M-pair mixed LOCAL/GLOBAL/SEMI_GLOBAL WITH_START batch, RC on 50%)",
           "w1: 1M pairs/GPU, thirds LOCAL(second best)/GLOBAL/SEMI_GLOBAL(TARGET,TARGET), WITH_START, q=150, "
           "t=150-300 (3% subs, 1% indels), RC 50% of queries, scores 1/4/6/1", 1_000_000, 1,
           W.WORKLOAD1_PARAMS, (1 / 3, 1 / 3, 1 / 3)),
    "w2": ("aligned pairs/s (2M-pair uneven-length GLOBAL WITH_TB batch, CIGAR out)",
           "w2: 2M pairs/GPU, GLOBAL WITH_TB, query log-uniform 50-1000, target = query with 1-8% subs and "
           "0.5-3% indels (len 1-10) per pair, scores 1/4/6/1", 2_000_000, 2,
           [Params(algo=GLOBAL, start_pos=WITH_TB)], (1.0,)),
    "w3": ("aligned pairs/s (ksw seed extension, z-drop 100, query 250-2000 bp)",
           "w3: 4M pairs/GPU, ksw extension, query U[250,2000], target = query with indel rate {0.5,2,5,10}% "
           "(len 1-3) + 1-5% subs per pair, h0 U[20,60], zdrop 100, scores 1/4/6/1; three launches on three "
           "streams (a GASAL2 batch holds at most 4 GiB of bases per side)", 4_000_000, 3,
           [Params(algo=KSW, zdrop=100)] * 3, (1 / 3, 1 / 3, 1 / 3)),
    "w0": ("aligned pairs/s (20k-pair LOCAL WITHOUT_START batch)",
           "w0: 20k pairs, LOCAL WITHOUT_START, q 100-150 with 0.1% N, t = q + 0-20 flanks, 2% subs, 0.5% "
           "indels", 20_000, 0, [Params(algo=LOCAL)], (1.0,)),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi clock / throttle sampling (50 ms) around the timed region;
    the summary keeps the samples taken between mark_start and mark_end."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), [x.strip() for x in line.split(",")]))

    def mark_start(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(0.12)  # let the sample covering the end arrive

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = [r for t, r in self.rows if self.t0 is None or (self.t0 - 0.06 <= t <= (self.t1 or t) + 0.06)]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        num = lambda x: x.replace(".", "").isdigit()
        sm = [float(r[1]) for r in rows if num(r[1])]
        mx = [float(r[2]) for r in rows if num(r[2])]
        pw = [float(r[3]) for r in rows if num(r[3])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(pw) if pw else None, "reasons": reasons, "samples": len(rows)}


def build_parts(name: str, n: int, seed: int, idx=None):
    """[(Params, Batch)] of workload `name` -- pairs [0, n), or the pairs
    listed in idx (ascending workload indexes) -- one entry per launch."""
    _, _, _, gen, params, shares = WORKLOADS[name]
    cuts = W._cuts(n, shares)
    if idx is None:
        batches = W.generate(gen, n, seed, cuts)
    else:
        idx = np.asarray(idx, dtype=np.int64)
        sub_cuts = [int(np.searchsorted(idx, c)) for c in cuts]
        batches = W.generate(gen, 0, seed, sub_cuts, idx=idx)
    return [(p, b) for p, b in zip(params, batches)]


def stratified(n: int, every: int) -> np.ndarray:
    """Every `every`-th pair of [0, n): the workload's pairs are i.i.d. in
    index order, so this is a uniform sample of each launch's pairs."""
    return np.arange(0, n, max(1, int(every)), dtype=np.int64)


def local_index(name: str, n: int, idx: np.ndarray):
    """For each launch: positions of workload indexes idx inside that launch."""
    cuts = W._cuts(n, WORKLOADS[name][5])
    out = []
    for lo, hi in zip(cuts[:-1], cuts[1:]):
        sel = idx[(idx >= lo) & (idx < hi)]
        out.append(sel - lo)
    return out


def alg_ops(parts) -> float:
    return float(sum(b.cells() * (OPS_PER_CELL[p.algo] + (TB_OPS if p.start_pos == WITH_TB else 0))
                     for p, b in parts))


# ------------------------------------------------------------------------------------------------------------
# reference arm
# ------------------------------------------------------------------------------------------------------------

def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.bindings import ref_host_align
    cores = os.cpu_count() or 1
    n = args.pairs or WORKLOADS[args.workload][2]
    every = max(1, n // args.ref_sample)
    idx = stratified(n, every)
    sample = build_parts(args.workload, n, W.SEED_BASE + WORKLOADS[args.workload][3], idx)
    chunk = 256  # bounds the reference's traceback tile buffer (longest pair's tiles x pairs per batch)

    chunks = [(p, [b.subset(np.arange(lo, min(b.n, lo + chunk))) for lo in range(0, b.n, chunk)]
               if p.start_pos == WITH_TB and b.n > chunk else [b]) for p, b in sample]

    def step():
        for p, cs in chunks:
            for c in cs:
                ref_host_align(p, c, threads=cores)

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.time()
        step()
        times.append(time.time() - t0)
    npairs = sum(b.n for _, b in sample)
    v = npairs / float(np.mean(times))
    line = {"impl": "reference", "metric": WORKLOADS[args.workload][0], "value": v, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (per-pair xoshiro256** streams)",
            "config": {"workload": WORKLOADS[args.workload][1], "pairs_per_step": npairs},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"every {every}th pair of the {n}-pair workload ({npairs} pairs per step, "
                                       f"traceback launches in chunks of {chunk}); the reference kernel headers compiled for the host "
                                       f"(MAX_QUERY_LEN 8192), OpenMP over pairs; ksw at the reference's "
                                       f"hard-coded z-drop 0"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------------------
# device-resident batches
# ------------------------------------------------------------------------------------------------------------

OUTS = ("score", "q_end", "t_end", "q_start", "t_start", "score2", "q_end2", "t_end2")


class DevPart:
    """One launch's batch in device memory plus its output buffers, with the
    gb_dev_batch_t / gb_dev_out_t address map."""

    def __init__(self, torch, p: Params, b, dev):
        def t_(a, dtype=None):
            return torch.from_numpy(np.ascontiguousarray(a).view(dtype or a.dtype)).to(dev)
        self.p, self.b = p, b
        self.t = {"q": t_(b.q), "t": t_(b.t), "qo": t_(b.q_off, np.int32), "to": t_(b.t_off, np.int32),
                  "ql": t_(b.q_len, np.int32), "tl": t_(b.t_len, np.int32)}
        if b.q_op is not None:
            self.t["qop"], self.t["top"] = t_(b.q_op), t_(b.t_op)
        if b.seed is not None:
            self.t["seed"] = t_(b.seed, np.int32)
        self.t["pq"] = torch.empty(b.q.shape[0] // 8, dtype=torch.int32, device=dev)
        self.t["pt"] = torch.empty(b.t.shape[0] // 8, dtype=torch.int32, device=dev)
        self.outs = {k: torch.empty(b.n, dtype=torch.int32, device=dev) for k in OUTS}
        self.cigar = torch.empty(b.q.shape[0], dtype=torch.uint8, device=dev)
        self.ncig = torch.empty(b.n, dtype=torch.int32, device=dev)
        m = {"q_bytes": b.q.shape[0], "t_bytes": b.t.shape[0]}
        for k, src in (("q", "q"), ("t", "t"), ("pq", "pq"), ("pt", "pt"), ("q_off", "qo"), ("t_off", "to"),
                       ("q_len", "ql"), ("t_len", "tl"), ("q_op", "qop"), ("t_op", "top"), ("seed", "seed")):
            m[k] = self.t[src].data_ptr() if src in self.t else None
        for k, v in self.outs.items():
            m["out_" + k] = v.data_ptr()
        if not p.second_best:
            m["out_score2"] = m["out_q_end2"] = m["out_t_end2"] = None
        m["out_cigar"] = self.cigar.data_ptr()
        m["out_n_cigar"] = self.ncig.data_ptr()
        self.map = m

    def fields(self):
        """Output arrays defined for this launch's options (name -> tensor)."""
        from gasal_b200.capi import Outputs
        names = Outputs.fields_for(None, self.p)
        d = {k: self.outs[k] for k in names}
        if has_cigar(self.p):
            d["n_cigar"] = self.ncig
        return d

    def cigar_of(self, i: int):
        o, n = int(self.b.q_off[i]), int(self.ncig[i].item())
        return self.cigar[o:o + n]


class Runner:
    """Launches every part on its own stream, joined into one timing stream."""

    def __init__(self, torch, gl, parts, dev, tb_priority=False, serial=False):
        self.torch, self.gl, self.parts, self.dev = torch, gl, parts, dev
        self.serial = serial  # every launch on the timing stream, one after another
        self.main = torch.cuda.Stream(device=dev)
        # optionally (tb_priority) a WITH_TB launch, which runs its traceback chunks one after another and
        # finishes last, gets the highest stream priority (the library gives its auxiliary stream the same)
        self.streams = [torch.cuda.Stream(device=dev, priority=-5 if tb_priority and d.p.start_pos == WITH_TB else 0)
                        for d in parts]

    def step(self, finish_times=False):
        torch = self.torch
        fork = torch.cuda.Event(enable_timing=finish_times)
        fork.record(self.main)
        dones = []
        for d, s in zip(self.parts, self.streams):
            if self.serial:
                s = self.main
            else:
                s.wait_event(fork)
            self.gl.align_dev(d.p, d.map, d.b.q_len, d.b.t_len, s.cuda_stream)
            done = torch.cuda.Event(enable_timing=finish_times)
            done.record(s)
            self.main.wait_event(done)
            dones.append(done)
        if finish_times:
            self.finish = (fork, dones)

    def launch_finish_ms(self):
        """Per launch, ms from the last timed step's start to that launch's
        end (the launches of a step run concurrently on their streams)."""
        fork, dones = self.finish
        return [fork.elapsed_time(e) for e in dones]

    def time(self, steps: int, warmup: int, dist=None, before_timed=None):
        torch = self.torch
        for _ in range(warmup):
            self.step()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        if before_timed:
            before_timed()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.main)
        for k in range(steps):
            self.step(finish_times=k == steps - 1)
        e1.record(self.main)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)


def outputs_equal(torch, a_parts, b_parts, a_idx=None):
    """Every defined output of b_parts equals a_parts' (at rows a_idx[k] of
    a_parts[k] when given); returns (equal, mismatched pair count)."""
    bad = 0
    for k, (a, b) in enumerate(zip(a_parts, b_parts)):
        sel = None if a_idx is None else torch.from_numpy(a_idx[k]).to(a.outs["score"].device)
        for name, tb_ in b.fields().items():
            ta = a.fields()[name]
            if sel is not None:
                ta = ta.index_select(0, sel)
            bad += int((ta != tb_).sum().item())
        if has_cigar(b.p):
            ia = None if a_idx is None else a_idx[k]
            nb = b.ncig.cpu().numpy()
            na = a.ncig.cpu().numpy() if ia is None else a.ncig.cpu().numpy()[ia]
            ca, cb = a.cigar.cpu().numpy(), b.cigar.cpu().numpy()
            for j in range(b.b.n):
                i = j if ia is None else int(ia[j])
                oa, ob = int(a.b.q_off[i]), int(b.b.q_off[j])
                if na[j] != nb[j] or not np.array_equal(ca[oa:oa + int(na[j])], cb[ob:ob + int(nb[j])]):
                    bad += 1
    return bad == 0, bad


# ------------------------------------------------------------------------------------------------------------
# the measured arm
# ------------------------------------------------------------------------------------------------------------

def train_band(torch, gl, args, rank, dev):
    """Train the ksw band model on a separate sample of the same workload
    (its ksw launch) and install it for every ksw call."""
    from gasal_b200 import band_train as BT
    t0 = time.time()
    name = args.workload
    shares = WORKLOADS[name][5]
    ksw_k = [p.algo for p in WORKLOADS[name][4]].index(KSW)
    n_train = int(args.band_train_pairs / shares[ksw_k])
    tparts = build_parts(name, n_train, W.SEED_BASE + 101 + 1000 * rank)
    tp, tb = tparts[ksw_k]
    tdb = BT.DeviceBatch(torch, tb, dev)
    feat = BT.features(torch, tdb)
    if args.band_labels == "max_off":
        lab, _ = BT.labels_max_off(torch, tp, tdb)
    else:
        lab = BT.labels(torch, tp, tdb)
    model = gl.BandModel(seed=11)
    trace = BT.train(torch, model, feat, lab, steps=600, batch=8192, tau=0.8, lr=3e-3)
    model.install(16, 1024)
    info = {"train_pairs": tb.n, "train_s": round(time.time() - t0, 1), "labels": args.band_labels,
            "label_hist_log2": {f"{k:.2f}": int(v) for k, v in zip(*np.unique(np.round(lab * 4) / 4,
                                                                                 return_counts=True))},
            "loss_first": trace[0], "loss_last": trace[-1]}
    log(f"band model trained in {info['train_s']} s; loss {trace[0]:.3f} -> {trace[-1]:.3f}")
    return model, info


def learned_band_leg(torch, gl, args, rank, dev, runner, kpart, dist, unbanded_value, job_pairs):
    """The headline step again with the learned band installed for the ksw
    launch (trained first, untimed): its throughput against the unbanded
    headline, its ksw outputs against the unbanded run's (bit-exact), and the
    certificate's statistics over the launch."""
    from gasal_b200 import shard
    ref = {k: v.clone() for k, v in kpart.fields().items()}
    model, info = train_band(torch, gl, args, rank, dev)
    try:
        ms = shard.max_over_ranks(runner.time(args.steps, args.warmup, dist), dist, dev)
        same = all(bool(torch.equal(v, ref[k])) for k, v in kpart.fields().items())
        with torch.cuda.stream(runner.main):
            st = gl.ksw_band_align(kpart.p, kpart.map, kpart.b.q_len, kpart.b.t_len, None, None,
                                   runner.main.cuda_stream)
    finally:
        gl.BandModel.uninstall()
        model.close()
    value = job_pairs * args.steps / (ms * 1e-3)
    return dict(info, value=value, unit=UNIT, ms_per_step=ms / args.steps, steps=args.steps,
                value_over_unbanded=value / unbanded_value, bit_exact_vs_unbanded=same, **st,
                acceptance_rate=st["accepted"] / max(1, st["pairs"]),
                computed_cells_fraction=st["cells"] / max(1, kpart.b.cells()))


def prep_bandwidth(torch, gl, dparts, hbm_gbs, reps=20):
    """Pack and reverse/complement kernels alone on the resident batch, each
    leg captured once as a CUDA graph of every launch's calls and replayed
    `reps` times between CUDA events on its stream (so host launch overhead is
    not timed; every step re-packs, so running them here changes nothing
    later).  Algorithmic bytes: pack 1.5 B per base (1 read, 0.5 written),
    reverse/complement 1 B per base of sequences with an operation (0.5 read,
    0.5 written)."""
    s = torch.cuda.Stream(device=dparts[0].outs["score"].device)
    out = {}

    def timed(calls, nbytes, launches):
        with torch.cuda.stream(s):
            calls()  # warm-up outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            calls()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(s):
            g.replay()
            e0.record(s)
            for _ in range(reps):
                g.replay()
            e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        gbs = nbytes / (ms * 1e-3) / 1e9
        del g
        return {"gbs": gbs, "frac_of_hbm": gbs / hbm_gbs, "ms_per_step": ms, "bytes_per_step": nbytes,
                "launches_per_step": launches, "timing": f"CUDA graph of the step's launches, {reps} replays"}

    def pack_all():
        for d in dparts:
            gl.pack_dev(d.map["q"], d.b.q.shape[0], d.map["pq"], torch.cuda.current_stream().cuda_stream)
            gl.pack_dev(d.map["t"], d.b.t.shape[0], d.map["pt"], torch.cuda.current_stream().cuda_stream)

    pack_bytes = sum(1.5 * (d.b.q.shape[0] + d.b.t.shape[0]) for d in dparts)
    out["pack"] = timed(pack_all, pack_bytes, 2 * len(dparts))
    rc = [d for d in dparts if d.b.q_op is not None and (d.b.q_op != 0).any()]
    if rc:
        rc_bytes = sum(float(np.sum(d.b.q_len[d.b.q_op != 0])) + float(np.sum(d.b.t_len[d.b.t_op != 0]))
                       for d in rc)

        def rc_all():
            for d in rc:
                gl.revcomp_dev(d.map, d.b.n, torch.cuda.current_stream().cuda_stream)

        out["revcomp"] = timed(rc_all, rc_bytes, len(rc))
    return out


def mixed_leg(torch, gl, parts, dparts, dev, args, dist, job_pairs, value):
    """The same step through the per-pair mixed dispatch: the workload's
    launches as ONE batch whose pairs each name their kind (interleaved at
    random), one gb_align_dev_mixed call per step, inputs resident; every
    output compared with the per-launch step's."""
    from gasal_b200 import shard
    kinds, b, kind, idx = W.concat_parts(parts, shuffle_seed=11)
    qb = np.cumsum([0] + [int(pb.q.shape[0]) for _, pb in parts])
    d = DevPart(torch, kinds[0], b, dev)
    for k in ("score2", "q_end2", "t_end2"):
        d.map["out_" + k] = d.outs[k].data_ptr()
    stream = torch.cuda.Stream(device=dev)
    host_ms = []

    def step():
        h0 = time.perf_counter()
        gl.align_dev_mixed(kinds, kind, d.map, b.q_len, b.t_len, stream.cuda_stream)
        host_ms.append((time.perf_counter() - h0) * 1e3)

    warm, steps = 2, max(1, min(args.steps, 3))
    for _ in range(warm):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = shard.max_over_ranks(e0.elapsed_time(e1), dist, dev)
    same = True
    for k, kp in enumerate(dparts):
        rows = torch.from_numpy(np.nonzero(kind == k)[0]).to(dev)
        src = torch.from_numpy(idx[kind == k]).to(dev)
        for f, t in kp.fields().items():
            mine = d.ncig if f == "n_cigar" else d.outs[f]
            same &= bool(torch.equal(mine[rows], t[src]))
        if has_cigar(kp.p):
            lens = kp.ncig.cpu().numpy().astype(np.int64)
            starts = kp.b.q_off.astype(np.int64)
            pos = np.repeat(starts, lens) + (np.arange(int(lens.sum())) - np.repeat(np.cumsum(lens) - lens, lens))
            pos_t = torch.from_numpy(pos).to(dev)
            same &= bool(torch.equal(kp.cigar[pos_t], d.cigar[pos_t + int(qb[k])]))
    del d
    torch.cuda.empty_cache()
    v = job_pairs * steps / (ms * 1e-3)
    return {"value": v, "unit": UNIT, "ms_per_step": ms / steps, "steps": steps, "warmup": warm,
            "value_over_per_launch": v / value, "bit_exact_vs_per_launch": same,
            "host_ms_per_call": float(np.median(host_ms)),
            "host_ms_note": "wall time of the call on the host, including its waits for buffers the previous "
                            "call's work still reads (the per-launch calls wait the same way)",
            "kinds": [p.key() for p in kinds],
            "path": "gb_align_dev_mixed: one call per step over one batch of every launch's pairs, kind per pair "
                    "(seeded random interleave); packed once, each kind on a forked stream, results scattered "
                    "back per pair"}


def e2e_leg(torch, gl, parts, args, dev, dist, job_pairs):
    """The storage API with host buffers: per step, every launch's pinned batch
    goes host->device, aligns, and every result array comes back."""
    from gasal_b200 import shard
    streams = []
    for p, b in parts:
        s = gl.Streams(1, -(-int(b.q.shape[0]) // b.n) + 8, -(-int(b.t.shape[0]) // b.n) + 8, b.n, p)
        streams.append((p, b, s))
    h2d = d2h = 0
    for p, b, _ in streams:
        h2d += int(b.q.shape[0] + b.t.shape[0]) + b.n * (4 * 4 + 2) + (4 * b.n if p.algo == KSW else 0)
        nf = 1 if p.algo == GLOBAL else (3 if p.algo == KSW else 5 + (3 if p.second_best else 0))
        d2h += 4 * b.n * nf
        if p.start_pos == WITH_TB:
            d2h += int(b.q.shape[0]) + 4 * b.n
    times = []
    ext = [torch.cuda.ExternalStream(s.view(0).stream, device=dev) for _, _, s in streams]
    n_timed = min(args.steps, args.e2e_steps)
    gs0 = None
    for it in range(args.warmup + n_timed):
        if it == args.warmup:
            gs0 = gl.graph_stats()
        # stage every storage's pinned pages before the timed region: gasal_is_aln_async_done resets a
        # storage's host pages when its batch completes (as the reference's does), so each step refills
        sizes = [s.fill_bulk(0, b) for _, b, s in streams]
        torch.cuda.synchronize()
        starts = [torch.cuda.Event(enable_timing=True) for _ in streams]
        ends = [torch.cuda.Event(enable_timing=True) for _ in streams]
        for k, ((p, b, s), (qi, ti)) in enumerate(zip(streams, sizes)):
            starts[k].record(ext[k])
            s.aln_async(0, qi, ti, b.n)
            ends[k].record(ext[k])
        for _, _, s in streams:
            s.wait(0)
        torch.cuda.synchronize()
        if it >= args.warmup:
            times.append(max(starts[0].elapsed_time(e) for e in ends))
    # the same with the host staging inside the timed region: every step refills each storage's pinned
    # pages from the caller's buffers (gasal_host_batch_fill_mt, all host threads) just before its
    # gasal_aln_async, so the fills of later storages overlap the GPU work of earlier ones
    gs1 = gl.graph_stats()
    ftimes, fill_s = [], []
    seq_bytes = sum(int(b.q.shape[0] + b.t.shape[0]) for _, b, _ in streams)
    for it in range(1 + n_timed):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in streams]
        e0.record(ext[0])
        fs = 0.0
        for k, (p, b, s) in enumerate(streams):
            t0 = time.perf_counter()
            qi, ti = s.fill_bulk(0, b)
            fs += time.perf_counter() - t0
            s.aln_async(0, qi, ti, b.n)
            ends[k].record(ext[k])
        for _, _, s in streams:
            s.wait(0)
        torch.cuda.synchronize()
        if it >= 1:
            ftimes.append(max(e0.elapsed_time(e) for e in ends))
            fill_s.append(fs)
    gs2 = gl.graph_stats()
    for _, _, s in streams:
        s.close()
    ms = shard.max_over_ranks(float(np.mean(times)), dist, dev)
    fms = shard.max_over_ranks(float(np.mean(ftimes)), dist, dev)
    fill_ms = float(np.mean(fill_s)) * 1e3
    return {"value": job_pairs / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms, "steps": n_timed,
            "path": f"gasal_c_aln_async + gasal_c_is_aln_async_done, one storage per launch ({len(parts)} streams), "
                    f"pinned host batches refilled (gasal_host_batch_fill_mt) before each step's timed region",
            "graphs_timed_steps": {k: gs1[k] - gs0[k] for k in gs1},
            "with_fill": {"value": job_pairs / (fms * 1e-3), "unit": UNIT, "ms_per_step": fms, "steps": n_timed,
                          "host_fill_ms_per_step": fill_ms, "host_fill_gbs": seq_bytes / (fill_ms * 1e-3) / 1e9,
                          "sequence_bytes_per_step": seq_bytes,
                          "graphs": {k: gs2[k] - gs1[k] for k in gs2},
                          "path": "per step and storage: gasal_host_batch_fill_mt of the query and target blocks "
                                  "(all host threads) + offsets/lengths/ops/seeds, then gasal_c_aln_async; later "
                                  "storages' fills overlap earlier storages' GPU work"}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="w4", choices=sorted(WORKLOADS))
    ap.add_argument("--pairs", type=int, default=0, help="pairs per GPU (default: the workload's size)")
    ap.add_argument("--ref-sample", type=int, default=4000, help="pairs per step of the reference arm")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-budget-s", type=float, default=12.0)
    ap.add_argument("--band", default="compare", choices=["off", "learned", "compare"],
                    help="ksw launches: off (unbanded), learned (the headline step runs with the learned band and "
                         "its certificate; the model is trained first on a separate sample of the workload), or "
                         "compare (headline unbanded, then the same step timed again with the learned band "
                         "installed, outputs compared)")
    ap.add_argument("--band-train-pairs", type=int, default=60_000)
    ap.add_argument("--band-labels", default="ladder", choices=["ladder", "max_off"],
                    help="band labels: the narrowest ladder band the certificate keeps, or log2(max_off + 16) "
                         "from the plain ksw's own maximum diagonal offset")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain full-DP form (one pair per thread, input order, no band)")
    ap.add_argument("--plain-budget-s", type=float, default=20.0,
                    help="device time the plain form's timed step may take; beyond it a stratified sample is used")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--serial", action="store_true",
                    help="kernel-level step: the launches one after another on one stream instead of concurrently")
    ap.add_argument("--tb-priority", default="off", choices=["on", "off"],
                    help="kernel-level step: run WITH_TB launches on the highest-priority stream (measured slower "
                         "on w4: the prioritised launch finishes early and the others then run on alone)")
    ap.add_argument("--mixed", default="on", choices=["on", "off"],
                    help="workloads of several launches: time the same step again as one per-pair mixed-dispatch "
                         "call (gb_align_dev_mixed) and compare its outputs with the per-launch step's")
    ap.add_argument("--split", default="weak", choices=["weak", "cells"],
                    help="N>1: weak = every rank aligns its own full-size seeded shard; cells = the ranks split one "
                         "workload into contiguous slices of equal DP cells (strong scaling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    from gasal_b200 import lib as gl
    from gasal_b200 import shard
    rank, world, local_rank = shard.rank_info()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    gl.lib()
    gl.set_reference_reverse(True)
    peak = gl.probe_int_peak()
    hbm = None
    try:
        hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        hbm_src = "MEASURED_PEAKS.json hbm_gbs (STREAM-style copy on this pool's B200s)"
    except (OSError, KeyError, ValueError):
        hbm, hbm_src = 6650.0, "fallback 6.65 TB/s (earlier measurement on this pool)"
    name = args.workload
    n_pairs = args.pairs or WORKLOADS[name][2]
    strong = args.split == "cells" and world > 1
    seed = W.SEED_BASE + WORKLOADS[name][3] if strong else shard.shard_seed(W.SEED_BASE + WORKLOADS[name][3], rank)
    t0 = time.time()
    if strong:
        all_cells = W.pair_cells(WORKLOADS[name][3], n_pairs, seed)
        lo, hi = shard.cell_shard_range(all_cells, rank, world)
        parts = build_parts(name, n_pairs, seed, np.arange(lo, hi, dtype=np.int64))
    else:
        parts = build_parts(name, n_pairs, seed)
    log(f"workload {name}: {n_pairs} pairs generated in {time.time() - t0:.1f}s "
        f"({W.generator_threads()} threads)")
    npairs = sum(b.n for _, b in parts)
    cells = sum(b.cells() for _, b in parts)
    if strong:
        args.no_plain = True  # the plain-form and oracle comparisons index the whole workload, not a slice
    job_pairs = n_pairs if strong else npairs * world  # pairs the whole job aligns per step
    job_cells = float(all_cells.sum()) if strong else float(cells) * world
    dev = torch.device("cuda", local_rank)
    dparts = [DevPart(torch, p, b, dev) for p, b in parts]

    model, band_info = None, None
    has_ksw = any(p.algo == KSW for p, _ in parts)
    if args.band == "learned" and has_ksw:
        model, band_info = train_band(torch, gl, args, rank, dev)

    # ---------------- kernel level: inputs resident in HBM -----------------
    runner = Runner(torch, gl, dparts, dev, tb_priority=args.tb_priority == "on", serial=args.serial)
    clk = ClockSampler(local_rank).__enter__()

    def arm():
        gl.kernel_timing(True)
        clk.mark_start()

    ms = runner.time(args.steps, args.warmup, dist, before_timed=arm)
    finish_ms = runner.launch_finish_ms()
    clk.mark_end()
    clk.__exit__()
    kt = gl.kernel_timing_read()
    gl.kernel_timing(False)
    ms = shard.max_over_ranks(ms, dist, dev)
    ms_step = ms / args.steps
    value = job_pairs * args.steps / (ms * 1e-3)
    ops = alg_ops(parts)
    achieved = ops / (ms_step * 1e-3) / 1e12
    launches = sum(n * gl.KERNELS_PER_MARK[k] for k, (_, n) in kt.items())

    prep = prep_bandwidth(torch, gl, dparts, hbm)

    # ---------------- the same step through the per-pair mixed dispatch ----------------
    mixed = None
    if len(parts) > 1 and args.mixed == "on":
        # each leg starts from the library's per-stream buffers released: the traceback tile budget is
        # at most half the free device memory, so tiles still held by an earlier leg would shrink it
        gl.release_workspaces()
        mixed = mixed_leg(torch, gl, parts, dparts, dev, args, dist, job_pairs, value)
        gl.release_workspaces()

    kpart = next((d for d in dparts if d.p.algo == KSW), None)
    if kpart is not None:
        # band statistics of one more (untimed) pass over the ksw launch: with the installed model, or,
        # without one, a band wider than every matrix (the unbanded computation's cells)
        wide = None
        if model is None:
            wide = torch.full((kpart.b.n,), 1 << 20, dtype=torch.int32, device=dev)
        with torch.cuda.stream(runner.main):
            st = gl.ksw_band_align(kpart.p, kpart.map, kpart.b.q_len, kpart.b.t_len,
                                   None if wide is None else wide.data_ptr(), None, runner.main.cuda_stream)
        band_info = dict(band_info or {}, mode=args.band, **st,
                         acceptance_rate=st["accepted"] / max(1, st["pairs"]),
                         computed_cells_fraction=st["cells"] / max(1, kpart.b.cells()))
        del wide

    if args.band == "compare" and kpart is not None:
        band_info["learned_leg"] = learned_band_leg(torch, gl, args, rank, dev, runner, kpart, dist, value,
                                                    job_pairs)

    # ---------------- end to end through the storage API ----------------
    gl.release_workspaces()
    e2e = e2e_leg(torch, gl, parts, args, dev, dist, job_pairs)

    # ---------------- the plain full-DP form on a stratified sample ----------------
    plain = None
    if not args.no_plain:
        plain = plain_leg(torch, gl, args, name, n_pairs, seed, dparts, model, dev, dist, value, world)

    in_mb = sum(int(b.q.shape[0] + b.t.shape[0]) + 16 * b.n for _, b in parts) / 1e6
    l2_note = (f"inputs {in_mb:.0f} MB > 126 MB L2, no flush" if in_mb > 126 else
               f"inputs {in_mb:.0f} MB fit the 126 MB L2 (no flush: each step re-reads them, as a caller "
               f"re-aligning resident batches would)")
    if rank == 0:
        cpu = None if args.no_cpu_baseline else cpu_baseline(name, n_pairs, seed, None if strong else dparts,
                                                             args.cpu_budget_s)
        computed = None
        if band_info is not None and kpart is not None:
            computed = cells - kpart.b.cells() + band_info["cells"]
        line = {
            "metric": WORKLOADS[name][0], "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong" if strong else "weak",
            "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded per-pair xoshiro256** streams, splitmix64-seeded)",
            "config": {"workload": WORKLOADS[name][1],
                       "pairs_per_step_per_gpu": npairs, "cells_per_step_per_gpu": cells,
                       "launches": [p.key() for p, _ in parts],
                       "band": ({"compare": "off (the learned band timed as a second leg, band.learned_leg)"}
                                .get(args.band, args.band) if has_ksw else None),
                       "parallelism": (f"one workload split into {world} contiguous slices of equal DP cells, no "
                                       f"collective in the data path" if strong else
                                       f"pair shards x{world} (a full-size seeded shard per rank), no collective "
                                       f"in the data path"),
                       "l2": l2_note,
                       "stream_priority": "WITH_TB launches on the highest-priority stream" if args.tb_priority == "on"
                                          else "all launches on default-priority streams",
                       "launch_streams": "one stream, launches in sequence" if args.serial else
                                         "one stream per launch, concurrent"},
            "gcups": job_cells / (ms_step * 1e-3) / 1e9,
            "gcups_computed": None if computed is None else computed * (job_cells / cells) / (ms_step * 1e-3) / 1e9,
            "roofline": {"bound": "int32", "achieved": achieved, "peak": peak["iadd_tops"], "unit": "Tops/s",
                         "frac": achieved / peak["iadd_tops"], "traffic": None,
                         "traffic_note": "no per-run DRAM counter; see the ncu summaries of the alignment kernels",
                         "kernel": "every alignment kernel of the step (DP, start passes, traceback; four launches "
                                   "on four streams): algorithmic integer ops / the step's wall clock",
                         "ops_per_step": ops,
                         "ops_per_cell": {"local": 11, "global": 9, "semi_global": 10, "ksw": 13,
                                          "traceback_extra": 4},
                         "peak_source": "measured live: 2-input int32 add issue rate (gb_probe_int_peak)",
                         "imnmx_tops": peak["imnmx_tops"], "dpx_tops": peak["dpx_tops"],
                         "dpx16x2_halfword_tops": peak["dpx16x2_halfword_tops"],
                         "align_span_ms_per_step": kt["span"][0] / args.steps},
            "prep_bandwidth": dict(prep, peak_gbs=hbm, peak_source=hbm_src),
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kt.items()},
            "launch_finish_ms": {p.key(): round(t, 2) for (p, _), t in zip(parts, finish_ms)},
            "launch_finish_note": "last timed step: ms from its start until each launch (own stream) finished; "
                                  "the gap between the last two is the time one launch ran alone",
            "kernel_ms_note": "summed per-kind CUDA-event times; kinds overlap across the four streams",
            "gpu_launches": launches,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clk.summary(),
            "band": band_info,
            "plain": plain,
            "mixed": mixed,
        }
        print(json.dumps(line), flush=True)
    if model is not None:
        gl.BandModel.uninstall()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def plain_leg(torch, gl, args, name, n_pairs, seed, dparts, model, dev, dist, value, world):
    """Batched vs plain full-DP form on one stratified sample of the
    workload, each timed over one step after a warm-up step, outputs compared
    with each other and with the full run's outputs for the same pairs."""
    from gasal_b200 import shard
    # size the sample from the plain form's rate on a 0.5% probe sample
    probe_every = 200
    pidx = stratified(n_pairs, probe_every)
    probe = [DevPart(torch, p, b, dev) for p, b in build_parts(name, n_pairs, seed, pidx)]
    saved = gl.get_tuning()
    if model is not None:
        gl.BandModel.uninstall()
    gl.set_tuning(**gl.PLAIN_FORM)
    try:
        r = Runner(torch, gl, probe, dev)
        probe_ms = r.time(1, 1)
    finally:
        gl.set_tuning(**saved)
        if model is not None:
            model.install(16, 1024)
    est_full_s = probe_ms * 1e-3 * probe_every
    every = 1 if est_full_s <= args.plain_budget_s else int(np.ceil(est_full_s / args.plain_budget_s))
    if every == 1:
        sample = dparts
        sidx = None
    else:
        sidx = stratified(n_pairs, every)
        sample = [DevPart(torch, p, b, dev) for p, b in build_parts(name, n_pairs, seed, sidx)]
    npairs = sum(d.b.n for d in sample)
    cells = sum(d.b.cells() for d in sample)
    rb = Runner(torch, gl, sample, dev)
    bms = shard.max_over_ranks(rb.time(1, 1), dist, dev)
    batched_out = [{k: v.clone() for k, v in d.fields().items()} for d in sample]
    batched_cig = [(d.cigar.clone(), d.ncig.clone()) for d in sample]
    if model is not None:
        gl.BandModel.uninstall()
    gl.set_tuning(**gl.PLAIN_FORM)
    try:
        rp = Runner(torch, gl, sample, dev)
        pms = shard.max_over_ranks(rp.time(1, 1), dist, dev)
    finally:
        gl.set_tuning(**saved)
        if model is not None:
            model.install(16, 1024)
    same = True
    for d, bo, (bc, bn) in zip(sample, batched_out, batched_cig):
        for k, v in d.fields().items():
            same &= bool(torch.equal(v, bo[k]))
        if d.p.start_pos == WITH_TB:
            same &= bool(torch.equal(d.cigar, bc)) and bool(torch.equal(d.ncig, bn))
    # the full run's outputs for the sampled pairs
    full_same = None
    if sidx is not None:
        lidx = local_index(name, n_pairs, sidx)
        # outputs of the sample currently hold the plain run's, equal to the batched sample run's when `same`
        full_same, bad = outputs_equal(torch, dparts, sample, lidx)
    pval = shard.job_throughput(npairs, world, 1, pms)
    bval = shard.job_throughput(npairs, world, 1, bms)
    return {"value": pval, "unit": UNIT, "ms_per_step": pms, "steps": 1, "warmup": 1,
            "sample": "full batch" if sidx is None else
                      f"stratified: every {every}th pair of the {n_pairs}-pair workload ({npairs} pairs, all "
                      f"launches); the plain form on the full batch would take ~{est_full_s:.0f} s",
            "gcups": cells * world / (pms * 1e-3) / 1e9,
            "form": "every pair one per thread in input order on a grid over the batch: no device work counter, "
                    "no length ordering, no warp-cooperative or warp-per-pair kernels, no band, start passes in "
                    "the forward launch",
            "batched_same_sample": {"value": bval, "ms_per_step": bms},
            "value_over_plain": bval / pval,
            "full_value_over_plain_sample_rate": value / pval,
            "bit_exact_vs_plain": bool(same),
            "full_run_equals_sample_run": full_same}


def cpu_baseline(name, n_pairs, seed, dparts, budget_s: float) -> dict:
    """Scalar C oracle, OpenMP on every host core, on a stratified subsample
    sized to about budget_s of CPU time; its outputs are compared with the GPU
    run's outputs for the same pairs."""
    from oracle.bindings import oracle_align
    cores = os.cpu_count() or 1
    probe_every = max(1, n_pairs // 3000)
    pidx = stratified(n_pairs, probe_every)
    probe = build_parts(name, n_pairs, seed, pidx)
    t0 = time.time()
    for p, b in probe:
        oracle_align(p, b, threads=cores)
    per_pair = (time.time() - t0) / max(1, len(pidx))
    m = int(min(n_pairs, max(len(pidx), budget_s / max(per_pair, 1e-9))))
    every = max(1, n_pairs // m)
    sidx = stratified(n_pairs, every)
    sample = build_parts(name, n_pairs, seed, sidx)
    t0 = time.time()
    outs = [oracle_align(p, b, threads=cores) for p, b in sample]
    dt = time.time() - t0
    n = len(sidx)
    line = {"value": n / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"stratified: every {every}th pair of the {n_pairs}-pair workload ({n} pairs, "
                      f"{100.0 * n / n_pairs:.2f}%), {dt:.1f} s"}
    if dparts is None:
        return line
    # parity of the full GPU run on these pairs
    lidx = local_index(name, n_pairs, sidx)
    bad = 0
    for (p, b), o, d, li in zip(sample, outs, dparts, lidx):
        exp = o.as_dict(p)
        for k, v in exp.items():
            if k == "cigar":
                cg = d.cigar.cpu().numpy()
                for j, i in enumerate(li):
                    oe, og = int(b.q_off[j]), int(d.b.q_off[i])
                    nc = int(exp["n_cigar"][j])
                    if not np.array_equal(v[oe:oe + nc], cg[og:og + nc]):
                        bad += 1
                continue
            got = (d.ncig if k == "n_cigar" else d.outs[k]).cpu().numpy()[li]
            bad += int((got.astype(np.int64) != v.astype(np.int64)).sum())
    line["oracle_check"] = {"pairs": n, "mismatched_values": bad,
                            "what": "every defined output (and CIGAR bytes) of the full GPU run at these pairs vs "
                                    "the oracle's"}
    return line


if __name__ == "__main__":
    main()
