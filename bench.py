#!/usr/bin/env python
"""Benchmark of the batched ConSGA alignment engine (libchsga) on one B200.

Workload (the batched-engine configuration): the config-2 variant-bubble DAG
(5 Mbp random ACGT backbone, a bubble every ~50 bp: 70% SNP, 20% 1-20 bp
indel, 10% 50-300 bp alternative allele; string vertices of 1-32 chars) and
reads with lengths log-uniform in [150, 10000] at 5% error (60% indels, 40%
substitutions), all generated with fixed seeds (synthetic stand-ins; the
reference ships no datasets). A step aligns one batch of --batch reads to
completion through the slot-interleaved engine (score-only, int32).

  value   GCUPS over the K timed steps: sum(read_len * num_chars) / device
          time (CUDA events around the device sequence, reads resident)
  e2e     batched + served: the same K batches streamed through the serving
          loop (chsga_server_submit / _poll with host buffers: reads copied
          in, scores copied out, continuous batching across batches, longest
          waiting read admitted first), cells / wall time from the first
          submit to the last result
  served  a Poisson arrival stream at ~80% of that capacity (80% 150 bp at
          1% error, 20% log-uniform 1-10 kbp at 5%): p50/p99 latency from
          submission to result, and the cost model's per-read time error
          against the analytic |V| x |read| model on those logs
The score rows of one step (slots x 25.5 MB per row buffer) exceed the 126 MB
L2, so no flush is needed between steps.

--impl reference times the reference's own CPU code (src/align.hpp's
align_combo compiled in oracle/_ref) on the host cores for the same workload,
one bounded sample of reads per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GCUPS on 1 B200 (batched+served vs plain per-read GPU), p50/p99 read latency"
WORKLOAD = ("config-2 graph (5 Mbp backbone, bubble every ~50 bp) with reads log-uniform "
            "150-10000 bp at 5% ONT-like error (the batched-engine configuration)")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="chsga", choices=["chsga", "reference"])
    p.add_argument("--batch", type=int, default=512, help="reads per step")
    p.add_argument("--slots", type=int, default=128)
    p.add_argument("--warmup-batch", type=int, default=128,
                   help="reads per warm-up step (lengths capped at 1 kbp)")
    p.add_argument("--no-profile", action="store_true")
    p.add_argument("--no-tune", action="store_true", help="skip the autotuner (use --slots)")
    p.add_argument("--row-kernel", default="auto", choices=["auto", "direct", "tiled", "dpx", "stream", "delta"],
                   help="with --no-tune: the row kernel")
    p.add_argument("--served-s", type=float, default=12.0, help="Poisson arrival window, seconds")
    p.add_argument("--backbone", type=int, default=0,
                   help="backbone length of the config-2-mix graph (0 = 5 Mbp); for small profiling captures")
    p.add_argument("--scale-cfg4", action="store_true",
                   help="config-4 run instead of the contract line: the 100 Mbp graph, "
                        "checkpointed tracebacks (-k 500) and batched score-only GCUPS")
    p.add_argument("--cfg4-reads", type=int, default=4,
                   help="with --scale-cfg4: how many 10 kbp reads to trace back")
    p.add_argument("--cfg5", action="store_true",
                   help="config-5 run instead of the contract line: the cost model trained on logs of "
                        "runs on the config-2 and config-4 graphs, then a Poisson stream of score and "
                        "traceback requests on the config-4 graph admitted by its footprint")
    p.add_argument("--cfg5-window-s", type=float, default=30.0, help="with --cfg5: arrival window")
    p.add_argument("--traceback-cfg1", action="store_true",
                   help="config-1 run instead of the contract line: tracebacks of 2,000 x 150 bp and "
                        "200 x 2 kbp reads with full score matrices, batched and one by one")
    p.add_argument("--tb-sample", type=int, default=0,
                   help="with --traceback-cfg1: that many 150 bp reads and a tenth as many 2 kbp ones")
    p.add_argument("--kernels-only", action="store_true",
                   help="time the batched steps only (no server, served run, plain sample, profiled "
                        "pass or CPU baseline): the command profiling captures run under ncu")
    p.add_argument("--launch-compare", action="store_true",
                   help="launch-mode comparison instead of the contract line: the same reads at 1, 8 "
                        "and 128 slots as CUDA-graph chains and as persistent launches, device time, "
                        "scores compared")
    p.add_argument("--shapes", default="1,8,128", help="with --launch-compare: slot counts to compare")
    p.add_argument("--top-compare", action="store_true",
                   help="device time per row-step for several top-region sizes at 1-128 slots, one JSON line")
    p.add_argument("--cpu-sample-s", type=float, default=15.0)
    p.add_argument("--plain-reads", type=int, default=64,
                   help="reads of the first timed batch (drawn at random) run through the plain path")
    return p.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9
                          for i in range(4) if r[5 + i].strip().lower() == "active"})
        load = [s for s in sm if mx and s > 0.3 * max(mx)] or sm
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def make_graph(backbone=0):
    import chsga_b200 as cb
    cfg = dict(cb.GRAPH_CONFIGS["cfg2"])
    if backbone:
        cfg["backbone_len"] = backbone
    g = cb.HostGraph.generate(**cfg)
    g.build_pch()
    return g


def make_reads(g, n, seed, len_max=10000):
    # 5% error, 60% indels / 40% substitutions
    return g.gen_reads(n, seed, 150, len_max, sub_rate=0.02, indel_rate=0.03, n_rate=0.0,
                       indel_len_max=3).to_list()


def algorithmic_row_bytes(st, slots, multi, score_bytes):
    """Bytes one row-kernel launch must move, with w = bytes per stored
    score: the previous and the new score of every char for every slot
    (2 w N R), the first/last boundary scores of every vertex written for
    the sweeps (w R (S + S_multi)), the previous row's final first score of
    every vertex and final last score of every first-char in-edge source
    (w R (S + E_first)), 2-bit labels plus the special-char map (3N/8), three
    words per vertex (offset, hierarchy position, in-edge offset: 12 S) and
    one word per first-char in-edge (4 E_first)."""
    N, S = st["num_chars"], st["num_strings"]
    e_first = st["num_char_edges"] - (N - S)
    w = score_bytes
    return (2 * w * N * slots + w * slots * (S + multi) + w * slots * (S + e_first)
            + 3 * N / 8 + 12 * S + 4 * e_first)


def algorithmic_delta_row_bytes(st, slots, multi):
    """Bytes one k_row_delta launch must move (128 slots, 2-bit delta rows):
    the previous and the new row's per-char deltas (2 bits per slot each,
    N R / 4 bytes per row), the previous and the new raw first score of every
    vertex (2 R S bytes each), and the boundary, in-edge and graph terms of
    algorithmic_row_bytes."""
    N, S = st["num_chars"], st["num_strings"]
    e_first = st["num_char_edges"] - (N - S)
    w = 2
    return (2 * N * slots / 4 + 2 * w * slots * S + w * slots * (S + multi) + w * slots * (S + e_first)
            + 3 * N / 8 + 12 * S + 4 * e_first)


def algorithmic_sweep_bytes(st, lay, slots, score_bytes, fl_first=True):
    """Bytes per row-step of the grid-wide sweep kernels below the top
    region (16-byte pull-list heads and vertex words, w bytes per score):
    up (k_pull_lv, k_pull_lv16): per target its head, first score read and written, one
    gathered score per edge, 8 bytes per edge after the first;
    down (k_down, k_down16): per position its vertex words, first score read,
    raw last score read (vertices of two or more chars), final first (unless
    fl_first is false: with delta rows the row kernel reads it from BV) and
    last written to FL; per target below the top its head, first score
    written, one gathered score per edge, 8 bytes per edge after the first."""
    S = st["num_strings"]
    wr = score_bytes * slots
    ut, ue = lay["sweep_up_targets"], lay["sweep_up_edges"]
    dt, de = lay["sweep_down_targets"], lay["sweep_down_edges"]
    up = ut * (16 + 2 * wr) + ue * wr + (ue - ut) * 8
    down = (S * (16 + (4 if fl_first else 3) * wr) - st["single_char_strings"] * wr + dt * (16 + wr) + de * wr
            + (de - dt) * 8)
    return up, down


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kname="k_row_stream"):
    """The ncu DRAM bytes of one row-kernel launch, scaled to the bench graph
    (profiles/k_row_traffic.json for k_row_stream, k_row_delta_traffic.json
    for k_row_delta)."""
    name = {"k_row_stream": "k_row_traffic.json", "k_row_delta": "k_row_delta_traffic.json"}.get(kname)
    if name is None:
        return None
    p = os.path.join(ROOT, "profiles", name)
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def host_threads():
    """Host threads this process may run on (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_harness(oracle, files):
    """The reference's own code (oracle/_ref) or, without it, the oracle, on
    every host thread of this process (set explicitly: a launcher such as
    torchrun sets OMP_NUM_THREADS=1); returns (harness, kind, threads used)."""
    n = host_threads()
    if oracle.ref_available():
        h, kind = oracle.RefHarness(files, threads=n), "reference"
        used = h.lib.ref_set_threads(0)
    else:
        h, kind = oracle.Oracle(files, threads=n), "port"
        used = h.lib.oracle_set_threads(0)
    return h, kind, int(used)


def cpu_baseline(g, reads, budget_s):
    """The reference's own align_combo (oracle/_ref) on the host cores, on a
    bounded sample of the workload's reads (shortest first, until about
    budget_s seconds of CPU work). Returns the baseline record, the indices
    of the sampled reads in `reads` and the reference's scores for them."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    st = g.stats()
    N = st["num_chars"]
    with tempfile.TemporaryDirectory() as d:
        files = g.write_files(os.path.join(d, "g"))
        h, kind, cores = cpu_harness(oracle, files)
        order = sorted(range(len(reads)), key=lambda i: len(reads[i]))
        # calibrate on one short read, then size the sample to the budget
        t = time.time()
        h.scores([reads[order[0]]])
        per_cell = (time.time() - t) / (len(reads[order[0]]) * N)
        picked, est = [], 0.0
        for i in order:
            c = per_cell * len(reads[i]) * N
            if picked and est + c > budget_s:
                break
            picked.append(i)
            est += c
        t = time.time()
        ref_scores = h.scores([reads[i] for i in picked])
        dt = time.time() - t
    bases = sum(len(reads[i]) for i in picked)
    cells = bases * N
    what = ("reference code (src/align.hpp align_combo, compiled unchanged) on a project-written "
            "OpenMP stand-in for parlaylib's scheduler" if kind == "reference" else
            "the CPU restatement of align_combo (oracle), OpenMP")
    info = {"value": cells / dt / 1e9, "unit": "GCUPS", "cores": cores, "kind": kind, "what": what,
            "sample": f"{len(picked)} reads ({bases} bases) of the first timed batch, shortest first, "
                      f"{dt:.1f} s on {cores} host threads"}
    return info, picked, ref_scores


def served_mix(g, n, seed):
    """80% 150 bp at 1% error, 20% log-uniform 1-10 kbp at 5% error."""
    import numpy as np
    rng = np.random.default_rng(seed)
    longs = int(round(0.2 * n))
    short = g.gen_reads(n - longs, seed, 150, 150, sub_rate=0.006, indel_rate=0.003,
                        n_rate=0.001).to_list()
    lng = make_reads(g, 3 * longs, seed + 1, len_max=10000) if longs else []
    lng = [r for r in lng if len(r) >= 1000][:longs] or lng[:longs]
    out = short + lng
    rng.shuffle(out)
    return out


def served_run(cb, ctx, g, N, opts, capacity_gcups, window_s):
    """Poisson arrivals at ~80% of the measured served capacity for window_s
    seconds; latency = result time - submit time (host clock)."""
    import numpy as np
    reads = served_mix(g, 4096, 4242)
    mean_len = float(np.mean([len(r) for r in reads]))
    rate = 0.8 * capacity_gcups * 1e9 / (mean_len * N)  # reads per second
    n = max(32, min(len(reads), int(rate * window_s)))
    reads = reads[:n]
    rng = np.random.default_rng(7)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    srv = cb.Server(ctx, slots=opts["slots"], steps_per_graph=opts["steps_per_graph"],
                    queue_capacity=4096, arena_bytes=64 << 20, tb_workers=1)
    res = {}
    tickets = [None] * n

    def producer():
        t0 = time.perf_counter()
        for i, (r, at) in enumerate(zip(reads, arrivals)):
            d = at - (time.perf_counter() - t0)
            if d > 0:
                time.sleep(d)
            tickets[i] = srv.submit(r)

    th = threading.Thread(target=producer)
    th.start()
    while th.is_alive() or len(res) < n:
        for d in srv.poll(1024, 50):
            res[d["ticket"]] = d
    th.join()
    st = srv.stats()
    srv.close()
    lat = np.array([(res[t]["done_ns"] - res[t]["submit_ns"]) / 1e6 for t in tickets])
    lens = np.array([len(r) for r in reads])
    short = lens <= 150
    # cost model: trained on the first half of the served logs (per-read
    # device time, and the slot share of the engine's buffers), tested on
    # the second half against the analytic |V| x |read| model
    feats = np.array([cb.cm_features(ctx, int(L), cb.REQ_SCORE, opts["slots"]) for L in lens])
    t_ms = np.array([max(1e-3, (res[t]["done_ns"] - res[t]["start_ns"]) / 1e6) for t in tickets])
    y = np.stack([t_ms, 4.0 * (N + 32) + lens], 1)
    half = n // 2
    m = cb.CostModel(0, seed=1)
    m.train(feats[:half], y[:half], epochs=1000, batch=min(64, half), lr=2e-3, seed=2)
    pred = m.predict(feats[half:])[:, 0]
    m.close()
    cells = lens * float(N)
    a = np.exp(np.mean(np.log(t_ms[:half] / cells[:half])))
    ana = a * cells[half:]
    return {
        "arrivals": "Poisson", "reads": n, "rate_reads_per_s": rate, "load": 0.8,
        "mix": "80% 150 bp @1% error, 20% log-uniform 1-10 kbp @5% error",
        "gcups": st["gcups"], "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "short_p50_ms": float(np.percentile(lat[short], 50)) if short.any() else None,
        "short_p99_ms": float(np.percentile(lat[short], 99)) if short.any() else None,
        "cost_model": {"train_reads": half, "test_reads": n - half,
                       "mean_abs_log_err_time": float(np.mean(np.abs(np.log(pred / t_ms[half:])))),
                       "analytic_mean_abs_log_err_time": float(np.mean(np.abs(np.log(ana / t_ms[half:]))))},
    }


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    g = make_graph(args.backbone)
    st = g.stats()
    N = st["num_chars"]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    with tempfile.TemporaryDirectory() as d:
        files = g.write_files(os.path.join(d, "g"))
        h, kind, cores = cpu_harness(oracle, files)
        # each step: the shortest reads of that step's batch until ~budget seconds
        budget = max(2.0, min(20.0, args.cpu_sample_s))
        t = time.time()
        probe = sorted(make_reads(g, 8, 999), key=len)[0]
        h.scores([probe])
        per_cell = (time.time() - t) / (len(probe) * N)
        samples = []
        for s in range(args.warmup + args.steps):
            reads = sorted(make_reads(g, 64, 1000 + s), key=len)
            pick, est = [], 0.0
            for r in reads:
                c = per_cell * len(r) * N
                if pick and est + c > budget:
                    break
                pick.append(r)
                est += c
            samples.append(pick)
        for s in range(args.warmup):
            h.scores(samples[s])
        cells, tt = 0, 0.0
        for s in range(args.warmup, args.warmup + args.steps):
            t = time.time()
            h.scores(samples[s])
            tt += time.time() - t
            cells += sum(len(r) for r in samples[s]) * N
    v = cells / tt / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GCUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": tt * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "num_chars": N, "batch": "bounded CPU sample per step"},
        "cpu_baseline": {"value": v, "unit": "GCUPS", "cores": cores, "kind": kind,
                         "what": ("reference code (src/align.hpp align_combo, compiled unchanged) on a "
                                  "project-written OpenMP stand-in for parlaylib's scheduler"
                                  if kind == "reference" else "the CPU restatement of align_combo"),
                         "sample": f"per step the shortest reads of a 64-read batch (shortest first) "
                                   f"up to ~{budget:.0f} s of CPU work, {cores} host threads"},
        "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_scale_cfg4(args):
    """Config 4: the 100 Mbp graph (about 139 M chars; one int32 row is
    0.56 GB, so a full 10 kbp matrix would take 5.6 TB) with -k 500.
      byte-compare  a 1001-base read: the checkpoint files row_0.bin,
                    row_500.bin and row_1000.bin the GPU writes against the
                    same rows from the reference's own row functions
                    (oracle/_ref, two rows held at a time)
      tracebacks    --cfg4-reads reads of 10 kbp at 5% error, each
                    checkpointed (16-bit rows; a 501-row recompute segment is
                    139 GB and fits the device in one level), each path
                    rescored against the score-only result; GCUPS over the
                    forward cells (recompute not counted)
      batched       score-only GCUPS with 128 slots
    Prints one JSON line."""
    import numpy as np

    import chsga_b200 as cb
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    t0 = time.time()
    g = cb.HostGraph.generate(**cb.GRAPH_CONFIGS["cfg4"])
    g.build_pch()
    st = g.stats()
    N = st["num_chars"]
    prep_s = time.time() - t0
    ctx = cb.Context(0).load(g)
    labels = ctypes_labels(g)
    out = {"mode": "scale-cfg4", "num_chars": N, "num_strings": st["num_strings"],
           "hierarchy_levels": st["pch_levels"], "graph_prep_s": prep_s}
    # checkpoint rows against the reference
    r1 = g.gen_reads(1, 43, 1001, 1001, sub_rate=0.02, indel_rate=0.03, indel_len_max=3).to_list()[0]
    with tempfile.TemporaryDirectory() as d:
        ck = os.path.join(d, "ck")
        t = time.perf_counter()
        ops, score, ckp = ctx.align_traceback(r1, k=500, ckpt_dir=ck, keep_files=True)
        gpu_s = time.perf_counter() - t
        cmp = {"read_len": len(r1), "k": 500, "gpu_seconds": gpu_s, "checkpointed": ckp,
               "score": score, "rescored": list(path_score(ops, r1, labels))}
        if oracle.ref_available():
            files = g.write_files(os.path.join(d, "g"))
            h, kind, cores = cpu_harness(oracle, files)
            t = time.time()
            rows = h.rows_at(r1, N, [0, 500, 1000]) if kind == "reference" else None
            cmp["reference_seconds"] = time.time() - t
            cmp["reference_threads"] = cores
            if rows is not None:
                same = []
                for j, i in enumerate((0, 500, 1000)):
                    got = np.fromfile(os.path.join(ck, f"row_{i}.bin"), dtype=np.int32)
                    same.append(bool(got.shape == rows[j].shape and np.array_equal(got, rows[j])))
                cmp["rows"] = [0, 500, 1000]
                cmp["byte_identical"] = same
        else:
            cmp["byte_identical"] = "reference build absent"
        out["checkpoint_compare"] = cmp
    # checkpointed tracebacks of 10 kbp reads
    reads = g.gen_reads(args.cfg4_reads, 44, 10000, 10000, sub_rate=0.02, indel_rate=0.03,
                        indel_len_max=3).to_list()
    want = ctx.align_scores_batched(reads, slots=min(128, max(2, 1 << (len(reads) - 1).bit_length())))
    tb = []
    for r, w in zip(reads, want):
        t = time.perf_counter()
        ops, score, ckp = ctx.align_traceback(r, k=500)
        dt = time.perf_counter() - t
        ps, last = path_score(ops, r, labels)
        tb.append({"len": len(r), "seconds": dt, "checkpointed": ckp, "score": score,
                   "score_only": int(w), "rescored": ps, "last_row": last,
                   "ok": bool(score == w == ps and last == len(r) - 1),
                   "gcups_forward_cells": len(r) * N / dt / 1e9})
    out["traceback"] = tb
    out["traceback_summary"] = {"reads": len(tb), "all_ok": all(x["ok"] for x in tb),
                                "gcups": sum(x["len"] for x in tb) * N / sum(x["seconds"] for x in tb) / 1e9}
    batch = make_reads(g, 256, 4545, len_max=2000)
    ctx.align_scores_batched(batch[:128], slots=128)  # warm-up
    ctx.align_scores_batched(batch, slots=128)
    p = ctx.profile()
    cells = sum(len(r) for r in batch) * N
    out["batched"] = {"reads": len(batch), "slots": 128, "gcups": cells / p["total_ms"] / 1e6,
                      "device_ms": p["total_ms"]}
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def path_score(ops, read, labels):
    """The traceback drivers' own check (src/ConSGA_traceback.cpp:190-209):
    the path's score under the unit costs and the last read row it uses."""
    score, last = 0, -1
    for row, v, op in ops:
        if op == 1:
            score += 0 if labels[int(v)] == read[int(row)] else 1
            last = int(row)
        else:
            score += 1
            if op == 0:
                last = int(row)
    return score, last


def run_traceback_cfg1(args):
    """Config 1: the 5 Mbp config-2 graph, 2,000 x 150 bp plus 200 x 2 kbp
    reads at 1% / 0.5% / 0.1% substitution / indel / N, full int32-sized
    matrices under the cap (the batched path keeps them 16-bit), every path
    rescored against the score-only result. The one-read path is timed on a
    sample for comparison. Prints one JSON line."""
    import chsga_b200 as cb
    g = make_graph(args.backbone)
    N = g.stats()["num_chars"]
    labels = ctypes_labels(g)
    n150, n2k = (2000, 200) if not args.tb_sample else (args.tb_sample, max(1, args.tb_sample // 10))
    reads = (g.gen_reads(n150, 11, 150, 150, sub_rate=0.01, indel_rate=0.005, n_rate=0.001).to_list() +
             g.gen_reads(n2k, 12, 2000, 2000, sub_rate=0.01, indel_rate=0.005, n_rate=0.001).to_list())
    ctx = cb.Context(0).load(g)
    want = ctx.align_scores_batched(reads, slots=128)
    ctx.align_traceback_batched(reads[:64], slots=64)  # warm-up
    t = time.perf_counter()
    got = ctx.align_traceback_batched(reads, slots=64)
    dt = time.perf_counter() - t
    bad = 0
    for r, w, (ops, score, ck) in zip(reads, want, got):
        ps, last = path_score(ops, r, labels)
        bad += int(not (score == w == ps and last == len(r) - 1 and not ck))
    cells = sum(len(r) for r in reads) * N
    sample = reads[:20] + reads[n150:n150 + 4]
    t = time.perf_counter()
    for r in sample:
        ctx.align_traceback(r)
    dt1 = time.perf_counter() - t
    cells1 = sum(len(r) for r in sample) * N
    line = {"mode": "traceback-cfg1", "num_chars": N, "reads": len(reads), "mismatches": bad,
            "batched": {"seconds": dt, "reads_per_s": len(reads) / dt, "gcups": cells / dt / 1e9,
                        "slots": "up to 64, by matrix memory"},
            "one_by_one": {"sample": f"{len(sample)} reads (20 x 150 bp, 4 x 2 kbp)", "seconds": dt1,
                           "gcups": cells1 / dt1 / 1e9},
            "speedup": (cells / dt) / (cells1 / dt1)}
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def run_top_compare(args):
    """Device time per row-step of the same reads with top regions of
    23000, 12000, 8000 (the default), 5000 and 3000 hierarchy vertices, at
    1, 8, 16, 32, 64 and 128 slots on the config-2-mix graph, and the
    per-kernel-group split (CUDA events between the groups) at 1, 8 and 128
    slots. Every run's scores must equal the first's. One JSON line."""
    import numpy as np

    import chsga_b200 as cb
    g = make_graph(args.backbone)
    ctx = cb.Context(0).load(g)
    pctx = cb.Context(0, flags=cb.FLAG_PROFILE).load(g)
    out = {"mode": "top-compare", "num_chars": g.stats()["num_chars"], "shapes": []}
    for R, n, seed, lm in ((1, 4, 31_000, 1000), (8, 32, 31_001, 2000), (16, 64, 31_004, 2000),
                           (32, 96, 31_005, 2000), (64, 160, 31_006, 2000), (128, 256, 31_002, 2000)):
        reads = make_reads(g, n, seed, len_max=lm)
        rec, ref = {"slots": R, "reads": n}, None
        for K in (23000, 12000, 8000, 5000, 3000):
            lay = g.check_layout(R, 16, K)
            ctx.align_scores_batched(reads, slots=R, steps_per_graph=16, top_vertices=K)
            best = None
            for _ in range(3):
                sc = ctx.align_scores_batched(reads, slots=R, steps_per_graph=16, top_vertices=K)
                p = ctx.profile()
                t = p["total_ms"] / max(1, p["steps"])
                best = t if best is None else min(best, t)
            ref = sc if ref is None else ref
            e = {"first_level": lay["top_first_level"], "top_vertices": lay["top_vertices"],
                 "us_per_row_step": best * 1e3, "same_scores": bool(np.array_equal(sc, ref))}
            if R in (1, 8, 128):
                pctx.align_scores_batched(reads[:max(2, R)], slots=R, steps_per_graph=16, top_vertices=K)
                pr = pctx.profile()
                st = max(1, pr["row_launches"])
                e["split_us"] = {k.replace("_ms", ""): 1e3 * pr[k] / st for k in
                                 ("row_ms", "sweep_up_ms", "top_ms", "sweep_down_ms", "other_ms")}
            rec[str(K)] = e
        out["shapes"].append(rec)
    pctx.close()
    ctx.close()
    print(json.dumps(out), flush=True)
    return 0


def run_launch_compare(args):
    """Device time of the same reads through the CUDA-graph chain of
    row-step kernels (with and without programmatic dependent launch between
    its kernels) and through the persistent row-step kernel, at 1, 8 and
    128 slots, on the config-2-mix graph; the one-slot chain also with the
    one-thread-per-vertex row kernel (the plain path's row kernel before the
    tile kernel). Every run's scores must equal the first's. One JSON line."""
    import numpy as np

    import chsga_b200 as cb
    g = make_graph(args.backbone)
    N = g.stats()["num_chars"]
    ctx = cb.Context(0).load(g)
    os.environ["CHSGA_PDL"] = "0"  # read when a context opens (on by default)
    ctx_nopdl = cb.Context(0).load(g)
    del os.environ["CHSGA_PDL"]
    os.environ["CHSGA_PULL_COOP"] = "1"
    ctx_coop = cb.Context(0).load(g)
    pctx_coop = cb.Context(0, flags=cb.FLAG_PROFILE).load(g)
    del os.environ["CHSGA_PULL_COOP"]
    os.environ["CHSGA_PULL_LEAN"] = "0"  # the unbounded upward form on every level
    ctx_gen = cb.Context(0).load(g)
    pctx_gen = cb.Context(0, flags=cb.FLAG_PROFILE).load(g)
    del os.environ["CHSGA_PULL_LEAN"]
    out = {"mode": "launch-compare", "num_chars": N, "shapes": []}
    want = [int(x) for x in args.shapes.split(",")]
    shapes = [(R, make_reads(g, n, seed, len_max=lm)) for R, n, seed, lm in
              ((1, 4, 31_000, 1000), (8, 32, 31_001, 2000), (128, 256, 31_002, 2000)) if R in want]
    for R, reads in shapes:
        cells = sum(len(r) for r in reads) * N
        runs = [("graphs", dict(use_graphs=cb.LAUNCH_GRAPHS, steps_per_graph=16)),
                ("graphs_no_pdl", dict(use_graphs=cb.LAUNCH_GRAPHS, steps_per_graph=16, ctx=ctx_nopdl)),
                ("persistent", dict(use_graphs=cb.LAUNCH_PERSISTENT, steps_per_graph=16)),
                ("persistent_64", dict(use_graphs=cb.LAUNCH_PERSISTENT, steps_per_graph=64))]
        if R == 1:
            runs.append(("graphs_direct_row", dict(use_graphs=cb.LAUNCH_GRAPHS, steps_per_graph=16,
                                                   row_kernel=cb.ROW_DIRECT)))
        if R >= 8:
            runs.append(("graphs_pull_unbounded", dict(use_graphs=cb.LAUNCH_GRAPHS, steps_per_graph=16,
                                                       ctx=ctx_gen)))
        if R >= 64:
            runs.append(("graphs_pull_coop", dict(use_graphs=cb.LAUNCH_GRAPHS, steps_per_graph=16,
                                                  ctx=ctx_coop)))
        if R == 128:
            # AUTO runs delta rows here; the 16-bit stream rows for comparison
            runs.append(("graphs_stream_rows", dict(use_graphs=cb.LAUNCH_GRAPHS, steps_per_graph=16,
                                                    row_kernel=cb.ROW_STREAM)))
        rec = {"slots": R, "reads": len(reads), "bases": sum(len(r) for r in reads)}
        ref = None
        for name, kw in runs:
            kw = dict(kw)
            cx = kw.pop("ctx", ctx)
            cx.align_scores_batched(reads, slots=R, **kw)  # warm-up (graph build, caches)
            best = None
            for _ in range(3):
                sc = cx.align_scores_batched(reads, slots=R, **kw)
                p = cx.profile()
                best = p["total_ms"] if best is None else min(best, p["total_ms"])
            if ref is None:
                ref = sc
            rec[name] = {"device_ms": best, "gcups": cells / best / 1e6, "launch_mode": int(p["launch_mode"]),
                         "ms_per_row_step": best / max(1, p["steps"]),
                         "same_scores": bool(np.array_equal(sc, ref))}
        out["shapes"].append(rec)
    # per-kernel-group times at one slot (CUDA events between the groups)
    pctx = cb.Context(0, flags=cb.FLAG_PROFILE).load(g)
    one = make_reads(g, 4, 31_000, len_max=1000)
    for name, rk in (("tile_row", cb.ROW_AUTO), ("direct_row", cb.ROW_DIRECT)):
        pctx.align_scores_batched(one[:2], slots=1, row_kernel=rk)
        pr = pctx.profile()
        st = max(1, pr["row_launches"])
        out["plain_profile_" + name] = {k.replace("_ms", "_us"): 1e3 * pr[k] / st for k in
                                        ("row_ms", "sweep_up_ms", "top_ms", "sweep_down_ms", "other_ms")}
    # per-kernel-group times at 128 slots, upward levels as k_pull_lv16 (two-edge form where it
    # applies), as the unbounded k_pull_lv16 and as k_pull_lv16c
    if 128 in want:
        reads128 = make_reads(g, 128, 31_003, len_max=1000)
        for name, cx in (("pull16", pctx), ("pull16_unbounded", pctx_gen), ("pull16c", pctx_coop)):
            cx.align_scores_batched(reads128, slots=128)
            pr = cx.profile()
            st = max(1, pr["row_launches"])
            out["batched_profile_" + name] = {k.replace("_ms", "_us"): 1e3 * pr[k] / st for k in
                                              ("row_ms", "sweep_up_ms", "top_ms", "sweep_down_ms", "other_ms")}
    pctx.close()
    pctx_coop.close()
    ctx_coop.close()
    pctx_gen.close()
    ctx_gen.close()
    ctx_nopdl.close()
    ctx.close()
    print(json.dumps(out), flush=True)
    return 0


def _served_logs(cb, ctx, g, reads, mode, slots, k=500, cap=0, tb_workers=1):
    """Runs the reads through a server and returns (features, targets,
    results): targets are the request's device time in ms (admission to
    completion) and its device bytes -- the measured peak of a traceback, the
    slot's share of the engine's 16-bit rows for a score read."""
    import numpy as np
    N = g.stats()["num_chars"]
    # the score lane has at least 2 slots; tracebacks run one read at a time
    srv = cb.Server(ctx, slots=max(2, slots), tb_workers=tb_workers, tb_k=k, tb_cap_bytes=cap,
                    queue_capacity=4096, arena_bytes=64 << 20)
    tk = [srv.submit(r, mode) for r in reads]
    res = srv.collect()
    srv.close()
    x, y, out = [], [], []
    for t, r in zip(tk, reads):
        d = res[t]
        if d["status"] != cb.OK:
            raise RuntimeError(f"request failed with status {d['status']}")
        x.append(cb.cm_features(ctx, len(r), mode, slots if mode == cb.REQ_SCORE else 1, k, cap))
        ms = max(1e-3, (d["done_ns"] - d["start_ns"]) / 1e6)
        by = d["peak_bytes"] if mode == cb.REQ_TRACEBACK else 4.0 * (N + 32) + len(r)
        y.append([ms, by])
        out.append(d)
    return np.array(x, np.float32), np.array(y, np.float32), out


def run_cfg5(args):
    """Config 5: served mode plus the learned cost model on the config-4
    graph resident in HBM.
      logs     the library's own runs on the config-2 graph (5 Mbp) and the
               config-4 graph (100 Mbp): score requests through the serving
               loop, full-matrix and checkpointed tracebacks; per request the
               8 features, device time and device bytes
      model    the FP32 MLP trained on the GPU on 3/4 of the logs; mean
               absolute log error on the held-out 1/4 for time and bytes,
               against the analytic |V| x |read| model (time = a |V| |read|
               with a fitted on the training logs, bytes = 4 |V| |read|)
      stream   Poisson arrivals on the config-4 graph for --cfg5-window-s
               seconds at ~80% of the score capacity measured in the logs:
               80% 150 bp at 1% error and 16% log-uniform 1-10 kbp at 5%
               error as score requests, 4% 150-600 bp traceback requests
               (k = 100, full matrices up to 200 bases),
               tracebacks admitted by the model's predicted footprint
               (CHSGA_FP_MODEL); p50/p99 per kind, GCUPS, the model's error on
               the stream. The 50,000-read stream of the configuration would
               take hours on one GPU; the window is a sample of it.
    Prints one JSON line."""
    import numpy as np

    import chsga_b200 as cb
    t0 = time.time()
    g2 = make_graph(args.backbone)
    g4 = cb.HostGraph.generate(**cb.GRAPH_CONFIGS["cfg4"])
    g4.build_pch()
    prep_s = time.time() - t0
    N2, N4 = g2.stats()["num_chars"], g4.stats()["num_chars"]
    ctx2 = cb.Context(0).load(g2)
    X, Y, src = [], [], []

    def add(x, y, tag):
        X.append(x)
        Y.append(y)
        src.extend([tag] * len(x))

    t = time.time()
    # config-2 graph: score reads (log-uniform 150-10k), tracebacks full-matrix and checkpointed
    add(*_served_logs(cb, ctx2, g2, make_reads(g2, 256, 5001), cb.REQ_SCORE, 128)[:2], "cfg2-score")
    add(*_served_logs(cb, ctx2, g2, make_reads(g2, 24, 5002, len_max=2000), cb.REQ_TRACEBACK, 1)[:2],
        "cfg2-tb-full")
    for k in (100, 250):
        add(*_served_logs(cb, ctx2, g2, make_reads(g2, 8, 5003 + k, len_max=2000), cb.REQ_TRACEBACK, 1,
                          k=k, cap=12 * N2 * 4)[:2], f"cfg2-tb-ckpt-k{k}")
    ctx2.close()
    ctx4 = cb.Context(0).load(g4)
    add(*_served_logs(cb, ctx4, g4, make_reads(g4, 64, 5101, len_max=2000), cb.REQ_SCORE, 64)[:2],
        "cfg4-score")
    # on the 139 M-char graph a 16-bit row is 278 MB: full matrices up to 200
    # bases, checkpointed above that with k = 100 (101-row segments, 28 GB)
    cap4 = 200 * N4 * 4
    add(*_served_logs(cb, ctx4, g4, g4.gen_reads(8, 5102, 100, 200, sub_rate=0.01, indel_rate=0.005)
                      .to_list(), cb.REQ_TRACEBACK, 1, k=100, cap=cap4)[:2], "cfg4-tb-full")
    add(*_served_logs(cb, ctx4, g4, g4.gen_reads(4, 5103, 400, 1500, sub_rate=0.02, indel_rate=0.03)
                      .to_list(), cb.REQ_TRACEBACK, 1, k=100, cap=cap4)[:2], "cfg4-tb-ckpt")
    log_s = time.time() - t
    X, Y = np.concatenate(X), np.concatenate(Y)
    rng = np.random.default_rng(0)
    order = rng.permutation(len(X))
    tr, te = order[: len(X) * 3 // 4], order[len(X) * 3 // 4:]
    m = cb.CostModel(0, seed=9)
    t = time.time()
    m.train(X[tr], Y[tr], epochs=1500, batch=64, lr=2e-3, seed=4)
    train_s = time.time() - t
    pred = m.predict(X[te])
    cells = (2 ** X[:, 1]) * (2 ** X[:, 0] - 1)
    a = np.exp(np.mean(np.log(Y[tr, 0] / cells[tr])))
    ana = np.stack([a * cells[te], 4 * cells[te]], 1)
    err_mlp = np.mean(np.abs(np.log(pred / Y[te])), 0)
    err_ana = np.mean(np.abs(np.log(ana / Y[te])), 0)
    out = {"mode": "cfg5", "num_chars_cfg2": N2, "num_chars_cfg4": N4, "graph_prep_s": prep_s,
           "logs": {"requests": len(X), "by_kind": {k: src.count(k) for k in sorted(set(src))},
                    "seconds": log_s},
           "cost_model": {"train": len(tr), "held_out": len(te), "train_seconds": train_s,
                          "mlp_mean_abs_log_err": {"time": float(err_mlp[0]), "bytes": float(err_mlp[1])},
                          "analytic_mean_abs_log_err": {"time": float(err_ana[0]),
                                                        "bytes": float(err_ana[1])}}}
    # stream on the config-4 graph
    short = g4.gen_reads(4000, 6001, 150, 150, sub_rate=0.006, indel_rate=0.003, n_rate=0.001).to_list()
    longr = [r for r in make_reads(g4, 3000, 6002, len_max=10000) if len(r) >= 1000]
    tbr = g4.gen_reads(400, 6003, 150, 600, sub_rate=0.01, indel_rate=0.005).to_list()
    mix = []
    pick = np.random.default_rng(6).random(8000)
    si = li = ti = 0
    for u in pick:
        if u < 0.80:
            mix.append((short[si % len(short)], cb.REQ_SCORE)); si += 1
        elif u < 0.96:
            mix.append((longr[li % len(longr)], cb.REQ_SCORE)); li += 1
        else:
            mix.append((tbr[ti % len(tbr)], cb.REQ_TRACEBACK)); ti += 1
    mean_len = float(np.mean([len(r) for r, _ in mix]))
    # capacity: the 64-slot lane advances 64 reads a row-step; its row-step
    # time from the score logs (a read of L bases spends L row-steps)
    y_sc = Y[[i for i, k in enumerate(src) if k == "cfg4-score"]]
    x_sc = X[[i for i, k in enumerate(src) if k == "cfg4-score"]]
    ms_per_row = float(np.median(y_sc[:, 0] / (2 ** x_sc[:, 0] - 1)))
    lane_gcups = 64 * N4 / (ms_per_row * 1e6)
    rate = 0.8 * lane_gcups * 1e9 / (mean_len * N4)
    n = max(16, min(len(mix), int(rate * args.cfg5_window_s)))
    mix = mix[:n]
    arrivals = np.cumsum(np.random.default_rng(7).exponential(1.0 / rate, n))
    srv = cb.Server(ctx4, cost_model=m, slots=64, tb_workers=2, footprint=cb.FP_MODEL, tb_k=100,
                    tb_cap_bytes=cap4, queue_capacity=4096, arena_bytes=64 << 20)
    tickets = [None] * n
    res = {}

    def producer():
        t1 = time.perf_counter()
        for i, ((r, mode), at) in enumerate(zip(mix, arrivals)):
            d = at - (time.perf_counter() - t1)
            if d > 0:
                time.sleep(d)
            tickets[i] = srv.submit(r, mode)

    t = time.time()
    th = threading.Thread(target=producer)
    th.start()
    while th.is_alive() or len(res) < n:
        for d in srv.poll(1024, 50):
            res[d["ticket"]] = d
    th.join()
    stream_s = time.time() - t
    st = srv.stats()
    srv.close()
    ok = all(res[t]["status"] == cb.OK for t in tickets)
    lat = {}
    for mode, name in ((cb.REQ_SCORE, "score"), (cb.REQ_TRACEBACK, "traceback")):
        v = np.array([(res[t]["done_ns"] - res[t]["submit_ns"]) / 1e6 for t, (r, md) in zip(tickets, mix)
                      if md == mode])
        lat[name] = {"n": int(len(v)), "p50_ms": float(np.percentile(v, 50)) if len(v) else None,
                     "p99_ms": float(np.percentile(v, 99)) if len(v) else None}
    # the model's error on the stream's own requests
    xs = np.array([cb.cm_features(ctx4, len(r), md, 64 if md == cb.REQ_SCORE else 1, 100,
                                  cap4 if md == cb.REQ_TRACEBACK else 0) for r, md in mix], np.float32)
    ys = np.array([max(1e-3, (res[t]["done_ns"] - res[t]["start_ns"]) / 1e6) for t in tickets])
    ps = m.predict(xs)[:, 0]
    cs = N4 * np.array([len(r) for r, _ in mix], np.float64)
    m.close()
    ctx4.close()
    out["stream"] = {"arrivals": "Poisson", "window_s": args.cfg5_window_s, "requests": n,
                     "rate_per_s": rate, "load": 0.8, "lane_capacity_gcups": lane_gcups,
                     "mix": "80% 150 bp @1% score, 16% 1-10 kbp @5% score, 4% 150-600 bp traceback (k 100)",
                     "admission": "traceback footprint predicted by the cost model (CHSGA_FP_MODEL)",
                     "all_ok": ok, "seconds": stream_s, "gcups": st["gcups"], "latency": lat,
                     "model_time_mean_abs_log_err": float(np.mean(np.abs(np.log(ps / ys)))),
                     "analytic_time_mean_abs_log_err": float(np.mean(np.abs(np.log(a * cs / ys))))}
    print(json.dumps(out), flush=True)
    return 0


def ctypes_labels(g):
    import ctypes
    v = g.view()
    return ctypes.string_at(v.labels, v.num_chars)


def profiled_roofline(cb, g, st, multi, device, R, opts, peak, src, row_bits, clk_mhz=None):
    """A profiled pass (CUDA events around every kernel group of every
    row-step) with R slots; the row kernel's achieved bandwidth against the
    algorithmic bytes of one launch, and the sweep kernels' per row-step.
    R = 1 is the plain one-read-per-launch path (align_scores)."""
    pctx = cb.Context(device, flags=cb.FLAG_PROFILE)
    pctx.load(g)
    if R == 1:
        sample = make_reads(g, 2, 77_001, len_max=1000)
        pctx.align_scores(sample)
    else:
        sample = make_reads(g, R, 77_777, len_max=1000)
        pctx.align_scores_batched(sample, **dict(opts, slots=R), row_bits=row_bits)
    pr = pctx.profile()
    pctx.close()
    w = pr["row_bits"] // 8
    row_avg_s = pr["row_ms"] / max(1, pr["row_launches"]) / 1e3
    # AUTO: delta rows for score-only steps at 128 slots (this pass is score-only)
    auto16 = "k_row_delta" if R == 128 else ("k_row_stream" if R >= 64 else ("k_row_dpx" if R >= 2 else "k_row_t1"))
    kname = {cb.ROW_DIRECT: "k_row_direct", cb.ROW_TILED: "k_row_tiled", cb.ROW_DPX: "k_row_dpx",
             cb.ROW_STREAM: "k_row_stream", cb.ROW_DELTA: "k_row_delta"}.get(
        opts["row_kernel"] if R > 1 else 0, auto16 if pr["row_bits"] == 16 else "k_row_direct")
    if pr["row_bits"] == 32 and kname in ("k_row_stream", "k_row_dpx", "k_row_delta"):
        kname = "k_row_direct"  # the 16-bit kernels do not run 32-bit rows
    ab = algorithmic_delta_row_bytes(st, R, multi) if kname == "k_row_delta" else \
        algorithmic_row_bytes(st, R, multi, w)
    tr = ncu_traffic(kname)
    total = pr["row_ms"] + pr["sweep_up_ms"] + pr["top_ms"] + pr["sweep_down_ms"] + pr["other_ms"]
    # working set of one row-step: two score rows, BV and FL, graph arrays
    S = st["num_strings"]
    work = 2 * w * st["num_chars"] * R + 2 * 2 * w * S * R + 3 * st["num_chars"] / 8 + 40 * S
    out = {
        "bound": "hbm", "kernel": f"{kname}<{R}>", "row_bits": int(pr["row_bits"]),
        "achieved": ab / row_avg_s / 1e9, "peak": peak, "unit": "GB/s",
        "frac": ab / row_avg_s / 1e9 / peak,
        "peak_source": f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback 6.65 TB/s",
        "algorithmic_bytes_per_launch": ab, "avg_launch_ms": row_avg_s * 1e3,
        "traffic": tr.get("bytes_per_launch_scaled") if tr else None,
        "traffic_source": tr.get("source") if tr else None,
        "l2_resident": bool(work < 126e6), "working_set_bytes": work,
        "row_step_ms": total / max(1, pr["row_launches"]),
        "kernel_share": {k: pr[k] / total for k in
                         ("row_ms", "sweep_up_ms", "top_ms", "sweep_down_ms", "other_ms")},
        "per_row_step_us": {k.replace("_ms", ""): 1e3 * pr[k] / max(1, pr["row_launches"]) for k in
                            ("row_ms", "sweep_up_ms", "top_ms", "sweep_down_ms", "other_ms")},
    }
    if kname == "k_row_delta":
        # delta rows move about a quarter of the 16-bit rows' bytes and are bound by
        # instruction issue; the 16-bit stream kernel on the same reads, for context
        out["limiter"] = "instruction issue (2-bit rows: a third of the 16-bit rows' bytes)"
        # the issue roofline: warp-instructions per char from the ncu capture
        # (profiles/k_row_delta_traffic.json) x chars per launch / launch time,
        # against one warp-instruction per cycle per scheduler (4 per SM) at
        # the SM clock sampled during the timed steps
        if tr and tr.get("warp_inst_per_char"):
            import torch
            sm_count = torch.cuda.get_device_properties(device).multi_processor_count
            inst = tr["warp_inst_per_char"] * st["num_chars"]
            mhz = clk_mhz or 1965.0
            ipeak = 4 * sm_count * mhz * 1e6
            out["issue"] = {"warp_inst_per_launch": inst, "warp_inst_per_char": tr["warp_inst_per_char"],
                            "achieved_warp_inst_per_s": inst / row_avg_s, "peak_warp_inst_per_s": ipeak,
                            "frac": inst / row_avg_s / ipeak,
                            "peak_source": f"4 schedulers x {sm_count} SMs x {mhz:.0f} MHz"}
        q = cb.Context(device, flags=cb.FLAG_PROFILE)
        q.load(g)
        q.align_scores_batched(sample, **dict(opts, slots=R, row_kernel=cb.ROW_STREAM), row_bits=16)
        qs = q.profile()
        q.close()
        s_avg = qs["row_ms"] / max(1, qs["row_launches"]) / 1e3
        s_ab = algorithmic_row_bytes(st, R, multi, 2)
        out["stream_rows"] = {"kernel": f"k_row_stream<{R}>", "avg_launch_ms": s_avg * 1e3,
                              "algorithmic_bytes_per_launch": s_ab, "achieved": s_ab / s_avg / 1e9,
                              "frac": s_ab / s_avg / 1e9 / peak,
                              "row_step_ms": sum(qs[k] for k in ("row_ms", "sweep_up_ms", "top_ms", "sweep_down_ms",
                                                                 "other_ms")) / max(1, qs["row_launches"])}
    # sweep kernels below the top region (the top region the run used)
    lay = g.check_layout(R, pr["row_bits"], opts["top_vertices"] if R > 1 else 0)
    up_b, down_b = algorithmic_sweep_bytes(st, lay, R, w, fl_first=kname != "k_row_delta")
    up_s = pr["sweep_up_ms"] / max(1, pr["row_launches"]) / 1e3
    down_s = pr["sweep_down_ms"] / max(1, pr["row_launches"]) / 1e3
    # 16-bit rows with R >= 8 run the packed forms of both sweeps
    packed = pr["row_bits"] == 16 and R >= 8
    out["sweeps"] = {
        "k_pull_lv16" if packed else "k_pull_lv": {
            "algorithmic_bytes_per_step": up_b, "avg_step_ms": up_s * 1e3,
            "achieved": up_b / up_s / 1e9 if up_s else None,
            "frac": up_b / up_s / 1e9 / peak if up_s else None},
        "k_down16" if packed else "k_down": {
            "algorithmic_bytes_per_step": down_b, "avg_step_ms": down_s * 1e3,
            "achieved": down_b / down_s / 1e9 if down_s else None,
            "frac": down_b / down_s / 1e9 / peak if down_s else None},
        "top_region": "levels >= %d (%d vertices) run in k_top, latency-bound" % (
            lay["top_first_level"], lay["top_vertices"]),
    }
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.scale_cfg4:
        return run_scale_cfg4(args)
    if args.traceback_cfg1:
        return run_traceback_cfg1(args)
    if args.launch_compare:
        return run_launch_compare(args)
    if args.top_compare:
        return run_top_compare(args)
    if args.cfg5:
        return run_cfg5(args)
    ws, rank, local = dist_env()
    if ws > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    import numpy as np

    import chsga_b200 as cb
    g = make_graph(args.backbone)
    st = g.stats()
    N = st["num_chars"]
    multi = st["num_strings"] - st["single_char_strings"]
    ctx = cb.Context(local)
    ctx.load(g)
    wb = args.warmup_batch or args.batch

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    from chsga_b200 import replicas

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, ws, device=f"cuda:{local}")

    # autotuner on a sample of the distribution (reads capped at 2 kbp)
    opts = dict(slots=args.slots, steps_per_graph=8,
                row_kernel=["auto", "direct", "tiled", "dpx", "stream", "delta"].index(args.row_kernel),
                top_vertices=0)
    tune = None
    if not args.no_tune:
        tsample = make_reads(g, 4 * args.slots, 60_000 + rank, len_max=2000)
        best, trials = ctx.autotune(tsample, repeats=1)
        opts = {k: best[k] for k in opts}
        tune = {"chosen": opts, "trials": [
            {k: (round(t[k], 1) if isinstance(t[k], float) else t[k]) for k in
             ("slots", "steps_per_graph", "row_kernel", "top_vertices", "measured_gcups")}
            for t in trials]}

    # warm-up: full passes of the engine (CUDA-graph instantiation, caches) on
    # batches of the same distribution capped at 1 kbp, so a warm-up step is
    # not held up by one 10 kbp read
    for w in range(args.warmup):
        reads = make_reads(g, wb, 50_000 + 1000 * rank + w, len_max=1000)
        ctx.align_scores_batched(reads, **opts)
    batches = [make_reads(g, args.batch, 1000 * rank + s) for s in range(args.steps)]
    cells = sum(len(r) for b in batches for r in b) * N
    h2d = sum(len(r) for b in batches for r in b) // args.steps + 16 * args.batch
    d2h = 4 * args.batch
    clocks = Clocks(local)
    barrier()
    clocks.start()
    dev_ms, lat, launches, steps_work = 0.0, [], 0, 0
    t0 = time.perf_counter()
    batched_scores = []
    for b in batches:
        batched_scores.append(ctx.align_scores_batched(b, **opts))
        p = ctx.profile()
        dev_ms += p["total_ms"]
        launches += int(p["launches"])
        steps_work += int(p["steps"])
        a, d = ctx.read_times(len(b))
        lat.extend(((d - a).astype(np.float64) / 1e6).tolist())
    wall = time.perf_counter() - t0
    srv_wall, sst = wall, {"gpu_launches": 0}
    if not args.kernels_only:
        # batched + served: the same batches streamed through the serving loop
        srv = cb.Server(ctx, slots=opts["slots"], steps_per_graph=opts["steps_per_graph"],
                        queue_capacity=4096, arena_bytes=64 << 20, tb_workers=1,
                        order=cb.ORDER_LONGEST)
        barrier()
        t1 = time.perf_counter()
        tickets = [[srv.submit(r) for r in b] for b in batches]
        served_res = {}
        while len(served_res) < len(batches) * args.batch:
            for d in srv.poll(4096, 100):
                served_res[d["ticket"]] = d
        srv_wall = time.perf_counter() - t1
        served_bad = sum(int(served_res[t]["status"] != cb.OK or served_res[t]["score"] != w)
                         for tk, ws_ in zip(tickets, batched_scores) for t, w in zip(tk, ws_))
        sst = srv.stats()
        srv.close()
    barrier()
    ck = clocks.stop()
    dev_s = max_over_ranks(dev_ms / 1e3)
    srv_s = max_over_ranks(srv_wall)
    total_cells = cells * ws
    value = total_cells / dev_s / 1e9
    e2e = total_cells / srv_s / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "row_storage": (("2-bit delta rows (per char and slot, T[c] - T[c-1] + 1 in 0..2 within a "
                         "vertex) plus the raw first score of every vertex in 16 bits, u16x2 DPX "
                         "arithmetic" if opts["slots"] == 128 and opts["row_kernel"] in (0, 5) else
                         "uint16 rows with u16x2 DPX arithmetic")
                        + ": int32 results exactly, since every row-i value is at most i + 1 (reads "
                          "of at most 65000 bases; longer reads run int32 rows)"),
        "config": {"workload": WORKLOAD, "num_chars": N, "num_strings": st["num_strings"],
                   "hierarchy_levels": st["pch_levels"], "batch_reads": args.batch,
                   "engine": opts, "parallelism": f"replicas x{ws}",
                   "l2": "score rows exceed L2 (no flush needed)"},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "what": "batched steps: device admission-to-completion per read"},
        "e2e": {"value": e2e, "unit": "GCUPS", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "what": "batched+served: the timed batches streamed through chsga_server, "
                        "first submit to last result, host buffers",
                "batched_call_gcups": total_cells / max_over_ranks(wall) / 1e9,
                "server_launches": int(sst["gpu_launches"])},
        "gpu_launches": launches,
        "clocks": ck,
    }
    if tune:
        line["autotune"] = tune
    if args.kernels_only:
        line["e2e"]["what"] = "kernels-only run: wall time of the batched calls"
    if rank == 0 and not args.kernels_only:
        # plain one-read-per-launch path on a random sample of the first
        # timed batch: its GCUPS, and its scores against the batched ones
        import random
        idx = sorted(random.Random(5).sample(range(len(batches[0])),
                                             min(args.plain_reads, len(batches[0]))))
        sample = [batches[0][i] for i in idx]
        plain_scores = ctx.align_scores(sample)
        pp = ctx.profile()
        pc = sum(len(r) for r in sample) * N
        plain_bad = int(np.sum(plain_scores != batched_scores[0][idx]))
        line["plain"] = {"value": pc / (pp["total_ms"] / 1e3) / 1e9, "unit": "GCUPS",
                         "sample": f"{len(sample)} reads drawn at random (seed 5) from the first timed "
                                   f"batch, {sum(len(r) for r in sample)} bases, device time"}
        line["batched_over_plain"] = value / line["plain"]["value"]
        line["served_over_plain"] = e2e / line["plain"]["value"]
        line["mismatches"] = {"batched_vs_plain": plain_bad, "batched_vs_plain_reads": len(sample),
                              "served_vs_batched": served_bad,
                              "served_vs_batched_reads": len(batches) * args.batch}
        line["served"] = served_run(cb, ctx, g, N, opts, e2e, args.served_s)
    if rank == 0 and not args.no_profile and not args.kernels_only:
        peak, src = measured_peak()
        R = opts["slots"]
        line["roofline"] = profiled_roofline(cb, g, st, multi, local, R, opts, peak, src, 0,
                                             clk_mhz=(line.get("clocks") or {}).get("sm_mhz"))
        line["roofline_plain"] = profiled_roofline(cb, g, st, multi, local, 1, opts, peak, src, 0)
        line["roofline_int32_rows"] = profiled_roofline(cb, g, st, multi, local, R, opts, peak, src, 32)
        cb_info, picked, ref_scores = cpu_baseline(g, batches[0], args.cpu_sample_s)
        line["cpu_baseline"] = cb_info
        line.setdefault("mismatches", {})
        line["mismatches"]["vs_reference"] = int(np.sum(batched_scores[0][picked] != ref_scores))
        line["mismatches"]["vs_reference_reads"] = len(picked)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
