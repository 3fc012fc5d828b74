#!/usr/bin/env python
"""Benchmark: gate-evals/s of path-delay-fault grading on B200.

One gate-eval is one (vector pair x gate) through the whole pipeline:
two-pattern simulation, robust marking, pruning, first-detect merge and
exact path counting.  A step grades one batch of synthetic pairs as a fresh
job (the state is reset inside the step).  The default workload is the plain
drop-in configuration: a 20,000-gate synthetic netlist (1,500 PI, 1,500 PO,
depth 60) and 32,768 random vector pairs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  For N > 1 (torchrun), each rank grades its
own 32,768 pairs of the same circuit; the ranks exchange first-detect ids
(all-reduce MIN) before counting, so the job equals one grading of all
N x 32,768 pairs (weak scaling).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))


def _load(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def pkg():
    return _load("pdf_b200", os.path.join(ROOT, "gpu-path-delay-coverage_b200", "__init__.py"))


def oracle():
    return _load("pdf_oracle", os.path.join(ROOT, "oracle", "oracle.py"))


# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for n, val in zip(names, f[4:8]):
                if val.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gpu_id_for_smi(torch, dev: int) -> str:
    """nvidia-smi index of CUDA device `dev`, matched by PCI bus/device id."""
    try:
        pr = torch.cuda.get_device_properties(dev)
        want = (int(pr.pci_domain_id), int(pr.pci_bus_id), int(pr.pci_device_id))
        out = subprocess.run(["nvidia-smi", "--query-gpu=index,pci.bus_id", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=20).stdout
        for ln in out.splitlines():
            idx, bus = [x.strip() for x in ln.split(",")]
            dom, b, rest = bus.split(":")
            d = rest.split(".")[0]
            if (int(dom, 16), int(b, 16), int(d, 16)) == want:
                return idx
    except Exception:
        pass
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    ids = [x for x in vis.split(",") if x.strip()]
    return ids[dev] if dev < len(ids) else str(dev)


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def traffic_summary(workload: str):
    p = os.path.join(ROOT, "profiles", f"k_forward_{workload}.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


# ---------------------------------------------------------------------------

MARK_MODES = {"default": (0, "default (LUT_NR)"), "robust": (1, "robust (LUT_R)"),
              "fixed-robust": (2, "FIXED robust (true n-input gates)"),
              "fixed-nonrobust": (3, "FIXED non-robust (true n-input gates)")}


def oracle_grade(O, nl, codes, n, mode: int, segs: int, threads: int):
    if segs > 1:
        return O.grade_seg(nl, codes, n, segs, mark_mode=mode, threads=threads)
    return O.grade(nl, codes, n, mark_mode=mode, threads=threads)


def cpu_baseline(P, O, nl, v, t, n_sample: int, threads: int, mode: int = 1, segs: int = 1) -> dict:
    """The oracle (a restatement of the reference algorithm; the reference has
    no CPU implementation) on a prefix of the workload's pairs."""
    codes = P.codes_from_planes(v[:, :P.words(n_sample)], t[:, :P.words(n_sample)], n_sample)
    t0 = time.perf_counter()
    r = oracle_grade(O, nl, codes, n_sample, mode, segs, threads)
    dt = time.perf_counter() - t0
    return {"value": nl.n_gates * n_sample / dt, "unit": "gate-evals/s", "cores": threads, "kind": "port",
            "sample": f"first {n_sample} of the workload's pairs, {nl.n_gates} gates, "
                      f"{dt:.2f} s, count {r.total}"}


def run_reference(args):
    """--impl reference: the CPU path (the oracle port) on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    P, O = pkg(), oracle()
    if args.workload in ("c4", "c5"):  # the batch's circuit nearest 20,000 gates stands for it
        spec = P.batch_workload()
        g, n = min(spec, key=lambda x: abs(x[0].n_gates - 20000))
        w = {"gen": g, "pairs": n}
    else:
        w = P.WORKLOADS[args.workload]
    nl = P.gen_netlist(w["gen"])
    n = w["pairs"]
    v, t = P.gen_pairs(P.pair_seed(w["gen"].seed), nl.n_pi, n)
    threads = os.cpu_count() or 1
    G = nl.n_gates
    n_sample = min(n, args.ref_sample or (n if G * n <= 2e9 else max(32, int(6.5e8 / G) // 32 * 32)))
    codes = P.codes_from_planes(v[:, :P.words(n_sample)], t[:, :P.words(n_sample)], n_sample)
    mode = MARK_MODES[args.mark_mode][0]
    for _ in range(args.warmup):
        oracle_grade(O, nl, codes, n_sample, mode, args.segs, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle_grade(O, nl, codes, n_sample, mode, args.segs, threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    val = nl.n_gates * n_sample / (ms / 1e3)
    line = {
        "impl": "reference", "metric": "gate-evals/s", "value": val, "unit": "gate-evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded)",
        "config": workload_config(P, args.workload if args.workload not in ("c4", "c5") else args.workload + "-member",
                                  nl, n_sample, args),
        "cpu_baseline": {"value": val, "unit": "gate-evals/s", "cores": threads, "kind": "port",
                         "sample": f"first {n_sample} of {n} pairs per step"},
        "e2e": {"value": val, "unit": "gate-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(P, name, nl, n_pairs, args=None) -> dict:
    cfg = {"workload": f"{name}: {nl.n_gates} gates, {nl.n_pi} PI, {int(nl.po.sum())} PO, "
                       f"depth {nl.n_levels - 1}, {n_pairs} pairs/rank",
           "gates": nl.n_gates, "pairs_per_rank": n_pairs,
           "mark_mode": MARK_MODES[args.mark_mode][1] if args else "robust (LUT_R)",
           "outputs": "path count and first-detect ids (sim/mark planes not requested)",
           "l2": "flushed between timed steps (256 MiB write)"}
    if args and args.segs > 1:
        cfg["segments"] = args.segs
    if args and args.tile_words:
        cfg["tile_words"] = args.tile_words
    if args and args.threads:
        cfg["threads"] = args.threads
    return cfg


def run_ours(args):
    import numpy as np
    import torch

    P = pkg()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    w = P.WORKLOADS[args.workload]
    nl = P.gen_netlist(w["gen"])
    n = args.pairs or w["pairs"]
    G, W = nl.n_gates, P.words(n)
    v, t = P.gen_pairs(P.pair_seed(w["gen"].seed) + rank, nl.n_pi, n)
    base = rank * n

    mode = MARK_MODES[args.mark_mode][0]
    c = P.Circuit(nl, device=local, mark_mode=mode, max_pairs=n, tile_words=args.tile_words, threads=args.threads,
                  seg_len=args.segs)
    s = P.State(c)
    stream = torch.cuda.current_stream().cuda_stream
    dv = torch.from_numpy(v.view(np.int32)).cuda()
    dt_ = torch.from_numpy(t.view(np.int32)).cuda()
    pairs = P.make_pairs(dv, dt_, n)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    D = _load("pdf_b200_dist", os.path.join(ROOT, "gpu-path-delay-coverage_b200", "dist.py")) if dist else None
    fx_t = torch.empty(c.n_first, dtype=torch.int32, device="cuda")  # one id per net, or per segment
    fy_t = torch.empty(c.n_first, dtype=torch.int32, device="cuda")

    # The graded quantities are the path count and the first-detect ids (what
    # fcount reports); the sim and mark planes stay inside the call.
    def step():
        s.reset_async(stream)
        if dist is None:
            P.grade_async(c, s, pairs, base, None, stream)
            return
        # pairs sharded over ranks: mark locally, MIN-reduce the first-detect
        # ids over NVLink (NCCL), then count locally
        P.grade_mark_async(c, s, pairs, base, None, stream)
        P.first_copy(s, fx_t, fy_t, False, stream)
        D.exchange_first_(fx_t, fy_t)
        P.first_copy(s, fx_t, fy_t, True, stream)
        P.grade_cover_async(c, s, stream)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    ref_total = s.snapshot()[2].value
    job_total = D.sum_u128(ref_total, "cuda") if dist else ref_total

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(gpu_id_for_smi(torch, local))
    sampler.start()
    time.sleep(0.3)
    s.profile(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record()
        step()
        ev[i][1].record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    prof_ms, prof_calls = s.profile_read()
    s.profile(False)
    ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    totals_ok = s.snapshot()[2].value == ref_total

    # e2e: the public calls with pinned host pairs (H2D inside the call) and
    # the batch count read back to the host, every step.
    hv = torch.from_numpy(v.view(np.int32)).pin_memory()
    ht = torch.from_numpy(t.view(np.int32)).pin_memory()
    hpairs = P.Pairs_t(hv.data_ptr(), ht.data_ptr(), n, W, 0)
    import ctypes as C
    e2e_ms = []
    for i in range(max(3, args.warmup) + args.steps):
        flush.fill_(i & 0xFF)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        s.reset_async(stream)
        tot = P.Totals_t()
        if dist is None:
            P.check(P.lib().pdf_grade(c.h, s.h, C.byref(hpairs), base, None, C.byref(tot),
                                      C.c_void_p(stream)), "pdf_grade")
        else:
            P.grade_mark_async(c, s, hpairs, base, None, stream)
            P.first_copy(s, fx_t, fy_t, False, stream)
            D.exchange_first_(fx_t, fy_t)
            P.first_copy(s, fx_t, fy_t, True, stream)
            P.grade_cover_async(c, s, stream)
            s.snapshot()
        if i >= max(3, args.warmup):
            e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_ms_mean = sum(e2e_ms) / len(e2e_ms)

    # e2e, streamed: the same public calls (pdf_grade_async, then
    # pdf_state_snapshot_on for the count) with each step's pinned host pairs
    # copied on a second stream into one of two device buffers while the
    # previous step grades; every step's copy and read-back is inside the
    # timed region, and every step's count is checked
    stream_ms, stream_ok = None, True
    if dist is None:
        cs = torch.cuda.Stream()
        comp = torch.cuda.current_stream()
        bufs = [(torch.empty_like(dv), torch.empty_like(dt_)) for _ in range(2)]
        copied = [torch.cuda.Event() for _ in range(2)]

        def issue_copy(j):
            b = j % 2
            with torch.cuda.stream(cs):
                bufs[b][0].copy_(hv, non_blocking=True)
                bufs[b][1].copy_(ht, non_blocking=True)
                copied[b].record(cs)

        def streamed(k):
            ok = True
            issue_copy(0)
            for i in range(k):
                b = i % 2
                comp.wait_event(copied[b])
                s.reset_async(stream)
                P.grade_async(c, s, P.make_pairs(bufs[b][0], bufs[b][1], n), base, None, stream)
                if i + 1 < k:
                    issue_copy(i + 1)  # buffer (i + 1) % 2 was last read by step i - 1, already read back
                tot = P.Totals_t()
                P.check(P.lib().pdf_state_snapshot_on(s.h, None, None, C.byref(tot), C.c_void_p(stream)),
                        "pdf_state_snapshot_on")
                ok &= tot.value == ref_total
            return ok

        streamed(max(3, args.warmup))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        stream_ok = streamed(args.steps)
        stream_ms = 1e3 * (time.perf_counter() - t0) / args.steps

    # max over ranks
    if dist:
        tt = torch.tensor([ms, e2e_ms_mean], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, e2e_ms_mean = tt.tolist()

    units = world * G * n
    value = units / (ms / 1e3)
    peaks = measured_peaks()
    # Algorithmic bytes per gate-eval: the pairs read (2 bits per PI and pair)
    # and the first-detect ids written (8 bytes per gate per call); the planes
    # of intermediate values never leave the chip except for rows re-read
    # later, which is traffic, not algorithm.
    B = 0.25 * nl.n_pi / G + 8.0 / n
    fwd_ms = prof_ms[0] / max(1, prof_calls)
    achieved = B * G * n / (fwd_ms / 1e3) / 1e9
    tr = traffic_summary(args.workload)
    line = {
        "metric": "gate-evals/s", "value": value, "unit": "gate-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": workload_config(P, args.workload, nl, n, args),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "kernel": "k_forward",
                     "kernel_ms": fwd_ms, "cover_ms": prof_ms[1] / max(1, prof_calls),
                     "bytes_per_gate_eval": B, "peak_source": peaks["source"] + " (hbm_gbs)",
                     "traffic": tr.get("dram_bytes_per_launch") if tr else None},
        "e2e": {"value": units / ((stream_ms or e2e_ms_mean) / 1e3), "unit": "gate-evals/s",
                "h2d_bytes_per_step": int(2 * nl.n_pi * W * 4), "d2h_bytes_per_step": 64,
                "mode": ("streamed: pinned host pairs copied on a second stream while the previous step "
                         "grades (pdf_grade_async + pdf_state_snapshot_on)") if stream_ms else
                        ("per step: host pairs in, mark, MIN-exchange of first-detect ids across ranks, cover, "
                         "count back" if dist else "one synchronous pdf_grade per step"),
                "value_one_call_per_step": units / (e2e_ms_mean / 1e3),
                "note": "one call per step: pdf_grade with the host pairs (H2D inside the call), then the next"},
        # k_forward, k_active, k_cover; with segments k_forward, k_seg_merge, k_seg_first, k_cover
        "gpu_launches": (4 if args.segs > 1 else 3) * args.steps,
        "clocks": clocks,
        "result_stable": bool(totals_ok and stream_ok),
        "batch_count": job_total,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        O = oracle()
        sample = args.cpu_sample or (n if G * n <= 2e9 else max(32, int(1.3e9 / G) // 32 * 32))
        line["cpu_baseline"] = cpu_baseline(P, O, nl, v, t, min(n, sample), os.cpu_count() or 1, mode, args.segs)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batched(args):
    """--workload c4: the mixed-size batch graded in one pass per step (the
    autotuned tile, replayed from a CUDA graph) against the same circuits
    graded one after another with the plain call."""
    import ctypes as C

    import numpy as np
    import torch

    P = pkg()
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    spec = P.batch_workload()[:args.circuits]
    nls = [P.gen_netlist(g) for g, _ in spec]
    counts = [n for _, n in spec]
    t0 = time.perf_counter()
    threads = args.threads
    if args.tile_words:
        tw, tune_ms = args.tile_words, None
    else:
        best, tune_ms = P.batch_autotune(nls, counts, mark_mode=P.MARK_ROBUST, reps=2, threads=args.threads)
        tw = best.tile_words
        threads = best.threads
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream().cuda_stream
    jobs, hosts = [], []
    for k, (nl, (g, n)) in enumerate(zip(nls, spec)):
        ld = (P.words(n) + tw - 1) // tw * tw
        v = np.zeros((nl.n_pi, ld), np.uint32)
        t = np.zeros((nl.n_pi, ld), np.uint32)
        check_v, check_t = P.gen_pairs(P.pair_seed(g.seed), nl.n_pi, n)
        v[:, :check_v.shape[1]] = check_v
        t[:, :check_t.shape[1]] = check_t
        c = P.Circuit(nl, mark_mode=P.MARK_ROBUST, max_pairs=n, tile_words=tw, threads=threads)
        st = P.State(c)
        dv = torch.from_numpy(v.view(np.int32)).cuda()
        dt = torch.from_numpy(t.view(np.int32)).cuda()
        jobs.append((c, st, dv, dt, n, 0))
        hosts.append((torch.from_numpy(v.view(np.int32)).pin_memory(), torch.from_numpy(t.view(np.int32)).pin_memory()))
    units = sum(nl.n_gates * n for nl, n in zip(nls, counts))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # the plain call as a user makes it: each circuit at its own default tile
    # (the batch's pair planes, whose pitch is a multiple of every tile)
    plain_jobs = []
    for (c, st, dv, dt, n, _), nl in zip(jobs, nls):
        c0 = P.Circuit(nl, mark_mode=P.MARK_ROBUST, max_pairs=n)
        plain_jobs.append((c0, P.State(c0), dv, dt, n, 0))

    def plain_pass(js):
        for c, st, dv, dt, n, _ in js:
            st.reset_async(stream)
            P.grade_async(c, st, P.make_pairs(dv, dt, n), 0, None, stream)

    def results(js=jobs):
        return [st.snapshot() for _, st, *_ in js]

    def time_plain(js):
        for _ in range(max(1, args.warmup)):
            plain_pass(js)
        torch.cuda.synchronize()
        res = results(js)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.fill_(1)
        e0.record()
        for _ in range(args.steps):
            plain_pass(js)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps, res

    # plain: every circuit alone, one after another
    plain_ms, plain_res = time_plain(plain_jobs)
    plain_bt_ms, plain_bt_res = time_plain(jobs)

    # batched: one graph replay per pass
    b = P.Batch(jobs)
    for _, st, *_ in jobs:
        st.reset_async(stream)
    b.run(stream)
    batch_res = results()
    same = all(np.array_equal(a[0], x[0]) and np.array_equal(a[1], x[1]) and a[2].value == x[2].value
               and a[2].flags == x[2].flags for ref in (plain_res, plain_bt_res) for a, x in zip(ref, batch_res))
    for c0, st0, *_ in plain_jobs:
        st0.close()
        c0.close()
    for _ in range(max(3, args.warmup)):
        b.run_async(stream)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(gpu_id_for_smi(torch, int(os.environ.get("LOCAL_RANK", "0"))))
    sampler.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record()
        b.run_async(stream)
        ev[i][1].record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = sum(x.elapsed_time(y) for x, y in ev) / args.steps

    # e2e: host pairs in (pinned), one pass, every job's count back
    tot = P.Totals_t()
    e2e = []
    h2d = sum(2 * hv.numel() * 4 for hv, _ in hosts)
    for i in range(2 + args.steps):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for (c, st, dv, dt, n, _), (hv, ht) in zip(jobs, hosts):
            dv.copy_(hv, non_blocking=True)
            dt.copy_(ht, non_blocking=True)
        b.run(stream)
        for _, st, *_ in jobs:
            P.check(P.lib().pdf_state_snapshot(st.h, None, None, C.byref(tot)), "pdf_state_snapshot")
        if i >= 2:
            e2e.append(1e3 * (time.perf_counter() - t1))
    e2e_ms = sum(e2e) / len(e2e)

    # e2e, streamed: two sets of device pair buffers, each bound to a batch;
    # the next pass's pinned host pairs are copied on a second stream while
    # this pass grades, and every job's count is read back after every pass
    # (pdf_state_snapshot_on, ordered on the grading stream)
    cs = torch.cuda.Stream()
    comp = torch.cuda.current_stream()
    sets = [[(dv, dt) for _, _, dv, dt, _, _ in jobs],
            [(torch.empty_like(dv), torch.empty_like(dt)) for _, _, dv, dt, _, _ in jobs]]
    b2 = P.Batch([(c, st, x, y, n, 0) for (c, st, _, _, n, _), (x, y) in zip(jobs, sets[1])])
    passes = [b, b2]
    copied = [torch.cuda.Event() for _ in range(2)]

    def issue_copy(j):
        with torch.cuda.stream(cs):
            for (x, y), (hv, ht) in zip(sets[j % 2], hosts):
                x.copy_(hv, non_blocking=True)
                y.copy_(ht, non_blocking=True)
            copied[j % 2].record(cs)

    def streamed(k):
        issue_copy(0)
        for i in range(k):
            comp.wait_event(copied[i % 2])
            passes[i % 2].run_async(stream)
            if i + 1 < k:
                issue_copy(i + 1)  # set (i + 1) % 2 was last read by pass i - 1, already read back
            for _, st, *_ in jobs:
                P.check(P.lib().pdf_state_snapshot_on(st.h, None, None, C.byref(tot), C.c_void_p(stream)),
                        "pdf_state_snapshot_on")

    streamed(2)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    streamed(args.steps)
    stream_ms = 1e3 * (time.perf_counter() - t1) / args.steps
    b2.close()
    peaks = measured_peaks()
    alg = sum(2 * nl.n_pi * P.words(n) * 4 + 8 * nl.n_gates for nl, n in zip(nls, counts))
    achieved = alg / (ms / 1e3) / 1e9
    info = b.info()
    line = {
        "metric": "gate-evals/s", "value": units / (ms / 1e3), "unit": "gate-evals/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": {"workload": f"c4: {len(nls)} netlists, gates log-uniform 500-200,000 "
                               f"({sum(nl.n_gates for nl in nls)} total), depth 20-150, pairs log-uniform "
                               f"1,024-65,536 ({sum(counts)} total), one batched pass per step",
                   "mark_mode": "robust (LUT_R)", "tile_words": tw, "ctas": info.ctas,
                   "autotune": {"tile_words": tw, "threads": threads, "ms_per_pass": tune_ms, "seconds": tune_s}
                   if tune_ms else None,
                   "threads": threads or "piece capacity + 64",
                   "outputs": "path count and first-detect ids per circuit",
                   "l2": "flushed between timed steps (256 MiB write)"},
        "plain": {"value": units / (min(plain_ms, plain_bt_ms) / 1e3), "ms_per_pass": min(plain_ms, plain_bt_ms),
                  "ms_per_pass_default_tiles": plain_ms, "ms_per_pass_batch_tile": plain_bt_ms,
                  "note": "the same circuits graded one after another (pdf_grade_async each), at each "
                          "circuit's default tile and at the batch's tile; the faster of the two"},
        "batched_vs_plain": min(plain_ms, plain_bt_ms) / ms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "kernel": "k_batch_forward + k_batch_active + k_batch_cover",
                     "peak_source": peaks["source"] + " (hbm_gbs)", "traffic": None},
        "e2e": {"value": units / (stream_ms / 1e3), "unit": "gate-evals/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": 64 * len(jobs),
                "mode": "streamed: pinned host pairs of the next pass copied on a second stream while this "
                        "pass grades (two buffer sets, two batches)",
                "value_one_pass_per_step": units / (e2e_ms / 1e3)},
        "gpu_launches": int(info.launches) * args.steps,  # forward per occupancy class, active, cover
        "clocks": clocks,
        "result_stable": bool(same),
    }
    if not args.no_cpu:
        O = oracle()
        k = int(np.argmin([abs(nl.n_gates - 20000) for nl in nls]))
        nl, (g, n) = nls[k], spec[k]
        v, t = P.gen_pairs(P.pair_seed(g.seed), nl.n_pi, n)
        line["cpu_baseline"] = cpu_baseline(P, O, nl, v, t, min(n, max(32, int(1.3e9 / nl.n_gates) // 32 * 32)),
                                            os.cpu_count() or 1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    return 0


def run_served(args):
    """--workload c5: jobs drawn from the mixed-size distribution arrive as a
    Poisson stream (200 jobs/s); each appends 4,096-pair batches until its
    65,536 pairs are graded.  Reports throughput and per-batch latency; every
    served result is checked against grading the job offline."""
    import ctypes as C

    import numpy as np
    import torch

    P = pkg()
    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n_jobs, per_job, batch, rate = args.jobs, 65536, 4096, 200.0
    spec = P.batch_workload()[:n_jobs]
    rng = np.random.default_rng(0x5EED0005)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    jobs = []
    for g, _ in spec:
        nl = P.gen_netlist(g)
        v, t = P.gen_pairs(P.pair_seed(g.seed), nl.n_pi, per_job)
        jobs.append((nl, v, t))
    units = sum(nl.n_gates * per_job for nl, _, _ in jobs)
    srv = P.Server(mark_mode=P.MARK_ROBUST, batch_pairs=batch, hbm_budget=int(args.hbm_gb * (1 << 30)),
                   workers=args.workers, tile_words=args.tile_words or 4)
    ids = [None] * n_jobs
    sampler = ClockSampler(gpu_id_for_smi(torch, int(os.environ.get("LOCAL_RANK", "0"))))
    sampler.start()
    time.sleep(0.3)
    t0 = time.perf_counter()
    k = 0
    while k < n_jobs or srv.stats().jobs_done < n_jobs:
        now = time.perf_counter() - t0
        while k < n_jobs and arrivals[k] <= now:
            nl, v, t = jobs[k]
            ids[k] = srv.submit(nl, v, t, per_job)
            k += 1
        if srv.stats().jobs_active + srv.stats().jobs_queued == 0:
            time.sleep(max(0.0, min(0.001, arrivals[k] - now)) if k < n_jobs else 0.0)
            continue
        srv.step()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    st = srv.stats()
    # every served result against the job graded offline in one call
    same = True
    for (nl, v, t), jid in zip(jobs, ids):
        fx, fy, tot = srv.result(jid)
        c = P.Circuit(nl, mark_mode=P.MARK_ROBUST, max_pairs=per_job)
        s2 = P.State(c)
        want = P.grade(c, s2, v, t, per_job)
        wfx, wfy, _ = s2.snapshot()
        same &= want.value == tot.value and np.array_equal(wfx, fx) and np.array_equal(wfy, fy)
        s2.close()
        c.close()
    line = {
        "metric": "gate-evals/s", "value": units / wall, "unit": "gate-evals/s", "n_gpus": 1, "steps": int(st.steps),
        "warmup": 0, "ms_per_step": 1e3 * st.busy_s / max(1, st.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": {"workload": f"c5: {n_jobs} jobs from the c4 size distribution, Poisson arrivals at "
                               f"{rate:.0f} jobs/s, {batch}-pair appends up to {per_job} pairs per job",
                   "mark_mode": "robust (LUT_R)", "hbm_budget_gib": args.hbm_gb,
                   "workers": args.workers or "library default", "tile_words": args.tile_words or 4,
                   "outputs": "path count and first-detect ids per job"},
        "latency_ms": {"p50": st.lat_p50_ms, "p99": st.lat_p99_ms, "max": st.lat_max_ms,
                       "per": "job batch, from ready (submission or previous batch) to result"},
        "wall_s": wall, "busy_s": st.busy_s, "batches": int(st.batches),
        # the arrival stream caps throughput: all the work over the span of the arrivals
        "offered_load": units / float(arrivals[-1]),
        "e2e": {"value": units / wall, "unit": "gate-evals/s",
                "h2d_bytes_per_step": int(sum(2 * nl.n_pi * (per_job // 32) * 4 for nl, _, _ in jobs) / max(1, st.steps)),
                "d2h_bytes_per_step": 64},
        "gpu_launches": int(st.launches),
        "clocks": clocks,
        "result_stable": bool(same),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    srv.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--mark-mode", choices=sorted(MARK_MODES), default="robust",
                    help="c1-c3: sensitisation table and gate semantics")
    ap.add_argument("--segs", type=int, default=1, help="c1-c3: path segments of this many nets (1-8)")
    ap.add_argument("--tile-words", type=int, default=0,
                    help="words per CTA column block (0 = default; c4: the autotuned width)")
    ap.add_argument("--threads", type=int, default=0,
                    help="threads per CTA, pieces of threads - 64 gates (0 = default; c4: the batch's circuits)")
    ap.add_argument("--pairs", type=int, default=0,
                    help="c1-c3: pairs per rank instead of the workload's (small cases for profiling)")
    # CPU samples: pairs per timed CPU run (0 = the whole workload up to 2e9
    # gate-evals, else about 1.3e9 gate-evals for the baseline and 6.5e8 per
    # reference-arm step: a few seconds on the host cores)
    ap.add_argument("--cpu-sample", type=int, default=0)
    ap.add_argument("--ref-sample", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--jobs", type=int, default=64, help="c5: jobs in the arrival stream")
    ap.add_argument("--circuits", type=int, default=256,
                    help="c4: the first N netlists of the batch (smaller cases for profiling)")
    ap.add_argument("--hbm-gb", type=float, default=64.0, help="c5: device memory for active jobs")
    ap.add_argument("--workers", type=int, default=0, help="c5: server threads preparing jobs (0 = library default)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c4":
        return run_batched(args)
    if args.workload == "c5":
        return run_served(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
