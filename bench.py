#!/usr/bin/env python
"""Benchmark: gate-evals/s of path-delay-fault grading on B200.

One gate-eval is one (vector pair x gate) through the whole pipeline:
two-pattern simulation, robust marking, pruning, first-detect merge and
exact path counting.  The default workload is the mixed-size batch (c4):
256 synthetic netlists of 500-200,000 gates (depth 20-150) with 1,024-65,536
vector pairs each, graded in one batched pass per step (a CUDA graph of one
forward launch per class of circuits, then the cover), beside the same
circuits graded one after another with the plain call.  Other workloads:
c1 (2,000 gates, 1,024 pairs), c2 (20,000 gates, 32,768 pairs), c3
(1,000,000 gates, Zipf fan-out, 262,144 pairs) and c5 (a Poisson stream of
c4-sized jobs served with continuous batching).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c1|c2|c3|c4|c5]

Prints one JSON line (rank 0).  For N > 1 (torchrun) on c1-c3, each rank
grades its own pairs of the same circuit; the ranks exchange first-detect ids
(all-reduce MIN) before counting, so the job equals one grading of all ranks'
pairs (weak scaling).  On c4 each rank grades the whole batch (replicas; the
ranks are timed together and the slowest sets the time).
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
    """SM clocks and clock-event (throttle) reasons sampled every 20 ms by
    NVML (nvidia-smi at 200 ms when NVML is missing); only the samples taken
    inside the timed region (mark_start .. mark_end) are reported."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("hw_power_brake_slowdown", 0x80), ("sw_power_cap", 0x4))

    def __init__(self, pci_bus_id: str | None, smi_index: str):
        self.pci = pci_bus_id
        self.smi_index = smi_index
        self.samples: list[tuple[float, float, float, int]] = []  # (t, sm MHz, max MHz, reason bits)
        self.stop_flag = threading.Event()
        self.thread = None
        self.proc = None
        self.t0 = self.t1 = None
        self.source = "nvml"

    def start(self):
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByPciBusId(self.pci.encode()) if self.pci else \
                N.nvmlDeviceGetHandleByIndex(int(self.smi_index))
            smax = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))

            def loop():
                while not self.stop_flag.is_set():
                    try:
                        sm = float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM))
                        rs = int(N.nvmlDeviceGetCurrentClocksEventReasons(h))
                        self.samples.append((time.perf_counter(), sm, smax, rs))
                    except Exception:
                        pass
                    self.stop_flag.wait(0.02)
            self.thread = threading.Thread(target=loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.source = "nvidia-smi"
        Q = "clocks.sm,clocks.max.sm,clocks_event_reasons.active"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.smi_index}", f"--query-gpu={Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return

        def read():
            for line in self.proc.stdout:
                f = [x.strip() for x in line.split(",")]
                try:
                    self.samples.append((time.perf_counter(), float(f[0]), float(f[1]), int(f[2], 16)))
                except (ValueError, IndexError):
                    pass
        self.thread = threading.Thread(target=read, daemon=True)
        self.thread.start()

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()

    def stop(self) -> dict:
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        t0 = self.t0 if self.t0 is not None else 0.0
        t1 = self.t1 if self.t1 is not None else float("inf")
        inside = [x for x in self.samples if t0 <= x[0] <= t1]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock sample in the timed region"],
                    "samples": 0, "source": self.source}
        reasons = sorted({n for _, _, _, r in inside for n, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(x[1] for x in inside), "sm_max_mhz": max(x[2] for x in inside),
                "reasons": reasons, "samples": len(inside), "source": self.source,
                "timed_region_s": round(t1 - t0, 3)}


def clock_sampler(torch, dev: int) -> ClockSampler:
    pci = None
    try:
        pr = torch.cuda.get_device_properties(dev)
        pci = f"{int(pr.pci_domain_id):08x}:{int(pr.pci_bus_id):02x}:{int(pr.pci_device_id):02x}.0"
    except Exception:
        pass
    return ClockSampler(pci, gpu_id_for_smi(torch, dev))


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


LANE_TILES = (32, 64, 128)  # tile widths of the lane kernel (a warp per gate)


def profile_summary(name: str):
    """A committed summary of an ncu capture (profiles/<name>.json), or None."""
    p = os.path.join(ROOT, "profiles", f"{name}.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def alg_bytes(nl, n_pairs: int) -> float:
    """Algorithmic bytes of grading n_pairs pairs on netlist nl: the 2-bit
    transition code and the 1-bit mark of every (net, pair), written once
    (0.375 B per gate-eval), and the 2-bit codes of the primary inputs read
    (0.25 B per PI and pair)."""
    return 0.375 * nl.n_gates * n_pairs + 0.25 * nl.n_pi * n_pairs


def roofline(alg: float, kernel_ms: float, kernel: str, prof: dict | None, units: float,
             sm_count: int, sm_mhz) -> dict:
    """HBM roofline of the forward kernel: algorithmic bytes per launch over
    its CUDA-event duration, against the measured copy bandwidth.  With an
    ncu summary of the same launch: its DRAM traffic (scaled to a full
    launch when the capture was a slice) and the issue slots its warp
    instructions fill at the sampled SM clock."""
    peaks = measured_peaks()
    achieved = alg / (kernel_ms / 1e3) / 1e9
    out = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
           "frac": achieved / peaks["hbm_gbs"], "traffic": None, "kernel": kernel, "kernel_ms": kernel_ms,
           "bytes_per_gate_eval": alg / units, "peak_source": peaks["source"] + " (hbm_gbs)"}
    if prof:
        scale = prof.get("scale", 1.0)
        if prof.get("dram_bytes_per_launch") is not None:
            out["traffic"] = prof["dram_bytes_per_launch"] * scale
            out["traffic_source"] = prof.get("source")
        if prof.get("warp_inst_per_launch") and sm_mhz:
            wi = prof["warp_inst_per_launch"] * scale
            slots = sm_count * 4 * sm_mhz * 1e6 * kernel_ms / 1e3
            out["issue_slots_frac"] = wi / slots
            out["issue_note"] = ("warp instructions per launch (ncu smsp__inst_executed.sum) over "
                                 "SMs x 4 schedulers x sampled SM clock x kernel time")
    # what the numbers say bounds the kernel: HBM or issue when either is
    # near its peak, else latency (dependent chains per warp, barriers)
    issue = out.get("issue_slots_frac")
    out["limiter"] = ("hbm" if out["frac"] >= 0.8 else "issue" if issue is not None and issue >= 0.8 else
                      "latency" if issue is not None else "unknown (no ncu summary for this kernel)")
    return out


# ---------------------------------------------------------------------------

MARK_MODES = {"default": (0, "default (LUT_NR)"), "robust": (1, "robust (LUT_R)"),
              "fixed-robust": (2, "FIXED robust (true n-input gates)"),
              "fixed-nonrobust": (3, "FIXED non-robust (true n-input gates)")}


def oracle_grade(O, nl, codes, n, mode: int, segs: int, threads: int):
    if segs > 1:
        return O.grade_seg(nl, codes, n, segs, mark_mode=mode, threads=threads)
    return O.grade(nl, codes, n, mark_mode=mode, threads=threads)


def cpu_sample(P, O, members, target_evals: float, threads: int, mode: int = 1, segs: int = 1,
               reps: int = 1, stride: int = 1) -> dict:
    """The CPU path (the oracle: a restatement of the reference algorithm;
    the reference has no CPU implementation) on a bounded sample of a
    workload: every `stride`-th member circuit graded on the same fraction of
    its pairs (a prefix of at least 32 pairs; the pair generator is
    prefix-stable), so the sample keeps the workload's mix of circuit sizes.
    A circuit whose sample is at least 1/threads of the whole runs on all
    threads (split over its pairs); the others run concurrently, one circuit
    per thread, largest first.  Returns the summed gate-evals over the wall
    seconds (input generation excluded).
    members: (netlist, GenParams, n_pairs)."""
    from concurrent.futures import ThreadPoolExecutor

    members = members[::stride]
    total = sum(nl.n_gates * n for nl, _, n in members)
    f = min(1.0, target_evals / total)
    jobs = []
    for nl, g, n in members:
        k = min(n, max(32, -(-int(f * n) // 32) * 32))
        v, t = P.gen_pairs(P.pair_seed(g.seed), nl.n_pi, k)
        jobs.append((nl, P.codes_from_planes(v, t, k), k))
    jobs.sort(key=lambda j: -j[0].n_gates * j[2])
    evals = sum(nl.n_gates * k for nl, _, k in jobs)
    secs, count = [], 0
    for _ in range(reps):
        t0 = time.perf_counter()
        big = [j for j in jobs if threads == 1 or j[0].n_gates * j[2] * threads >= evals]
        rest = [j for j in jobs if not (threads == 1 or j[0].n_gates * j[2] * threads >= evals)]
        for nl, codes, k in big:
            count += oracle_grade(O, nl, codes, k, mode, segs, threads).total
        if rest:  # ctypes releases the GIL during each oracle call
            with ThreadPoolExecutor(max_workers=threads) as ex:
                count += sum(ex.map(lambda j: oracle_grade(O, j[0], j[1], j[2], mode, segs, 1).total, rest))
        secs.append(time.perf_counter() - t0)
    dt = sum(secs) / len(secs)
    what = (f"the circuit on its first {jobs[0][2]} of {members[0][2]} pairs" if len(members) == 1 else
            f"{'every' if stride == 1 else f'every {stride}th'} circuit of the batch ({len(members)}), each on "
            f"the first {100 * f:.2g}% of its pairs (at least 32)"
            f"{'; small circuits one per thread' if threads > 1 else ''}")
    return {"value": evals / dt, "unit": "gate-evals/s", "cores": threads, "kind": "port",
            "sample": f"{what}: {evals:.3g} gate-evals in {dt:.2f} s", "seconds": dt, "gate_evals": evals,
            "count": count}


def cpu_baselines(P, members, args):
    """The CPU path on all host cores (about 1e9 gate-evals) and on one core
    (about 6e7, every 16th circuit of a batch), each on the workload's own
    mix of circuits."""
    O = oracle()
    mode = MARK_MODES[args.mark_mode][0]
    allc = cpu_sample(P, O, members, args.cpu_sample or 1e9, os.cpu_count() or 1, mode, args.segs)
    one = cpu_sample(P, O, members, (args.cpu_sample or 1e9) / 16, 1, mode, args.segs,
                     stride=16 if len(members) >= 64 else 1)
    for r in (allc, one):
        for k in ("seconds", "gate_evals", "count"):
            r.pop(k)
    return allc, one


def workload_members(P, args):
    """(netlist, GenParams, n_pairs) of every circuit of the workload."""
    if args.workload in ("c4", "c5"):
        spec = P.batch_workload()[:args.circuits]
        return [(P.gen_netlist(g), g, n) for g, n in spec]
    w = P.WORKLOADS[args.workload]
    return [(P.gen_netlist(w["gen"]), w["gen"], args.pairs or w["pairs"])]


def run_reference(args):
    """--impl reference: the CPU path (the oracle port; the reference has no
    CPU implementation and its GPU code needs a Fermi toolchain) on the host
    cores, over a bounded sample of the same workload per step.  Loads the
    workload generator and the oracle, never the grader library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    P, O = pkg(), oracle()
    members = workload_members(P, args)
    threads = os.cpu_count() or 1
    mode = MARK_MODES[args.mark_mode][0]
    target = args.ref_sample or 1e9  # gate-evals per step: a few seconds on 16 cores
    for _ in range(args.warmup):
        cpu_sample(P, O, members, target, threads, mode, args.segs)
    runs = [cpu_sample(P, O, members, target, threads, mode, args.segs) for _ in range(args.steps)]
    secs = sum(r["seconds"] for r in runs)
    evals = sum(r["gate_evals"] for r in runs)
    val = evals / secs
    nl = members[0][0]
    line = {
        "impl": "reference", "metric": "gate-evals/s", "value": val, "unit": "gate-evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded)",
        "config": (batch_config(members, args) if args.workload in ("c4", "c5")
                   else workload_config(P, args.workload, nl, members[0][2], args)),
        "cpu_baseline": {"value": val, "unit": "gate-evals/s", "cores": threads, "kind": "port",
                         "sample": runs[0]["sample"] + " per step"},
        "e2e": {"value": val, "unit": "gate-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "native_libraries": loaded_libraries(),
    }
    print(json.dumps(line), flush=True)
    return 0


def loaded_libraries() -> list[str]:
    """This repository's shared libraries mapped into the process."""
    out = set()
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                path = ln.split()[-1] if ln.strip() else ""
                if path.startswith(ROOT) and path.endswith(".so"):
                    out.add(os.path.relpath(path, ROOT))
    except OSError:
        pass
    return sorted(out)


def batch_config(members, args) -> dict:
    gates = sum(nl.n_gates for nl, _, _ in members)
    pairs = sum(n for _, _, n in members)
    return {"workload": f"c4: {len(members)} netlists, gates log-uniform 500-200,000 ({gates} total), "
                        f"depth 20-150, pairs log-uniform 1,024-65,536 ({pairs} total), one batched pass "
                        f"per step",
            "netlists": len(members), "gates": gates, "pairs": pairs,
            "gate_evals_per_pass": sum(nl.n_gates * n for nl, _, n in members),
            "mark_mode": MARK_MODES[args.mark_mode][1],
            "outputs": "path count and first-detect ids per circuit",
            "l2": "flushed between timed steps (256 MiB write); the pass's planes (GBs) exceed L2"}


def workload_config(P, name, nl, n_pairs, args=None) -> dict:
    cfg = {"workload": f"{name}: {nl.n_gates} gates, {nl.n_pi} PI, {int(nl.po.sum())} PO, "
                       f"depth {nl.n_levels - 1}, {n_pairs} pairs/rank",
           "gates": nl.n_gates, "pairs_per_rank": n_pairs,
           "mark_mode": MARK_MODES[args.mark_mode][1] if args else "robust (LUT_R)",
           "outputs": ("path count, first-detect ids, and the sim and mark planes of every (net, pair) "
                       "written to device memory" if args and args.planes else
                       "path count and first-detect ids (sim/mark planes not requested)"),
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
    # fcount reports); with --planes the sim and mark planes are written to
    # device memory as well (every (net, pair) code and mark, 3 bits each).
    outs = None
    if args.planes:
        tile = c.info().tile_words
        planes = [torch.empty((G, -(-W // tile) * tile), dtype=torch.int32, device="cuda") for _ in range(3)]
        outs = P.make_outputs(*planes)

    def step():
        s.reset_async(stream)
        if dist is None:
            P.grade_async(c, s, pairs, base, outs, stream)
            return
        # pairs sharded over ranks: mark locally, MIN-reduce the first-detect
        # ids over NVLink (NCCL), then count locally
        P.grade_mark_async(c, s, pairs, base, outs, stream)
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
    sampler = clock_sampler(torch, local)
    sampler.start()
    time.sleep(0.1)
    s.profile(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.mark_start()
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record()
        step()
        ev[i][1].record()
    torch.cuda.synchronize()
    sampler.mark_end()
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
            P.check(P.lib().pdf_grade(c.h, s.h, C.byref(hpairs), base, C.byref(outs) if outs else None,
                                      C.byref(tot), C.c_void_p(stream)), "pdf_grade")
        else:
            P.grade_mark_async(c, s, hpairs, base, outs, stream)
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
                P.grade_async(c, s, P.make_pairs(bufs[b][0], bufs[b][1], n), base, outs, stream)
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
    fwd_ms = prof_ms[0] / max(1, prof_calls)
    tile = c.info().tile_words
    kname = "k_forward_lanes" if tile in LANE_TILES else "k_forward"
    prof = profile_summary(f"{kname}_{args.workload}_tile{tile}") if not args.planes and args.segs == 1 and \
        args.mark_mode == "robust" and not args.pairs else None
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    line = {
        "metric": "gate-evals/s", "value": value, "unit": "gate-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": workload_config(P, args.workload, nl, n, args),
        "roofline": dict(roofline(alg_bytes(nl, n), fwd_ms, f"{kname} (tile {tile} words)", prof, G * n,
                                  sm_count, clocks.get("sm_mhz")), cover_ms=prof_ms[1] / max(1, prof_calls)),
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
        line["cpu_baseline"], line["cpu_baseline_1core"] = cpu_baselines(P, [(nl, w["gen"], n)], args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batched(args):
    """--workload c4: the mixed-size batch graded in one pass per step (one
    forward launch per class of circuits and the cover, replayed from a CUDA
    graph) against the same circuits graded one after another with the
    plain call (pdf_grade_async each)."""
    import ctypes as C

    import numpy as np
    import torch

    P = pkg()
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        # replicas: every rank grades the whole batch on its own GPU (the
        # circuits share nothing); the process group only times the ranks
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        args.no_tile_sweep = True  # the plain arm's per-circuit tile sweep runs at N = 1

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    members = workload_members(P, args)
    nls = [m[0] for m in members]
    counts = [m[2] for m in members]
    t0 = time.perf_counter()
    threads = args.threads
    if args.tile_words:
        tw, tune_ms = args.tile_words, None
    else:
        best, tune_ms = P.batch_autotune(nls, counts, mark_mode=P.MARK_ROBUST, reps=2, device=local,
                                         threads=args.threads)
        tw = best.tile_words
        threads = best.threads
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.current_stream().cuda_stream
    jobs, hosts = [], []
    for nl, g, n in members:
        ld = (P.words(n) + 127) // 128 * 128  # a pitch every tile width divides
        v, t = P.gen_pairs(P.pair_seed(g.seed), nl.n_pi, n, ld)
        c = P.Circuit(nl, device=local, mark_mode=P.MARK_ROBUST, max_pairs=n, tile_words=tw, threads=threads)
        st = P.State(c)
        hv = torch.from_numpy(v.view(np.int32)).pin_memory()
        ht = torch.from_numpy(t.view(np.int32)).pin_memory()
        jobs.append((c, st, hv.cuda(), ht.cuda(), n, 0))
        hosts.append((hv, ht))
    units = sum(nl.n_gates * n for nl, n in zip(nls, counts))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # the plain call as a user makes it: each circuit at its own default tile
    plain_jobs = []
    for (c, st, dv, dt, n, _), nl in zip(jobs, nls):
        c0 = P.Circuit(nl, device=local, mark_mode=P.MARK_ROBUST, max_pairs=n)
        plain_jobs.append((c0, P.State(c0), dv, dt, n, 0))

    def plain_pass(js, marks=None):
        for k, (c, st, dv, dt, n, _) in enumerate(js):
            if marks:
                marks[k].record()
            st.reset_async(stream)
            P.grade_async(c, st, P.make_pairs(dv, dt, n), 0, None, stream)
        if marks:
            marks[len(js)].record()

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
    # and each circuit at the tile that grades it fastest alone (every tile
    # width timed per circuit): the best the plain call can do
    sweep_ms, sweep_tiles, sweep_same = 0.0, {}, True
    if not args.no_tile_sweep:
        for (c, st, dv, dt, n, _), nl, ref in zip(jobs, nls, plain_res):
            best = None
            for tile in (4, 8) + LANE_TILES:
                c1 = P.Circuit(nl, device=local, mark_mode=P.MARK_ROBUST, max_pairs=n, tile_words=tile)
                s1 = P.State(c1)
                pr = P.make_pairs(dv, dt, n)
                s1.reset_async(stream)
                P.grade_async(c1, s1, pr, 0, None, stream)
                got = s1.snapshot()
                sweep_same &= bool(np.array_equal(got[0], ref[0]) and got[2].value == ref[2].value)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(3):
                    s1.reset_async(stream)
                    P.grade_async(c1, s1, pr, 0, None, stream)
                e1.record()
                torch.cuda.synchronize()
                t_ms = e0.elapsed_time(e1) / 3
                if best is None or t_ms < best[0]:
                    best = (t_ms, tile)
                s1.close()
                c1.close()
            sweep_ms += best[0]
            sweep_tiles[best[1]] = sweep_tiles.get(best[1], 0) + 1
    if args.timeline:  # per-circuit duration of one plain pass (fill of the GPU against time)
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(len(jobs) + 1)]
        plain_pass(plain_jobs, marks)
        torch.cuda.synchronize()
        rows = [{"gates": nl.n_gates, "depth": nl.n_levels - 1, "pairs": n, "tile_words": c.info().tile_words,
                 "ctas": -(-P.words(n) // c.info().tile_words), "ms": marks[k].elapsed_time(marks[k + 1])}
                for k, ((c, _, _, _, n, _), nl) in enumerate(zip(plain_jobs, nls))]
        with open(args.timeline, "w") as f:
            json.dump({"plain_pass_ms": plain_ms, "circuits": rows}, f)

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
    b.profile(True)  # forward span and cover of every timed pass, from events inside the graph
    for _ in range(max(3, args.warmup)):
        b.run_async(stream)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    fwd_ms, cov_ms = [], []
    sampler = clock_sampler(torch, local)
    sampler.start()
    time.sleep(0.1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler.mark_start()
    for i in range(args.steps):
        flush.fill_(i & 0xFF)
        ev[i][0].record()
        b.run_async(stream)
        ev[i][1].record()
        f, cv = b.profile_read()  # waits for this pass
        fwd_ms.append(f)
        cov_ms.append(cv)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler.mark_end()
    clocks = sampler.stop()
    b.profile(False)
    ms = max_over_ranks(sum(x.elapsed_time(y) for x, y in ev) / args.steps)
    passes_run = 1 + max(3, args.warmup) + args.steps
    stable = all(a[2].value == passes_run * x[2].value for a, x in zip(results(), batch_res))

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
    if dist:
        dist.barrier()
    t1 = time.perf_counter()
    streamed(args.steps)
    stream_ms = max_over_ranks(1e3 * (time.perf_counter() - t1) / args.steps)
    e2e_ms = max_over_ranks(e2e_ms)
    b2.close()
    info = b.info()
    kernel_ms = sum(fwd_ms) / len(fwd_ms)
    sm_count = torch.cuda.get_device_properties(local).multi_processor_count
    prof = profile_summary(f"k_batch_forward_c4_tile{tw}") if args.circuits == 256 else None
    plain_best = min(plain_ms, plain_bt_ms, sweep_ms or float("inf"))
    line = {
        "metric": "gate-evals/s", "value": world * units / (ms / 1e3), "unit": "gate-evals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": dict(batch_config(members, args), tile_words=tw, threads=threads or "default",
                       parallelism=f"replicas x{world}" if world > 1 else "one GPU",
                       ctas=info.ctas, forward_launches=int(info.forward_launches),
                       autotune={"tile_words": tw, "threads": threads, "ms_per_pass": tune_ms,
                                 "seconds": round(tune_s, 1)} if tune_ms else None),
        "plain": {"value": units / (plain_best / 1e3), "ms_per_pass": plain_best,
                  "ms_per_pass_default_tiles": plain_ms, "ms_per_pass_batch_tile": plain_bt_ms,
                  "ms_per_pass_best_tile_per_circuit": sweep_ms or None,
                  "best_tiles": {str(k): v for k, v in sorted(sweep_tiles.items())} or None,
                  "note": "the same circuits graded one after another (pdf_grade_async each): at each "
                          "circuit's default tile, at the batch's tile, and each at the tile that graded "
                          "it fastest (every tile timed per circuit, 3 calls each); the fastest of these"},
        "batched_vs_plain": plain_best / ms,
        "roofline": dict(roofline(sum(alg_bytes(nl, n) for nl, n in zip(nls, counts)), kernel_ms,
                                  f"forward span of the pass (k_batch_forward{'_lanes' if tw in LANE_TILES else ''}, "
                                  f"every class)", prof, units, sm_count, clocks.get("sm_mhz")),
                         cover_ms=sum(cov_ms) / len(cov_ms)),
        "e2e": {"value": world * units / (stream_ms / 1e3), "unit": "gate-evals/s",
                "h2d_bytes_per_step": int(world * h2d), "d2h_bytes_per_step": 64 * len(jobs) * world,
                "mode": "streamed: pinned host pairs of the next pass copied on a second stream while this "
                        "pass grades (two buffer sets, two batches)",
                "value_one_pass_per_step": world * units / (e2e_ms / 1e3)},
        "gpu_launches": int(info.launches) * args.steps * world,  # forward per class, active, covers, spill cover
        "clocks": clocks,
        "same_config": True,
        "result_stable": bool(same and stable and sweep_same),
        "native_libraries": loaded_libraries(),
    }
    if not args.no_cpu and rank == 0 and world == 1:
        line["cpu_baseline"], line["cpu_baseline_1core"] = cpu_baselines(P, members, args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
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
    # past the 256 circuits of the distribution, the list again with other pairs
    base = P.batch_workload()
    rng = np.random.default_rng(0x5EED0005)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    jobs, nls = [], {}
    for k in range(n_jobs):
        g = base[k % len(base)][0]
        if g.seed not in nls:
            nls[g.seed] = P.gen_netlist(g)
        nl = nls[g.seed]
        v, t = P.gen_pairs(P.pair_seed(g.seed) + k // len(base), nl.n_pi, per_job)
        jobs.append((nl, v, t))
    units = sum(nl.n_gates * per_job for nl, _, _ in jobs)

    def server():
        return P.Server(mark_mode=P.MARK_ROBUST, batch_pairs=batch, hbm_budget=int(args.hbm_gb * (1 << 30)),
                        workers=args.workers, tile_words=args.tile_words or 4)

    # warm-up: a server of its own serves the first `warmup` jobs of the list
    # to completion (kernel modules loaded, allocator and host pools warm);
    # the timed server starts empty
    if args.warmup:
        srv = server()
        for nl, v, t in jobs[:args.warmup]:
            srv.submit(nl, v, t, per_job)
        while srv.stats().jobs_done < min(args.warmup, n_jobs):
            srv.step()
        srv.close()
        torch.cuda.synchronize()
    srv = server()
    ids = [None] * n_jobs
    sampler = clock_sampler(torch, int(os.environ.get("LOCAL_RANK", "0")))
    sampler.start()
    time.sleep(0.1)
    sampler.mark_start()
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
    sampler.mark_end()
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
        "warmup": args.warmup, "ms_per_step": 1e3 * st.busy_s / max(1, st.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded)",
        "config": {"workload": f"c5: {n_jobs} jobs from the c4 size distribution (its 256 circuits in turn), "
                               f"Poisson arrivals at "
                               f"{rate:.0f} jobs/s, {batch}-pair appends up to {per_job} pairs per job",
                   "mark_mode": "robust (LUT_R)", "hbm_budget_gib": args.hbm_gb,
                   "workers": args.workers or "library default", "tile_words": args.tile_words or 4,
                   "outputs": "path count and first-detect ids per job"},
        "latency_ms": {"p50": st.lat_p50_ms, "p99": st.lat_p99_ms, "max": st.lat_max_ms,
                       "per": "job batch, from ready (submission or previous batch) to result"},
        "wall_s": wall, "busy_s": st.busy_s, "gpu_s": st.gpu_s, "batches": int(st.batches),
        # the arrival stream caps throughput: all the work over the span of the arrivals
        "offered_load": units / float(arrivals[-1]),
        "served_fraction_of_offered": float(arrivals[-1]) / wall,
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
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c4", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--mark-mode", choices=sorted(MARK_MODES), default="robust",
                    help="c1-c3: sensitisation table and gate semantics")
    ap.add_argument("--segs", type=int, default=1, help="c1-c3: path segments of this many nets (1-8)")
    ap.add_argument("--tile-words", type=int, default=0,
                    help="words per CTA column block (0 = default; c4: the autotuned width)")
    ap.add_argument("--threads", type=int, default=0,
                    help="threads per CTA, pieces of threads - 64 gates (0 = default; c4: the batch's circuits)")
    ap.add_argument("--pairs", type=int, default=0,
                    help="c1-c3: pairs per rank instead of the workload's (small cases for profiling)")
    # CPU samples, in gate-evals per timed CPU run (0: about 1e9 for the
    # baseline and per reference-arm step, 6e7 for the one-core figure; a
    # few seconds on the host cores)
    ap.add_argument("--cpu-sample", type=float, default=0)
    ap.add_argument("--ref-sample", type=float, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--jobs", type=int, default=512, help="c5: jobs in the arrival stream")
    ap.add_argument("--planes", action="store_true",
                    help="c1-c3: also write the sim and mark planes of every (net, pair) to device memory")
    ap.add_argument("--no-tile-sweep", action="store_true",
                    help="c4: skip timing the plain call of each circuit at every tile")
    ap.add_argument("--timeline", default="",
                    help="c4: write the per-circuit durations of one plain pass to this JSON file")
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
