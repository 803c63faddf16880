"""Benchmark: Goldilocks LDE + Poseidon2 Merkle commitment throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]

A step is one full commitment of the large commitment: 2^22 rows x 176 base columns (128 base
columns plus 24 quadratic-extension columns stored as adjacent c0/c1 base columns) of seeded
synthetic Goldilocks elements: iNTT to monomials, coset LDE factor 2, Poseidon2 leaf hashing of
every row across the 176 columns (22 rate-8 absorptions), node layers up to a cap of 16.  Inputs
are resident in HBM when the timed region starts (5.9 GB, far larger than the 126 MB L2).  Rank 0
prints one JSON line; it also carries the 128 x 2^20 single-size batch and the uneven 300-job
batch (batched against one call per job) as extra keys.

--impl reference times the reference's CPU algorithm for the same workload on the host cores
(the oracle's C restatement of boojum's NTT / LDE / Poseidon2 Merkle routines, all threads, a
bounded sample of the rows per step); boojum itself (Rust) cannot be built here.
Under torchrun each rank runs its own replica (the jobs are independent: weak scaling).
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG_DIR = os.path.join(ROOT, "zksync-crypto-gpu_b200")

# (log2 rows, base columns, log2 LDE factor, log2 cap)
LARGE = (22, 176, 1, 4)
BATCH = (20, 128, 1, 4)
WORKLOADS = {
    LARGE: "2^22 rows x 176 base columns (128 base + 24 extension pairs), iNTT + coset LDE x2 + Poseidon2 Merkle tree (cap 16)",
    BATCH: "128 columns x 2^20 rows, iNTT + coset LDE x2 + Poseidon2 Merkle tree (cap 16)",
}
SEED = "glc-bench"
MODMUL_PER_PERM = 472


def job_units(shape):
    """elements, permutations, algorithmic bytes and modmuls of one commitment."""
    log_n, cols, log_lde, log_cap = shape
    n, f = 1 << log_n, 1 << log_lde
    perms_leaves = f * n * ((cols + 7) // 8)
    perms_nodes = f * n - (1 << log_cap)
    bytes_ = 8 * n * cols * (1 + f) + 64 * f * n
    modmul = cols * (n // 2 * log_n + n) + f * cols * (n + n // 2 * log_n) + MODMUL_PER_PERM * (perms_leaves + perms_nodes)
    return {"elements": n * cols, "perms_leaves": perms_leaves, "perms_nodes": perms_nodes, "bytes": bytes_,
            "modmul": modmul}


def stage_units(shape):
    """Algorithmic modmuls and bytes per stage of one commitment (the split of job_units)."""
    log_n, cols, log_lde, log_cap = shape
    n, f = 1 << log_n, 1 << log_lde
    return {
        "monomials": {"modmul": cols * (n // 2 * log_n + n), "bytes": 32 * n * cols},  # iNTT + bit reversal
        "ntt": {"modmul": f * cols * (n + n // 2 * log_n), "bytes": 16 * f * n * cols},
        "leaves": {"modmul": MODMUL_PER_PERM * f * n * ((cols + 7) // 8), "bytes": f * (8 * n * cols + 32 * n)},
        "nodes": {"modmul": MODMUL_PER_PERM * (f * n - (1 << log_cap)), "bytes": 64 * f * n},
    }


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def load_by_path(name):
    """A module of the package loaded from its file, without importing the package (whose
    __init__ loads libglc.so): the CPU reference arm maps only the oracle's libraries."""
    spec = importlib.util.spec_from_file_location("_glc_bench_" + name, os.path.join(PKG_DIR, name + ".py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def profile_facts():
    """Figures taken from committed ncu captures (profiles/traffic.json): DRAM traffic per leaf
    launch and the probe's instruction mix; None when absent."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            return json.load(fh)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout_s=3.0):
        """Block until the sampler has produced a line (nvidia-smi takes a moment to start), so
        the timed region is covered; returns the index of the next sample."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout_s:
            time.sleep(0.01)
        return len(self.lines)

    def stop(self, since=0):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines[since:]:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [x for x in sm if mx and x > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample_shape(shape):
    """The bounded CPU sample of a workload: the same columns, LDE factor and cap over 2^16 rows."""
    log_n, cols, log_lde, log_cap = shape
    return (min(log_n, 16), cols, log_lde, log_cap)


def cpu_baseline(shape, threads=None, ev=None):
    """The oracle's commitment (C restatement of the reference algorithm, all host threads) on a
    bounded sample of the workload: the same columns, LDE factor and cap over 2^16 rows."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    consts = load_by_path("p2_constants")
    O.set_round_constants(consts.env_round_constants() or consts.grain_lfsr_round_constants())
    threads = threads or os.cpu_count() or 1
    s = cpu_sample_shape(shape)
    if ev is None:
        ev = load_by_path("synthetic").random_field_elements(SEED + "-cpu", s[1] << s[0])
    t0 = time.perf_counter()
    O.commit(np.ascontiguousarray(ev), *s, threads=threads)
    dt = time.perf_counter() - t0
    frac = "1/%d of the rows" % (1 << (shape[0] - s[0]))
    return {"value": (s[1] << s[0]) / dt, "unit": "elements/s", "cores": threads, "kind": "port",
            "sample": "%d columns x 2^%d rows (%s), LDE x%d, cap %d; %.2f s" % (s[1], s[0], frac, 1 << s[2], 1 << s[3], dt),
            "seconds": dt}


def run_reference(args, rank, world):
    if rank != 0:
        return
    s = cpu_sample_shape(LARGE)
    ev = load_by_path("synthetic").random_field_elements(SEED + "-cpu", s[1] << s[0])
    steps = []
    for _ in range(args.warmup):
        cpu_baseline(LARGE, ev=ev)
    for _ in range(args.steps):
        steps.append(cpu_baseline(LARGE, ev=ev))
    v = statistics.median(x["value"] for x in steps)
    ms = statistics.median(x["seconds"] for x in steps) * 1e3
    cb = dict(steps[0])
    cb["value"] = v
    cb.pop("seconds", None)
    line = {"impl": "reference", "metric": "LDE+Merkle commit elements/s", "value": v, "unit": "elements/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded ChaCha20 Goldilocks elements",
            "config": {"workload": WORKLOADS[LARGE], "sample_rows": "2^%d of 2^%d per step (CPU-bounded sample)"
                                                                   % (s[0], LARGE[0])},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "boojum's Rust CPU path cannot be built here (no Rust toolchain); the oracle restates it in C"}
    print(json.dumps(line), flush=True)


def canon_dev(t):
    """x mod p for int64-viewed u64 values: x >= p exactly when -(2^32 - 1) <= x < 0 as int64."""
    import torch
    return torch.where((t < 0) & (t >= -4294967295), t + 4294967295, t)


def same_values(torch, a, b, chunk=1 << 27):
    if a.numel() != b.numel():
        return False
    for i in range(0, a.numel(), chunk):
        if not torch.equal(canon_dev(a[i:i + chunk]), canon_dev(b[i:i + chunk])):
            return False
    return True


def reference_kernels(torch, job, shape, steps):
    """The reference's own CUDA kernels (boojum-cuda native, compiled for sm_100a) driven with the
    reference's per-call launch plans on the same workload, into buffers of their own; then their
    LDE, trees and cap compared bit for bit with this library's.  None when not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import refkern
    except Exception:
        return None
    if not refkern.available():
        return None
    log_n, cols, log_lde, log_cap = shape
    n, f = 1 << log_n, 1 << log_lde
    refkern.call("ref_context_create", 15, 15)
    s = torch.cuda.current_stream().cuda_stream
    mono = torch.empty(cols * n, dtype=torch.int64, device="cuda")
    lde = torch.empty(f * cols * n, dtype=torch.int64, device="cuda")
    trees = torch.empty(f * 8 * n, dtype=torch.int64, device="cuda")
    layers = log_n - (log_cap - log_lde) + 1

    def step():
        refkern.call("ref_batch_ntt", job.evals.data_ptr(), mono.data_ptr(), log_n, cols, n, n, False, True, 0, 0, s)
        refkern.call("ref_bit_reverse", mono.data_ptr(), n, mono.data_ptr(), n, log_n, cols, s)
        for c in range(f):
            coset = int(format(c, "0%db" % log_lde)[::-1], 2)
            dst = lde.data_ptr() + c * cols * n * 8
            refkern.call("ref_batch_ntt", mono.data_ptr(), dst, log_n, cols, n, n, False, False, log_lde, coset, s)
            refkern.call("ref_p2_build_merkle_tree", dst, cols * n, trees.data_ptr() + c * 8 * n * 8, 8 * n, 0,
                         layers, s)

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    refkern.call("ref_context_destroy")
    ccap = 1 << (log_cap - log_lde)
    cap = torch.empty(4 << log_cap, dtype=torch.int64, device="cuda")
    for c in range(f):
        cap.view(4, f * ccap)[:, c * ccap:(c + 1) * ccap] = trees[c * 8 * n + 8 * n - 8 * ccap:
                                                                  c * 8 * n + 8 * n - 4 * ccap].view(4, ccap)
    # each coset's subtree is compared up to its cap: the buffer tail past the cap is written by
    # neither side
    parity = same_values(torch, cap, job.cap) and same_values(torch, lde, job.lde) and all(
        same_values(torch, trees[c * 8 * n: c * 8 * n + 8 * n - 4 * ccap], job.trees[c * 8 * n: c * 8 * n + 8 * n - 4 * ccap])
        for c in range(f))
    del mono, lde, trees, cap
    torch.cuda.empty_cache()
    return {"ms_per_step": e0.elapsed_time(e1) / steps, "parity": bool(parity)}


def modmul_probe(glc, torch, stream):
    """Modular-multiply rate of this device (roofline denominator for the integer kernels)."""
    lib = glc._lib.lib()
    blocks, iters = 148 * 32, 2048
    scratch = torch.empty(blocks * 256, dtype=torch.int64, device="cuda")
    glc._lib.check(lib.glc_modmul_probe(scratch.data_ptr(), blocks, 64, stream.cuda_stream), "probe")
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    glc._lib.check(lib.glc_modmul_probe(scratch.data_ptr(), blocks, iters, stream.cuda_stream), "probe")
    p1.record()
    torch.cuda.synchronize()
    return blocks * 256 * 8 * iters / (p0.elapsed_time(p1) / 1e3)


def make_job(glc, torch, shape, seed, monomials=True):
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    sz = glc.CommitJob.sizes(*shape)
    dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
    job = glc.CommitJob(evals=dev("evals"), log_n=shape[0], cols=shape[1], log_lde=shape[2], log_cap=shape[3],
                        lde=dev("lde"), trees=dev("trees"), cap=dev("cap"), monomials=dev("monomials") if monomials else None)
    syn.fill_device(job.evals, seed)
    return job, sz


def measure_commit(glc, torch, shape, steps, warmup, world, barrier, clocks=None, e2e=True):
    """Times `steps` commitments of `shape` (inputs resident in HBM) with per-stage events, then
    the same through the C ABI end to end with the input copied from pinned host memory."""
    log_n, cols, log_lde, log_cap = shape
    f = 1 << log_lde
    job, sz = make_job(glc, torch, shape, "%s-%d-%d" % (SEED, log_n, cols))
    stream = torch.cuda.current_stream()
    n_ev = 3 + 4 * f
    events = [torch.cuda.Event(enable_timing=True) for _ in range(n_ev)]
    for e in events:  # torch creates the underlying cudaEvent_t on first record
        e.record()
    torch.cuda.synchronize()
    ev_arr = (C.c_void_p * n_ev)(*[e.cuda_event for e in events])
    jstruct = job._struct()
    lib = glc._lib.lib()

    def step(profiled):
        if profiled:
            glc._lib.check(lib.glc_commit_profiled(C.addressof(jstruct), stream.cuda_stream, ev_arr, n_ev),
                           "glc_commit_profiled")
        else:
            glc._lib.check(lib.glc_commit(C.addressof(jstruct), stream.cuda_stream), "glc_commit")

    for _ in range(warmup):
        step(False)
    torch.cuda.synchronize()
    barrier()
    # ---- timed region: inputs resident in HBM ----
    i_clk = clocks.wait_first() if clocks else 0
    stage = {"monomials": 0.0, "ntt": 0.0, "leaves": 0.0, "nodes": 0.0, "caps": 0.0}
    l0 = lib.glc_launch_count()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t_start.record()
    for _ in range(steps):
        step(True)
        torch.cuda.synchronize()  # read the stage events of this step
        stage["monomials"] += events[0].elapsed_time(events[1])
        for c in range(f):  # cosets run on parallel streams: the stage sums can exceed the step
            b = 2 + 4 * c
            stage["ntt"] += events[b].elapsed_time(events[b + 1])
            stage["leaves"] += events[b + 1].elapsed_time(events[b + 2])
            stage["nodes"] += events[b + 2].elapsed_time(events[b + 3])
        stage["caps"] += max(events[2 + 4 * c + 3].elapsed_time(events[n_ev - 1]) for c in range(f))
    t_end.record()
    torch.cuda.synchronize()
    launches = (lib.glc_launch_count() - l0) // max(1, steps)
    clk = clocks.stop(since=i_clk) if clocks else None
    barrier()
    ms = t_start.elapsed_time(t_end) / steps
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    out = {"ms": ms, "stage": {k: v / steps for k, v in stage.items()}, "launches": launches, "clocks": clk,
           "job": job, "sz": sz}
    if not e2e:
        return out

    # ---- end to end through the C ABI with host buffers ----
    # Every step copies its evaluations from pinned host memory and reads its cap back.
    # Pipelined form: two device input buffers, so step i+1's copy (on a copy stream) overlaps
    # step i's commitment; a buffer is refilled only after the commitment that read it is done.
    # The serial form (copy, commit, read back, one after the other) is reported beside it.
    h_in = torch.empty(sz["evals"], dtype=torch.int64, pin_memory=True)
    h_in.copy_(job.evals)
    h_cap = [torch.empty(sz["cap"], dtype=torch.int64, pin_memory=True) for _ in range(2)]
    evals2 = [job.evals, torch.empty_like(job.evals)]
    jobs2 = [job, glc.CommitJob(evals=evals2[1], log_n=log_n, cols=cols, log_lde=log_lde, log_cap=log_cap,
                                lde=job.lde, trees=job.trees, cap=job.cap, monomials=job.monomials)]
    js2 = [j._struct() for j in jobs2]
    copy_stream = torch.cuda.Stream()
    copied = [torch.cuda.Event() for _ in range(2)]
    consumed = [torch.cuda.Event() for _ in range(2)]

    def e2e_pipelined(nsteps):
        copy_stream.wait_stream(stream)
        for i in range(nsteps):
            b = i % 2
            if i >= 2:
                copy_stream.wait_event(consumed[b])
            with torch.cuda.stream(copy_stream):
                evals2[b].copy_(h_in, non_blocking=True)
            copied[b].record(copy_stream)
            stream.wait_event(copied[b])
            glc._lib.check(lib.glc_commit(C.addressof(js2[b]), stream.cuda_stream), "glc_commit")
            consumed[b].record(stream)
            h_cap[b].copy_(job.cap, non_blocking=True)

    def e2e_serial(nsteps):
        for _ in range(nsteps):
            job.evals.copy_(h_in, non_blocking=True)
            step(False)
            h_cap[0].copy_(job.cap, non_blocking=True)

    def timed(fn, nsteps):
        fn(2)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn(nsteps)
        e1.record()
        torch.cuda.synchronize()
        r = e0.elapsed_time(e1) / nsteps
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([r], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            r = float(t.item())
        return r

    e_steps = max(3, steps)
    e2e_ms = timed(e2e_pipelined, e_steps)
    serial_ms = timed(e2e_serial, e_steps)
    units = job_units(shape)
    out["e2e"] = {"value": units["elements"] * world / (e2e_ms / 1e3), "unit": "elements/s", "ms_per_step": e2e_ms,
                  "h2d_bytes_per_step": sz["evals"] * 8, "d2h_bytes_per_step": sz["cap"] * 8, "steps": e_steps,
                  "form": "pipelined: step i+1's host-to-device copy overlaps step i's commitment (two input buffers)",
                  "serial_ms_per_step": serial_ms}
    del evals2[1], jobs2[1], h_in
    return out


def leaf_alone_ms(glc, torch, job, shape):
    """One coset's leaf launch alone on the stream (in the step it shares the GPU with the other
    coset's kernels, which stretches its duration): median of 3, CUDA events."""
    log_n, cols = shape[0], shape[1]
    lr = []
    for _ in range(3):
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        glc.GLHasher.compute_leaf_hashes(job.lde[:cols << log_n], job.trees[:4 << log_n], 0, False, False)
        a1.record()
        torch.cuda.synchronize()
        lr.append(a0.elapsed_time(a1))
    return statistics.median(lr)


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    glc, torch, ctx = _setup_device(local_rank)

    def barrier():
        if world > 1:
            dist.barrier()

    shape = LARGE
    log_n, cols, log_lde, log_cap = shape
    f = 1 << log_lde
    clocks = ClockSampler(local_rank)
    clocks.start()
    m = measure_commit(glc, torch, shape, args.steps, args.warmup, world, barrier, clocks=clocks, e2e=True)
    ms, job = m["ms"], m["job"]
    stage, e2e, clk, launches = m["stage"], m["e2e"], m["clocks"], m["launches"]
    units = job_units(shape)
    value = units["elements"] * world / (ms / 1e3)
    stream = torch.cuda.current_stream()
    mm_peak = modmul_probe(glc, torch, stream)
    peaks, peak_kind = measured_peaks()
    facts = profile_facts()
    leaf_ms = stage["leaves"] / f  # per launch, inside the step
    leaf_modmul = MODMUL_PER_PERM * units["perms_leaves"] / f
    achieved = leaf_modmul / (leaf_ms / 1e3) / 1e9
    alone = leaf_alone_ms(glc, torch, job, shape)
    traffic = facts.get("p2_leaves_kernel_bytes_per_launch_2e22x176")
    t_roof = max(units["bytes"] / (peaks["hbm_gbs"] * 1e9), units["modmul"] / mm_peak)
    ref = None
    if rank == 0 and not args.no_ref_kernels:
        try:
            ref = reference_kernels(torch, job, shape, max(1, min(args.steps, 3)))
        except Exception as ex:  # reported, never fatal
            print("reference kernels not timed: %s" % ex, file=sys.stderr)
    extras = {}
    if world == 1 and not args.no_extras:
        del m, job
        torch.cuda.empty_cache()
        mb = measure_commit(glc, torch, BATCH, max(3, args.steps // 2), args.warmup, 1, barrier, e2e=False)
        ub = job_units(BATCH)
        extras["single_size_batch_128x2e20"] = {
            "workload": WORKLOADS[BATCH], "ms_per_step": mb["ms"], "value": ub["elements"] / (mb["ms"] / 1e3),
            "unit": "elements/s",
            "roofline_job_frac": max(ub["bytes"] / (peaks["hbm_gbs"] * 1e9), ub["modmul"] / mm_peak) / (mb["ms"] / 1e3),
            "leaf_frac_in_step": MODMUL_PER_PERM * ub["perms_leaves"] / (1 << BATCH[2]) / (mb["stage"]["leaves"] / (1 << BATCH[2]) / 1e3) / mm_peak}
        del mb
        torch.cuda.empty_cache()
        try:
            budget = min(args.budget_gb, 120.0)
            extras["uneven_batch_300_jobs"] = uneven_batch(glc, torch, budget_gb=budget, streams=args.streams,
                                                           with_reference=not args.no_ref_kernels)
            small = [j for j in uneven_jobs() if j[0] <= 15]
            extras["uneven_batch_small_jobs"] = uneven_batch(glc, torch, budget_gb=budget, streams=args.streams,
                                                             with_reference=not args.no_ref_kernels, jobs=small)
            extras["uneven_batch_small_jobs"]["workload"] = ("uneven batch, small jobs only (log2 rows <= 15): %d of "
                                                             "the 300 jobs" % len(small))
        except Exception as ex:
            print("uneven batch not run: %s" % ex, file=sys.stderr)
    cpu = cpu_baseline(shape) if (rank == 0 and world == 1) else None
    if cpu:
        cpu.pop("seconds", None)
    line = {
        "metric": "LDE+Merkle commit elements/s",
        "value": value, "unit": "elements/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: seeded ChaCha20 uniform Goldilocks elements (glc_fill_random)",
        "config": {"workload": WORKLOADS[shape], "log_rows": log_n, "base_columns": cols,
                   "extension_columns": 24, "lde_factor": f, "cap": 1 << log_cap,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs 5.9 GB > 126 MB L2, no flush"},
        "hashes_per_s": (units["perms_leaves"] + units["perms_nodes"]) * world / (ms / 1e3),
        "algorithmic_gbs": units["bytes"] * world / (ms / 1e3) / 1e9,
        "stages_ms": stage,
        # per stage: algorithmic work, its roofline time, and that over the stage's in-step time
        # (the coset stages run on two streams at once, so their in-step times overlap)
        "stages_roofline": {k: dict(u, roof_ms=max(u["bytes"] / (peaks["hbm_gbs"] * 1e9), u["modmul"] / mm_peak) * 1e3,
                                    frac=max(u["bytes"] / (peaks["hbm_gbs"] * 1e9), u["modmul"] / mm_peak) * 1e3
                                    / max(1e-9, stage[k]))
                            for k, u in stage_units(shape).items()},
        "roofline": {"bound": "int", "kernel": "p2_leaves_kernel", "achieved": achieved,
                     "peak": mm_peak / 1e9, "unit": "Gmodmul/s", "frac": achieved * 1e9 / mm_peak,
                     "launch_ms_in_step": leaf_ms, "launch_ms_alone": alone,
                     "frac_alone": leaf_modmul / (alone / 1e3) / mm_peak,
                     "hbm_gbs_alone": (traffic or 0) / (alone / 1e3) / 1e9,
                     "hbm_frac_alone": (traffic or 0) / (alone / 1e3) / 1e9 / peaks["hbm_gbs"],
                     "traffic": traffic,
                     "probe_warp_inst_per_modmul": facts.get("probe_warp_inst_per_modmul"),
                     "peak_source": "glc_modmul_probe measured live in this run (8 independent multiply chains per "
                                    "thread on every SM)"},
        "roofline_job": {"bytes": units["bytes"], "modmul": units["modmul"], "t_roof_ms": t_roof * 1e3,
                         "frac": t_roof * 1e3 / ms, "hbm_gbs": peaks["hbm_gbs"], "hbm_source": peak_kind,
                         "modmul_peak_gs": mm_peak / 1e9},
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    if ref:
        line["reference_kernels_sm100a"] = {"ms_per_step": ref["ms_per_step"],
                                            "value": units["elements"] / (ref["ms_per_step"] / 1e3),
                                            "unit": "elements/s", "speedup": ref["ms_per_step"] / ms,
                                            "what": "boojum-cuda native kernels recompiled for sm_100a, reference launch plans"}
        line["parity_vs_reference_kernels"] = ref["parity"]
    line.update(extras)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.destroy()


def _setup_device(local_rank=0):
    import torch
    glc = importlib.import_module("zksync-crypto-gpu_b200")
    torch.cuda.set_device(local_rank)
    ctx = glc.Context.create(15, 15)
    consts = importlib.import_module("zksync-crypto-gpu_b200.p2_constants")
    rc = consts.env_round_constants()
    if rc:
        glc.poseidon2.set_round_constants(rc)
    tune_path = os.path.join(ROOT, "zksync-crypto-gpu_b200", "tuning_b200.txt")
    if os.path.exists(tune_path):
        glc.tuning.load(tune_path)
    return glc, torch, ctx


def uneven_jobs(n_jobs=300, seed=7):
    """The uneven batch: log2 rows uniform in 12..22, columns in {8,16,32,64,128}, LDE factor 2 or
    4 (50/50), cap 16; drawn from a seeded generator."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(12, 23)), int(rng.choice([8, 16, 32, 64, 128])), int(rng.choice([1, 2])), 4)
            for _ in range(n_jobs)]


def uneven_batch(glc, torch, budget_gb=120.0, streams=8, with_reference=True, jobs=None):
    """Batched (multi-stream + CUDA graph) vs plain one-call-per-job on the uneven batch.  The 300
    jobs hold ~100 GB of inputs and ~300 GB of outputs, so they run in waves that fit a device
    budget; every form processes every job.  Also splits the time of the small jobs (at most
    2^15 rows) from the rest."""
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    jobs = jobs or uneven_jobs()
    budget = int(budget_gb * (1 << 30))
    waves, cur, used = [], [], 0
    for j in sorted(jobs, key=lambda j: -(j[1] << j[0])):
        sz = glc.CommitJob.sizes(*j)
        b = 8 * (sz["evals"] + sz["lde"] + sz["trees"] + sz["cap"])
        if cur and used + b > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(j)
        used += b
    waves.append(cur)
    stream = torch.cuda.current_stream()
    t = {"plain": 0.0, "batched": 0.0, "graph": 0.0, "fused": 0.0, "reference_kernels": 0.0}
    fused = all(l <= 22 for l, _, _, _ in jobs)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import refkern
        have_ref = with_reference and refkern.available()
    except Exception:
        have_ref = False
    if have_ref:
        refkern.call("ref_context_create", 15, 15)
    elements = sum(c << l for l, c, _, _ in jobs)
    caps_equal = True
    for wi, wave in enumerate(waves):
        bufs = []
        for i, (l, c, e, cap) in enumerate(wave):
            sz = glc.CommitJob.sizes(l, c, e, cap)
            dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
            jb = glc.CommitJob(evals=dev("evals"), log_n=l, cols=c, log_lde=e, log_cap=cap, lde=dev("lde"),
                               trees=dev("trees"), cap=dev("cap"))
            syn.fill_device(jb.evals, "uneven-%d-%d" % (wi, i))
            bufs.append(jb)
        # warm up every form once (also the graph instantiation), then time one pass of each
        for jb in bufs:
            glc.commit.commit(jb)
        graph = glc.CommitGraph(bufs, n_streams=streams)
        graph.launch()
        torch.cuda.synchronize()
        caps_graph = [jb.cap.clone() for jb in bufs]
        # the fused form: one cooperative launch for every stage of every job of the wave
        forms = ("plain", "batched", "graph") + (("fused",) if fused else ())
        if fused:
            glc.commit.commit_batch_fused(bufs, stream)
            torch.cuda.synchronize()
        for form in forms:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if form == "plain":
                for jb in bufs:
                    glc.commit.commit(jb, stream)
            elif form == "batched":
                glc.commit.commit_batch(bufs, n_streams=streams)
            elif form == "graph":
                graph.launch()
            else:
                glc.commit.commit_batch_fused(bufs, stream)
            e1.record()
            torch.cuda.synchronize()
            t[form] += e0.elapsed_time(e1)
            caps_equal &= all(bool((a == jb.cap).all()) for a, jb in zip(caps_graph, bufs))
        graph.close()
        if have_ref:
            # the reference's own kernels, one call sequence per job (its per-call form)
            s_ = stream.cuda_stream
            mono = torch.empty(max(jb.cols << jb.log_n for jb in bufs), dtype=torch.int64, device="cuda")

            def ref_job(jb):
                n, f = 1 << jb.log_n, 1 << jb.log_lde
                refkern.call("ref_batch_ntt", jb.evals.data_ptr(), mono.data_ptr(), jb.log_n, jb.cols, n, n, False, True,
                             0, 0, s_)
                refkern.call("ref_bit_reverse", mono.data_ptr(), n, mono.data_ptr(), n, jb.log_n, jb.cols, s_)
                layers = jb.log_n - (jb.log_cap - jb.log_lde) + 1
                for c in range(f):
                    coset = int(format(c, "0%db" % jb.log_lde)[::-1], 2)
                    dst = jb.lde.data_ptr() + c * jb.cols * n * 8
                    refkern.call("ref_batch_ntt", mono.data_ptr(), dst, jb.log_n, jb.cols, n, n, False, False,
                                 jb.log_lde, coset, s_)
                    refkern.call("ref_p2_build_merkle_tree", dst, jb.cols * n, jb.trees.data_ptr() + c * 8 * n * 8,
                                 8 * n, 0, layers, s_)
            for jb in bufs[:4]:
                ref_job(jb)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for jb in bufs:
                ref_job(jb)
            e1.record()
            torch.cuda.synchronize()
            t["reference_kernels"] += e0.elapsed_time(e1)
            del mono
        del bufs
        torch.cuda.empty_cache()
    line = {"workload": "uneven batch: 300 jobs, log2 rows U{12..22}, columns {8..128}, LDE x2/x4, cap 16",
            "metric": "LDE+Merkle commit elements/s", "unit": "elements/s", "waves": len(waves),
            "plain": {"ms": t["plain"], "value": elements / (t["plain"] / 1e3)},
            "batched_streams": {"ms": t["batched"], "value": elements / (t["batched"] / 1e3)},
            "batched_graph": {"ms": t["graph"], "value": elements / (t["graph"] / 1e3)},
            "speedup_graph_vs_plain": t["plain"] / t["graph"], "speedup_streams_vs_plain": t["plain"] / t["batched"],
            "reference_kernels_per_call": ({"ms": t["reference_kernels"],
                                            "value": elements / (t["reference_kernels"] / 1e3),
                                            "speedup_graph_vs_reference": t["reference_kernels"] / t["graph"]}
                                           if have_ref else None),
            "caps_identical_across_forms": caps_equal, "streams": streams}
    if fused:
        line["batched_fused_one_launch"] = {"ms": t["fused"], "value": elements / (t["fused"] / 1e3),
                                            "speedup_vs_plain": t["plain"] / t["fused"],
                                            "speedup_vs_graph": t["graph"] / t["fused"],
                                            "speedup_vs_reference": (t["reference_kernels"] / t["fused"]
                                                                     if have_ref else None)}
    return line


def run_uneven(args):
    glc, torch, ctx = _setup_device()
    budget = min(args.budget_gb, 120.0)
    print(json.dumps(uneven_batch(glc, torch, budget, args.streams, not args.no_ref_kernels)), flush=True)
    small = [j for j in uneven_jobs() if j[0] <= 15]
    line = uneven_batch(glc, torch, budget, args.streams, not args.no_ref_kernels, jobs=small)
    line["workload"] = "uneven batch, small jobs only (log2 rows <= 15): %d of the 300 jobs" % len(small)
    print(json.dumps(line), flush=True)
    ctx.destroy()


def serve_jobs(n, seed=11):
    """Serving mix: log2 rows U[16,23], columns U[8,256], LDE factor 2 or 4, cap 16."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(16, 24)), int(rng.integers(8, 257)), int(rng.choice([1, 2])), 4) for _ in range(n)]


def run_serve(args):
    """Poisson arrivals of commitment jobs served with continuous batching under an HBM budget,
    against the plain sequential form (one request on the device at a time).  First the
    saturation throughput (all jobs submitted at once), then an offered-load sweep: half of
    saturation, 0.9 of it, and the configured rate; p50/p99 latency per point.  Host inputs: one
    pinned buffer of seeded synthetic elements, each request reading its prefix."""
    import numpy as np
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    jobs = serve_jobs(args.serve_jobs)
    max_elems = max(c << l for l, c, _, _ in jobs)
    host = torch.empty(max_elems, dtype=torch.int64, pin_memory=True)
    chunk = 1 << 28
    d = torch.empty(min(chunk, max_elems), dtype=torch.int64, device="cuda")
    for i in range(0, max_elems, chunk):
        k = min(chunk, max_elems - i)
        syn.fill_device(d[:k], "serve", i)
        host[i:i + k].copy_(d[:k])
    del d
    torch.cuda.empty_cache()
    base = host.numpy().view(np.uint64)
    make = lambda i, l, c: base[:c << l]
    budget = int(args.budget_gb * (1 << 30))
    arms = {"continuous_batching": dict(max_inflight=args.inflight, streams=args.streams, size_priority=True),
            "plain_sequential": dict(max_inflight=1, streams=1, size_priority=False)}
    elements = sum(c << l for l, c, _, _ in jobs)
    out = {"workload": "serving: %d jobs, log2 rows U[16,23], columns U[8,256], LDE x2/x4, cap 16" % len(jobs),
           "budget_gb": args.budget_gb, "elements": elements}

    def point(arm, rate):
        with glc.serve.Server(hbm_budget_bytes=budget, **arms[arm]) as srv:
            r = glc.serve.poisson_load(srv, jobs, rate_per_s=rate, seed=3, make_input=make)
            st = srv.stats()
        r.pop("caps")
        r["offered_per_s"] = rate if rate > 0 else None
        r["peak_inflight"] = st["peak_inflight"]
        r["peak_gb"] = st["peak_bytes"] / (1 << 30)
        return r

    sat = {arm: point(arm, 0) for arm in arms}
    out["saturation"] = sat
    s = sat["continuous_batching"]["jobs_per_s"]
    rates = [("half_saturation", 0.5 * s), ("near_saturation", 0.9 * s), ("configured_200_per_s", args.rate)]
    out["sweep"] = {name: {arm: point(arm, rate) for arm in arms} for name, rate in rates}
    print(json.dumps(out), flush=True)
    ctx.destroy()


def run_ef(args):
    """Extension-field layout conversion of the 24 extension columns of the 2^22-row trace
    (vectorized <-> tuples, 16 bytes read + 16 written per element): HBM roofline."""
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    rows, cols = 1 << args.ef_log_rows, 24
    v = torch.empty(2 * cols * rows, dtype=torch.int64, device="cuda")
    syn.fill_device(v, "ef")
    t = torch.empty_like(v)
    peaks, kind = measured_peaks()
    out = {"workload": "GoldilocksExt2 layouts: 24 extension columns x 2^%d rows" % args.ef_log_rows,
           "hbm_gbs_peak": peaks["hbm_gbs"], "peak_source": kind}
    for name, fn, a, b in (("vectorized_to_tuples", glc.extension_field.vectorized_to_tuples, v, t),
                           ("tuples_to_vectorized", glc.extension_field.tuples_to_vectorized, t, v)):
        for _ in range(args.warmup):
            fn(a, b, rows, cols)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn(a, b, rows, cols)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        gbs = 32 * rows * cols / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "GB/s": gbs, "frac_of_hbm": gbs / peaks["hbm_gbs"]}
    print(json.dumps(out), flush=True)
    ctx.destroy()


def run_witness(args):
    """Witness-to-trace fill of the large commitment's trace: 2^22 rows (--witness-log-rows) x 176 columns (150
    variable, 25 witness, 1 multiplicity) gathered from 2^28 witness values by seeded random u32
    indexes (3% placeholders), multiplicities for 3/4 of the rows.  HBM-bound gather: per element
    4 bytes of index and 8 of value read, 8 written (algorithmic); the value read is a separate
    32-byte DRAM sector at random indexes.  Also the reference's select kernel on the same indexes,
    compared element for element."""
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    log_n, nv, nw, nm = args.witness_log_rows, 150, 25, 1
    n = 1 << log_n
    n_values = 1 << 28
    values = torch.empty(n_values, dtype=torch.int64, device="cuda")
    syn.fill_device(values, "witness-values")
    gen = torch.Generator(device="cuda").manual_seed(17)
    def indexes(count):
        ix = torch.randint(0, n_values, (count,), generator=gen, device="cuda", dtype=torch.int64)
        ph = torch.rand(count, generator=gen, device="cuda") < 0.03
        return (ix | (ph.to(torch.int64) << 31)).to(torch.int32)
    vi, wi = indexes(nv * n), indexes(nw * n)
    mult = torch.randint(0, 1 << 20, (3 * n // 4,), generator=gen, device="cuda", dtype=torch.int32)
    trace = torch.empty((nv + nw + nm) * n, dtype=torch.int64, device="cuda")
    fill = lambda: glc.trace.fill_from_remote_witness_data(vi, wi, values, mult, trace, nv, nw, nm, n)
    peaks, kind = measured_peaks()
    for _ in range(max(args.warmup, 1)):
        fill()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fill()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    elems = (nv + nw + nm) * n
    gathered = (nv + nw) * n
    alg = 20 * gathered + 12 * n * nm
    sectors = (4 + 32 + 8) * gathered + 12 * n * nm
    out = {"workload": "witness-to-trace fill: 2^%d rows x 176 columns (150 variable, 25 witness, 1 multiplicity) "
                       "from 2^28 values, random indexes, 3%% placeholders" % log_n,
           "ms": ms, "elements_per_s": elems / (ms / 1e3), "algorithmic_gbs": alg / (ms / 1e3) / 1e9,
           "sector_gbs": sectors / (ms / 1e3) / 1e9, "hbm_gbs_peak": peaks["hbm_gbs"], "peak_source": kind,
           "frac_sector_traffic_of_hbm": sectors / (ms / 1e3) / 1e9 / peaks["hbm_gbs"]}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import refkern
        have_ref = refkern.available()
    except Exception:
        have_ref = False
    if have_ref:
        ref = torch.empty_like(trace)
        s_ = torch.cuda.current_stream().cuda_stream
        def ref_fill():
            refkern.call("ref_select", vi.data_ptr(), values.data_ptr(), ref.data_ptr(), nv * n, s_)
            refkern.call("ref_select", wi.data_ptr(), values.data_ptr(), ref.data_ptr() + 8 * nv * n, nw * n, s_)
        ref_fill()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            ref_fill()
        e1.record()
        torch.cuda.synchronize()
        rms = e0.elapsed_time(e1) / args.steps
        out["reference_select_kernel"] = {"ms_for_the_selects": rms, "speedup_of_the_selects": None,
                                          "parity": bool((ref[:gathered] == trace[:gathered]).all())}
        # this build's selects alone (the multiplicity column is not part of the reference kernel)
        e0.record()
        for _ in range(args.steps):
            glc.ops_complex.select(vi, values, trace[:nv * n])
            glc.ops_complex.select(wi, values, trace[nv * n:gathered])
        e1.record()
        torch.cuda.synchronize()
        ours = e0.elapsed_time(e1) / args.steps
        out["reference_select_kernel"]["speedup_of_the_selects"] = rms / ours
        out["selects_ms"] = ours
    print(json.dumps(out), flush=True)
    ctx.destroy()


def run_queries(args):
    """Query openings on the 128 x 2^20 commitment (LDE x2, cap 16): for 100 seeded query indexes
    of one coset, gather the 100 rows of the 128 LDE columns (gather_rows) and the 17-layer Merkle
    paths of the 2^20-leaf subtree (gather_merkle_paths)."""
    import numpy as np
    glc, torch, ctx = _setup_device()
    log_n, cols, log_lde, log_cap = BATCH
    n = 1 << log_n
    jb, _ = make_job(glc, torch, BATCH, "queries", monomials=False)
    glc.commit.commit(jb)
    q = 100
    idx = torch.from_numpy(np.random.default_rng(5).integers(0, n, q).astype(np.int32)).cuda()
    layers = log_n - (log_cap - log_lde)
    rows = torch.empty(q * cols, dtype=torch.int64, device="cuda")
    paths = torch.empty(layers * 4 * q, dtype=torch.int64, device="cuda")
    lde0, tree0 = jb.lde[:cols * n], jb.trees[:8 * n]
    calls = {"gather_rows": lambda: glc.GLHasher.gather_rows(idx, 0, lde0, n, cols, rows, q, cols),
             "gather_merkle_paths": lambda: glc.GLHasher.gather_merkle_paths(idx, tree0, paths, layers)}
    out = {"workload": "query openings: 100 indexes, 128 columns x 2^20 rows, 17-layer paths (cap 16 over 2 cosets)"}
    for name, fn in calls.items():
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        reps = 200
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        us = e0.elapsed_time(e1) / reps * 1e3
        out[name] = {"us_per_call": us, "queries_per_s": q / (us / 1e6)}
    print(json.dumps(out), flush=True)
    ctx.destroy()


def run_profile_case(args):
    """A small commitment for profiler captures: --cols columns x 2^--log-n rows (default 176 x
    2^18, 369 MB of inputs, still larger than L2), LDE x2, cap 16; warm-up plus a few plain
    glc_commit calls."""
    glc, torch, ctx = _setup_device()
    shape = (args.log_n, args.cols, 1, 4)
    jb, _ = make_job(glc, torch, shape, "profile", monomials=False)
    for _ in range(args.warmup):
        glc.commit.commit(jb)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        glc.commit.commit(jb)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"workload": "profile case: %d columns x 2^%d rows, LDE x2, cap 16" % (args.cols, args.log_n),
                      "ms_per_step": ms, "value": (args.cols << args.log_n) / (ms / 1e3), "unit": "elements/s"}),
          flush=True)
    ctx.destroy()


def run_fused_trace(args):
    """The fused launch on the uneven batch's small jobs (log2 rows <= 15), with its per-item
    trace: where the CTAs spent their time (commit.fused_trace_summary) and the launch's time."""
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    jobs = [j for j in uneven_jobs() if j[0] <= 15]
    bufs = []
    for i, (l, c, e, cap) in enumerate(jobs):
        sz = glc.CommitJob.sizes(l, c, e, cap)
        dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
        bufs.append(glc.CommitJob(evals=dev("evals"), log_n=l, cols=c, log_lde=e, log_cap=cap, lde=dev("lde"),
                                  trees=dev("trees"), cap=dev("cap")))
        syn.fill_device(bufs[-1].evals, "uneven-0-%d" % i)
    trace = torch.zeros(4 << 20, dtype=torch.int64, device="cuda")
    for _ in range(max(args.warmup, 1)):
        glc.commit.commit_batch_fused(bufs)
    ms = []
    for _ in range(max(args.steps, 1)):
        trace.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        glc.commit.commit_batch_fused(bufs, trace=trace)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    summary = glc.commit.fused_trace_summary(trace.cpu().numpy().view("uint64"))
    print(json.dumps({"workload": "fused launch, uneven batch small jobs (log2 rows <= 15): %d jobs" % len(jobs),
                      "ms_per_launch": sorted(ms)[len(ms) // 2], "trace_of_last_launch": summary,
                      "timeouts": glc.commit.fused_timeouts()}), flush=True)
    ctx.destroy()


def run_probe(args):
    """The modular-multiply probe alone (the roofline denominator), for instruction-mix captures."""
    glc, torch, ctx = _setup_device()
    rate = modmul_probe(glc, torch, torch.cuda.current_stream())
    print(json.dumps({"workload": "glc_modmul_probe: 148 x 32 blocks x 256 threads, 8 chains x 2048 multiplies",
                      "Gmodmul_s": rate / 1e9}), flush=True)
    ctx.destroy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-ref-kernels", action="store_true", help="skip the reference-kernel timing and parity leg")
    ap.add_argument("--no-extras", action="store_true", help="skip the 128 x 2^20 and uneven-batch extra keys")
    ap.add_argument("--workload", default="commit",
                    choices=["commit", "uneven", "serve", "profile", "ef", "queries", "probe", "fused-trace",
                             "witness"],
                    help="commit: the contract line; others print their own JSON")
    ap.add_argument("--log-n", type=int, default=18, help="rows of the profile case (log2)")
    ap.add_argument("--cols", type=int, default=176, help="columns of the profile case")
    ap.add_argument("--ef-log-rows", type=int, default=22, help="rows of the extension-layout workload (log2)")
    ap.add_argument("--witness-log-rows", type=int, default=22, help="rows of the witness-fill workload (log2)")
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-jobs", type=int, default=400)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--inflight", type=int, default=8)
    args = ap.parse_args()
    if args.workload != "commit":
        {"uneven": run_uneven, "serve": run_serve, "profile": run_profile_case, "ef": run_ef,
         "queries": run_queries, "probe": run_probe, "fused-trace": run_fused_trace,
         "witness": run_witness}[args.workload](args)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
