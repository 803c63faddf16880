"""Benchmark: Goldilocks LDE + Poseidon2 Merkle commitment throughput on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one full commitment of the headline workload (128 columns x 2^20 rows of seeded
synthetic Goldilocks elements: iNTT to monomials, LDE factor 2, Poseidon2 leaf hashing of every
row across the 128 columns, node layers up to a cap of 16).  Inputs are resident in HBM when
the timed region starts (1 GiB, larger than the 126 MB L2).  Rank 0 prints one JSON line.

--impl reference times the reference's CPU algorithm for the same workload on the host cores
(the oracle's C restatement of boojum's NTT / LDE / Poseidon2 Merkle routines, all threads, a
bounded sample per step); boojum itself (Rust) cannot be built here.
Under torchrun each rank runs its own replica (the jobs are independent: weak scaling).
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LOG_N, COLS, LOG_LDE, LOG_CAP = 20, 128, 1, 4
WORKLOAD = "128 columns x 2^20 rows, iNTT + coset LDE x2 + Poseidon2 Merkle tree (cap 16)"
SEED = "glc-bench-c2"
MODMUL_PER_PERM = 472


def job_units(log_n=LOG_N, cols=COLS, log_lde=LOG_LDE, log_cap=LOG_CAP):
    """elements, permutations, algorithmic bytes and modmuls of one commitment."""
    n, f = 1 << log_n, 1 << log_lde
    perms_leaves = f * n * ((cols + 7) // 8)
    perms_nodes = f * n - (1 << log_cap)
    bytes_ = 8 * n * cols * (1 + f) + 64 * f * n
    modmul = cols * (n // 2 * log_n + n) + f * cols * (n + n // 2 * log_n) + MODMUL_PER_PERM * (perms_leaves + perms_nodes)
    return {"elements": n * cols, "perms_leaves": perms_leaves, "perms_nodes": perms_nodes, "bytes": bytes_,
            "modmul": modmul}


def stage_units(log_n=LOG_N, cols=COLS, log_lde=LOG_LDE, log_cap=LOG_CAP):
    """Algorithmic modmuls and bytes per stage of one commitment (the split of job_units)."""
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


def cpu_baseline(threads=None):
    """The oracle's commitment (C restatement of the reference algorithm) on a bounded sample
    of the same workload shape: 128 columns x 2^16 rows, LDE x2, cap 16."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    consts = importlib.import_module("zksync-crypto-gpu_b200.p2_constants")
    O.set_round_constants(consts.env_round_constants() or consts.grain_lfsr_round_constants())
    threads = threads or os.cpu_count() or 1
    log_n = 16
    ev = syn.random_field_elements(SEED + "-cpu", COLS << log_n)
    t0 = time.perf_counter()
    O.commit(np.ascontiguousarray(ev), log_n, COLS, LOG_LDE, LOG_CAP, threads=threads)
    dt = time.perf_counter() - t0
    return {"value": (COLS << log_n) / dt, "unit": "elements/s", "cores": threads, "kind": "port",
            "sample": "128 columns x 2^16 rows (1/16 of the rows), LDE x2, cap 16; %.2f s" % dt, "seconds": dt}


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps = []
    for _ in range(args.warmup):
        cpu_baseline()
    for _ in range(args.steps):
        steps.append(cpu_baseline())
    v = statistics.median(s["value"] for s in steps)
    ms = statistics.median(s["seconds"] for s in steps) * 1e3
    cb = dict(steps[0])
    cb["value"] = v
    cb.pop("seconds", None)
    line = {"impl": "reference", "metric": "LDE+Merkle commit elements/s", "value": v, "unit": "elements/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic: seeded ChaCha20 Goldilocks elements",
            "config": {"workload": WORKLOAD, "sample_rows": "2^16 of 2^20 per step (CPU-bounded sample)"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "boojum's Rust CPU path cannot be built here (no Rust toolchain); the oracle restates it in C"}
    print(json.dumps(line), flush=True)


def reference_kernels_ms(glc, torch, job, steps):
    """The reference's own CUDA kernels (boojum-cuda native, compiled for sm_100a) driven with the
    reference's per-call launch plans on the same workload; None when not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import refkern
    except Exception:
        return None
    if not refkern.available():
        return None
    n, f = 1 << LOG_N, 1 << LOG_LDE
    refkern.call("ref_context_create", 15, 15)
    s = torch.cuda.current_stream().cuda_stream
    mono = torch.empty(COLS * n, dtype=torch.int64, device="cuda")
    layers = LOG_N - (LOG_CAP - LOG_LDE) + 1

    def step():
        refkern.call("ref_batch_ntt", job.evals.data_ptr(), mono.data_ptr(), LOG_N, COLS, n, n, False, True, 0, 0, s)
        refkern.call("ref_bit_reverse", mono.data_ptr(), n, mono.data_ptr(), n, LOG_N, COLS, s)
        for c in range(f):
            coset = int(format(c, "0%db" % LOG_LDE)[::-1], 2)
            dst = job.lde.data_ptr() + c * COLS * n * 8
            refkern.call("ref_batch_ntt", mono.data_ptr(), dst, LOG_N, COLS, n, n, False, False, LOG_LDE, coset, s)
            refkern.call("ref_p2_build_merkle_tree", dst, COLS * n, job.trees.data_ptr() + c * 8 * n * 8, 8 * n, 0,
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
    del mono
    return e0.elapsed_time(e1) / steps


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    glc = importlib.import_module("zksync-crypto-gpu_b200")
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    consts = importlib.import_module("zksync-crypto-gpu_b200.p2_constants")
    torch.cuda.set_device(local_rank)
    ctx = glc.Context.create(15, 15)
    rc = consts.env_round_constants()
    if rc:
        glc.poseidon2.set_round_constants(rc)
    tune_path = os.path.join(ROOT, "zksync-crypto-gpu_b200", "tuning_b200.txt")
    if os.path.exists(tune_path):
        glc.tuning.load(tune_path)
    n, f = 1 << LOG_N, 1 << LOG_LDE
    sz = glc.CommitJob.sizes(LOG_N, COLS, LOG_LDE, LOG_CAP)
    dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
    job = glc.CommitJob(evals=dev("evals"), log_n=LOG_N, cols=COLS, log_lde=LOG_LDE, log_cap=LOG_CAP,
                        lde=dev("lde"), trees=dev("trees"), cap=dev("cap"), monomials=dev("monomials"))
    syn.fill_device(job.evals, "%s-rank%d" % (SEED, rank))
    stream = torch.cuda.current_stream()
    n_ev = 3 + 4 * f
    events = [torch.cuda.Event(enable_timing=True) for _ in range(n_ev)]
    for e in events:  # torch creates the underlying cudaEvent_t on first record
        e.record()
    torch.cuda.synchronize()
    assert all(e.cuda_event for e in events)
    ev_arr = (C.c_void_p * n_ev)(*[e.cuda_event for e in events])
    jstruct = job._struct()
    lib = glc._lib.lib()

    def step(profiled):
        if profiled:
            glc._lib.check(lib.glc_commit_profiled(C.addressof(jstruct), stream.cuda_stream, ev_arr, n_ev),
                           "glc_commit_profiled")
        else:
            glc._lib.check(lib.glc_commit(C.addressof(jstruct), stream.cuda_stream), "glc_commit")

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    barrier()
    # ---- timed region: inputs resident in HBM ----
    clocks = ClockSampler(local_rank)
    clocks.start()
    i_clk = clocks.wait_first()
    stage = {"monomials": 0.0, "ntt": 0.0, "leaves": 0.0, "nodes": 0.0, "caps": 0.0}
    l0 = lib.glc_launch_count()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t_start.record()
    for _ in range(args.steps):
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
    launches = (lib.glc_launch_count() - l0) // max(1, args.steps)
    clk = clocks.stop(since=i_clk)
    barrier()
    ms = t_start.elapsed_time(t_end) / args.steps
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    units = job_units()
    value = units["elements"] * world / (ms / 1e3)

    # ---- end to end through the C ABI with host buffers ----
    # Every step copies its 1 GiB of evaluations from pinned host memory and reads its cap back.
    # Pipelined form: two device input buffers, so step i+1's copy (on a copy stream) overlaps
    # step i's commitment; a buffer is refilled only after the commitment that read it is done.
    # The serial form (copy, commit, read back, one after the other) is reported beside it.
    h_in = torch.empty(sz["evals"], dtype=torch.int64, pin_memory=True)
    h_in.copy_(job.evals)
    h_cap = [torch.empty(sz["cap"], dtype=torch.int64, pin_memory=True) for _ in range(2)]
    evals2 = [job.evals, torch.empty_like(job.evals)]
    jobs2 = [job, glc.CommitJob(evals=evals2[1], log_n=LOG_N, cols=COLS, log_lde=LOG_LDE, log_cap=LOG_CAP,
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
            t = torch.tensor([r], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            r = float(t.item())
        return r

    e_steps = max(3, args.steps)
    e2e_ms = timed(e2e_pipelined, e_steps)
    serial_ms = timed(e2e_serial, e_steps)
    e2e = {"value": units["elements"] * world / (e2e_ms / 1e3), "unit": "elements/s", "ms_per_step": e2e_ms,
           "h2d_bytes_per_step": sz["evals"] * 8, "d2h_bytes_per_step": sz["cap"] * 8, "steps": e_steps,
           "form": "pipelined: step i+1's host-to-device copy overlaps step i's commitment (two input buffers)",
           "serial_ms_per_step": serial_ms}
    del evals2[1], jobs2[1]

    # ---- modular-multiply peak of this device (roofline denominator for integer kernels) ----
    blocks = 148 * 32
    scratch = torch.empty(blocks * 256, dtype=torch.int64, device="cuda")
    iters = 2048
    glc._lib.check(lib.glc_modmul_probe(scratch.data_ptr(), blocks, 64, stream.cuda_stream), "probe")
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    glc._lib.check(lib.glc_modmul_probe(scratch.data_ptr(), blocks, iters, stream.cuda_stream), "probe")
    p1.record()
    torch.cuda.synchronize()
    mm_peak = blocks * 256 * 8 * iters / (p0.elapsed_time(p1) / 1e3)

    peaks, peak_kind = measured_peaks()
    leaf_ms = stage["leaves"] / (args.steps * f)  # per launch
    leaf_modmul = MODMUL_PER_PERM * units["perms_leaves"] / f
    achieved = leaf_modmul / (leaf_ms / 1e3) / 1e9
    # the same leaf launch alone on the stream (in the step it shares the GPU with the other
    # coset's NTT, which stretches its duration): one coset of the LDE, 3 launches, events
    lr = []
    for _ in range(3):
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        glc.GLHasher.compute_leaf_hashes(job.lde[:COLS << LOG_N], job.trees[:4 << LOG_N], 0, False, False)
        a1.record()
        torch.cuda.synchronize()
        lr.append(a0.elapsed_time(a1))
    leaf_alone_ms = statistics.median(lr)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as fh:
            traffic = json.load(fh).get("p2_leaves_kernel_bytes_per_launch")
    t_roof = max(units["bytes"] / (peaks["hbm_gbs"] * 1e9), units["modmul"] / mm_peak)
    ref_ms = None
    if rank == 0 and not args.no_ref_kernels:
        try:
            ref_ms = reference_kernels_ms(glc, torch, job, max(1, min(args.steps, 3)))
        except Exception as ex:  # reported, never fatal
            ref_ms = None
            print("reference kernels not timed: %s" % ex, file=sys.stderr)
    cpu = cpu_baseline() if (rank == 0 and world == 1) else None
    if cpu:
        cpu.pop("seconds", None)
    line = {
        "metric": "LDE+Merkle commit elements/s",
        "value": value, "unit": "elements/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: seeded ChaCha20 uniform Goldilocks elements (glc_fill_random, seed %r)" % SEED,
        "config": {"workload": WORKLOAD, "columns": COLS, "log_rows": LOG_N, "lde_factor": f, "cap": 1 << LOG_CAP,
                   "parallelism": "replicas" if world > 1 else "single", "l2": "inputs 1 GiB > 126 MB L2, no flush"},
        "hashes_per_s": (units["perms_leaves"] + units["perms_nodes"]) * world / (ms / 1e3),
        "algorithmic_gbs": units["bytes"] * world / (ms / 1e3) / 1e9,
        "stages_ms": {k: v / args.steps for k, v in stage.items()},
        # per stage: algorithmic work, its roofline time, and that over the stage's in-step time
        # (the coset stages run on two streams at once, so their in-step times overlap)
        "stages_roofline": {k: dict(u, roof_ms=max(u["bytes"] / (peaks["hbm_gbs"] * 1e9), u["modmul"] / mm_peak) * 1e3,
                                    frac=max(u["bytes"] / (peaks["hbm_gbs"] * 1e9), u["modmul"] / mm_peak) * 1e3
                                    / max(1e-9, stage[k] / args.steps))
                            for k, u in stage_units().items()},
        "roofline": {"bound": "int", "kernel": "p2_leaves_kernel", "achieved": achieved,
                     "peak": mm_peak / 1e9, "unit": "Gmodmul/s", "frac": achieved * 1e9 / mm_peak,
                     "launch_ms_in_step": leaf_ms, "launch_ms_alone": leaf_alone_ms,
                     "hbm_gbs_alone": (traffic or 0) / (leaf_alone_ms / 1e3) / 1e9,
                     "hbm_frac_alone": (traffic or 0) / (leaf_alone_ms / 1e3) / 1e9 / peaks["hbm_gbs"],
                     "frac_alone": leaf_modmul / (leaf_alone_ms / 1e3) / mm_peak,
                     "traffic": traffic,
                     "peak_source": "glc_modmul_probe measured live in this run (8 independent chains per thread)"},
        "roofline_job": {"bytes": units["bytes"], "modmul": units["modmul"], "t_roof_ms": t_roof * 1e3,
                         "frac": t_roof * 1e3 / ms, "hbm_gbs": peaks["hbm_gbs"], "hbm_source": peak_kind,
                         "modmul_peak_gs": mm_peak / 1e9},
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    if ref_ms:
        line["reference_kernels_sm100a"] = {"ms_per_step": ref_ms, "value": units["elements"] / (ref_ms / 1e3),
                                            "unit": "elements/s", "speedup": ref_ms / ms,
                                            "what": "boojum-cuda native kernels recompiled for sm_100a, reference launch plans"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.destroy()


# ---------------------------------------------------------------------------------------------
# Secondary workloads (their own JSON lines; the default run prints the contract line above).
# ---------------------------------------------------------------------------------------------

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


def run_uneven(args):
    """Batched (multi-stream + CUDA graph) vs plain one-call-per-job on the uneven batch.  The 300
    jobs hold ~100 GB of inputs and ~300 GB of outputs, so they run in waves that fit a device
    budget; every form processes every job."""
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    jobs = uneven_jobs()
    budget = int(args.budget_gb * (1 << 30))
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
    t = {"plain": 0.0, "batched": 0.0, "graph": 0.0, "reference_kernels": 0.0}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    try:
        import refkern
        have_ref = refkern.available()
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
        graph = glc.CommitGraph(bufs, n_streams=args.streams)
        graph.launch()
        torch.cuda.synchronize()
        caps_graph = [jb.cap.clone() for jb in bufs]
        for form in ("plain", "batched", "graph"):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            if form == "plain":
                for jb in bufs:
                    glc.commit.commit(jb, stream)
            elif form == "batched":
                glc.commit.commit_batch(bufs, n_streams=args.streams)
            else:
                graph.launch()
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
            "caps_identical_across_forms": caps_equal, "streams": args.streams}
    print(json.dumps(line), flush=True)
    ctx.destroy()


def run_large(args):
    """2^22 rows x (128 base + 24 extension) = 176 base columns, LDE x2, cap 16 (~18 GB resident)."""
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    l, c, e, cap = 22, 176, 1, 4
    sz = glc.CommitJob.sizes(l, c, e, cap)
    dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
    jb = glc.CommitJob(evals=dev("evals"), log_n=l, cols=c, log_lde=e, log_cap=cap, lde=dev("lde"),
                       trees=dev("trees"), cap=dev("cap"))
    syn.fill_device(jb.evals, "large")
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
    units = job_units(l, c, e, cap)
    peaks, _ = measured_peaks()
    lib = glc._lib.lib()
    blocks, iters = 148 * 32, 2048
    scratch = torch.empty(blocks * 256, dtype=torch.int64, device="cuda")
    lib.glc_modmul_probe(scratch.data_ptr(), blocks, 64, None)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    lib.glc_modmul_probe(scratch.data_ptr(), blocks, iters, None)
    p1.record()
    torch.cuda.synchronize()
    mm_peak = blocks * 256 * 8 * iters / (p0.elapsed_time(p1) / 1e3)
    t_roof = max(units["bytes"] / (peaks["hbm_gbs"] * 1e9), units["modmul"] / mm_peak)
    print(json.dumps({"workload": "2^22 rows x 176 base columns (128 + 24 extension pairs), LDE x2, cap 16",
                      "ms_per_step": ms, "value": units["elements"] / (ms / 1e3), "unit": "elements/s",
                      "hashes_per_s": (units["perms_leaves"] + units["perms_nodes"]) / (ms / 1e3),
                      "roofline": {"t_roof_ms": t_roof * 1e3, "frac": t_roof * 1e3 / ms, "modmul": units["modmul"],
                                   "bytes": units["bytes"], "modmul_peak_gs": mm_peak / 1e9,
                                   "hbm_gbs": peaks["hbm_gbs"]}}), flush=True)
    ctx.destroy()


def run_serve(args):
    """Poisson arrivals of commitment jobs (log2 rows U[16,23], columns U[8,256], LDE x2/x4) served
    with continuous batching under an HBM budget; p50/p99 latency, against the plain sequential
    form (one request on the device at a time).  Host inputs: one pinned buffer of seeded
    synthetic elements, each request reading its prefix."""
    import numpy as np
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    rng = np.random.default_rng(11)
    jobs = [(int(rng.integers(16, 24)), int(rng.integers(8, 257)), int(rng.choice([1, 2])), 4)
            for _ in range(args.serve_jobs)]
    max_elems = max(c << l for l, c, _, _ in jobs)
    d = torch.empty(max_elems, dtype=torch.int64, device="cuda")
    syn.fill_device(d, "serve")
    host = torch.empty(max_elems, dtype=torch.int64, pin_memory=True)
    host.copy_(d)
    del d
    torch.cuda.empty_cache()
    base = host.numpy().view(np.uint64)
    make = lambda i, l, c: base[:c << l]
    out = {"workload": "serving: Poisson(%g/s) arrivals, %d jobs, log2 rows U[16,23], columns U[8,256], LDE x2/x4"
                       % (args.rate, len(jobs)), "budget_gb": args.budget_gb}
    for name, inflight, streams, prio in (("continuous_batching", args.inflight, args.streams, True),
                                          ("continuous_batching_flat_priority", args.inflight, args.streams, False),
                                          ("plain_sequential", 1, 1, False)):
        with glc.serve.Server(hbm_budget_bytes=int(args.budget_gb * (1 << 30)), max_inflight=inflight,
                              streams=streams, size_priority=prio) as srv:
            r = glc.serve.poisson_load(srv, jobs, rate_per_s=args.rate, seed=3, make_input=make)
            st = srv.stats()
        r.pop("caps")
        r["peak_inflight"] = st["peak_inflight"]
        r["peak_gb"] = st["peak_bytes"] / (1 << 30)
        out[name] = r
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
           "hbm_gbs_peak": peaks["hbm_gbs"],
           "peak_source": kind}
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


def run_queries(args):
    """Query openings on the headline commitment (128 columns x 2^20 rows, LDE x2, cap 16): for
    100 seeded query indexes of one coset, gather the 100 rows of the 128 LDE columns
    (gather_rows) and the 17-layer Merkle paths of the 2^20-leaf subtree (gather_merkle_paths)."""
    import numpy as np
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    n = 1 << LOG_N
    sz = glc.CommitJob.sizes(LOG_N, COLS, LOG_LDE, LOG_CAP)
    dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
    jb = glc.CommitJob(evals=dev("evals"), log_n=LOG_N, cols=COLS, log_lde=LOG_LDE, log_cap=LOG_CAP, lde=dev("lde"),
                       trees=dev("trees"), cap=dev("cap"))
    syn.fill_device(jb.evals, "queries")
    glc.commit.commit(jb)
    q = 100
    idx = torch.from_numpy(np.random.default_rng(5).integers(0, n, q).astype(np.int32)).cuda()
    layers = LOG_N - (LOG_CAP - LOG_LDE)
    rows = torch.empty(q * COLS, dtype=torch.int64, device="cuda")
    paths = torch.empty(layers * 4 * q, dtype=torch.int64, device="cuda")
    lde0, tree0 = jb.lde[:COLS * n], jb.trees[:8 * n]
    calls = {"gather_rows": lambda: glc.GLHasher.gather_rows(idx, 0, lde0, n, COLS, rows, q, COLS),
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
    """A small commitment for profiler captures: 128 columns x 2^log_n rows (default 2^18, 256 MiB of
    inputs, still larger than L2), LDE x2, cap 16; warm-up plus a few plain glc_commit calls."""
    glc, torch, ctx = _setup_device()
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    l = args.log_n
    sz = glc.CommitJob.sizes(l, COLS, LOG_LDE, LOG_CAP)
    dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
    jb = glc.CommitJob(evals=dev("evals"), log_n=l, cols=COLS, log_lde=LOG_LDE, log_cap=LOG_CAP, lde=dev("lde"),
                       trees=dev("trees"), cap=dev("cap"))
    syn.fill_device(jb.evals, "profile")
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
    print(json.dumps({"workload": "profile case: %d columns x 2^%d rows, LDE x2, cap 16" % (COLS, l),
                      "ms_per_step": ms, "value": (COLS << l) / (ms / 1e3), "unit": "elements/s"}), flush=True)
    ctx.destroy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-ref-kernels", action="store_true")
    ap.add_argument("--workload", default="commit", choices=["commit", "uneven", "large", "serve", "profile", "ef", "queries"],
                    help="commit: the contract line; others print their own JSON")
    ap.add_argument("--log-n", type=int, default=18, help="rows of the profile case (log2)")
    ap.add_argument("--ef-log-rows", type=int, default=22, help="rows of the extension-layout workload (log2)")
    ap.add_argument("--streams", type=int, default=8)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--serve-jobs", type=int, default=40)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--inflight", type=int, default=8)
    args = ap.parse_args()
    if args.workload != "commit":
        {"uneven": run_uneven, "large": run_large, "serve": run_serve,
         "profile": run_profile_case, "ef": run_ef, "queries": run_queries}[args.workload](args)
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
