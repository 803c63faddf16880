"""Serving: continuous batching of commitment requests (glc_server_*), plus a Poisson load
generator that reports throughput and p50/p99 latency."""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np

from ._lib import GlcError, call, lib


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_inflight", C.c_uint32), ("streams", C.c_uint32),
                ("flat_priority", C.c_uint32)]


class ServeRequest(C.Structure):
    _fields_ = [("host_evals", C.c_void_p), ("log_n", C.c_uint32), ("cols", C.c_uint32), ("log_lde", C.c_uint32),
                ("log_cap", C.c_uint32), ("host_cap", C.c_void_p), ("keep_resident", C.c_uint32)]


class ServeResult(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int), ("queue_s", C.c_double), ("latency_s", C.c_double),
                ("device_lde", C.c_void_p), ("device_trees", C.c_void_p)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("completed", "rejected", "pending", "inflight", "used_bytes", "peak_bytes",
                                         "peak_inflight")]


_SIG = {
    "glc_server_create": [C.c_void_p, C.c_void_p],
    "glc_server_submit": [C.c_void_p, C.c_void_p, C.c_void_p],
    "glc_server_cancel": [C.c_void_p, C.c_uint64],
    "glc_server_wait": [C.c_void_p, C.c_uint64, C.c_double, C.c_void_p],
    "glc_server_release": [C.c_void_p, C.c_uint64],
    "glc_server_get_stats": [C.c_void_p, C.c_void_p],
    "glc_server_destroy": [C.c_void_p],
}


def _bind():
    L = lib()
    for k, a in _SIG.items():
        f = getattr(L, k)
        f.restype = C.c_int
        f.argtypes = a
    return L


@dataclass
class Pending:
    ticket: int
    cap: np.ndarray
    evals: np.ndarray  # kept alive until the request finishes (the device reads it)
    shape: tuple


class Server:
    """Owns a glc_server on the current device.  submit() takes host numpy arrays (uint64)."""

    def __init__(self, hbm_budget_bytes: int, max_inflight: int = 16, streams: int = 8, size_priority: bool = True):
        _bind()
        self._h = C.c_void_p()
        cfg = ServerConfig(hbm_budget_bytes, max_inflight, streams, 0 if size_priority else 1)
        call("glc_server_create", C.byref(cfg), C.byref(self._h))
        self._pending: dict[int, Pending] = {}

    def submit(self, evals: np.ndarray, log_n: int, cols: int, log_lde: int, log_cap: int,
               keep_resident: bool = False) -> int:
        evals = np.ascontiguousarray(evals, dtype=np.uint64)
        if evals.size != cols << log_n:
            raise ValueError("evals must hold cols << log_n elements")
        cap = np.zeros(4 << log_cap, dtype=np.uint64)
        req = ServeRequest(evals.ctypes.data, log_n, cols, log_lde, log_cap, cap.ctypes.data, int(keep_resident))
        t = C.c_uint64()
        call("glc_server_submit", self._h, C.byref(req), C.byref(t))
        self._pending[t.value] = Pending(t.value, cap, evals, (log_n, cols, log_lde, log_cap))
        return t.value

    def cancel(self, ticket: int) -> None:
        call("glc_server_cancel", self._h, ticket)

    def wait(self, ticket: int, timeout_s: float = -1.0):
        """Returns (cap, ServeResult); raises GlcError on a failed request or a timeout."""
        r = ServeResult()
        call("glc_server_wait", self._h, ticket, timeout_s, C.byref(r))
        p = self._pending.pop(ticket)
        if r.status:
            raise GlcError(r.status, "request %d" % ticket, "")
        return p.cap, r

    def release(self, ticket: int) -> None:
        call("glc_server_release", self._h, ticket)

    def stats(self) -> dict:
        s = ServerStats()
        call("glc_server_get_stats", self._h, C.byref(s))
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            call("glc_server_destroy", self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def poisson_load(server: Server, jobs: list[tuple], rate_per_s: float, seed: int = 0, make_input=None):
    """Submits jobs (log_n, cols, log_lde, log_cap) at Poisson arrival times, waits for all, and
    returns per-job latencies plus aggregate throughput.  make_input(i, log_n, cols) -> evals."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=len(jobs)) if rate_per_s > 0 else np.zeros(len(jobs))
    inputs = [make_input(i, j[0], j[1]) for i, j in enumerate(jobs)]
    tickets = []
    t0 = time.perf_counter()
    next_t = t0
    for i, j in enumerate(jobs):
        next_t += gaps[i]
        d = next_t - time.perf_counter()
        if d > 0:
            time.sleep(d)
        tickets.append(server.submit(inputs[i], *j))
    lat, queue, caps = [], [], []
    for t in tickets:
        cap, r = server.wait(t)
        lat.append(r.latency_s)
        queue.append(r.queue_s)
        caps.append(cap)
    wall = time.perf_counter() - t0
    elements = sum(c << l for l, c, _, _ in jobs)
    lat_ms = np.array(lat) * 1e3
    return {"jobs": len(jobs), "wall_s": wall, "jobs_per_s": len(jobs) / wall, "elements_per_s": elements / wall,
            "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99)),
            "mean_queue_ms": float(np.mean(queue) * 1e3), "caps": caps}
