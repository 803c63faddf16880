"""Commitment jobs: evaluations -> monomials -> coset LDE -> Poseidon2 subtrees -> cap.

The sequence shivini runs around boojum-cuda for one commitment
(crates/shivini/src/data_structures/storage.rs:155-330, cache.rs:353-418), as one call
(glc_commit), as a batch of uneven jobs on concurrent streams (glc_commit_batch), or as a
captured CUDA graph replayed with one launch (CommitGraph), or, for jobs of at most 2^22 rows, as
one persistent cooperative launch that runs every stage of every job (commit_batch_fused).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from ._buffers import as_slice, stream_handle
from ._lib import call, lib


class _Job(C.Structure):
    _fields_ = [("evals", C.c_void_p), ("evals_stride", C.c_uint64), ("log_n", C.c_uint32), ("cols", C.c_uint32),
                ("log_lde", C.c_uint32), ("log_cap", C.c_uint32), ("monomials", C.c_void_p), ("lde", C.c_void_p),
                ("trees", C.c_void_p), ("cap", C.c_void_p)]


@dataclass
class CommitJob:
    """Device buffers of one commitment (see glc_commit_job in include/glc.h)."""
    evals: object
    log_n: int
    cols: int
    log_lde: int
    log_cap: int
    lde: object
    trees: object
    cap: object
    monomials: object = None
    evals_stride: int | None = None

    @staticmethod
    def sizes(log_n: int, cols: int, log_lde: int, log_cap: int) -> dict:
        n, f = 1 << log_n, 1 << log_lde
        return {"evals": cols * n, "lde": f * cols * n, "trees": f * 8 * n, "cap": 4 << log_cap, "monomials": cols * n}

    def _struct(self) -> _Job:
        n = 1 << self.log_n
        sz = self.sizes(self.log_n, self.cols, self.log_lde, self.log_cap)
        stride = n if self.evals_stride is None else self.evals_stride
        ep, el = as_slice(self.evals)
        lp, ll = as_slice(self.lde)
        tp, tl = as_slice(self.trees)
        cp, cl = as_slice(self.cap)
        if el < (self.cols - 1) * stride + n or ll < sz["lde"] or tl < sz["trees"] or cl < sz["cap"]:
            raise ValueError("commit: a buffer is shorter than the job needs")
        mp = None
        if self.monomials is not None:
            mp, ml = as_slice(self.monomials)
            if ml < sz["monomials"]:
                raise ValueError("commit: monomials buffer too short")
        return _Job(ep, stride, self.log_n, self.cols, self.log_lde, self.log_cap, mp, lp, tp, cp)


def commit(job: CommitJob, stream=None) -> None:
    """One commitment on one stream (glc_commit)."""
    s = job._struct()
    call("glc_commit", C.addressof(s), stream_handle(stream))


def _array(jobs):
    arr = (_Job * len(jobs))(*[j._struct() for j in jobs])
    return arr


def commit_batch(jobs: list[CommitJob], n_streams: int = 0, stream=None) -> None:
    """Many commitments as one unit on `stream` (glc_commit_batch)."""
    arr = _array(jobs)
    call("glc_commit_batch", C.addressof(arr) if jobs else None, len(jobs), n_streams, stream_handle(stream))


class MappedWord:
    """A 32-bit word of page-locked host memory mapped into the device (glc_mapped_word_create):
    `value` reads and writes it from the host, `device` is its address for kernels."""

    def __init__(self):
        h, d = C.c_void_p(), C.c_void_p()
        call("glc_mapped_word_create", C.byref(h), C.byref(d))
        self._host, self.device = h.value, d.value
        self._word = C.c_uint32.from_address(self._host)

    @property
    def value(self) -> int:
        return self._word.value

    @value.setter
    def value(self, v: int) -> None:
        self._word.value = v

    def close(self) -> None:
        if self._host:
            call("glc_mapped_word_destroy", self._host)
            self._host = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def commit_batch_fused_cancellable(jobs: list[CommitJob], cancel: MappedWord, status: MappedWord | None = None,
                                   stream=None) -> None:
    """commit_batch_fused that stops claiming and starting items once `cancel.value` is non-zero
    (glc_commit_batch_fused_cancellable); `status.value` becomes 1 when every item ran, 2 when a
    cancel skipped some (outputs incomplete)."""
    arr = _array(jobs)
    call("glc_commit_batch_fused_cancellable", C.addressof(arr) if jobs else None, len(jobs), cancel.device,
         status.device if status is not None else None, stream_handle(stream))


def commit_batch_fused(jobs: list[CommitJob], stream=None, trace=None) -> None:
    """Many commitments (2^log_n <= 2^22 rows each) in ONE persistent launch
    (glc_commit_batch_fused): work items of every stage of every job, each waiting only for the
    items it reads from.  `trace`: a device buffer of 4 * N 8-byte words, cleared by the caller,
    that receives the per-item records of the first N items (glc_commit_batch_fused_traced; see
    fused_trace_summary)."""
    arr = _array(jobs)
    if trace is None:
        call("glc_commit_batch_fused", C.addressof(arr) if jobs else None, len(jobs), stream_handle(stream))
    else:
        tp, tl = as_slice(trace)
        call("glc_commit_batch_fused_traced", C.addressof(arr) if jobs else None, len(jobs), tp, tl // 4,
             stream_handle(stream))


FUSED_KINDS = ("ntt", "bitrev", "leaves", "nodes", "caps")


def fused_trace_summary(records) -> dict:
    """Where the CTAs of one fused launch spent their time, from its trace (an (n, 4) array of
    uint64 records as glc_commit_batch_fused_traced writes them; all-zero rows are unwritten).
    Per item kind: items, CTA-milliseconds of work (start -> end) and of waiting (claim -> start:
    entry search and producers), first start and last end (ms from the first claim); the
    CTA-milliseconds between one item's end and the same CTA's next claim; and the launch span."""
    import numpy as np
    r = np.asarray(records, dtype=np.uint64).reshape(-1, 4)
    r = r[r[:, 2] > 0].astype(np.int64)
    if len(r) == 0:
        return {"items": 0}
    t00 = r[:, 0].min()
    claim, start, end = (r[:, 0] - t00) / 1e6, (r[:, 1] - t00) / 1e6, (r[:, 2] - t00) / 1e6
    kind, cta = r[:, 3] & 0xFF, (r[:, 3] >> 8) & 0xFFFFFFFF
    out = {"items": int(len(r)), "ctas": int(len(np.unique(cta))), "span_ms": float(end.max())}
    for k, name in enumerate(FUSED_KINDS):
        m = kind == k
        if m.any():
            out[name] = {"items": int(m.sum()), "work_cta_ms": float((end - start)[m].sum()),
                         "wait_cta_ms": float((start - claim)[m].sum()), "first_start_ms": float(start[m].min()),
                         "last_end_ms": float(end[m].max())}
    order = np.lexsort((claim, cta))
    same = cta[order][1:] == cta[order][:-1]
    out["between_items_cta_ms"] = float((claim[order][1:] - end[order][:-1])[same].sum())
    out["cta_ms_total"] = float(out["ctas"] * end.max())
    return out


def fused_timeouts() -> int:
    """Expired waits of commit_batch_fused on this device since load (0 unless something is wrong)."""
    v = C.c_uint64()
    call("glc_commit_batch_fused_timeouts", C.byref(v))
    return v.value


class CommitGraph:
    """A batch captured once into a CUDA graph (glc_commit_graph_*); replay with launch()."""

    def __init__(self, jobs: list[CommitJob], n_streams: int = 0):
        self._arr = _array(jobs)
        self._h = C.c_void_p()
        call("glc_commit_graph_create", C.addressof(self._arr), len(jobs), n_streams, C.byref(self._h))

    def launch(self, stream=None) -> None:
        call("glc_commit_graph_launch", self._h, stream_handle(stream))

    def close(self) -> None:
        if self._h:
            call("glc_commit_graph_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
