"""fused_trace_summary on a hand-made trace of two CTAs: per-kind work and wait, the time
between items, the span, and all-zero (unwritten) records skipped.  No GPU needed."""
import numpy as np

from conftest import load_package


def test_fused_trace_summary():
    glc = load_package()
    ms = 1_000_000  # the records hold nanoseconds
    base = 5 * ms
    # (claim, start, end, kind) per item; CTA 0 runs items 0 and 2, CTA 1 runs item 1
    items = [(0, 1, 3, 0, 0), (0, 2, 4, 2, 1), (4, 4, 9, 3, 0)]
    rec = np.zeros((5, 4), dtype=np.uint64)
    for i, (c, s, e, kind, cta) in enumerate(items):
        rec[i] = [base + c * ms, base + s * ms, base + e * ms, (7 << 40) | (cta << 8) | kind]
    out = glc.commit.fused_trace_summary(rec)
    assert out["items"] == 3 and out["ctas"] == 2
    assert out["span_ms"] == 9.0 and out["cta_ms_total"] == 18.0
    assert out["ntt"] == {"items": 1, "work_cta_ms": 2.0, "wait_cta_ms": 1.0, "first_start_ms": 1.0,
                          "last_end_ms": 3.0}
    assert out["leaves"]["work_cta_ms"] == 2.0 and out["leaves"]["wait_cta_ms"] == 2.0
    assert out["nodes"]["work_cta_ms"] == 5.0 and out["nodes"]["wait_cta_ms"] == 0.0
    assert "bitrev" not in out and "caps" not in out
    assert out["between_items_cta_ms"] == 1.0  # CTA 0: item 0 ends at 3, item 2 claimed at 4
    assert glc.commit.fused_trace_summary(np.zeros((3, 4), dtype=np.uint64)) == {"items": 0}
