"""Per-device twiddle/power tables: the counterpart of boojum-cuda's context::Context
(crates/boojum-cuda/src/context.rs:157-297)."""
from __future__ import annotations

from ._lib import call

OMEGA_LOG_ORDER = 30


class Context:
    """Tables of the current device.  Context.create(...) mirrors Context::create (context.rs:171);
    destroy() mirrors Context::destroy (context.rs:284).  One per device, like the reference's
    __constant__ descriptors."""

    def __init__(self, w_coarse_log: int, g_coarse_log: int):
        self.w_coarse_log = w_coarse_log
        self.g_coarse_log = g_coarse_log
        self._alive = True

    @classmethod
    def create(cls, powers_of_w_coarse_log_count: int = 15, powers_of_g_coarse_log_count: int = 15) -> "Context":
        call("glc_context_create", powers_of_w_coarse_log_count, powers_of_g_coarse_log_count)
        return cls(powers_of_w_coarse_log_count, powers_of_g_coarse_log_count)

    def destroy(self) -> None:
        if self._alive:
            call("glc_context_destroy")
            self._alive = False
