"""Regenerates the launch-tuning table on the current GPU (tuning_b200.txt was made this way on a
B200): the autotuner over every NTT size at its default batch (128 columns, at most 2^28
elements), then again at the two benchmarked commitment shapes (2^20 rows x 128 columns and
2^22 rows x 176 columns), each pass also re-timing the leaf-kernel variants.

    python zksync-crypto-gpu_b200/make_tuning.py [output path, default: tuning_b200.txt here]
"""
from __future__ import annotations

import importlib
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(out: str) -> None:
    sys.path.insert(0, os.path.dirname(HERE))
    glc = importlib.import_module(os.path.basename(HERE))
    ctx = glc.Context.create()
    try:
        glc.tuning.autotune(1, 24, cols=0, reps=3)
        glc.tuning.autotune(20, 20, cols=128, reps=5)
        glc.tuning.autotune(22, 22, cols=176, reps=5)
        glc.tuning.save(out)
    finally:
        ctx.destroy()
    print(open(out).read(), end="")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "tuning_b200.txt"))
