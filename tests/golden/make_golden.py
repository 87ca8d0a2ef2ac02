"""Regenerate the committed fixtures under tests/golden/ from the oracle.

  python tests/golden/make_golden.py

fetch_counts.json  executed-fetch counts per kind (instrumented FP64 CPU
                   restatement) for each benchmark workload, the voxel-grid
                   one included (the stress workload's first frame stands for
                   its eight); bench.py turns them into algorithmic bytes
                   per ray.
plain_96x54.npz    FP64-oracle L/T of the plain workload at 96x54 (float32),
precision_96x54.npz  and of the three-layer workload.  The oracle must
                   reproduce them (tests/test_oracle_goldens.py) and the GPU
                   benchmark form is compared with them
                   (tests/test_gpu_fullsize.py::test_committed_goldens).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle import pyoracle  # noqa: E402
from pedalsky_b200 import scenes  # noqa: E402


def main():
    pyoracle.build()
    noise = pyoracle.bake_noise()
    counts = {}
    for name, make in (("precision_1080p", lambda: scenes.precision_1080p()),
                       ("plain_320x180", lambda: scenes.plain_320x180()),
                       ("stress_2160p", lambda: scenes.stress_2160p(frame_index=0))):
        s = make()
        luts = pyoracle.bake_luts(s.frame, s.world)
        _, _, c = pyoracle.render(s, noise, luts, precision=pyoracle.FP64, counters=True)
        counts[name] = {"width": s.width, "height": s.height, "counts": c}
        print(name, c)
    s = scenes.grid_512()
    luts = pyoracle.bake_luts(s.frame, s.world)
    c = pyoracle.grid_counts(s, noise, luts, s.extra["grid"], s.extra["grid_spec"])
    counts["grid_512"] = {"width": s.width, "height": s.height, "counts": c}
    print("grid_512", c)
    (HERE / "fetch_counts.json").write_text(json.dumps(counts, indent=1) + "\n")
    for name, make in (("plain_96x54", lambda: scenes.plain_320x180(96, 54)),
                       ("precision_96x54", lambda: scenes.precision_1080p(96, 54))):
        s = make()
        luts = pyoracle.bake_luts(s.frame, s.world)
        L, T = pyoracle.render(s, noise, luts, precision=pyoracle.FP64)
        np.savez_compressed(HERE / f"{name}.npz", L=L, T=T)
        print(name, float(L[..., :3].max()), float(T[..., :3].min()))


if __name__ == "__main__":
    main()
