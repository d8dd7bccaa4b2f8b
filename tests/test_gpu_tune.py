"""The autotuner's choices for the T-operator (tile shape wmax = widest column piece, 128 / 192 / 256,
and item depth bper = point blocks per work item) change only how the work is spread over the SMs: every
element of T is the same sum of the same per-128-point tensor-core partials, grouped into the same fixed
point blocks.  Each choice is pinned through a tune file in a fresh process (the tuner's table lives for
the process), and h after three split-precision steps must equal the default choice bit for bit.  The point
blocks are sized from the point count, the basis and the SM count only: at 150,000 points on 148 SMs the
default layout's items fill whole waves with blocks of 16 Xt tiles instead of 32, and the same holds there.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
import papers_b200
s = papers_b200.QuinticSolver.new_with_psi_sz(6, int(sys.argv[3]), 3, 0.5, reduced_basis=True, precision="fp16x3")
for _ in range(3):
    s.donaldson_step()
np.save(sys.argv[2], s.h_block)
"""


def _run(tmp_path, name, env_extra, points=40000):
    env = dict(os.environ)
    env.pop("CY3Q_TUNE_FILE", None)
    env.pop("CY3Q_GRAM_WMAX", None)
    env.update(env_extra)
    out = str(tmp_path / f"{name}.npy")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, out, str(points)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


def test_tuned_tile_shapes_and_depths_give_identical_h(tmp_path):
    import torch

    sm = torch.cuda.get_device_properties(0).multi_processor_count
    # k = 6 reduced: 2N = 410 -> ldk 448; 40,000 points -> 40,064 padded (313 Xt tiles, 10 blocks of 32)
    key = f"448 40064 1 {sm}"
    base = _run(tmp_path, "default", {"CY3Q_AUTOTUNE": "0"})
    assert np.all(np.isfinite(base))
    for wmax, bper in [(256, 10), (192, 3), (128, 1), (128, 10)]:
        tf = tmp_path / f"tune_{wmax}_{bper}.txt"
        tf.write_text(f"{key} {wmax} {bper}\n")
        h = _run(tmp_path, f"w{wmax}_b{bper}", {"CY3Q_TUNE_FILE": str(tf)})
        assert np.array_equal(h, base), json.dumps({"wmax": wmax, "bper": bper,
                                                    "max_abs_diff": float(np.max(np.abs(h - base)))})


def test_wave_sized_point_blocks_give_identical_h(tmp_path):
    import torch

    sm = torch.cuda.get_device_properties(0).multi_processor_count
    points = 150000
    # 150,000 points -> 150,016 padded, 1,172 Xt tiles (74 blocks of 16 on 148 SMs)
    key = f"448 150016 1 {sm}"
    base = _run(tmp_path, "default150k", {"CY3Q_AUTOTUNE": "0"}, points)
    assert np.all(np.isfinite(base))
    for wmax, bper in [(256, 74), (192, 5), (128, 1)]:
        tf = tmp_path / f"tune150k_{wmax}_{bper}.txt"
        tf.write_text(f"{key} {wmax} {bper}\n")
        h = _run(tmp_path, f"w{wmax}_b{bper}_150k", {"CY3Q_TUNE_FILE": str(tf)}, points)
        assert np.array_equal(h, base), json.dumps({"wmax": wmax, "bper": bper,
                                                    "max_abs_diff": float(np.max(np.abs(h - base)))})
