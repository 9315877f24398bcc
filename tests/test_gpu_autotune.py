"""Format autotuner (autotune.choose_format): picks the fastest layout of the candidates,
returns it ready to use (same products), and caches the choice by matrix shape class."""
import json

import numpy as np
import pytest
import torch

from mats import case, within_bound


def test_matrix_key_classes():
    from gpu_spmv_b200.autotune import matrix_key

    row = np.arange(0, 5 * 1000 + 1, 5)  # uniform rows
    assert matrix_key(row).endswith("cv0")
    lens = np.r_[np.ones(999, int), [5000]]
    row2 = np.r_[0, np.cumsum(lens)]
    assert matrix_key(row2).endswith("cv2")
    assert matrix_key(row, "f32").startswith("f32/")


@pytest.mark.gpu
def test_choose_format(port, tmp_path):
    from gpu_spmv_b200 import autotune

    rng = np.random.default_rng(2)
    row, col, val = case("powerlaw_small", rng)
    n = len(row) - 1
    cache = tmp_path / "fmt.json"
    A, t = autotune.choose_format(row, col, val, reps=5, cache_path=str(cache))
    assert set(t) == set(autotune.FORMAT_CANDIDATES)
    assert A.autotuned_format == min(t, key=t.get)
    x = rng.uniform(-1, 1, n)
    y = A.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    _, mag = port.csr_truth(row, col, val, x)
    assert within_bound(y, port.csr_spmv(row, col, val, x), mag)
    assert json.loads(cache.read_text())[autotune.matrix_key(row)] == A.autotuned_format
    A2, t2 = autotune.choose_format(row, col, val, reps=5, cache_path=str(cache))
    assert list(t2) == [A.autotuned_format]
