"""The launch-shape autotuner's selection rule (cp_tune_select), driven with
synthetic timings on the CPU (a host-only call of the C-ABI library)."""
import ctypes as C

import numpy as np
import pytest


def select(lib, ms, default=0, min_gain=0.02):
    ms = np.ascontiguousarray(ms, dtype=np.float64)
    nv, reps = ms.shape
    return int(lib.cp_tune_select(nv, reps, ms.ctypes.data_as(C.POINTER(C.c_double)), default, min_gain))


def test_picks_the_smallest_median(cuda_lib):
    ms = [[5.0, 5.1, 9.0], [4.0, 4.2, 4.1], [6.0, 6.0, 6.0], [4.5, 1.0, 4.6]]
    # medians 5.1, 4.1, 6.0, 4.5: shape 1 (the outlier 1.0 of shape 3 does not count)
    assert select(cuda_lib, ms, default=0) == 1


def test_keeps_the_default_within_the_noise_margin(cuda_lib):
    ms = [[10.0, 10.0, 10.0], [9.9, 9.9, 9.9], [12.0, 12.0, 12.0], [11.0, 11.0, 11.0]]
    assert select(cuda_lib, ms, default=0, min_gain=0.02) == 0  # 1 % faster: not enough
    assert select(cuda_lib, ms, default=0, min_gain=0.0) == 1
    ms[1] = [9.0, 9.0, 9.0]
    assert select(cuda_lib, ms, default=0, min_gain=0.02) == 1  # 10 % faster


def test_failed_launches_and_ties(cuda_lib):
    ms = [[-1.0, -1.0], [np.nan, 3.0], [3.0, 3.0], [np.inf, np.inf]]
    # shape 0 and 3 have no timing; shapes 1 and 2 tie at 3.0: the lower index
    assert select(cuda_lib, ms, default=0) == 1
    assert select(cuda_lib, [[-1.0], [-1.0]], default=0) == -1
    # a default without a timing does not block the winner
    assert select(cuda_lib, ms, default=3) == 1


@pytest.mark.parametrize("seed", range(5))
def test_agrees_with_a_numpy_restatement(cuda_lib, seed):
    rng = np.random.default_rng(seed)
    ms = rng.uniform(1.0, 2.0, size=(4, 5))
    d = int(rng.integers(0, 4))
    med = np.median(ms, axis=1)
    best = int(np.argmin(med))
    want = d if (best != d and not med[best] < 0.98 * med[d]) else best
    assert select(cuda_lib, ms, default=d) == want
