"""The schedule autotuner's decision rules (CPU: synthetic cycle counts, no engine call)."""
import numpy as np

from axtb_b200.autotune import DEFAULT, crossover


def test_crossover_is_the_last_bin_below_which_two_stage_always_wins():
    nao = np.arange(30, 600, 7)
    one = nao.astype(float) ** 2 * 600.0 + 2e6   # one-stage: a per-column chain short of work at small n
    two = nao.astype(float) ** 2 * 700.0         # two-stage: no fixed cost, a larger slope
    cut, bins = crossover(nao, two, one)
    # 700 n^2 = 600 n^2 + 2e6 at n ~ 141: every bin below the cut favours the two-stage reduction
    assert 96 <= cut <= 160
    assert all(b[3] <= b[4] for b in bins if b[1] <= cut)
    assert bins[0][0] == 0 and sum(b[2] for b in bins) == len(nao)


def test_crossover_never_and_always():
    nao = np.array([40, 80, 200, 400])
    cut, _ = crossover(nao, np.full(4, 2.0), np.full(4, 1.0))  # two-stage never cheaper
    assert cut == 0
    cut, _ = crossover(nao, np.full(4, 1.0), np.full(4, 2.0))  # always cheaper
    assert cut == 416
    assert DEFAULT["grid_min_nao"] == 1024 and DEFAULT["band_max_nao"] == 64
