"""The schedule autotuner's decision rules (CPU: synthetic cycle counts, no engine call)."""
import numpy as np

from axtb_b200.autotune import DEFAULT, crossover


def test_crossover_is_the_first_bin_from_which_two_stage_always_wins():
    nao = np.arange(30, 600, 7)
    one = nao.astype(float) ** 2 * 600.0          # the one-stage cost grows like n^2 (latency chain)
    two = nao.astype(float) ** 2 * 250.0 + 4e6    # the two-stage has a fixed overhead
    cut, bins = crossover(nao, two, one)
    # 600 n^2 = 250 n^2 + 4e6 at n ~ 107: the bin holding it and every larger bin favour two-stage
    assert 96 <= cut <= 128
    assert all(b[3] <= b[4] for b in bins if b[0] >= cut)
    assert bins[0][0] == 0 and sum(b[2] for b in bins) == len(nao)


def test_crossover_never_and_always():
    nao = np.array([40, 80, 200, 400])
    cut, _ = crossover(nao, np.full(4, 2.0), np.full(4, 1.0))  # two-stage never cheaper
    assert cut == 416  # past the largest bin: no molecule of the sample uses it
    cut, _ = crossover(nao, np.full(4, 1.0), np.full(4, 2.0))  # always cheaper
    assert cut == 32
    assert DEFAULT["grid_min_nao"] == 1024
