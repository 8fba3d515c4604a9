"""The schedule autotuner's decision rules (CPU: synthetic cycle counts, no engine call)."""
import numpy as np

from axtb_b200.autotune import DEFAULT, crossover


def test_crossover_minimises_the_total():
    nao = np.arange(30, 600, 7)
    one = nao.astype(float) ** 2 * 600.0 + 2e6   # one-stage: a per-column chain short of work at small n
    two = nao.astype(float) ** 2 * 700.0         # two-stage: no fixed cost, a larger slope
    cut, bins = crossover(nao, two, one)
    # 700 n^2 = 600 n^2 + 2e6 at n ~ 141: the bins below the cut favour the two-stage reduction
    assert 96 <= cut <= 160
    assert all(b[3] <= b[4] for b in bins if b[1] <= cut)
    assert bins[0][0] == 0 and sum(b[2] for b in bins) == len(nao)


def test_crossover_tolerates_a_losing_bin_inside_a_winning_range():
    nao = np.array([40, 100, 300, 350, 500])
    one = np.array([10.0, 10.0, 10.0, 10.0, 10.0])
    two = np.array([9.0, 10.5, 8.0, 8.0, 14.0])  # loses a little at 100 AOs, wins at 300-350
    cut, _ = crossover(nao, two, one)
    assert cut == 352


def test_crossover_never_and_always():
    nao = np.array([40, 80, 200, 400])
    cut, _ = crossover(nao, np.full(4, 2.0), np.full(4, 1.0))  # two-stage never cheaper
    assert cut == 0
    cut, _ = crossover(nao, np.full(4, 1.0), np.full(4, 2.0))  # always cheaper
    assert cut == 416
    assert DEFAULT["grid_min_nao"] == 1024 and DEFAULT["band_max_nao"] == 64
