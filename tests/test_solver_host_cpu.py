"""Host-side decision logic of the solvers, without a GPU: the sweep autotuner's choice."""
from edge_to_b200.solvers import CuMultiGrid, pick_sweep_pattern


def _retime(table, fail=()):
    def f(pattern):
        key = tuple(pattern)
        return table[key], key not in fail, 0
    return f


def test_sweep_choice_tie_goes_to_fewer_sweeps():
    m = CuMultiGrid.SWEEP_MARGIN
    # the fastest is also the cheapest: kept
    runs = [[85.2, [1, 1, 1, 1, 1], 195], [88.7, [1, 2, 2, 2, 2], 147], [99.5, [2, 2, 2, 2, 2], 149]]
    best = pick_sweep_pattern(runs, _retime({(1, 1, 1, 1, 1): 85.0}), m)
    assert best[1] == [1, 1, 1, 1, 1] and best[0] == 170.2
    # more sweeps 3 % faster on both timings: within the margin, the cheapest is kept
    runs = [[100.0, [1, 1, 1], 10], [97.0, [1, 2, 2], 8]]
    best = pick_sweep_pattern(runs, _retime({(1, 1, 1): 100.0, (1, 2, 2): 97.0}), m)
    assert best[1] == [1, 1, 1]
    # 20 % faster: the pattern with more sweeps wins
    runs = [[100.0, [1, 1, 1], 10], [80.0, [1, 2, 2], 8]]
    best = pick_sweep_pattern(runs, _retime({(1, 1, 1): 100.0, (1, 2, 2): 80.0}), m)
    assert best[1] == [1, 2, 2] and best[0] == 160.0
    # the fastest fails to converge when timed again: the cheapest is kept
    runs = [[100.0, [1, 1, 1], 10], [60.0, [2, 2, 2], 8]]
    best = pick_sweep_pattern(runs, _retime({(1, 1, 1): 100.0, (2, 2, 2): 60.0}, fail={(2, 2, 2)}), m)
    assert best[1] == [1, 1, 1]
    # the input list is not modified
    assert runs[0][0] == 100.0


def test_sweep_choice_falls_back_when_no_contender_converges_again():
    m = CuMultiGrid.SWEEP_MARGIN
    fallback = [3, 3, 3]
    # the only contender (fastest = cheapest) fails on its retime
    runs = [[100.0, [1, 1, 1], 10], [120.0, [2, 2, 2], 8]]
    best = pick_sweep_pattern(runs, _retime({(1, 1, 1): 100.0}, fail={(1, 1, 1)}), m, fallback=fallback)
    assert best == (0.0, [3, 3, 3], 0)
    # both contenders fail on their retimes
    runs = [[100.0, [1, 1, 1], 10], [60.0, [2, 2, 2], 8]]
    best = pick_sweep_pattern(runs, _retime({(1, 1, 1): 100.0, (2, 2, 2): 60.0}, fail={(1, 1, 1), (2, 2, 2)}), m,
                              fallback=fallback)
    assert best == (0.0, [3, 3, 3], 0)
