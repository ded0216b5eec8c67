"""The batched sweep's seeded draw (host only)."""
import numpy as np

from pyib_b200.batch import SWEEP_CELLS_PER_DIAMETER, sweep_cases


def test_sweep_draw_is_seeded_and_in_range():
    a = sweep_cases(64, seed=0)
    b = sweep_cases(64, seed=0)
    assert [(c.cells_per_diameter, c.amplitude_d, c.reynolds) for c in a] == \
           [(c.cells_per_diameter, c.amplitude_d, c.reynolds) for c in b]
    assert len(a) == 64
    for c in a:
        assert c.cells_per_diameter in SWEEP_CELLS_PER_DIAMETER
        assert 0.05 <= c.amplitude_d <= 0.3
        assert 0.1 <= c.reynolds <= 10.0
        assert c.half_widths_d == (2.0, 4.0) and c.cavity
    # draw order per case: D, then A/D, then Re0
    rng = np.random.default_rng(0)
    d0 = int(rng.choice(SWEEP_CELLS_PER_DIAMETER))
    a0 = float(rng.uniform(0.05, 0.3))
    r0 = float(10.0 ** rng.uniform(-1.0, 1.0))
    assert (a[0].cells_per_diameter, a[0].amplitude_d, a[0].reynolds) == (d0, a0, r0)
    # two levels: (4N)^3 + (4N)^3 - (2N)^3 = 120 N^3 cells
    lay = a[0].layout().build()
    assert int(lay.cell_active.sum()) == 120 * a[0].cells_per_diameter ** 3


def test_case_cost_counts_the_layout_cells():
    from pyib_b200.batch import case_cost
    from pyib_b200.cases import CASES
    for c in sweep_cases(8, seed=1):
        assert case_cost(c, steps=3) == 3 * 120 * c.cells_per_diameter ** 3
    d8 = CASES["d8_oscillating_sphere"]
    assert case_cost(d8) == int(d8.layout().build().cell_active.sum())


def test_partition_is_deterministic_complete_and_balanced():
    from pyib_b200.batch import case_cost, partition
    cases = sweep_cases(64, seed=0)
    for world in (1, 2, 4, 8):
        parts, load = partition(cases, world)
        assert parts == partition(cases, world)[0]
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(64))                       # every case exactly once
        assert all(p == sorted(p) for p in parts)             # sweep order within a rank
        costs = [case_cost(c) for c in cases]
        assert load == [sum(costs[q] for q in p) for p in parts]
        # longest-first greedy: no rank exceeds the mean by more than the largest case
        assert max(load) <= sum(costs) / world + max(costs)
    # more ranks than cases: the extra ranks get nothing
    parts, _ = partition(cases[:3], 5)
    assert sorted(len(p) for p in parts) == [0, 0, 1, 1, 1]
