"""Batched sweep on the GPU: concurrent stepping gives the same fields as one case at a time."""
import numpy as np
import pytest

from pyib_b200.batch import BatchRun
from pyib_b200.cases import SphereCase

pytestmark = pytest.mark.gpu


def _cases():
    # uneven sizes and viscosities, small enough for a test
    return [SphereCase(name="b8", cells_per_diameter=8, half_widths_d=(2.0, 4.0), reynolds=1.0, amplitude_d=0.2),
            SphereCase(name="b12", cells_per_diameter=12, half_widths_d=(2.0, 4.0), reynolds=5.0,
                       amplitude_d=0.1),
            SphereCase(name="b8b", cells_per_diameter=8, half_widths_d=(2.0, 4.0), reynolds=0.5,
                       amplitude_d=0.3)]


def test_concurrent_equals_sequential():
    con = BatchRun(_cases())
    seq = BatchRun(_cases())
    assert len(con.tables) == 2                     # equal resolutions share their tables
    con.tune()
    seq.tune()
    t1, s1 = con.advance(2, concurrent=True)
    t2, s2 = seq.advance(2, concurrent=False)
    assert s1 == s2                                 # same CG iterations, case by case summed
    for a, b in zip(con.runs, seq.runs):
        assert np.array_equal(np.asarray(a.s), np.asarray(b.s))
        assert np.array_equal(np.asarray(a.drv.ib_force_L), np.asarray(b.drv.ib_force_L))
        assert a.loads.latest["body_force"].tolist() == b.loads.latest["body_force"].tolist()
    con.close()
    seq.close()


def _per_case(run):
    return [(np.asarray(r.s).copy(), np.asarray(r.drv.ib_force_L).copy(), r.loads.latest["body_force"].tolist(),
             r.drv.helmholtz_total_iterations_last_step) for r in run.runs]


@pytest.mark.parametrize("precision", ["float64", "mixed"])
def test_batched_equals_sequential(precision):
    """One pyib_batch over all cases (the CG iterations of every case as one launch per
    kernel stage) gives every case the bits of its own steps, in both precisions."""
    bat = BatchRun(_cases(), precision=precision)
    seq = BatchRun(_cases(), precision=precision)
    bat.tune()
    seq.tune()
    for _ in range(2):
        _, s1 = bat.advance(1, batched=True)
        _, s2 = seq.advance(1, concurrent=False)
        assert s1 == s2
        for a, b in zip(_per_case(bat), _per_case(seq)):
            assert np.array_equal(a[0], b[0])
            assert np.array_equal(a[1], b[1])
            assert a[2] == b[2]
            assert a[3] == b[3]
    t = bat.batch_timing()
    assert t["batched_launches"] > 0 and t["chunk_seconds"] > 0 and t["graph_captures"] >= 1
    bat.close()
    seq.close()
