"""Host-side helpers of ``bench.py`` and of the batched sweep (no GPU needed)."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402
import _pyib_b200_import  # noqa: E402

_pyib_b200_import.load()
from pyib_b200.batch import BatchRun  # noqa: E402


def test_matvec_kernel_names_follow_the_tuned_form():
    mv = [0.3, 0.06, 0.02, 0.08, 0.02, 0.11, 0.024]
    apart = bench.matvec_kernel_ms(mv, False)
    assert list(apart) == ["curl_interp", "curl_interp_patch", "viscous", "viscous_patch", "integr_rot_dot",
                           "integr_rot_patch_reduce"]
    assert apart["viscous"] == 0.08
    fused = bench.matvec_kernel_ms(mv, True)
    # the fused kernel takes slot 1; slot 3 (the viscous template) is not a kernel of its own
    assert list(fused) == ["curl_interp_viscous", "curl_interp_patch", "viscous_patch", "integr_rot_dot",
                           "integr_rot_patch_reduce"]
    assert fused["curl_interp_viscous"] == 0.06 and fused["viscous_patch"] == 0.02


def test_sweep_stats_keep_each_case_iterations():
    st = BatchRun._stats(None, [[10, 20], [5], [7, 8, 9]])
    assert st == {"cg_iterations": 59, "max_case_iterations": 30, "per_case_iterations": [30, 5, 24]}


def test_bit_identity_flag_needs_every_rank():
    # the sweep line's flag is the minimum over ranks, taken as -max(-x); one process here
    agree = -bench.reduce_max(None, -1.0) > 0.5
    differ = -bench.reduce_max(None, -0.0) > 0.5
    assert agree and not differ
