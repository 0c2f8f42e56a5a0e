"""bench.py's host-side bookkeeping without a device: the clocks record
taken from nvidia-smi samples during the timed region (its median under load
and the throttle reasons are what decide whether a number stands), the
reference arm's replicas per host process, and the algorithmic work and
whole-job value the bench line is computed from."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "md-force-routines_b200")]

import bench  # noqa: E402


def _row(sm, mx=1965, pw="650.25", reasons=("Not Active",) * 4, active="0x0000000000000000"):
    return ", ".join(["0", str(sm), str(mx), pw, active, *reasons]) + "\n"


def test_clocks_median_under_load_ignores_idle_samples():
    lines = [_row(345), _row(1965), _row(1965), _row(1950), _row(1965), _row(210)]
    c = bench.summarise_clocks(lines)
    assert c["sm_mhz"] == 1965.0          # the two idle samples (< half the peak) are left out
    assert c["sm_max_mhz"] == 1965.0
    assert c["power_w_max"] == 650.25
    assert c["samples"] == 6
    assert c["reasons"] == []


def test_clocks_reasons_seen_active_are_reported():
    power = ("Not Active", "Not Active", "Not Active", "Active")
    hot = ("Not Active", "Active", "Not Active", "Not Active")
    lines = [_row(1800, reasons=power), _row(1700, reasons=hot), _row(1965)]
    assert bench.summarise_clocks(lines)["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]


def test_clocks_tolerate_missing_fields_and_bad_lines():
    lines = ["garbage\n", "\n", _row(1965, pw="[N/A]"), _row(1965, pw="[N/A]")]
    c = bench.summarise_clocks(lines)
    assert c["samples"] == 2 and c["sm_mhz"] == 1965.0 and c["power_w_max"] is None
    assert bench.summarise_clocks([]) == {"sm_mhz": None, "sm_max_mhz": None,
                                          "reasons": ["no samples"]}


def test_clock_stuck_low_is_visible():
    """A leftover clock lock shows as a median well below the max clock with
    no reason active (the record keeps both so the run can be rejected)."""
    c = bench.summarise_clocks([_row(990)] * 10)
    assert c["sm_mhz"] == 990.0 and c["sm_max_mhz"] == 1965.0 and c["reasons"] == []


def test_reference_arm_balance():
    """The reference arm's replicas per host process: each replica once,
    largest first onto the least loaded process."""
    assert bench.balance([10, 10, 10], 3) == [[0], [1], [2]]
    sizes = [1000, 5000, 3000, 3000, 2000, 1000]
    groups = bench.balance(sizes, 2)
    assert sorted(i for g in groups for i in g) == list(range(len(sizes)))
    assert groups == [[1, 4, 5], [2, 3, 0]]
    loads = [sum(sizes[i] for i in g) for g in groups]
    assert loads == [8000, 7000]
    # uneven ensemble (sizes as the 64-replica draws span): imbalance below the largest replica
    import numpy as np

    rng = np.random.default_rng(4)
    sizes = [int(x) for x in rng.integers(5000, 40000, size=64)]
    loads = [sum(sizes[i] for i in g) for g in bench.balance(sizes, 16)]
    assert max(loads) - min(loads) <= max(sizes)


def test_roofline_work_figures_of_the_ensemble():
    """The algorithmic work the bench line divides by, for the 20 x 1e4
    ensemble (r_c 6, 64^3): N rc^3/2 pairs x 48 FLOP = 1.037 GFLOP per pair
    launch, and the step's roofline time at 72.4 TFLOP/s and 6650 GB/s."""
    from p3m_b200.configs import cfg3

    reps = cfg3(20)
    assert bench.pp_flop(reps) == 20 * 10 ** 4 * 6.0 ** 3 / 2 * 48
    flop = 20 * 10 ** 4 * (6.0 ** 3 / 2 * 48 + 3 * 32 * 8)
    byts = 20 * (66.0 * 64 ** 3 + 120.0 * 10 ** 4)
    t = bench.step_roofline_s(reps, 72.4, 6650.0)
    assert t == flop / 72.4e12 + byts / 6650e9
    assert 0.0715e-3 < t < 0.0725e-3
    # whole-job value: all ranks' particles over the slowest rank's time
    assert bench.job_value(2 * 10 ** 5, 2000, 1, 938.75) == 2 * 10 ** 5 * 2000 / 0.93875
    assert bench.job_value(2 * 10 ** 5, 10, 4, 5.0) == 4 * bench.job_value(2 * 10 ** 5, 10, 1, 5.0)
