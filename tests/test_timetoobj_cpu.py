"""Host-side summary of the time-to-objective measurement (no GPU)."""
import pytest

from gpair_b200 import timetoobj as T


def _row(width, plain, batch, warm, winner, reached=(True, True, True), fallback=False):
    return dict(width=width, nuv=10, J_star=1.0, target=1.0001, objective_from="plain",
                plain_s=plain[0], plain_iters=plain[1], plain_reached=reached[0],
                batch_s=batch[0], batch_iters=batch[1], batch_reached=reached[1],
                warm_s=warm[0], warm_net_s=0.001, warm_iters=warm[1], warm_reached=reached[2],
                fallback=fallback, race_s=min(warm[0], batch[0]), race_winner=winner)


def test_summary_sums_ratios_and_rows():
    rows = [_row(64, (1.0, 100), (0.2, 30), (0.1, 5), "warm"),
            _row(128, (3.0, 1000), (1.0, 1000), (0.5, 40), "flat", reached=(True, False, True), fallback=True)]
    s = T.summarize(rows)
    assert s["problems"] == 2
    assert s["plain_s"] == pytest.approx(4.0) and s["batch_s"] == pytest.approx(1.2)
    assert s["speedup_batch_vs_plain"] == pytest.approx(4.0 / 1.2)
    assert s["speedup_warm_vs_plain"] == pytest.approx(4.0 / 0.6)
    assert s["batch_reached"] == 1 and s["fallbacks"] == 1
    assert s["race_winners"] == {"warm": 1, "flat": 1, "flat_fr": 0, "none": 0}
    assert s["median_ratio_warm_vs_plain"] == pytest.approx((10.0 + 6.0) / 2)
    pp = s["per_problem_iters"]
    assert pp["columns"] == ["width", "plain", "batch", "warm"]
    # a run that missed the target is reported with a negative iteration count
    assert pp["rows"] == [[64, 100, 30, 5], [128, 1000, -1000, 40]]
