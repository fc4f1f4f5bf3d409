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


class _FakeRec:
    """Stands in for a Reconstructor: cg() returns a fixed outcome and records its arguments."""

    def __init__(self, reached, iters):
        self.reached, self.iters, self.calls = reached, iters, []

    def set_image(self, img):
        pass

    def cg(self, iters, **kw):
        self.calls.append(kw)
        return {"reached": self.reached, "iterations": self.iters}


class _FakeProblem:
    def start_image(self):
        return None


class _FakeFlag:
    ptr = 0

    def reset(self):
        pass


@pytest.mark.parametrize("outcomes, expect", [
    ((True, False, False), "warm"),
    ((False, True, False), "flat"),
    ((False, False, True), "flat_fr"),
    ((False, False, False), "none"),
])
def test_race_winner_and_runner_settings(monkeypatch, outcomes, expect):
    import gpair_b200.warmstart as W
    monkeypatch.setattr(W, "features", lambda rec, p: None)
    monkeypatch.setattr(W, "warm_start", lambda net, rec, p, f: None)
    warm, flat, fr = (_FakeRec(r, 10 + i) for i, r in enumerate(outcomes))
    out = T.race(warm, flat, _FakeProblem(), None, 100, 1.0, _FakeFlag(), rec3=fr)
    assert out["race_winner"] == expect
    assert (out["race_warm_iters"], out["race_flat_iters"], out["race_flat_fr_iters"]) == (10, 11, 12)
    # every runner uses the batched search, the shared stop flag and the same target;
    # the third runner alone uses the Fletcher-Reeves beta
    for rec, method in ((warm, 2), (flat, 2), (fr, 1)):
        (kw,) = rec.calls
        assert kw["method"] == method and kw["target_J"] == 1.0 and kw["stop_flag"] == 0


def test_race_without_third_runner(monkeypatch):
    import gpair_b200.warmstart as W
    monkeypatch.setattr(W, "features", lambda rec, p: None)
    monkeypatch.setattr(W, "warm_start", lambda net, rec, p, f: None)
    out = T.race(_FakeRec(False, 7), _FakeRec(True, 5), _FakeProblem(), None, 100, 1.0, _FakeFlag())
    assert out["race_winner"] == "flat" and "race_flat_fr_iters" not in out
