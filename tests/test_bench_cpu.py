"""Host-side pieces of bench.py that need no GPU."""
import bench


class _FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _sampler(lines):
    s = bench.ClockSampler(0)
    s.proc = _FakeProc()
    s.lines = list(lines)
    return s


def test_clock_sampler_median_max_and_reasons():
    # index, sm MHz, max MHz, power, active mask, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
             "0, 1900, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
             "0, 1950, 1965, 980.0, 0x4, Not Active, Not Active, Not Active, Active",
             "garbage line",
             "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, Not Active"]
    out = _sampler(lines).stop()
    assert out["sm_mhz"] == 1950.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"] and out["samples"] == 3


def test_clock_sampler_reports_thermal_and_hw_slowdown():
    lines = ["0, 1500, 1965, 900, 0x48, Active, Not Active, Active, Not Active"]
    out = _sampler(lines).stop()
    assert out["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"]


def test_clock_sampler_without_nvidia_smi():
    s = bench.ClockSampler(0)
    assert s.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_cpu_sample_problem_keeps_the_data():
    import gpair_b200 as g
    p = g.workload_problem("tiny")
    s = bench.cpu_sample_problem(p, 16)
    assert s.width == 16 and s.nuv == p.nuv and s.npow == p.npow and s.nbis == p.nbis
    assert (s.data == p.data).all() and s.model.shape == (16 * 16,)
