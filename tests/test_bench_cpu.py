"""Host-side pieces of bench.py that need no GPU."""
import bench
from gpair_b200.clocks import ClockSampler


class _FakeProc:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0

    def kill(self):
        pass


def _sampler(lines):
    s = ClockSampler(0)
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
    s = ClockSampler(0)
    assert s.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_reference_sample_is_one_channel_indexed_by_the_reference():
    """The CPU sample holds the middle channel and every SAMPLE_HA_STRIDE-th hour
    angle of the workload's tables, indexed by the reference's own getoifits.c;
    this project's indexer gives the same indices."""
    import os

    import numpy as np
    import pytest

    import gpair_b200 as g
    from gpair_b200 import synth
    from oracle import oracle as O

    if not os.path.exists(O.REF_LIB):
        pytest.skip("the reference's getoifits.c is not built here")
    w, oi = synth.make_workload_data("tiny")
    s = bench.reference_sample("tiny", oi, width=16)
    _, oifits_mod = bench.data_modules()
    cfg = w.array
    nbl, ntr = cfg.n_tel * (cfg.n_tel - 1) // 2, oi.t3[0].t3amp.shape[0] // cfg.n_ha
    ha = np.arange(0, cfg.n_ha, bench.SAMPLE_HA_STRIDE)
    rows_v2 = (ha[:, None] * nbl + np.arange(nbl)[None, :]).ravel()
    rows_t3 = (ha[:, None] * ntr + np.arange(ntr)[None, :]).ravel()
    sub = bench.subset_channels(oi, [s["channel"]], oifits_mod, rows_v2, rows_t3)
    ix = g.index_oifits(sub)
    assert s["channel"] == 1 and s["channels"] == 2 and s["width"] == 16
    assert s["npow"] == ix.npow == len(ha) * nbl
    assert s["nbis"] == ix.nbis == len(ha) * ntr
    assert s["data_scale"] == 2 * cfg.n_ha / len(ha)
    assert np.array_equal(s["uv"], ix.uv) and np.array_equal(s["uvpnt"], ix.uvpnt)
    assert np.array_equal(s["sign"], ix.sign)
    assert s["model"].shape == (16 * 16,)


def test_reference_arm_maps_no_library_of_this_project():
    """`bench.py --impl reference` in a fresh process: the reference's compiled
    cpu.c / getoifits.c run, libgpair_b200.so is never mapped."""
    import json
    import os
    import subprocess
    import sys

    import pytest

    from oracle import oracle as O

    if not os.path.exists(O.REF_LIB):
        pytest.skip("the reference's cpu.c is not built here")
    r = subprocess.run([sys.executable, os.path.join(bench.ROOT, "bench.py"), "--impl", "reference", "--workload",
                        "tiny", "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    libs = line["native_libraries"]
    assert any(x.startswith("oracle/") for x in libs), libs
    assert not any("libgpair_b200" in x for x in libs), libs
    assert line["higher_is_better"] is True and line["unit"] == bench.UNIT and line["metric"] == bench.METRIC
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["cpu_baseline"]["cores"] == (os.cpu_count() or 1)
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_small_workload_reference_cg_runs_on_the_reference_code():
    """The CPU side of the 64x64 plain-method block: the reference's own compiled
    code builds the data (getoifits.c, init_data, set_model) at the workload's
    own size, and a few CG iterations through its cpu.c descend from the flat
    start."""
    import os

    import pytest

    from oracle import oracle as O

    if not os.path.exists(O.REF_LIB) or not os.path.exists(O.REF_MAIN_LIB):
        pytest.skip("reference library not built")
    ref = bench.reference_problem("small")
    assert ref["width"] == 64 and ref["npow"] == 900 and ref["nbis"] == 600
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)  # cpu.c's image2vis prints on every call
    try:
        out = bench.small_plain_cg_cpu(3)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)
    assert out["kind"] == "reference" and out["cores"] == 1
    assert out["grad_evals"] >= 3 and out["J"] > 0


def test_stage_report_instance_workloads_match_the_profiled_problems():
    """stage_report's instance:SEED workloads are the many-instance generator's
    problems (the small-image trial-forward profiles use seeds 30,000,000 and
    30,000,040)."""
    from gpair_b200 import stage_report
    p = stage_report.problem("instance:30000000")
    assert p.width == 64 and p.nuv == 6871 and p.nbis == 4576
    p = stage_report.problem("instance:30000040")
    assert p.width == 128 and p.nuv == 5664 and p.nbis == 3776
