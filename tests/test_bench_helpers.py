"""Host-side helpers of bench.py (no GPU): the summary of the nvidia-smi clock
samples that goes into the bench line, and the DRAM-traffic figure chosen for
the roofline of the dominant kernel family."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _row(mhz, reasons=("Not Active",) * 4, mx=1965):
    return f"0, {mhz}, {mx}, 900.0, 0x0, " + ", ".join(reasons) + "\n"


def test_clock_summary_counts_only_the_timed_region():
    b = _bench()
    rows = [_row(900), _row(1965), _row(1965), _row(1950)]
    out = b.parse_clock_samples(rows, skip=1)  # the idle sample before the region is dropped
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}
    # a region shorter than the sampling period keeps the one sample there is
    assert b.parse_clock_samples(rows[:1], skip=1)["samples"] == 1
    assert b.parse_clock_samples([], skip=0) is None
    assert b.parse_clock_samples(["garbage\n", "0, [N/A], 1965, x, y, a, b, c, d\n"]) is None


def test_clock_summary_reports_throttle_reasons():
    b = _bench()
    rows = [_row(1965), _row(1800, ("Not Active", "Not Active", "Not Active", "Active")),
            _row(1700, ("Active", "Not Active", "Not Active", "Not Active"))]
    out = b.parse_clock_samples(rows)
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert out["sm_mhz"] == 1800.0 and out["samples"] == 3


def test_traffic_figures_cover_the_production_families():
    b = _bench()
    t = b.TRAFFIC_PER_CELL
    # the pipelined sweep moves about the contract's 42 words of 4 B a cell per launch
    assert 160 < t["energy_sweeps:fp32:redblack:pipe"] < 190
    assert 8 * t["energy_sweeps:fp32:redblack"] < 1.1 * t["energy_sweeps:fp32:redblack:pipe"]
    for fam in ("energy_assemble", "h2t_meltpool"):
        assert f"{fam}:fp32:redblack" in t


def test_clock_sampler_end_to_end_with_a_stand_in_nvidia_smi(tmp_path, monkeypatch):
    """Clocks.start/stop around a short region, with a stand-in nvidia-smi on PATH
    that prints one sample row every 50 ms."""
    import time
    b = _bench()
    fake = tmp_path / "nvidia-smi"
    fake.write_text("#!/bin/sh\nwhile true; do echo '0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, "
                    "Not Active, Not Active'; sleep 0.05; done\n")
    fake.chmod(0o755)
    monkeypatch.setenv("PATH", f"{tmp_path}:{os.environ.get('PATH', '')}")
    c = b.Clocks(0)
    c.start()
    time.sleep(0.3)
    out = c.stop()
    assert out is not None and out["samples"] >= 1, out
    assert out["sm_mhz"] == 1965.0 and out["reasons"] == []
