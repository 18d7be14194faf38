"""bench.py's committed inputs, on the CPU: the ncu traffic record that the roofline object of
the bench line reads, and the peak it divides by when no measured peak is present."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_traffic_record_has_what_the_roofline_reads():
    b = _bench()
    tr = b.load_traffic()
    assert tr is not None
    for key in ("vertices", "warmup", "dram_bytes_per_launch", "algorithmic_bytes_per_launch", "cbar_at_capture",
                "summary"):
        assert key in tr, key
    assert tr["dram_bytes_per_launch"] == tr["dram_bytes_read_per_launch"] + tr["dram_bytes_write_per_launch"]
    assert abs(tr["dram_bytes_per_launch"] / tr["vertices"] - tr["dram_bytes_per_vertex"]) < 0.1
    # the algorithmic bytes follow the Newton iteration's byte model at the captured contact count
    alg = tr["vertices"] * (b.ITER_BYTES_BASE + b.ITER_BYTES_PER_CONTACT * tr["cbar_at_capture"])
    assert abs(alg - tr["algorithmic_bytes_per_launch"]) / alg < 1e-3
    assert os.path.exists(os.path.join(ROOT, tr["summary"]))


def test_peak_is_measured_or_the_stated_fallback():
    b = _bench()
    peak, kind = b.load_peaks()
    if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")):
        assert kind == "measured" and peak > 0
    else:
        assert (peak, kind) == (6650.0, "fallback")
