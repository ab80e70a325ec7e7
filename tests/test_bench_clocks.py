"""bench.py's clock record keeps only the nvidia-smi samples taken inside the timed loop.

Host logic only: a synthetic sample log (idle clocks before and after the loop, one sample with
the power cap active inside it) goes through ClockSampler.stop(); no GPU and no nvidia-smi.
"""
import datetime
import importlib.util
import os
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _DoneProcess:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        pass

    def kill(self):
        pass


def _sampler_with_log(bench, t0, rows):
    c = bench.ClockSampler("0")
    c.t0, c.t1 = t0, t0 + datetime.timedelta(milliseconds=150)
    f = tempfile.NamedTemporaryFile("w+", delete=False)
    f.write("\n".join(rows))
    f.flush()
    c.proc, c.f = _DoneProcess(), f
    return c


def test_clock_samples_outside_the_timed_loop_are_dropped():
    bench = _bench()
    t0 = datetime.datetime.now()
    rows = []
    for k in range(-10, 20):   # every 20 ms from 200 ms before the loop to 380 ms after its start
        t = t0 + datetime.timedelta(milliseconds=20 * k)
        inside = 0 <= k <= 7
        rows.append("%s, 0, %d, 1965, %.1f, 0x0, Not Active, Not Active, Not Active, %s" % (
            t.strftime("%Y/%m/%d %H:%M:%S.%f")[:-3], 1965 if inside else 345, 600.0 if inside else 90.0,
            "Active" if k == 3 else "Not Active"))
    rec = _sampler_with_log(bench, t0, rows).stop()
    assert rec["sm_mhz"] == 1965.0 and rec["sm_max_mhz"] == 1965.0
    assert 8 <= rec["samples"] <= 10          # the loop's samples plus at most one on each edge
    assert rec["reasons"] == ["sw_power_cap"]
    assert rec["power_w_max"] == 600.0


def test_clock_samples_with_unparsable_timestamps_are_all_kept():
    bench = _bench()
    rows = ["not-a-time, 0, 1900, 1965, 300.0, 0x0, Not Active, Not Active, Not Active, Not Active"] * 4
    rec = _sampler_with_log(bench, datetime.datetime.now(), rows).stop()
    assert rec["samples"] == 4 and rec["sm_mhz"] == 1900.0 and rec["reasons"] == []
