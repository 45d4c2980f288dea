"""bench.py's clock sampler on the CPU, against a stand-in nvidia-smi that
streams fixed samples: the summary keeps the samples of the timed region,
reports the active throttle reasons, and says when nothing was sampled."""
import os
import stat
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def fake_smi(tmp_path, line):
    p = tmp_path / "nvidia-smi"
    p.write_text("#!/bin/sh\nwhile true; do echo '%s'; sleep 0.02; done\n" % line)
    p.chmod(p.stat().st_mode | stat.S_IEXEC)
    return str(tmp_path)


def test_samples_of_the_timed_region(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", fake_smi(tmp_path, "1965, 1965, Not Active, Not Active, "
                                                   "Not Active, Active")
                       + os.pathsep + os.environ["PATH"])
    sys.path.insert(0, ROOT)
    import bench
    cs = bench.ClockSampler(0)
    cs.start()
    time.sleep(0.3)
    cs.begin()
    time.sleep(0.5)
    cs.end()
    time.sleep(0.2)
    cs.stop()
    s = cs.summary()
    assert s["window"] == "timed region" and s["samples"] >= 5
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"]
    # every kept sample lies inside the region
    assert len(cs.samples) > s["samples"]


def test_no_sampler_available(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))  # no nvidia-smi at all
    sys.path.insert(0, ROOT)
    import bench
    cs = bench.ClockSampler(0)
    cs.start()
    cs.begin()
    cs.end()
    cs.stop()
    assert cs.summary()["reasons"] == ["unsampled"]
