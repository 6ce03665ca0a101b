"""The bench's clock record: the nvidia-smi sampler's rows become the median SM
clock under load, the maximum clock and the throttle reasons seen (a run with
hw_slowdown, hw_thermal_slowdown or sw_thermal_slowdown is re-measured; a
sw_power_cap is kept and noted).  CPU only: nvidia-smi is replaced by a fake."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HEADER_FREE_ROWS = """\
2026/12/04 01:00:00.000, 1965, 1965, 512.3, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active
2026/12/04 01:00:00.100, 1965, 1965, 780.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active
2026/12/04 01:00:00.200, 1830, 1965, 998.7, 0x0000000000000004, Not Active, Not Active, Not Active, Active
2026/12/04 01:00:00.300, 345, 1965, 120.0, 0x0000000000000001, Not Active, Not Active, Not Active, Not Active
garbled line
"""


class _FakeProc:
    def __init__(self, out):
        self.out = out

    def terminate(self):
        pass

    def communicate(self, timeout=None):
        return self.out, ''

    def kill(self):
        pass


def _clocks(monkeypatch, out):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setattr(bench.subprocess, 'Popen', lambda *a, **k: _FakeProc(out))
    return bench.Clocks().stop()


def test_clock_record_median_under_load_and_reasons(monkeypatch):
    ck = _clocks(monkeypatch, HEADER_FREE_ROWS)
    assert ck['samples'] == 4
    assert ck['sm_max_mhz'] == 1965.0
    assert ck['sm_mhz'] == 1965.0              # idle sample (345 MHz) left out of the median
    assert ck['reasons'] == ['sw_power_cap']


def test_clock_record_of_a_throttled_run(monkeypatch):
    rows = HEADER_FREE_ROWS.replace('Not Active, Not Active, Not Active, Active',
                                    'Active, Not Active, Active, Not Active')
    ck = _clocks(monkeypatch, rows)
    assert ck['reasons'] == ['hw_slowdown', 'sw_thermal_slowdown']


def test_clock_record_without_samples(monkeypatch):
    assert _clocks(monkeypatch, '') is None
