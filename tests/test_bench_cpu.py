"""Host logic of bench.py that runs without a GPU: the clock sampler keeps
only the samples taken inside the timed region (or the nearest one when the
region is shorter than the sampling period) and reports the throttle reasons
seen there; the ncu traffic figure is read from the committed profile
summary; library options given on the command line reach the simulation."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def line(sm, mx=1965, reasons=('Not Active',) * 4):
    return '%d, %d, 700.0, %s' % (sm, mx, ', '.join(reasons))


def test_clock_sampler_window():
    c = bench.ClockSampler(0, period_ms=25)
    c.t0, c.t1 = 10.0, 10.1
    c.lines = [(9.0, line(345)),                     # idle, before the region
               (10.02, line(1965)),
               (10.07, line(1950, reasons=('Not Active', 'Not Active', 'Not Active', 'Active'))),
               (10.12, line(1965)),                  # inside the slack after the region
               (11.0, line(400))]                    # long after
    s = c.summary()
    assert s['samples'] == 3
    assert s['sm_mhz'] == 1965.0 and s['sm_max_mhz'] == 1965.0
    assert s['reasons'] == ['sw_power_cap']


def test_clock_sampler_nearest_sample():
    c = bench.ClockSampler(0, period_ms=200)
    c.t0, c.t1 = 10.0, 10.01
    c.lines = [(9.3, line(300)), (9.95, line(1965)), (12.0, line(300))]
    s = c.summary()
    assert s['samples'] == 1 and s['sm_mhz'] == 1965.0


def test_clock_sampler_without_nvidia_smi():
    c = bench.ClockSampler(0)
    c.t0, c.t1 = 0.0, 1.0
    assert c.summary() == {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}


def test_profile_traffic_figure():
    t = bench.ncu_traffic_per_particle()
    assert t is not None and 40.0 < t < 60.0      # bytes per particle from the committed ncu summary


def test_options_reach_the_simulation():
    class Args:
        reorder = 40

    class Sim:
        def __init__(self):
            self.opts = {}

        def set_option(self, k, v):
            self.opts[k] = v

    s = bench.apply_options(Sim(), Args())
    assert s.opts == {'reorder': 40}
    assert bench.apply_options(Sim(), None).opts == {}
