"""Live ring-buffer mode, host side (no GPU): FrameClock (camera.ts:306-426)
slot/mask/guard/shuffle rules and the analysis tick's stale-result rule
(main.ts:366-398), against a stand-in engine."""
import math

import numpy as np
import pytest

from hackathon_b200.live import FrameClock, LiveAnalyzer, shuffle_order


def test_slots_duplicates_missed_and_gap_reset():
    c = FrameClock(fps=100.0, T=8)           # 10 ms grid
    assert c.place(1000.0) == dict(slot=0, n=0)
    assert c.place(1010.4) == dict(slot=1, n=1)
    assert c.place(1012.0) is None           # rounds to n = 1 again
    assert c.duplicates == 1
    assert c.place(1040.0) == dict(slot=4, n=4)
    assert c.missed == 2                     # n = 2, 3 never arrived
    assert c.place(1095.0) == dict(slot=2, n=10)   # Math.round(9.5) = 10
    assert c.validCount == 2                 # window n = 3..10 holds frames 4 and 10
    c.place(1200.0)                          # n = 20: gap of 10 > T restarts the clock
    assert c.resets == 1 and c.newestN == 0


def test_valid_count_window():
    c = FrameClock(fps=100.0, T=8)
    for n in range(12):
        c.place(1000.0 + 10 * n)
    assert c.validCount == 8
    c.drop(11)
    c.drop(3)                                # already overwritten by 11: no effect
    assert c.validCount == 7


def test_media_time_switch_resets():
    c = FrameClock(fps=30.0, T=16)
    c.place(0.0, "captureTime")
    c.place(33.4, "watchdog")                # capture and watchdog stamps mix freely
    assert c.resets == 0
    c.place(5000.0, "mediaTime")
    assert c.resets == 1 and c.newestN == 0 and c.timeSource == "mediaTime"


def test_snapshot_guard_and_order():
    c = FrameClock(fps=100.0, T=8)
    for n in range(11):                      # frames 0..10; frame 7 dropped
        p = c.place(1000.0 + 10 * n)
        if n == 7:
            c.drop(p["n"])
    s = c.snapshot(guard=2)
    # time index j holds frame n = 3 + j in slot n mod 8
    assert s.order.tolist() == [(3 + j) % 8 for j in range(8)]
    assert s.mask.tolist() == [0, 0, 1, 1, 0, 1, 1, 1]   # guard masks j < 2; frame 7 dropped
    assert s.used == 5 and s.newestN == 10


def test_shuffle_is_a_joint_permutation():
    c = FrameClock(fps=100.0, T=16)
    for n in range(20):
        c.place(10.0 * n)
    s0 = c.snapshot(guard=3)
    rng = np.random.default_rng(5)
    s1 = c.snapshot(guard=3, shuffle=True, rand=rng.random)
    pairs0 = sorted(zip(s0.order.tolist(), s0.mask.tolist()))
    pairs1 = sorted(zip(s1.order.tolist(), s1.mask.tolist()))
    assert pairs0 == pairs1 and s1.used == s0.used
    assert s1.order.tolist() != s0.order.tolist()
    o, m = shuffle_order([0, 1, 2], [1, 1, 0], lambda: 0.0)   # j = 0 every step
    assert o.tolist() == [1, 2, 0] and m.tolist() == [1, 0, 1]


class _Engine:
    """Stand-in for DdmEngine: records calls; the analysis completes when
    the test says so."""

    def __init__(self):
        self.ingested, self.calls, self.done = [], [], False
        self.saturated = False

    def ingest_frames(self, frames, slots, scale=None):
        self.ingested.append(int(slots[0]))

    def compute_temporal(self, order, mask, live=False):
        self.calls.append((np.array(order), np.array(mask), live))
        self.done = False

    @property
    def analysis_done(self):
        return self.done

    def read_radial(self):
        return "radial"


def test_tick_collect_stale_guard_widening():
    clock = FrameClock(fps=100.0, T=16)
    eng = _Engine()
    la = LiveAnalyzer(eng, clock, opt={}, worker=None, guard=4)
    frame = np.zeros((8, 8), np.uint16)
    for n in range(10):
        la.on_frame(frame, 10.0 * n)
    assert la.start() == "collecting"        # 10 < 12 = 0.75 T
    for n in range(10, 20):
        la.on_frame(frame, 10.0 * n)
    assert la.start() == "started" and la.busy
    order, mask, live = eng.calls[-1]
    assert live and mask[:4].sum() == 0      # the guard's time indices
    assert la.finish(block=False) is None    # still running
    for n in range(20, 26):                  # 6 frames arrive during the analysis
        la.on_frame(frame, 10.0 * n)
    eng.done = True
    r = la.finish(block=False)
    assert r["status"] == "stale" and la.stale == 1
    assert la.guard == min(128, math.ceil(6 * 1.5) + 4) == 13


def test_back_pressure_drops_the_frame():
    clock = FrameClock(fps=100.0, T=16)
    eng = _Engine()
    la = LiveAnalyzer(eng, clock)
    eng.saturated = True
    la.on_frame(np.zeros((8, 8)), 0.0)
    assert la.throttled == 1 and clock.validCount == 0 and eng.ingested == []
