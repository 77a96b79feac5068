"""Step scheduler of a closed loop.

Public interface as the reference's ``LoopControl`` (specula/loop_control.py):
``add(obj, idx)``, ``remove_all()``, ``niters()``, ``run(...)``,
``start(...)``, ``iter()`` and ``finish()``, with the same meaning of the
arguments.  Objects are grouped by trigger order; within one step every
group runs ``check_ready`` on all its members, then ``trigger``, then
``post_trigger``, and groups run in increasing order.  Times are the
integer nanosecond ticks of ``BaseTimeObj``.

The implementation is this package's own: a sorted table of stages, a
``LoopClock`` record for the time bookkeeping and a rolling window of step
timestamps for the optional rate report.  Every object of a loop launches
on the current CUDA stream of its device, so a step issues its kernels
without host synchronisation; ``iter`` itself never waits on the GPU.
"""
import bisect
import time
from collections import deque
from dataclasses import dataclass

from specula_b200.base_time_obj import BaseTimeObj


@dataclass
class LoopClock:
    """Integer-tick time bookkeeping of one run."""
    t: int = 0              # tick of the step about to run
    dt: int = 0             # ticks per step
    t0: int = 0             # first tick
    duration: int = 0       # ticks to run after t0
    stop_tick: int = 0      # raise StopIteration once t reaches it (0: never)

    @property
    def end(self):
        return self.t0 + self.duration


class LoopControl(BaseTimeObj):
    # steps averaged by the rate report
    REPORT_WINDOW = 10

    def __init__(self, verbose=False):
        super().__init__(target_device_idx=-1, precision=1)
        self.verbose = verbose
        self._orders = []          # sorted trigger orders
        self._stages = {}          # order -> objects in insertion order
        self.clock = LoopClock()
        self._watch = None         # data object whose refresh ends a step early
        self._report = False
        self._stamps = deque(maxlen=self.REPORT_WINDOW + 1)

    # ---- membership ------------------------------------------------------
    def add(self, obj, idx):
        """Schedule ``obj`` in trigger group ``idx`` (lower runs first)."""
        if obj is None:
            raise ValueError('LoopControl.add: got None where a processing object was expected')
        if idx not in self._stages:
            bisect.insort(self._orders, idx)
            self._stages[idx] = []
        self._stages[idx].append(obj)

    def remove_all(self):
        self._orders = []
        self._stages = {}

    def _each(self):
        for idx in self._orders:
            yield from self._stages[idx]

    # ---- time ------------------------------------------------------------
    @property
    def t(self):
        """Tick of the step that ``iter`` runs next."""
        return self.clock.t

    @property
    def dt(self):
        """Ticks per step."""
        return self.clock.dt

    def niters(self):
        """Number of steps of the configured run (0 with a zero time step)."""
        c = self.clock
        return c.end / c.dt if c.dt else 0

    # ---- running ---------------------------------------------------------
    def start(self, run_time, dt, t0=0, stop_on_data=None, stop_at_time=None, speed_report=False):
        """Set the clock up and call ``setup()`` on every object in trigger order."""
        self.clock = LoopClock(t=self.seconds_to_t(t0), dt=self.seconds_to_t(dt), t0=self.seconds_to_t(t0),
                               duration=self.seconds_to_t(run_time),
                               stop_tick=self.seconds_to_t(stop_at_time) if stop_at_time else 0)
        self._watch = stop_on_data
        self._report = bool(speed_report)
        self._stamps.clear()
        for obj in self._each():
            obj.setup()

    def iter(self):
        """One loop step at the current tick, then advance the clock."""
        now = self.clock.t
        for idx in self._orders:
            stage = self._stages[idx]
            for obj in stage:
                obj.check_ready(now)
            for obj in stage:
                try:
                    obj.trigger()
                except Exception as exc:
                    exc.add_note(f'raised while triggering {type(obj).__name__} (trigger order {idx}, t={now})')
                    raise
            for obj in stage:
                obj.post_trigger()
        if self._watch is not None and self._watch.generation_time == now:
            # the watched output was refreshed: this step ends here and the
            # clock stays, as the reference's stop_on_data does
            return
        if self.clock.stop_tick and now >= self.clock.stop_tick:
            raise StopIteration
        if self._report:
            self._rate_report(now)
        self.clock.t = now + self.clock.dt

    def _rate_report(self, now):
        self._stamps.append(time.perf_counter())
        if len(self._stamps) == self._stamps.maxlen:
            span = self._stamps[-1] - self._stamps[0]
            print(f't={self.t_to_seconds(now):.6f} {(len(self._stamps) - 1) / span:.2f} Hz')
            self._stamps.clear()
            self._stamps.append(time.perf_counter())

    def run(self, run_time, dt, t0=0, stop_on_data=None, stop_at_time=None, speed_report=False):
        """``start``, steps until ``run_time`` has elapsed, then ``finish``."""
        self.start(run_time, dt, t0=t0, stop_on_data=stop_on_data, stop_at_time=stop_at_time,
                   speed_report=speed_report)
        while self.clock.t < self.clock.end:
            self.iter()
        self.finish()

    def finish(self):
        """``finalize()`` on every object in trigger order."""
        for obj in self._each():
            obj.finalize()
