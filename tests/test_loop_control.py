"""Host logic of the step scheduler and the input slots (no device)."""
import pytest

from specula_b200.base_value import BaseValue
from specula_b200.connections import InputList, InputValue
from specula_b200.loop_control import LoopControl


class Recorder:
    def __init__(self, name, log, fail_at=None):
        self.name, self.log, self.fail_at = name, log, fail_at
        self.t = None

    def setup(self):
        self.log.append((self.name, 'setup'))

    def check_ready(self, t):
        self.t = t
        self.log.append((self.name, 'ready', t))

    def trigger(self):
        if self.fail_at is not None and self.t == self.fail_at:
            raise RuntimeError('boom')
        self.log.append((self.name, 'trigger'))

    def post_trigger(self):
        self.log.append((self.name, 'post'))

    def finalize(self):
        self.log.append((self.name, 'finalize'))


def test_groups_run_in_order_with_phases_per_group():
    log = []
    loop = LoopControl()
    a, b, c = Recorder('a', log), Recorder('b', log), Recorder('c', log)
    loop.add(c, 5)
    loop.add(a, 0)
    loop.add(b, 0)
    loop.run(0.002, 0.001)
    # setup in trigger order, then per step: group 0 (ready, ready, trigger, trigger, post, post), then group 5
    assert log[:3] == [('a', 'setup'), ('b', 'setup'), ('c', 'setup')]
    step0 = log[3:12]
    assert step0 == [('a', 'ready', 0), ('b', 'ready', 0), ('a', 'trigger'), ('b', 'trigger'), ('a', 'post'),
                     ('b', 'post'), ('c', 'ready', 0), ('c', 'trigger'), ('c', 'post')]
    assert log[12] == ('a', 'ready', 1_000_000)
    assert log[-3:] == [('a', 'finalize'), ('b', 'finalize'), ('c', 'finalize')]
    assert loop.t == 2_000_000 and loop.dt == 1_000_000 and loop.niters() == 2


def test_stop_at_time_and_stop_on_data():
    log = []
    loop = LoopControl()
    loop.add(Recorder('a', log), 0)
    loop.start(1.0, 0.001, stop_at_time=0.002)
    loop.iter()
    loop.iter()
    with pytest.raises(StopIteration):
        loop.iter()
    data = BaseValue(value=[0.0])
    data.generation_time = 0
    loop.start(1.0, 0.001, stop_on_data=data)
    loop.iter()                 # the watched data carries this step's time: the clock stays
    assert loop.t == 0


def test_exception_names_the_object():
    loop = LoopControl()
    loop.add(Recorder('a', [], fail_at=1_000_000), 0)
    loop.start(1.0, 0.001)
    loop.iter()
    with pytest.raises(RuntimeError) as ei:
        loop.iter()
    assert any('Recorder' in n for n in getattr(ei.value, '__notes__', []))


def test_add_rejects_none_and_remove_all():
    loop = LoopControl()
    with pytest.raises(ValueError):
        loop.add(None, 0)
    log = []
    loop.add(Recorder('a', log), 2)
    loop.remove_all()
    loop.run(0.001, 0.001)
    assert log == []


def test_input_slots_type_check_and_times():
    v = InputValue(type=BaseValue)
    assert v.get(-1) is None and v.get_time() is None
    with pytest.raises(ValueError):
        v.set(3.0)
    x = BaseValue(value=[1.0])
    x.generation_time = 7
    v.set(x)
    assert v.get(x.target_device_idx) is x and v.get_time() == 7
    lst = InputList(type=BaseValue, optional=True)
    assert lst.optional and lst.get(-1) is None and lst.get_time() == []
    y = BaseValue(value=[2.0])
    y.generation_time = 9
    lst.set([x, y])
    assert lst.get(x.target_device_idx) == [x, y] and lst.get_time() == [7, 9]
    with pytest.raises(ValueError):
        lst.set([x, 'no'])
