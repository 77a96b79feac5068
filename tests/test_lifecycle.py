"""Input freshness of the processing-object life cycle (no device): an
object is due when one of its inputs carries a generation time newer than
the one it consumed last (any time >= 0 for an input never consumed), an
object without inputs is always due, and a due object stays due until it
is triggered (base_processing_obj.py:38-58, 60-160)."""
from specula_b200.base_processing_obj import BaseProcessingObj
from specula_b200.base_value import BaseValue
from specula_b200.connections import InputList, InputValue


class Counter(BaseProcessingObj):
    def __init__(self):
        super().__init__(target_device_idx=-1, precision=1)
        self.runs = 0

    def trigger_code(self):
        self.runs += 1


def _value(t):
    v = BaseValue(value=[0.0], target_device_idx=-1)
    v.generation_time = t
    return v


def test_object_without_inputs_is_always_due():
    c = Counter()
    for t in range(3):
        assert c.check_ready(t)
        c.trigger()
    assert c.runs == 3


def test_single_input_due_on_new_times_only():
    c = Counter()
    c.inputs['in'] = InputValue(type=BaseValue)
    v = _value(-1)
    c.inputs['in'].set(v)
    assert not c.check_ready(0)             # never produced
    v.generation_time = 0
    assert c.check_ready(0)                 # first value, time 0
    assert c.local_inputs['in'] is v
    c.trigger()
    assert not c.check_ready(1)             # nothing newer
    assert c.check_ready(1) is False
    v.generation_time = 5
    assert c.check_ready(5)
    assert c.check_ready(6)                 # still due: not triggered yet
    c.trigger()
    assert not c.check_ready(6)
    assert c.runs == 2
    assert c.current_time == 6


def test_list_input_due_when_any_member_is_newer():
    c = Counter()
    c.inputs['lst'] = InputList(type=BaseValue)
    a, b = _value(-1), _value(-1)
    c.inputs['lst'].set([a, b])
    assert not c.check_ready(0)
    b.generation_time = 2
    assert c.check_ready(2)
    assert c.local_inputs['lst'] == [a, b]
    c.trigger()
    assert not c.check_ready(3)
    a.generation_time = 1                   # newer than a's consumed -1
    assert c.check_ready(3)
    c.trigger()
    assert not c.check_ready(4)
    assert c.runs == 2


def test_any_fresh_input_makes_the_object_due():
    c = Counter()
    c.inputs['a'] = InputValue(type=BaseValue)
    c.inputs['b'] = InputValue(type=BaseValue, optional=True)     # never connected
    a = _value(3)
    c.inputs['a'].set(a)
    assert c.check_ready(3)
    assert c.local_inputs['b'] is None
    c.trigger()
    assert not c.check_ready(4)
    b = _value(4)
    c.inputs['b'].set(b)
    assert c.check_ready(4)                 # the newly connected input carries time 4
    c.trigger()
    assert not c.check_ready(5)
    assert c.runs == 2


def test_lenslet_grid_and_calibrator_boxes():
    """Lenslet.get(i, j) = [x, y, side] on the make_xy grid (x along j), and
    the calibrator's per-lenslet pixel boxes, as the oracle's sub-aperture
    detection builds them (sh_subap_calibrator.py:47-60)."""
    import numpy as np
    from specula_b200.data_objects.lenslet import Lenslet
    from specula_b200.processing_objects.sh_subap_calibrator import lenslet_boxes
    for n, side in ((1, 8), (4, 24), (8, 64), (12, 72), (20, 160), (40, 240)):
        lens = Lenslet(n)
        assert (lens.dimx, lens.dimy) == (n, n)
        centres = (np.arange(n) - (n - 1) / 2.0) / (n / 2.0)
        for i in range(n):
            for j in range(n):
                x, y, size = lens.get(i, j)
                assert abs(x - centres[j]) < 1e-12 and abs(y - centres[i]) < 1e-12 and size == 2.0 / n
        boxes, np_sub = lenslet_boxes(n, side)
        assert np_sub == round(side / 2.0 * 2.0 / n)
        want = []
        for i in range(n):
            for j in range(n):
                xc, yc = side / 2.0 * (1 + centres[j]), side / 2.0 * (1 + centres[i])
                want.append((int(np.round(xc - np_sub / 2)), int(np.round(xc + np_sub / 2)),
                             int(np.round(yc - np_sub / 2)), int(np.round(yc + np_sub / 2))))
        assert boxes == want
