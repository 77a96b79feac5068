"""DataStore (processing_objects/data_store.py): recorded series written in
the reference's FITS / pickle layout and read back (FITS also with the
independent harness reader); on CPU objects here, on the GPU in
tests/test_gpu_data_store.py."""
import os
import pickle

import numpy as np
import pytest
import torch

from tests.golden import fits_min


def run_store(tmp_path, fmt, device_idx, steps=5, flush_steps=2):
    from specula_b200.connections import InputValue
    from specula_b200.base_value import BaseValue
    from specula_b200.data_objects.slopes import Slopes
    from specula_b200.data_objects.pixels import Pixels
    from specula_b200.data_objects.electric_field import ElectricField
    from specula_b200.processing_objects.data_store import DataStore
    dev = torch.device('cuda', device_idx) if device_idx >= 0 else torch.device('cpu')
    ds = DataStore(str(tmp_path), data_format=fmt, flush_steps=flush_steps, target_device_idx=device_idx)
    modes = BaseValue(value=torch.zeros(3, device=dev), target_device_idx=device_idx)
    sl = Slopes(length=4, target_device_idx=device_idx)
    px = Pixels(5, 6, target_device_idx=device_idx)
    ef = ElectricField(4, 4, 0.1, target_device_idx=device_idx)
    for name, obj in (('modes', modes), ('slopes', sl), ('pixels', px), ('ef', ef)):
        ds.inputs[name] = InputValue(type=type(obj))
        ds.inputs[name].set(obj)
    ds.setParams({'main': {'total_time': 1.0}})
    ds.setReplayParams({'data_source': {}})
    ds.setup()
    rng = np.random.default_rng(0)
    want = {k: [] for k in ('modes', 'slopes', 'pixels', 'ef')}
    times = []
    for k in range(steps):
        t = (k + 1) * 1_000_000
        modes.value = torch.as_tensor(rng.standard_normal(3).astype(np.float32), device=dev)
        sl.slopes.copy_(torch.as_tensor(rng.standard_normal(4).astype(np.float32)))
        px.pixels.copy_(torch.as_tensor(rng.standard_normal((5, 6)).astype(np.float32)))
        ef.A.copy_(torch.as_tensor(rng.random((4, 4)).astype(np.float32)))
        ef.phaseInNm.copy_(torch.as_tensor(rng.standard_normal((4, 4)).astype(np.float32)))
        for o in (modes, sl, px, ef):
            o.generation_time = t
        want['modes'].append(modes.value.cpu().numpy().copy())      # copies: CPU tensors share memory
        want['slopes'].append(sl.slopes.cpu().numpy().copy())
        want['pixels'].append(px.pixels.cpu().numpy().copy())
        want['ef'].append(np.stack((ef.A.cpu().numpy(), ef.phaseInNm.cpu().numpy())))
        times.append(t)
        ds.check_ready(t)
        ds.trigger()
        ds.post_trigger()
    ds.finalize()
    return ds, {k: np.array(v) for k, v in want.items()}, np.array(times, dtype=np.float32)


@pytest.mark.parametrize('fmt', ['fits', 'pickle'])
def test_store_writes_reference_layout(tmp_path, fmt):
    ds, want, times = run_store(tmp_path, fmt, -1)
    assert os.path.dirname(ds.tn_dir) == str(tmp_path)
    assert os.path.exists(os.path.join(ds.tn_dir, 'params.yml'))
    assert os.path.exists(os.path.join(ds.tn_dir, 'replay_params.yml'))
    for name, arr in want.items():
        if fmt == 'fits':
            path = os.path.join(ds.tn_dir, name + '.fits')
            (h0, d0), (h1, d1) = fits_min.read_hdus(path)
            assert np.array_equal(d0, arr) and np.array_equal(d1, times)
        else:
            with open(os.path.join(ds.tn_dir, name + '.pickle'), 'rb') as f:
                d = pickle.load(f)
            assert np.array_equal(d['data'], arr) and np.array_equal(d['times'], times)


def test_unknown_format_and_type(tmp_path):
    from specula_b200.processing_objects.data_store import DataStore
    with pytest.raises(TypeError):
        DataStore(str(tmp_path), data_format='hdf5', target_device_idx=-1)
    with pytest.raises(TypeError):
        DataStore._value_of(object())
