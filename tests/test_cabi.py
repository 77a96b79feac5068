"""The C-ABI library loads without a GPU, exports every function declared in
include/specula_b200.h, and rejects bad arguments before touching the device."""
import ctypes as C
import os
import re

import pytest

from specula_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'include', 'specula_b200.h')


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
    return sorted(set(re.findall(r'\b(sb_\w+)\s*\(', src)))


@pytest.fixture(scope='module')
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        from specula_b200.csrc import build
        build.build()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n


def test_binding_table_matches_header():
    assert sorted(_lib.SIGNATURES) == declared_functions()


def test_version_and_error_string(lib):
    assert lib.sb_version() >= 100
    assert isinstance(lib.sb_last_error(), bytes)


def test_argument_validation_without_device(lib):
    plan = _lib.ShPlan()
    rc = lib.sb_sh_forward(C.byref(plan), None, None, None, 0, C.c_float(1.0), None, None, 0, None)
    assert rc == -1
    assert b'null' in lib.sb_last_error()
    rc = lib.sb_modalrec(None, 3, 4, 4, None, None, None)
    assert rc == -1
    assert lib.sb_atmo_evolve(None, 1, 16, None, None) == -1
    layers = (_lib.AtmoLayer * 17)()
    pos = C.c_double(0)
    assert lib.sb_atmo_evolve(layers, 17, 16, C.byref(pos), None) == -2


def test_fused_atmosphere_and_batched_mirror_validation_without_device(lib):
    """sb_atmo_propagate_batched and sb_dm_project_batched reject bad
    arguments (status and message) before any device work."""
    layers = (_lib.AtmoLayer * 4)()
    inputs = (_lib.AtmoLayerInputs * 4)()
    consts = _lib.AtmoInputs()
    consts.pixel_pitch = 0.05
    consts.delta_time = 0.001
    buf = C.c_void_p(16)                     # never dereferenced: validation fails first
    f = _lib.SIGNATURES['sb_atmo_propagate_batched']
    assert len(f[1]) == 17
    # no layers per realisation
    rc = lib.sb_atmo_propagate_batched(layers, inputs, 0, 4, 16, C.byref(consts), buf, 1 << 20, None, None, None,
                                       buf, 256, buf, buf, 256, None)
    assert rc == -1 and b'sb_atmo_propagate_batched' in lib.sb_last_error()
    # mirror phase stride below one pupil
    rc = lib.sb_atmo_propagate_batched(layers, inputs, 2, 2, 16, C.byref(consts), buf, 1 << 20, None, None, None,
                                       buf, 255, buf, buf, 256, None)
    assert rc == -1
    # work area too small for the per-layer parameters
    rc = lib.sb_atmo_propagate_batched(layers, inputs, 2, 2, 16, C.byref(consts), buf, 8, None, None, None,
                                       buf, 256, buf, buf, 256, None)
    assert rc == -4 and b'work needs' in lib.sb_last_error()
    # batched mirror: too many modes, misaligned rows
    rc = lib.sb_dm_project_batched(buf, 2000, 100, 100, buf, 2000, 4, C.c_float(-1.0), buf, buf, 1000, None)
    assert rc == -2 and b'at most' in lib.sb_last_error()
    rc = lib.sb_dm_project_batched(buf, 10, 100, 101, buf, 10, 4, C.c_float(-1.0), buf, buf, 1000, None)
    assert rc == -1 and b'16-byte' in lib.sb_last_error()


STRUCTS = {'sb_sh_plan': _lib.ShPlan, 'sb_ccd_params': _lib.CcdParams, 'sb_slopec_plan': _lib.SlopecPlan,
           'sb_iir_plan': _lib.IirPlan, 'sb_atmo_layer': _lib.AtmoLayer, 'sb_prop_layer': _lib.PropLayer,
           'sb_atmo_inputs': _lib.AtmoInputs, 'sb_atmo_layer_inputs': _lib.AtmoLayerInputs,
           'sb_sh_lgs_tables': _lib.ShLgsTables, 'sb_prop_sampling': _lib.PropSampling,
           'sb_mc_group': _lib.McGroup}


def test_struct_layouts_match_header(tmp_path):
    """Compile a probe against the header with gcc and compare every struct's
    size and field offsets with the ctypes mirrors."""
    import shutil
    import subprocess
    if shutil.which('gcc') is None:
        pytest.skip('gcc not available')
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "specula_b200.h"', 'int main(void){']
    for cname, py in STRUCTS.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append('return 0;}')
    src = tmp_path / 'probe.c'
    src.write_text('\n'.join(lines))
    exe = tmp_path / 'probe'
    subprocess.run(['gcc', '-I', os.path.dirname(HEADER), str(src), '-o', str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split('\n')
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in STRUCTS.items():
        assert got[(cname, 'size')] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_static_scratch_limit_without_device(lib):
    """sb_sh_forward_static's 64 KB array holds the partial sums of grids up
    to 128 x 128 lenslets; larger grids are rejected before any device work."""
    plan = _lib.ShPlan()
    plan.np_sub, plan.cutsize, plan.subap_npx = 8, 12, 6
    plan.n_lenses = 128
    plan.field_ld = 128 * 8
    assert 0 < lib.sb_sh_scratch_bytes(C.byref(plan)) <= 64 * 1024
    plan.n_lenses = 130
    plan.field_ld = 130 * 8
    assert lib.sb_sh_scratch_bytes(C.byref(plan)) > 64 * 1024
    buf = C.c_void_p(16)                     # never dereferenced: the size check fails first
    rc = lib.sb_sh_forward_static(C.byref(plan), buf, buf, buf, 16, C.c_float(1.0), buf, None)
    assert rc == -4 and b'static array' in lib.sb_last_error()


def test_monte_carlo_step_validation_without_device(lib):
    """sb_mc_* reject an empty or oversized group list, a null handle and a
    missing workspace before any device work."""
    groups = (_lib.McGroup * 9)()
    assert lib.sb_mc_workspace_bytes(groups, 0) == 0
    assert lib.sb_mc_workspace_bytes(groups, 9) == 0 and b'groups' in lib.sb_last_error()
    groups[0].n_batch = 0
    assert lib.sb_mc_workspace_bytes(groups, 1) == 0 and b'no realisations' in lib.sb_last_error()
    assert lib.sb_mc_step(None, None) == -1
    h = C.c_void_p()
    assert lib.sb_mc_create(groups, 1, None, 0, C.byref(h), None) == -1
    lib.sb_mc_destroy(None)


def test_row_band_and_stage_validation_without_device(lib):
    """The row-band entry points and sb_mc_stage reject bad bands, null
    pointers and unknown stages before any device work."""
    plan = _lib.ShPlan()
    plan.n_lenses, plan.np_sub, plan.cutsize, plan.subap_npx, plan.field_ld = 20, 8, 14, 8, 160
    buf = C.c_void_p(16)                       # never dereferenced: validation fails first
    rc = lib.sb_sh_forward_rows(C.byref(plan), 2, 0, 4, buf, buf, buf, 16, buf, buf, 1 << 20, None)
    assert rc == -1 and b'dft_mode' in lib.sb_last_error()
    ccd = _lib.CcdParams()
    sl = _lib.SlopecPlan()
    rc = lib.sb_ccd_slopec_rows(C.byref(plan), None, 10, C.c_float(1.0), 0, 4, buf, C.byref(ccd), buf, buf,
                                C.byref(sl), buf, buf, buf, buf, None)
    assert rc == -1 and b'null' in lib.sb_last_error()
    ccd.state = buf
    sl.xw = sl.yw = sl.mw = buf
    rc = lib.sb_ccd_slopec_rows(C.byref(plan), buf, 10, C.c_float(1.0), 18, 4, buf, C.byref(ccd), buf, buf,
                                C.byref(sl), buf, buf, buf, buf, None)
    assert rc == -1 and b'lenslet rows 18..21 of 20' in lib.sb_last_error()
    assert lib.sb_slopec_cutoff(buf, buf, buf, 0, buf, None) == -1
    assert lib.sb_mc_stage(None, 0, -1, None) == -1


def test_lenslet_contraction_validation_without_device(lib):
    """sb_intmat_lenslet_ifunc and sb_intmat_contract_lenslets reject null
    pointers, unsupported lenslet sizes and a misaligned layout before any
    device work."""
    buf = C.c_void_p(256)                      # never dereferenced: validation fails first
    assert lib.sb_intmat_lenslet_ifunc(None, 10, 64, buf, 4, 8, 4, 32, buf, buf, None) == -1
    assert b'bad args' in lib.sb_last_error()
    rc = lib.sb_intmat_lenslet_ifunc(buf, 10, 64, buf, 4, 16, 4, 64, buf, buf, None)
    assert rc != 0 and b'np_sub=16' in lib.sb_last_error()
    rc = lib.sb_intmat_lenslet_ifunc(buf, 10, 64, buf, 4, 8, 4, 16, buf, buf, None)
    assert rc == -1 and b'field stride' in lib.sb_last_error()
    assert lib.sb_intmat_contract_lenslets(buf, None, 0, 8, buf, 10, C.c_float(1.0), buf, None) == -1
    rc = lib.sb_intmat_contract_lenslets(buf, None, 4, 16, buf, 10, C.c_float(1.0), buf, None)
    assert rc != 0 and b'np_sub=16' in lib.sb_last_error()
    rc = lib.sb_intmat_contract_lenslets(buf, None, 4, 8, C.c_void_p(260), 10, C.c_float(1.0), buf, None)
    assert rc == -1 and b'16-byte aligned' in lib.sb_last_error()
