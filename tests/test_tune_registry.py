"""Host side of the tile-shape tuning registry (no GPU): variant counts and
names, registration, lookup and removal per (family, shape key)."""
import pytest

from specula_b200 import _lib


def test_families_and_names():
    lib = _lib.load()
    assert lib.sb_tune_variants(_lib.SB_TUNE_DM_BATCHED) == 12
    assert lib.sb_tune_variants(_lib.SB_TUNE_SH_FP32) == 6
    assert b'by TMA' in lib.sb_tune_variant_name(_lib.SB_TUNE_SH_FP32, 0)
    assert b'TMA' not in lib.sb_tune_variant_name(_lib.SB_TUNE_SH_FP32, 3)
    assert lib.sb_tune_variants(_lib.SB_TUNE_MODALREC_BATCHED) == 3
    assert b'rows per CTA' in lib.sb_tune_variant_name(_lib.SB_TUNE_MODALREC_BATCHED, 2)
    assert lib.sb_tune_variants(99) == 0
    assert b'per pass' in lib.sb_tune_variant_name(_lib.SB_TUNE_DM_BATCHED, 3)
    assert lib.sb_tune_variant_name(_lib.SB_TUNE_SH_FP32, 7) == b''


def test_set_get_remove():
    lib = _lib.load()
    fam = _lib.SB_TUNE_DM_BATCHED
    k1, k2 = lib.sb_tune_key(500, 275000, 7), lib.sb_tune_key(500, 275000, 8)
    assert k1 != k2
    assert lib.sb_tune_get(fam, k1) == 0
    _lib.call('sb_tune_set', fam, k1, 3)
    assert lib.sb_tune_get(fam, k1) == 3
    assert lib.sb_tune_get(fam, k2) == 0
    assert lib.sb_tune_get(_lib.SB_TUNE_SH_FP32, k1) == 0
    _lib.call('sb_tune_set', fam, k1, -1)
    assert lib.sb_tune_get(fam, k1) == 0
    with pytest.raises(RuntimeError, match='EINVAL'):
        _lib.call('sb_tune_set', fam, k1, 12)
    with pytest.raises(RuntimeError, match='EINVAL'):
        _lib.call('sb_tune_set', 42, k1, 0)
    assert lib.sb_tune_get(42, k1) == -1
