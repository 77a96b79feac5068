"""sb_propagate through AtmoPropagation on the GPU against the reference's
fields for interpolated layers (LGS cone effect, off-axis NGS and LGS,
shifted / rotated / magnified layers), within 1e-6; the zero-amplitude
pixels of an interpolated layer get its lit mean phase in place, as in the
reference."""
import numpy as np
import pytest

from tests.cases import rel_max_err
from tests.test_prop_interp import build, prop_golden  # noqa: F401

pytestmark = pytest.mark.gpu


def test_interpolated_propagation_matches_reference(cuda, prop_golden):  # noqa: F811
    g = prop_golden
    prop, layers, pup, sources = build(0, g)
    for lay in layers:
        lay.generation_time = 1
    pup.generation_time = 1
    prop.setup()
    assert prop._interpolated
    for t in (1, 2):
        for lay in layers:
            lay.generation_time = t
        pup.generation_time = t
        prop.check_ready(t)
        prop.trigger()
        prop.post_trigger()
        for name in sources:
            ef = prop.outputs['out_%s_ef' % name]
            assert rel_max_err(ef.A.cpu().numpy(), g['prop/%s/A' % name]) <= 1e-6, (t, name)
            assert rel_max_err(ef.phaseInNm.cpu().numpy(), g['prop/%s/phase' % name]) <= 1e-6, (t, name)
    assert rel_max_err(layers[3].phaseInNm.cpu().numpy(), g['prop/layer3/phase_after']) <= 1e-6
