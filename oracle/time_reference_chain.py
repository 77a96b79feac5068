"""Time the reference's own CPU chain on the ELT bench workload, object by
object, next to the oracle port on the same host threads (test
infrastructure: it checks that the port the bench times as the reference arm
costs what the reference costs).

    SPECULA_REF=<SPECULA checkout> python oracle/time_reference_chain.py [steps]

The reference is imported on CPU with the harness-only stand-ins for
astropy.io.fits and matplotlib (tests/golden/_refstubs).  Nothing else in the
repository runs this script.
"""
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get('SPECULA_REF')
if not REF:
    sys.exit('time_reference_chain.py: set SPECULA_REF to the root of a SPECULA source tree')
sys.path.insert(0, os.path.join(ROOT, 'tests', 'golden', '_refstubs'))
sys.path.insert(0, REF)
sys.path.insert(0, ROOT)
import specula
specula.init(-1, precision=1)
from specula.processing_objects.sh import SH
from specula.processing_objects.sh_slopec import ShSlopec
from specula.processing_objects.ccd import CCD
from specula.processing_objects.integrator import Integrator
from specula.processing_objects.dm import DM
from specula.processing_objects.modalrec import Modalrec
from specula.processing_objects.atmo_evolution import AtmoEvolution
from specula.processing_objects.atmo_propagation import AtmoPropagation
from specula.data_objects.subap_data import SubapData
from specula.data_objects.ifunc import IFunc
from specula.data_objects.recmat import Recmat
from specula.data_objects.source import Source
from specula.data_objects.pupilstop import Pupilstop
from specula.data_objects.simul_params import SimulParams
from specula.base_value import BaseValue
from specula.loop_control import LoopControl
from specula_b200.scao import elt_config, valid_subaps, RAD2ASEC
from specula_b200.lib.make_mask import make_mask

c = elt_config()
sp = SimulParams(pixel_pupil=c.pixel_pupil, pixel_pitch=c.pitch, time_step=c.time_step)
pupil = make_mask(c.pixel_pupil, c.obsratio, 1.0)
nv = int(pupil.sum())
d_sub = c.diameter_m / c.n_lenses
lamd = c.wavelength_nm * 1e-9 / d_sub * RAD2ASEC
pxs = c.pxscale_over_lamd * lamd
n_valid_est = max(1, int(round(pupil.sum() / (c.pixel_pupil / c.n_lenses) ** 2)))
S0 = c.photons_per_subap * n_valid_est / (pupil.sum() * c.pitch ** 2 * c.time_step)
see = BaseValue(value=c.seeing); ws = BaseValue(value=np.array(c.wind_speed)); wd = BaseValue(value=np.array(c.wind_direction))
import tempfile
atmo = AtmoEvolution(sp, L0=c.L0, heights=c.heights, Cn2=c.cn2, data_dir=tempfile.mkdtemp(), pixel_phasescreens=c.pixel_phasescreens, seed=c.screen_seed, target_device_idx=-1)
atmo.inputs['seeing'].set(see); atmo.inputs['wind_speed'].set(ws); atmo.inputs['wind_direction'].set(wd)
pup = Pupilstop(sp, obs_diam=c.obsratio, target_device_idx=-1)
rng = np.random.default_rng(c.seed)
IF = rng.standard_normal((c.n_modes, nv), dtype=np.float32) * 10
dm = DM(sp, 0, ifunc=IFunc(ifunc=IF, mask=pupil, target_device_idx=-1), target_device_idx=-1)
src = Source([0.0, 0.0], 8, c.wavelength_nm)
prop = AtmoPropagation(sp, {'on_axis_source': src}, target_device_idx=-1)
prop.inputs['atmo_layer_list'].set(atmo.layer_list)
prop.inputs['common_layer_list'].set([pup, dm.outputs['out_layer']])
sh = SH(wavelengthInNm=c.wavelength_nm, subap_wanted_fov=c.subap_npx * pxs, sensor_pxscale=pxs, subap_on_diameter=c.n_lenses, subap_npx=c.subap_npx, fov_ovs_coeff=c.fov_ovs_coeff, target_device_idx=-1)
sh.inputs['in_ef'].set(prop.outputs['out_on_axis_source_ef'])
side = c.n_lenses * c.subap_npx
ccd = CCD(sp, size=[side, side], dt=c.time_step, bandw=1.0, photon_noise=True, readout_noise=True, readout_level=3.0, quantum_eff=1.0, target_device_idx=-1)
ccd.inputs['in_i'].set(sh.outputs['out_i'])
idxs, dmap = valid_subaps(pupil, c.n_lenses, c.subap_npx, c.subap_threshold)
sd = SubapData(idxs=idxs, display_map=dmap, nx=c.n_lenses, ny=c.n_lenses, target_device_idx=-1)
sl = ShSlopec(sd, target_device_idx=-1)
sl.inputs['in_pixels'].set(ccd.outputs['out_pixels'])
R = rng.standard_normal((c.n_modes, 2 * len(idxs)), dtype=np.float32) / math.sqrt(2 * len(idxs))
rec = Modalrec(recmat=Recmat(R, target_device_idx=-1), target_device_idx=-1)
rec.inputs['in_slopes'].set(sl.outputs['out_slopes'])
integ = Integrator(sp, int_gain=[c.gain] * c.n_modes, delay=c.delay, target_device_idx=-1)
integ.inputs['delta_comm'].set(rec.outputs['out_modes'])
dm.inputs['in_command'].set(integ.outputs['out_comm'])
objs = [atmo, prop, sh, ccd, sl, rec, integ, dm]
t0 = time.perf_counter()
for o in objs: o.setup()
print('setup s', time.perf_counter() - t0, flush=True)
per = {type(o).__name__: 0.0 for o in objs}
nsteps = int(sys.argv[1]) if len(sys.argv) > 1 else 6
tot = 0.0
for k in range(nsteps + 1):
    tt = k * 1000000
    for v in (see, ws, wd): v.generation_time = tt
    ts = time.perf_counter()
    for o in objs:
        a = time.perf_counter()
        o.check_ready(tt); o.trigger(); o.post_trigger()
        if k > 0: per[type(o).__name__] += time.perf_counter() - a
    if k > 0: tot += time.perf_counter() - ts
print(f'reference: {tot / nsteps * 1e3:.1f} ms/step', {k: round(v / nsteps * 1e3, 2) for k, v in per.items()})

# the oracle port on the same system (the bench's reference arm)
from oracle.loop import OracleScaoLoop  # noqa: E402
port = OracleScaoLoop(c, IF, R, idxs, pupil, S0)
port.step()
t0 = time.perf_counter()
for _ in range(nsteps):
    port.step()
print(f'port: {(time.perf_counter() - t0) / nsteps * 1e3:.1f} ms/step')
try:
    from threadpoolctl import threadpool_info
    print('BLAS threads', max(i.get('num_threads', 1) for i in threadpool_info() if i.get('user_api') == 'blas'))
except Exception:
    pass
