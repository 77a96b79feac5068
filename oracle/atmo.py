"""Oracle: turbulence screens, their per-step shift and the on-axis
propagation (test infrastructure only).

Restates specula/lib/calc_phasescreen.py:6-105 with
specula/lib/calc_spatialfrequency.py, the screen preparation of
specula/processing_objects/atmo_evolution.py:142-252, its per-step update
:254-300, and the on-axis (no interpolation) branch of
specula/processing_objects/atmo_propagation.py:105-144 with
specula/data_objects/electric_field.py:35-43,77-82.

The fractional-degree wind rotation calls scipy.ndimage.rotate exactly as
the reference CPU path does (atmo_evolution.py:293 via base_time_obj.py:40-54).
"""
import numpy as np
from scipy.ndimage import rotate as _scipy_rotate


def spatial_frequency(dim, dtype=np.float64):
    """row^2 + col^2 with the null frequency at [dim/2-1, dim/2-1]
    (calc_spatialfrequency.py: the four rotated quarters reduce to this)."""
    c = np.arange(dim, dtype=dtype) - (dim // 2 - 1)
    return (c[:, None] ** 2 + c[None, :] ** 2).astype(dtype)


def calc_phasescreen(L0, dimension, pixel_pitch, seed=0, precision=0):
    """Von Karman phase screen in radians at 500 nm (calc_phasescreen.py:6-105)."""
    n = int(np.ceil(np.log2(float(dimension))))
    dimension = 2 ** n
    dtype = np.float32 if precision == 1 else np.float64
    cdtype = np.complex64 if precision == 1 else np.complex128
    m_dim = dimension * pixel_pitch
    h = dimension // 2
    rng = np.random.RandomState(seed)
    u1 = rng.random((h + 1, 2 * h + 1))
    v1 = rng.random((h + 1, 2 * h + 1))
    re = (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * v1)).astype(dtype)
    u2 = rng.random((h + 1, 2 * h + 1))
    v2 = rng.random((h + 1, 2 * h + 1))
    im = (np.sqrt(-2.0 * np.log(u2)) * np.cos(2.0 * np.pi * v2)).astype(dtype)
    ps = np.zeros((dimension, dimension), dtype=cdtype)
    ps[h:2 * h, 0:2 * h] = re[1:h + 1, 1:2 * h + 1] + 1j * im[1:h + 1, 1:2 * h + 1]
    ps[0:h - 1, 0:2 * h] = np.rot90(re, 2)[1:h, 1:2 * h + 1] - 1j * np.rot90(im, 2)[1:h, 1:2 * h + 1]
    ps[h, 0:h] = re[0, 1:h + 1] + 1j * im[0, 1:h + 1]
    ps[h, h:2 * h] = np.flipud(re)[0, 0:h] - 1j * np.flipud(im)[0, 0:h]
    ps[2 * h - 1, :] = 0
    ps[:, 2 * h - 1] = 0
    f2 = spatial_frequency(dimension, dtype) / m_dim ** 2
    ps *= (f2 + 1. / L0 ** 2) ** (-11. / 12.)
    ps *= np.sqrt(0.033 / 2. / m_dim ** 2) * (2 * np.pi) ** (2. / 3.) * np.sqrt(0.06) * (1 / pixel_pitch) ** (5. / 6.)
    ps = np.roll(ps, (-h + 1, -h + 1), axis=(0, 1))
    ps = np.fft.ifft2(ps, norm='forward')
    ps = np.roll(ps, (h - 1, h - 1), axis=(0, 1))
    return np.real(ps)


def prepare_strips(square_screens, n_layers, pixel_layer, Cn2, wavelength_nm=500.0, precision=1):
    """Cut square screens into per-layer strips (pixel_layer x square_dim),
    scale by sqrt(Cn2), de-mean, convert to nm and flip odd layers
    (atmo_evolution.py:164-226, single-L0 branch)."""
    dtype = np.float32 if precision == 1 else np.float64
    dim = square_screens[0].shape[0]
    per_square = dim // pixel_layer
    strips = []
    sq = -1
    ps_index = 0
    for i in range(n_layers):
        if i % per_square == 0:
            sq += 1
            ps_index = 0
        s = np.array(square_screens[sq][pixel_layer * ps_index: pixel_layer * (ps_index + 1), :], dtype=dtype)
        s *= np.sqrt(np.asarray(Cn2, dtype=dtype)[i])
        s -= np.mean(s)
        s *= wavelength_nm / (2 * np.pi)
        s = np.array(s, dtype=dtype)
        if i % 2 != 0:
            s = np.flip(s, axis=1)
        ps_index += 1
        strips.append(s)
    return strips


class AtmoEvolutionOracle:
    """Per-step layer update (atmo_evolution.py:254-300)."""

    def __init__(self, strips, pixel_layer, pixel_pitch, wavelength_nm=500.0, zenith_deg=0.0, precision=1):
        self.dtype = np.float32 if precision == 1 else np.float64
        self.strips = strips
        self.L = int(pixel_layer)
        self.pitch = pixel_pitch
        self.lam = wavelength_nm
        # a numpy scalar of the object dtype, which makes r0 and the screen
        # scale follow that dtype (atmo_evolution.py:57-58)
        self.airmass = 1.0 / np.cos(np.radians(zenith_deg), dtype=self.dtype)
        self.last_position = np.zeros(len(strips), dtype=self.dtype)
        self.sizes = np.array([s.shape[1] for s in strips])
        self.last_t = 0

    def step(self, t_ns, seeing, wind_speed, wind_direction):
        """``t_ns``: loop time in integer nanoseconds (base_time_obj.py:16)."""
        delta_time = float(t_ns - self.last_t) / 1e9
        r0 = 0.9759 * 0.5 / (seeing * 4.848) * self.airmass ** (-3. / 5.)
        r0l = r0 * (self.lam / 500.0) ** (6. / 5.)
        scale = (self.pitch / r0l) ** (5. / 6.)
        ws = np.asarray(wind_speed, dtype=float)
        wd = np.asarray(wind_direction, dtype=float)
        new = self.last_position + ws * delta_time / self.pitch
        _, wdi = np.modf(wd / 90.0)
        wdf_full, _ = np.modf(wd)
        new = np.where(new + self.L >= self.sizes, 0, new)
        quo = np.floor(new).astype(np.int64)
        rem = (new - quo).astype(self.dtype)
        layers = []
        for k, p in enumerate(self.strips):
            pos = int(quo[k])
            lp = (1.0 - rem[k]) * p[0:self.L, pos:pos + self.L] + rem[k] * p[0:self.L, pos + 1:pos + 1 + self.L]
            lp = np.rot90(lp, wdi[k])
            if not wdf_full[k] == 0:
                lp = _scipy_rotate(lp, wdf_full[k], reshape=False, order=1)
            layers.append(lp * scale)
        self.last_position = new
        self.last_t = t_ns
        return layers


def propagate_on_axis(layers_A, layers_phase, pupil_size, dtype=np.float32):
    """Reset the field then multiply amplitudes and add phases of every layer's
    centred crop (atmo_propagation.py:105-125, electric_field.py:35-43,77-82)."""
    A = np.ones((pupil_size, pupil_size), dtype=dtype)
    P = np.zeros((pupil_size, pupil_size), dtype=dtype)
    for a, p in zip(layers_A, layers_phase):
        t0 = (p.shape[0] - pupil_size) // 2
        t1 = (p.shape[1] - pupil_size) // 2
        A *= a[t0:t0 + pupil_size, t1:t1 + pupil_size]
        P += np.asarray(p[t0:t0 + pupil_size, t1:t1 + pupil_size])
    return A, P
