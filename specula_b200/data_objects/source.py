"""Point source (mirrors specula/data_objects/source.py:8-90).

``phot_density()`` needs the reference's photometric tables
(specula/lib/n_phot.py); here a source built with ``phot_density_value``
returns that value, and AtmoPropagation copies it into the field's S0."""
import numpy as np

from specula_b200 import ASEC2RAD


class Source:
    def __init__(self, polar_coordinates: list, magnitude: float, wavelengthInNm: float,
                 height: float = float('inf'), band: str = '', zeroPoint: float = 0,
                 error_coord: tuple = (0., 0.), verbose: bool = False, phot_density_value: float = None):
        self.polar_coordinates = np.array(polar_coordinates, dtype=float) + np.array(error_coord, dtype=float)
        self.magnitude = magnitude
        self.wavelengthInNm = wavelengthInNm
        self.height = height
        self.band = band
        self.zeroPoint = zeroPoint
        self.verbose = verbose
        self._phot_density_value = phot_density_value

    @property
    def r(self):
        return self.polar_coordinates[0] * ASEC2RAD

    @property
    def r_arcsec(self):
        return self.polar_coordinates[0]

    @property
    def phi(self):
        return self.polar_coordinates[1] * np.pi / 180.

    def phot_density(self):
        if self._phot_density_value is None:
            raise NotImplementedError('Source.phot_density: give phot_density_value= (photometric tables '
                                      'are not part of specula_b200)')
        return self._phot_density_value
