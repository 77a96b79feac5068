"""Generic value container (mirrors specula/base_value.py:4-56)."""
from specula_b200.base_data_obj import BaseDataObj


class BaseValue(BaseDataObj):
    def __init__(self, description='', value=None, target_device_idx=None, precision=None):
        super().__init__(target_device_idx=target_device_idx, precision=precision)
        self._description = description
        self._value = value

    def set_value(self, val):
        self._value = val

    @property
    def value(self):
        return self._value

    @value.setter
    def value(self, val):
        self._value = val

    @property
    def ptr_value(self):
        return self._value

    @ptr_value.setter
    def ptr_value(self, val):
        self._value = val
