"""Typed input slots of processing objects.

Interface as the reference's ``InputValue`` / ``InputList``
(specula/connections.py): a slot is built with the accepted data-object type
and an ``optional`` flag; ``set`` connects a producer's output (wrong types
raise ``ValueError``), ``get(device_idx)`` returns what the consumer reads on
its device and ``get_time()`` the producer's generation time(s).

A value that already lives on the consumer's device is handed over as is.
A value on another device is mirrored: the first ``get`` makes a device copy
(``copyTo``), later calls refresh that copy in place (``transferDataTo``), so
the consumer keeps reading fixed addresses, which captured CUDA graphs need.
Mirrors are kept per consumer device and dropped when the slot is re-connected.
"""


class _Slot:
    """What both slot kinds share: the accepted type and the mirror cache."""

    def __init__(self, type, optional=False):
        self._accepts = type
        self.optional = optional
        self._mirrors = {}          # (consumer device, position) -> device copy

    def type(self):
        return self._accepts

    def _require(self, value, what):
        if not isinstance(value, self._accepts):
            raise ValueError(f'{what}: expected {self._accepts.__name__}, got {type(value).__name__}')

    def _on_device(self, value, device_idx, pos=0):
        if value.target_device_idx == device_idx:
            return value
        key = (device_idx, pos)
        copy = self._mirrors.get(key)
        if copy is None:
            copy = self._mirrors[key] = value.copyTo(device_idx)
        else:
            value.transferDataTo(copy)
        return copy


class InputValue(_Slot):
    """One connected data object."""

    def __init__(self, type, optional=False):
        super().__init__(type, optional)
        self._source = None

    def set(self, value):
        self._require(value, 'InputValue.set')
        self._source = value
        self._mirrors = {}

    def get(self, target_device_idx):
        if self._source is None:
            return None
        return self._on_device(self._source, target_device_idx)

    def get_time(self):
        return None if self._source is None else self._source.generation_time


class InputList(_Slot):
    """A list of connected data objects of one type."""

    def __init__(self, type, optional=False):
        super().__init__(type, optional)
        self._sources = None

    def set(self, new_list):
        items = list(new_list)
        for k, v in enumerate(items):
            self._require(v, f'InputList.set (element {k})')
        self._sources = new_list
        self._mirrors = {}

    def get(self, target_device_idx):
        if self._sources is None:
            return None
        return [self._on_device(v, target_device_idx, k) for k, v in enumerate(self._sources)]

    def get_time(self):
        return [] if self._sources is None else [v.generation_time for v in self._sources]
