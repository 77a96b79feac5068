"""Typed input slots of processing objects (mirrors specula/connections.py:2-80)."""


class InputValue:
    def __init__(self, type, optional=False):
        self.wrapped_type = type
        self.wrapped_value = None
        self.cloned_value = None
        self.optional = optional

    def get_time(self):
        if self.wrapped_value is not None:
            return self.wrapped_value.generation_time

    def get(self, target_device_idx):
        if self.wrapped_value is None:
            return None
        if self.wrapped_value.target_device_idx == target_device_idx:
            return self.wrapped_value
        if self.cloned_value is None:
            self.cloned_value = self.wrapped_value.copyTo(target_device_idx)
        else:
            self.wrapped_value.transferDataTo(self.cloned_value)
        return self.cloned_value

    def set(self, value):
        if not isinstance(value, self.wrapped_type):
            raise ValueError(f'Value must be of type {self.wrapped_type} instead of {type(value)}')
        self.wrapped_value = value

    def type(self):
        return self.wrapped_type


class InputList:
    def __init__(self, type, optional=False):
        self.wrapped_type = type
        self.wrapped_list = None
        self.cloned_list = []
        self.optional = optional

    def get_time(self):
        if self.wrapped_list is None:
            return []
        return [x.generation_time for x in self.wrapped_list]

    def get(self, target_device_idx):
        if self.wrapped_list is None:
            return None
        if not self.cloned_list:
            for w in self.wrapped_list:
                self.cloned_list.append(w if w.target_device_idx == target_device_idx else w.copyTo(target_device_idx))
        else:
            for i, (w, c) in enumerate(zip(self.wrapped_list, self.cloned_list)):
                if w.target_device_idx == target_device_idx:
                    self.cloned_list[i] = w
                else:
                    w.transferDataTo(c)
        return self.cloned_list

    def set(self, new_list):
        for v in new_list:
            if not isinstance(v, self.wrapped_type):
                raise ValueError(f'List element must be of type {self.wrapped_type}')
        self.wrapped_list = new_list
        self.cloned_list = []

    def type(self):
        return self.wrapped_type
