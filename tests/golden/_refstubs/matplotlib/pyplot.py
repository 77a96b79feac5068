"""Harness-only stand-in for matplotlib.pyplot: every attribute is a no-op."""


def __getattr__(name):
    def _noop(*a, **k):
        return None
    return _noop
