"""No-op pyplot stand-in: plotting is out of scope."""


def __getattr__(name):
    def _noop(*args, **kwargs):
        return None
    return _noop
