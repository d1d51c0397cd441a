"""No-op nibabel stand-in: NIfTI output is out of scope."""


def __getattr__(name):
    def _noop(*args, **kwargs):
        return None
    return _noop
