"""Test-only stand-in for h5py (absent here): names the reference imports."""


class File:  # noqa: D101
    def __init__(self, *a, **k):
        raise RuntimeError("h5py is not available")


class Group:  # noqa: D101
    pass


class Datatype:  # noqa: D101
    pass
