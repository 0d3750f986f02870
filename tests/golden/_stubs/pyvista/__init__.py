"""Test-only stand-in for pyvista (absent here): names the reference imports, no rendering."""


class PolyData:  # noqa: D101
    @classmethod
    def from_irregular_faces(cls, *a, **k):
        raise RuntimeError("pyvista is not available")


class Plotter:  # noqa: D101
    def __init__(self, *a, **k):
        raise RuntimeError("pyvista is not available")


class CellArray:  # noqa: D101
    @classmethod
    def from_regular_cells(cls, *a, **k):
        raise RuntimeError("pyvista is not available")


class _Themes:
    class DocumentProTheme:  # noqa: D106
        pass


themes = _Themes()
