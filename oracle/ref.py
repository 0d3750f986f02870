"""Load the reference's own compiled extension (oracle/_ref) and, where the reference
tree is present, its Python package -- ORACLE / TEST INFRASTRUCTURE ONLY.

``load_cvl()`` imports ``oracle/_ref/cvl*.so`` (built by oracle/build_ref.sh) as the
module ``pyvl.cvl``; it travels to the GPU host prebuilt.  ``load_pyvl()`` additionally
imports the reference's Python package from its source tree (only available where
that tree is mounted, i.e. when generating golden vectors), with the test-only
stand-ins in tests/golden/_stubs for the plotting/IO modules the hot path never uses.
"""

from __future__ import annotations

import importlib.machinery
import importlib.util
import os
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_SO = HERE / "_ref" / ("cvl" + sysconfig.get_config_var("EXT_SUFFIX"))
STUBS = HERE.parent / "tests" / "golden" / "_stubs"


def available() -> bool:
    return REF_SO.exists()


def load_cvl():
    """Return the reference's compiled ``cvl`` module (registered as ``pyvl.cvl``)."""
    if "pyvl.cvl" in sys.modules:
        return sys.modules["pyvl.cvl"]
    if not REF_SO.exists():
        raise FileNotFoundError(f"{REF_SO} is missing; run oracle/build_ref.sh")
    loader = importlib.machinery.ExtensionFileLoader("pyvl.cvl", str(REF_SO))
    spec = importlib.util.spec_from_file_location("pyvl.cvl", str(REF_SO), loader=loader)
    mod = importlib.util.module_from_spec(spec)
    loader.exec_module(mod)
    sys.modules["pyvl.cvl"] = mod
    return mod


def reference_root(given: str | Path | None = None) -> Path:
    """The reference checkout: ``given``, else $PYVL_REFERENCE_ROOT."""
    if given is None:
        given = os.environ.get("PYVL_REFERENCE_ROOT")
    if not given:
        raise FileNotFoundError("the reference checkout is not known: pass its path or set PYVL_REFERENCE_ROOT")
    return Path(given)


def load_pyvl(reference_root_dir: str | Path | None = None):
    """Import the reference Python package on top of the compiled extension."""
    root = reference_root(reference_root_dir) / "python"
    if not (root / "pyvl" / "__init__.py").exists():
        raise FileNotFoundError(f"reference python package not found under {root}")
    load_cvl()
    for p in (str(STUBS), str(root)):
        if p not in sys.path:
            sys.path.insert(0, p)
    import pyvl  # noqa: PLC0415

    return pyvl
