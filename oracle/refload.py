"""Loads the reference's Python package on top of the oracle -- TEST INFRASTRUCTURE ONLY.

PyEulerALE's class ``SpatialDiscretization`` (``src/py_euler_ale/core.py``) imports its native
module as ``from .euler_ale import spatial_discretization as disc`` (``core.py:17``). Here the
package ``py_euler_ale`` is assembled from the reference's own, unmodified ``__init__.py`` and
``core.py`` with ``euler_ale.spatial_discretization`` bound to the f2py-compatible oracle facade
of ``oracle/shim.py``. It only works where the reference sources are present
(PYEULERALE_REFERENCE names the checkout); its results are committed as fixtures under
``tests/golden/``.
"""

from __future__ import annotations

import importlib.util
import os
import sys
import types
from pathlib import Path

from . import shim

# A checkout of the reference sources, named by PYEULERALE_REFERENCE (no default: the tests that
# need the sources skip without it).
DEFAULT_REFERENCE = (Path(os.environ["PYEULERALE_REFERENCE"])
                     if os.environ.get("PYEULERALE_REFERENCE") else None)


def reference_available(root: Path | None = DEFAULT_REFERENCE) -> bool:
    return root is not None and (root / "src" / "py_euler_ale" / "core.py").is_file()


def load_reference_package(root: Path | None = DEFAULT_REFERENCE) -> types.ModuleType:
    """Returns the reference package ``py_euler_ale`` running on the C++ oracle."""
    if "py_euler_ale" in sys.modules and getattr(sys.modules["py_euler_ale"], "_on_oracle", False):
        return sys.modules["py_euler_ale"]
    if root is None:
        raise RuntimeError("set PYEULERALE_REFERENCE to a checkout of the reference sources")
    pkg_dir = root / "src" / "py_euler_ale"
    native = types.ModuleType("py_euler_ale.euler_ale")
    native.spatial_discretization = shim.SpatialDiscretizationModule()
    sys.modules["py_euler_ale.euler_ale"] = native
    spec = importlib.util.spec_from_file_location(
        "py_euler_ale", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    pkg = importlib.util.module_from_spec(spec)
    pkg.euler_ale = native
    pkg._on_oracle = True
    sys.modules["py_euler_ale"] = pkg
    spec.loader.exec_module(pkg)
    return pkg
