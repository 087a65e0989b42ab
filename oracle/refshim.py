"""Import shim for running the reference materialite package in this container
(test infrastructure: used only to generate golden fixtures and to pin the oracle).

The reference imports pyvista, h5py, matplotlib and cupy at module level for plotting,
file import and its GPU process models; none of them is on the SmallStrainFFT path.
Empty placeholder modules are registered for them before import, which changes no
arithmetic.  The reference is read from ``MATERIALITE_REFERENCE`` (default
``/root/reference``) and is never needed on a machine that only runs the GPU tests.
"""

import os
import sys
import types

_STUBS = ["pyvista", "h5py", "matplotlib", "matplotlib.pyplot", "matplotlib.colors",
          "cupy", "cupyx", "cupyx.scipy", "cupyx.scipy.ndimage", "mpl_toolkits",
          "mpl_toolkits.mplot3d"]


def reference_root():
    return os.environ.get("MATERIALITE_REFERENCE", "/root/reference")


def available():
    return os.path.isfile(os.path.join(reference_root(), "materialite", "__init__.py"))


def import_reference():
    """Return the reference ``materialite`` module (raises ImportError if absent)."""
    if not available():
        raise ImportError("reference materialite checkout not found")
    for name in _STUBS:
        sys.modules.setdefault(name, types.ModuleType(name))
    root = reference_root()
    if root not in sys.path:
        sys.path.insert(0, root)
    import materialite  # noqa: E402
    return materialite
