"""Import shim for running the reference materialite package in this container
(test infrastructure: used only to generate golden fixtures and to pin the oracle).

The reference imports pyvista, h5py, matplotlib and cupy at module level for plotting,
file import and its GPU process models; none of them is on the SmallStrainFFT path.
Empty placeholder modules are registered for them before import, which changes no
arithmetic.  The reference checkout is named by the ``MATERIALITE_REFERENCE``
environment variable (there is no default); it is never needed on a machine that only runs
the GPU tests.
"""

import os
import sys
import types

_STUBS = ["pyvista", "h5py", "matplotlib", "matplotlib.pyplot", "matplotlib.colors",
          "cupy", "cupyx", "cupyx.scipy", "cupyx.scipy.ndimage", "mpl_toolkits",
          "mpl_toolkits.mplot3d"]


def reference_root():
    """The reference checkout named by MATERIALITE_REFERENCE, or None when unset."""
    return os.environ.get("MATERIALITE_REFERENCE") or None


def available():
    root = reference_root()
    return root is not None and os.path.isfile(os.path.join(root, "materialite", "__init__.py"))


def import_reference():
    """Return the reference ``materialite`` module (raises ImportError if absent)."""
    if not available():
        raise ImportError("reference materialite checkout not found: set MATERIALITE_REFERENCE "
                          "to the directory that contains the materialite package")
    for name in _STUBS:
        sys.modules.setdefault(name, types.ModuleType(name))
    root = reference_root()
    if root not in sys.path:
        sys.path.insert(0, root)
    import materialite  # noqa: E402
    return materialite
