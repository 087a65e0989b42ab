"""Readers of microstructure files for the SmallStrainFFT path.

``import_evpfft`` reads the EVP-FFT input format that ``Material.export_to_evpfft``
writes (materialite/importers.py:153-200): "e1 e2 e3 x y z grain phase" per point with
1-based indices, in any point order.
"""

import numpy as np
import pandas as pd

from .material import Material
from .tensor import Orientation


def import_evpfft(file, spacing=(1, 1, 1), origin=(0, 0, 0), grain_label="grain",
                  phase_label="phase", orientation_label="orientation",
                  euler_angles_to_radians=True):
    """A Material from an EVP-FFT file; the angles are read as degrees when
    ``euler_angles_to_radians`` (the reference's name), else as radians."""
    cols = ["e1", "e2", "e3", "x_id", "y_id", "z_id", grain_label, phase_label]
    df = pd.read_csv(file, header=None, sep=r"\s+", names=cols)
    df = df.sort_values(by=["x_id", "y_id", "z_id"]).reset_index(drop=True)
    dims = df[["x_id", "y_id", "z_id"]].max().to_numpy().astype(int)
    if len(df) != int(np.prod(dims)):
        raise ValueError("EVP-FFT file does not hold one line per point of its grid")
    angles = df[["e1", "e2", "e3"]].to_numpy(dtype=np.float64)
    orientations = Orientation.from_euler_angles(angles, in_degrees=euler_angles_to_radians)
    if orientations.rotation_matrix.ndim == 2:
        orientations = Orientation(orientations.rotation_matrix[None], "p")
    material = Material(dimensions=dims, spacing=spacing, origin=origin)
    return material.create_fields({grain_label: df[grain_label].to_numpy(),
                                   phase_label: df[phase_label].to_numpy(),
                                   orientation_label: orientations})
