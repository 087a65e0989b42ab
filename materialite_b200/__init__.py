"""materialite_b200: materialite's SmallStrainFFT solve on NVIDIA B200 (sm_100a).

Mirrors the reference package's names for the pieces on the SmallStrainFFT path:
``Material`` and its features, the Mandel tensor objects, ``SlipSystem``, the EVP-FFT and
JSON file formats (``import_evpfft``, ``Material.export_to_evpfft``, ``read_from_json``,
``write_to_json``) and, in
``materialite_b200.small_strain_fft``, ``SmallStrainFFT`` with its constitutive models.
"""

from .importers import import_evpfft
from .json_operations import read_from_json, write_to_json
from .material import Box, Feature, Material, Sphere, Superellipsoid
from .slip_system import SlipSystem
from .tensor import (Order2SymmetricTensor, Order2Tensor, Order4SymmetricTensor, Orientation,
                     Scalar, Vector)

__all__ = ["Box", "Feature", "Material", "Sphere", "Superellipsoid", "SlipSystem",
           "Order2SymmetricTensor", "Order2Tensor", "Order4SymmetricTensor", "Orientation",
           "Scalar", "Vector", "import_evpfft", "read_from_json", "write_to_json"]
