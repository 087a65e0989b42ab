"""Drop-in SmallStrainFFT and constitutive models
(materialite/models/small_strain_fft/__init__.py:13-19)."""

from .elastic import Elastic
from .elastic_viscoplastic import ElasticViscoplastic
from .hardening_laws import armstrong_frederick, linear, perfect_plasticity, voce
from .isotropic_elastic_plastic import IsotropicElasticPlastic
from .load_schedule import LoadSchedule
from .multiphase import Multiphase
from .small_strain_fft import SmallStrainFFT
