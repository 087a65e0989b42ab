"""Crystal elasto-viscoplasticity
(materialite/models/small_strain_fft/elastic_viscoplastic.py:20-294).

The backward-Euler update (power-law slip rates, Newton on the stress with the
consistent tangent) runs per voxel in double precision in libssfft
(csrc/constitutive.cuh).  ``latent_ratio`` is an extension with no reference
counterpart: the hardening increment of each system is weighted by
q + (1 - q) |gdot_a| / sum |gdot|; q = 1 is the reference."""

import numpy as np

from ..engine import PhaseSpec
from .hardening_laws import HARDENING_LAWS


class ElasticViscoplastic:
    def __init__(self, stiffness, slip_systems, reference_slip_rate, rate_exponent,
                 slip_resistance, hardening_function, hardening_properties, latent_ratio=1.0):
        self.stiffness = stiffness
        self._ref_modulus = float(np.asarray(stiffness.directional_modulus([1, 0, 0]).components))
        self.slip_systems = slip_systems
        self.reference_slip_rate = float(reference_slip_rate)
        self.rate_exponent = float(rate_exponent)
        self.initial_slip_resistance = float(slip_resistance)
        self.hardening_function = hardening_function
        self.hardening_properties = hardening_properties
        self.latent_ratio = float(latent_ratio)
        self.state_variables = dict()
        self.available_state_variables = ["slip_resistances", "plastic_strains",
                                          "slip_system_shear_strains"]
        n = len(slip_systems)
        from ..tensor import Order2SymmetricTensor, Scalar
        self._state_variable_info = dict(zip(self.available_state_variables,
                                             [(Scalar, n), (Order2SymmetricTensor, 0), (Scalar, n)]))

    def phase_spec(self):
        name = getattr(self.hardening_function, "__name__", None)
        if name not in HARDENING_LAWS:
            raise NotImplementedError(
                f"hardening law {name!r} has no device implementation; use "
                "perfect_plasticity, linear, voce or armstrong_frederick")
        return PhaseSpec("evp", np.asarray(self.stiffness.components, dtype=np.float64),
                         schmid=self.slip_systems.schmid_mandel(),
                         reference_slip_rate=self.reference_slip_rate,
                         rate_exponent=self.rate_exponent,
                         slip_resistance=self.initial_slip_resistance, hardening=name,
                         hardening_props=self.hardening_properties,
                         latent_ratio=self.latent_ratio)

    def generate_outputs(self, output_variables=None):
        if output_variables is not None:
            return {k: self.state_variables.get(k, None) for k in output_variables}
        return dict()

    def __repr__(self):
        return (f"ElasticViscoplastic(stiffness={self.stiffness.voigt}, \n"
                f"slip_systems={self.slip_systems}, \n"
                f"reference_slip_rate={self.reference_slip_rate}, "
                f"rate_exponent={self.rate_exponent}, "
                f"initial_slip_resistance={self.initial_slip_resistance}, "
                f"hardening_function={getattr(self.hardening_function, '__name__', '?')}, "
                f"hardening_properties={self.hardening_properties})")
