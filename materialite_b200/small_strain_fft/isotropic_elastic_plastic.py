"""J2 small-strain plasticity
(materialite/models/small_strain_fft/isotropic_elastic_plastic.py:17-192).

Isotropic elasticity with a von Mises yield surface and radial return. The return
mapping runs per voxel in double precision in libssfft (csrc/constitutive.cuh). Its
iteration is the reference's: a fixed-point update of the equivalent plastic strain
increment with the constant inverse Jacobian -1/(3G), every point iterated until all have
converged (tolerance 1e-7, at most 100 iterations). When every point is elastic the update
returns the elastic stress and leaves the plastic state untouched, as the reference does."""

import numpy as np

from ..engine import PhaseSpec
from .hardening_laws import HARDENING_LAWS


class IsotropicElasticPlastic:
    def __init__(self, modulus, shear_modulus, yield_stress, hardening_function,
                 hardening_properties):
        from ..tensor import Order2SymmetricTensor, Order4SymmetricTensor, Scalar
        self.modulus = modulus
        self.shear_modulus = shear_modulus
        self.bulk_modulus = shear_modulus * modulus / (3 * (3 * shear_modulus - modulus))
        self.stiffness = Order4SymmetricTensor.from_isotropic_constants(modulus, shear_modulus)
        self.yield_stress = Scalar(yield_stress)
        self.hardening_function = hardening_function
        self.hardening_properties = hardening_properties
        self.state_variables = dict()
        self.available_state_variables = ["yield_stresses", "plastic_strains",
                                          "eq_plastic_strains"]
        self._state_variable_info = dict(zip(self.available_state_variables,
                                             [(Scalar, 0), (Order2SymmetricTensor, 0),
                                              (Scalar, 0)]))

    def phase_spec(self):
        name = getattr(self.hardening_function, "__name__", None)
        if name not in HARDENING_LAWS:
            raise NotImplementedError(
                f"hardening law {name!r} has no device implementation; use "
                "perfect_plasticity, linear, voce or armstrong_frederick")
        return PhaseSpec("j2", np.asarray(self.stiffness.components, dtype=np.float64),
                         slip_resistance=float(np.asarray(self.yield_stress.components)),
                         hardening=name, hardening_props=self.hardening_properties,
                         modulus=float(self.modulus), shear_modulus=float(self.shear_modulus))

    def generate_outputs(self, output_variables=None):
        if output_variables is not None:
            return {k: self.state_variables.get(k, None) for k in output_variables}
        return dict()

    def __repr__(self):
        return (f"IsotropicElasticPlastic(modulus={self.modulus}, "
                f"shear_modulus={self.shear_modulus}, "
                f"yield_stress={self.yield_stress.components}, "
                f"hardening_function={self.hardening_function.__name__}, "
                f"hardening_properties={self.hardening_properties})")
