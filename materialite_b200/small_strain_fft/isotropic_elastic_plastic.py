"""J2 elastic-plastic model (materialite/models/small_strain_fft/isotropic_elastic_plastic.py).

Not implemented on the device path yet; SmallStrainFFT raises NotImplementedError when a
phase uses it (there is no CPU fallback)."""


class IsotropicElasticPlastic:
    def __init__(self, modulus, shear_modulus, yield_stress, hardening_function,
                 hardening_properties):
        self.modulus = modulus
        self.shear_modulus = shear_modulus
        self.yield_stress = yield_stress
        self.hardening_function = hardening_function
        self.hardening_properties = hardening_properties
        self.available_state_variables = ["plastic_strains", "eq_plastic_strains"]
        self.state_variables = dict()

    def phase_spec(self):
        raise NotImplementedError(
            "IsotropicElasticPlastic has no device implementation in materialite_b200")
