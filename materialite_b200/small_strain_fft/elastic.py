"""Elastic constitutive model (materialite/models/small_strain_fft/elastic.py:16-49).

The per-voxel update sigma = K_spec : eps runs in libssfft; this object carries the
stiffness, holds the state the reference exposes (``state_variables``), and describes
the phase to the solver."""

import numpy as np

from ..engine import PhaseSpec


class Elastic:
    def __init__(self, stiffness):
        self.stiffness = stiffness
        self.state_variables = dict()
        self.available_state_variables = None
        self._state_variable_info = dict()

    def phase_spec(self):
        return PhaseSpec("elastic", np.asarray(self.stiffness.components, dtype=np.float64))

    def generate_outputs(self, output_variables=None):
        if output_variables is not None:
            return {k: self.state_variables.get(k, None) for k in output_variables}
        return dict()

    def __repr__(self):
        return f"Elastic(stiffness={np.round(self.stiffness.voigt, 3)})"
