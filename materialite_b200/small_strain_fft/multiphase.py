"""Per-phase constitutive dispatch (materialite/models/small_strain_fft/multiphase.py:18-95).

On the device every point carries a phase index into the solver's phase table; this
object groups the phase models and point indices and merges their output variables as
the reference does (zeros where a phase lacks a variable)."""

import numpy as np


class Multiphase:
    def __init__(self, phases, models, indices, num_points):
        self.phases = phases
        self.models = models
        self.indices = indices
        self.num_points = num_points
        self.available_state_variables = []
        for m in self.models:
            if m.available_state_variables is not None:
                self.available_state_variables += m.available_state_variables

    def phase_of_point(self):
        out = np.full(self.num_points, -1, dtype=np.int32)
        for k, idx in enumerate(self.indices):
            out[np.asarray(idx, dtype=np.int64)] = k
        if np.any(out < 0):
            raise ValueError("every point needs a phase with a constitutive model")
        return out

    def check_output_variables(self, output_variables):
        for v in output_variables or []:
            if v not in self.available_state_variables:
                raise ValueError(f"output variable {v} is not available in any constitutive "
                                 "models in this simulation")
