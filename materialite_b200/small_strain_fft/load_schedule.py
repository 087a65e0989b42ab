# Portions of this file restate the interface and the boundary-condition closures of materialite's
# materialite/models/small_strain_fft/load_schedule.py: Copyright 2025 United States Government as represented by the Administrator
# of the National Aeronautics and Space Administration.  All Rights Reserved.  Licensed
# under the Apache License, Version 2.0 (http://www.apache.org/licenses/LICENSE-2.0);
# distributed on an "AS IS" BASIS, WITHOUT WARRANTIES OR CONDITIONS OF ANY KIND.

"""Mixed strain/stress boundary conditions as closures of (t, dt)
(materialite/models/small_strain_fft/load_schedule.py:17-119)."""

import numpy as np

from ..tensor import Order2SymmetricTensor


class LoadSchedule:
    def __init__(self, strain_increment, stress_increment, stress, stress_mask):
        self.strain_increment = strain_increment
        self.stress_increment = stress_increment
        self.stress = stress
        self.stress_mask = np.asarray(stress_mask)
        if np.any(np.logical_and(self.stress_mask != 1, self.stress_mask != 0)):
            raise ValueError("stress mask can only have zeros and ones")

    @staticmethod
    def apply_stress_mask(strain, stress, stress_mask):
        return (Order2SymmetricTensor(strain.components * (1 - stress_mask)),
                Order2SymmetricTensor(stress.components * stress_mask))

    @classmethod
    def from_constant_rates(cls, strain_rate, stress_rate, stress_mask, start_time=0):
        strain_rate, stress_rate = cls.apply_stress_mask(strain_rate, stress_rate, stress_mask)
        return cls(lambda t, dt: strain_rate * dt, lambda t, dt: stress_rate * dt,
                   lambda t, dt: stress_rate * (t + dt - start_time), stress_mask)

    @classmethod
    def from_constant_uniaxial_strain_rate(cls, magnitude=1.0, direction="z", start_time=0):
        rates = {"x": [magnitude, 0, 0], "y": [0, magnitude, 0], "z": [0, 0, magnitude]}
        masks = {"x": [0, 1, 1], "y": [1, 0, 1], "z": [1, 1, 0]}
        stress_mask = np.concatenate([masks[direction], np.ones(3)])
        strain_rate = Order2SymmetricTensor(np.concatenate([rates[direction], np.zeros(3)]))
        return cls.from_constant_rates(strain_rate, Order2SymmetricTensor.zero(), stress_mask,
                                       start_time)

    @classmethod
    def from_ramp(cls, times, strains, stresses, stress_mask):
        start_time = times[0]
        dtime = times[1] - start_time
        strains, stresses = cls.apply_stress_mask(strains, stresses, stress_mask)
        strain_rate = (strains[1] - strains[0]) / dtime
        stress_rate = (stresses[1] - stresses[0]) / dtime
        return cls(lambda t, dt: strain_rate * dt, lambda t, dt: stress_rate * dt,
                   lambda t, dt: stress_rate * (t + dt - start_time) + stresses[0], stress_mask)

    @classmethod
    def from_cyclic_stress(cls, stress_amplitude, frequency, stress_mask=np.ones(6), start_time=0,
                           ramp_rate=0):
        amp = Order2SymmetricTensor(stress_amplitude.components * stress_mask)
        f = lambda t: amp * ((1 + ramp_rate * (t - start_time))
                             * np.sin(2 * np.pi * frequency * (t - start_time)))
        return cls(lambda t, dt: Order2SymmetricTensor.zero(), lambda t, dt: f(t + dt) - f(t),
                   lambda t, dt: f(t + dt), stress_mask)

    @classmethod
    def from_cyclic_strain(cls, strain_amplitude, frequency, stress_mask, start_time=0,
                           ramp_rate=0):
        amp = Order2SymmetricTensor(strain_amplitude.components * (1 - stress_mask))
        f = lambda t: amp * ((1 + ramp_rate * (t - start_time))
                             * np.sin(2 * np.pi * frequency * (t - start_time)))
        return cls(lambda t, dt: f(t + dt) - f(t), lambda t, dt: Order2SymmetricTensor.zero(),
                   lambda t, dt: Order2SymmetricTensor.zero(), stress_mask)
