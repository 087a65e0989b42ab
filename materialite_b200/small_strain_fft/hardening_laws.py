"""Slip-resistance laws of materialite's crystal plasticity
(materialite/models/small_strain_fft/hardening_laws.py:18-90).

On the GPU path the law is selected by name and evaluated in the constitutive kernel
(csrc/constitutive.cuh, ``harden_iso``); these host versions state the same closed forms
for inspection and host-side checks.  A user-written law has no device version and is
rejected by SmallStrainFFT."""

import numpy as np

from ..tensor import Scalar


def _slip_increment(plastic_slip_rates, time_increment):
    try:
        return time_increment * plastic_slip_rates.abs.sum("s")
    except ValueError:
        return time_increment * plastic_slip_rates.abs


def perfect_plasticity(properties, old_accumulated_slip, old_slip_resistances,
                       plastic_slip_rates, time_increment):
    return old_slip_resistances


def linear(properties, old_accumulated_slip, old_slip_resistances, plastic_slip_rates,
           time_increment):
    return (old_slip_resistances
            + properties["hardening_rate"] * _slip_increment(plastic_slip_rates, time_increment))


def voce(properties, old_accumulated_slip, old_slip_resistances, plastic_slip_rates,
         time_increment):
    dg = _slip_increment(plastic_slip_rates, time_increment)
    th0, th1, tau1 = properties["theta_0"], properties["theta_1"], properties["tau_1"]
    ratio = np.abs(th0 / tau1)
    e_i = Scalar(np.exp(-ratio * old_accumulated_slip.components), old_accumulated_slip.dims_str)
    e_c = Scalar(np.exp(-ratio * dg.components), dg.dims_str)
    return (old_slip_resistances + dg * th1 - e_i * (e_c - 1) * ((ratio * tau1 - th1) / ratio)
            - e_i * (e_c * ((old_accumulated_slip + dg) * ratio + 1) - 1
                     - old_accumulated_slip * ratio) * (th1 / ratio))


def armstrong_frederick(properties, old_accumulated_slip, old_slip_resistances,
                        plastic_slip_rates, time_increment):
    h = properties["direct_hardening"]
    r = properties["dynamic_recovery"]
    dg = _slip_increment(plastic_slip_rates, time_increment)
    return old_slip_resistances + (old_slip_resistances * (-r) + h) * (dg / (dg * r + 1))


HARDENING_LAWS = {f.__name__: f for f in (perfect_plasticity, linear, voce, armstrong_frederick)}
