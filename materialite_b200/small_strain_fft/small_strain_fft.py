"""SmallStrainFFT: the drop-in model class
(materialite/models/small_strain_fft/small_strain_fft.py:30-398).

``SmallStrainFFT(load_schedule=..., constitutive_model=...)(material)`` returns a new
Material with ``stress`` and ``strain`` (and requested state variables), like the
reference.  The solve runs on the GPU through libssfft; the time loop, the LoadSchedule
closures and output collection run here, as in the reference.  There is no CPU path:
without a CUDA device and the built library the call raises.

Extensions beyond the reference's keywords: ``precision`` ("fp64", the reference's
arithmetic and the default, or "mixed": float fields/FFTs/Krylov vectors with double
residuals, norms and crystal-plasticity Newton) and ``device`` (CUDA ordinal).
"""

import logging
from collections import defaultdict

import numpy as np

from ..engine import SolverHandle, SolveStats, solve, unique_rotations
from ..tensor import Order2SymmetricTensor, Scalar
from .multiphase import Multiphase


class Model:
    """Plugin base (materialite/models/model.py:16-30)."""

    def __call__(self, material, **kwargs):
        return self.run(material, **kwargs)

    def run(self, *args, **kwargs):
        raise NotImplementedError

    def verify_material(self, material, required_field_labels):
        labels = list(material.get_fields())
        if not all(l in labels for l in required_field_labels):
            raise AttributeError(f"{type(self)} requires the Material to have fields with labels "
                                 f"{required_field_labels}. The actual field labels are {labels}.")
        return material


# Which phase kinds carry each state variable (the constitutive models'
# available_state_variables).
STATE_VARIABLE_KINDS = {
    "slip_resistances": ("evp",), "slip_system_shear_strains": ("evp",),
    "plastic_strains": ("evp", "j2"), "yield_stresses": ("j2",),
    "eq_plastic_strains": ("j2",),
}


class SmallStrainFFT(Model):
    def __init__(self, load_schedule, end_time=1, initial_time_increment=None,
                 max_time_increment=None, min_time_increment=1.0e-9, start_time=0.0,
                 constitutive_model=None, precision="fp64", device=0):
        self.load_schedule = load_schedule
        self.end_time = end_time
        self.initial_time_increment = (self.end_time if initial_time_increment is None
                                       else initial_time_increment)
        self.max_time_increment = (self.initial_time_increment if max_time_increment is None
                                   else max_time_increment)
        self.min_time_increment = min_time_increment
        self.start_time = start_time
        self._constitutive_model = constitutive_model
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self.device = device
        self._logger = logging.getLogger("SmallStrainFFT")
        self.last_stats = None

    def _get_constitutive_model(self, material, phase_label, constitutive_model):
        """small_strain_fft.py:384-398."""
        if phase_label is not None and constitutive_model is not None:
            raise ValueError("cannot specify phase and constitutive model")
        if phase_label is None and constitutive_model is None:
            raise ValueError("must specify phase label or provide a constitutive model")
        if phase_label is not None:
            df = material.extract_regional_field(phase_label)
            phases = df[phase_label].to_list()
            models = df["constitutive_model"].to_list()
            idx = material.get_region_indices(region_label=phase_label)
            return Multiphase(phases, models, [idx.get(p, np.zeros(0, dtype=np.int64))
                                               for p in phases], material.num_points)
        return constitutive_model

    def run(self, material, orientation_label="orientation", phase_label=None,
            output_variables=None, output_times=None, global_tolerance=1.0e-3,
            strain_correction_tolerance=1.0e-2, linear_solver_tolerance=1.0e-5,
            postprocessor=None):
        dims = tuple(int(d) for d in material.dimensions)
        V = int(np.prod(dims))
        model = self._get_constitutive_model(material, phase_label, self._constitutive_model)
        if isinstance(model, Multiphase):
            models = model.models
            phase_of_point = model.phase_of_point()
            model.check_output_variables(output_variables)
        else:
            models = [model]
            phase_of_point = None
        specs = [m.phase_spec() for m in models]
        orientations = material.extract(orientation_label)
        R = np.asarray(orientations.rotation_matrix, dtype=np.float64).reshape(V, 3, 3)
        table, index = unique_rotations(R)
        ls = self.load_schedule
        handle = SolverHandle(dims, np.asarray(ls.stress_mask, dtype=float), self.precision,
                              global_tolerance=global_tolerance,
                              strain_correction_tolerance=strain_correction_tolerance,
                              linear_solver_tolerance=linear_solver_tolerance, device=self.device)
        try:
            handle.set_phases(specs)
            handle.set_microstructure(table, index, phase_of_point)
            device_vars = [v for v in (output_variables or [])
                           if v in STATE_VARIABLE_KINDS and handle.nslip]
            phase_kinds = [sp.kind for sp in specs]
            comps = lambda f: (lambda t, dt: np.asarray(f(t, dt).components, dtype=float))
            stats = SolveStats()
            nslip = handle.nslip
            phase_slips = [len(m.slip_systems) if hasattr(m, "slip_systems") else 0
                           for m in models]

            def hook(history, h, variables):
                outs = self._outputs(h, variables, device_vars, V, nslip, phase_of_point,
                                     phase_slips, phase_kinds)
                outs["stress"] = Order2SymmetricTensor(h.field("stress"), "p")
                outs["strain"] = Order2SymmetricTensor(h.field("strain"), "p")
                if postprocessor is not None:
                    outs = postprocessor(outs)
                for k, v in outs.items():
                    history[k].append(v)

            final, history = solve(handle, comps(ls.strain_increment), comps(ls.stress_increment),
                                   comps(ls.stress), end_time=self.end_time,
                                   initial_time_increment=self.initial_time_increment,
                                   max_time_increment=self.max_time_increment,
                                   min_time_increment=self.min_time_increment,
                                   start_time=self.start_time, output_times=output_times,
                                   output_variables=output_variables, stats=stats,
                                   outputs_hook=hook)
            final_outs = self._outputs(handle, output_variables, device_vars, V, nslip,
                                       phase_of_point, phase_slips, phase_kinds)
            final_outs["stress"] = Order2SymmetricTensor(final["stress"], "p")
            final_outs["strain"] = Order2SymmetricTensor(final["strain"], "p")
            self.last_stats = stats
        finally:
            handle.close()
        if output_times is None:
            return material.create_fields(final_outs)
        if postprocessor is None:
            stacked = {}
            for k, v in history.items():
                if v and v[0] is not None:
                    stacked[k] = type(v[0]).from_stack(v, new_dim="t", axis=len(v[0].dims_str))
                else:
                    stacked[k] = v
            return material.create_fields(stacked)
        new_material = material.create_fields(final_outs)
        new_material.state.update(dict(history))
        return new_material

    @staticmethod
    def _outputs(handle, variables, device_vars, V, nslip, phase_of_point, phase_slips,
                 phase_kinds):
        """generate_outputs of the constitutive models (elastic_viscoplastic.py:278-285,
        isotropic_elastic_plastic.py:177-183, multiphase.py:63-95): state variables of the
        plastic phases, None for variables a single-phase model does not have, zeros
        where a phase lacks them."""
        outs = {}
        for v in variables or []:
            if v not in device_vars:
                outs[v] = None
                continue
            data = handle.field(v)
            kinds = STATE_VARIABLE_KINDS[v]
            if phase_of_point is not None:
                lacks = np.array([k not in kinds for k in phase_kinds])[phase_of_point]
                data[lacks] = 0.0
            elif phase_kinds[0] not in kinds:
                outs[v] = None
                continue
            if v == "plastic_strains":
                outs[v] = Order2SymmetricTensor(data, "p")
            elif v in ("yield_stresses", "eq_plastic_strains"):
                outs[v] = Scalar(data[:, 0], "p")
            else:
                evp_slips = [n for n, k in zip(phase_slips, phase_kinds) if k == "evp"]
                width = max(evp_slips) if evp_slips else nslip
                outs[v] = Scalar(data[:, :width], "ps")
        return outs
