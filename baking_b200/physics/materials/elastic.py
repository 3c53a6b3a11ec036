"""Neo-Hookean material (the reference's ``physics/materials/elastic.py:4-49``).

tau = mu (F F^T - I) + lambda log(J) I; J <= 0 or non-finite sets error flag 0.
"""

from __future__ import annotations

from ... import _lib, arrays


def ComputeElasticStress(deformation_gradients, kirchhoff_stresses, shear_modulus, lame_lambda, error_flags):
    n = deformation_gradients.shape[0]
    pitch = arrays.common_pitch(deformation_gradients, kirchhoff_stresses)
    _lib.call("bk_compute_elastic_stress", n, pitch, arrays.ptr(deformation_gradients), arrays.ptr(kirchhoff_stresses),
              shear_modulus, lame_lambda, error_flags.data_ptr(), _lib.stream_handle())


class ElasticMaterial:
    """Material plugin base: ``ComputeStress``, ``AdvanceState`` (reference elastic.py:29-49)."""

    def __init__(self, material_config):
        material_config.Validate()
        self.material_config = material_config

    def ComputeStress(self, particle_state, kirchhoff_stresses, error_flags):
        ComputeElasticStress(particle_state.deformation_gradients, kirchhoff_stresses,
                             self.material_config.shear_modulus, self.material_config.lame_lambda, error_flags)

    def AdvanceState(self, input_state, output_state, time_step):
        output_state.material_state = None
