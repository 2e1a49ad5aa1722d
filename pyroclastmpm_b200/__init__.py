"""B200-native update-stress-last MPM step for PyroclastMPM users.

- ``pyroclastmpm_b200.MPM2D`` / ``MPM3D``: the reference's Python module API
  (``set_globals``, ``ParticlesContainer``, ``NodesContainer``, ``USL``,
  materials and boundary conditions), backed by the C ABI.
- ``pyroclastmpm_b200._capi.Simulation``: direct binding of the C ABI
  (include/pmpm.h).
"""
from ._capi import Batch, PmpmError, Simulation, lib, material_point_update  # noqa: F401

__all__ = ["Simulation", "Batch", "PmpmError", "lib", "material_point_update"]
