"""curcuma_b200: GFN-FF energy + analytic gradient on NVIDIA B200 (sm_100a).

A drop-in for curcuma's ``-method gfnff -gpu cuda`` path: host setup (topology and
parameters) once per molecule, then energy + gradient per geometry on the GPU through the
C ABI declared in ``include/gfnff_b200.h``.
"""
from .gfnff import FP64, MIXED, GFNFF, atomic_masses, maxwell_boltzmann, write_parameters, write_topology_cache  # noqa: F401
from .sharding import shard_by_cost  # noqa: F401

__all__ = ["GFNFF", "FP64", "MIXED", "atomic_masses", "maxwell_boltzmann", "shard_by_cost", "write_parameters",
           "write_topology_cache"]
