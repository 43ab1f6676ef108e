"""fftsvd_b200 — FFTSVD boundary-element PBE matvec and GMRES solve on NVIDIA B200.

The compute path is the in-tree CUDA library libfftsvd_b200.so (sm_100a);
this package is its host-side mirror:

* ``surface``  — Surface objects and the reference-named entry points
  (generateSurfaceOperator, generateRHS, solveSurfaceOperator, collectPotentials);
* ``meshes``   — seeded synthetic surfaces and charge sets;
* ``frontend`` — the reference's input readers (parameters, PDB/CRD/XYZR, SIZ/CRG,
  vert/face meshes, SRF) and the FFTSVDpbe input sequence;
* ``lib``      — the ctypes binding (fails loudly when the library is absent).
"""
from .lib import FFTSVDError, load  # noqa: F401
from .surface import (Surface, collectPotentials, generateRHS, generateSurfaceOperator,  # noqa: F401
                      solvation_energy, solveSurfaceOperator, two_region_maps, two_region_precond)

__all__ = ["Surface", "FFTSVDError", "generateSurfaceOperator", "generateRHS", "solveSurfaceOperator",
           "collectPotentials", "solvation_energy", "two_region_maps", "two_region_precond", "load"]
