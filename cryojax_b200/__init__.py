"""cryojax_b200: B200 (sm_100a) Fourier-slice + CTF image simulation.

A from-scratch CUDA implementation of cryoJAX's FourierSliceExtraction /
AstigmaticCTF / LinearImageModel path behind a C-ABI library
(include/cryojax_b200.h), with a host-side mirror of the reference's
simulator API in ``cryojax_b200.simulator``.
"""

from . import constants, rotations, simulator  # noqa: F401
from ._native import CryojaxB200Error, load_library  # noqa: F401

__all__ = ["simulator", "rotations", "constants", "load_library", "CryojaxB200Error"]
