"""B200-native BIGSTICK M-scheme Hamiltonian application and Lanczos.

Layers:
  model   -- inputs (.sps/.int, synthetic interactions) and the host-side
             table build (libbsghost.so, the stand-in for the Fortran host)
  engine  -- the sm_100a engine behind the C ABI (libbsgpu.so)
"""
from . import model  # noqa: F401

__all__ = ["model", "engine"]
