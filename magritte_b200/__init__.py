"""B200-native radiation hot path of Magritte (UCL): ray tracing through the
point-cloud neighbour graph, the Feautrier formal solve over every ray pair
and frequency bin, J and approximate-Lambda accumulation, and the
statistical-equilibrium + Ng (ALI) iteration, as hand-written sm_100a CUDA
kernels behind a C ABI (``include/magritte_b200.h``)."""
from .simulation import Simulation, MagritteError  # noqa: F401
from . import model  # noqa: F401

__all__ = ["Simulation", "MagritteError", "model"]
