"""B200-native Kohn-Sham H|psi> + LOBPCG engine (sm_100a).

The compute path is the C ABI of ``include/qumasun_b200.h`` implemented in
``csrc/`` (hand-written CUDA); this package is the host-side binding:

* :mod:`qumasun_b200.cell`   -- synthetic diamond cells, analytic V and projector tables;
* :mod:`qumasun_b200.engine` -- Context / Hamiltonian over the shared library.
"""
from .engine import (Context, Hamiltonian, LearnedPreconditioner, Poisson, QGError, density,  # noqa: F401
                     lib, occupancy)

__all__ = ["Context", "Hamiltonian", "LearnedPreconditioner", "Poisson", "QGError", "density", "lib",
           "occupancy"]
