"""B200-native AMLS eigensolver for K x = lambda M x.

Python face of libamls_b200.so, mirroring the reference's C++ API:
``AmlsOptions`` / ``AmlsSolver.solve`` (src/amls/solver.hpp:18-52),
``recursive_bisection`` (src/partition/partitioner.hpp:8-31) and the batched
dense generalized eigensolver (src/linalg/dense_eigensolver.hpp:11-31).
"""
from .solver import (AmlsOptions, AmlsSolver, Solution, read_matrix_market,  # noqa: F401
                     recursive_bisection, sygvx_batched, write_matrix_market)
from ._lib import AmlsStatusError, NotSPDError  # noqa: F401
