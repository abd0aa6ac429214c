"""sbb — B200-native FP64 CSR SpMV (y = alpha*A*x + beta*y).

Host-side mirror of JieyangChen7/Sparse-BLAS's entry points over libsbb.so:

* ``sbb.api``    the reference's spMV_mgpu_baseline / _v1 / _v2 and helpers,
                 host numpy arrays in, y updated in place;
* ``sbb.device`` plans over device-resident (torch CUDA) arrays;
* ``sbb.gen``    seeded synthetic matrices for the benchmark configurations.
"""
from . import api  # noqa: F401
from ._lib import lib, last_error  # noqa: F401
