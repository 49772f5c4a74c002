"""B200-native explicit time advance for NOVA (stencil RHS + RK stage + FFT projection).

The compute path is libnova_b200.so (hand-written CUDA for sm_100a behind the
C ABI in include/nova_gpu.h).  ``novaclone_b200.nova`` binds it with the
reference's names; ``python -m novaclone_b200.build`` compiles it in-tree.
"""
from .nova import (Field, Mesh, NovaError, advance, ex, load_library, poisson, run_desc, tools)  # noqa: F401

__all__ = ["Mesh", "Field", "ex", "poisson", "tools", "advance", "run_desc", "NovaError", "load_library"]
