"""eggsync -- B200 (sm_100a) EGG-SynC synchronisation clustering.

The compute path is libeggsync.so (CUDA kernels + C ABI, include/eggsync.h);
this package is its Python front end, mirroring the reference's
python/algorithms.py entry points.
"""
from .algorithms import (DEFAULT_LAMBDA, EGG_SynC, EggError, egg_grid, egg_step, egg_sync,  # noqa: F401
                         egg_sync_batch, impl)

__all__ = ["EGG_SynC", "impl", "egg_sync", "egg_sync_batch", "egg_step", "egg_grid", "EggError", "DEFAULT_LAMBDA"]
