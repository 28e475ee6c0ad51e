"""eggsync -- B200 (sm_100a) EGG-SynC synchronisation clustering.

The compute path is libeggsync.so (CUDA kernels + C ABI, include/eggsync.h);
this package is its Python front end, mirroring the reference's
python/algorithms.py entry points.
"""
from .algorithms import (DEFAULT_LAMBDA, EGG_SynC, EggError, GPU_DynamicalClustering, egg_grid,  # noqa: F401
                         egg_step, egg_sync, egg_sync_batch, impl, knn_mean, mdl_cost, mdl_search, normalize,
                         simple_sync)

__all__ = ["EGG_SynC", "GPU_DynamicalClustering", "impl", "egg_sync", "egg_sync_batch", "egg_step", "egg_grid",
           "normalize", "simple_sync", "knn_mean", "mdl_cost", "mdl_search", "EggError", "DEFAULT_LAMBDA"]
