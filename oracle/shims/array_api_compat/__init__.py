"""Oracle shim: the reference imports ``array_api_compat`` (pinned 1.15.0 in its
uv.lock) only to resolve the namespace of host arrays. NumPy 2.x is itself an
array-API namespace, so every host array resolves to ``numpy``. Test
infrastructure only."""

import numpy as _np


def array_namespace(*arrays):
    return _np


def is_jax_array(array):
    return False


def is_cupy_array(array):
    return False


def is_numpy_array(array):
    return isinstance(array, _np.ndarray)
