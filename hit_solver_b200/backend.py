"""Array-backend selection (OOP/parallel/backend.py:8-38) for the b200 path.

``select_array_module("b200")`` returns :mod:`torch`: torch CUDA tensors are
the only array type of this backend.  The reference's own ``numpy`` and
``cupy`` backends are the reference implementation and are not provided here
(there is no CPU fallback).
"""

from __future__ import annotations

import numpy as np


def select_array_module(backend: str):
    if backend in ("b200", "auto"):
        import torch

        if not torch.cuda.is_available():
            raise RuntimeError("B200 backend requested, but no CUDA device is available.")
        from . import _lib

        _lib.load()
        return torch
    if backend in ("numpy", "cupy"):
        raise RuntimeError(
            f"backend '{backend}' is the reference implementation; this package runs the "
            "b200 backend only")
    raise ValueError("backend must be 'auto', 'numpy', 'cupy', or 'b200'")


def array_module(values):
    module = type(values).__module__.split(".")[0]
    if module == "torch":
        import torch

        return torch
    return np


def to_numpy(values):
    """Host copy of a torch tensor (any device) or pass-through of numpy data."""
    if type(values).__module__.split(".")[0] == "torch":
        return values.detach().cpu().numpy()
    return np.asarray(values)
