"""``with_torch``: numpy inputs become torch tensors, outputs go back to numpy."""

import functools

import numpy as np
import torch


def _to_torch(x):
    if isinstance(x, np.ndarray):
        return torch.as_tensor(x)
    return x


def _to_numpy(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    if isinstance(x, tuple):
        return tuple(_to_numpy(v) for v in x)
    if isinstance(x, list):
        return [_to_numpy(v) for v in x]
    return x


def with_torch(fn):
    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        was_numpy = any(isinstance(a, np.ndarray) for a in args) or any(
            isinstance(v, np.ndarray) for v in kwargs.values()
        )
        args = tuple(_to_torch(a) for a in args)
        kwargs = {k: _to_torch(v) for k, v in kwargs.items()}
        out = fn(*args, **kwargs)
        return _to_numpy(out) if was_numpy else out

    return wrapper
