"""Containers handed across the package boundary.

``Arrays`` is the reference's attribute bag (lcode/plasma3d/data.py:6-34);
here its attributes are CUDA tensors.  Objects given to user diagnostics wrap
each tensor in ``DeviceArray`` so that the reference's ``get(array)`` idiom
(``array.get()`` for device arrays, lcode/diagnostics/utils.py:11-14) works
unchanged.
"""
from __future__ import annotations

import numpy as np
import torch


class DeviceArray:
    """Read-only view of a CUDA tensor with the cupy-style ``get()``."""

    __slots__ = ("t",)

    def __init__(self, t: torch.Tensor):
        self.t = t

    def get(self) -> np.ndarray:
        return self.t.detach().cpu().numpy()

    def __array__(self, dtype=None, copy=None):
        a = self.get()
        return a if dtype is None else a.astype(dtype)

    @property
    def shape(self):
        return tuple(self.t.shape)

    @property
    def ndim(self):
        return self.t.dim()

    @property
    def size(self):
        return self.t.numel()

    @property
    def dtype(self):
        return np.dtype(str(self.t.dtype).replace("torch.", ""))

    def __getitem__(self, idx):
        r = self.t[idx]
        return DeviceArray(r) if r.dim() > 0 else r.item()

    def __len__(self):
        return self.t.shape[0]

    def copy(self):
        return DeviceArray(self.t.clone())

    def sum(self, axis=None):
        r = self.t.sum() if axis is None else self.t.sum(dim=axis)
        return DeviceArray(r) if r.dim() > 0 else r.item()

    def __repr__(self):
        return f"DeviceArray(shape={self.shape}, dtype={self.dtype}, device={self.t.device})"


class Arrays:
    """Attribute bag of arrays (device tensors inside this package)."""

    def __init__(self, xp=None, **kwargs):
        self.xp = xp
        for name, array in kwargs.items():
            setattr(self, name, array)

    def names(self):
        return [k for k in self.__dict__ if k != "xp"]

    def copy(self) -> "Arrays":
        return Arrays(self.xp, **{k: (v.clone() if isinstance(v, torch.Tensor) else
                                      np.array(v)) for k, v in self.__dict__.items()
                                  if k != "xp"})

    def wrapped(self) -> "Arrays":
        """The same arrays as DeviceArray views (for user diagnostics)."""
        return Arrays(np, **{k: (DeviceArray(v) if isinstance(v, torch.Tensor) else v)
                             for k, v in self.__dict__.items() if k != "xp"})

    def to_numpy(self) -> "Arrays":
        return Arrays(np, **{k: (v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else v)
                             for k, v in self.__dict__.items() if k != "xp"})

    def save(self, *args, **kwargs):
        """np.savez_compressed of every array (lcode/plasma3d/data.py:31-34)."""
        data = {k: v for k, v in self.to_numpy().__dict__.items() if k != "xp"}
        np.savez_compressed(*args, **kwargs, **data)
