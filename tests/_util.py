"""Shared helpers for the tests (numpy oracle arrays <-> device tensors)."""

import numpy as np
import torch


def to_dev(a, g):
    """numpy array (oracle layout) -> contiguous device tensor of the grid's precision."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    if np.iscomplexobj(a):
        t = t.to(g.cdtype)
    else:
        t = t.to(g.dtype)
    return t.to(g.device).contiguous()


def to_np(t):
    return t.detach().cpu().numpy().astype(np.complex128 if t.is_complex() else np.float64)


def rel_l2(a, b):
    if isinstance(a, np.ndarray):
        a, b = [a], [b]
    num = sum(float(np.sum(np.abs(x - y) ** 2)) for x, y in zip(a, b))
    den = sum(float(np.sum(np.abs(y) ** 2)) for y in b)
    return (num / den) ** 0.5 if den > 0 else num ** 0.5
