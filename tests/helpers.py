"""Shared helpers for the parity tests (no product code here)."""
import numpy as np
import torch


def rel_fro(x, ref):
    x = np.asarray(x.cpu() if torch.is_tensor(x) else x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.linalg.norm(ref.ravel())
    return float(np.linalg.norm((x - ref).ravel()) / (den if den > 0 else 1.0))


def max_abs(x, ref):
    x = np.asarray(x.cpu() if torch.is_tensor(x) else x, dtype=np.float64)
    return float(np.max(np.abs(x - np.asarray(ref, dtype=np.float64)))) if x.size else 0.0


def to_np(t):
    return np.asarray(t.detach().cpu().numpy() if torch.is_tensor(t) else t, dtype=np.float64)


def f32_round(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)
