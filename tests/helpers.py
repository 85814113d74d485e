"""Helpers shared by the tests (comparison metrics, golden loading)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def relerr(a, b):
    """max |a - b| / max |b| (absolute when b is all zeros)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    d = float(np.max(np.abs(a - b))) if a.size else 0.0
    return d / den if den > 0 else d


def normrel(a, b):
    """||a - b|| / ||b|| over all entries."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))
