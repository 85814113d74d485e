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


def write_mpmbin(path, x, v, F, C, P, m, vol, lam, mu, dFc, dLdx=None, dLdv=None, dLdF=None):
    """A cereal binary archive of std::vector<MaterialPoint> (the reference's
    .mpmbin): uint64 count, then per point x, v, F, C, P, m, vol, lam, mu, dFc,
    dLdx, dLdv, dLdF, momentum, vector, vector_max; vectors as int32 rows + 3
    floats, matrices as int32 rows, int32 cols + 9 floats in row order."""
    import struct

    n = len(x)
    z3 = np.zeros((n, 3))
    z33 = np.zeros((n, 3, 3))
    dLdx = z3 if dLdx is None else dLdx
    dLdv = z3 if dLdv is None else dLdv
    dLdF = z33 if dLdF is None else dLdF
    vec = lambda a: struct.pack("<i3f", 3, *np.asarray(a, dtype=np.float32))
    mat = lambda a: struct.pack("<ii9f", 3, 3, *np.asarray(a, dtype=np.float32).reshape(9))
    f = lambda a: struct.pack("<f", np.float32(a))
    with open(path, "wb") as fh:
        fh.write(struct.pack("<Q", n))
        for p in range(n):
            fh.write(vec(x[p]) + vec(v[p]) + mat(F[p]) + mat(C[p]) + mat(P[p]) + f(m[p]) + f(vol[p]) + f(lam[p]) +
                     f(mu[p]) + mat(dFc[p]) + vec(dLdx[p]) + vec(dLdv[p]) + mat(dLdF[p]) + mat(z33[p]) + mat(z33[p]) +
                     mat(z33[p]))
