"""Shared test helpers: fixtures loading and error norms."""
import glob
import os

import numpy as np

from tests.golden.make_golden import params_from_json

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "golden_*.npz")))


def load_golden(path):
    d = np.load(path)
    p = params_from_json(str(d["params"]))
    return p, d


def golden_ids():
    return [os.path.basename(g)[7:-4] for g in GOLDEN]


def colwise_rel(a, b, floor=1e-300):
    """max over columns of max|a-b| / max|b| (normwise relative error per
    particle attribute or per mesh component)."""
    a = np.atleast_2d(a)
    b = np.atleast_2d(b)
    num = np.abs(a - b).max(axis=0)
    den = np.maximum(np.abs(b).max(axis=0), floor)
    r = num / den
    r[np.abs(b).max(axis=0) == 0] = num[np.abs(b).max(axis=0) == 0]
    return float(r.max())


def mesh_rel(a, b, ncomp):
    """per-component normwise relative error of GIdx planes"""
    return colwise_rel(a.reshape(ncomp, -1).T, b.reshape(ncomp, -1).T)


def magnitude_mesh(oracle, parts):
    """Per-cell, per-component sum of |contribution| (the deposit of |f| N
    |v|): the scale that rounding errors of a deposit are relative to."""
    q = np.array(parts, dtype=np.float64, copy=True)
    q[:, 3:] = np.abs(q[:, 3:])
    return oracle.deposit(q)


def mesh_rel_mag(a, b, mag, ncomp):
    """max over components of max|a-b| / max(magnitude) of that component"""
    a = a.reshape(ncomp, -1)[3:]
    b = b.reshape(ncomp, -1)[3:]
    m = np.abs(mag.reshape(ncomp, -1)[3:]).max(axis=1)
    err = np.abs(a - b).max(axis=1)
    return float((err / np.maximum(m, 1e-300)).max())


def flavor_cols(nf):
    nh = nf * nf
    return list(range(3 + 10, 3 + 10 + nh)) + list(range(3 + 12 + nh, 3 + 12 + 2 * nh))
