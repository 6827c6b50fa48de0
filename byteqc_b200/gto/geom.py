"""Seeded geometry generators for the measured workloads.

* ``water_cluster(k, seed)``: k rigid waters (O-H 0.9572 A, H-O-H 104.52 deg)
  placed at the first k sites of a cubic lattice of spacing 3.1 A, each site
  jittered by a uniform +-0.2 A per axis and each molecule given a uniformly
  random orientation (random unit quaternion), all from ``seed``.
* ``linear_alkane(n)``: all-trans CnH(2n+2) with C-C 1.54 A, C-H 1.09 A and
  tetrahedral angles.
"""
import math

import numpy as np

ROH = 0.9572
THETA_HOH = math.radians(104.52)


def _random_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def water_cluster(k, seed=0, spacing=3.1, jitter=0.2):
    """List of (symbol, xyz[A]) for k waters."""
    rng = np.random.default_rng(seed)
    n = max(1, int(math.ceil(k ** (1. / 3) - 1e-9)))
    sites = [(i, j, l) for i in range(n) for j in range(n) for l in range(n)][:k]
    h = 0.5 * THETA_HOH
    local = np.array([[0., 0., 0.],
                      [ROH * math.sin(h), 0., ROH * math.cos(h)],
                      [-ROH * math.sin(h), 0., ROH * math.cos(h)]])
    atoms = []
    for s in sites:
        center = np.array(s, dtype=float) * spacing + rng.uniform(-jitter, jitter, 3)
        rot = _random_rotation(rng)
        xyz = local @ rot.T + center
        for sym, r in zip(('O', 'H', 'H'), xyz):
            atoms.append((sym, tuple(r)))
    return atoms


def linear_alkane(n, rcc=1.54, rch=1.09):
    """All-trans CnH(2n+2) in the xy plane (carbon zigzag along x)."""
    tet = math.acos(-1. / 3)            # 109.47 deg
    half = 0.5 * tet
    dx = rcc * math.sin(half)
    dy = rcc * math.cos(half)
    carbons = [np.array([i * dx, (i % 2) * dy, 0.]) for i in range(n)]
    atoms = [('C', tuple(c)) for c in carbons]
    hs = []
    for i, c in enumerate(carbons):
        # bisector direction pointing away from the backbone
        ydir = -1. if i % 2 == 0 else 1.
        out = np.array([0., ydir, 0.])
        # two out-of-plane hydrogens of a CH2 (or the CH3 pair)
        for s in (1., -1.):
            v = math.cos(half) * out + math.sin(half) * np.array([0., 0., s])
            hs.append(c + rch * v / np.linalg.norm(v))
        ends = ([-1] if i == 0 else []) + ([n] if i == n - 1 else [])
        for k in ends:
            # a methyl hydrogen sits where the zigzag's next carbon would be
            virtual = np.array([k * dx, (k % 2) * dy, 0.])
            v = virtual - c
            hs.append(c + rch * v / np.linalg.norm(v))
    atoms += [('H', tuple(h)) for h in hs]
    return atoms
