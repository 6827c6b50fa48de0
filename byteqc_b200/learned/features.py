"""Atom-pair features, local frames and AO-block rotations of the learned
initial-density model.

Every atom pair (A, B) within PAIR_CUTOFF (on-site pairs A == B included) is
one sample.  Its density block D_AB (AOs of A x AOs of B) is predicted in a
local frame of the pair, so the network sees rotation-invariant inputs and
produces rotation-invariant outputs:

* frame: z along A -> B (on-site: towards the nearest neighbour), x towards
  the nearest other atom to the pair centre, projected off z; y = z x x;
* features (FEAT_DIM = 64, zero padded): one-hot pair type (9), distance
  r_AB on 16 Gaussian radial functions, local coordinates and element flags
  of the 4 atoms nearest to the pair centre, counts of H and heavy atoms
  within 3.5 A of A and of B;
* target: the local-frame block minus the local-frame SAD block (the SAD
  block is zero off-site), flattened and padded to OUT_DIM.

The AO block of a shell of angular momentum l rotates with the orthogonal
matrix U_l solving Y_m(R^T u) = sum_m' Y_m'(u) U_m'm for the real solid
harmonics Y of the basis (found by least squares on sample directions).
"""
import numpy as np

from ..gto import mole as gto

ANG = 0.52917721092           # Angstrom per Bohr
PAIR_CUTOFF = 5.0             # Angstrom
FEAT_DIM = 64
OUT_DIM = 208                 # >= 14 x 14 (largest DZ-shaped block), multiple of 16
# output width per basis shape: the largest atom-pair block, rounded up to 16
OUT_DIMS = {'cc-pvdz': 208, 'cc-pvtz': 912}   # 14 x 14 and 30 x 30 AOs
ELEMENT_RANK = {'O': 3, 'N': 2, 'C': 1, 'H': 0}
PAIR_TYPES = ['O', 'C', 'H', 'OO', 'CC', 'HH', 'OH', 'CH', 'OC']
RBF_CENTRES = np.linspace(0.5, 6.0, 16)
RBF_WIDTH = 0.35


def _sym(mol, a):
    return mol.atom[a][0]


def pair_type(sa, sb, onsite):
    if onsite:
        return PAIR_TYPES.index(sa)
    return PAIR_TYPES.index(sa + sb)


def canonical_pairs(mol, cutoff=PAIR_CUTOFF):
    """(A, B) with rank(A) >= rank(B) (ties: A <= B) and r_AB <= cutoff."""
    xyz = mol.atom_coords() * ANG
    syms = [a[0] for a in mol.atom]
    out = []
    for a in range(mol.natm):
        for b in range(mol.natm):
            ra, rb = ELEMENT_RANK[syms[a]], ELEMENT_RANK[syms[b]]
            if ra < rb or (ra == rb and a > b):
                continue
            if np.linalg.norm(xyz[a] - xyz[b]) <= cutoff:
                out.append((a, b))
    return out


def local_frame(xyz, a, b):
    """Rows (ex, ey, ez) of the pair frame, and the pair centre."""
    n = len(xyz)
    centre = 0.5 * (xyz[a] + xyz[b])
    others = [c for c in range(n) if c != a and c != b]
    if a != b:
        ez = xyz[b] - xyz[a]
    else:
        if others:
            c0 = min(others, key=lambda c: (round(float(np.linalg.norm(xyz[c] - xyz[a])), 6), c))
            ez = xyz[c0] - xyz[a]
            others = [c for c in others if c != c0]
        else:
            ez = np.array([0., 0., 1.])
    ez = ez / np.linalg.norm(ez)
    ex = None
    for c in sorted(others, key=lambda c: (round(float(np.linalg.norm(xyz[c] - centre)), 6), c)):
        v = xyz[c] - centre
        v = v - v.dot(ez) * ez
        if np.linalg.norm(v) > 1e-3:
            ex = v / np.linalg.norm(v)
            break
    if ex is None:
        t = np.array([1., 0., 0.]) if abs(ez[0]) < 0.9 else np.array([0., 1., 0.])
        ex = t - t.dot(ez) * ez
        ex /= np.linalg.norm(ex)
    ey = np.cross(ez, ex)
    return np.stack([ex, ey, ez]), centre


_DIRS = None


def _rank(d):
    """Order of distances d (.., N), ties within 1e-6 A broken by atom index."""
    q = np.round(np.where(np.isfinite(d), d, 1e9), 6)
    idx = np.broadcast_to(np.arange(d.shape[-1]), d.shape)
    return np.lexsort((idx, q), axis=-1)


def _harmonics(l, u):
    """Real solid harmonics of degree l (basis order) at directions u (n, 3)."""
    pw = gto.cart_powers(l)
    mono = np.stack([u[:, 0] ** a * u[:, 1] ** b * u[:, 2] ** c for a, b, c in pw], axis=1)
    return mono @ gto.cart2sph(l)


def shell_rotation(l, R):
    """U_l for the frame rotation R (local = R @ global)."""
    global _DIRS
    if l == 0:
        return np.ones((1, 1))
    if _DIRS is None:
        rng = np.random.default_rng(12345)
        d = rng.normal(size=(64, 3))
        _DIRS = d / np.linalg.norm(d, axis=1)[:, None]
    A = _harmonics(l, _DIRS)
    B = _harmonics(l, _DIRS @ R)        # rows: Y(R^T u_k)
    U, *_ = np.linalg.lstsq(A, B, rcond=None)
    return U


def atom_shell_ls(mol, a):
    """Angular momentum of each AO shell block of atom a (one per contraction)."""
    ls = []
    for i in range(mol.nbas):
        if mol.bas_atom(i) == a:
            ls += [mol.bas_angular(i)] * mol.bas_nctr(i)
    return ls


def atom_rotation(mol, a, R, cache=None):
    ls = atom_shell_ls(mol, a)
    blocks = [shell_rotation(l, R) for l in ls]
    n = sum(b.shape[0] for b in blocks)
    U = np.zeros((n, n))
    o = 0
    for b in blocks:
        k = b.shape[0]
        U[o:o + k, o:o + k] = b
        o += k
    return U


def pair_features(mol, a, b, xyz=None):
    """FEAT_DIM features and the frame of pair (a, b)."""
    xyz = mol.atom_coords() * ANG if xyz is None else xyz
    syms = [t[0] for t in mol.atom]
    R, centre = local_frame(xyz, a, b)
    f = np.zeros(FEAT_DIM)
    f[pair_type(syms[a], syms[b], a == b)] = 1.
    r = np.linalg.norm(xyz[b] - xyz[a])
    f[9:25] = np.exp(-((r - RBF_CENTRES) / RBF_WIDTH) ** 2) if a != b else 0.
    others = [c for c in range(len(xyz)) if c != a and c != b]
    others.sort(key=lambda c: (round(float(np.linalg.norm(xyz[c] - centre)), 6), c))
    for k, c in enumerate(others[:4]):
        loc = R @ (xyz[c] - centre) / 3.
        f[25 + 5 * k:28 + 5 * k] = loc
        f[28 + 5 * k] = 1. if syms[c] == 'H' else 0.
        f[29 + 5 * k] = 0. if syms[c] == 'H' else 1.
    for j, x in enumerate((a, b)):
        d = np.linalg.norm(xyz - xyz[x], axis=1)
        near = (d < 3.5) & (d > 1e-8)
        nh = sum(1 for c in np.flatnonzero(near) if syms[c] == 'H')
        f[45 + 2 * j] = nh / 4.
        f[46 + 2 * j] = (near.sum() - nh) / 4.
    return f, R


# ---------------------------------------------------------------------------
# vectorised versions (all pairs of a molecule at once)

_AINV = {}


def _ainv(l):
    global _DIRS
    if _DIRS is None:
        shell_rotation(1, np.eye(3))
    if l not in _AINV:
        _AINV[l] = np.linalg.pinv(_harmonics(l, _DIRS))
    return _AINV[l]


def shell_rotations(l, R):
    """U_l for a stack of frames R (P, 3, 3) -> (P, 2l+1, 2l+1)."""
    P = len(R)
    if l == 0:
        return np.ones((P, 1, 1))
    if l == 1:
        return R.copy()
    ainv = _ainv(l)                                     # also sets up _DIRS
    u = np.einsum('kd,pde->pke', _DIRS, R)            # rows (R^T u_k)^T
    pw = gto.cart_powers(l)
    mono = np.stack([u[..., 0] ** a * u[..., 1] ** b * u[..., 2] ** c for a, b, c in pw], axis=-1)
    B = mono @ gto.cart2sph(l)                          # (P, K, 2l+1)
    return np.einsum('mk,pkn->pmn', ainv, B)


def frames_all(xyz, pairs):
    """Frames (P, 3, 3) and centres (P, 3) of all pairs, same rules as local_frame."""
    pairs = np.asarray(pairs)
    a, b = pairs[:, 0], pairs[:, 1]
    P, N = len(pairs), len(xyz)
    centre = 0.5 * (xyz[a] + xyz[b])
    onsite = a == b
    excl = np.zeros((P, N), bool)
    excl[np.arange(P), a] = True
    excl[np.arange(P), b] = True
    ez = xyz[b] - xyz[a]
    if onsite.any():
        d = np.linalg.norm(xyz[None, :, :] - xyz[a[onsite]][:, None, :], axis=2)
        d[np.arange(onsite.sum()), a[onsite]] = np.inf
        if N > 1:
            c0 = _rank(d)[:, 0]
            ez[onsite] = xyz[c0] - xyz[a[onsite]]
            excl[np.flatnonzero(onsite), c0] = True
        else:
            ez[onsite] = np.array([0., 0., 1.])
    ez = ez / np.linalg.norm(ez, axis=1)[:, None]
    dc = np.linalg.norm(xyz[None, :, :] - centre[:, None, :], axis=2)
    dc[excl] = np.inf
    order = _rank(dc)[:, :min(8, N)]
    ex = np.zeros((P, 3))
    found = np.zeros(P, bool)
    for j in range(order.shape[1]):
        c = order[:, j]
        ok = np.isfinite(dc[np.arange(P), c]) & ~found
        v = xyz[c] - centre
        v = v - np.sum(v * ez, axis=1)[:, None] * ez
        nv = np.linalg.norm(v, axis=1)
        ok &= nv > 1e-3
        ex[ok] = v[ok] / nv[ok][:, None]
        found |= ok
    for p in np.flatnonzero(~found):
        t = np.array([1., 0., 0.]) if abs(ez[p, 0]) < 0.9 else np.array([0., 1., 0.])
        t = t - t.dot(ez[p]) * ez[p]
        ex[p] = t / np.linalg.norm(t)
    ey = np.cross(ez, ex)
    return np.stack([ex, ey, ez], axis=1), centre


def features_all(mol, pairs, xyz=None):
    """(P, FEAT_DIM) features and (P, 3, 3) frames of all pairs."""
    xyz = mol.atom_coords() * ANG if xyz is None else xyz
    syms = np.array([t[0] for t in mol.atom])
    pairs = np.asarray(pairs)
    a, b = pairs[:, 0], pairs[:, 1]
    P, N = len(pairs), len(xyz)
    R, centre = frames_all(xyz, pairs)
    f = np.zeros((P, FEAT_DIM))
    types = [pair_type(syms[i], syms[j], i == j) for i, j in pairs]
    f[np.arange(P), types] = 1.
    r = np.linalg.norm(xyz[b] - xyz[a], axis=1)
    rbf = np.exp(-((r[:, None] - RBF_CENTRES[None]) / RBF_WIDTH) ** 2)
    rbf[a == b] = 0.
    f[:, 9:25] = rbf
    dc = np.linalg.norm(xyz[None, :, :] - centre[:, None, :], axis=2)
    dc[np.arange(P), a] = np.inf
    dc[np.arange(P), b] = np.inf
    near = _rank(dc)[:, :min(4, N)]
    isH = syms == 'H'
    for k in range(near.shape[1]):
        c = near[:, k]
        valid = np.isfinite(dc[np.arange(P), c])
        loc = np.einsum('pij,pj->pi', R, xyz[c] - centre) / 3.
        f[valid, 25 + 5 * k:28 + 5 * k] = loc[valid]
        f[valid, 28 + 5 * k] = isH[c][valid]
        f[valid, 29 + 5 * k] = ~isH[c][valid]
    d = np.linalg.norm(xyz[:, None, :] - xyz[None, :, :], axis=2)
    nearm = (d < 3.5) & (d > 1e-8)
    nh = (nearm & isH[None, :]).sum(1)
    nheavy = (nearm & ~isH[None, :]).sum(1)
    f[:, 45] = nh[a] / 4.
    f[:, 46] = nheavy[a] / 4.
    f[:, 47] = nh[b] / 4.
    f[:, 48] = nheavy[b] / 4.
    return f, R


def atom_rotations(mol, atoms, R):
    """Block-diagonal AO rotations (P, n, n) of atoms (all of one element)."""
    ls = atom_shell_ls(mol, int(atoms[0]))
    n = sum(2 * l + 1 for l in ls)
    U = np.zeros((len(R), n, n))
    cache = {}
    o = 0
    for l in ls:
        if l not in cache:
            cache[l] = shell_rotations(l, R)
        k = 2 * l + 1
        U[:, o:o + k, o:o + k] = cache[l]
        o += k
    return U
