"""Samples (features, local-frame targets) from converged densities, and the
assembly of a predicted density from per-pair blocks.  All pairs of a
molecule are processed at once, grouped by element pair."""
import numpy as np

from .features import ANG, OUT_DIM, atom_rotations, canonical_pairs, features_all


def _slices(mol):
    s = mol.aoslice_by_atom()
    return s[:, 2].astype(int), s[:, 3].astype(int)


class PairFrames:
    """Pairs, features and per-element-pair groups with their AO rotations."""

    def __init__(self, mol):
        self.mol = mol
        self.pairs = np.asarray(canonical_pairs(mol))
        self.feats, R = features_all(mol, self.pairs, mol.atom_coords() * ANG)
        syms = np.array([t[0] for t in mol.atom])
        key = np.array([syms[a] + '|' + syms[b] for a, b in self.pairs])
        self.groups = []
        for k in np.unique(key):
            idx = np.flatnonzero(key == k)
            a, b = self.pairs[idx, 0], self.pairs[idx, 1]
            Ua = atom_rotations(mol, a, R[idx])
            Ub = atom_rotations(mol, b, R[idx])
            self.groups.append((idx, a, b, Ua, Ub))

    def _index(self, a, b, na, nb):
        s0, _ = _slices(self.mol)
        rows = s0[a][:, None] + np.arange(na)[None, :]
        cols = s0[b][:, None] + np.arange(nb)[None, :]
        return rows[:, :, None], cols[:, None, :]


def pair_frames(mol):
    return PairFrames(mol)


def samples(mol, dm, dm_sad, out_dim=OUT_DIM, dtype=np.float64):
    """Features, targets (local-frame block minus local SAD block, padded to
    out_dim) and masks of every canonical pair of mol; the training set
    keeps them in FP32 (dtype), which is what the network trains on."""
    pf = PairFrames(mol)
    P = len(pf.pairs)
    tgt = np.zeros((P, out_dim), dtype=dtype)
    mask = np.zeros((P, out_dim), dtype=dtype)
    diff = dm - dm_sad
    for idx, a, b, Ua, Ub in pf.groups:
        na, nb = Ua.shape[1], Ub.shape[1]
        r, c = pf._index(a, b, na, nb)
        blk = diff[r, c]                                    # (G, na, nb)
        loc = np.einsum('gij,gjk,glk->gil', Ua, blk, Ub)     # U_a blk U_b^T
        tgt[idx, :na * nb] = loc.reshape(len(idx), -1)
        mask[idx, :na * nb] = 1.
    return pf.feats, tgt, mask


def assemble(mol, pf, pred, dm_sad):
    """Density from the SAD density plus the predicted local-frame residual
    blocks rotated back to the molecular frame; symmetric by construction."""
    dm = dm_sad.copy()
    for idx, a, b, Ua, Ub in pf.groups:
        na, nb = Ua.shape[1], Ub.shape[1]
        loc = pred[idx, :na * nb].reshape(len(idx), na, nb)
        blk = np.einsum('gji,gjk,gkl->gil', Ua, loc, Ub)     # U_a^T loc U_b
        r, c = pf._index(a, b, na, nb)
        on = a == b
        if on.any():
            sym = 0.5 * (blk[on] + blk[on].transpose(0, 2, 1))
            np.add.at(dm, (r[on], c[on]), sym)
        off = ~on
        if off.any():
            np.add.at(dm, (r[off], c[off]), blk[off])
            np.add.at(dm, (c[off].transpose(0, 2, 1), r[off].transpose(0, 2, 1)),
                      blk[off].transpose(0, 2, 1))
    return dm


def assemble_device(mol, pf, pred, dm_sad):
    """assemble() on the device: pred (pairs x width) and dm_sad are torch
    tensors; the blocks are rotated back with batched matrix products and
    added with one index_add per element pair."""
    import torch
    dev = dm_sad.device
    nao = dm_sad.shape[-1]
    dm = dm_sad.clone()
    flat = dm.view(-1)
    for idx, a, b, Ua, Ub in pf.groups:
        na, nb = Ua.shape[1], Ub.shape[1]
        it = torch.as_tensor(idx, device=dev)
        loc = pred[it, :na * nb].to(torch.float64).reshape(len(idx), na, nb)
        Ua_t = torch.as_tensor(Ua, dtype=torch.float64, device=dev)
        Ub_t = torch.as_tensor(Ub, dtype=torch.float64, device=dev)
        blk = Ua_t.transpose(1, 2) @ loc @ Ub_t                  # U_a^T loc U_b
        r, c = pf._index(a, b, na, nb)
        lin = torch.as_tensor((r * nao + c).astype(np.int64), device=dev)       # (G, na, nb)
        lin_t = torch.as_tensor((c * nao + r).astype(np.int64), device=dev)
        on = torch.as_tensor(a == b, device=dev)
        if bool((a == b).any()):
            sym = 0.5 * (blk[on] + blk[on].transpose(1, 2))
            flat.index_add_(0, lin[on].reshape(-1), sym.reshape(-1))
        off = ~on
        if bool((a != b).any()):
            flat.index_add_(0, lin[off].reshape(-1), blk[off].reshape(-1))
            flat.index_add_(0, lin_t[off].reshape(-1), blk[off].reshape(-1))
    return dm
