"""Initial density from the trained MLP (SAD plus predicted pair blocks)."""
import os

import numpy as np
import torch

from . import dataset
from .model import DensityMLP

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, 'weights_ccpvdz.npz')
# trained models per basis shape
WEIGHTS = {'cc-pvdz': DEFAULT_WEIGHTS, 'cc-pvtz': os.path.join(HERE, 'weights_ccpvtz.npz')}
_MODELS = {}


def weights_for(mol):
    """The trained weights for the basis shape of mol (mol.basis_name, the
    cc-pVDZ shape when it is not set), or None when none was trained."""
    path = WEIGHTS.get(getattr(mol, 'basis_name', 'cc-pvdz'))
    return path if path is not None and os.path.exists(path) else None


def load_model(path=DEFAULT_WEIGHTS):
    if path not in _MODELS:
        if not os.path.exists(path):
            raise FileNotFoundError('no trained density model at %s' % path)
        _MODELS[path] = DensityMLP().load(dict(np.load(path)))
    return _MODELS[path]


def mlp_density(mf, dm_sad=None, path=DEFAULT_WEIGHTS):
    """Predicted AO density (device tensor) for the molecule of mf."""
    from ..scf.guess import init_guess
    mol = mf.mol
    if dm_sad is None:
        dm_sad = init_guess(mf, 'sad')
    model = load_model(path)
    pf = dataset.pair_frames(mol)
    pred = model.predict(pf.feats)
    dm = dataset.assemble_device(mol, pf, pred, dm_sad)
    ne = float(torch.sum(dm * mf.get_ovlp()))
    if ne > 0:
        dm *= mol.nelectron / ne
    return dm
