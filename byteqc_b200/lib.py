"""Loader of the CUDA library (the counterpart of cuobc/lib/__init__.py:41-42).

The engine has no CPU path: if ``libbyteqc_b200.so`` is missing or cannot be
loaded, every entry point raises instead of falling back.
"""
import ctypes
import os

from .gto.mole import BAS_SLOTS  # noqa: F401  (layout constants re-exported)

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, 'libbyteqc_b200.so')

_lib = None

# exported symbols, as declared in include/byteqc_b200.h
SYMBOLS = ('GINTinit_basis_prod_cpu', 'GINTinit_basis_prod_gpu', 'GINTdel_basis_prod',
           'GINTbuild_jk', 'GINTfill_int2e', 'BQCbuild_jk', 'BQCbuild_jk_mol', 'BQCbuild_jk_class', 'BQCcount_quartets',
           'BQCfp64_fma_peak', 'BQCdm_cond', 'BQCschwarz', 'BQCint1e', 'BQClaunch_counter',
           'BQCbuild_jk_noalloc', 'BQCmlp_linear_fwd', 'BQCmlp_linear_bwd', 'BQCmlp_adam',
           'BQCmlp_to_bf16', 'BQCset_class_variant', 'BQCversion', 'BQCplan_create',
           'BQCplan_destroy', 'BQCbuild_jk_plan')


def load_library(name='libbyteqc_b200'):
    """Load the engine library; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError('%s is not built: run byteqc_b200.build.build() '
                           '(the J/K engine has no CPU fallback)' % LIBPATH)
    lib = ctypes.CDLL(LIBPATH)
    lib.BQCversion.restype = ctypes.c_char_p
    lib.BQClaunch_counter.restype = ctypes.c_ulonglong
    for fn in ('GINTbuild_jk', 'BQCbuild_jk', 'BQCdm_cond', 'BQCschwarz', 'BQCint1e'):
        getattr(lib, fn).restype = ctypes.c_int
    # double arguments must be declared where a bare Python float is passed
    lib.BQCbuild_jk.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 3 + \
        [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
         ctypes.c_void_p]
    lib.BQCbuild_jk_class.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + \
        [ctypes.c_void_p] * 3 + [ctypes.c_double] + [ctypes.c_void_p] * 3 + \
        [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
         ctypes.c_void_p]
    lib.BQCcount_quartets.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + \
        [ctypes.c_void_p] * 3 + [ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                 ctypes.c_void_p]
    lib.BQCbuild_jk_noalloc.restype = ctypes.c_int
    lib.BQCplan_create.restype = ctypes.c_int
    lib.BQCplan_create.argtypes = [ctypes.c_void_p] * 4
    lib.BQCplan_destroy.restype = None
    lib.BQCplan_destroy.argtypes = [ctypes.c_void_p]
    lib.BQCbuild_jk_plan.restype = ctypes.c_int
    lib.BQCbuild_jk_plan.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                              ctypes.c_double, ctypes.c_void_p]
    lib.BQCbuild_jk_mol.restype = ctypes.c_int
    lib.BQCbuild_jk_mol.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_double] + \
        [ctypes.c_void_p] * 3 + [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_void_p, ctypes.c_void_p]
    vp, ci, cf = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    lib.BQCmlp_linear_fwd.argtypes = [vp] * 6 + [ci] * 4 + [vp]
    lib.BQCmlp_linear_bwd.argtypes = [vp] * 8 + [ci] * 3 + [vp]
    lib.BQCmlp_adam.argtypes = [vp] * 5 + [ci, cf, cf, cf, cf, ci, vp]
    lib.BQCmlp_to_bf16.argtypes = [vp, vp, ctypes.c_size_t, vp]
    lib.GINTinit_basis_prod_cpu.restype = None
    lib.GINTinit_basis_prod_gpu.restype = None
    lib.GINTdel_basis_prod.restype = None
    _lib = lib
    return lib


class ContractionProdType(ctypes.Structure):
    """Layout of cuobc/lib/gint/gint.h:101-107."""
    _fields_ = [
        ('l_bra', ctypes.c_int),
        ('l_ket', ctypes.c_int),
        ('nprim_12', ctypes.c_int),
        ('npairs', ctypes.c_int),
    ]


class BasisProdCache(ctypes.Structure):
    """Layout of cuobc/lib/gint/gint.h:118-147."""
    _fields_ = [
        ('nbas', ctypes.c_int),
        ('ncptype', ctypes.c_int),
        ('cptype', ctypes.POINTER(ContractionProdType)),
        ('bas_pairs_locs', ctypes.POINTER(ctypes.c_int)),
        ('primitive_pairs_locs', ctypes.POINTER(ctypes.c_int)),
        ('bas_pair2shls', ctypes.POINTER(ctypes.c_int)),
        ('aexyz', ctypes.POINTER(ctypes.c_double)),
        ('bas_coords', ctypes.POINTER(ctypes.c_double)),
        ('bas_pair2bra', ctypes.POINTER(ctypes.c_int)),
        ('bas_pair2ket', ctypes.POINTER(ctypes.c_int)),
        ('ao_loc', ctypes.POINTER(ctypes.c_int)),
        ('a12', ctypes.POINTER(ctypes.c_double)),
        ('e12', ctypes.POINTER(ctypes.c_double)),
        ('x12', ctypes.POINTER(ctypes.c_double)),
        ('y12', ctypes.POINTER(ctypes.c_double)),
        ('z12', ctypes.POINTER(ctypes.c_double)),
    ]
