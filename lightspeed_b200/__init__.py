"""lightspeed_b200 -- a B200 (sm_100a) engine for the Lightspeed IntBox
Coulomb/exchange (J/K) path.

`import lightspeed_b200 as ls` gives the reference's names for that path:
ls.Tensor, ls.Primitive, ls.Basis (with Basis.from_gbs_file), ls.PairList,
ls.Ewald, ls.ResourceList, ls.IntBox.coulomb / ls.IntBox.exchange, and
ls.Molecule. J and K always run on the GPU through liblsjk.so; there is no
CPU path, and the first call that needs the device fails loudly without one.
"""
import os as _os

from ._lightspeed import (Tensor, Primitive, Basis, Pair, PairListL, PairList, Ewald, ResourceList, IntBox,
                          PREC_MIXED, PREC_FP64, set_precision, get_precision, stats, reset_stats,
                          engine_version, stream_handle, fma_peak_tflops, coulomb_device, exchange_device,
                          graph_begin, graph_end, Graph, class_counts, Stream, flops_split,
                          set_autotune, get_tune_table, set_tune_table, set_merge, get_merge)
from .molecule import Atom, Molecule, units
from . import gbs as _gbs

_PKG_DIR = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_PKG_DIR, "liblsjk.so")


def _basis_from_gbs_file(molecule, filename, normalize=True, spherical=None):
    import sys
    return _gbs.basis_from_gbs_file(sys.modules[__name__], molecule, filename, normalize=normalize,
                                    spherical=spherical)


def _basis_from_gbs_lines(molecule, lines, name="bas", normalize=True, spherical=None):
    import sys
    return _gbs.basis_from_gbs_lines(sys.modules[__name__], molecule, lines, name=name, normalize=normalize,
                                     spherical=spherical)


def _basis_from_gbs_str(molecule, strval, **kwargs):
    return _basis_from_gbs_lines(molecule, strval.split("\n"), **kwargs)


Basis.from_gbs_file = staticmethod(_basis_from_gbs_file)
Basis.from_gbs_lines = staticmethod(_basis_from_gbs_lines)
Basis.from_gbs_str = staticmethod(_basis_from_gbs_str)
Basis.basisdir = _gbs.BASIS_DIR

__all__ = ["Tensor", "Primitive", "Basis", "Pair", "PairListL", "PairList", "Ewald", "ResourceList", "IntBox",
           "Atom", "Molecule", "units", "PREC_MIXED", "PREC_FP64", "set_precision", "get_precision", "stats",
           "reset_stats", "engine_version", "set_merge", "get_merge", "LIB_PATH"]
