"""polybin3d_b200 — B200-native (sm_100a) binned polyspectrum hot path of PolyBin3D.

Drop-in for `pb.PolyBin3D(..., backend='cuda')`, `pb.PSpec`, `pb.BSpec`:
Pk_ideal, Pk_unwindowed, Bk_ideal, Bk_unwindowed and compute_fisher keep the reference's
signatures and return layouts.  Host: Python on torch tensors; compute: hand-written CUDA
behind the C ABI in include/polybin3d_b200.h (libpb_b200.so).
"""
from .base import PolyBin3D
from .pspec import PSpec
from .bspec import BSpec

__all__ = ["PolyBin3D", "PSpec", "BSpec"]
