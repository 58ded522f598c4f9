"""pspaqr_public_b200 -- B200-native factorize-and-solve path of pspaQR.

Sparsified QR (spaQR) preconditioner + GMRES: host nested-dissection ordering
and symbolic structure in C++, FP64 tile QR / RRQR sparsification /
preconditioner apply as hand-written sm_100a kernels, all behind the C ABI in
``include/spaqr_b200.h``.
"""
from .tree import ParTree, SpqError, dist_gmres, random_reference, scale_columns  # noqa: F401

__all__ = ["ParTree", "SpqError", "dist_gmres", "random_reference", "scale_columns"]
