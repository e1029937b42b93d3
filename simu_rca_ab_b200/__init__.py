"""simu_rca_ab_b200: a B200 (sm_100a) row-column-array delay-and-sum I/Q beamformer.

Drop-in for the RCA beamformer of Jeanrop/Simu_RCA_ab
(MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.{m,cu}) with the
``Python/beamformer`` call style.  The compute path is librcabf.so (C ABI in
include/rcabf.h, hand-written CUDA for sm_100a); this package is its host
binding.
"""
from .params import RCAError, RCAWarning, normalize  # noqa: F401

__all__ = ["bf_rca", "bf_rca_nosum", "BfIQRCA", "Engine", "RCAError", "RCAWarning", "normalize"]


def __getattr__(name):
    # the CUDA-backed names load librcabf on first use
    if name in ("bf_rca", "bf_rca_nosum", "BfIQRCA", "Engine", "default_engine", "GeometryHandle"):
        from . import beamformer
        return getattr(beamformer, name)
    raise AttributeError(name)
