"""cuphu_b200 -- B200-native (sm_100a) cuPHU unwrapping path.

Drop-in for ``cuphu.unwrap(igram, corr, nlooks, init='laplace', ...)`` and
``cuphu.io.InputDataset/OutputDataset``: statistical-cost weights, residues,
the IRLS-reweighted Jacobi-PCG Laplace solve, tile stitching, connected
components and flow integration run as hand-written CUDA kernels in
``lib/libcuphu_b200.so`` behind the C ABI of ``include/cuphu_b200.h``.
"""
from cuphu_b200._conncomp import regrow_conncomp
from cuphu_b200._gpu import gpu_count, gpu_info, gpu_name
from cuphu_b200._looks import get_effective_looks
from cuphu_b200._tune import autotune
from cuphu_b200._unwrap import unwrap

__version__ = "0.1.0"

__all__ = ["__version__", "autotune", "get_effective_looks", "gpu_count", "gpu_info",
           "gpu_name", "regrow_conncomp", "unwrap"]
