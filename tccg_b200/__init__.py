"""tccg_b200: a B200-native tensor-contraction generator with TCCG's surface.

``C = alpha * A * B + beta * C`` for column-major tensors described in TCCG's
``.tccg`` format, computed by hand-written sm_100a CUDA kernels (tcgen05/TMA
for BF16 and split-BF16x3, CUDA cores for FP32/FP64) behind a C ABI
(include/tccg_b200.h).
"""
from .spec import (Contraction, Index, Tensor, TccgSyntaxError, TccgUnsupported, fuse_indices,
                   make_contraction, parse_file, parse_text, to_tccg_text)

from .api import Compiled, compile, contract
from .autograd import GettFunction, grad_contractions
from .plan import Plan, Tuning

__version__ = "0.1.0"

__all__ = ["Contraction", "Index", "Tensor", "TccgSyntaxError", "TccgUnsupported",
           "fuse_indices", "make_contraction", "parse_file", "parse_text", "to_tccg_text",
           "Compiled", "compile", "contract", "GettFunction", "grad_contractions", "Plan",
           "Tuning"]
