"""B200-native blind-rotation engine for Toothpaste's CGGI/BMMP path.

The compute path is hand-written sm_100a CUDA behind the C ABI declared in
include/toothpaste_gpu.h (libtoothpaste_gpu.so, built in-tree by build.py).
"""
from ._native import GOLDILOCKS, TP_BR_BMMP_BINARY, TP_BR_CGGI_BINARY, TP_BR_CGGI_TERNARY, TpError  # noqa: F401
from .blind_rotation import (BatchGraph, BlindRotationContext, GpuBlindRotator, NegacyclicFunctionEvaluator,  # noqa: F401
                             ntt_backward, ntt_forward, sample_extract_batch)
from .key_switching import (GpuAutomorphismEvaluator, GpuLWEtoLWEConverter, GpuLWEtoRLWEPacker,  # noqa: F401,E402
                            GpuRLWEtoRLWEConverter, GpuTraceEvaluator, modulus_switch_batch)
from .sap import GpuSAPDecomposer  # noqa: F401,E402
from .scheme_switching import GpuLWEtoRGSWConverter  # noqa: F401,E402
from .serving import BootstrapServer  # noqa: F401,E402
