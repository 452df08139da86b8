"""
zkgpu — the BN254 prover hot path of the reference's zkgpu package, rebuilt
for NVIDIA B200 (sm_100a).

The public modules keep the reference's names and behaviour, so they are a
drop-in for its GPU calls:

- zkgpu.field256_gpu : Field256, BN254_FR, BN254_FQ (Montgomery mul/add/sub, NTT)
- zkgpu.curve_gpu    : G1 add / add_affine / double and conversions
- zkgpu.msm_gpu      : msm_pippenger_gpu
- zkgpu.curve        : Point, the affine point value these return

All arithmetic runs in libzkb200.so (hand-written sm_100a CUDA behind a C
ABI, include/zkb200.h), called through ctypes with torch tensors as device
buffers. There is no CPU fallback: without a CUDA device the operations
raise RuntimeError. Importing the package needs neither a GPU nor the
library; the first operation loads both.
"""

from zkgpu.curve import JACOBIAN_IDENTITY, G, P, Point, R
from zkgpu.field256_gpu import BN254_FQ, BN254_FR, LIMBS, Field256
from zkgpu.msm_gpu import msm_pippenger_gpu, msm_pippenger_rows, pippenger_window_size

__all__ = [
    "BN254_FQ",
    "BN254_FR",
    "G",
    "JACOBIAN_IDENTITY",
    "LIMBS",
    "P",
    "Point",
    "R",
    "Field256",
    "msm_pippenger_gpu",
    "msm_pippenger_rows",
    "pippenger_window_size",
]
