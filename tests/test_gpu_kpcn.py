"""The learned denoiser's tensor-core kernels against FP32/FP64 references on the CPU."""
from __future__ import annotations

import numpy as np
import pytest

from webgpuraytracer_b200 import _lib

pytestmark = pytest.mark.gpu


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def bf16_value(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("m,n,k", [(128, 32, 64), (300, 96, 200), (257, 16, 8), (1000, 256, 576), (64, 200, 1232)])
def test_tc_gemm_matches_fp32(m, n, k):
    rng = np.random.default_rng(m * 7 + n + k)
    a = bf16_bits(rng.standard_normal((m, k)).astype(np.float32))
    b = bf16_bits(rng.standard_normal((n, k)).astype(np.float32))
    c = np.zeros((m, n), np.float32)
    L = _lib.lib()
    rc = L.wgpt_gemm_bf16(0, _lib.ptr(a), _lib.ptr(b), _lib.ptr(c), m, n, k)
    assert rc == 0, _lib.STATUS_NAMES.get(rc, rc)
    ref = bf16_value(a).astype(np.float64) @ bf16_value(b).astype(np.float64).T
    err = np.abs(c - ref)
    # FP32 accumulation of k products of BF16 values (exact in FP32): rounding only
    tol = 1e-5 * np.sqrt(k) * np.abs(bf16_value(a)).max() * np.abs(bf16_value(b)).max() * 4
    assert err.max() <= max(tol, 1e-4), f"max abs error {err.max()} (tol {tol})"
