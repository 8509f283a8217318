"""The gravity surrogate's tensor-core kernels against PyTorch FP32 references
of the same operations on the same BF16-rounded values."""
import ctypes as C

import numpy as np
import pytest

from bqp_b200 import _native as N

pytestmark = pytest.mark.gpu


def _gemm(a_bf16, b_bf16):
    import torch
    m, k = a_bf16.shape
    n = b_bf16.shape[0]
    c = torch.empty((m, n), dtype=torch.float32, device="cuda")
    N.check(N.lib().bqp_gemm_bf16_device(m, n, k, C.c_void_p(a_bf16.data_ptr()), C.c_void_p(b_bf16.data_ptr()),
                                         C.c_void_p(c.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return c


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (256, 512, 256), (1024, 256, 1024)])
def test_tensor_core_gemm_matches_fp32_reference(m, n, k):
    import torch
    g = torch.Generator().manual_seed(m + n + k)
    a = torch.randn(m, k, generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(torch.bfloat16)
    ref = a.float() @ b.float().T  # FP32 products of the BF16 values
    got = _gemm(a.cuda(), b.cuda()).cpu()
    err = (got - ref).abs().max().item()
    # FP32 accumulation in a different order: a few ulp of the partial sums
    assert err <= 1e-5 * np.sqrt(k) * ref.abs().max().item() + 1e-5, err
    # and not a trivially wrong layout: every element checked, signs too
    assert torch.allclose(got, ref, rtol=1e-4, atol=1e-3)
