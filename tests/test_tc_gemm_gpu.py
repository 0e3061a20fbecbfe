"""tcgen05 TF32 GEMM (C -= A B) against an FP64 numpy product.

TF32 keeps 10 mantissa bits of each operand, so the tolerance is relative
to sum |A||B| per entry: 2^-10 (plus FP32 accumulation).

Shapes whose leading dimensions are multiples of 4 floats run the TMA-fed
pipelined kernel (128 x 256 tiles, 4 stages: k > 128 wraps the stage ring);
the others run the register-staged kernel."""
import ctypes as C

import numpy as np
import pytest
import torch

from dust_b200._lib import check, lib

pytestmark = pytest.mark.gpu


def run(m, n, k, seed):
    g = torch.Generator().manual_seed(seed)
    A = torch.randn(m, k, generator=g, dtype=torch.float32)
    B = torch.randn(k, n, generator=g, dtype=torch.float32)
    C0 = torch.randn(m, n, generator=g, dtype=torch.float32)
    # column-major device copies: store transposes row-major
    dA = A.t().contiguous().cuda()
    dB = B.t().contiguous().cuda()
    dC = C0.t().contiguous().cuda()
    p = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float))
    s = torch.cuda.current_stream().cuda_stream
    check(lib().dust_tc_gemm_tf32_minus(m, n, k, p(dA), m, p(dB), k, p(dC), m, C.c_void_p(s)),
          "dust_tc_gemm_tf32_minus")
    got = dC.cpu().t().double().numpy()
    ref = C0.double().numpy() - A.double().numpy() @ B.double().numpy()
    scale = np.abs(A.double().numpy()) @ np.abs(B.double().numpy()) + 1.0
    return np.max(np.abs(got - ref) / scale)


@pytest.mark.parametrize("m,n,k", [(128, 128, 32), (256, 384, 64), (200, 130, 70),
                                   (1000, 700, 256), (64, 33, 5), (300, 520, 1000),
                                   (128, 256, 4096), (513, 257, 96), (4, 8, 12)])
def test_tc_gemm_matches_fp64(m, n, k):
    err = run(m, n, k, seed=m + n + k)
    assert err < 2.0 ** -9
