"""The tcgen05 tile GEMM (tensor memory accumulator, shared-memory operands in
the core-matrix layout) against a float64 reference, for K-major and MN-major
operands.  BF16 inputs, FP32 accumulation."""
import ctypes as C

import numpy as np
import pytest

from q_psdm_b200 import _lib

pytestmark = pytest.mark.gpu


def _run(a, b, a_mn, b_mn):
    import torch
    L = _lib.lib()
    f = L.qpsdm_internal_tc_gemm
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                  C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    N, K = b.shape
    da = torch.from_numpy(a).to(torch.bfloat16).cuda()
    db = torch.from_numpy(b).to(torch.bfloat16).cuda()
    out = torch.zeros((128, N), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = f(da.data_ptr(), db.data_ptr(), out.data_ptr(), N, K, a_mn, b_mn, err.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert int(err.item()) == 0, "tensor-core wait timed out"
    ref = da.double().cpu().numpy() @ db.double().cpu().numpy().T
    return out.cpu().numpy(), ref


@pytest.mark.parametrize("N,K", [(128, 128), (16, 128), (128, 16), (64, 64), (256, 64)])
@pytest.mark.parametrize("a_mn,b_mn", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_tc_gemm(cuda, N, K, a_mn, b_mn):
    rng = np.random.default_rng(N * 1000 + K + 10 * a_mn + b_mn)
    a = rng.standard_normal((128, K)).astype(np.float32)
    b = rng.standard_normal((N, K)).astype(np.float32)
    got, ref = _run(a, b, a_mn, b_mn)
    # bf16 inputs are exact in the reference; only FP32 accumulation differs
    assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()


def test_bounded_wait_times_out_and_context_survives(cuda):
    """A tensor-core CTA waiting on an mbarrier that nothing arrives on (no
    MMA issued, nothing in flight) gives up after its limit, frees its tensor
    memory and returns: the entry point reports QPSDM_ETIMEOUT, and the next
    normal tensor-core call on the same context succeeds."""
    import time

    import torch
    L = _lib.lib()
    f = L.qpsdm_internal_tc_wait_timeout
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    assert f(2000, err.data_ptr(), None) == _lib.ETIMEOUT     # 2 ms limit
    assert time.perf_counter() - t0 < 5.0
    assert int(err.item()) == 1
    rng = np.random.default_rng(1)
    a = rng.standard_normal((128, 64)).astype(np.float32)
    b = rng.standard_normal((64, 64)).astype(np.float32)
    got, ref = _run(a, b, 0, 0)
    assert np.abs(got - ref).max() <= 1e-3 * np.abs(ref).max()
