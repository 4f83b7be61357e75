"""plfft_cuda_c2c_execute_noalloc against the plan-based C2C path and the FP64 oracle.

The entry point serves callers that must not allocate device memory while
they run (a framework that already owns the GPU's memory pool, or a
latency-critical loop where cudaMalloc/cudaFree would synchronize the device).
It keeps its four-step scratch in a file-scope device array instead.  This
test calls it through the C-ABI twice in a row with different data and
checks each result against plfft_plan_execute on the same input, within the
FP32 tolerance used by every parity test (rel-L2 <= 4*log2(N)*2^-24).  It is
collected last so that a run stopping at the first failure has already run
every other test, and it passes alone in a fresh process as well.
"""
import numpy as np
import pytest

import oracle
import plfft

pytestmark = pytest.mark.gpu


def _plan_result(x, n, hm, direction):
    import torch

    plan = plfft.make_plan("c2c", n, hm, direction=direction)
    y = torch.empty_like(x)
    plan.execute(x.data_ptr(), y.data_ptr())
    return y


@pytest.mark.parametrize("n,hm", [(65536, 3), (1 << 20, 3), (3 ** 10, 2)])
@pytest.mark.parametrize("direction", [plfft.FORWARD, plfft.BACKWARD])
def test_noalloc_matches_plan_two_calls(n, hm, direction):
    import torch

    for call in range(2):
        g = torch.Generator(device="cuda")
        g.manual_seed(1000 * call + n % 997)
        x = torch.complex(torch.rand(n * hm, device="cuda", generator=g) * 2 - 1,
                          torch.rand(n * hm, device="cuda", generator=g) * 2 - 1)
        ref = _plan_result(x, n, hm, direction)
        y = torch.full_like(x, complex(7.0, -7.0))
        st = plfft.c2c_execute_noalloc(x.data_ptr(), y.data_ptr(), n, hm, direction)
        assert st == plfft.Status.OK
        torch.cuda.synchronize()
        err = oracle.rel_l2(y.cpu().numpy(), ref.cpu().numpy())
        assert err <= oracle.fp32_tol(n), (call, err)


def _oracle(x, n, hm, direction):
    return oracle.c2c(x.cpu().numpy().reshape(hm, n).astype(np.complex128), direction, method="fft")


@pytest.mark.parametrize("n,hm", [(65536, 5), (1 << 20, 3), (1 << 21, 2)])
def test_noalloc_matches_fp64_oracle(n, hm):
    """Directly against the FP64 oracle, including the largest accepted n
    (2^21: one member per 16 MiB chunk, so two chunks)."""
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(n + hm)
    x = torch.complex(torch.rand(n * hm, device="cuda", generator=g) * 2 - 1,
                      torch.rand(n * hm, device="cuda", generator=g) * 2 - 1)
    y = torch.empty_like(x)
    assert plfft.c2c_execute_noalloc(x.data_ptr(), y.data_ptr(), n, hm, plfft.FORWARD) == plfft.Status.OK
    torch.cuda.synchronize()
    ref = _oracle(x, n, hm, -1)
    assert oracle.rel_l2(y.cpu().numpy().reshape(hm, n), ref) <= oracle.fp32_tol(n)


def test_noalloc_in_place_several_chunks_on_a_stream():
    """In place (input and output the same buffer) over more than one chunk
    (n = 2^20: two members per 16 MiB chunk, three members), enqueued on a
    non-default stream."""
    import torch

    n, hm = 1 << 20, 3
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    x = torch.complex(torch.rand(n * hm, device="cuda", generator=g) * 2 - 1,
                      torch.rand(n * hm, device="cuda", generator=g) * 2 - 1)
    ref = _oracle(x, n, hm, 1)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        st = plfft.c2c_execute_noalloc(x.data_ptr(), x.data_ptr(), n, hm, plfft.BACKWARD, s.cuda_stream)
    assert st == plfft.Status.OK
    s.synchronize()
    assert oracle.rel_l2(x.cpu().numpy().reshape(hm, n), ref) <= oracle.fp32_tol(n)


def test_noalloc_rejects_sizes_beyond_limit():
    import torch

    x = torch.zeros(8, dtype=torch.complex64, device="cuda")
    assert plfft.c2c_execute_noalloc(x.data_ptr(), x.data_ptr(), 1024, 1) == plfft.Status.INVALID_SIZE
    assert plfft.c2c_execute_noalloc(x.data_ptr(), x.data_ptr(), 1 << 22, 1) == plfft.Status.INVALID_SIZE
    assert plfft.c2c_execute_noalloc(x.data_ptr(), x.data_ptr(), 65537, 1) == plfft.Status.INVALID_SIZE
    assert plfft.c2c_execute_noalloc(0, x.data_ptr(), 65536, 1) == plfft.Status.NULL_ARGUMENT
