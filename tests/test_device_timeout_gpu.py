"""Device-side timeouts are reported to the host, and the plan stays usable.

Every wait of the power-of-two kernels on a bulk copy is bounded in time;
when the bound runs out the CTA records PLFFT_DEVICE_TIMEOUT in its plan's
host-mapped status word, lets the copies it did issue land, and returns.
The test makes one wait run out without any fault: with the test hook
PLFFT_B200_TEST_STALL_CTA set at plan creation, one CTA of the plan's first
run issues none of its loads, so its barrier never completes and its wait
(shortened to PLFFT_B200_TEST_WAIT_US) gives up while nothing is in flight.
The host must report the timeout -- through plfft_cuda_get_last_status()
for plfft_plan_execute and through plfft_cuda_plan_get_device_status() for
stream-ordered execution -- and the next execution of the same plan must be
correct.
"""
import numpy as np
import pytest

import oracle
import plfft

pytestmark = pytest.mark.gpu

N, HOWMANY = 1024, 4096


@pytest.fixture
def stalled(monkeypatch):
    monkeypatch.setenv("PLFFT_B200_TEST_STALL_CTA", "5")
    monkeypatch.setenv("PLFFT_B200_TEST_WAIT_US", "3000")


def _data():
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    return torch.complex(torch.rand(N * HOWMANY, device="cuda", generator=g) * 2 - 1,
                         torch.rand(N * HOWMANY, device="cuda", generator=g) * 2 - 1)


def _check(x, y):
    ref = oracle.c2c(x.cpu().numpy().reshape(HOWMANY, N).astype(np.complex128), -1, method="fft")
    assert oracle.rel_l2(y.cpu().numpy().reshape(HOWMANY, N), ref) <= oracle.fp32_tol(N)


def test_timeout_reported_by_plan_execute(stalled):
    import torch

    plan = plfft.make_plan("c2c", N, HOWMANY)
    assert "c2c-pow2" in plan.describe(), plan.describe()
    x = _data()
    y = torch.zeros_like(x)
    with pytest.raises(plfft.PlfftError) as e:
        plan.execute(x.data_ptr(), y.data_ptr())
    assert e.value.status == plfft.Status.DEVICE_TIMEOUT
    # the context is intact and the plan runs normally afterwards
    y.zero_()
    plan.execute(x.data_ptr(), y.data_ptr())
    _check(x, y)


def test_timeout_reported_for_stream_ordered_execution(stalled):
    import torch

    plan = plfft.make_plan("c2c", N, HOWMANY)
    x = _data()
    y = torch.zeros_like(x)
    s = torch.cuda.Stream()
    plan.execute_async(x.data_ptr(), y.data_ptr(), 0, s.cuda_stream)
    assert plan.device_status(s.cuda_stream) == plfft.Status.DEVICE_TIMEOUT
    # reading the status cleared it; a clean run reports OK
    assert plan.device_status(s.cuda_stream) == plfft.Status.OK
    plan.execute_async(x.data_ptr(), y.data_ptr(), 0, s.cuda_stream)
    assert plan.device_status(s.cuda_stream) == plfft.Status.OK
    _check(x, y)


def test_no_timeout_without_the_hook():
    import torch

    plan = plfft.make_plan("c2c", N, HOWMANY)
    x = _data()
    y = torch.empty_like(x)
    for _ in range(3):
        plan.execute_async(x.data_ptr(), y.data_ptr())
    assert plan.device_status() == plfft.Status.OK
    plan.execute(x.data_ptr(), y.data_ptr())
    _check(x, y)
