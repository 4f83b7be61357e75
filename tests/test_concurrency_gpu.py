"""Concurrent execution of one plan (reference include/plfft.h:520-523 allows
calling plfft_plan_execute on one plan from several threads at once).

On the device this is stream-ordered execution on two streams with a
workspace each (plfft_cuda_execute_async): the two executions may overlap on
the GPU and must not share scratch.  The schedules used need workspace:
the two-pass four-step (n = 65536) and a multi-launch Bluestein convolution
(n = 4099).
On the host, two threads call plfft_plan_execute on the same plan with
their own host buffers.
"""
import threading

import numpy as np
import pytest

import oracle
import plfft

pytestmark = pytest.mark.gpu


def _rand(n, hm, seed):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.complex(torch.rand(n * hm, device="cuda", generator=g) * 2 - 1,
                         torch.rand(n * hm, device="cuda", generator=g) * 2 - 1)


@pytest.mark.parametrize("n,hm", [(65536, 24), (4099, 150)])
def test_two_streams_one_plan_own_workspaces(n, hm):
    import torch

    plan = plfft.make_plan("c2c", n, hm)
    ws_bytes = plan.workspace_size()
    assert ws_bytes > 0, plan.describe()
    xs = [_rand(n, hm, 10 + i) for i in range(2)]
    ys = [torch.empty_like(xs[0]) for _ in range(2)]
    wss = [torch.empty(ws_bytes, dtype=torch.uint8, device="cuda") for _ in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    torch.cuda.synchronize()
    for _ in range(4):  # alternate enqueues so the executions interleave
        for i in range(2):
            plan.execute_async(xs[i].data_ptr(), ys[i].data_ptr(), wss[i].data_ptr(), streams[i].cuda_stream)
    torch.cuda.synchronize()
    for i in range(2):
        ref = oracle.c2c(xs[i].cpu().numpy().reshape(hm, n).astype(np.complex128), -1, method="fft")
        assert oracle.rel_l2(ys[i].cpu().numpy().reshape(hm, n), ref) <= oracle.fp32_tol(n), (i, plan.describe())


def test_two_host_threads_one_plan():
    n, hm = 4096, 256
    plan = plfft.make_plan("c2c", n, hm)
    rng = np.random.default_rng(3)
    xs = [(rng.uniform(-1, 1, (hm, n)) + 1j * rng.uniform(-1, 1, (hm, n))).astype(np.complex64) for _ in range(2)]
    ys = [np.zeros_like(x) for x in xs]
    errors = []

    def work(i):
        try:
            for _ in range(5):
                plan.execute(xs[i].ctypes.data, ys[i].ctypes.data)
        except Exception as e:  # reported after the join
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for i in range(2):
        ref = oracle.c2c(xs[i].astype(np.complex128), -1, method="fft")
        assert oracle.rel_l2(ys[i], ref) <= oracle.fp32_tol(n)
