"""Grouped mixed-length C2C (plfft_cuda_group_*) vs the FP64 oracle.

Each transform of the group is checked against the oracle at the FP32 gate
(rel-L2 <= 4*log2(N)*2^-24); the lengths cover every task class: on-chip
smooth, Rader, Bluestein, four-step, and long Rader/Bluestein convolutions.
"""
import numpy as np
import pytest

import oracle
import plfft

pytestmark = pytest.mark.gpu


def _run_group(lengths, direction, seed, gap=0, rigor=None):
    import torch

    lengths = np.asarray(lengths, np.int64)
    offs = np.concatenate([[0], np.cumsum(lengths + gap)[:-1]]).astype(np.int64)
    total = int(offs[-1] + lengths[-1])
    rng = np.random.default_rng(seed)
    x = (rng.uniform(-1, 1, total) + 1j * rng.uniform(-1, 1, total)).astype(np.complex64)
    g = plfft.Group(lengths, offs, offs, direction, rigor=rigor)
    d_in = torch.from_numpy(x).cuda()
    d_out = torch.zeros(total, dtype=torch.complex64, device="cuda")
    g.execute_async(d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    y = d_out.cpu().numpy()
    return g, x, y, offs


def _check(lengths, x, y, offs, direction):
    for n, o in zip(lengths, offs):
        ref = oracle.c2c(x[o:o + n][None].astype(np.complex128), direction, method="fft" if n > 2048 else "dft")[0]
        err = oracle.rel_l2(y[o:o + n], ref)
        assert err <= oracle.fp32_tol(n), (n, err)


CLASSES = [16, 1, 2, 3, 100, 1024, 8192, 6561,        # on chip
           1009, 97, 8191 + 2 * 0,                     # Rader (8191 -> 8190 smooth? no: Bluestein)
           1031, 4099, 1058,                           # Bluestein on chip
           16384, 65536, 3 ** 10, 10000 * 3,            # four-step
           12289, 40961,                                # long Rader (12288, 40960 smooth)
           9001, 65521]                                 # long Bluestein


@pytest.mark.parametrize("direction", [-1, 1])
def test_group_all_classes(direction):
    g, x, y, offs = _run_group(CLASSES, direction, seed=1)
    d = g.describe()
    assert "four-step=" in d and g.launch_count() >= 2, d
    _check(CLASSES, x, y, offs, direction)


def test_group_replay_and_gaps():
    """Graph replay with new data and non-contiguous offsets."""
    import torch

    lengths = [64, 257, 4096, 17, 20000, 1031]
    g, x, y, offs = _run_group(lengths, -1, seed=2, gap=5)
    _check(lengths, x, y, offs, -1)
    total = len(x)
    x2 = (np.random.default_rng(3).standard_normal(total) + 0j).astype(np.complex64)
    d_in = torch.from_numpy(x2).cuda()
    d_out = torch.zeros(total, dtype=torch.complex64, device="cuda")
    for _ in range(2):
        g.execute_async(d_in.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    _check(lengths, x2, d_out.cpu().numpy(), offs, -1)


def test_group_synthetic_mix_sample():
    """A 300-transform sample of the grouped workload's length distribution."""
    from helpers import grouped_lengths

    lengths = grouped_lengths(300, seed=7, max_len=65536)
    g, x, y, offs = _run_group(lengths, -1, seed=4)
    rng = np.random.default_rng(0)
    pick = rng.choice(len(lengths), 40, replace=False)
    _check([lengths[i] for i in pick], x, y, [offs[i] for i in pick], -1)


# the schedule shapes the grouped autotuner chooses from: four-step tile
# width, same-length on-chip transforms merged into one task (runs of equal
# lengths with equal offset steps), largest radix of the stage lists
SHAPE_LENGTHS = ([64] * 40 + [1000] * 9 + [17] * 3 + [4096] * 5 + [8192] * 3 + [16384] * 2 +
                 [12289, 9001, 1031, 97, 6561, 6561])


@pytest.mark.parametrize("gap", [0, 3])
@pytest.mark.parametrize("shape", ["16,1,16", "8,16,8", "32,64,32", "64,16,16", "16,4,16"])
def test_group_shapes(monkeypatch, shape, gap):
    monkeypatch.setenv("PLFFT_B200_GROUP_SHAPE", shape)
    g, x, y, offs = _run_group(SHAPE_LENGTHS, -1, seed=5, gap=gap)
    t, m, r = shape.split(",")
    assert "tile=%s merge=%s radix=%s" % (t, m, r) in g.describe(), g.describe()
    _check(SHAPE_LENGTHS, x, y, offs, -1)


def test_group_tuned_and_wisdom():
    """MEASURE rigor times candidate schedules and keeps the fastest; a second
    group of the same problem takes the choice from the wisdom."""
    from helpers import grouped_lengths

    plfft.wisdom_forget()
    lengths = grouped_lengths(120, seed=11, max_len=20000)
    g, x, y, offs = _run_group(lengths, 1, seed=6, rigor=plfft.Rigor.MEASURE)
    d = g.describe()
    assert "tile=" in d, d
    pick = np.random.default_rng(1).choice(len(lengths), 20, replace=False)
    _check([lengths[i] for i in pick], x, y, [offs[i] for i in pick], 1)
    g2, x2, y2, offs2 = _run_group(lengths, 1, seed=7, rigor=plfft.Rigor.MEASURE)
    assert g2.describe() == d
    _check([lengths[i] for i in pick], x2, y2, [offs2[i] for i in pick], 1)
    with pytest.raises(plfft.PlfftError):
        _run_group([16, 32], -1, seed=8, rigor=7)
