"""The reference's ESTIMATE plan for batched C2C, executed with its own kernels.

Test infrastructure only (fixture generation).  Restates, for the
interpreter in neon_a64.py, how the reference composes its NEON kernels for
a C2C transform when the planner stops at the first applicable strategy
(rigor ESTIMATE: plfft.cpp:149-153 gives a zero time budget, which keeps
ALLOW_PRUNING, planner/policy.hpp:45-66; planner.cpp:317-345 then takes the
first candidate):

  strategy order       planner/planner.cpp:51-175: direct(n) for a base
                       kernel length, cooley_tukey_ab(r) for r = 40 .. 2,
                       cooley_tukey_ac(r) for r = 40 .. 2, (convolutions),
                       loop
  base kernel lengths  providers/aot/aot_kernel_data.cpp:296-308: 2..20 for
                       floating point, {2, 4, 8, 16} for fixed point
  cooley_tukey_ab/ac   planner/strategies/cooley_tukey.hpp:622-748 (DIT):
                       stage 1 = sub-problem of length m = n / r, stage 2 =
                       twiddled radix-r level; stage 1 writes a buffer of
                       n * howmany elements that stage 2 reads
  ab level             cooley_tukey.hpp:82-143: the unit row by the
                       untwiddled kernel, rows 1..howmany-1 by ab_t_dit
  ac level             cooley_tukey.hpp:331-385: row 0 untwiddled over
                       howmany1 columns, rows i >= 1 twiddled with row
                       (i - 1) of the table
  loop                 planner/strategies/loop.hpp: one plan per member
  kernel variant       providers/aot/aot_kernel_data.cpp:182-256: howmany 1
                       -> uun, idist = odist = 1 -> uu, idist = 1 -> us,
                       odist = 1 -> gu, else gs
  twiddles             generate_twiddles.hpp:72-132 with premultiplied
                       pairs: for j = 1..n1-1, i = 1..n2-1,
                       W = (cos t, sin t), (-sin t, cos t), t = dir 2 pi i j / n;
                       fixed point converts each with convert_to
                       (plfft_convert.hpp:36-54: truncate x * 2^(bits-1),
                       saturate)
"""
import numpy as np

CT_RADICES = [40, 39, 38, 36, 35, 34, 33, 32, 30, 28, 26, 25, 24, 22, 21, 20, 19, 18, 17, 16, 15, 14, 13,
              12, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2]

DTYPES = {
    # name: (kernel infix, complex element bytes, base lengths)
    "f32": ("ccc", 8, list(range(2, 21))),
    "q15": ("q15_jjj", 4, [2, 4, 8, 16]),
    "q7": ("q7_ppp", 2, [2, 4, 8, 16]),
}


def variant(howmany, idist, odist):
    if howmany == 1:
        return "uun"
    if idist == 1 and odist == 1:
        return "uu"
    if idist == 1:
        return "us"
    if odist == 1:
        return "gu"
    return "gs"


def twiddles(dtype, dirn, n1, n2):
    """generate_twiddles(dir, n1, n2, premul=True, interleave=1) as the
    kernels read it: complex elements of the data type, flattened."""
    n = n1 * n2
    base = dirn * 2.0 * np.pi / n
    vals = []
    for j in range(1, n1):
        for i in range(1, n2):
            a, b = np.cos(base * i * j), np.sin(base * i * j)
            vals += [(a, b), (-b, a)]
    v = np.array(vals, np.float64).reshape(-1, 2)
    if dtype == "f32":
        return v.astype(np.float32)
    bits = 16 if dtype == "q15" else 8
    t = np.trunc(v.astype(np.float32).astype(np.float64) * float(1 << (bits - 1)))
    lim = 1 << (bits - 1)
    return np.clip(t, -lim, lim - 1).astype(np.int16 if bits == 16 else np.int8)


class Planner:
    def __init__(self, machine, dtype, dirn):
        self.m = machine
        self.dtype = dtype
        self.dirn = dirn
        self.k, self.esz, self.ns = DTYPES[dtype]
        self.d = "f" if dirn < 0 else "b"

    def plan(self, n, istride, ostride, howmany, idist, odist):
        if n in self.ns:
            return Direct(self, n, istride, ostride, howmany, idist, odist)
        for r in CT_RADICES:
            if r < n and n % r == 0 and r in self.ns and howmany == 1:
                return CooleyTukeyAB(self, r, n, istride, ostride)
        for r in CT_RADICES:
            if (r < n and n % r == 0 and r in self.ns and istride == howmany * idist and odist == 1
                    and howmany > 1):
                return CooleyTukeyAC(self, r, n, istride, ostride, howmany, idist)
        if n > 1 and howmany > 1:
            return Loop(self, n, istride, ostride, howmany, idist, odist)
        raise NotImplementedError(f"no ESTIMATE plan restated for n={n} howmany={howmany}")

    def call(self, name, args):
        self.m.call(name, [int(a) for a in args])


class Direct:
    def __init__(self, p, n, istride, ostride, howmany, idist, odist):
        self.p, self.a = p, (istride, ostride, howmany, idist, odist)
        self.name = f"plfft_{n}_{p.k}n{p.d}_{variant(howmany, idist, odist)}_neon"

    def execute(self, x, y):
        self.p.call(self.name, [x, y, *self.a])


class AbLevel:
    """ab_twid_direct_plan (c2c): radix-n level over howmany rows."""

    def __init__(self, p, n, istride, ostride, howmany, idist, odist):
        self.p, self.n = p, n
        self.istride, self.ostride, self.howmany, self.idist, self.odist = istride, ostride, howmany, idist, odist
        self.kn = f"plfft_{n}_{p.k}n{p.d}_uun_neon"
        self.kt = f"plfft_ab_{n}_{p.k}t{p.d}_dit_{variant(howmany, idist, odist)}_neon"
        w = twiddles(p.dtype, p.dirn, howmany, n)
        self.w = p.m.alloc(max(1, w.nbytes))
        p.m.write(self.w, w)

    def execute(self, x, y):
        e = self.p.esz
        self.p.call(self.kn, [x, y, self.istride, self.ostride, 1, 0, 0])
        if self.howmany > 1:
            self.p.call(self.kt, [x + e * self.idist, y + e * self.odist, self.istride, self.ostride, self.w,
                                  self.howmany - 1, self.idist, self.odist])


class AcLevel:
    """ac_twid_direct_plan (c2c): radix-n level, howmany0 rows of howmany1 columns."""

    def __init__(self, p, n, istride, ostride, howmany0, idist0, odist0, howmany1):
        self.p, self.n = p, n
        self.istride, self.ostride = istride, ostride
        self.howmany0, self.idist0, self.odist0, self.howmany1 = howmany0, idist0, odist0, howmany1
        v = variant(howmany1, 1, 1)
        self.kn = f"plfft_{n}_{p.k}n{p.d}_{v}_neon"
        self.kt = f"plfft_ac_{n}_{p.k}t{p.d}_dit_{v}_neon"
        w = twiddles(p.dtype, p.dirn, howmany0, n)
        self.w = p.m.alloc(max(1, w.nbytes))
        p.m.write(self.w, w)

    def execute(self, x, y):
        e = self.p.esz
        self.p.call(self.kn, [x, y, self.istride, self.ostride, self.howmany1, 1, 1])
        for i in range(1, self.howmany0):
            off = (i - 1) * 2 * (self.n - 1)  # premultiplied pairs per row
            self.p.call(self.kt, [x + e * i * self.idist0, y + e * i * self.odist0, self.istride, self.ostride,
                                  self.w + e * off, self.howmany1, 1, 1])


class CooleyTukeyAB:
    def __init__(self, p, r, n, istride, ostride):
        m = n // r
        self.p, self.n = p, n
        self.stage1 = p.plan(m, istride * r, r, r, istride, 1)
        self.stage2 = AbLevel(p, r, 1, ostride * m, m, r, ostride)
        self.buf = p.m.alloc(p.esz * n)

    def execute(self, x, y):
        self.stage1.execute(x, self.buf)
        self.stage2.execute(self.buf, y)


class CooleyTukeyAC:
    def __init__(self, p, r, n, istride, ostride, howmany, idist):
        m = n // r
        self.p, self.n = p, n
        self.stage1 = p.plan(m, istride * r, howmany * r, howmany * r, idist, 1)
        self.stage2 = AcLevel(p, r, howmany, ostride * m, m, howmany * r, ostride, howmany)
        self.buf = p.m.alloc(p.esz * n * howmany)

    def execute(self, x, y):
        self.stage1.execute(x, self.buf)
        self.stage2.execute(self.buf, y)


class Loop:
    def __init__(self, p, n, istride, ostride, howmany, idist, odist):
        self.p = p
        self.howmany, self.idist, self.odist = howmany, idist, odist
        self.inner = p.plan(n, istride, ostride, 1, 0, 0)

    def execute(self, x, y):
        e = self.p.esz
        for i in range(self.howmany):
            self.inner.execute(x + e * i * self.idist, y + e * i * self.odist)


def describe(node):
    if isinstance(node, Direct):
        return node.name
    if isinstance(node, Loop):
        return f"(loop {node.howmany} {describe(node.inner)})"
    if isinstance(node, (CooleyTukeyAB, CooleyTukeyAC)):
        kind = "ab" if isinstance(node, CooleyTukeyAB) else "ac"
        return f"(ct-{kind} {node.n} {describe(node.stage1)} {node.stage2.kt})"
    return type(node).__name__


def run_c2c(machine, dtype, dirn, x, n, howmany, istride=1, idist=None, ostride=1, odist=None):
    """Execute the ESTIMATE plan on buffer x (flat array of complex elements in
    the type's storage: complex64, or int16/int8 pairs as [..., 2]).
    Returns the output buffer (same layout as x) and the plan description."""
    idist = n if idist is None else idist
    odist = n if odist is None else odist
    p = Planner(machine, dtype, dirn)
    node = p.plan(n, istride, ostride, howmany, idist, odist)
    xa = machine.alloc(x.nbytes)
    machine.write(xa, x)
    out_elems = (howmany - 1) * odist + (n - 1) * ostride + 1
    ya = machine.alloc(out_elems * p.esz)
    node.execute(xa, ya)
    if dtype == "f32":
        y = machine.read(ya, np.complex64, out_elems)
    else:
        y = machine.read(ya, np.int16 if dtype == "q15" else np.int8, 2 * out_elems).reshape(-1, 2)
    return y, describe(node)
