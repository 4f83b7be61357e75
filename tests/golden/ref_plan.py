"""The reference's ESTIMATE plans for batched C2C, R2C and C2R, executed with
its own kernels.

Test infrastructure only (fixture generation).  Restates, for the
interpreter in neon_a64.py, how the reference composes its NEON kernels when
the planner stops at the first applicable strategy (rigor ESTIMATE:
plfft.cpp:149-153 gives a zero time budget, which keeps ALLOW_PRUNING,
planner/policy.hpp:45-66; planner.cpp:317-345 then takes the first
candidate):

  strategy order       planner/planner.cpp:51-175: direct(n) for a base
                       kernel length, cooley_tukey_ab(r) for r = 40 .. 2,
                       cooley_tukey_ac(r) for r = 40 .. 2, (convolutions),
                       loop
  base kernel lengths  providers/aot/aot_kernel_data.cpp:296-308: 2..20 for
                       floating point, {2, 4, 8, 16} for fixed point
  cooley_tukey_ab/ac   planner/strategies/cooley_tukey.hpp:622-748: C2C and
                       R2C decimate in time (stage 1 = sub-problem of length
                       m = n / r, stage 2 = twiddled radix-r level), C2R in
                       frequency (stage 1 = twiddled level, stage 2 = the
                       sub-problem); the stages meet in a buffer of n *
                       howmany complex elements
  ab levels            cooley_tukey.hpp:82-143 (C2C: unit row untwiddled,
                       rows 1.. twiddled), :145-248 (R2C: half-output unit
                       row, conjugate-reversed rows, middle row for even
                       howmany), :250-323 (C2R: Hermitian-input rows)
  ac levels            cooley_tukey.hpp:331-552 (the same per column block)
  loop                 planner/strategies/loop.hpp: one plan per member
  kernel variant       providers/aot/aot_kernel_data.cpp:182-256: howmany 1
                       -> uun, idist = odist = 1 -> uu, idist = 1 -> us,
                       odist = 1 -> gu, else gs
  kernel names         providers/aot/aot_kernel_lookup.cpp (n: untwiddled,
                       t: twiddled, f/b: direction, oh/ih: half-spectrum
                       output/input, j: conjugate-reversed second output,
                       ol/il: middle row)
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
    # name: (complex infix, real-in infix, real-out infix, complex bytes, real bytes, base lengths)
    "f32": ("ccc", "scc", "ccs", 8, 4, list(range(2, 21))),
    "q15": ("q15_jjj", "q15_hjj", "q15_jjh", 4, 2, [2, 4, 8, 16]),
    "q7": ("q7_ppp", "q7_rpp", "q7_ppr", 2, 1, [2, 4, 8, 16]),
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
    def __init__(self, machine, dtype, kind, dirn):
        self.m = machine
        self.dtype = dtype
        self.kind = kind  # "c2c", "r2c" (forward) or "c2r" (backward)
        self.dirn = dirn
        self.k, self.kr, self.kcr, self.esz, self.rsz, self.ns = DTYPES[dtype]
        self.d = "f" if dirn < 0 else "b"

    def in_size(self):
        return self.rsz if self.kind == "r2c" else self.esz

    def out_size(self):
        return self.rsz if self.kind == "c2r" else self.esz

    def plan(self, n, istride, ostride, howmany, idist, odist):
        if n in self.ns:
            return Direct(self, n, istride, ostride, howmany, idist, odist)
        for r in CT_RADICES:
            if r < n and n % r == 0 and r in self.ns and howmany == 1:
                return CooleyTukeyAB(self, r, n, istride, ostride)
        for r in CT_RADICES:
            if not (r < n and n % r == 0 and r in self.ns and howmany > 1):
                continue
            if self.kind != "c2r" and istride == howmany * idist and odist == 1:
                return CooleyTukeyAC(self, r, n, istride, ostride, howmany, idist, odist)
            if self.kind == "c2r" and idist == 1 and ostride == howmany * odist:
                return CooleyTukeyAC(self, r, n, istride, ostride, howmany, idist, odist)
        if n > 1 and howmany > 1:
            return Loop(self, n, istride, ostride, howmany, idist, odist)
        raise NotImplementedError(f"no ESTIMATE plan restated for n={n} howmany={howmany}")

    def call(self, name, args):
        self.m.call(name, [int(a) for a in args])

    def table(self, n1, n2):
        w = twiddles(self.dtype, self.dirn, n1, n2)
        a = self.m.alloc(max(1, w.nbytes))
        self.m.write(a, w)
        return a


class Direct:
    def __init__(self, p, n, istride, ostride, howmany, idist, odist):
        self.p, self.a = p, (istride, ostride, howmany, idist, odist)
        v = variant(howmany, idist, odist)
        if p.kind == "c2c":
            self.name = f"plfft_{n}_{p.k}n{p.d}_{v}_neon"
        elif p.kind == "r2c":
            self.name = f"plfft_{n}_{p.kr}nfoh_{v}_neon"
        else:
            self.name = f"plfft_{n}_{p.kcr}nb_{v}_neon"

    def execute(self, x, y):
        self.p.call(self.name, [x, y, *self.a])


class AbLevel:
    """ab_twid_direct_plan: radix-n level over howmany rows (complex data)."""

    def __init__(self, p, n, istride, ostride, howmany, idist, odist):
        self.p, self.n = p, n
        self.istride, self.ostride, self.howmany, self.idist, self.odist = istride, ostride, howmany, idist, odist
        k, d = p.k, p.d
        if p.kind == "c2c":
            self.kn = f"plfft_{n}_{k}n{d}_uun_neon"
            self.kt = f"plfft_ab_{n}_{k}t{d}_dit_{variant(howmany, idist, odist)}_neon"
            self.w = p.table(howmany, n)
        elif p.kind == "r2c":
            self.kn = f"plfft_{n}_{k}nfoh_uun_neon"
            self.kt = f"plfft_ab_{n}_{k}tfj_dit_{variant(howmany, idist, odist)}_neon"
            self.kol = f"plfft_ab_{n}_{k}tfol_dit_uun_neon"
            self.w = p.table(howmany, n)
        else:
            # rows 0 .. howmany/2 of the Hermitian input
            self.rows = howmany // 2 + 1
            self.kn = f"plfft_{n}_{k}nbih_uun_neon"
            half = "il" if n % 2 == 0 else "ih"
            self.kt = f"plfft_ab_{n}_{k}tb{half}_dif_{variant(2, idist, odist)}_neon"
            self.w = p.table(howmany, n)

    def execute(self, x, y):
        p, e, n = self.p, self.p.esz, self.n
        is_, os_, hm, id_, od = self.istride, self.ostride, self.howmany, self.idist, self.odist
        if p.kind == "c2c":
            p.call(self.kn, [x, y, is_, os_, 1, 0, 0])
            if hm > 1:
                p.call(self.kt, [x + e * id_, y + e * od, is_, os_, self.w, hm - 1, id_, od])
        elif p.kind == "r2c":
            p.call(self.kn, [x, y, is_, os_, 1, 0, 0])
            halflo = (hm + 1) // 2
            if halflo > 1:
                yy = (n // 2 - 1) * os_ + (hm - 1) * od
                p.call(self.kt, [x + e * id_, y + e * od, y + e * yy, is_, os_, self.w, halflo - 1, id_, od])
            if hm % 2 == 0:
                p.call(self.kol, [x + e * halflo * id_, y + e * halflo * od, is_, os_,
                                  self.w + e * 2 * (halflo - 1) * (n - 1), 1, 0, 0])
        else:
            xx = (n - 1) // 2 * is_
            p.call(self.kn, [x, x + e * xx, y, is_, os_, 1, 0, 0])
            if self.rows > 1:
                p.call(self.kt, [x + e * id_, x + e * (n // 2 * is_ - id_), y + e * od, is_, os_, self.w,
                                 self.rows - 1, id_, od])


class AcLevel:
    """ac_twid_direct_plan: radix-n level, howmany0 rows of howmany1 columns."""

    def __init__(self, p, n, istride, ostride, howmany0, idist0, odist0, howmany1):
        self.p, self.n = p, n
        self.istride, self.ostride = istride, ostride
        self.howmany0, self.idist0, self.odist0, self.howmany1 = howmany0, idist0, odist0, howmany1
        v = variant(howmany1, 1, 1)
        k, d = p.k, p.d
        if p.kind == "c2c":
            self.kn = f"plfft_{n}_{k}n{d}_{v}_neon"
            self.kt = f"plfft_ac_{n}_{k}t{d}_dit_{v}_neon"
        elif p.kind == "r2c":
            self.kn = f"plfft_{n}_{k}nfoh_{v}_neon"
            self.kt = f"plfft_ac_{n}_{k}tfj_dit_{v}_neon"
            self.kol = f"plfft_ac_{n}_{k}tfol_dit_{v}_neon"
        else:
            self.kn = f"plfft_{n}_{k}nbih_{v}_neon"
            self.kt = f"plfft_ac_{n}_{k}tb{'il' if n % 2 == 0 else 'ih'}_dif_{v}_neon"
        self.w = p.table(howmany0, n)

    def execute(self, x, y):
        p, e, n = self.p, self.p.esz, self.n
        is_, os_, h0, id0, od0, h1 = self.istride, self.ostride, self.howmany0, self.idist0, self.odist0, self.howmany1
        row = lambda i: self.w + e * (i - 1) * 2 * (n - 1)  # noqa: E731  premultiplied pairs per row
        if p.kind == "c2c":
            p.call(self.kn, [x, y, is_, os_, h1, 1, 1])
            for i in range(1, h0):
                p.call(self.kt, [x + e * i * id0, y + e * i * od0, is_, os_, row(i), h1, 1, 1])
        elif p.kind == "r2c":
            p.call(self.kn, [x, y, is_, os_, h1, 1, 1])
            halflo = (h0 + 1) // 2
            yy = (n // 2 - 1) * os_ + h0 * od0
            for i in range(1, halflo):
                p.call(self.kt, [x + e * i * id0, y + e * i * od0, y + e * (yy - i * od0), is_, os_, row(i), h1, 1, 1])
            if h0 % 2 == 0:
                p.call(self.kol, [x + e * halflo * id0, y + e * halflo * od0, is_, os_, row(halflo), h1, 1, 1])
        else:
            xx = (n - 1) // 2 * is_
            p.call(self.kn, [x, x + e * xx, y, is_, os_, h1, 1, 1])
            for i in range(1, h0 // 2 + 1):
                p.call(self.kt, [x + e * i * id0, x + e * (n // 2 * is_ - i * id0), y + e * i * od0, is_, os_, row(i),
                                 h1, 1, 1])


class CooleyTukeyAB:
    def __init__(self, p, r, n, istride, ostride):
        m = n // r
        self.p, self.n = p, n
        self.buf = p.m.alloc(p.esz * n)
        if p.kind != "c2r":
            self.stage1 = p.plan(m, istride * r, r, r, istride, 1)
            self.stage2 = AbLevel(p, r, 1, ostride * m, m, r, ostride)
        else:
            self.stage1 = AbLevel(p, r, istride * m, 1, m, istride, r)
            self.stage2 = p.plan(m, r, ostride * r, r, 1, ostride)

    def execute(self, x, y):
        self.stage1.execute(x, self.buf)
        self.stage2.execute(self.buf, y)


class CooleyTukeyAC:
    def __init__(self, p, r, n, istride, ostride, howmany, idist, odist):
        m = n // r
        self.p, self.n = p, n
        self.buf = p.m.alloc(p.esz * n * howmany)
        if p.kind != "c2r":
            self.stage1 = p.plan(m, istride * r, howmany * r, howmany * r, idist, 1)
            self.stage2 = AcLevel(p, r, howmany, ostride * m, m, howmany * r, ostride, howmany)
        else:
            self.stage1 = AcLevel(p, r, istride * m, howmany, m, istride, howmany * r, howmany)
            self.stage2 = p.plan(m, howmany * r, ostride * r, howmany * r, 1, odist)

    def execute(self, x, y):
        self.stage1.execute(x, self.buf)
        self.stage2.execute(self.buf, y)


class Loop:
    def __init__(self, p, n, istride, ostride, howmany, idist, odist):
        self.p = p
        self.howmany, self.idist, self.odist = howmany, idist, odist
        self.inner = p.plan(n, istride, ostride, 1, 0, 0)

    def execute(self, x, y):
        ei, eo = self.p.in_size(), self.p.out_size()
        for i in range(self.howmany):
            self.inner.execute(x + ei * i * self.idist, y + eo * i * self.odist)


def describe(node):
    if isinstance(node, Direct):
        return node.name
    if isinstance(node, Loop):
        return f"(loop {node.howmany} {describe(node.inner)})"
    if isinstance(node, (CooleyTukeyAB, CooleyTukeyAC)):
        kind = "ab" if isinstance(node, CooleyTukeyAB) else "ac"
        lvl = node.stage2 if isinstance(node.stage2, (AbLevel, AcLevel)) else node.stage1
        sub = node.stage1 if lvl is node.stage2 else node.stage2
        return f"(ct-{kind} {node.n} {describe(sub)} {lvl.kt})"
    return type(node).__name__


def _storage(dtype, count, real):
    if dtype == "f32":
        return np.float32 if real else np.complex64, count
    it = np.int16 if dtype == "q15" else np.int8
    return it, count if real else 2 * count


def run(machine, dtype, kind, dirn, x, n, howmany, istride=1, idist=None, ostride=1, odist=None):
    """Execute the ESTIMATE plan on buffer x (flat array: complex64 / float32,
    or int16 / int8 values, complex elements as (re, im) pairs).  Returns the
    flat output buffer and the plan description."""
    nin = n // 2 + 1 if kind == "c2r" else n
    nout = n // 2 + 1 if kind == "r2c" else n
    idist = nin if idist is None else idist
    odist = nout if odist is None else odist
    p = Planner(machine, dtype, kind, dirn)
    node = p.plan(n, istride, ostride, howmany, idist, odist)
    xa = machine.alloc(x.nbytes)
    machine.write(xa, x)
    out_elems = (howmany - 1) * odist + (nout - 1) * ostride + 1
    ya = machine.alloc(out_elems * p.out_size())
    node.execute(xa, ya)
    dt, cnt = _storage(dtype, out_elems, kind == "c2r")
    return machine.read(ya, dt, cnt), describe(node)


def run_c2c(machine, dtype, dirn, x, n, howmany, istride=1, idist=None, ostride=1, odist=None):
    y, desc = run(machine, dtype, "c2c", dirn, x, n, howmany, istride, idist, ostride, odist)
    return (y if dtype == "f32" else y.reshape(-1, 2)), desc
