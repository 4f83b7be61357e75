"""Interpreter for the AArch64 / NEON instruction subset of PLFFT's kernels.

Test infrastructure only: the fixture generators in this folder use it, in
a container that holds the reference sources, to execute the reference's
own generated NEON kernels (src/providers/aot/asm/neon/*.S, read as text)
on seeded inputs.  Their outputs become committed fixtures; nothing at test
time reads the reference.

Semantics implemented (Arm A64 definitions):
  scalar  ldr/str (B/H/S/D/Q and X registers), ldp/stp, add/sub (immediate,
          register, shifted register), lsl, asr, mul, movz, mov, cmp,
          movn, b / b.lt / b.ge, ret, adrp + page offsets of read-only data
  loads   ld1r (replicate one element to every lane), dup (by element)
  FP32    fadd, fsub, fmul (vector and by element), fmla / fmls (vector and
          by element; a fused multiply-add rounded once: the product is
          exact in double, the sum is formed with an exact two-sum and
          rounded to single precision once, ties broken by the two-sum's
          error term)
  integer sqadd, sqsub, srshr, sqrdmulh, smull(2), smlal(2), smlsl(2)
          (vector and by element), sqrshrn(2) on 8- and 16-bit lanes
  permute rev16, rev32, rev64, zip1, trn1, trn2, uzp1, uzp2, ext
  sign    fneg (any lane width: the sign bit flipped), sqneg
"""
import re

import numpy as np

MASK64 = (1 << 64) - 1

# lane arrangement -> (lanes, bytes per lane)
_ARR = {"8b": (8, 1), "16b": (16, 1), "4h": (4, 2), "8h": (8, 2), "2s": (2, 4), "4s": (4, 4),
        "1d": (1, 8), "2d": (2, 8)}
_INT = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}


def _s64(v):
    v &= MASK64
    return v - (1 << 64) if v >> 63 else v


class Kernels:
    """Parsed functions (name -> instruction list), labels and read-only data."""

    def __init__(self, paths):
        self.funcs, self.labels, self.rodata = {}, {}, {}
        for p in paths:
            self._parse(open(p).read())

    def _parse(self, text):
        cur, ro = None, None
        for raw in text.splitlines():
            line = raw.split("//")[0].strip()
            if not line or line.startswith("#") or line.startswith("/*") or line.startswith("*"):
                continue
            m = re.match(r"FUNC_NAME\((\w+)\):", line)
            if m:
                cur, ro = m.group(1), None
                self.funcs[cur] = []
                continue
            m = re.match(r"(\.rodata\.\w+):", line)
            if m:
                ro, cur = m.group(1), None
                self.rodata[ro] = bytearray()
                continue
            m = re.match(r"(\.L[\w.]+):", line)
            if m and cur:
                self.labels[(cur, m.group(1))] = len(self.funcs[cur])
                continue
            if line.startswith(".byte") and ro:
                self.rodata[ro] += bytes(int(b, 16) for b in line[5:].split(","))
                continue
            if line.startswith(".") or line.startswith("FUNC_") or line.startswith("RODATA"):
                continue
            if cur:
                op, _, rest = line.partition("\t") if "\t" in line else line.partition(" ")
                self.funcs[cur].append((op.strip(), [a.strip() for a in _split_operands(rest.strip())]))


def _split_operands(s):
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "[{":
            depth += 1
        elif ch in "]}":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return out


def _fma32(a, b, d, negate=False):
    """float32 d + a*b (or d - a*b) rounded once, elementwise."""
    p = a.astype(np.float64) * b.astype(np.float64)  # exact
    if negate:
        p = -p
    dd = d.astype(np.float64)
    s = p + dd
    bb = s - p
    e = (p - (s - bb)) + (dd - bb)  # s + e == p + d exactly (two-sum)
    r = s.astype(np.float32)
    r64 = r.astype(np.float64)
    # |e| is at most half an ulp of s in double, so s + e rounds like s unless
    # s sits exactly halfway between r and its neighbour nb on s's side;
    # then the sign of e decides
    nb = np.where(s > r64, np.nextafter(r, np.float32(np.inf)), np.nextafter(r, np.float32(-np.inf)))
    at_mid = (s == (r64 + nb.astype(np.float64)) * 0.5) & (e != 0)
    if np.any(at_mid):
        toward_nb = np.sign(e) == np.sign(nb.astype(np.float64) - r64)
        r = np.where(at_mid & toward_nb, nb, r)
    return r.astype(np.float32)


class Machine:
    """Flat byte memory, 31 X registers + sp, 32 V registers (16 bytes)."""

    def __init__(self, kernels, mem_bytes=1 << 26):
        self.k = kernels
        self.mem = np.zeros(mem_bytes, np.uint8)
        self.top = 4096  # bump allocator for buffers
        self.ro_addr = {}
        for name, data in kernels.rodata.items():
            a = self.alloc(len(data))
            self.mem[a:a + len(data)] = np.frombuffer(bytes(data), np.uint8)
            self.ro_addr[name] = a
        self.stack_top = mem_bytes - 256

    def alloc(self, nbytes):
        a = (self.top + 63) & ~63
        self.top = a + nbytes
        assert self.top < len(self.mem) - (1 << 20), "interpreter memory exhausted"
        return a

    def write(self, addr, arr):
        b = np.ascontiguousarray(arr).view(np.uint8).ravel()
        self.mem[addr:addr + b.size] = b

    def read(self, addr, dtype, count):
        nb = np.dtype(dtype).itemsize * count
        return self.mem[addr:addr + nb].copy().view(dtype)

    # ---------------------------------------------------------------
    def call(self, name, args):
        self.x = [0] * 31
        self.sp = self.stack_top - 64  # 16-byte aligned; arguments 9.. live at [sp], [sp + 8], ...
        self.v = [np.zeros(16, np.uint8) for _ in range(32)]
        for i, a in enumerate(args[:8]):
            self.x[i] = int(a) & MASK64
        for i, a in enumerate(args[8:]):  # AAPCS64: integer arguments past the eighth on the stack
            self.mem[self.sp + 8 * i:self.sp + 8 * i + 8] = np.array([int(a) & MASK64], np.uint64).view(np.uint8)
        code = self.k.funcs[name]
        pc, steps = 0, 0
        while True:
            op, ops = code[pc]
            steps += 1
            assert steps < 50_000_000, "runaway kernel"
            nxt = self.step(name, op, ops)
            if nxt == "ret":
                return
            pc = pc + 1 if nxt is None else nxt

    # ---------------------------------------------------------------
    def reg(self, s):
        if s == "sp":
            return self.sp
        if s == "xzr":
            return 0
        return self.x[int(s[1:])]

    def setreg(self, s, val):
        if s == "sp":
            self.sp = val & MASK64
        elif s != "xzr":
            self.x[int(s[1:])] = val & MASK64

    @staticmethod
    def imm(s):
        return int(s.lstrip("#"), 0)

    def addr(self, s):
        inner = s.strip()[1:-1].split(",")
        base = self.reg(inner[0].strip())
        if len(inner) == 1:
            return base
        second = inner[1].strip()
        if second.startswith("#"):
            return base + self.imm(second)
        off = _s64(self.reg(second))
        if len(inner) > 2:
            sh = int(inner[2].strip().split("#")[1])
            off <<= sh
        return base + off

    def vreg(self, s):
        return self.v[int(re.match(r"\{?[vqsdhb](\d+)", s).group(1))]

    @staticmethod
    def arr(s):
        return s.split(".")[1].rstrip("}") if "." in s else None

    def lanes(self, s, kind="i"):
        """The lanes of a register operand as int64 ('i') or float32 ('f')."""
        n, w = _ARR[self.arr(s)]
        r = self.vreg(s)
        if kind == "f":
            return r.view(np.float32)[:n].copy()
        return r.view(_INT[w])[:n].astype(np.int64)

    def put(self, s, vals, kind="i"):
        n, w = _ARR[self.arr(s)]
        r = self.vreg(s)
        if kind == "f":
            r.view(np.float32)[:n] = vals
        else:
            r.view(_INT[w])[:n] = np.asarray(vals).astype(_INT[w])
        if n * w == 8:
            r[8:] = 0

    def elem(self, s, kind="i"):
        m = re.match(r"v(\d+)\.([bhsd])\[(\d+)\]", s)
        r = self.v[int(m.group(1))]
        i = int(m.group(3))
        if kind == "f":
            return r.view(np.float32)[i]
        return int(r.view(_INT[{"b": 1, "h": 2, "s": 4, "d": 8}[m.group(2)]])[i])

    # ---------------------------------------------------------------
    _VBYTES = {"b": 1, "h": 2, "s": 4, "d": 8, "q": 16}

    def step(self, fname, op, o):
        if op in ("ldr", "str"):
            r, a = o[0], self.addr(o[1])
            if r[0] == "x":
                if op == "ldr":
                    self.setreg(r, int(self.mem[a:a + 8].view(np.uint64)[0]))
                else:
                    self.mem[a:a + 8] = np.array([self.reg(r)], np.uint64).view(np.uint8)
                return None
            nb = self._VBYTES[r[0]]
            v = self.vreg(r)
            if op == "ldr":
                v[:] = 0
                v[:nb] = self.mem[a:a + nb]
            else:
                self.mem[a:a + nb] = v[:nb]
            return None
        if op in ("ldp", "stp"):
            a = self.addr(o[2])
            for i, r in enumerate(o[:2]):
                if op == "ldp":
                    self.setreg(r, int(self.mem[a + 8 * i:a + 8 * i + 8].view(np.uint64)[0]))
                else:
                    self.mem[a + 8 * i:a + 8 * i + 8] = np.array([self.reg(r)], np.uint64).view(np.uint8)
            return None
        if op == "ld1r":
            n, w = _ARR[self.arr(o[0])]
            a = self.addr(o[1])
            v = self.vreg(o[0])
            v[:] = np.tile(self.mem[a:a + w], 16 // w)
            if n * w == 8:
                v[8:] = 0
            return None
        if op == "adrp":
            self.setreg(o[0], self.ro_addr[re.search(r"\((.*)\)", o[1]).group(1)])
            return None
        if op in ("add", "sub"):
            if "PAGEOFF" in o[2]:
                self.setreg(o[0], self.reg(o[1]))
                return None
            a = _s64(self.reg(o[1]))
            b = self.imm(o[2]) if o[2].startswith("#") else _s64(self.reg(o[2]))
            if len(o) > 3:
                b <<= int(o[3].split("#")[1])
            self.setreg(o[0], a + b if op == "add" else a - b)
            return None
        if op == "lsl":
            self.setreg(o[0], self.reg(o[1]) << self.imm(o[2]))
            return None
        if op == "asr":
            self.setreg(o[0], _s64(self.reg(o[1])) >> self.imm(o[2]))
            return None
        if op == "mul":
            self.setreg(o[0], _s64(self.reg(o[1])) * _s64(self.reg(o[2])))
            return None
        if op == "movz":
            self.setreg(o[0], self.imm(o[1]))
            return None
        if op == "movn":
            self.setreg(o[0], ~self.imm(o[1]))
            return None
        if op == "mov":
            self.setreg(o[0], self.reg(o[1]))
            return None
        if op == "cmp":
            self.cmp = (_s64(self.reg(o[0])), _s64(self.reg(o[1])))
            return None
        if op in ("b.lt", "b.ge", "b"):
            if op == "b" and o[0].startswith("#"):
                return None  # branch to the next instruction
            taken = op == "b" or (self.cmp[0] < self.cmp[1]) == (op == "b.lt")
            return self.k.labels[(fname, o[0])] if taken else None
        if op == "ret":
            return "ret"
        return self.vstep(op, o)

    def vstep(self, op, o):
        d = o[0]
        if op in ("fadd", "fsub", "fmul", "fmla", "fmls"):
            a = self.lanes(o[1], "f")
            b = np.float32(self.elem(o[2], "f")) if "[" in o[2] else self.lanes(o[2], "f")
            b = np.broadcast_to(np.asarray(b, np.float32), a.shape)
            if op == "fadd":
                r = a + b
            elif op == "fsub":
                r = a - b
            elif op == "fmul":
                r = a * b
            else:
                r = _fma32(a, b, self.lanes(d, "f"), negate=op == "fmls")
            self.put(d, r.astype(np.float32), "f")
        elif op in ("sqadd", "sqsub"):
            _, w = _ARR[self.arr(d)]
            lo, hi = -(1 << (8 * w - 1)), (1 << (8 * w - 1)) - 1
            a, b = self.lanes(o[1]), self.lanes(o[2])
            self.put(d, np.clip(a + b if op == "sqadd" else a - b, lo, hi))
        elif op == "srshr":
            s = self.imm(o[2])
            self.put(d, (self.lanes(o[1]) + (1 << (s - 1))) >> s)
        elif op == "sqrdmulh":
            _, w = _ARR[self.arr(d)]
            bits = 8 * w
            a = self.lanes(o[1])
            b = self.elem(o[2]) if "[" in o[2] else self.lanes(o[2])
            r = (2 * a * b + (1 << (bits - 1))) >> bits
            self.put(d, np.clip(r, -(1 << (bits - 1)), (1 << (bits - 1)) - 1))
        elif op in ("smull", "smull2", "smlal", "smlal2", "smlsl", "smlsl2"):
            hi = op.endswith("2")
            nd, wd = _ARR[self.arr(d)]
            src = self.vreg(o[1]).view(_INT[wd // 2])
            a = (src[nd:2 * nd] if hi else src[:nd]).astype(np.int64)
            if "[" in o[2]:
                b = self.elem(o[2])
            else:
                bv = self.vreg(o[2]).view(_INT[wd // 2])
                b = (bv[nd:2 * nd] if hi else bv[:nd]).astype(np.int64)
            prod = a * b
            acc = self.vreg(d).view(_INT[wd])[:nd].astype(np.int64)
            if op.startswith("smull"):
                res = prod
            elif op.startswith("smlal"):
                res = acc + prod
            else:
                res = acc - prod
            m = 1 << (8 * wd)
            res = ((res + m // 2) % m) - m // 2  # wraps at the lane width
            self.vreg(d).view(_INT[wd])[:nd] = res.astype(_INT[wd])
        elif op in ("sqrshrn", "sqrshrn2"):
            s = self.imm(o[2])
            ns_, ws = _ARR[self.arr(o[1])]
            a = self.vreg(o[1]).view(_INT[ws])[:ns_].astype(np.int64)
            bits = 4 * ws
            r = np.clip((a + (1 << (s - 1))) >> s, -(1 << (bits - 1)), (1 << (bits - 1)) - 1)
            v = self.vreg(d).view(_INT[ws // 2])
            if op == "sqrshrn":
                v[:ns_] = r
                self.vreg(d)[8:] = 0
            else:
                v[ns_:2 * ns_] = r
        elif op in ("rev16", "rev32", "rev64"):
            n, w = _ARR[self.arr(d)]
            group = {"rev16": 2, "rev32": 4, "rev64": 8}[op] // w
            a = self.vreg(o[1]).view(_INT[w])[:n].copy()
            self.put(d, a.reshape(-1, group)[:, ::-1].ravel().astype(np.int64))
        elif op == "zip1":
            n, w = _ARR[self.arr(d)]
            a = self.vreg(o[1]).view(_INT[w])[:n].copy()
            b = self.vreg(o[2]).view(_INT[w])[:n].copy()
            r = np.empty(n, _INT[w])
            r[0::2], r[1::2] = a[: n // 2], b[: n // 2]
            self.put(d, r.astype(np.int64))
        elif op in ("trn1", "trn2"):
            n, w = _ARR[self.arr(d)]
            a = self.vreg(o[1]).view(_INT[w])[:n].copy()
            b = self.vreg(o[2]).view(_INT[w])[:n].copy()
            off = 0 if op == "trn1" else 1
            r = np.empty(n, _INT[w])
            r[0::2], r[1::2] = a[off::2], b[off::2]
            self.put(d, r.astype(np.int64))
        elif op == "fneg":
            # flip the sign bit of every lane (exact for any bit pattern)
            n, w = _ARR[self.arr(d)]
            a = self.vreg(o[1]).view(_INT[w])[:n].astype(np.int64)
            self.put(d, a ^ (-(1 << (8 * w - 1))))
        elif op == "sqneg":
            _, w = _ARR[self.arr(d)]
            self.put(d, np.clip(-self.lanes(o[1]), -(1 << (8 * w - 1)), (1 << (8 * w - 1)) - 1))
        elif op in ("uzp1", "uzp2"):
            n, w = _ARR[self.arr(d)]
            a = self.vreg(o[1]).view(_INT[w])[:n].copy()
            b = self.vreg(o[2]).view(_INT[w])[:n].copy()
            off = 0 if op == "uzp1" else 1
            self.put(d, np.concatenate([a[off::2], b[off::2]]).astype(np.int64))
        elif op == "ext":
            n, _ = _ARR[self.arr(d)]
            cat = np.concatenate([self.vreg(o[1])[:n].copy(), self.vreg(o[2])[:n].copy()])
            i = self.imm(o[3])
            v = self.vreg(d)
            v[:n] = cat[i:i + n]
            if n == 8:
                v[8:] = 0
        elif op == "dup":
            n, w = _ARR[self.arr(d)]
            self.put(d, np.full(n, self.elem(o[1]), np.int64))
        else:
            raise NotImplementedError(op)
        return None
