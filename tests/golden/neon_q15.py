"""Interpreter for the AArch64/NEON instruction subset of PLFFT's Q0.15 kernels.

Test infrastructure only: make_q15_golden.py uses it, in the container that
holds the reference sources, to execute the reference's own generated q15
kernels (src/providers/aot/asm/neon/plfft_*q15*.S, read as text) on seeded
inputs.  The outputs become the committed fixture tests/golden/q15_reference.npz
that pins the bit-exact Q0.15 path.  Nothing at test time reads the reference.

Semantics implemented (Arm A64 definitions): integer loads/stores of
S/D/Q/X registers, address arithmetic, compare-and-branch, and the vector
ops sqadd, sqsub, srshr, sqrdmulh, smull(2), smlal(2), smlsl(2) (vector and
by-element), sqrshrn(2), rev32, zip1, trn1, trn2.
"""
import re

import numpy as np

MASK64 = (1 << 64) - 1


def _s64(v):
    v &= MASK64
    return v - (1 << 64) if v >> 63 else v


def _sat16(a):
    return np.clip(a, -32768, 32767)


class Kernels:
    """Parsed functions (name -> instruction list) and read-only data."""

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
        if ch == "[":
            depth += 1
        elif ch == "]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return out


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
        self.sp = self.stack_top
        self.v = [np.zeros(16, np.uint8) for _ in range(32)]
        self.nzcv = 0
        for i, a in enumerate(args):
            self.x[i] = int(a) & MASK64
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

    def imm(self, s):
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
        return self.v[int(re.match(r"[vqsdh](\d+)", s).group(1))]

    @staticmethod
    def arr(s):
        return s.split(".")[1] if "." in s else None

    def lanes16(self, s):
        """int64 array of the 16-bit lanes named by an arrangement (4h -> 4, 8h -> 8)."""
        r = self.vreg(s)
        n = 8 if self.arr(s) == "8h" else 4
        return r.view(np.int16)[:n].astype(np.int64)

    def put16(self, s, vals, clear_hi=True):
        r = self.vreg(s)
        n = 8 if self.arr(s) == "8h" else 4
        r.view(np.int16)[:n] = vals.astype(np.int16)
        if n == 4 and clear_hi:
            r[8:] = 0

    def elem16(self, s):
        m = re.match(r"v(\d+)\.h\[(\d+)\]", s)
        return int(self.v[int(m.group(1))].view(np.int16)[int(m.group(2))])

    # ---------------------------------------------------------------
    _VBYTES = {"s": 4, "d": 8, "q": 16}

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
        if op in ("sqadd", "sqsub"):
            a, b = self.lanes16(o[1]), self.lanes16(o[2])
            self.put16(d, _sat16(a + b if op == "sqadd" else a - b))
        elif op == "srshr":
            s = self.imm(o[2])
            self.put16(d, (self.lanes16(o[1]) + (1 << (s - 1))) >> s)
        elif op == "sqrdmulh":
            a = self.lanes16(o[1])
            b = self.elem16(o[2]) if "[" in o[2] else self.lanes16(o[2])
            self.put16(d, _sat16((2 * a * b + (1 << 15)) >> 16))
        elif op in ("smull", "smull2", "smlal", "smlal2", "smlsl", "smlsl2"):
            hi = op.endswith("2")
            a = self.vreg(o[1]).view(np.int16)[4:8 if hi else 4].astype(np.int64) if hi else \
                self.vreg(o[1]).view(np.int16)[:4].astype(np.int64)
            if "[" in o[2]:
                b = self.elem16(o[2])
            else:
                bv = self.vreg(o[2]).view(np.int16)
                b = (bv[4:8] if hi else bv[:4]).astype(np.int64)
            prod = a * b
            acc = self.vreg(d).view(np.int32).astype(np.int64)
            if op.startswith("smull"):
                res = prod
            elif op.startswith("smlal"):
                res = acc + prod
            else:
                res = acc - prod
            res = ((res + (1 << 31)) % (1 << 32)) - (1 << 31)  # 32-bit wrap
            self.vreg(d).view(np.int32)[:] = res.astype(np.int32)
        elif op in ("sqrshrn", "sqrshrn2"):
            s = self.imm(o[2])
            a = self.vreg(o[1]).view(np.int32).astype(np.int64)
            r = _sat16((a + (1 << (s - 1))) >> s).astype(np.int16)
            v = self.vreg(d)
            if op == "sqrshrn":
                v.view(np.int16)[:4] = r
                v[8:] = 0
            else:
                v.view(np.int16)[4:8] = r
        elif op == "rev32":
            a = self.lanes16(o[1])
            sw = a.reshape(-1, 2)[:, ::-1].ravel()
            self.put16(d, sw)
        elif op == "zip1":
            t = self.arr(d)
            n, m = self.vreg(o[1]).copy(), self.vreg(o[2]).copy()
            v = self.vreg(d)
            if t == "2s":
                v[:] = 0
                v[0:4], v[4:8] = n[0:4], m[0:4]
            elif t == "2d":
                v[0:8], v[8:16] = n[0:8], m[0:8]
            else:
                raise NotImplementedError(f"zip1 .{t}")
        elif op in ("trn1", "trn2"):
            n = self.vreg(o[1]).view(np.int16).copy()
            m = self.vreg(o[2]).view(np.int16).copy()
            off = 0 if op == "trn1" else 1
            r = np.empty(8, np.int16)
            r[0::2], r[1::2] = n[off::2], m[off::2]
            self.vreg(d).view(np.int16)[:] = r
        else:
            raise NotImplementedError(op)
        return None
