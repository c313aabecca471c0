"""A small AArch64 (A64 + AdvSIMD) interpreter for the reference's kernels.

TEST INFRASTRUCTURE ONLY.  The reference's SGEMM/DGEMM kernels are single
``asm volatile`` blocks of AArch64 NEON assembly (NN_LIB/test_SMM_NT.c:6,
NN_LIB/test_temp.c:6, NN_LIB/test_temp_L1.c:4, NN_LIB/DGEMM_NN.c:5) that
cannot be compiled or run on an x86 host.  This module executes the
reference's own instruction text: it extracts the assembly string from the C
source, expands its ``.macro`` blocks, resolves labels, and interprets the
instruction subset those kernels use (integer address arithmetic, flags and
branches, vector loads/stores, and IEEE single/double multiply, add and fused
multiply-add with round-to-nearest-even).  Its outputs are the golden vectors
that pin the oracle's restatement of the reference's rounding order
(``tests/golden/make_golden.py`` runs it; nothing at test or bench time
imports the reference).

Fused multiply-add is computed exactly: the oracle's C library calls
``fmaf``/``fma`` (correctly rounded by C99), one call per vector instruction.
"""
from __future__ import annotations

import ctypes
import re

import numpy as np

from oracle import oracle as _orc

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def _fma_fns():
    L = _orc.lib()
    f = L.orc_fma_f32_vec
    f.restype = None
    f.argtypes = [ctypes.c_long, _f32p, _f32p, _f32p, _f32p]
    d = L.orc_fma_f64_vec
    d.restype = None
    d.argtypes = [ctypes.c_long, _f64p, _f64p, _f64p, _f64p]
    return f, d


# --------------------------------------------------------------------------
# extraction of the assembly text from the C source
# --------------------------------------------------------------------------

def _strip_c_comments(src: str) -> str:
    out, i, n, in_str = [], 0, len(src), False
    while i < n:
        c = src[i]
        if in_str:
            out.append(c)
            if c == "\\" and i + 1 < n:
                out.append(src[i + 1])
                i += 2
                continue
            if c == '"':
                in_str = False
            i += 1
            continue
        if c == '"':
            in_str = True
            out.append(c)
            i += 1
        elif src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    return "".join(out)


def extract_asm(path: str, func: str) -> tuple[list[str], list[str]]:
    """Returns (assembly lines, operand names) of the asm block in `func`."""
    src = _strip_c_comments(open(path, encoding="utf-8", errors="replace").read())
    m = re.search(r"\b" + re.escape(func) + r"\s*\([^)]*\)\s*\{", src)
    if not m:
        raise ValueError(f"{func} not found in {path}")
    a = src.index("asm", m.end())
    p = src.index("(", a)
    # collect string literals up to the first ':' outside strings at depth 1
    i, depth, lits = p + 1, 1, []
    while True:
        c = src[i]
        if c == '"':
            j = i + 1
            while src[j] != '"':
                j += 2 if src[j] == "\\" else 1
            lits.append(src[i + 1:j])
            i = j + 1
            continue
        if c == ":" and depth == 1:
            break
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        i += 1
    ops_end = src.index(";", i)
    names = re.findall(r"\[(\w+)\]\s*\"", src[i:ops_end])
    text = "".join(lits).replace("\\n", "\n").replace("\\t", " ")
    return text.split("\n"), names


# --------------------------------------------------------------------------
# program: macro expansion, labels, decoded instructions
# --------------------------------------------------------------------------

def build_program(lines: list[str]):
    macros, body, cur = {}, [], None
    for raw in lines:
        s = raw.strip()
        if not s:
            continue
        if s.startswith(".macro"):
            cur = s.split()[1]
            macros[cur] = []
            continue
        if s.startswith(".endm"):
            cur = None
            continue
        (macros[cur] if cur else body).append(s)

    def expand(seq, depth=0):
        out = []
        for s in seq:
            w = s.split()[0]
            if w in macros and len(s.split()) == 1:
                out.extend(expand(macros[w], depth + 1))
            else:
                out.append(s)
        return out

    flat = expand(body)
    prog, labels = [], {}
    for s in flat:
        if s.endswith(":") and " " not in s:
            labels[s[:-1]] = len(prog)
            continue
        if s.startswith("."):
            raise ValueError(f"unsupported directive {s}")
        m = re.match(r"([a-z][a-z0-9.]*)\s*(.*)", s)
        prog.append((m.group(1), m.group(2).strip()))
    return prog, labels


# --------------------------------------------------------------------------
# machine
# --------------------------------------------------------------------------

_MASK = (1 << 64) - 1


class Memory:
    """Flat address space of a few buffers.  The reference's software-pipelined
    loops load one vector past the end of A or B on their last iteration (a
    load whose value is never used); reads that fall in the GUARD bytes after
    a buffer return NaN bit patterns, so a guard value that reached the result
    would show up as NaN.  Writes outside a buffer raise."""
    GUARD = 4096

    def __init__(self):
        self.regions = []  # (base, uint8 array)
        self.guard_reads = 0

    def add(self, base: int, arr: np.ndarray) -> int:
        self.regions.append((base, arr.view(np.uint8).reshape(-1)))
        return base

    def _find(self, addr: int, n: int):
        for base, a in self.regions:
            if base <= addr and addr + n <= base + a.size:
                return a, addr - base
        raise IndexError(f"access of {n} bytes at {addr:#x} outside every buffer")

    def read(self, addr: int, n: int) -> np.ndarray:
        for base, a in self.regions:
            if base <= addr and addr + n <= base + a.size:
                o = addr - base
                return a[o:o + n].copy()
            if base <= addr < base + a.size + self.GUARD:
                # straddles or lies in the guard zone after the buffer
                self.guard_reads += 1
                out = np.frombuffer(np.full(n // 4, np.nan, np.float32).tobytes(), np.uint8).copy()
                o = addr - base
                k = max(0, min(n, a.size - o))
                out[:k] = a[o:o + k]
                return out
        raise IndexError(f"access of {n} bytes at {addr:#x} outside every buffer")

    def write(self, addr: int, data: np.ndarray) -> None:
        data = np.ascontiguousarray(data).view(np.uint8).reshape(-1)
        a, o = self._find(addr, data.size)
        a[o:o + data.size] = data


class Machine:
    def __init__(self, prog, labels, params: dict, mem: Memory, sp: int):
        self.prog, self.labels, self.params, self.mem = prog, labels, params, mem
        self.x = [0] * 31
        self.sp = sp
        self.v = np.zeros((32, 16), np.uint8)
        self.N = self.Z = self.C = self.V = False
        self.fma32, self.fma64 = _fma_fns()
        self.count = 0
        self.cache = {}

    # ---- register helpers ----
    def rx(self, tok: str) -> int:
        tok = tok.strip()
        if tok == "sp":
            return self.sp
        if tok in ("xzr", "wzr"):
            return 0
        return self.x[int(tok[1:])]

    def wx(self, tok: str, val: int) -> None:
        tok = tok.strip()
        val &= _MASK
        if tok == "sp":
            self.sp = val
        elif tok not in ("xzr", "wzr"):
            self.x[int(tok[1:])] = val

    def f32(self, i):
        return self.v[i].view(np.float32)

    def f64(self, i):
        return self.v[i].view(np.float64)

    @staticmethod
    def vreg(tok):
        m = re.match(r"[vqdsb](\d+)", tok.strip())
        return int(m.group(1))

    def imm(self, tok):
        tok = tok.strip().lstrip("#")
        return int(tok, 0)

    def addr(self, ops):
        """memory operand(s): '[xN]', '[xN, #i]', '[xN], #i' -> (address, writeback)"""
        m = re.match(r"\[(\w+)(?:\s*,\s*#(-?\w+))?\]\s*(?:,\s*#(-?\w+))?$", ops.strip())
        base, off, post = m.group(1), m.group(2), m.group(3)
        a = self.rx(base) + (int(off, 0) if off else 0)
        wb = (base, self.rx(base) + int(post, 0)) if post else None
        return a & _MASK, wb

    def flags_sub(self, a, b):
        r = (a - b) & _MASK
        self.N = bool(r >> 63)
        self.Z = r == 0
        self.C = (a & _MASK) >= (b & _MASK)
        sa, sb, sr = a >> 63 & 1, b >> 63 & 1, r >> 63 & 1
        self.V = (sa != sb) and (sr != sa)
        return r

    # ---- float helpers (exact FMA through C) ----
    def fma_f32(self, a, b, c):
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        c = np.ascontiguousarray(c, np.float32)
        out = np.empty_like(a)
        self.fma32(a.size, a, b, c, out)
        return out

    def fma_f64(self, a, b, c):
        a = np.ascontiguousarray(a, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        c = np.ascontiguousarray(c, np.float64)
        out = np.empty_like(a)
        self.fma64(a.size, a, b, c, out)
        return out

    # ---- execution ----
    def run(self, max_steps=50_000_000):
        pc, prog = 0, self.prog
        while pc < len(prog):
            self.count += 1
            if self.count > max_steps:
                raise RuntimeError("step limit")
            op, args = prog[pc]
            pc += 1
            nxt = self.step(op, args)
            if nxt is not None:
                pc = nxt

    def _vec_operands(self, args):
        parts = [p.strip() for p in re.split(r",(?![^\[]*\])", args)]
        return parts

    def step(self, op, args):
        if op == "prfm":
            return None
        if op in ("b", "beq", "bne", "bgt", "blt", "bge", "ble"):
            take = {"b": True, "beq": self.Z, "bne": not self.Z,
                    "bgt": (not self.Z) and (self.N == self.V), "blt": self.N != self.V,
                    "bge": self.N == self.V, "ble": self.Z or (self.N != self.V)}[op]
            return self.labels[args.strip()] if take else None
        if op in ("fmul", "fmla", "fadd"):
            return self._farith(op, args)
        if op == "faddp":
            return self._faddp(args)
        if op == "fmadd":
            d, n, m, a = [t.strip() for t in args.split(",")]
            dbl = d.startswith("d")
            vd, vn, vm, va = (self.vreg(t) for t in (d, n, m, a))
            if dbl:
                r = self.fma_f64(self.f64(vn)[:1], self.f64(vm)[:1], self.f64(va)[:1])
                self.v[vd] = 0
                self.f64(vd)[0] = r[0]
            else:
                r = self.fma_f32(self.f32(vn)[:1], self.f32(vm)[:1], self.f32(va)[:1])
                self.v[vd] = 0
                self.f32(vd)[0] = r[0]
            return None
        if op == "ins":
            d, s = [t.strip() for t in args.split(",")]
            md = re.match(r"v(\d+)\.([sd])\[(\d)\]", d)
            ms = re.match(r"v(\d+)\.([sd])\[(\d)\]", s)
            if md.group(2) == "s":
                self.f32(int(md.group(1)))[int(md.group(3))] = self.f32(int(ms.group(1)))[int(ms.group(3))]
            else:
                self.f64(int(md.group(1)))[int(md.group(3))] = self.f64(int(ms.group(1)))[int(ms.group(3))]
            return None
        if op == "dup":
            d, s = [t.strip() for t in args.split(",")]
            assert s == "wzr" and d.endswith(".4s")
            self.v[self.vreg(d)] = 0
            return None
        if op in ("ldr", "str", "ldp", "stp"):
            return self._ldst(op, args)
        if op in ("ld1", "ld2", "ld3", "ld4", "st1", "st2", "st3", "st4"):
            return self._ldst_struct(op, args)
        return self._integer(op, args)

    def _farith(self, op, args):
        d, n, m = self._vec_operands(args)
        md = re.match(r"v(\d+)\.(\d)([sd])", d)
        vd, lanes, kind = int(md.group(1)), int(md.group(2)), md.group(3)
        vn = self.vreg(n)
        view = self.f32 if kind == "s" else self.f64
        nv = view(vn)[:lanes].copy()
        mm = re.match(r"v(\d+)\.([sd])\[(\d)\]", m)
        if mm:
            mv = np.full(lanes, view(int(mm.group(1)))[int(mm.group(3))])
        else:
            mv = view(self.vreg(m))[:lanes].copy()
        dv = view(vd)[:lanes].copy()
        if op == "fmul":
            r = nv * mv
        elif op == "fadd":
            r = nv + mv
        else:
            r = (self.fma_f32 if kind == "s" else self.fma_f64)(nv, mv, dv)
        full = lanes * (4 if kind == "s" else 8) == 16
        if not full:
            self.v[vd] = 0  # 64-bit vector writes clear the upper half
        view(vd)[:lanes] = r
        return None

    def _faddp(self, args):
        d, *rest = self._vec_operands(args)
        d = d.strip()
        if d.startswith("v"):
            n, m = rest
            vd, vn, vm = self.vreg(d), self.vreg(n), self.vreg(m)
            a, b = self.f32(vn).copy(), self.f32(vm).copy()
            self.f32(vd)[:] = np.array([a[0] + a[1], a[2] + a[3], b[0] + b[1], b[2] + b[3]],
                                       np.float32)
        elif d.startswith("s"):
            vd, vn = self.vreg(d), self.vreg(rest[0])
            a = self.f32(vn).copy()
            self.v[vd] = 0
            self.f32(vd)[0] = a[0] + a[1]
        else:
            vd, vn = self.vreg(d), self.vreg(rest[0])
            a = self.f64(vn).copy()
            self.v[vd] = 0
            self.f64(vd)[0] = a[0] + a[1]
        return None

    def _ldst(self, op, args):
        if op in ("ldr", "str"):
            m = re.match(r"(\w+)\s*,\s*(.*)$", args)
            reg, mem = m.group(1), m.group(2)
            if mem.startswith("%["):
                self.wx(reg, int(self.params[mem[2:-1]]))
                return None
            size = {"q": 16, "d": 8, "s": 4}[reg[0]]
            a, wb = self.addr(mem)
            vr = self.vreg(reg)
            if op == "ldr":
                data = self.mem.read(a, size)
                self.v[vr] = 0
                self.v[vr][:size] = data
            else:
                self.mem.write(a, self.v[vr][:size])
            if wb:
                self.wx(*wb)
            return None
        m = re.match(r"(\w+)\s*,\s*(\w+)\s*,\s*(.*)$", args)
        r1, r2, mem = m.group(1), m.group(2), m.group(3)
        a, wb = self.addr(mem)
        v1, v2 = self.vreg(r1), self.vreg(r2)
        if op == "ldp":
            data = self.mem.read(a, 32)
            self.v[v1] = data[:16]
            self.v[v2] = data[16:]
        else:
            self.mem.write(a, np.concatenate([self.v[v1], self.v[v2]]))
        if wb:
            self.wx(*wb)
        return None

    def _ldst_struct(self, op, args):
        """ldN / stN, N = 1..4, on 32- or 64-bit elements: the single-lane form
        {Vt.s, ...}[lane] moves element `lane` of each register to / from N
        consecutive elements; the multiple-structure form {Vt.4s, ...}
        interleaves N registers element by element (N = 1 with several
        registers: consecutive registers)."""
        m = re.match(r"\{([^}]*)\}(\[(\d)\])?\s*,\s*(.*)$", args)
        regs = [r.strip() for r in m.group(1).split(",")]
        lane = int(m.group(3)) if m.group(3) is not None else None
        a, wb = self.addr(m.group(4))
        nst = int(op[2])
        load = op.startswith("ld")
        arr = re.match(r"v\d+\.(\d*)([sd])", regs[0])
        esize = 4 if arr.group(2) == "s" else 8
        dt = np.float32 if esize == 4 else np.float64
        vr = [self.vreg(r) for r in regs]

        def view(r):
            return self.v[r].view(dt)
        if lane is not None:
            assert len(vr) == nst, args
            if load:
                data = self.mem.read(a, esize * nst).view(dt)
                for i, r in enumerate(vr):
                    view(r)[lane] = data[i]
            else:
                self.mem.write(a, np.array([view(r)[lane] for r in vr], dt))
        else:
            lanes = int(arr.group(1)) if arr.group(1) else 16 // esize
            nbytes = esize * lanes * len(vr)
            if nst == 1:
                # consecutive registers, no interleave
                if load:
                    data = self.mem.read(a, nbytes)
                    for i, r in enumerate(vr):
                        self.v[r] = 0
                        self.v[r][:esize * lanes] = data[i * esize * lanes:(i + 1) * esize * lanes]
                else:
                    self.mem.write(a, np.concatenate([self.v[r][:esize * lanes] for r in vr]))
            else:
                assert len(vr) == nst, args
                if load:
                    data = self.mem.read(a, nbytes).view(dt).reshape(lanes, nst)
                    for i, r in enumerate(vr):
                        self.v[r] = 0
                        view(r)[:lanes] = data[:, i]
                else:
                    data = np.stack([view(r)[:lanes] for r in vr], axis=1).astype(dt)
                    self.mem.write(a, data.reshape(-1).view(np.uint8))
        if wb:
            self.wx(*wb)
        return None

    def _integer(self, op, args):
        t = [s.strip() for s in args.split(",")]
        if op == "mov":
            self.wx(t[0], self.imm(t[1]) if t[1].startswith("#") else self.rx(t[1]))
        elif op in ("add", "sub"):
            a = self.rx(t[1])
            if t[2].startswith("#"):
                b = self.imm(t[2])
            else:
                b = self.rx(t[2])
                if len(t) > 3:
                    sh = re.match(r"lsl\s*#(\d+)", t[3])
                    b = b << int(sh.group(1))
            self.wx(t[0], a + b if op == "add" else a - b)
        elif op == "subs":
            self.wx(t[0], self.flags_sub(self.rx(t[1]), self.imm(t[2])))
        elif op == "cmp":
            self.flags_sub(self.rx(t[0]), self.imm(t[1]))
        elif op == "ands":
            r = self.rx(t[1]) & self.imm(t[2])
            self.N, self.Z, self.C, self.V = bool(r >> 63), r == 0, False, False
            self.wx(t[0], r)
        elif op == "lsr":
            self.wx(t[0], self.rx(t[1]) >> self.imm(t[2]))
        elif op == "lsl":
            self.wx(t[0], self.rx(t[1]) << self.imm(t[2]))
        elif op == "udiv":
            b = self.rx(t[2])
            self.wx(t[0], 0 if b == 0 else self.rx(t[1]) // b)
        elif op == "mul":
            self.wx(t[0], self.rx(t[1]) * self.rx(t[2]))
        elif op == "msub":
            self.wx(t[0], self.rx(t[3]) - self.rx(t[1]) * self.rx(t[2]))
        else:
            raise NotImplementedError(f"{op} {args}")
        return None


# --------------------------------------------------------------------------
# running a reference kernel
# --------------------------------------------------------------------------

BASE_A, BASE_B, BASE_C, BASE_SB, STACK_TOP = 0x10_0000_0000, 0x20_0000_0000, 0x30_0000_0000, \
    0x40_0000_0000, 0x7F_0000_0000


def run_kernel(path: str, func: str, A: np.ndarray, B: np.ndarray, C: np.ndarray,
               M: int, N: int, K: int, sb_elems: int = 0, stack_bytes: int = 1 << 20):
    """Executes the reference kernel `func` of `path` on copies of A and B;
    writes into C (which keeps its initial contents where the kernel does not
    store).  Returns the number of instructions executed."""
    lines, names = extract_asm(path, func)
    prog, labels = build_program(lines)
    mem = Memory()
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B)
    mem.add(BASE_A, A)
    mem.add(BASE_B, B)
    mem.add(BASE_C, C)
    stack = np.zeros(stack_bytes, np.uint8)
    mem.add(STACK_TOP - stack_bytes, stack)
    params = {"C": BASE_C, "A": BASE_A, "B": BASE_B, "M": M, "N": N, "K": K}
    if sb_elems:
        sb = np.zeros(sb_elems, A.dtype)
        mem.add(BASE_SB, sb)
        params["SB"] = BASE_SB
    missing = [n for n in names if n not in params]
    if missing:
        raise ValueError(f"unbound asm operands {missing}")
    mach = Machine(prog, labels, params, mem, sp=STACK_TOP)
    mach.run()
    if mach.sp != STACK_TOP:
        raise RuntimeError("stack pointer not restored")
    return mach.count


def run_asm(path: str, func: str, buffers: dict, params: dict, offsets: dict | None = None,
            stack_bytes: int = 1 << 20, _cache: dict = {}) -> int:
    """Executes the asm block of `func` with named buffers (numpy arrays,
    updated in place) and scalar operands.  `offsets` gives, per buffer
    operand, the element offset its pointer operand starts at.  Returns the
    number of instructions executed."""
    key = (path, func)
    if key not in _cache:
        lines, names = extract_asm(path, func)
        _cache[key] = (build_program(lines), names)
    (prog, labels), names = _cache[key]
    mem = Memory()
    p = dict(params)
    base = 0x10_0000_0000
    for name, arr in buffers.items():
        mem.add(base, arr)
        p[name] = base + (offsets or {}).get(name, 0) * arr.itemsize
        base += 0x10_0000_0000
    stack = np.zeros(stack_bytes, np.uint8)
    mem.add(STACK_TOP - stack_bytes, stack)
    missing = [n for n in names if n not in p]
    if missing:
        raise ValueError(f"unbound asm operands {missing}")
    mach = Machine(prog, labels, p, mem, sp=STACK_TOP)
    mach.run()
    if mach.sp != STACK_TOP:
        raise RuntimeError("stack pointer not restored")
    return mach.count
