"""compute_quotient_values on the GPU: a chip's constraints as a register program.

The reference evaluates each chip's AIR over the quotient domain with
Plonky3's ProverConstraintFolder (vm/src/machine/utils.rs:201-350,
vm/src/machine/folder.rs:170-330): for every point the folder walks the
chip's `eval`, and each `assert_zero` / `assert_zero_ext` does
acc = acc * alpha + constraint; the quotient is acc * inv_zerofier.

Here the chip's constraints arrive as a straight-line program over base and
extension registers -- what a Rust shim emits by walking the chip's symbolic
constraints (Plonky3's SymbolicExpression, the same DAG the reference already
builds to infer constraint degrees, vm/src/machine/utils.rs:359-398).
`ConstraintBuilder` is that emitter for Python callers and tests: it mirrors
the AirBuilder surface (main / preprocessed / permutation columns, local and
next rows, public values, first-row / last-row / transition selectors,
permutation challenges, cumulative sums, assert_zero) and allocates registers.

Program format (one instruction = 4 u32: op, dst, a, b; `b` = 1 reads the
next row for the trace loads):
  MAIN/PREP dst<-col a        PERM ext dst<-EF column a
  CONST dst<-a (Monty)        PUBLIC dst<-public_values[a]
  FIRST/LAST/TRANSITION dst   ADD/SUB/MUL dst<-a op b (base)
  EADD/ESUB/EMUL (extension)  EMB ext dst<-base a   EMULB ext dst<-ext a * base b
  CHALLENGE ext dst<-perm_challenges[a]   REGIONAL ext dst<-regional sum
  GLOBAL dst<-global cumulative sum coordinate a (0..13)
  ASSERT base a / EASSERT ext a: acc = acc * alpha + register
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from . import fields as F

OPS = {"MAIN": 1, "PREP": 2, "PERM": 3, "CONST": 4, "PUBLIC": 5, "FIRST": 6, "LAST": 7, "TRANSITION": 8,
       "ADD": 9, "SUB": 10, "MUL": 11, "EADD": 12, "ESUB": 13, "EMUL": 14, "EMB": 15, "EMULB": 16,
       "CHALLENGE": 17, "REGIONAL": 18, "GLOBAL": 19, "ASSERT": 20, "EASSERT": 21}
MAX_BASE_REGS = 64
MAX_EXT_REGS = 16


class Expr:
    """A value of the program: base (`ext` False) or degree-4 extension."""

    def __init__(self, b: "ConstraintBuilder", vid: int, ext: bool):
        self.b, self.vid, self.ext = b, vid, ext

    def _bin(self, other, op):
        return self.b._binop(op, self, self.b._lift(other))

    def __add__(self, o):
        return self._bin(o, "ADD")

    def __radd__(self, o):
        return self.b._lift(o)._bin(self, "ADD")

    def __sub__(self, o):
        return self._bin(o, "SUB")

    def __rsub__(self, o):
        return self.b._lift(o)._bin(self, "SUB")

    def __mul__(self, o):
        return self._bin(o, "MUL")

    def __rmul__(self, o):
        return self.b._lift(o)._bin(self, "MUL")

    def __neg__(self):
        return self.b.const(0) - self


class _When:
    def __init__(self, b: "ConstraintBuilder", sel: Expr):
        self.b, self.sel = b, sel

    def assert_zero(self, x):
        self.b.assert_zero(self.sel * self.b._lift(x))

    def assert_eq(self, x, y):
        self.assert_zero(self.b._lift(x) - self.b._lift(y))


class ConstraintBuilder:
    """Records a chip's constraints as SSA values, then emits a register program."""

    def __init__(self):
        self._ops = []  # (op, dst vid or None, ext flag of dst, a, b, operand vids)
        self._n = 0

    # ---- values
    def _new(self, op, ext, a=0, b=0, args=()):
        vid = self._n
        self._n += 1
        self._ops.append((op, vid, ext, a, b, tuple(args)))
        return Expr(self, vid, ext)

    def _lift(self, x):
        if isinstance(x, Expr):
            return x
        return self.const(int(x))

    def main(self, col: int, next_row: bool = False) -> Expr:
        return self._new("MAIN", False, col, int(next_row))

    def preprocessed(self, col: int, next_row: bool = False) -> Expr:
        return self._new("PREP", False, col, int(next_row))

    def permutation(self, col: int, next_row: bool = False) -> Expr:
        return self._new("PERM", True, col, int(next_row))

    def const(self, canonical: int) -> Expr:
        return self._new("CONST", False, int(canonical))

    def public(self, i: int) -> Expr:
        return self._new("PUBLIC", False, i)

    def is_first_row(self) -> Expr:
        return self._new("FIRST", False)

    def is_last_row(self) -> Expr:
        return self._new("LAST", False)

    def is_transition(self) -> Expr:
        return self._new("TRANSITION", False)

    def challenge(self, i: int) -> Expr:
        return self._new("CHALLENGE", True, i)

    def regional_cumulative_sum(self) -> Expr:
        return self._new("REGIONAL", True)

    def global_cumulative_sum(self, coord: int) -> Expr:
        return self._new("GLOBAL", False, coord)

    def _binop(self, op, x: Expr, y: Expr) -> Expr:
        if not x.ext and not y.ext:
            return self._new(op, False, args=(x.vid, y.vid))
        if op == "MUL" and x.ext != y.ext:
            e, s = (x, y) if x.ext else (y, x)
            return self._new("EMULB", True, args=(e.vid, s.vid))
        xe = x if x.ext else self._new("EMB", True, args=(x.vid,))
        ye = y if y.ext else self._new("EMB", True, args=(y.vid,))
        return self._new("E" + op, True, args=(xe.vid, ye.vid))

    # ---- assertions (AirBuilder surface)
    def assert_zero(self, x):
        x = self._lift(x)
        self._ops.append(("EASSERT" if x.ext else "ASSERT", None, False, 0, 0, (x.vid,)))

    def assert_eq(self, x, y):
        self.assert_zero(self._lift(x) - self._lift(y))

    def when_first_row(self) -> _When:
        return _When(self, self.is_first_row())

    def when_last_row(self) -> _When:
        return _When(self, self.is_last_row())

    def when_transition(self) -> _When:
        return _When(self, self.is_transition())

    def when(self, cond) -> _When:
        return _When(self, self._lift(cond))

    # ---- emission
    def program(self, field) -> np.ndarray:
        """(n, 4) uint32 program with registers allocated by last use."""
        f = F.field_id(field)
        last = {}
        for k, (_, _, _, _, _, args) in enumerate(self._ops):
            for v in args:
                last[v] = k
        free = {False: list(range(MAX_BASE_REGS - 1, -1, -1)), True: list(range(MAX_EXT_REGS - 1, -1, -1))}
        reg, kind = {}, {}
        out = []
        for k, (op, dst, ext, a, b, args) in enumerate(self._ops):
            regs = [reg[v] for v in args]
            for v in args:  # operands read before the destination is written: their registers may be reused
                if last[v] == k and v in reg:
                    free[kind[v]].append(reg.pop(v))
            d = 0
            if dst is not None:
                if dst not in last:  # never used: still evaluated into a scratch register
                    pass
                if not free[ext]:
                    raise ValueError(f"program needs more than {MAX_EXT_REGS if ext else MAX_BASE_REGS} "
                                     f"{'extension' if ext else 'base'} registers")
                d = free[ext].pop()
                if dst in last:
                    reg[dst], kind[dst] = d, ext
                else:
                    free[ext].append(d)
            if op == "CONST":
                a = F.monty(f, a)
            if args:
                a = regs[0]
                b = regs[1] if len(regs) > 1 else 0
            out.append((OPS[op], d, a, b))
        return np.array(out, dtype=np.uint32).reshape(-1, 4)


def compute_quotient_values(ctx, program: np.ndarray, log_trace: int, log_quotient_degree: int, main,
                            preprocessed=None, permutation=None, public_values=(), perm_challenges=None,
                            regional_sum=None, global_sum=None, alpha=None, out=None, chunks: bool = False):
    """pico_gpu_quotient_values: the chip's quotient on the quotient domain
    GENERATOR * <w_Q>, Q = 2^(log_trace + log_quotient_degree), natural order,
    (Q, 4) Monty words.  main / preprocessed / permutation are (ProverData,
    matrix index) pairs of resident commits (None: absent), committed with
    the standard LDE shift and a blowup >= log_quotient_degree.  `out`: a
    device tensor of Q x 4 int32 to fill in place, else a host array is
    returned.  chunks=True (PICO_QUOTIENT_CHUNKS): the output is the
    2^log_quotient_degree chunks split_evals makes, chunk j (rows j n ..
    (j + 1) n) holding points j, j + D, ...; a host result is then shaped
    (D, n, 4), ready for commit_quotient_chunks."""
    from .pcs import _is_device

    lib = ctx.lib

    def ref(x):
        r = abi.TraceRef()
        if x is not None:
            pd, idx = x
            r.commit = pd.handle
            r.mat_idx = idx
        return r

    prog = np.ascontiguousarray(program, dtype=np.uint32).reshape(-1, 4)
    pub = np.ascontiguousarray(np.asarray(public_values, dtype=np.uint32).reshape(-1))
    chal = np.ascontiguousarray(np.zeros((0, 4), np.uint32) if perm_challenges is None else perm_challenges,
                                dtype=np.uint32).reshape(-1, 4)
    reg = np.ascontiguousarray(np.zeros(4, np.uint32) if regional_sum is None else regional_sum, dtype=np.uint32)
    glob = np.ascontiguousarray(np.zeros(14, np.uint32) if global_sum is None else global_sum, dtype=np.uint32)
    al = np.ascontiguousarray(alpha, dtype=np.uint32)
    Q = 1 << (log_trace + log_quotient_degree)
    flags = abi.PICO_QUOTIENT_CHUNKS if chunks else 0
    if out is None:
        host = np.zeros((Q, 4), dtype=np.uint32)
        optr = host.ctypes.data
    else:
        if not _is_device(out):
            raise ValueError("out must be a device tensor")
        flags |= abi.PICO_OUTPUT_DEVICE
        optr = out.data_ptr()
    abi.check(lib.pico_gpu_quotient_values(
        ctx.handle, ref(preprocessed), ref(main), ref(permutation), log_trace, log_quotient_degree,
        prog.ctypes.data, prog.shape[0], pub.ctypes.data if pub.size else None, pub.size,
        chal.ctypes.data if chal.size else None, chal.shape[0], reg.ctypes.data, glob.ctypes.data, al.ctypes.data,
        optr, flags))
    if out is not None:
        return out
    return host.reshape(1 << log_quotient_degree, 1 << log_trace, 4) if chunks else host


def quotient_chunk_domains(field, log_trace: int, log_quotient_degree: int):
    """The chunks' domains (split_domains of the quotient domain GENERATOR * <w_Q>):
    chunk j lives on GENERATOR * w_Q^j * <w_n>."""
    from .pcs import TwoAdicDomain

    f = F.field_id(field)
    p = F.P[f]
    wq = F.two_adic_generator(f, log_trace + log_quotient_degree)
    return [TwoAdicDomain(log_trace, F.GENERATOR[f] * pow(wq, j, p) % p) for j in range(1 << log_quotient_degree)]


def commit_quotient_chunks(pcs, chunks, log_trace: int, log_quotient_degree: int, keep: bool = True):
    """Commit a chip's quotient chunks as the prover does after
    compute_quotient_values (vm/src/machine/prover.rs:513-538): chunk j, n EF4
    values (host (n, 4) arrays or device tensors, e.g. views of a chunked
    output), on its split domain, as an extension matrix."""
    doms = quotient_chunk_domains(pcs.field, log_trace, log_quotient_degree)
    traces = [c.reshape(1 << log_trace, 1, 4) for c in chunks]
    return pcs.commit(list(zip(doms, traces)), keep=keep)
