"""Generates field_asm.cuh: GF(2^255-19) multiply and square for sm_100a.

Eight 32-bit limbs, least significant first; inputs and outputs below 2^256
(not canonical). The 512-bit product is accumulated by operand scanning in 64-bit slots:
every partial product a_i*b_j is added as one 64-bit quantity (its low half
then its high half, back to back in one PTX carry chain), so the pair maps
to one wide multiply-add. Slots at even positions i+j go to one accumulator
and slots at odd positions to another, merged by one add chain at the end:
with a single accumulator a word is the high half of one slot and the low
half of the next, and the misaligned register pairs cost extra instructions
on the multiply pipe (on B200: 0.387 multiplications/clk/SM with one
accumulator, 0.411 with two). The 512-bit result is folded with
2^256 = 38 (mod 2^255-19) the same way.
(A one-level Karatsuba variant, 48 wide products plus carry corrections on
the ALU, measured no faster on sm_100a: the ALU work it adds cancels the
multiply-pipe work it saves.)

Each routine is one asm block so the carry flag never crosses a
compiler-visible boundary.

    python gen_field_asm.py > field_asm.cuh       # write the header
    python gen_field_asm.py --check               # simulate the PTX on random inputs
"""
import random
import sys


class Emit:
    """Accumulates PTX lines and tracks which accumulator words hold data."""

    def __init__(self, acc="t", words=17):
        self.lines = []
        self.acc = acc
        self.live = [False] * words

    def w(self, k):
        return f"{self.acc}{k}"

    def chain(self, prods, carry_to=None):
        """prods: list of (position, x, y); positions ascend by 2 so the 64-bit
        slots do not overlap. Adds every x*y at its position in one carry
        chain; the final carry goes to `carry_to` when given (a word that
        may be fresh), else is known to be zero."""
        ops = []
        for n, (p, x, y) in enumerate(prods):
            for half, q in (("lo", p), ("hi", p + 1)):
                ops.append((half, q, x, y))
        for n, (half, q, x, y) in enumerate(ops):
            first, last = n == 0, n == len(ops) - 1
            cc_in = not first
            cc_out = not last or carry_to is not None
            addend = self.w(q) if self.live[q] else "0"
            op = ("madc" if cc_in else "mad") + f".{half}" + (".cc" if cc_out else "") + ".u32"
            self.lines.append(f"{op} {self.w(q)}, {x}, {y}, {addend};")
            self.live[q] = True
        if carry_to is not None:
            src = self.w(carry_to) if self.live[carry_to] else "0"
            self.lines.append(f"addc.u32 {self.w(carry_to)}, {src}, 0;")
            self.live[carry_to] = True


def merge(E, O, L):
    """E += O over words 1..15 (the sum is below 2^512: no carry out)."""
    first = True
    for k in range(1, 16):
        dst = f"t{k}"
        src = dst if E.live[k] else "0"
        if O.live[k]:
            L.append(("add.cc.u32" if first else "addc.cc.u32") + f" {dst}, {src}, o{k};")
            first = False
        elif not first:
            L.append(f"addc.cc.u32 {dst}, {src}, 0;")
        else:
            continue
        E.live[k] = True
    L[-1] = L[-1].replace("addc.cc.u32", "addc.u32")


def mul_body(A, Bv):
    """Row i adds a_i * b into two accumulators: E takes the 64-bit slots at
    even positions i + j, O those at odd positions. Each accumulator only
    ever sees slots of one alignment, so every slot is an aligned register
    pair. Of a row's two chains, the one whose last slot ends at word i + 7
    carries into word i + 8; the other ends at word i + 8 and its carry is
    zero (each accumulator holds a subset of rows 0..i, below 2^(32*(i+9)))."""
    E, O = Emit("t"), Emit("o")
    O.lines = E.lines
    for i in range(8):
        j0 = i % 2  # j with i + j even
        ev = [(i + j, A(i), Bv(j)) for j in range(j0, 8, 2)]
        od = [(i + j, A(i), Bv(j)) for j in range(1 - j0, 8, 2)]
        E.chain(ev, carry_to=i + 8 if j0 == 0 else None)
        O.chain(od, carry_to=i + 8 if j0 == 1 else None)
    merge(E, O, E.lines)
    return E.lines


def sq_body(A):
    """Off-diagonal products a_i a_j (i < j) at odd positions into O, at even
    positions into E; then E += O, doubled, plus the squares a_i^2 (even
    positions, into E)."""
    E, O = Emit("t"), Emit("o")
    O.lines = E.lines
    for i in range(7):
        js = list(range(i + 1, 8))
        for acc, par in ((O, 1), (E, 0)):
            prods = [(i + j, A(i), A(j)) for j in js if (i + j) % 2 == par]
            if prods:
                c = prods[-1][0] + 2
                acc.chain(prods, carry_to=c if c <= 15 else None)
    L = E.lines
    merge(E, O, L)
    for k in range(16):
        if not E.live[k]:
            L.append(f"mov.u32 t{k}, 0;")
            E.live[k] = True
    # double t1..t15 (t0 is still empty; the doubled sum is below 2^512)
    L.append("add.cc.u32 t1, t1, t1;")
    for k in range(2, 15):
        L.append(f"addc.cc.u32 t{k}, t{k}, t{k};")
    L.append("addc.u32 t15, t15, t15;")
    # diagonal squares a_i^2 at position 2i: one chain of 64-bit slots
    diag = [(2 * i, A(i), A(i)) for i in range(8)]
    E.chain(diag, carry_to=None)
    return L


def reduce_tail():
    """t0..t15 -> %0..%7 with 2^256 = 38; the result is below 2^256."""
    e = Emit("r")
    L = []
    # r = t_lo, then r += 38 * t_hi by two chains of 64-bit slots
    for k in range(8):
        L.append(f"mov.u32 r{k}, t{k};")
        e.live[k] = True
    even = [(k, f"t{8 + k}", "38") for k in range(0, 8, 2)]
    odd = [(k, f"t{8 + k}", "38") for k in range(1, 8, 2)]
    e.chain(even, carry_to=8)
    e.chain(odd, carry_to=None)
    L += e.lines
    # value = r0..r7 + r8 * 2^256 with r8 < 39: fold once more
    L.append("mad.lo.cc.u32 r0, r8, 38, r0;")
    for k in range(1, 8):
        L.append(f"addc.cc.u32 r{k}, r{k}, 0;")
    L.append("addc.u32 r8, 0, 0;")
    # a carry here leaves r0..r7 below 38*39, so this add cannot carry
    L.append("mad.lo.u32 r0, r8, 38, r0;")
    for k in range(8):
        L.append(f"mov.u32 %{k}, r{k};")
    return L


def reduce_tail_fold16():
    """t0..t15 -> %0..%7 with 2^256 = 38, the high words folded by 16-bit
    halves: t = h 2^16 + l gives 38 t = 38 l + (38 h) 2^16, where 38 l and
    38 h are below 2^22 (narrow multiplies, no 64-bit result), and the byte
    permutes split (38 h) 2^16 into (38 h) << 16, added to its own word, and
    (38 h) >> 16, below 2^6, added to the next word. No wide multiply-add."""
    L = []
    for k in range(8):
        t = f"t{8 + k}"
        L.append(f"and.b32 l{k}, {t}, 65535;")
        L.append(f"prmt.b32 h{k}, {t}, 0, 17458;")  # 0x4432: t >> 16
        L.append(f"mul.lo.u32 l{k}, l{k}, 38;")
        L.append(f"mul.lo.u32 h{k}, h{k}, 38;")
    for k in range(8):
        L.append(f"prmt.b32 x{k}, h{k}, 0, 4164;")  # 0x1044: (38 h) << 16
        L.append(f"prmt.b32 y{k}, h{k}, 0, 17458;")  # (38 h) >> 16
    # the small addends of each word: 38 l_k plus the spill of word k - 1
    L.append("mov.u32 s0, l0;")
    for k in range(1, 8):
        L.append(f"add.u32 s{k}, l{k}, y{k - 1};")
    L.append("add.cc.u32 r0, t0, x0;")
    for k in range(1, 8):
        L.append(f"addc.cc.u32 r{k}, t{k}, x{k};")
    L.append("addc.u32 r8, y7, 0;")
    L.append("add.cc.u32 r0, r0, s0;")
    for k in range(1, 8):
        L.append(f"addc.cc.u32 r{k}, r{k}, s{k};")
    L.append("addc.u32 r8, r8, 0;")
    # value = r0..r7 + r8 * 2^256 with r8 < 66: fold once more
    L.append("mad.lo.cc.u32 r0, r8, 38, r0;")
    for k in range(1, 8):
        L.append(f"addc.cc.u32 r{k}, r{k}, 0;")
    L.append("addc.u32 r8, 0, 0;")
    # a carry here leaves r0..r7 below 38*66, so this add cannot carry
    L.append("mad.lo.u32 r0, r8, 38, r0;")
    for k in range(8):
        L.append(f"mov.u32 %{k}, r{k};")
    return L


FOLD16 = "--fold16" in sys.argv
TAIL_REGS = "\\n\\t.reg .u32 l<8>;\\n\\t.reg .u32 h<8>;\\n\\t.reg .u32 x<8>;\\n\\t.reg .u32 y<8>;\\n\\t.reg .u32 s<8>;"


def tail():
    return reduce_tail_fold16() if FOLD16 else reduce_tail()


def emit_fn(name, body, nin, extra=""):
    out = []
    ins = ", ".join(f'"r"(a[{i}])' for i in range(8))
    if nin == 2:
        ins += ", " + ", ".join(f'"r"(b[{i}])' for i in range(8))
    sig = (
        "const uint32_t* __restrict__ a, const uint32_t* __restrict__ b"
        if nin == 2
        else "const uint32_t* __restrict__ a"
    )
    out.append(f"__device__ __forceinline__ void {name}(uint32_t* __restrict__ r, {sig}) {{")
    regs = TAIL_REGS if FOLD16 else ""
    out.append('    asm("{\\n\\t.reg .u32 t<17>;\\n\\t.reg .u32 o<17>;\\n\\t.reg .u32 r<9>;' + regs + '\\n\\t' + extra + '"')
    for line in body + tail():
        out.append(f'        "{line}\\n\\t"')
    out.append('        "}"')
    outs = ", ".join(f'"=r"(r[{i}])' for i in range(8))
    out.append(f"        : {outs}")
    out.append(f"        : {ins});")
    out.append("}")
    return "\n".join(out)


def operands():
    A = lambda i: f"%{8 + i}"
    Bv = lambda j: f"%{16 + j}"
    return A, Bv


def header():
    A, Bv = operands()
    parts = [
        "// Generated by gen_field_asm.py — do not edit by hand.",
        "// GF(2^255-19): r = a*b and r = a^2, eight 32-bit limbs, result below 2^256.",
        "#pragma once",
        "#include <cstdint>",
        "",
        emit_fn("fe_mul_asm", mul_body(A, Bv), 2),
        "",
        emit_fn("fe_sq_asm", sq_body(A), 1),
        "",

    ]
    return "\n".join(parts)


# ---- a small interpreter of the PTX subset above, for --check ----------------

M32 = (1 << 32) - 1


def simulate(lines, args):
    regs = {}
    cc = 0

    def val(x):
        if x.startswith("%"):
            return args[int(x[1:])]
        if x[0].isdigit():
            return int(x)
        return regs[x]

    out = {}
    for line in lines:
        line = line.rstrip(";")
        op, rest = line.split(" ", 1)
        ops = [s.strip() for s in rest.split(",")]
        parts = op.split(".")
        base = parts[0]
        dst = ops[0]
        if base in ("mad", "madc", "mul"):
            half = parts[1]
            x, y = val(ops[1]), val(ops[2])
            prod = x * y
            v = (prod & M32) if half == "lo" else (prod >> 32)
            if base == "mul":
                res = v
                carry = 0
            else:
                add = val(ops[3])
                cin = cc if base == "madc" else 0
                s = v + add + cin
                res, carry = s & M32, s >> 32
            if ".cc" in op:
                cc = carry
            elif base != "mul" and carry:
                raise AssertionError(f"carry lost in {line}")
        elif base in ("add", "addc"):
            s = val(ops[1]) + val(ops[2]) + (cc if base == "addc" else 0)
            res, carry = s & M32, s >> 32
            if ".cc" in op:
                cc = carry
            elif carry:
                raise AssertionError(f"carry lost in {line}")
        elif base == "mov":
            res = val(ops[1])
        elif base == "neg":
            res = (-val(ops[1])) & M32
        elif base == "and":
            res = val(ops[1]) & val(ops[2])
        elif base == "prmt":
            src = val(ops[1]) | (val(ops[2]) << 32)
            sel = val(ops[3])
            res = 0
            for i in range(4):
                b = (sel >> (4 * i)) & 0xF
                assert b < 8, "sign-replicating selectors are not used"
                res |= ((src >> (8 * b)) & 0xFF) << (8 * i)
        elif base in ("sub", "subc"):
            d = val(ops[1]) - val(ops[2]) - (cc if base == "subc" else 0)
            res, borrow = d & M32, 1 if d < 0 else 0
            if ".cc" in op:
                cc = borrow
            elif borrow:
                raise AssertionError(f"borrow lost in {line}")
        else:
            raise ValueError(op)
        if dst.startswith("%"):
            out[int(dst[1:])] = res
        else:
            regs[dst] = res
    return [out[k] for k in range(8)]


def limbs(v):
    return [(v >> (32 * k)) & M32 for k in range(8)]


def check(n=20000):
    P = 2**255 - 19
    A, Bv = operands()
    mul = mul_body(A, Bv) + tail()
    sq = sq_body(A) + tail()

    rng = random.Random(1)
    special = [0, 1, 2**256 - 1, 2**255, 2**256 - 38, P, 2 * P, 2**255 - 1, 38]
    vals = special + [rng.getrandbits(256) for _ in range(n)]
    for i, a in enumerate(vals):
        b = vals[(i * 13 + 7) % len(vals)] if i % 3 else rng.getrandbits(256)
        r = simulate(mul, {**{8 + k: v for k, v in enumerate(limbs(a))}, **{16 + k: v for k, v in enumerate(limbs(b))}})
        rv = sum(x << (32 * k) for k, x in enumerate(r))
        assert rv < 2**256 and rv % P == a * b % P, (hex(a), hex(b))
        r = simulate(sq, {8 + k: v for k, v in enumerate(limbs(a))})
        rv = sum(x << (32 * k) for k, x in enumerate(r))
        assert rv < 2**256 and rv % P == a * a % P, hex(a)
    # extremes that stress every carry: all-ones limbs
    for a in [2**256 - 1, 2**256 - 2, (2**256 - 1) ^ (1 << 200)]:
        for b in [2**256 - 1, 2**255 + 12345]:
            r = simulate(mul, {**{8 + k: v for k, v in enumerate(limbs(a))}, **{16 + k: v for k, v in enumerate(limbs(b))}})
            rv = sum(x << (32 * k) for k, x in enumerate(r))
            assert rv % P == a * b % P
    print(f"ok: {len(vals)} multiplications and squarings; mul {len(mul)} ops, sq {len(sq)} ops")


if __name__ == "__main__":
    if "--check" in sys.argv:
        check()
    else:
        print(header())
