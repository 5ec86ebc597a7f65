"""Generates field_asm.cuh: GF(2^255-19) multiply and square for sm_100a.

Eight 32-bit limbs, least significant first, values below 2^256 (not
canonical). The 512-bit product is built row by row with two PTX carry
chains per row (low halves, then high halves), and folded with
2^256 = 38 (mod 2^255-19). Each routine is one asm block so the carry flag
never crosses a compiler-visible boundary.

Run: python gen_field_asm.py > field_asm.cuh
"""


def mul_body():
    L = []
    A = lambda i: f"%{8 + i}"
    B = lambda j: f"%{16 + j}"
    T = lambda k: f"t{k}"
    # row 0: low halves straight into t0..t7, high halves into t1..t8
    for j in range(8):
        L.append(f"mul.lo.u32 {T(j)}, {A(0)}, {B(j)};")
    for j in range(8):
        op = "mad.hi.cc.u32" if j == 0 else ("madc.hi.u32" if j == 7 else "madc.hi.cc.u32")
        acc = "0" if j == 7 else T(j + 1)
        L.append(f"{op} {T(j + 1)}, {A(0)}, {B(j)}, {acc};")
    for i in range(1, 8):
        for j in range(8):
            op = "mad.lo.cc.u32" if j == 0 else "madc.lo.cc.u32"
            L.append(f"{op} {T(i + j)}, {A(i)}, {B(j)}, {T(i + j)};")
        L.append(f"addc.u32 {T(i + 8)}, 0, 0;")
        for j in range(8):
            op = "mad.hi.cc.u32" if j == 0 else ("madc.hi.u32" if j == 7 else "madc.hi.cc.u32")
            L.append(f"{op} {T(i + j + 1)}, {A(i)}, {B(j)}, {T(i + j + 1)};")
    return L


def sq_body():
    L = []
    A = lambda i: f"%{8 + i}"
    T = lambda k: f"t{k}"
    # off-diagonal products a_i a_j, i < j: low half to t[i+j], high to t[i+j+1]
    for j in range(1, 8):
        L.append(f"mul.lo.u32 {T(j)}, {A(0)}, {A(j)};")
    for j in range(1, 8):
        first, last = j == 1, j == 7
        op = "mad.hi.cc.u32" if first else ("madc.hi.u32" if last else "madc.hi.cc.u32")
        acc = "0" if last else T(j + 1)
        L.append(f"{op} {T(j + 1)}, {A(0)}, {A(j)}, {acc};")
    for i in range(1, 7):
        js = list(range(i + 1, 8))
        for n, j in enumerate(js):
            op = "mad.lo.cc.u32" if n == 0 else "madc.lo.cc.u32"
            L.append(f"{op} {T(i + j)}, {A(i)}, {A(j)}, {T(i + j)};")
        L.append(f"addc.u32 {T(i + 8)}, 0, 0;")
        for n, j in enumerate(js):
            first, last = n == 0, n == len(js) - 1
            if first and last:
                op = "mad.hi.u32"
            elif first:
                op = "mad.hi.cc.u32"
            elif last:
                op = "madc.hi.u32"
            else:
                op = "madc.hi.cc.u32"
            L.append(f"{op} {T(i + j + 1)}, {A(i)}, {A(j)}, {T(i + j + 1)};")
    # double t1..t14 into t1..t15
    L.append("add.cc.u32 t1, t1, t1;")
    for k in range(2, 15):
        L.append(f"addc.cc.u32 {T(k)}, {T(k)}, {T(k)};")
    L.append("addc.u32 t15, 0, 0;")
    # diagonal squares
    L.append(f"mul.lo.u32 t0, {A(0)}, {A(0)};")
    L.append(f"mad.hi.cc.u32 t1, {A(0)}, {A(0)}, t1;")
    for i in range(1, 8):
        L.append(f"madc.lo.cc.u32 {T(2 * i)}, {A(i)}, {A(i)}, {T(2 * i)};")
        op = "madc.hi.u32" if i == 7 else "madc.hi.cc.u32"
        L.append(f"{op} {T(2 * i + 1)}, {A(i)}, {A(i)}, {T(2 * i + 1)};")
    return L


def reduce_tail():
    """t0..t15 -> %0..%7 with 2^256 = 38, result below 2^256."""
    R = lambda k: f"%{k}"
    T = lambda k: f"t{k}"
    L = []
    for k in range(8):
        op = "mad.lo.cc.u32" if k == 0 else "madc.lo.cc.u32"
        L.append(f"{op} {R(k)}, {T(8 + k)}, 38, {T(k)};")
    L.append("addc.u32 c, 0, 0;")
    for k in range(8):
        op = "mad.hi.cc.u32" if k == 0 else ("madc.hi.u32" if k == 7 else "madc.hi.cc.u32")
        dst = "c" if k == 7 else R(k + 1)
        L.append(f"{op} {dst}, {T(8 + k)}, 38, {dst};")
    # value = %0..%7 + c * 2^256 with c < 39: fold once more
    L.append("mad.lo.cc.u32 %0, c, 38, %0;")
    for k in range(1, 8):
        L.append(f"addc.cc.u32 {R(k)}, {R(k)}, 0;")
    L.append("addc.u32 c, 0, 0;")
    # a carry here leaves %0..%7 below 38*39, so this add cannot carry
    L.append("mad.lo.u32 %0, c, 38, %0;")
    return L


def emit(name, body, nin):
    out = []
    ins = ", ".join(f'"r"(a[{i}])' for i in range(8))
    if nin == 2:
        ins += ", " + ", ".join(f'"r"(b[{i}])' for i in range(8))
    sig = "const uint32_t* __restrict__ a, const uint32_t* __restrict__ b" if nin == 2 else "const uint32_t* __restrict__ a"
    out.append(f"__device__ __forceinline__ void {name}(uint32_t* __restrict__ r, {sig}) {{")
    out.append("    asm(\"{\\n\\t.reg .u32 t<16>;\\n\\t.reg .u32 c;\\n\\t\"")
    for line in body + reduce_tail():
        out.append(f'        "{line}\\n\\t"')
    out.append('        "}"')
    outs = ", ".join(f'"=r"(r[{i}])' for i in range(8))
    out.append(f"        : {outs}")
    out.append(f"        : {ins});")
    out.append("}")
    return "\n".join(out)


if __name__ == "__main__":
    print("// Generated by gen_field_asm.py — do not edit by hand.")
    print("// GF(2^255-19): r = a*b and r = a^2, eight 32-bit limbs, result below 2^256.")
    print("#pragma once")
    print("#include <cstdint>")
    print()
    print(emit("fe_mul_asm", mul_body(), 2))
    print()
    print(emit("fe_sq_asm", sq_body(), 1))
