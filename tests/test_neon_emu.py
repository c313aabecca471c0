"""CPU unit tests of the AArch64 interpreter that produced the golden fixtures
(oracle/neon_emu.py), on hand-written instruction snippets: addressing
modes, flags and branches, by-element and pairwise float arithmetic, exact
fused multiply-add, structure stores and 64-bit vector writes."""
import numpy as np

from oracle import neon_emu as emu


def run(lines, A=None, B=None, C=None, params=None):
    prog, labels = emu.build_program(lines)
    mem = emu.Memory()
    p = dict(params or {})
    for name, base, arr in (("A", emu.BASE_A, A), ("B", emu.BASE_B, B), ("C", emu.BASE_C, C)):
        if arr is not None:
            mem.add(base, arr)
            p[name] = base
    stack = np.zeros(4096, np.uint8)
    mem.add(emu.STACK_TOP - 4096, stack)
    m = emu.Machine(prog, labels, p, mem, sp=emu.STACK_TOP)
    m.run()
    return m


def test_loads_post_index_and_stores():
    A = np.arange(16, dtype=np.float32)
    C = np.zeros(16, np.float32)
    run(["ldr x1, %[A]", "ldr x2, %[C]", "ldr q0, [x1], #16", "ldp q1, q2, [x1], #32",
         "str q2, [x2]", "stp q0, q1, [x2, #16]", "ldr q3, [x1]", "str q3, [x2], #48",
         "str q3, [x2]"], A=A, C=C)
    assert np.array_equal(C[:4], A[12:16])  # the post-indexed store overwrote A[8:12]
    assert np.array_equal(C[4:12], A[0:8])
    assert np.array_equal(C[12:16], A[12:16])


def test_fmla_by_element_and_fmul():
    A = np.array([1.5, -2.0, 3.25, 0.5], np.float32)
    B = np.array([2.0, 4.0, -1.0, 8.0], np.float32)
    C = np.zeros(8, np.float32)
    run(["ldr x1, %[A]", "ldr x2, %[B]", "ldr x3, %[C]", "ldr q0, [x1]", "ldr q1, [x2]",
         "fmul v2.4s, v0.4s, v1.s[1]", "fmla v2.4s, v0.4s, v1.s[3]", "str q2, [x3]",
         "fmul v4.4s, v0.4s, v1.4s", "str q4, [x3, #16]"], A=A, B=B, C=C)
    assert np.array_equal(C[:4], A * 4.0 + A * 8.0)
    assert np.array_equal(C[4:], A * B)


def test_fma_is_single_rounded():
    # a*b + c with a*b needing more than 24 bits: FMA and mul-then-add differ
    a = np.float32(1 + 2 ** -12)
    c = np.float32(-(1 + 2 ** -11))
    A = np.array([a, 0, 0, 0], np.float32)
    Cacc = np.array([c, 0, 0, 0], np.float32)
    out = np.zeros(4, np.float32)
    run(["ldr x1, %[A]", "ldr x2, %[B]", "ldr x3, %[C]", "ldr q0, [x1]", "ldr q5, [x2]",
         "fmla v5.4s, v0.4s, v0.4s", "str q5, [x3]"], A=A, B=Cacc, C=out)
    exact = float(a) * float(a) + float(c)  # exactly 2^-24
    assert out[0] == np.float32(exact)
    assert out[0] != np.float32(np.float32(a * a) + c)


def test_faddp_and_scalar_forms():
    A = np.array([1, 2, 3, 4, 10, 20, 30, 40], np.float32)
    C = np.zeros(8, np.float32)
    run(["ldr x1, %[A]", "ldr x3, %[C]", "ldp q0, q1, [x1]", "faddp v2.4s, v0.4s, v1.4s",
         "str q2, [x3]", "faddp s4, v0.2s", "str s4, [x3, #16]"], A=A, C=C)
    assert np.array_equal(C[:4], [3, 7, 30, 70])
    assert C[4] == 3 and np.all(C[5:] == 0)


def test_st4_lane_store_and_ins():
    A = np.arange(16, dtype=np.float32)
    C = np.zeros(8, np.float32)
    run(["ldr x1, %[A]", "ldr x3, %[C]", "ldp q5, q6, [x1]", "ldp q7, q8, [x1, #32]",
         "st4 {v5.s, v6.s, v7.s, v8.s}[2], [x3]", "ins v5.s[0], v8.s[3]",
         "str s5, [x3, #16]"], A=A, C=C)
    assert np.array_equal(C[:4], [2, 6, 10, 14])
    assert C[4] == 15


def test_branches_flags_and_integer_ops():
    C = np.zeros(4, np.int64)
    m = run(["mov x1, #10", "mov x2, #0", "loop:", "add x2, x2, x1", "subs x1, x1, #1",
             "bgt loop", "mov x4, #17", "mov x5, #5", "udiv x6, x4, x5",
             "msub x7, x6, x5, x4", "lsl x8, x7, #3", "ands x9, x4, #7", "cmp x9, #1",
             "beq done", "mov x2, #0", "done:"], C=C)
    assert m.x[2] == 55 and m.x[6] == 3 and m.x[7] == 2 and m.x[8] == 16 and m.x[9] == 1


def test_macro_expansion_and_stack():
    C = np.zeros(4, np.float32)
    m = run([".macro BUMP", "add x1, x1, #2", ".endm", "mov x1, #0", "BUMP", "BUMP",
             "mov x6, #64", "sub sp, sp, x6", "mov x2, sp", "add sp, sp, x6"], C=C)
    assert m.x[1] == 4 and m.x[2] == emu.STACK_TOP - 64 and m.sp == emu.STACK_TOP


def test_64bit_vector_write_clears_upper_half():
    A = np.array([1, 2, 3, 4], np.float32)
    C = np.zeros(4, np.float32)
    run(["ldr x1, %[A]", "ldr x3, %[C]", "ldr q0, [x1]", "ldr q1, [x1]",
         "fmul v1.2s, v0.2s, v0.s[1]", "str q1, [x3]"], A=A, C=C)
    assert np.array_equal(C, [2, 4, 0, 0])


def test_guard_zone_reads_are_nan():
    A = np.ones(4, np.float32)
    C = np.zeros(8, np.float32)
    run(["ldr x1, %[A]", "ldr x3, %[C]", "ldr q0, [x1, #16]", "str q0, [x3]"], A=A, C=C)
    assert np.isnan(C[:4]).all()


def test_interleaved_structure_loads_and_stores():
    # ld2 / ld3 de-interleave, st2 interleaves, lane forms move one element per register
    A = np.arange(24, dtype=np.float32)
    C = np.zeros(32, np.float32)
    run(["ldr x1, %[A]", "ldr x2, %[C]",
         "ld2 {v0.4s, v1.4s}, [x1]",          # v0 = A[0,2,4,6], v1 = A[1,3,5,7]
         "str q0, [x2]", "str q1, [x2, #16]",
         "ld3 {v2.4s, v3.4s, v4.4s}, [x1]",   # v2 = A[0,3,6,9], v3 = A[1,4,7,10]
         "str q2, [x2, #32]", "str q3, [x2, #48]",
         "st2 {v2.s, v3.s}[1], [x2, #64]",    # A[3], A[4]
         "ld2 {v5.s, v6.s}[2], [x1, #8]",     # lane 2 of v5 / v6 <- A[2], A[3]
         "str q5, [x2, #72]", "str q6, [x2, #88]",
         "st2 {v0.4s, v1.4s}, [x1]"], A=A, C=C)    # interleaves back: A unchanged
    assert np.array_equal(C[0:4], [0, 2, 4, 6]) and np.array_equal(C[4:8], [1, 3, 5, 7])
    assert np.array_equal(C[8:12], [0, 3, 6, 9]) and np.array_equal(C[12:16], [1, 4, 7, 10])
    assert np.array_equal(C[16:18], [3, 4])
    assert C[18 + 2] == 2.0 and C[22 + 2] == 3.0
    assert np.array_equal(A, np.arange(24, dtype=np.float32))
