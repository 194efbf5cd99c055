"""Generates jump_tables.inc: the GF(2) matrices of J^(2^b), b = 4..27, where
J is the xoshiro128+ jump() (advance by 2^64 steps, Rust-CUDA/src/main.rs:
1452, 1473-1487).  xoshiro128+ is linear over GF(2), so J is a 128 x 128 bit
matrix whose column j is jump() applied to the unit state e_j; its powers by
repeated squaring let one GPU thread compute stream 16*m = J^(16 m) master
directly instead of performing 16 m sequential jumps.

Usage: python gen_jump_tables.py OUT_FILE   (run by cudapic_b200/build.py)
"""
import sys

JUMP = (0x8764000B, 0xF542D2D3, 0x6FA035C3, 0x77F2DB5B)
M32 = 0xFFFFFFFF
FIRST_LEVEL = 4   # streams are produced in chunks of 2^4 consecutive jumps
LEVELS = 24       # levels 4..27: up to 2^28 streams


def _next(s):
    s0, s1, s2, s3 = s
    t = (s1 << 9) & M32
    s2 ^= s0
    s3 ^= s1
    s1 ^= s2
    s0 ^= s3
    s2 ^= t
    s3 = ((s3 << 11) | (s3 >> 21)) & M32
    return [s0, s1, s2, s3]


def _jump(s):
    acc = [0, 0, 0, 0]
    for word in JUMP:
        for b in range(32):
            if (word >> b) & 1:
                acc = [a ^ x for a, x in zip(acc, s)]
            s = _next(s)
    return acc


def _to_int(s):
    return s[0] | (s[1] << 32) | (s[2] << 64) | (s[3] << 96)


def _matvec(cols, v):
    r = 0
    j = 0
    while v:
        if v & 1:
            r ^= cols[j]
        v >>= 1
        j += 1
    return r


def jump_power_columns():
    unit = []
    for j in range(128):
        s = [0, 0, 0, 0]
        s[j // 32] = 1 << (j % 32)
        unit.append(_to_int(_jump(s)))
    levels = [unit]
    for _ in range(FIRST_LEVEL + LEVELS - 1):
        m = levels[-1]
        levels.append([_matvec(m, c) for c in m])
    return levels[FIRST_LEVEL:FIRST_LEVEL + LEVELS]


def main(out_path):
    tables = jump_power_columns()
    lines = ["// generated by gen_jump_tables.py -- do not edit",
             "// c_jump_pow[l][j] = column j of J^(2^(l+%d)) as (s0, s1, s2, s3)" % FIRST_LEVEL,
             "#define CUDAPIC_JUMP_FIRST_LEVEL %d" % FIRST_LEVEL,
             "#define CUDAPIC_JUMP_LEVELS %d" % LEVELS,
             "__constant__ uint4 c_jump_pow[%d][128] = {" % LEVELS]
    for cols in tables:
        row = []
        for c in cols:
            w = [(c >> (32 * k)) & M32 for k in range(4)]
            row.append("{0x%08xu,0x%08xu,0x%08xu,0x%08xu}" % tuple(w))
        lines.append("  {" + ",".join(row) + "},")
    lines.append("};")
    with open(out_path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])
