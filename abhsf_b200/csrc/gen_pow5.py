"""Writes pow5_table.inc: for every decimal exponent q in [-342, 308], 5^q
normalised to 128 bits and truncated, T(q) = floor(5^q * 2^(127 - e5(q))) with
e5(q) = floor(log2 5^q), so that 2^127 <= T(q) < 2^128, as two 64-bit words,
and e5(q).  The device Matrix Market parser (mtx_device.cu) multiplies a
decimal significand by T(q) to round w * 10^q to a double (the method of
D. Lemire, "Number parsing at a gigabyte per second", Software: Practice and
Experience 51(8), 2021), with exact integer arithmetic here:

    python abhsf_b200/csrc/gen_pow5.py > abhsf_b200/csrc/pow5_table.inc
"""
Q_MIN, Q_MAX = -342, 308


def entry(q: int) -> tuple[int, int]:
    if q >= 0:
        p = 5 ** q
        e5 = p.bit_length() - 1
        t = p << (127 - e5) if e5 <= 127 else p >> (e5 - 127)
    else:
        d = 5 ** (-q)
        e5 = -d.bit_length()  # floor(log2 5^q): 5^-q is never a power of two
        t = (1 << (127 - e5)) // d
    assert (1 << 127) <= t < (1 << 128), q
    return t, e5


def main() -> None:
    print("// 5^q normalised to 128 bits (truncated) and floor(log2 5^q), q = -342 .. 308, as")
    print("// initializer lists (high word, low word per q).  Written by")
    print("// abhsf_b200/csrc/gen_pow5.py; do not edit.")
    print(f"#define ABHSF_POW5_MIN ({Q_MIN})")
    print(f"#define ABHSF_POW5_MAX {Q_MAX}")
    print("#define ABHSF_POW5_WORDS \\")
    for q in range(Q_MIN, Q_MAX + 1):
        t, _ = entry(q)
        print(f"    0x{t >> 64:016x}ull, 0x{t & ((1 << 64) - 1):016x}ull, \\")
    print("")
    print("#define ABHSF_POW5_EXPS \\")
    row = []
    for q in range(Q_MIN, Q_MAX + 1):
        row.append(str(entry(q)[1]))
        if len(row) == 16:
            print("    " + ", ".join(row) + ", \\")
            row = []
    print("    " + ", ".join(row))


if __name__ == "__main__":
    main()
