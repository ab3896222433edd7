"""Parameter constants of the lvl1 gate path (mirror of ``csrc/params.h``)."""

LVL0_N = 636
LVL0_ALPHA = 9.25e-5
LVL1_NBIT = 10
LVL1_N = 1024
LVL1_K = 1
LVL1_L = 2
LVL1_BGBIT = 8
LVL1_ALPHA = 2.0 ** -25
LVL10_BASEBIT = 2
LVL10_T = 7
MU32 = 1 << 29

TLWE0_WORDS = LVL0_N + 1          # 637
TLWE1_WORDS = LVL1_N + 1          # 1025
TRLWE1_WORDS = 2 * LVL1_N         # 2048
TRGSW1_WORDS = 4 * TRLWE1_WORDS   # 8192
BK_WORDS = LVL0_N * TRGSW1_WORDS
BKKB_WORDS = (LVL0_N // 2) * 3 * TRGSW1_WORDS
KSK_WORDS = LVL1_N * LVL10_T * 2 * TLWE0_WORDS

LVL2_N = 2048
LVL2_L = 4
LVL2_BGBIT = 10
LVL2_ALPHA = 2.0 ** -44
MU64 = 1 << 61
LVL20_BASEBIT = 2
LVL20_T = 7
TLWE2_WORDS = LVL2_N + 1           # 2049 (uint64)
TRLWE2_WORDS = 2 * LVL2_N          # 4096 (uint64)
TRGSW2_WORDS = 8 * TRLWE2_WORDS
BK2_WORDS = LVL0_N * TRGSW2_WORDS
BK2KB_WORDS = (LVL0_N // 2) * 3 * TRGSW2_WORDS
KSK20_WORDS = LVL2_N * LVL20_T * 2 * TLWE0_WORDS

# gate ids of the C-ABI (include/cufhe_b200.h)
NAND, OR, ORYN, ORNY, AND, ANDYN, ANDNY, NOR, XOR, XNOR, NOT, COPY, MUX, NMUX = range(14)
GATE_NAMES = ["Nand", "Or", "OrYN", "OrNY", "And", "AndYN", "AndNY", "Nor", "Xor", "Xnor",
              "Not", "Copy", "Mux", "NMux"]

# truth tables (test/plain.h:1-70)
TRUTH = {
    NAND: lambda a, b, c=None: 1 - (a & b),
    OR: lambda a, b, c=None: a | b,
    ORYN: lambda a, b, c=None: a | (1 - b),
    ORNY: lambda a, b, c=None: (1 - a) | b,
    AND: lambda a, b, c=None: a & b,
    ANDYN: lambda a, b, c=None: a & (1 - b),
    ANDNY: lambda a, b, c=None: (1 - a) & b,
    NOR: lambda a, b, c=None: 1 - (a | b),
    XOR: lambda a, b, c=None: a ^ b,
    XNOR: lambda a, b, c=None: 1 - (a ^ b),
    NOT: lambda a, b=None, c=None: 1 - a,
    COPY: lambda a, b=None, c=None: a,
    MUX: lambda a, b, c: (a & b) | ((1 - a) & c),
    NMUX: lambda a, b, c: 1 - ((a & b) | ((1 - a) & c)),
}

# precision forms of the external product
FP64_FFNT = 0
INT8_EXACT = 1
