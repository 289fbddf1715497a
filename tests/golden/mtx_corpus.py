"""Matrix Market texts that exercise the reference reader's value rule
(ReadMatrixFile, reference include/load_matrix.h:88-93): values that end the
line, values followed by a space, a tab or a carriage return, zero values,
missing and unparsable values, exponents and signs.  Seeded and written
here; make_golden.py stores the reference reader's output for each."""
import numpy as np


def corpus():
    rng = np.random.default_rng(11)
    texts = {}
    lines = []
    n = 40
    endings = ["", " ", "\t", "\r", "  ", " % note"]
    for i in range(120):
        r, c = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
        kind = i % 10
        if kind == 0:
            val = ""                       # missing
        elif kind == 1:
            val = " 0"                     # zero
        elif kind == 2:
            val = " abc"                   # unparsable
        elif kind == 3:
            val = f" {rng.standard_normal():.6e}"
        elif kind == 4:
            val = f" {-rng.uniform(1, 100):.4f}"
        elif kind == 5:
            val = " -0.0"
        else:
            val = f" {rng.uniform(-5, 5):.9g}"
        lines.append(f"{r} {c}{val}{endings[i % len(endings)]}")
    texts["mixed_endings"] = ("%%MatrixMarket matrix coordinate real general\n% comment\n"
                              f"{n} {n} {len(lines)}\n" + "\n".join(lines) + "\n")
    # every value followed by a space: the reference keeps the values
    m = 30
    kept = [f"{int(rng.integers(1, m + 1))}\t{int(rng.integers(1, m + 1))} {rng.standard_normal():.17g} "
            for _ in range(80)]
    texts["trailing_space"] = f"%%MatrixMarket matrix coordinate real general\n{m} {m} {len(kept)}\n" + \
        "\n".join(kept) + "\n"
    return texts
