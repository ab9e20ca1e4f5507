"""The committed tile-shape table (read beside the library by the pass autotuner).

Every line names a precision, a grid size, a line length, a stride, a pass kind and a shape choice
that the engine builds: shapes 0-2 for lines of 256 to 2048 points, shape 3 (seven lines per CTA)
only for 1024-point lines. A malformed or out-of-range line would be skipped or refused by the
engine at run time; here it fails on the CPU.
"""
import os
import re

TABLE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tdse_nd_mpi_b200",
                     "shape_table.tsv")
LINE = re.compile(r"^(fp64|fp32)\tn=(\d+)\tL=(\d+)\tlog2S=(\d+)\t(double|sandwich)\tms=([-0-9.,]+)\tchoice=(\d+)$")


def test_shape_table_lines_are_valid():
    with open(TABLE) as f:
        lines = [l.rstrip("\n") for l in f if l.strip()]
    assert any(l.startswith("# device=") for l in lines)
    seen = set()
    for l in lines:
        if l.startswith("#"):
            continue
        m = LINE.match(l)
        assert m, l
        prec, n, L, log2S, kind, ms, choice = m.groups()
        n, L, log2S, choice = int(n), int(L), int(log2S), int(choice)
        assert L & (L - 1) == 0 and 256 <= L <= 2048, l
        assert n % L == 0 and (1 << log2S) <= n // L, l
        assert 0 <= choice <= 3 and (choice < 3 or L == 1024), l
        times = [float(x) for x in ms.split(",")]
        assert len(times) >= 3 and times[choice] > 0, l
        # the choice is the default unless another shape was measured at least 2% faster
        if choice:
            assert times[choice] < 0.98 * times[0], l
        key = (prec, n, L, log2S, kind)
        assert key not in seen, l
        seen.add(key)
