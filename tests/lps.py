"""Small LPs used by the tests: hand models from the reference's unit tests, a long-row model,
and readers for the reference's .lpm fixtures (read by path where the reference is mounted)."""
import os

import numpy as np
from ps26119.generators import Lp, from_dense, csc_from_triplets

inf = np.inf


def wyndor():
    """Wyndor (max 3x + 5y; x <= 4, 2y <= 12, 3x + 2y <= 18): optimum 36 at (2, 6),
    y = (0, 1.5, 1) — reference tests/unit/test_pdhg.cpp:38-41, test_c_api.cpp:13-19."""
    return from_dense([3, 5], [[1, 0], [0, 2], [3, 2]], [-inf] * 3, [4, 12, 18], [0, 0], [inf, inf], sense=-1,
                      name="wyndor")


def mixed_rows():
    """min with >= rows, an equality, a ranged row and bounded/free columns
    (reference tests/unit/test_pdhg.cpp:43-47)."""
    return from_dense([2, 3, -1, 0.5], [[1, 1, 0, 0], [0, 1, 1, 0], [1, 0, 0, 1], [1, -1, 1, 1]],
                      [2, 1, 1, -3], [inf, 1, 4, 3], [0, 0, -1, -inf], [10, 10, 2, inf], name="mixed_rows")


def max_ranged():
    """MAX model with a ranged row and a free column, optimum 21.5
    (reference data/hand/max_ranged.lpm, tests/unit/test_batch.cpp:66-73)."""
    cs = np.array([0, 3, 6, 7], dtype=np.int32)
    ri = np.array([0, 1, 2, 0, 1, 2, 0], dtype=np.int32)
    v = np.array([1.0, 1.0, 1.0, 1.0, -1.0, 3.0, 1.0])
    return Lp(3, 3, np.array([3.0, 2.0, -1.0]), np.array([0.0, -inf, -1.0]), np.array([3.0, inf, 5.0]),
              np.array([-inf, -1.0, 1.0]), np.array([4.0, 2.0, inf]), cs, ri, v, -1, 7.5, "max_ranged")


def long_row(m=1500, n=3000):
    """Row 0 has n entries and column 0 has m entries (both > 1024): the long-row case of the
    reference's tests/unit/test_gpu.cpp:128-188."""
    rows, cols, vals = [], [], []
    obj = np.empty(n)
    for j in range(n):
        obj[j] = -1.0 - (j % 13) * 0.1
        rows.append(0), cols.append(j), vals.append(1.0 + (j % 5) * 0.25)
        i = 1 + j % (m - 1)
        rows.append(i), cols.append(j), vals.append(0.5 + (j % 7) * 0.1)
        if j == 0:
            for r in range(1, m):
                if r != i:
                    rows.append(r), cols.append(j), vals.append(0.3)
    cs, ri, v = csc_from_triplets(m, n, np.array(rows), np.array(cols), np.array(vals))
    return Lp(m, n, obj, np.zeros(n), np.full(n, 10.0), np.full(m, -inf), np.full(m, 50.0), cs, ri, v, 1, 0.0,
              "long_row")


def infeasible():
    """x0 + x1 <= 1 and x0 + x1 >= 3 (reference tests/unit/test_gpu.cpp:195)."""
    return from_dense([1, 1], [[1, 1], [1, 1]], [-inf, 3], [1, inf], [0, 0], [inf, inf], name="infeasible")


def unbounded():
    """The 7x7 MAX model of reference tests/unit/test_gpu.cpp:196-206."""
    lp = from_dense([5, -1, 4, -5, 0, 0, -5],
                    [[0, 5, 0, 0, 0, 2, 0], [0, 5, -5, 0, 0, 0, -1], [0, 0, 0, -1, 0, 0, 5], [-3, 0, 0, 0, 0, -3, 4],
                     [0, 4, -1, -5, 0, 0, 0], [4, 0, 0, 0, 0, -4, 4], [0, 0, 0, 0, -5, -2, 0]],
                    [-inf, -inf, -15, -21, 24, -inf, -inf], [31, 23, inf, inf, 24, -24, -9],
                    [0, 4, 1, -inf, 0, 1, -inf], [inf, 9, inf, 2, inf, 4, inf], sense=-1, name="unbounded")
    return lp


def read_lpm(path):
    """Reader of the reference's .lpm text format (reference tools/lpm.py docstring)."""
    sections = {}
    head = {}
    cur = None
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#") or line.startswith("LPM"):
                continue
            word = line.split()[0]
            if word in ("NAME", "SENSE", "ROWS", "COLS", "NNZ", "OFFSET"):
                head[word] = line.split(None, 1)[1] if len(line.split()) > 1 else ""
                cur = None
            elif word in ("OBJ", "COL_LOWER", "COL_UPPER", "ROW_LOWER", "ROW_UPPER", "COL_START", "ROW_INDEX",
                          "VALUE", "ROW_NAMES", "COL_NAMES", "INTEGER"):
                cur = word
                sections[cur] = []
            elif word == "END":
                break
            elif cur is not None:
                sections[cur].extend(line.split())
    m, n = int(head["ROWS"]), int(head["COLS"])
    num = lambda k: np.array([float(t) for t in sections.get(k, [])], dtype=np.float64)
    cs = np.array([int(t) for t in sections["COL_START"]], dtype=np.int32)
    ri = np.array([int(t) for t in sections.get("ROW_INDEX", [])], dtype=np.int32)
    return Lp(m, n, num("OBJ"), num("COL_LOWER"), num("COL_UPPER"), num("ROW_LOWER"), num("ROW_UPPER"), cs, ri,
              num("VALUE"), -1 if head.get("SENSE", "MIN").upper() == "MAX" else 1, float(head.get("OFFSET", 0)),
              head.get("NAME", os.path.basename(path)))


NETLIB = ["afiro", "sc50a", "sc50b", "kb2", "adlittle", "blend", "share2b", "sc105", "stocfor1", "recipe"]
