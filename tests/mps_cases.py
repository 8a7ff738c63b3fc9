"""MPS inputs for the reader's parity tests.

`CASES` are small hand-written files, each aimed at one rule of the
reference reader (src/io/mps_reader.hpp:15-304) or of the validation after
it (src/model/model.hpp:117-178).  `random_mps` writes a seeded LP in a
randomly varied but legal layout (fixed or free columns, set names present
or not, one or two pairs per line, D exponents, comments, CRLF, markers,
ranges, every bound type) so that large files exercise the same rules.
"""
from __future__ import annotations

import numpy as np

CASES = {
    # every row type, RHS with a set name, two pairs per line, all bound types
    "basic": """NAME          BASIC
ROWS
 N  COST
 L  LIM1
 G  LIM2
 E  MYEQN
 L  LIM3
COLUMNS
    X1        COST         1.0   LIM1         1.0
    X1        LIM2         1.0
    X2        COST         2.0   LIM1         1.0
    X2        MYEQN       -1.0
    X3        COST        -1.0   MYEQN        1.0
    X4        COST         0.5   LIM3         2.5
    X5        LIM3         1.0   LIM2        -3.0
    X6        COST         1.0   LIM1         4.0
    X7        LIM1         1.0
RHS
    RHS       LIM1         4.0   LIM2         1.0
    RHS       MYEQN        7.0   LIM3        10.0
BOUNDS
 UP BND       X1           4.0
 LO BND       X2          -1.0
 UP BND       X2           1.0
 MI BND       X3
 FX BND       X4           2.0
 FR BND       X5
 PL BND       X6
 LO BND       X7           1.5
ENDATA
""",
    # RANGES on each row type, both signs; a range on an unknown row
    "ranges": """NAME RANGES
ROWS
 N obj
 G g1
 G g2
 L l1
 L l2
 E e1
 E e2
 E e3
COLUMNS
 x obj 1 g1 1
 x g2 1 l1 1
 x l2 1 e1 1
 x e2 1 e3 1
RHS
 rhs g1 1 g2 2
 rhs l1 3 l2 4
 rhs e1 5 e2 6
 rhs e3 7
RANGES
 rng g1 2 g2 -2
 rng l1 3 l2 -3
 rng e1 4 e2 -4
 rng nosuch 9
 e3 0
ENDATA
""",
    # OBJSENSE on its own line, then MAXIMIZE on the next; RHS on the
    # objective gives minus the offset; D exponents
    "objsense_next_line": """NAME
OBJSENSE
    MAXIMIZE
ROWS
 N  profit
 L  cap
COLUMNS
    a  profit  3.5D+00  cap  1.0d0
    b  profit  2.0E0    cap  2D-1
RHS
    RHS  profit  -12.5
    RHS  cap     1.0D1
BOUNDS
 UP BND a 4
ENDATA
""",
    # OBJSENSE MAX on the header line; OBJNAME picks the second N row;
    # the first N row is then an ignored free row
    "objname": """NAME OBJN
OBJSENSE MAX
OBJNAME second
ROWS
 N first
 N second
 E r1
COLUMNS
 x first 100 second 1
 x r1 1
 y second 2 r1 1
 y first 7
RHS
 B r1 4 first 3
 B second 8
ENDATA
""",
    # OBJSENSE and OBJNAME given inside COLUMNS: the section goes on
    "header_inside_columns": """NAME MID
ROWS
 N c1
 N c2
 G r1
COLUMNS
 x c1 1 r1 1
OBJSENSE MAXIMIZE
 y c1 2 r1 1
OBJNAME c2
 y c2 5
 z c2 -1 r1 2
 z c1 9
RHS
 r1 3
ENDATA
""",
    # integer markers, BV, LI/UI, integer bound rounding, binary promotion
    "integers": """NAME INTS
ROWS
 N obj
 L c
COLUMNS
    x0 obj 1 c 1
    MARKER                 'MARKER'                 'INTORG'
    i1 obj 1 c 1
    i2 obj 1 c 1
    i3 obj 1 c 1
    MARKER                 'MARKER'                 'INTEND'
    y obj 1 c 1
    i4 obj 1 c 1
    z obj 1 c 1
    MARK2 'MARKER' 'INTORG'
    i5 obj 1 c 1
    MARK3 'MARKER' 'INTEND'
    x0 c 2
RHS
    R c 10
BOUNDS
 UP B i1 1
 LO B i2 0.3
 UP B i2 7.9999999999
 LO B i3 -2.5
 UP B i3 2.5
 BV B y
 LI B i4 -3.2
 UI B i4 4.7
 UI B z 0.5
 SC B x0 9
 UP B i5 1e30
ENDATA
""",
    # duplicates summed, sums to zero dropped, explicit zeros dropped, a
    # column that reappears later, unknown rows ignored, the objective
    # entered twice
    "duplicates": """NAME DUP
ROWS
 N obj
 E a
 E b
 E c
COLUMNS
 x a 1.5 b 2
 x a 0.25 c 0
 x nosuch 3 obj 1
 y a 1 b 1
 y b -1 obj 2
 x c 4 obj 0.5
 x a 0.125
 y c 1e-300 c -1e-300
RHS
 R a 1 nosuch 2
ENDATA
""",
    # CRLF, comments, blank and white-space-only lines, tabs, a lower-case
    # header, a data line in column 0, lines after ENDATA
    "layout": "NAME\tLAYOUT\r\n* a comment\r\n\r\nrows\r\n N\tz\r\n   \r\n L\tr\r\n"
              "COLUMNS\r\n\tu\tz\t1\tr\t1\r\n*   another comment\r\nv z 2 r 3\r\nRHS\r\n r 6\r\n"
              "BOUNDS\r\n UP bnd u 4\r\nENDATA\r\n x z 99\r\nGARBAGE\r\n",
    # negative UP rule, bounds at and past 1e20, crossed bounds inside the
    # repair tolerance
    "bound_rules": """NAME BR
ROWS
 N obj
 G r
COLUMNS
 a obj 1 r 1
 b obj 1 r 1
 c obj 1 r 1
 d obj 1 r 1
 e obj 1 r 1
 f obj 1 r 1
RHS
 rhs r 1e20
BOUNDS
 UP bnd a -5
 LO bnd b 2
 UP bnd b -1e-12
 LO bnd b -3
 UP bnd c 1e20
 LO bnd c -1e21
 LO bnd d 1.0000000001
 UP bnd d 1
 UP bnd e -0
 MI bnd f
 UP bnd f -2
ENDATA
""",
    # bounds written without the set name (three tokens)
    "bounds_no_set": """NAME NOSET
ROWS
 N obj
 L r
COLUMNS
 x obj 1 r 1
 y obj -1 r 1
RHS
 r 5
BOUNDS
 UP x 3
 LO y 1
 FX x 2
 FR bnd y
ENDATA
""",
    # QUADOBJ (lower entries swapped up) and QMATRIX (lower entries dropped)
    "quadobj": """NAME QP
ROWS
 N obj
 G r
COLUMNS
 x obj 1 r 1
 y obj 1 r 1
 z obj 0 r 1
RHS
 r 1
QUADOBJ
 x x 2
 y x 0.5
 z y 1
 y y 4
 q x 1
ENDATA
""",
    "qmatrix": """NAME QM
ROWS
 N obj
 G r
COLUMNS
 x obj 1 r 1
 y obj 1 r 1
RHS
 r 1
QMATRIX
 x x 2
 x y 0.5
 y x 0.5
 y y 4
ENDATA
""",
    # SOS content and RANGES/RHS with an even token count
    "sos_and_even": """NAME SOS
ROWS
 N obj
 L a
 G b
COLUMNS
 x obj 1 a 1
 y obj 1 b 1
RHS
 a 2 b 1
RANGES
 a 1
SOS
 S1 SOS s1 1
 x 1
 y 2
ENDATA
""",
    # no ENDATA, last line without a newline
    "no_endata": "NAME E\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r 1\nRHS\n rhs r 2",
    # empty model
    "empty": "NAME EMPTY\nROWS\n N obj\nCOLUMNS\nRHS\nENDATA\n",
    # ---- failures
    "err_duplicate_row": "NAME D\nROWS\n N o\n L r\n G r\nCOLUMNS\n x o 1 r 1\nENDATA\n",
    "err_unknown_bound_column": "NAME U\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r 1\nBOUNDS\n UP b nope 1\nENDATA\n",
    "err_infeasible_column": "NAME I\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r 1\nBOUNDS\n LO b x 5\n UP b x 3\nENDATA\n",
    "err_integer_rounding_infeasible": "NAME I\nROWS\n N o\n L r\nCOLUMNS\n MARKER 'MARKER' 'INTORG'\n"
                                       " x o 1 r 1\n MARKER 'MARKER' 'INTEND'\nBOUNDS\n LO b x 0.2\n UP b x 0.8\n"
                                       "ENDATA\n",
    "err_nonfinite_cost": "NAME N\nROWS\n N o\n L r\nCOLUMNS\n x o nan r 1\nENDATA\n",
    "err_nonfinite_matrix": "NAME N\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r inf\nENDATA\n",
    # std::stod failures: the reference lets the exception escape
    "err_bad_number": "NAME B\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r 1\n y o abc r 1\nENDATA\n",
    "err_out_of_range": "NAME B\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r 1e400\nENDATA\n",
    "err_bad_rhs": "NAME B\nROWS\n N o\n L r\nCOLUMNS\n x o 1 r 1\nRHS\n rhs r x1\nENDATA\n",
}


def _num(rng, v: float) -> str:
    """A decimal that reads back as exactly v, in a random spelling."""
    s = repr(float(v))
    k = rng.integers(0, 4)
    if k == 1 and "e" in s:
        s = s.replace("e", "D")
    elif k == 2 and "e" in s:
        s = s.replace("e", "d")
    elif k == 3 and v == int(v) and abs(v) < 1e15:
        s = str(int(v))
    return s


def random_mps(lp, seed: int, integer_frac: float = 0.1, ranges: bool = True, sense: int = 1) -> str:
    """The LP (nir_lp_view layout) as an MPS text with a seeded layout."""
    rng = np.random.default_rng([0x3B5, seed])
    nl = "\r\n" if rng.random() < 0.3 else "\n"
    fixed = rng.random() < 0.5
    out = [f"NAME RAND{seed}"]
    if sense < 0:
        out.append("OBJSENSE MAX" if rng.random() < 0.5 else "OBJSENSE\n    MAX")
    out.append("ROWS")
    out.append(" N  OBJ")
    lo, up = lp.rowlo, lp.rowup
    fin = lambda b: np.isfinite(b) & (np.abs(b) < 1e20)
    rtype = []
    for i in range(lp.nrow):
        if not fin(lo[i]) and fin(up[i]):
            t = "L"
        elif fin(lo[i]) and not fin(up[i]):
            t = "G"
        elif fin(lo[i]) and fin(up[i]) and lo[i] == up[i]:
            t = "E"
        elif fin(lo[i]) and fin(up[i]) and ranges:
            t = "R"
        else:
            t = "N"  # a free row: written as G with rhs -1e30
        rtype.append(t)
        letter = {"L": "L", "G": "G", "E": "E", "R": "G", "N": "G"}[t]
        out.append(f" {letter}  R{i}")
        if rng.random() < 0.002:
            out.append("* comment between rows")
    out.append("COLUMNS")
    in_int = False
    ints = rng.random(lp.ncol) < integer_frac
    for j in range(lp.ncol):
        if ints[j] != in_int:
            out.append(f"    M{j}  'MARKER'  '{'INTORG' if ints[j] else 'INTEND'}'")
            in_int = bool(ints[j])
        pairs = []
        if lp.cost[j] != 0.0:
            pairs.append(("OBJ", lp.cost[j]))
        s, e = lp.col_start[j], lp.col_start[j + 1]
        pairs += [(f"R{lp.row_index[k]}", lp.value[k]) for k in range(s, e)]
        # split one entry into two duplicates now and then
        if pairs and rng.random() < 0.05:
            r, v = pairs[-1]
            pairs[-1] = (r, v * 0.5)
            pairs.append((r, v - v * 0.5))
        q = 0
        while q < len(pairs):
            two = rng.random() < 0.5 and q + 1 < len(pairs)
            items = pairs[q:q + (2 if two else 1)]
            toks = [f"C{j}"] + [f"{r} {_num(rng, v)}" for r, v in items]
            if fixed:
                line = "    " + "  ".join(f"{t:<10}" for t in toks)
            else:
                line = (" " if rng.random() < 0.9 else "\t") + " ".join(toks)
            out.append(line)
            q += len(items)
    if in_int:
        out.append("    MEND  'MARKER'  'INTEND'")
    out.append("RHS")
    if lp.obj_offset != 0.0:
        out.append(f"    RHS  OBJ  {_num(rng, -lp.obj_offset)}")
    for i in range(lp.nrow):
        t = rtype[i]
        b = {"L": up[i], "G": lo[i], "E": lo[i], "R": lo[i], "N": -1e30}[t]
        if b != 0.0:
            out.append((f"    RHS  R{i}  " if rng.random() < 0.7 else f" R{i} ") + _num(rng, b))
    if ranges and "R" in rtype:
        out.append("RANGES")
        for i in range(lp.nrow):
            if rtype[i] == "R":
                out.append(f"    RNG  R{i}  {_num(rng, up[i] - lo[i])}")
    out.append("BOUNDS")
    for j in range(lp.ncol):
        a, b = lp.collo[j], lp.colup[j]
        fa, fb = fin(a), fin(b)
        if not fa and not fb:
            out.append(f" FR BND C{j}")
            continue
        if fa and fb and a == b:
            out.append(f" FX BND C{j} {_num(rng, a)}")
            continue
        if not fa:
            out.append(f" MI BND C{j}")
        elif a != 0.0:
            out.append(f" LO BND C{j} {_num(rng, a)}")
        if fb:
            out.append(f" UP BND C{j} {_num(rng, b)}")
    out.append("ENDATA")
    return nl.join(out) + nl


# number spellings std::stod accepts, and tokens it rejects or overflows on
_GOOD = ["1", "-2.5", "3e2", "4D-1", "0.0", "-0", ".5", "5.", "+7", "1e20", "-1e20", "1e19", "00012", "2.25d+1",
        "0.1", "1.0000000000000000000001", "123456789012345678901234", "7E-3", "-0.0"]
_BAD = ["abc", "1e400", "1e-400", "x1", "inf", "nan", "0x10", "1.5x", "2d", "1e"]


def _fuzz_num(rng, pbad):
    return str(rng.choice(_BAD)) if rng.random() < pbad else str(rng.choice(_GOOD))


def fuzz_mps(rng):
    """A random MPS text: a mostly valid skeleton (NAME, OBJSENSE / OBJNAME
    forms, ROWS with odd types and duplicates, COLUMNS with markers, column-0
    lines and headers inside, RHS with and without set names, RANGES,
    BOUNDS of every type, a quadratic block) with comments, CRLF and, now
    and then, tokens that are not numbers or not names."""
    pbad = rng.choice([0.0, 0.0, 0.002, 0.02])
    nr, nc = int(rng.integers(1, 30)), int(rng.integers(1, 40))
    rows = [f"R{i}" for i in range(nr)]
    cols = [f"C{j}" for j in range(nc)]
    L = []

    def noise():
        if rng.random() < 0.05:
            L.append(str(rng.choice(["", "* c", "   ", "\t*", "*"])))

    L.append("NAME " + ("M%d" % rng.integers(99) if rng.random() < 0.8 else ""))
    if rng.random() < 0.3:
        L += ["OBJSENSE", "    " + str(rng.choice(["MAX", "MIN", "MAXIMIZE"]))] if rng.random() < 0.5 else \
             ["OBJSENSE " + str(rng.choice(["MAX", "MIN"]))]
    if rng.random() < 0.15:
        L.append("OBJNAME " + str(rng.choice(["OBJ", "F2", "R0"])))
    L.append(str(rng.choice(["ROWS", "rows", "Rows"])))
    L.append(" N OBJ")
    if rng.random() < 0.3:
        L.append(" N F2")
    for r in rows:
        L.append(f" {rng.choice(list('LGEXle'))} {r}")
        noise()
    if rng.random() < 0.05:
        L.append(f" L {rows[0]}")  # duplicate row
    L.append("COLUMNS")
    in_int = False
    for c in cols:
        if rng.random() < 0.15:
            in_int = not in_int
            L.append(f"    M{rng.integers(9)} 'MARKER' '{'INTORG' if in_int else 'INTEND'}'")
        k = int(rng.integers(0, 5))
        names = ["OBJ"] * (rng.random() < 0.7) + list(rng.choice(rows + ["F2", "zz"], size=k))
        i = 0
        while i < len(names):
            two = rng.random() < 0.5 and i + 1 < len(names)
            t = [c] + [f"{nm} {_fuzz_num(rng, pbad)}" for nm in names[i:i + (2 if two else 1)]]
            L.append((" " if rng.random() < 0.95 else "") + " ".join(t))
            i += 2 if two else 1
            noise()
        if rng.random() < 0.03:
            L.append("OBJSENSE MAX")
    if in_int and rng.random() < 0.7:
        L.append("    MX 'MARKER' 'INTEND'")
    L.append("RHS")
    for r in rng.choice(rows + ["OBJ"], size=int(rng.integers(0, nr + 1))):
        L.append((" RHS " if rng.random() < 0.6 else " ") + f"{r} {_fuzz_num(rng, pbad)}")
    if rng.random() < 0.5:
        L.append("RANGES")
        for r in rng.choice(rows, size=int(rng.integers(0, nr + 1))):
            L.append(f" RNG {r} {_fuzz_num(rng, pbad)}")
    if rng.random() < 0.8:
        L.append("BOUNDS")
        for _ in range(int(rng.integers(0, 2 * nc))):
            bt = str(rng.choice(["UP", "LO", "FX", "FR", "MI", "PL", "BV", "LI", "UI", "SC", "up", "fx"]))
            c = str(rng.choice(cols + (["nope"] if rng.random() < 0.02 else [])))
            if bt.upper() in ("FR", "MI", "PL", "BV"):
                L.append(f" {bt} BND {c}")
            elif rng.random() < 0.8:
                L.append(f" {bt} BND {c} {_fuzz_num(rng, pbad)}")
            else:
                L.append(f" {bt} {c} {_fuzz_num(rng, pbad)}")
    if rng.random() < 0.2:
        L.append(str(rng.choice(["QUADOBJ", "QMATRIX", "QSECTION"])))
        for _ in range(int(rng.integers(0, 6))):
            L.append(f" {rng.choice(cols)} {rng.choice(cols)} {_fuzz_num(rng, pbad)}")
    if rng.random() < 0.9:
        L.append("ENDATA")
    nl = str(rng.choice(["\n", "\r\n"]))
    return nl.join(L) + (nl if rng.random() < 0.9 else "")
