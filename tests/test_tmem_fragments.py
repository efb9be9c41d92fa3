"""The tensor-memory LU and solve fragments (csrc/gen/radm2_{decomp,solve}{_rcp,}_tm.inc: the
reciprocal-pivot and the division form for the 128-slot map; radm2_{decomp,solve}{_rcp,}_tm_wide.inc:
both forms for the 256-slot map) against the plain ones they stand in for, read as text on
the CPU.

- Every tcgen05 load and store piece covers exactly its slots' columns (radm2_tmem.h,
  radm2_tmem_wide.h): in slot order, two 32-bit columns per double, starting on a multiple of
  its own width, inside the thread's 256 columns (512 with the wide map).
- With the tensor-memory temporaries read back as G(s), the eliminations, the substitution
  rows and each row's stored values are the plain fragments' own, in the same order.
"""
import os
import re

import pytest
from conftest import PKG

GEN = os.path.join(PKG, "csrc", "gen")


def read(name):
    with open(os.path.join(GEN, name)) as f:
        return f.read()


def tmem_cols(tag):
    text = read("radm2_tmem%s.h" % tag)
    m = re.search(r"radm2_tmem%s_col\[(\d+)\] = \{([^}]*)\}" % tag, text)
    return [int(v) for v in m.group(2).split(",")]


MAPS = {"": (tmem_cols(""), 256), "_wide": (tmem_cols("_wide"), 512)}  # tag: (columns, columns per thread)
PIECE = re.compile(r"tcgen05\.(ld|st)\.sync\.aligned\.32x32b\.x(\d+)\.b32")


# (form, map): reciprocal pivots (the fast solver) or divisions (reference arithmetic), with
# the 128-slot and with the 256-slot map
FORMS = [("_rcp", ""), ("", ""), ("_rcp", "_wide"), ("", "_wide")]


def test_wide_map_holds_the_most_used_slots():
    narrow, wide = MAPS[""][0], MAPS["_wide"][0]
    assert sum(c >= 0 for c in narrow) == 128 and sum(c >= 0 for c in wide) == 256
    assert sorted(c for c in wide if c >= 0) == list(range(0, 512, 2))
    assert all(wide[s] >= 0 for s in range(len(narrow)) if narrow[s] >= 0)


@pytest.mark.parametrize("form,tag", FORMS)
def test_load_and_store_pieces_cover_their_columns(form, tag):
    COL, ncol = MAPS[tag]
    n = 0
    for name in ("radm2_decomp%s_tm%s.inc" % (form, tag), "radm2_solve%s_tm%s.inc" % (form, tag)):
        for line in read(name).splitlines():
            if "tcgen05.ld" in line:
                widths = [int(w) for op, w in PIECE.findall(line)]
                slots = [int(s) for s in re.findall(r'"=r"\(tl(\d+)\)', line)]
                bases = [int(b) for b in re.findall(r"TM_BASE \+ (\d+)u", line)]
                assert len(widths) == len(bases) and sum(widths) == 2 * len(slots)
                assert line.count("tcgen05.wait::ld") == 1 and line.rstrip().endswith(");")
                i = 0
                for w, b in zip(widths, bases):
                    assert w in (2, 4, 8, 16) and b % w == 0 and b + w <= ncol
                    for q in range(w // 2):
                        assert COL[slots[i + q]] == b + 2 * q
                    i += w // 2
                n += 1
            elif "tcgen05.st" in line:
                (op, w), = PIECE.findall(line)
                w = int(w)
                b = int(re.search(r"TM_BASE \+ (\d+)u", line).group(1))
                assert w in (2, 4, 8, 16) and b % w == 0 and b + w <= ncol
                assert line.count("__double2loint") == w // 2
                n += 1
    assert n > 100


def normalise(text):
    """Statements of a fragment with tensor-memory temporaries written as G(s) and the
    load blocks, declarations and waits removed."""
    out = []
    skip = 0
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("{ unsigned"):
            skip = 1
            continue
        if skip:
            if s == "}":
                skip = 0
            continue
        if (not s or s.startswith("/*") or s.startswith("*") or s.startswith("#") or s in ("{", "}")
                or s.startswith("LU_T u") or re.fullmatch(r"LU_T w\d+;", s) or s.startswith("double g")
                or "wait::st" in s or s.startswith("LU_PIVOT_CHECK")):
            continue
        if s.startswith("{ "):  # the plain fragment opens an elimination step on its first line
            s = s[2:]
        s = re.sub(r"\b[ug](\d+)\b", r"G(\1)", s)
        out.append(s)
    return out


@pytest.mark.parametrize("form,tag", FORMS)
def test_solves_are_the_plain_solves(form, tag):
    plain = [s for s in normalise(read("radm2_solve%s.inc" % form))]
    tm = normalise(read("radm2_solve%s_tm%s.inc" % (form, tag)))
    assert tm == plain


def stores_by_row(text, tm, COL=None):
    rows, cur = [], None
    for line in text.splitlines():
        m = re.match(r"\{ /\* row (\d+) \*/", line)
        if m:
            cur = {}
            rows.append(cur)
            continue
        if cur is None:
            continue
        g = re.match(r"\s*G\((\d+)\) = (.*);$", line)
        if g:
            cur[int(g.group(1))] = g.group(2)
        if tm and "tcgen05.st" in line:
            b = int(re.search(r"TM_BASE \+ (\d+)u", line).group(1))
            vals = re.findall(r"__double2loint\((.*?)\)\), \"r\"\(__double2hiint", line)
            for q, v in enumerate(vals):
                cur[COL.index(b + 2 * q)] = v
    return rows


@pytest.mark.parametrize("form,tag", FORMS)
def test_factorisation_is_the_plain_factorisation(form, tag):
    plain_text, tm_text = read("radm2_decomp%s.inc" % form), read("radm2_decomp%s_tm%s.inc" % (form, tag))
    elim = lambda lines: [s for s in lines if "const LU_T a =" in s or "+= a *" in s]  # noqa: E731
    assert elim(normalise(tm_text)) == elim(normalise(plain_text))
    sp, st = stores_by_row(plain_text, False), stores_by_row(tm_text, True, MAPS[tag][0])
    assert len(sp) == len(st) == 59
    def norm(v):
        v = v.strip()
        while v.startswith("((") and v.endswith(")"):
            v = v[1:-1]
        return v

    for k, (a, b) in enumerate(zip(sp, st)):
        assert set(a) == set(b), k
        for slot in a:
            va, vb = norm(a[slot]), norm(b[slot])
            # a row without eliminations: the plain form stores 1/G(d), the tensor-memory
            # form 1/w<row> with w<row> just loaded from slot d
            assert va == vb or (va == "(LU_T)1 / G(%d)" % slot and vb == "(LU_T)1 / w%d" % k), (k, slot, va, vb)
