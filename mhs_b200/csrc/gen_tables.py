"""Emit ``tables.inc``: the constant data the device engine is compiled against.

Run once, by hand, whenever the half-space image coefficients change::

    python mhs_b200/csrc/gen_tables.py <path to mhs/kernels/_image_table.py>

Two kinds of data are written.

1. The mollified-Mindlin IMAGE coefficients. These are the kernel itself: a
   symbolic derivation (mhs tools/gen_image_table.py) reduces the half-space
   image to records ``coeff(z, nu) * D1^a D2^b D3^c / R2^n`` (R-family,
   closed form) and ``coeff(nu) * D1^a D2^b D3^c / (R2^n Q^q)`` (Q-family,
   quadrature).  Parity with mhs needs exactly these rational coefficients, so
   the records are read from mhs's generated table (mhs/kernels/_image_table.py)
   and re-laid out for the device:

   * R-family: the distinct monomials ``(a, b, c, n)`` sorted by ``n`` then
     rank, and every record as ``(slot, monomial, c[pz][pnu])`` with ``slot``
     the flattened DG ``(i, j, m)`` or DDG ``(i, j, p, m)`` index and ``c`` the
     rational coefficient of ``z^pz nu^pnu`` (pz, pnu <= 2);
   * Q-family: the distinct monomials ``(a, b, c, n, q)`` sorted by ``(n, q)``
     and every record as ``(slot, monomial, c[pnu])`` (no Q coefficient
     depends on the depth).

   The host library turns ``c`` into per-material numbers once per call.

2. ``C(-m/2, j)`` for the binomial edge series (odd m in -1..9, j < 32),
   exact rationals rounded once to double -- independent of mhs.
"""
from __future__ import annotations

import ast
import pathlib
import os
import sys
from fractions import Fraction

HERE = pathlib.Path(__file__).resolve().parent


def _load(path: pathlib.Path) -> dict:
    """Parse the generated table module without importing its package."""
    tree = ast.parse(path.read_text())
    out = {}
    for node in tree.body:
        if isinstance(node, ast.Assign) and len(node.targets) == 1:
            name = getattr(node.targets[0], "id", None)
            if name in ("DG_RECORDS", "DDG_RECORDS", "Q_DG_RECORDS",
                        "Q_DDG_RECORDS", "N_ORDERS", "MAX_RANK"):
                out[name] = ast.literal_eval(node.value)
    return out


def _flat(ix) -> int:
    s = 0
    for i in ix:
        s = s * 3 + i
    return s


def _num(x: Fraction) -> str:
    return repr(float(x))


def main(src: str) -> None:
    t = _load(pathlib.Path(src))
    lines = ["// GENERATED by gen_tables.py -- do not edit by hand.",
             "// Image-family coefficients re-laid out from mhs's generated table",
             "// (mhs/kernels/_image_table.py); binomial series constants exact.",
             "// Included once per address space: MHS_TBL is the storage qualifier of",
             "// the kernel-time tables, MHS_TBLC of the per-material coefficients.", ""]

    # ---------------- R family ----------------
    rmono = set()
    for rec in t["DG_RECORDS"]:
        rmono.add(tuple(rec[3:7]))
    for rec in t["DDG_RECORDS"]:
        rmono.add(tuple(rec[4:8]))
    rmono = sorted(rmono, key=lambda m: (m[3], m[0] + m[1] + m[2], m))
    ridx = {m: i for i, m in enumerate(rmono)}
    lines.append(f"#define MHS_R_NMONO {len(rmono)}")
    lines.append("// (a, b, c, n): D1^a D2^b D3^c / R2^n on the reflected element")
    lines.append("MHS_TBL int mhs_r_mono[MHS_R_NMONO][4] = {")
    lines += [f"  {{{a}, {b}, {c}, {n}}}," for a, b, c, n in rmono]
    lines.append("};")

    def rrecs(records, nix):
        rows = []
        for rec in records:
            slot = _flat(rec[:nix])
            mono = ridx[tuple(rec[nix:nix + 4])]
            c = [[Fraction(0)] * 3 for _ in range(3)]
            for pz, pnu, num, den in rec[nix + 4]:
                c[pz][pnu] += Fraction(num, den)
            rows.append((mono, slot, c))
        rows.sort(key=lambda r: (r[0], r[1]))
        return rows

    rlists = {}
    for name, records, nix in (("DG", t["DG_RECORDS"], 3),
                               ("DDG", t["DDG_RECORDS"], 4)):
        rows = rrecs(records, nix)
        rlists[name] = rows
        lines.append(f"#define MHS_R_N{name} {len(rows)}")
        lines.append(f"// (monomial, slot) sorted by monomial; slot = flattened "
                     f"{'(i,j,m)' if nix == 3 else '(i,j,p,m)'}")
        lines.append(f"MHS_TBL short mhs_r_{name.lower()}_idx[MHS_R_N{name}][2] = {{")
        lines += [f"  {{{m}, {s}}}," for m, s, _ in rows]
        lines.append("};")
        lines.append(f"// c[pz][pnu]: coefficient of z^pz nu^pnu")
        lines.append(f"MHS_TBLC double mhs_r_{name.lower()}_c[MHS_R_N{name}][3][3] = {{")
        for _, _, c in rows:
            lines.append("  {" + ", ".join(
                "{" + ", ".join(_num(v) for v in row) + "}" for row in c) + "},")
        lines.append("};")

    # ---------------- Q family ----------------
    qmono = set()
    for rec in t["Q_DG_RECORDS"]:
        qmono.add(tuple(rec[3:8]))
    for rec in t["Q_DDG_RECORDS"]:
        qmono.add(tuple(rec[4:9]))
    qmono = sorted(qmono, key=lambda m: (m[3], m[4], m[0] + m[1] + m[2], m))
    qidx = {m: i for i, m in enumerate(qmono)}
    lines.append(f"#define MHS_Q_NMONO {len(qmono)}")
    lines.append("// (a, b, c, n, q): D1^a D2^b D3^c / (R2^n Q^q), Q = R2 - D3")
    lines.append("MHS_TBL int mhs_q_mono[MHS_Q_NMONO][5] = {")
    lines += [f"  {{{a}, {b}, {c}, {n}, {q}}}," for a, b, c, n, q in qmono]
    lines.append("};")
    qlists = {}
    for name, records, nix in (("DG", t["Q_DG_RECORDS"], 3),
                               ("DDG", t["Q_DDG_RECORDS"], 4)):
        rows = []
        for rec in records:
            slot = _flat(rec[:nix])
            mono = qidx[tuple(rec[nix:nix + 5])]
            c = [Fraction(0)] * 3
            for pz, pnu, num, den in rec[nix + 5]:
                assert pz == 0, "a Q-family coefficient depends on depth"
                c[pnu] += Fraction(num, den)
            rows.append((mono, slot, c))
        rows.sort(key=lambda r: (r[0], r[1]))
        lines.append(f"#define MHS_Q_N{name} {len(rows)}")
        lines.append(f"MHS_TBL short mhs_q_{name.lower()}_idx[MHS_Q_N{name}][2] = {{")
        lines += [f"  {{{m}, {s}}}," for m, s, _ in rows]
        lines.append("};")
        lines.append(f"MHS_TBLC double mhs_q_{name.lower()}_c[MHS_Q_N{name}][3] = {{")
        lines += ["  {" + ", ".join(_num(v) for v in c) + "}," for _, _, c in rows]
        lines.append("};")
        qlists[name] = rows

    # ---------------- binomial series ----------------
    lines.append("// C(-m/2, j) for m = -1, 1, 3, 5, 7, 9 (row (m+1)/2), j = 0..31")
    lines.append("MHS_TBL double mhs_binom_half[6][32] = {")
    for m in (-1, 1, 3, 5, 7, 9):
        a = Fraction(-m, 2)
        vals, cur = [], Fraction(1)
        for j in range(32):
            vals.append(cur)
            cur = cur * (a - j) / (j + 1)
        lines.append("  {" + ", ".join(_num(v) for v in vals) + "},")
    lines.append("};")
    # 1 / k as the compiler rounds 1.0 / (double)k, for loops whose k is not
    # a compile-time constant
    lines.append("MHS_TBL double mhs_inv_int[128] = {")
    lines.append("  0.0, " + ", ".join(repr(1.0 / k) for k in range(1, 128)))
    lines.append("};")
    (HERE / "tables.inc").write_text("\n".join(lines) + "\n")
    # X-macro lists of the Q family for straight-line device code: the
    # monomials each contraction reads (global index, exponents) and its
    # records in table order (record, monomial, slot).
    ql = ["// GENERATED by gen_tables.py -- do not edit by hand.",
          "// Q-family lists as X-macros over the records of tables.inc.", ""]
    for name in ("DG", "DDG"):
        used = sorted({m for m, _, _ in qlists[name]})
        ql.append(f"#define MHS_Q_MONO_{name}(X) \\")
        ql += [f"  X({i}, {qmono[i][0]}, {qmono[i][1]}, {qmono[i][2]}, {qmono[i][3]}, {qmono[i][4]}) \\"
               for i in used]
        ql.append("")
        ql.append(f"#define MHS_Q_TERMS_{name}(X) \\")
        ql += [f"  X({r}, {m}, {sl}) \\" for r, (m, sl, _) in enumerate(qlists[name])]
        ql.append("")
    (HERE / "tables_q.inc").write_text("\n".join(ql) + "\n")
    # X-macro lists of the R family: every monomial (index, exponents) and
    # each contraction's records in table order (record, monomial, slot).
    rl = ["// GENERATED by gen_tables.py -- do not edit by hand.",
          "// R-family lists as X-macros over the records of tables.inc.", ""]
    rl.append("#define MHS_R_MONO(X) \\")
    rl += [f"  X({i}, {a}, {b}, {c}, {n}) \\" for i, (a, b, c, n) in enumerate(rmono)]
    rl.append("")
    for name in ("DG", "DDG"):
        rl.append(f"#define MHS_R_TERMS_{name}(X) \\")
        rl += [f"  X({r}, {m}, {sl}) \\" for r, (m, sl, _) in enumerate(rlists[name])]
        rl.append("")
    (HERE / "tables_r.inc").write_text("\n".join(rl) + "\n")
    print(f"wrote {HERE / 'tables.inc'}: R {len(rmono)} monomials, "
          f"Q {len(qmono)} monomials")


def _table_path() -> str:
    """mhs/kernels/_image_table.py of the reference tree: the first argument,
    else under $MHS_REFERENCE_SRC (the reference's src/ directory)."""
    if len(sys.argv) > 1:
        return sys.argv[1]
    root = os.environ.get("MHS_REFERENCE_SRC")
    if not root:
        sys.exit("usage: gen_tables.py <mhs/kernels/_image_table.py> "
                 "(or set MHS_REFERENCE_SRC to the reference's src/ directory)")
    return os.path.join(root, "mhs", "kernels", "_image_table.py")


if __name__ == "__main__":
    main(_table_path())
