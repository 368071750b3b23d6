"""Writes mpm_pow_tables.h: the constant tables of the f64 log / exp used by
powf_m (mpm_math.cuh) and by the oracle's or_powf, which must agree bit for
bit and therefore read the same table file.

    python gen_pow_tables.py            # rewrites mpm_pow_tables.h beside this file

Every entry is the f64 value nearest the exact quantity, computed with
60-digit decimal arithmetic:
  POW_INVC[j]  = RN(1 / c_j), c_j = 1 + (j + 1/2) / 128, j = 0..127
                 (centre of the j-th 1/128 slice of the mantissa range [1, 2))
  POW_NLOGC[j] = RN(-log(POW_INVC[j]))   (log of the rounded reciprocal, so
                 log m = POW_NLOGC[j] + log(m * POW_INVC[j]) holds exactly)
  POW_EXP2[i]  = RN(2^(i / 64)), i = 0..63
"""
from __future__ import annotations

import os
from decimal import Decimal, getcontext

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "mpm_pow_tables.h")


def _rows(name: str, n: int, vals: list[float]) -> str:
    items = [float.hex(v) for v in vals]
    lines = [f"MPM_POW_TABLE double {name}[{n}] = {{"]
    for i in range(0, n, 4):
        lines.append("    " + ", ".join(items[i:i + 4]) + ",")
    lines.append("};")
    return "\n".join(lines)


def render() -> str:
    getcontext().prec = 60
    invc = [256.0 / (257 + 2 * j) for j in range(128)]          # IEEE division: RN(256 / (257 + 2j))
    nlogc = [float(-(Decimal(v).ln())) for v in invc]            # Decimal(v) is exact
    exp2 = [float(Decimal(2) ** (Decimal(i) / Decimal(64))) for i in range(64)]
    head = [
        "// Generated by gen_pow_tables.py; do not edit.",
        "// Tables of the f64 log / exp behind powf_m (mpm_math.cuh) and the oracle's",
        "// or_powf.  The includer defines MPM_POW_TABLE (storage class and qualifiers).",
        "// POW_INVC[j]  = RN(1 / c_j), c_j = 1 + (j + 1/2) / 128",
        "// POW_NLOGC[j] = RN(-log(POW_INVC[j]))",
        "// POW_EXP2[i]  = RN(2^(i / 64))",
        "#ifndef MPM_POW_TABLE",
        "#error define MPM_POW_TABLE before including mpm_pow_tables.h",
        "#endif",
    ]
    return "\n".join(head + [_rows("POW_INVC", 128, invc), _rows("POW_NLOGC", 128, nlogc),
                             _rows("POW_EXP2", 64, exp2)]) + "\n"


if __name__ == "__main__":
    with open(OUT, "w") as f:
        f.write(render())
    print(OUT)
