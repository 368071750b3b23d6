"""Writes mpm_mc_table.h: the marching-cubes case table of the reference, the
data contract that fixes which triangles (and in which vertex order) each of
the 256 cube cases produces, so the vertex buffer equals the reference's.

    python gen_mc_table.py <reference checkout>   # rewrites mpm_mc_table.h beside this file

Reads, from the reference checkout:
  src/lib/gpu/marchingCubes/triTable.wgsl  MC_TRI_TABLE: per case up to 15 edge
                                           indices (5 triangles), -1 after the last
  src/lib/gpu/marchingCubes/prelude.wgsl   MC_TRI_COUNTS: triangles per case
and checks that the two agree (every case lists exactly 3 x count edges, then
only -1) before writing both.  The edge numbering is the reference's
(prelude.wgsl: vertex id = x + 2z + 4y; edges along x, then y, then z), which
the kernels use as well.  The header is included by the CUDA passes
(mpm_mc.cu) and by the oracle (oracle/mc_oracle.c), so both triangulate with
the same numbers.
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "mpm_mc_table.h")


def read_tables(ref_root: str):
    mc = os.path.join(ref_root, "src", "lib", "gpu", "marchingCubes")
    with open(os.path.join(mc, "triTable.wgsl")) as f:
        text = f.read()
    body = text[text.index("MC_TRI_TABLE"):]
    rows = re.findall(r"array<i32,\s*16>\(([^)]*)\)", body)
    tri = [[int(v) for v in r.split(",")] for r in rows]
    with open(os.path.join(mc, "prelude.wgsl")) as f:
        prelude = f.read()
    m = re.search(r"MC_TRI_COUNTS\s*=\s*array<u32,\s*256>\(([^;]*)\);", prelude, re.S)
    if not m:
        raise ValueError("MC_TRI_COUNTS not found")
    counts = [int(v.strip().rstrip("u")) for v in m.group(1).split(",") if v.strip()]
    if len(tri) != 256 or any(len(r) != 16 for r in tri) or len(counts) != 256:
        raise ValueError("unexpected table shape")
    for c in range(256):
        k = 3 * counts[c]
        if any(not 0 <= e < 12 for e in tri[c][:k]) or any(e != -1 for e in tri[c][k:]):
            raise ValueError(f"case {c}: triangle list and count disagree")
    return tri, counts


def render(tri, counts) -> str:
    out = ["// mpm_mc_table.h -- generated by gen_mc_table.py from the reference's",
           "// marchingCubes/triTable.wgsl (MC_TRI_TABLE) and prelude.wgsl (MC_TRI_COUNTS).",
           "// Do not edit by hand.  Case c = bit v set when cube vertex v is above the",
           "// isovalue (vertex id = x + 2z + 4y); entries are edge ids, 3 per triangle,",
           "// -1 after the last triangle.",
           "#pragma once",
           "#include <stdint.h>",
           "",
           "static const int8_t MPM_MC_TRI_TABLE[256][16] = {"]
    for c in range(256):
        out.append("    {" + ", ".join(f"{v:2d}" for v in tri[c]) + f"}},  /* {c} */")
    out.append("};")
    out.append("")
    out.append("static const uint8_t MPM_MC_TRI_COUNTS[256] = {")
    for i in range(0, 256, 16):
        out.append("    " + ", ".join(str(v) for v in counts[i:i + 16]) + ",")
    out.append("};")
    return "\n".join(out) + "\n"


def main(argv):
    if len(argv) != 2:
        print(__doc__)
        return 2
    tri, counts = read_tables(argv[1])
    with open(OUT, "w") as f:
        f.write(render(tri, counts))
    print(f"wrote {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
