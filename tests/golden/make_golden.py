"""Generates tests/golden/lss_symmetric_dirichlet_kat.json from the reference's
own known-answer test of symmetric_dirichlet, read as text
(test/math/utest-lss-symmetric-dirichlet.cpp: the commpattern of
build_commpattern, the set_row / symmetric_dirichlet calls and every
BOOST_CHECK_EQUAL of test_complete_system), with each rank's local indices
mapped to global node ids.  Note the reference's get_value(icol, irow) order.

Run where the reference tree is available, with its root as the argument:
    python tests/golden/make_golden.py <reference root>
"""
from __future__ import annotations

import json
import os
import re
import sys

SRC = "test/math/utest-lss-symmetric-dirichlet.cpp"


def parse(text: str) -> dict:
    cp = text[text.index("void build_commpattern"):text.index("void build_system")]
    gids = [list(map(int, m.split(","))) for m in re.findall(r"gid \+= ([\d,]+);", cp)]
    body = text[text.index("BOOST_AUTO_TEST_CASE( test_complete_system )"):]
    body = body[:body.index("BOOST_AUTO_TEST_CASE( finalize_mpi )")]
    set_rows = [tuple(float(x) for x in m) for m in
                re.findall(r"set_row\((\d+), (\d+), ([\d.]+), ([\d.]+)\)", body)]
    dirichlet = re.findall(r"symmetric_dirichlet\((\d+), (\d+), ([\d.]+)\.?,", body)
    branches = [body[body.index("if(irank == 0)\n  {"):body.index("else\n  {")], body[body.index("else\n  {"):]]
    matrix, rhs = [], []
    for rank, part in enumerate(branches):
        g = gids[rank]
        for col, row, val in re.findall(r"matrix\(\)->get_value\((\d+), (\d+), val\);\s*BOOST_CHECK_EQUAL\(val, "
                                        r"(-?[\d.]+)\);", part):
            matrix.append({"row": g[int(row)], "col": g[int(col)], "value": float(val), "rank": rank})
        for idx, val in re.findall(r"rhs\(\)->get_value\((\d+), val\);\s*BOOST_CHECK_EQUAL\(val, (-?[\d.]+)\);",
                                   part):
            rhs.append({"row": g[int(idx)], "value": float(val), "rank": rank})
    # the Dirichlet call: rank 0 uses its local node 1, rank 1 its local node 0 (the same global node)
    bc_nodes = sorted({gids[0][int(dirichlet[0][0])], gids[1][int(dirichlet[1][0])]})
    return {
        "source": f"{SRC} (test_complete_system)",
        "nodes": 4,
        "neq": 1,
        "graph": "chain 0-1-2-3 (each node coupled to itself and its neighbours)",
        "set_row": {"diag": set_rows[0][2], "offdiag": set_rows[0][3]},
        "dirichlet": {"node": bc_nodes[0], "eq": int(dirichlet[0][1]), "value": float(dirichlet[0][2])},
        "matrix_checks": matrix,
        "rhs_checks": rhs,
    }


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference root>")
    root = sys.argv[1]
    text = open(os.path.join(root, SRC)).read()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lss_symmetric_dirichlet_kat.json")
    with open(out, "w") as f:
        json.dump(parse(text), f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
