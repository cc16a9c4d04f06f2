"""The algorithmic byte counts the bench's rooflines divide by: every map
entry and dataset element a loop touches once, read-and-written data twice
(per-loop), and the union over a fused chain.  Checked on the 720k-cell mesh
against the per-call figures worked out by hand for it (FP32): res_calc
66.23 MB, bres_calc 0.21 MB (76 B per boundary edge, its nodes and cells
counted once per edge), 317.2 MB per outer iteration; 565.3 MB in FP64."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oplus2_matlab_b200 import mesh as M  # noqa: E402


def test_per_loop_and_chain_bytes_720k():
    m = M.naca0012(400, 600)
    assert (m.ncell, m.nnode, m.nedge, m.nbedge) == (720000, 721801, 1438600, 2800)
    mb = 1e6
    assert round(bench.res_calc_bytes(m) / mb, 2) == 66.23
    assert round(bench.bres_calc_bytes(m) / mb, 2) == 0.21
    assert round(bench.iteration_bytes(m) / mb, 1) == 317.2
    # union of res_calc, bres_calc, update, adt_calc: q, adt and res once
    # each way, plus qold and pcell -- 103.7 MB
    chain = bench.chain_bytes(m, "res_calc+bres_calc+update+adt_calc")
    assert round(chain / mb, 1) == 103.7
    assert chain < bench.res_calc_bytes(m) + bench.bres_calc_bytes(m) + 17 * 4 * m.ncell + \
        (16 + 4 * 4 + 4) * m.ncell + 2 * 4 * m.nnode
    # FP64 doubles every dataset byte, not the maps
    assert round(bench.iteration_bytes(m, 8) / mb, 1) == 565.3
