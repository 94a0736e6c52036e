"""The benchmark's byte model (CPU): the algorithmic HBM bytes per launch that
the roofline fractions divide, and the neighbour-row bytes the gather view
reports, on a small hand-counted scene."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def test_kernel_bytes_d3q27_counts():
    # 10 bulk, 6 layer, 4 boundary nodes, k = kb = 32; 7 visited nodes
    # holding 50 layer-support records
    N, nb, nl, nbd, k = 20, 10, 6, 4, 32
    kb = bench.kernel_bytes(3, N, nb, nl, nbd, k, k, (7, 50))
    row, st = 4 * 27, 4 * k * 4  # algorithmic rows: the 27 populations, unpadded
    assert kb["macro_pml"] == N * (4 * row + 32) + nl * row
    assert kb["pml_gather"] == 50 * 16 + 7 * (2 * row + 32) + nl * row
    assert kb["filter"] == N * 2 * row + (nb + nl) * 8 * k
    assert kb["rk_stage1"] == (nb + nl) * (st + 2 * row)
    assert kb["rk_stage2"] == kb["rk_stage3"] == kb["rk_stage4"] == (nb + nl) * (st + 3 * row)
    assert kb["edge_collide"] == nbd * (2 * row + 8 * k)
    assert kb["edge_interp"] == nbd * (8 * k + row)


def test_kernel_bytes_d2q9_gathers_the_moving_populations():
    kb = bench.kernel_bytes(2, 20, 10, 6, 4, 16, 16, (7, 50))
    st = 4 * 16 * 3
    assert kb["rk_stage1"] == 16 * (st + 2 * 32)
    assert kb["pml_gather"] == 50 * 16 + 7 * (2 * 32 + 32) + 6 * 32


def test_gather_bytes_one_row_per_reference():
    # the loads move the padded 112-B row (seven 16-B chunks)
    gb = bench.gather_bytes(10, 6, 4, 32, 32, (7, 50))
    assert gb["filter"] == gb["rk_stage1"] == gb["rk_stage4"] == 16 * 32 * 112
    assert gb["pml_gather"] == 50 * 112
    assert gb["edge_collide"] == gb["edge_interp"] == 4 * 32 * 112
    # every step kernel with a gather is covered, and only those
    assert set(gb) == set(bench.kernel_bytes(3, 20, 10, 6, 4, 32, 32, (7, 50))) - {"macro_pml"}


def test_dominant_kernel_counts_the_rk_stages_as_one():
    # the PML gather is the longest single launch, but the four RK stages
    # (one kernel, four launches a step) take the largest share
    kb = bench.kernel_bytes(3, 20, 10, 6, 4, 32, 32, (7, 50))
    prof = {n: (5, 0.30) for n in kb}
    prof.update({"pml_gather": (5, 0.40), "rk_stage1": (5, 0.34), "rk_stage2": (5, 0.36),
                 "rk_stage3": (5, 0.36), "rk_stage4": (5, 0.36)})
    top, per_launch, avg_ms, members = bench.dominant_kernel(kb, prof)
    assert top == "rk_stage1..4" and members == list(bench.RK_STAGES)
    assert per_launch == sum(kb[n] for n in bench.RK_STAGES) / 4
    assert abs(avg_ms - (0.34 + 3 * 0.36) / 20) < 1e-12
    # a kernel that takes more than the four stages together is dominant
    prof["filter"] = (5, 2.0)
    top, per_launch, avg_ms, members = bench.dominant_kernel(kb, prof)
    assert top == "filter" and members == ["filter"] and per_launch == kb["filter"] and avg_ms == 2.0 / 5
