"""bench.py's roofline accounting, without a GPU: the algorithmic bytes of each lattice
stage (the numerators of every roofline fraction on the bench line) and the committed
ncu summary it reads the DRAM traffic from."""
import bench


def test_stage_bytes_follow_the_stated_terms():
    """Each stage is the sum of the terms its docstring lists (N points, M vertices, d = 5,
    three image channels, FP32 rows of four values)."""
    N, M, d, C, p, vdp = 1000, 300, 5, 3, 4, 4
    axes = d + 1
    slot = bench.stage_bytes(N, M, d, C, p, vdp, vertex_rows=False, nbr_half=False)
    assert slot["splat"] == N * C * 4 + N * axes * 8 + M * (16 + 4 * vdp)
    assert slot["compact"] == M * (4 + 16 + 4 * vdp) + M * (16 + p * vdp + 8 + 16)
    assert slot["neighbours"] == M * 16 + 2 * axes * M * 16 + axes * M * 8
    assert slot["blur"] == axes * (2 * M * p * vdp + M * 8) + M * 4
    assert slot["slice"] == N * axes * 8 + M * 4 * vdp + N * C * 4
    vrows = bench.stage_bytes(N, M, d, C, p, vdp, vertex_rows=True, nbr_half=True)
    assert vrows["splat"] == slot["splat"] + M * (16 + 4 + 4) + M * 8 * axes
    assert vrows["compact"] == 0
    assert vrows["neighbours"] == M * 16 + axes * M * 16 + axes * M * 8 + axes * M * 4
    assert vrows["blur"] == axes * (2 * M * p * vdp + M * 8)
    assert vrows["slice"] == slot["slice"]
    # 16-bit rows: the blur moves half the row bytes and writes FP32 rows at the end
    half = bench.stage_bytes(N, M, d, C, 2, vdp, vertex_rows=True, nbr_half=True)
    assert half["blur"] == axes * (2 * M * 2 * vdp + M * 8) + M * (4 * vdp - 2 * vdp)


def test_stage_bytes_of_the_4k_frame_match_the_profile_summary():
    """The per-frame algorithmic bytes the committed 4K traffic summary compares the DRAM
    counters with: M = 1,494,033 vertices of the 3840x2160 frame, vertex-ordered rows and
    one neighbour lookup per axis (splat 653, neighbours 275, blur 359, slice 522 MB)."""
    b = bench.stage_bytes(3840 * 2160, 1494033, vertex_rows=True, nbr_half=True)
    mb = {k: round(v / 1e6) for k, v in b.items()}
    assert mb == {"splat": 653, "compact": 0, "neighbours": 275, "blur": 359, "slice": 522}


def test_ncu_traffic_reads_the_committed_summary():
    t = bench.ncu_traffic()
    for stage in ("splat", "compact", "neighbours", "blur", "slice"):
        assert stage + "_dram_bytes" in t
    assert t["splat_dram_bytes"] > 0 and t["compact_dram_bytes"] == 0
    assert all(v < 2e9 for v in t.values())   # one frame's traffic, not a batch's
