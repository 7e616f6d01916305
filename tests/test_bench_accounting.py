"""The bench's algorithmic-byte accounting (the numerators of every roofline
fraction it reports) against the survey's worked example for the 128^3 APIC
workload: P = 3,969,024 particles, N = 2,097,152 cells, F = 6,340,608 faces."""
import bench

P, N, F = 3_969_024, 128 ** 3, 3 * 129 * 128 * 128


def test_face_count_of_the_workload():
    assert F == 6_340_608


def test_stage_bytes_match_the_worked_example():
    b = bench.stage_bytes(P, 0, N, F)
    mb = {k: round(v / 1e6, 1) for k, v in b.items()}
    assert mb == {"bin_sort": 565.0, "p2g": 267.7, "forces_div": 61.2, "project": 61.2,
                  "g2p": 311.1}


def test_flip_stage_bytes_formulas():
    b = bench.stage_bytes_flip(P, N, F)
    assert b == {"bin_sort": 64 * P + 12 * N, "p2g": 24 * P + 4 * F + 2 * N,
                 "forces_div": 8 * F + 5 * N, "project": 8 * F + 5 * N, "g2p": 48 * P + 8 * F}


def test_pcg_bytes_per_iteration_and_overheads():
    # 47 B per processed cell per iteration (98.6 MB at N = 128^3), 13 N of
    # set-up and 25 N per FP64 residual replacement; processed cells are the
    # active tiles' cells
    tiles = N // 512
    one = bench.pcg_bytes({"n_active_tiles": tiles, "iters": 1, "replacements": 0})
    two = bench.pcg_bytes({"n_active_tiles": tiles, "iters": 2, "replacements": 0})
    assert round((two - one) / 1e6, 1) == 98.6
    assert bench.pcg_bytes({"n_active_tiles": tiles, "iters": 0, "replacements": 0}) == 13 * N
    rep = bench.pcg_bytes({"n_active_tiles": tiles, "iters": 0, "replacements": 1})
    assert rep - 13 * N == 25 * N
