"""CPU: the byte counts behind bench.py's throughput and roofline numbers.

Per product (one orientation, b right-hand sides, e bytes per complex entry):
    e (near + coupling + transfer + leaf-basis entries)    stores, each read once
  + e b (N_trial + 2 N_test)                               x read, y read and written
  + 2 e b (coefficients of both sides)                     x-hat and y-hat written and read once
and for the near-field launch: e near entries + e b (N_trial + N_test)."""
import bench

INFO = {"near_entries": 1000, "coupling_entries": 200, "transfer_entries_test": 30, "transfer_entries_trial": 40,
        "basis_entries_test": 50, "basis_entries_trial": 60, "ntest": 70, "ntrial": 80, "ncoeff_test": 9,
        "ncoeff_trial": 11}


def test_product_bytes():
    for e, b in ((16, 1), (16, 16), (8, 16)):
        stores = 1000 + 200 + 30 + 40 + 50 + 60
        want = e * stores + e * b * (80 + 2 * 70) + 2 * e * b * (9 + 11)
        assert bench.product_bytes(INFO, b, e) == want


def test_near_stage_bytes():
    assert bench.stage_bytes(INFO, 16, 16) == 16 * 1000 + 16 * 16 * (80 + 70)
    assert bench.stage_bytes(INFO, 16, 8) == 8 * 1000 + 8 * 16 * (80 + 70)


def test_traffic_from_profiles_reads_the_committed_summary():
    t = bench.traffic_from_profiles()
    assert t is not None and t > 1.3e9  # the 65,536-point near-field launch moves about 1.4 GB
