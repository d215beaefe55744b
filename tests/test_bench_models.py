"""Host-side byte models of bench.py (no GPU): the roofline numerators of the
merge kernels and of the whole insert step, and the ncu traffic figure read
from the committed insert profile."""
import bench

STATS = {"last_keys": 2_000_000, "last_applied": 1_150_000, "last_rewritten": 1_280_000,
         "last_gathered": 62_300_000, "last_written": 63_600_000, "last_hub_read": 1_300_000,
         "last_hub_written": 1_310_000, "last_hub_touched": 1_800}


def test_merge_bytes_cover_tiers_one_and_two_only():
    so = STATS["last_gathered"] - STATS["last_hub_read"]
    sn = STATS["last_written"] - STATS["last_hub_written"]
    nr = STATS["last_rewritten"] - STATS["last_hub_touched"]
    want = 4 * so + 8 * STATS["last_applied"] + 4 * sn + 40 * nr
    assert bench.kernel_bytes("upd_merge", STATS) == want


def test_step_roofline_counts_inputs_keys_and_all_tiers():
    r = bench.step_roofline([STATS, STATS], 1.0, 6553.6, "measured")
    want = (8 * bench.BATCH + 16 * STATS["last_keys"] + 4 * STATS["last_gathered"]
            + 8 * STATS["last_applied"] + 4 * STATS["last_written"] + 40 * STATS["last_rewritten"])
    assert r["bytes_per_step"] == want
    assert abs(r["achieved"] - want / 1e-3 / 1e9) < 1e-9
    assert abs(r["frac"] - r["achieved"] / 6553.6) < 1e-12
    assert r["unit"] == "GB/s" and r["bound"] == "hbm"


def test_merge_traffic_is_read_from_the_insert_profile():
    traffic, src = bench.ncu_traffic("upd_merge")
    assert src == "profiles/insert_rmat22_batch1e6.md"
    assert traffic and traffic > 1e8
    assert bench.ncu_traffic("no_such_kernel") == (None, None)
