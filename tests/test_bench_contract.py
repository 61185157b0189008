"""Host-side pieces of bench.py's JSON line: the roofline traffic comes from
the committed ncu capture of the plan that actually ran, and the plan
description names each plan's own parameters."""
import json
import os

import bench


def _traffic(workload, mode, B, R=0):
    p = bench.committed_profile(workload, mode, B, R)
    return p.get("dram_bytes_per_launch") if p else None


def test_traffic_is_looked_up_per_plan_and_group_variant():
    # FCI(12,12): plan 5 and plan 7 with group variants 2 and 3 were captured
    assert _traffic("fci12_12", 5, 1) > 0
    assert _traffic("fci12_12", 7, 3) > 0
    assert _traffic("fci12_12", 7, 2) > 0
    # plans or variants without a capture report no traffic
    assert _traffic("fci12_12", 7, 4) is None
    assert _traffic("fci12_12", 1, 1) is None
    assert _traffic("fci14_14_fc2", 6, 2) > 0
    assert _traffic("fci14_14_fc2", 6, 3) is None
    assert _traffic("no_such_workload", 5, 1) is None


def test_every_traffic_entry_points_at_a_committed_summary():
    prof = os.path.join(bench.ROOT, "profiles")
    for name in os.listdir(prof):
        if not name.endswith("_traffic.json"):
            continue
        d = json.load(open(os.path.join(prof, name)))
        assert d["plans"]
        for key, plan in d["plans"].items():
            mode = int(key.split(":")[0])
            assert mode in bench.PLAN_NAMES
            # group plans carry their variant, blocked and shared panels a suffix
            stem = key.replace(":blk", "").replace(":row", "").replace(":cp", "").replace(":hs", "")
            assert (":" in stem) == (mode in (6, 7))
            assert plan["dram_bytes_per_launch"] > 0 and plan["kernels"]
            assert os.path.exists(os.path.join(bench.ROOT, plan["summary"]))


def test_plan_description_names_each_plans_parameters():
    d = bench.sigma_plan_desc(7, 512, 16, 3)
    assert d["beta_singles_threads"] == 512 and d["product_engine"] == "16 column threads"
    assert "split over 4 warps, 2 column" in d["group_kernel"]
    assert "tcgen05" in bench.sigma_plan_desc(7, 512, 64, 3)["product_engine"]
    d = bench.sigma_plan_desc(6, 512, 18, 2)
    assert d["product_ctas_per_sm"] == 2 and d["product_panel"] == "256-column blocks"
    d = bench.sigma_plan_desc(6, 512, 33, 2)
    assert d["product_ctas_per_sm"] == 1 and "shared by all CTAs" in d["product_panel"]
    assert bench.sigma_plan_desc(6, 512, 2, 2)["product_panel"] == "whole alpha row per CTA"
    d = bench.sigma_plan_desc(6, 512, 66, 5)
    assert d["product_ctas_per_sm"] == 2 and "compact" in d["product_panel"]
    assert bench.profile_key(6, 66, 5) == "6:5:cp"
    assert bench.profile_key(6, 66, 5, 0) == "6:5:hs:cp"
    assert bench.sigma_plan_desc(6, 0, 66, 5)["beta_singles"] == "hole-string products"
    assert "1 column" in bench.sigma_plan_desc(6, 256, 0, 1)["group_kernel"]
    assert "split over 4 warps, 1 column" in bench.sigma_plan_desc(6, 256, 0, 4)["group_kernel"]
    assert "hole-string" in bench.sigma_plan_desc(6, 256, 0, 5)["group_kernel"]
    assert "4 GiB" in bench.sigma_plan_desc(6, 256, 0, 7)["group_kernel"]
    assert "64-column" in bench.sigma_plan_desc(7, 256, 16, 6)["group_kernel"]
    d = bench.sigma_plan_desc(3, 256, 0, 512)
    assert d["alpha_pass_threads"] == 256 and d["beta_pass_threads"] == 512
    d = bench.sigma_plan_desc(5, 256, 16, 2)
    assert d["row_kernel_threads"] == 256 and d["rows_per_cta"] == 2
    assert set(bench.SIGMA_KERNELS) == set(bench.PLAN_NAMES) == set(range(8))


def test_tensor_pipe_figures_come_from_committed_captures():
    tp = bench.committed_tensor_pipe("fci12_12")
    assert "not measured in the run" in tp["source"]
    names = [k["kernel"] for k in tp["kernels"]]
    assert any(n.startswith("k_gram") for n in names)
    for k in tp["kernels"]:
        assert 0 < k["active_pct"] <= 100
        assert os.path.exists(os.path.join(bench.ROOT, k["summary"]))
    assert bench.committed_tensor_pipe("cas10_10") is None


def test_default_workload_is_the_largest_single_gpu_configuration():
    import sys
    old = sys.argv
    try:
        sys.argv = ["bench.py"]
        import argparse
        seen = {}
        real = argparse.ArgumentParser.parse_args

        def grab(self, *a, **k):
            ns = real(self, *a, **k)
            seen["ns"] = ns
            raise SystemExit(0)
        argparse.ArgumentParser.parse_args = grab
        try:
            bench.main()
        except SystemExit:
            pass
        finally:
            argparse.ArgumentParser.parse_args = real
    finally:
        sys.argv = old
    assert seen["ns"].workload == "fci16_16"
    assert bench.SOLVES_OF["fci16_16"] == "fci14_14_fc2"


def test_reference_calibration_separates_fixed_and_row_costs():
    class Fake:
        """A reference whose call costs 4 s plus 1 ms per row."""
        def step(self, rows):
            return 4.0 + 1e-3 * rows, rows
    fixed, per_row = bench.calibrate(Fake(), 2000, 20000)
    assert abs(fixed - 4.0) < 1e-9 and abs(per_row - 1e-3) < 1e-12
    assert bench.sample_rows(fixed, per_row, 15.0, 20000, 10 ** 9) == 11000


def test_reference_calibration_is_bounded_when_noise_hides_the_rows():
    class Noisy:
        """Fixed cost 3 s with noise larger than the rows' cost: the second
        call, with ten times the rows, comes out faster."""
        def __init__(self):
            self.t = iter([5.0, 3.2, 3.1])
        def step(self, rows):
            return next(self.t), rows
    fixed, per_row = bench.calibrate(Noisy(), 2000, 165636)
    assert fixed == 0.0 and per_row == 3.1 / 165636
    rows = bench.sample_rows(fixed, per_row, 15.0, 165636, 165636900)
    assert rows <= 64 * 165636 and rows * per_row <= 15.0 + 1e-9
    assert bench.calib_sizes(165636900) == (2000, 165636)


def test_reference_threads_are_bounded_by_memory():
    # one full-length private buffer per thread: a huge vector gets one thread
    assert bench.host_threads(10 ** 13, 1) == 1
    assert 1 <= bench.host_threads(1000, 1) <= (os.cpu_count() or 1)
    # the reference's int-sized buffer block: FCI(16e,16o) fits 12 threads
    assert bench.host_threads(165636900, 1) <= 12
