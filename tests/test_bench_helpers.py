"""bench.py's host-side helpers: backprojection batch counting and the clock-sample parser."""
import bench


def test_batches_of_in_order_pushes():
    # 128 steps of 32 views in order, 128-view batches: one batch per 4 steps
    assert bench.count_bp_batches([32 * i for i in range(128)], 32, 128) == [128] * 32
    # a partial last batch is flushed at the end
    assert bench.count_bp_batches([32 * i for i in range(5)], 32, 128) == [128, 32]
    # the driver's 20-step run at 512-view batches: a full batch and a 128-view flush
    assert bench.count_bp_batches([32 * i for i in range(5, 25)], 32, 512) == [512, 128]


def test_batches_break_on_discontinuity():
    # the views restart (the workload wraps around): the waiting batch is backprojected first
    assert bench.count_bp_batches([0, 32, 0, 32], 32, 128) == [64, 64]
    # a push larger than a batch fills several batches
    assert bench.count_bp_batches([0], 300, 128) == [128, 128, 44]


class _Done:
    def terminate(self):
        pass

    def wait(self, timeout=None):
        return 0


def test_clock_parser_reads_median_max_and_reasons():
    c = bench.ClockSampler(0)
    c.proc = _Done()
    c.lines = ["0, 1965, 1965, 600.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1900, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1950, 1965, 800.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "garbage line"]
    r = c.stop()
    assert r["sm_mhz"] == 1950 and r["sm_max_mhz"] == 1965 and r["samples"] == 3
    assert r["reasons"] == ["sw_power_cap"]


def test_clock_parser_without_nvidia_smi():
    assert bench.ClockSampler(0).stop()["reasons"] == ["nvidia-smi unavailable"]
