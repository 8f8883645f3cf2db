"""bench.py's host-side helpers: backprojection batch counting and the clock-sample parser."""
import bench


def test_batches_of_in_order_pushes():
    # 128 steps of 32 views in order, 128-view batches: one batch per 4 steps
    assert bench.count_bp_batches([32 * i for i in range(128)], 32, 128) == [128] * 32
    # a partial last batch is flushed at the end
    assert bench.count_bp_batches([32 * i for i in range(5)], 32, 128) == [128, 32]
    # the driver's 20-step run at 512-view batches: a full batch and a 128-view flush
    assert bench.count_bp_batches([32 * i for i in range(5, 25)], 32, 512) == [512, 128]


def test_batches_break_on_discontinuity_only_for_contiguous_batches():
    # FP32_EXACT batches hold consecutive views: a restart closes the waiting batch
    assert bench.count_bp_batches([0, 32, 0, 32], 32, 128, contiguous=True) == [64, 64]
    # the staged precisions take views in any order
    assert bench.count_bp_batches([0, 32, 0, 32], 32, 128) == [128]
    # a push larger than a batch fills several batches
    assert bench.count_bp_batches([0], 300, 128) == [128, 128, 44]


def test_step_chunks_read_every_view_once_in_quarter_order():
    import fdk_b200 as F

    p = F.config("c3")
    seen = sorted(v for b in range(128) for f, n in bench.step_chunks(p, b, order="quarter") for v in range(f, f + n))
    assert seen == list(range(4096))
    # each step: 8 views from each quarter, partners v + k N/4 in the same step
    ch = bench.step_chunks(p, 3, order="quarter")
    assert [n for _, n in ch] == [8] * 4 and [f - ch[0][0] for f, _ in ch] == [0, 1024, 2048, 3072]
    # a scan whose quarter does not split into 8-view chunks reads 32 consecutive views
    assert bench.step_chunks(F.config("c5"), 2, order="quarter") == [(64, 32)]
    assert bench.step_chunks(p, 3, order="sequential") == [(96, 32)]


def test_read_order_follows_the_pairing(monkeypatch):
    import fdk_b200 as F

    monkeypatch.delenv("FDK_BP_SYM", raising=False)
    assert bench.pairs_views(F.config("c3"), "fp32") and not bench.pairs_views(F.config("c3"), "mixed")
    monkeypatch.setenv("FDK_BP_SYM", "1")
    assert bench.pairs_views(F.config("c3"), "mixed") and not bench.pairs_views(F.config("c5"), "mixed")


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


def test_metric_and_l2_note_follow_the_workload():
    import fdk_b200 as F

    c3, c1 = F.config("c3"), F.config("c1")
    assert bench.metric_name(c3, "mixed") == bench.METRIC
    assert bench.metric_name(c1, "mixed").startswith("FDK GUPS at 256^3 x 256 views")
    assert "fp32 precision" in bench.metric_name(c3, "fp32")
    assert bench.l2_note(c3, "mixed").startswith("inputs larger than L2")
    c1.nz = 64  # 16 MiB of volume state: smaller than L2
    assert bench.l2_note(c1, "fp32").startswith("inputs smaller than L2")


def test_band_launches_from_the_launch_count():
    # the driver's 20-step C3 run: 2 filter kernels per step, a 512- and a 128-view batch, each
    # two conversion launches and 16 bands
    assert bench.band_launches(20 * 2 + 2 * (2 + 16), 20, 2, 2, "mixed") == 16
    # FP32 filters with one FFT launch per step and converts nothing
    assert bench.band_launches(20 + 2 * 16, 20, 1, 2, "fp32") == 16
    assert bench.conversion_launches("fp32_exact") == 0
