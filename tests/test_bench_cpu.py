"""The bench's roofline arithmetic on CPU: per-phase CUDA-event times and the
tree statistics of the 250k / 1M-point matvec give each phase's achieved rate
against its peak, for every branch the dominant phase can take."""
import pytest

import bench

STATS = {"pairs_up": 476_380_160, "pairs_down": 35_120_308_320, "pairs_leaf": 1_093_206_582,
         "pairs_p2p": 592_857_390, "surface_points": 152, "m2l_rank": 256, "m2l_pairs": 1_426_620,
         "m2l_tile_rows": 1_500_000, "c2e_columns": 28_000}
PHASES = {"gather": (0.015, 1), "up_pairs": (0.61, 5), "up_c2e": (0.62, 7), "down_pairs": (2.08, 7),
          "down_c2e": (0.66, 8), "leaf_pairs": (1.19, 3), "scatter": (0.008, 1), "m2l": (2.52, 3)}
PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def test_m2l_dominant_phase():
    r = bench.roofline(PHASES, STATS, "mixed", PEAKS, "tensor")
    assert r["bound"] == "tensor" and "m2l_ws_kernel" in r["kernel"]
    flops = 2 * 2.0 * 256 * 256 * STATS["m2l_pairs"]
    assert r["achieved"] == pytest.approx(flops / 2.52e-3 / 1e12)
    assert r["peak"] == pytest.approx(795.0) and r["frac"] == pytest.approx(r["achieved"] / 795.0)
    assert r["launches_per_step"] == 3 and r["hbm_measured_gbs"] == 6650.0
    assert r["traffic"] == pytest.approx(bench.M2L_TRAFFIC_250K) and r["traffic"] > 1e9
    p = r["pair_kernels"]
    # the V pairs run in the M2L phase, not in the down pairs
    npairs = STATS["pairs_up"] + STATS["pairs_down"] - STATS["m2l_pairs"] * 152 ** 2 + STATS["pairs_leaf"]
    assert p["ms_per_step"] == pytest.approx(0.61 + 2.08 + 1.19)
    assert p["achieved"] == pytest.approx(npairs * bench.FLOPS_PER_PAIR / (3.88e-3) / 1e12)
    assert p["peak"] == pytest.approx(bench.FP32_NOMINAL_TFLOPS) and 0 < p["frac"] < 1.5


def test_pair_dominant_phase_fp64():
    # M2L as pair segments of the down pass: no M2L phase, the V pairs count
    phases = dict(PHASES, down_pairs=(40.0, 7), m2l=(0.0, 0))
    r = bench.roofline(phases, STATS, "fp64", {}, "pairs")
    assert r["kernel"] == "p2p_kernel (down_pairs)" and r["bound"] == "fp64"
    assert r["achieved"] == pytest.approx(STATS["pairs_down"] * bench.FLOPS_PER_PAIR / 40e-3 / 1e12)
    assert r["peak"] == pytest.approx(bench.FP32_NOMINAL_TFLOPS / 2)
    assert r["pair_kernels"]["bound"] == "fp64" and "hbm_measured_gbs" not in r


def test_c2e_dominant_phase_and_uncompressed_m2l():
    r = bench.roofline(dict(PHASES, up_c2e=(9.0, 7)), STATS, "fp64", PEAKS, "fourier")
    assert r["kernel"] == "c2e_kernel (up_c2e)"
    assert r["achieved"] == pytest.approx(2.0 * 456 * 456 * STATS["c2e_columns"] / 9e-3 / 1e12)
    full = bench.roofline(PHASES, dict(STATS, m2l_rank=0), "mixed", PEAKS, "tensor")
    assert "m2l_img_kernel" in full["kernel"]
    assert full["achieved"] == pytest.approx(2.0 * 456 * 456 * STATS["m2l_pairs"] / 2.52e-3 / 1e12)


def test_fourier_m2l_dominant_phase_fp64():
    """FP64 matvec with its Fourier-space M2L as the longest phase: 9 complex
    multiply-adds (72 flops) per V pair and frequency (11^2 x 6 = 726 for
    p = 6: transform length 2 p - 1) against the nominal FP64 SIMT rate."""
    phases = dict(PHASES, m2l=(6.0, 3))
    r = bench.roofline(phases, STATS, "fp64", PEAKS, "fourier")
    assert "fft_accumulate_family_kernel (FP64" in r["kernel"] and r["bound"] == "fp64"
    assert r["achieved"] == pytest.approx(72.0 * 726 * STATS["m2l_pairs"] / 6e-3 / 1e12)
    assert r["peak"] == pytest.approx(bench.FP32_NOMINAL_TFLOPS / 2)
    assert r["ms_per_launch"] == pytest.approx(2.0)
    assert "l2" not in r  # no parent-grouped statistics, no L2 roofline


def test_fourier_m2l_l2_roofline():
    """The parent-grouped accumulation's L2 roofline: per launch one kernel
    spectrum (6 complex FP64 values a frequency) per (record, difference)
    group and 8 x 3 source spectra per record, over the launch time, against
    the measured L2 read rate."""
    stats = dict(STATS, m2l_family=1, m2l_groups=570_000, m2l_records=25_000, m2l_frequencies=726)
    r = bench.roofline(dict(PHASES, m2l=(6.0, 1)), stats, "fp64", PEAKS, "fourier", l2_gbs=12000.0)
    l2 = r["l2"]
    nbytes = (570_000 * 6 + 25_000 * 24) * 16 * 726
    assert l2["bytes_per_launch"] == nbytes and l2["unit"] == "GB/s" and l2["peak"] == 12000.0
    assert l2["achieved"] == pytest.approx(nbytes / 6e-3 / 1e9)
    assert l2["frac"] == pytest.approx(l2["achieved"] / 12000.0)
    # FP32 spectra: 8-byte complex values
    r32 = bench.roofline(dict(PHASES, m2l=(6.0, 1)), stats, "mixed", PEAKS, "fourier", l2_gbs=12000.0)
    assert r32["l2"]["bytes_per_launch"] == nbytes // 2


def test_reference_arm_does_not_load_the_library():
    """The reference arm reads the workload generator without importing the
    package (whose import maps libnnkifmm.so)."""
    import subprocess
    import sys
    code = ("import sys, bench; m = bench.workloads_module(); w = m.matvec_at_scale(200, 800); "
            "assert w['coarse'].shape == (200, 3); "
            "assert 'nnkifmm' not in sys.modules and 'nnkifmm._lib' not in sys.modules; "
            "maps = open('/proc/self/maps').read(); assert 'libnnkifmm' not in maps; print('ok')")
    out = subprocess.run([sys.executable, "-c", code], cwd=bench.ROOT, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and "ok" in out.stdout, out.stderr


def test_pair_kernels_of_the_250k_matvec():
    """The live phase split and statistics of the 250k / 1M-point mixed
    matvec: the pair phases reach 41% of the nominal FP32 rate (32 flops per
    pair), the M2L phase 19% of the TF32 rate."""
    r = bench.roofline(PHASES, STATS, "mixed", PEAKS, "tensor")
    assert r["pair_kernels"]["frac"] == pytest.approx(0.41, abs=0.01)
    assert r["frac"] == pytest.approx(0.186, abs=0.005)


class FakeNVML:
    """Read-only NVML stand-in: an SM clock and a reason mask that change
    once a few samples have been taken."""
    NVML_CLOCK_SM = 1
    nvmlClocksThrottleReasonSwPowerCap = 0x4

    def __init__(self):
        self.calls = 0
        self.shut = False

    def nvmlInit(self):
        pass

    def nvmlShutdown(self):
        self.shut = True

    def nvmlDeviceGetHandleByIndex(self, i):
        return ("gpu", i)

    def nvmlDeviceGetMaxClockInfo(self, h, kind):
        return 1965

    def nvmlDeviceGetClockInfo(self, h, kind):
        self.calls += 1
        return 1965 if self.calls < 4 else 1800

    def nvmlDeviceGetCurrentClocksEventReasons(self, h):
        return 0x1 if self.calls < 4 else 0x1 | 0x4  # idle, then power cap


def test_clock_sampler_on_a_fake_nvml(monkeypatch):
    import sys
    import time
    fake = FakeNVML()
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    c = bench.Clocks(0, period=0.002)
    c.start()
    time.sleep(0.05)
    out = c.stop()
    assert fake.shut and out["samples"] >= 5 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"] and out["source"].startswith("nvml")
    assert out["sm_mhz"] in (1800.0, 1965.0, (1800.0 + 1965.0) / 2)


def test_clock_sampler_without_nvml(monkeypatch):
    import sys
    monkeypatch.setitem(sys.modules, "pynvml", None)  # import fails
    monkeypatch.setattr(bench.subprocess, "Popen", lambda *a, **k: (_ for _ in ()).throw(OSError("no nvidia-smi")))
    c = bench.Clocks(0)
    c.start()
    assert c.stop()["reasons"] == ["nvidia-smi unavailable"]


def test_throughputs():
    t = bench.throughputs(2, 250_000, 1_000_000, STATS, 7.8)
    assert t["targets_per_s"] == pytest.approx(2 * 250_000 / 7.8e-3)
    assert t["sources_per_s"] == pytest.approx(2 * 1_000_000 / 7.8e-3)
    assert t["near_pairs_per_s"] == pytest.approx(2 * STATS["pairs_p2p"] / 7.8e-3)
