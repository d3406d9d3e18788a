"""bench.py's host-side accounting on the CPU: the algorithmic bytes per time
step are the fused minimum 84 N + 48 (S_x + S_y + S_z) in 3D and
52 N + 32 (S_x + S_z) in 2D, whose worked values at the benchmark workloads
are 902.4 MB (3D 200^3, 20-cell CPML) and 9.344 MB (2D 400^2); the whole-job
value, the config dict both arms print, and the CPU baseline's sample."""
import bench


def test_algorithmic_bytes_worked_values():
    assert bench.algorithmic_bytes({"shape": (200, 200, 200)}) == 902_400_000
    assert bench.algorithmic_bytes({"shape": (400, 400)}) == 9_344_000
    # 3D 400 x 400 x 200: 84 * 32e6 + 48 * 2 * 20 * (400*200 + 400*200 + 400*400)
    assert bench.algorithmic_bytes({"shape": (400, 400, 200)}) == 84 * 32_000_000 + 48 * 40 * 320_000


def test_split_pml_algorithmic_bytes():
    """Split-field PML: 84 B per cell plus the 24 split fields read and
    written (8 B each) on every cell of the 20-cell shell."""
    n = 200
    shell = n ** 3 - (n - 40) ** 3
    assert bench.algorithmic_bytes({"shape": (n, n, n), "scheme": "SPML"}) == 84 * n ** 3 + 192 * shell


def test_whole_job_value_is_weak_scaling_aggregate():
    # 2 replicas of 8e6 cells x 1000 steps, 3 timed runs in 1.5 s
    assert bench.whole_job_value(2, 8_000_000, 1000, 3, 1500.0) == 2 * 8e6 * 1000 * 3 / 1.5 / 1e9
    assert bench.max_over_ranks(12.5, None) == 12.5


def test_both_arms_share_one_config_dict():
    from seiswave_taichi_b200 import synthetic as S
    cfg = S.config1(n=64, nt=10)
    a, b = bench.workload_config(cfg, 1), bench.workload_config(cfg, 1)
    assert a == b and a["grid"] == [64, 64] and a["time_steps"] == 10 and a["parallelism"] == "replicas1"
    assert bench.workload_config(cfg, 4)["parallelism"] == "replicas4"


def test_cpu_sample_text_names_the_sample():
    cfg = {"nt": 1000, "shape": (200, 200, 200)}
    assert bench.cpu_sample_text(cfg, 1000, 65.3).startswith("all 1000 of the 1000 time steps of the full 200x200x200")
    assert bench.cpu_sample_text(cfg, 625, 214.7).startswith("the first 625 of the 1000 time steps")


def test_cpu_segments_cover_the_run_and_respect_the_cap(monkeypatch):
    """The oracle runs the whole loop in consecutive segments when it fits the
    cap, else only its first steps; the segments tile the run from step 0."""
    from seiswave_taichi_b200 import synthetic as S
    cfg = S.config1(n=48, nt=12)
    segs, total = bench.cpu_segments(cfg, 4)
    assert total == 12 and [n for n, _ in segs] == [3, 3, 3, 3] and all(t >= 0 for _, t in segs)
    monkeypatch.setattr(bench, "CPU_FULL_RUN_MAX_UPDATES", 48 * 48 * 5)
    segs, total = bench.cpu_segments(cfg, 2)
    assert total == 5 and sum(n for n, _ in segs) == 5
