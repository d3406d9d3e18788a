"""bench.py's roofline accounting on the CPU: the algorithmic bytes per time
step are the fused minimum 84 N + 48 (S_x + S_y + S_z) in 3D and
52 N + 32 (S_x + S_z) in 2D, whose worked values at the benchmark workloads
are 902.4 MB (3D 200^3, 20-cell CPML) and 9.344 MB (2D 400^2)."""
import bench


def test_algorithmic_bytes_worked_values():
    assert bench.algorithmic_bytes({"shape": (200, 200, 200)}) == 902_400_000
    assert bench.algorithmic_bytes({"shape": (400, 400)}) == 9_344_000
    # 3D 400 x 400 x 200: 84 * 32e6 + 48 * 2 * 20 * (400*200 + 400*200 + 400*400)
    assert bench.algorithmic_bytes({"shape": (400, 400, 200)}) == 84 * 32_000_000 + 48 * 40 * 320_000
