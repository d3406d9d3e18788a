"""Regenerate tests/golden/oracle_small.npz: small runs of the CPU oracle
(oracle/sw_oracle.cpp, the restatement of the reference's kernels) kept as
regression fixtures.  SeisWave_Taichi itself cannot run in this image
(Taichi is not installed), so these vectors pin the oracle and the GPU
kernels to one another over time, not to a run of the reference.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE.parents[1]))

from cases import case2d, case3d, oracle2d, oracle3d  # noqa: E402


def cases():
    """(name, case, scheme, steps); the same definitions drive the tests."""
    return [
        ("vs2d", case2d(shape=(48, 40), N=2, nt=60, npml=8, nrec=5, MT="explosive", src_scale=1e5), "VS", 60),
        ("sv2d", case2d(shape=(44, 50), N=3, nt=50, npml=8), "SV", 50),
        ("tensor3d", case3d(shape=(24, 22, 26), N=2, nt=40, npml=6), "TENSOR", 40),
        ("cpml3d", case3d(shape=(26, 24, 22), N=2, nt=40, npml=6, scheme="CPML"), "CPML", 40),
        ("spml3d", case3d(shape=(24, 26, 22), N=2, nt=40, npml=6, scheme="SPML"), "SPML", 40),
        ("rsg2d", case2d(shape=(46, 42), N=2, nt=60, npml=8), "RSG", 60),
    ]


def wavelet_of(c, scheme):
    from seiswave_taichi_b200 import BaseFun
    if scheme == "VS":
        return BaseFun.series("ricker2", c["nt"], c["dt"], c["freq"], c.get("src_scale", 1.0),
                              t0=np.float32(1.5 / float(c["freq"])))
    if scheme == "SV":
        return BaseFun.series("ricker", c["nt"], c["dt"], c["freq"], 1.0)
    if scheme == "TENSOR":
        return BaseFun.series("ricker2", c["nt"], c["dt"], c["freq"], c["src_scale"], t0=0.03)
    return BaseFun.series("ricker", c["nt"], c["dt"], c["freq"], c["src_scale"])


def rsg_sources(c):
    """update_RSG's caller-given source value of each step (a Ricker series)."""
    from seiswave_taichi_b200 import BaseFun
    return BaseFun.series("ricker", c["nt"], c["dt"], c["freq"], 1.0)


def run(name, c, scheme, steps):
    if scheme == "RSG":
        # update_RSG records no receiver (Elastic2D_CPML.py:277-353): keep vx and vz
        o = oracle2d(c).run("RSG", 0, steps, rsg_sources=rsg_sources(c).astype(np.float64))
        return {f"{name}_vx": np.asarray(o.vx), f"{name}_vz": np.asarray(o.vz)}
    if scheme in ("VS", "SV"):
        o = oracle2d(c, wavelet=wavelet_of(c, scheme)).run(scheme, 0, steps)
    else:
        o = oracle3d(c, wavelet=wavelet_of(c, scheme)).run(0, steps)
    return {f"{name}_data": np.asarray(o.data), f"{name}_vx": np.asarray(o.vx)}


def main():
    from seiswave_taichi_b200.pml import diff_coff
    out = {}
    for name, c, scheme, steps in cases():
        out.update(run(name, c, scheme, steps))
    for n in range(1, 9):
        out[f"diff_coff_{n}"] = np.asarray(diff_coff(n), np.float32)
    np.savez_compressed(HERE / "oracle_small.npz", **out)
    print("wrote", HERE / "oracle_small.npz", sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
