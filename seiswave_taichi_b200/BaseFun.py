"""Source wavelets of src/BaseFun.py, evaluated on the host in float32.

The reference evaluates these @ti.func's inside its kernels in float32
(default_fp) and returns ti.f32; here they are tabulated once per run, one value
per time step, in the same operation order.

* Ricker   (BaseFun.py:4-11)  -src_scale*2a*tau*exp(-a tau^2), t0 = 1.5/freq
  (the first derivative of a Gaussian, despite its name)
* Ricker2  (BaseFun.py:13-19) src_scale*(1-2a tau^2)*exp(-a tau^2), t0 given
* Ricker3  (BaseFun.py:21-27) Ricker wavelet shifted by 1.5/freq + t0
with a = pi^2 freq^2 and tau = nt*dt - t0.

Constant folding follows Taichi's frontend: `pi**2` is an expression of
Python values only, so Taichi evaluates it in Python (float64) and the result
enters the float32 arithmetic rounded once (f32(pi^2) = 9.869604, where
f32(pi)*f32(pi) would give 9.869605).  Integer powers of float32 values
(`freq**2`, `tau**2`) are single float32 products, as Taichi lowers them.
"""
from __future__ import annotations

import numpy as np

_f = np.float32
_PI = _f(np.pi)
_PI2 = _f(np.pi ** 2)  # pi**2 folded in float64, then rounded once (BaseFun.py:6,15)


def _steps(nt) -> np.ndarray:
    return np.asarray(nt, dtype=np.int64).astype(np.float32)


def Ricker(nt, dt, freq, src_scale):
    """BaseFun.py:4-11 for step index nt (scalar or array)."""
    freq, dt, s = _f(freq), _f(dt), _f(src_scale)
    t0 = _f(1.5) / freq
    a = _PI2 * (freq * freq)
    t = _steps(nt) * dt
    tau = t - t0
    with np.errstate(under="ignore"):
        return ((((-s) * _f(2)) * a) * tau) * np.exp((-a) * (tau * tau))


def Ricker2(nt, dt, t0, freq, src_scale):
    """BaseFun.py:13-19 for step index nt (scalar or array)."""
    freq, dt, t0, s = _f(freq), _f(dt), _f(t0), _f(src_scale)
    a = _PI2 * (freq * freq)
    t = _steps(nt) * dt
    tau = t - t0
    with np.errstate(under="ignore"):
        return (s * (_f(1) - (_f(2) * a) * (tau * tau))) * np.exp((-a) * (tau * tau))


def Ricker3(nt, dt, t0, freq, src_scale):
    """BaseFun.py:21-27 for step index nt (scalar or array)."""
    freq, dt, t0, s = _f(freq), _f(dt), _f(t0), _f(src_scale)
    ts = _f(1) / freq
    t = _steps(nt) * dt
    tau = _PI * ((t - _f(1.5) * ts) - t0) / ts
    with np.errstate(under="ignore"):
        return (s * (_f(1) - _f(2) * (tau * tau))) * np.exp(-(tau * tau))


def series(kind: str, nt: int, dt, freq, src_scale=1.0, t0=None) -> np.ndarray:
    """Tabulate a wavelet for steps 0..nt-1 (float32)."""
    steps = np.arange(int(nt))
    if kind == "ricker":
        return np.asarray(Ricker(steps, dt, freq, src_scale), dtype=np.float32)
    if kind == "ricker2":
        return np.asarray(Ricker2(steps, dt, t0, freq, src_scale), dtype=np.float32)
    if kind == "ricker3":
        return np.asarray(Ricker3(steps, dt, t0, freq, src_scale), dtype=np.float32)
    raise ValueError(f"unknown wavelet {kind!r}")
