"""Deterministic noise tapes and synthetic SV paths for parity tests.

A tape for one tick holds ``normals[k, i]`` (the k-th normal draw of particle
i within the tick) and ``uniforms[k, i]``.  Values come from splitmix64 on an
integer counter (exact uint64 arithmetic, so identical on every machine) and a
Box-Muller transform in float64 rounded to float32.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = x.astype(np.uint64) + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def _counters(seed: int, stream: int, tick: int, slots: int, n: int) -> np.ndarray:
    k = np.arange(slots, dtype=np.uint64)[:, None]
    i = np.arange(n, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        base = np.uint64((seed * 1_000_003 + stream * 7_919 + tick) & 0xFFFFFFFFFFFF)
        return (base << np.uint64(32)) ^ (k << np.uint64(16)) ^ i


def _unit(z: np.ndarray) -> np.ndarray:
    """(0, 1] with 24 bits, exactly representable in float32."""
    return ((z >> np.uint64(40)).astype(np.float64) + 1.0) * (1.0 / 16777216.0)


def tape_normals(seed: int, tick: int, slots: int, n: int) -> np.ndarray:
    c = _counters(seed, 1, tick, slots, n)
    u1 = _unit(splitmix64(c))
    u2 = _unit(splitmix64(c ^ np.uint64(0x5555555555555555))) - (1.0 / 16777216.0)
    z = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    return z.astype(np.float32)


def tape_uniforms(seed: int, tick: int, slots: int, n: int) -> np.ndarray:
    c = _counters(seed, 2, tick, slots, n)
    return _unit(splitmix64(c)).astype(np.float32)


def tape(seed: int, tick: int, n: int, normal_slots: int, uniform_slots: int = 2):
    return tape_normals(seed, tick, normal_slots, n), tape_uniforms(seed, tick, uniform_slots, n)


def init_normals(seed: int, n: int, slots: int = 1) -> np.ndarray:
    """Initial draws: [n] for one slot, else [slots, n] (slot 0 is the same
    either way; a two-factor initialisation draws slots 0, 1 and 2)."""
    z = tape_normals(seed, 10_000_000, slots, n)
    return z[0] if slots == 1 else z


def sv_path(T: int, mu: float, rho: float, sigma_z: float, seed: int):
    """Synthetic 1-factor SV path h_t = mu + rho (h_{t-1} - mu) + sigma_z eps,
    h_0 ~ stationary, y_t = exp(h_t / 2) eta_t with Gaussian eta."""
    c = np.arange(3 * T + 3, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40)
    u = _unit(splitmix64(c))
    u2 = _unit(splitmix64(c ^ np.uint64(0x3333333333333333))) - (1.0 / 16777216.0)
    g = np.sqrt(-2.0 * np.log(u)) * np.cos(2.0 * np.pi * u2)
    h = np.empty(T)
    y = np.empty(T)
    hv = mu + sigma_z / np.sqrt(1.0 - rho * rho) * g[0]
    for t in range(T):
        hv = mu + rho * (hv - mu) + sigma_z * g[1 + 3 * t]
        eta = g[2 + 3 * t]
        h[t] = hv
        y[t] = np.exp(hv / 2.0) * eta
    return h, y.astype(np.float32)


def sv2_path(T: int, mu: float, rho_fast: float, sigma_fast: float, rho_slow: float, sigma_slow: float,
             seed: int, nu_obs: float = 0.0):
    """Synthetic two-factor SV path h_t = mu + f_t + s_t with AR(1) factors
    f_t = rho_f f_{t-1} + sigma_f eps, s_t = rho_s s_{t-1} + sigma_s eps', both
    started from their stationary laws; y_t = exp(h_t / 2) eta_t with Gaussian
    eta, or Student-t eta when nu_obs > 0 (chi-square from nu_obs squared
    normals, nu_obs rounded)."""
    k = int(round(nu_obs)) if nu_obs > 0 else 0
    per = 3 + k
    c = np.arange(per * T + 2, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40) + np.uint64(1 << 39)
    u = _unit(splitmix64(c))
    u2 = _unit(splitmix64(c ^ np.uint64(0x3333333333333333))) - (1.0 / 16777216.0)
    g = np.sqrt(-2.0 * np.log(u)) * np.cos(2.0 * np.pi * u2)
    f = sigma_fast / np.sqrt(1.0 - rho_fast * rho_fast) * g[0]
    s = sigma_slow / np.sqrt(1.0 - rho_slow * rho_slow) * g[1]
    h = np.empty(T)
    y = np.empty(T)
    for t in range(T):
        b = 2 + per * t
        f = rho_fast * f + sigma_fast * g[b]
        s = rho_slow * s + sigma_slow * g[b + 1]
        eta = g[b + 2]
        if k:
            eta = eta / np.sqrt(np.sum(g[b + 3:b + 3 + k] ** 2) / k)
        h[t] = mu + f + s
        y[t] = np.exp(h[t] / 2.0) * eta
    return h, y.astype(np.float32)


SCENARIOS = ("regime", "spike", "jumps", "fat_tails", "crisis")


def scenario_path(name: str, T: int, seed: int):
    """The scenario sweep on the 1-factor SV model (base mu=-1, rho=0.97,
    sigma_z=0.15, Gaussian eta; counter-based draws as sv_path):
      regime    mu steps from -1 to +1 at T/2
      spike     +3 added to h at a seeded 1% of ticks (a shock the AR(1) carries on)
      jumps     compound Poisson in h: rate 0.01 per tick, N(0, 2^2) sizes
      fat_tails Student-t eta with nu = 5 (chi-square from 5 squared normals)
      crisis    sigma_z = 0.4, rho = 0.99
    Returns (h[T], y[T] float32, filter params (rho, sigma_z, mu), nu of the
    filter's likelihood)."""
    mu, rho, sz = -1.0, 0.97, 0.15
    if name == "crisis":
        rho, sz = 0.99, 0.4
    k = 5 if name == "fat_tails" else 0
    per = 5 + k
    c = np.arange(per * T + 2, dtype=np.uint64) + np.uint64(seed) * np.uint64(1 << 40) + np.uint64(3 << 38)
    u = _unit(splitmix64(c))
    u2 = _unit(splitmix64(c ^ np.uint64(0x3333333333333333))) - (1.0 / 16777216.0)
    g = np.sqrt(-2.0 * np.log(u)) * np.cos(2.0 * np.pi * u2)
    h = np.empty(T)
    y = np.empty(T)
    hv = mu + sz / np.sqrt(1.0 - rho * rho) * g[0]
    for t in range(T):
        b = 1 + per * t
        m = mu
        if name == "regime" and t >= T // 2:
            m = 1.0
        hv = m + rho * (hv - m) + sz * g[b]
        if name == "spike" and u[b + 2] < 0.01:
            hv += 3.0
        if name == "jumps" and u[b + 3] < 0.01:    # Poisson(0.01): two or more jumps per tick are ~5e-5
            hv += 2.0 * g[b + 4]
        eta = g[b + 1]
        if k:
            eta = eta / np.sqrt(np.sum(g[b + 5:b + 5 + k] ** 2) / k)
        h[t] = hv
        y[t] = np.exp(hv / 2.0) * eta
    nu = 5.0 if name == "fat_tails" else 30.0
    return h, y.astype(np.float32), (rho, sz, mu), nu
