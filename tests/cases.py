"""Initial states of the test cases, generated on the host with numpy.

Parity tests feed the same array to the CUDA solver (fvb_set_state) and to
the oracle, so both start from identical bits; test_cases.py checks the
device initial-state kernels against these formulas.
"""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & M64
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M64
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M64
    return x ^ (x >> np.uint64(31))


def unit_draw(seed: int, k: np.ndarray) -> np.ndarray:
    """k-th uniform [0,1) draw of stream `seed` (same as the device kernel)."""
    with np.errstate(over="ignore"):
        base = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15)) & M64
        x = splitmix64((base + np.asarray(k, dtype=np.uint64)) & M64)
    return (x >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def centers(n: int, x0: float, y0: float, length: float):
    h = length / n
    i = np.arange(n)
    x = x0 + (i + 0.5) * h
    return np.meshgrid(x, y0 + (i + 0.5) * h, indexing="xy")  # X[j, i], Y[j, i]


def vortex(n: int, x0=-5.0, y0=-5.0, length=10.0, beta=5.0, u0=1.0, v0=1.0, gamma=1.4, xc=None, yc=None):
    """Isentropic vortex with mean flow (rt_dg_euler_2d.cu:1334-1356 shifted):
    primitives (4, n, n) at cell centres."""
    xc = x0 + 0.5 * length if xc is None else xc
    yc = y0 + 0.5 * length if yc is None else yc
    X, Y = centers(n, x0, y0, length)
    dx, dy = X - xc, Y - yc
    r2 = dx * dx + dy * dy
    f = beta / (2 * np.pi) * np.exp(0.5 * (1 - r2))
    T = 1 - (gamma - 1) * beta * beta / (8 * gamma * np.pi ** 2) * np.exp(1 - r2)
    T = np.maximum(T, 1e-6)
    rho = T ** (1 / (gamma - 1))
    p = T ** (gamma / (gamma - 1))
    return np.stack([rho, u0 - f * dy, v0 + f * dx, p])


def kh(n: int, seed: int = 12345, noise: float = 1e-3, x0=0.0, y0=0.0, length=1.0):
    """Kelvin-Helmholtz double shear layer: rho 2 / u -0.5 for |y-0.5|<0.25,
    rho 1 / u +0.5 outside, p 2.5, v = 0.01 sin(4 pi x) + noise U[-1,1]."""
    X, Y = centers(n, x0, y0, length)
    inside = np.abs(Y - (y0 + 0.5 * length)) < 0.25 * length
    k = np.arange(n * n, dtype=np.uint64).reshape(n, n)
    v = 0.01 * np.sin(4 * np.pi * (X - x0) / length) + noise * (2 * unit_draw(seed, k) - 1)
    return np.stack([np.where(inside, 2.0, 1.0), np.where(inside, -0.5, 0.5), v, np.full((n, n), 2.5)])


def riemann4(n: int, seed: int, x0=0.0, y0=0.0, length=1.0, width: float = 2.0):
    """Four-quadrant Riemann problem; quadrant q = (x >= xm) + 2 (y >= ym)
    takes draws 4q..4q+3 of stream `seed` for rho, u, v, p.  The interfaces
    are tanh-smoothed over `width` cells (0 = sharp jumps), blending the four
    quadrant states bilinearly."""
    X, Y = centers(n, x0, y0, length)
    h = length / n
    xm, ym = x0 + 0.5 * length, y0 + 0.5 * length
    if width > 0:
        wx = 0.5 * (1 + np.tanh((X - xm) / (width * h)))
        wy = 0.5 * (1 + np.tanh((Y - ym) / (width * h)))
    else:
        wx = (X >= xm).astype(float)
        wy = (Y >= ym).astype(float)
    wq = [(1 - wx) * (1 - wy), wx * (1 - wy), (1 - wx) * wy, wx * wy]
    out = np.zeros((4, n, n))
    lo_hi = [(0.1, 1.9), (-1.0, 2.0), (-1.0, 2.0), (0.1, 1.9)]
    for q in range(4):
        for m, (a, b) in enumerate(lo_hi):
            out[m] += wq[q] * (a + b * unit_draw(seed, 4 * q + m))
    return out


def sod(n: int, length=1.0):
    """Circular Sod of fv_up7_ducros_2d.cu:629-637 evaluated in FP64."""
    X, Y = centers(n, 0.0, 0.0, length)
    h = length / n
    r = np.sqrt((X - 0.5 * length) ** 2 + (Y - 0.5 * length) ** 2)
    phi = 0.5 * (1 + np.tanh((0.25 * length - r) / h))
    z = np.zeros_like(r)
    return np.stack([0.125 + 10.875 * phi, z, z, 0.1 + 9.9 * phi])


def pad(interior: np.ndarray, g: int) -> np.ndarray:
    n = interior.shape[-1]
    Q = np.zeros((4, n + 2 * g, n + 2 * g), interior.dtype)
    Q[:, g:g + n, g:g + n] = interior
    return Q


def prim_to_cons(w: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    r, u, v, p = w
    return np.stack([r, r * u, r * v, p / (gamma - 1) + 0.5 * r * (u * u + v * v)])


def cons_to_prim(c: np.ndarray, gamma: float = 1.4) -> np.ndarray:
    r, m, n_, E = c
    u, v = m / r, n_ / r
    return np.stack([r, u, v, (gamma - 1) * (E - 0.5 * r * (u * u + v * v))])


def rel_linf(a: np.ndarray, b: np.ndarray) -> float:
    """max over variables of max|a-b| / max|b|."""
    out = 0.0
    for q in range(a.shape[0]):
        s = np.max(np.abs(b[q]))
        out = max(out, float(np.max(np.abs(a[q] - b[q])) / (s if s > 0 else 1.0)))
    return out


def smooth(n: int, seed: int, x0=0.0, y0=0.0, length=1.0):
    """Smooth periodic random state (sums of a few Fourier modes): a
    well-conditioned input for tolerance checks at any resolution."""
    rng = np.random.default_rng(seed)
    X, Y = centers(n, x0, y0, length)
    kx = 2 * np.pi / length

    def field(base, amp):
        f = np.full((n, n), base)
        for _ in range(3):
            a, b = rng.integers(1, 4, 2)
            ph = rng.uniform(0, 2 * np.pi)
            f = f + amp * rng.uniform(0.3, 1.0) * np.sin(a * kx * (X - x0) + b * kx * (Y - y0) + ph)
        return f

    return np.stack([field(1.0, 0.2), field(0.0, 0.5), field(0.0, 0.5), field(1.0, 0.2)])
