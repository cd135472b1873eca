"""Seeded synthetic inputs for the plane-Couette benchmarks.

The reference quotes its benchmark on its own analytic initial field
(pcf_fluctuations_jax.py:77-97); the B200 benchmark workload is the seeded
divergence-free perturbation described for the Couette DNS configuration:

    u' = curl(psi_a e_z) + curl(psi_b e_y),
    psi(x, y, z) = (1 - x^2)^2 sum_k w_k [alpha_k cos(k.y') + beta_k sin(k.y')],
    w_k = exp(-|k|^2 / 16),  alpha, beta ~ N(0, 1)  (numpy PCG64, seeds 2 / 3),

over integer mode indices |k_y| <= Ny/3, |k_z| <= Nz/3 (y' = 2 pi y / L_y,
z' = 2 pi z / L_z), i.e. u0 = d_y psi_a - d_z psi_b, u1 = -d_x psi_a,
u2 = d_x psi_b, which vanishes with its wall-normal derivative at x = +-1 and
is divergence free.  The projected state is scaled to perturbation energy
``energy`` (the reference's integral convention, channelflow_kmm.py:1302-1308).
Generating the samples is host-side input preparation; projecting and scaling
them runs on the GPU through the solver's own ``state_from_physical`` and
``diagnostics``.
"""

from __future__ import annotations

import math

import numpy as np


def couette_perturbation_fields(N, domain, seeds=(2, 3)) -> tuple[np.ndarray, ...]:
    """Physical samples (u0, u1, u2), shape N, on the quadrature mesh."""
    Nx, Ny, Nz = (int(n) for n in N)
    (a, b), (y0, y1), (z0, z1) = domain
    Ly, Lz = y1 - y0, z1 - z0
    X = np.cos(np.pi + (2 * np.arange(Nx) + 1) * np.pi / (2 * Nx))
    x = a + (X + 1.0) * (b - a) / 2.0
    y = y0 + np.arange(Ny) * Ly / Ny
    z = z0 + np.arange(Nz) * Lz / Nz
    xs = 2.0 * (x - a) / (b - a) - 1.0  # reference coordinate in [-1, 1]
    dxs = 2.0 / (b - a)
    env = (1.0 - xs**2) ** 2
    denv = -4.0 * xs * (1.0 - xs**2) * dxs
    ky_max, kz_max = Ny // 3, Nz // 3
    kys = np.arange(-ky_max, ky_max + 1)
    kzs = np.arange(-kz_max, kz_max + 1)

    def psi_parts(seed):
        rng = np.random.Generator(np.random.PCG64(seed))
        alpha = rng.standard_normal((kys.size, kzs.size))
        beta = rng.standard_normal((kys.size, kzs.size))
        w = np.exp(-(kys[:, None] ** 2 + kzs[None, :] ** 2) / 16.0)
        yp = 2.0 * np.pi * y / Ly
        zp = 2.0 * np.pi * z / Lz
        phase = kys[:, None, None, None] * yp[None, None, :, None] + (
            kzs[None, :, None, None] * zp[None, None, None, :]
        )  # (ky, kz, Ny, Nz)
        c, s = np.cos(phase), np.sin(phase)
        A = (w * alpha)[:, :, None, None]
        B = (w * beta)[:, :, None, None]
        f = np.sum(A * c + B * s, axis=(0, 1))
        fy = np.sum((A * (-s) + B * c) * (2 * np.pi / Ly) * kys[:, None, None, None], axis=(0, 1))
        fz = np.sum((A * (-s) + B * c) * (2 * np.pi / Lz) * kzs[None, :, None, None], axis=(0, 1))
        return f, fy, fz

    fa, fa_y, _ = psi_parts(seeds[0])
    fb, _, fb_z = psi_parts(seeds[1])
    u0 = env[:, None, None] * (fa_y[None] - fb_z[None])
    u1 = -denv[:, None, None] * fa[None]
    u2 = denv[:, None, None] * fb[None]
    return u0, u1, u2


def scale_to_energy(fields, energy_now: float, target: float):
    """Scale physical fields linearly so the projected energy equals target."""
    s = math.sqrt(target / energy_now)
    return tuple(f * s for f in fields)


def helmholtz2d_forcing(N=(64, 64), seed=1) -> np.ndarray:
    """Seeded forcing of the 2-D Helmholtz case: orthogonal Chebyshev x
    Fourier coefficients (a + i b)/sqrt(2) (1 + j)^-2 (1 + |k|)^-2 with
    a, b ~ N(0, 1) (numpy PCG64), made Hermitian in k (a real f), Nyquist
    mode zero."""
    Nx, Ny = N
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.standard_normal((Nx, Ny))
    b = rng.standard_normal((Nx, Ny))
    j = np.arange(Nx)[:, None]
    k = np.fft.fftfreq(Ny, 1.0 / Ny)[None, :]
    c = (a + 1j * b) / np.sqrt(2.0) * (1.0 + j) ** -2 * (1.0 + np.abs(k)) ** -2
    c[:, Ny // 2] = 0.0
    kk = (-np.arange(Ny)) % Ny
    return 0.5 * (c + np.conj(c[:, kk]))
