"""Seeded synthetic SDOT problems of the five benchmark shapes.

All problems live on the unit square: proj_domain = sample_domain =
[0, 1]^2, so the reference's area_scalar is 1 and its mass normalisation
(ot_op.cuh:154, 199-206) makes both the target density and the site masses
sum to 1.  Pixel (ix, iy) covers [ix/W, (ix+1)/W] x [iy/H, (iy+1)/H] and is
stored at picture[ix + iy*W], the reference's ``grid = i_x + i_y*size[0]``
(basic_function.cuh:805).  Sites are indexed i = a + G_x*b on the jittered
G_x x G_y grid.  The random stream is numpy PCG64 seeded with
1000*config + instance; draws happen in a fixed order (jitter, then the
mixture parameters) so the same seed gives the same problem everywhere.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

UNIT_DOMAIN = np.array([0.0, 1.0, 0.0, 1.0])


@dataclass
class SDOTProblem:
    """One instance: sites, masses and a normalised density image."""

    name: str
    xy: np.ndarray          # (N, 2) float64 site coordinates
    nu: np.ndarray          # (N,) float64 target masses, sum 1
    picture: np.ndarray     # (W*H,) float64 density per pixel, sum 1
    size: tuple             # (W, H): pixels along x, along y
    proj_domain: np.ndarray = None
    grid: tuple = None      # (G_x, G_y) of the site lattice

    def __post_init__(self):
        if self.proj_domain is None:
            self.proj_domain = UNIT_DOMAIN.copy()

    @property
    def n(self) -> int:
        return int(self.xy.shape[0])


def rng_for(config: int, instance: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(1000 * config + instance))


def jittered_grid(rng, gx: int, gy: int, jitter: float = 0.25):
    """Site (a, b) at ((a+0.5+u)/gx, (b+0.5+v)/gy), u, v ~ U[-jitter, jitter]."""
    j = rng.uniform(-jitter, jitter, size=(gy, gx, 2))
    a = np.arange(gx)[None, :]
    b = np.arange(gy)[:, None]
    x = (a + 0.5 + j[..., 0]) / gx
    y = (b + 0.5 + j[..., 1]) / gy
    return np.stack([x.ravel(), y.ravel()], axis=1)


def gaussian_mixture(rng, k: int, w: int, h: int, floor: float = 1e-3):
    """Anisotropic Gaussian mixture at pixel centres + floor, sum 1."""
    ctr = rng.uniform(0.1, 0.9, size=(k, 2))
    sig = rng.uniform(0.02, 0.15, size=(k, 2))
    th = rng.uniform(0.0, np.pi, size=k)
    amp = rng.uniform(0.2, 1.0, size=k)
    px = (np.arange(w) + 0.5) / w
    py = (np.arange(h) + 0.5) / h
    X, Y = np.meshgrid(px, py)          # Y rows -> iy, X cols -> ix
    img = np.zeros((h, w))
    for c in range(k):
        dx = X - ctr[c, 0]
        dy = Y - ctr[c, 1]
        ct, st = np.cos(th[c]), np.sin(th[c])
        u = ct * dx + st * dy
        v = -st * dx + ct * dy
        img += amp[c] * np.exp(-0.5 * ((u / sig[c, 0]) ** 2 + (v / sig[c, 1]) ** 2))
    img += floor
    img /= img.sum()
    return img.ravel()                  # index ix + iy*w


def beam_masses(gx: int, gy: int, sigma: float = 0.35):
    """nu_i proportional to exp(-|c_i - (0.5,0.5)|^2 / (2 sigma^2)) at the
    unjittered lattice positions, normalised to 1."""
    a = (np.arange(gx)[None, :] + 0.5) / gx
    b = (np.arange(gy)[:, None] + 0.5) / gy
    m = np.exp(-((a - 0.5) ** 2 + (b - 0.5) ** 2) / (2 * sigma * sigma)).ravel()
    return m / m.sum()


def make(config: int, instance: int = 0, *, g: int = None, res: int = None, k: int = None,
         beam: bool = None) -> SDOTProblem:
    """Problem of benchmark shape ``config`` (1..5); keyword overrides shrink
    it for tests while keeping the same generator.

    1: N=4096 (64^2), 256^2 image, K=8, uniform masses
    2: N=65536 (256^2), 1024^2 image, K=16, beam masses
    3: one of 64 instances, N log-uniform in [1024, 32768], 512^2, K in [4,16]
    4: N=16384 (128^2), 256^2, K in [2,16]
    5: N=262144 (512^2), 2048^2, K=24, beam masses
    """
    rng = rng_for(config, instance)
    if config == 1:
        gx = gy = g or 64
        r, kk, bm = res or 256, k or 8, False
    elif config == 2:
        gx = gy = g or 256
        r, kk, bm = res or 1024, k or 16, True
    elif config == 3:
        n = int(round(np.exp(rng.uniform(np.log(1024), np.log(32768)))))
        gx = gy = g or int(round(np.sqrt(n)))
        r = res or 512
        kk = k or int(rng.integers(4, 17))
        bm = False
    elif config == 4:
        gx = gy = g or 128
        r = res or 256
        kk = k or int(rng.integers(2, 17))
        bm = False
    elif config == 5:
        gx = gy = g or 512
        r, kk, bm = res or 2048, k or 24, True
    else:
        raise ValueError(f"unknown config {config}")
    if beam is not None:
        bm = beam
    xy = jittered_grid(rng, gx, gy)
    pic = gaussian_mixture(rng, kk, r, r)
    nu = beam_masses(gx, gy) if bm else np.full(gx * gy, 1.0 / (gx * gy))
    return SDOTProblem(f"config{config}/{instance}", xy, nu, pic, (r, r), UNIT_DOMAIN.copy(), (gx, gy))
