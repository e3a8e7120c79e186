"""Per-element material fields in the solver's input format.

The solver reads two raw little-endian float64 files, ``<prefix>_k.bin`` and
``<prefix>_rhoc.bin``, each holding ``N**3`` values in element order
``e = ix*N*N + iy*N + iz`` (x slowest), plus an optional ``<prefix>_meta.json``
(scripts/gen_field.py:5-6, 106-113 of the reference).  This module writes the
same files for the four material models of the reference generator, so the
solver (and the reference's validation scripts) can be fed without the
reference tree:

* ``homogeneous``  -- constant k and rho*c (scripts/gen_field.py:88-89).
* ``quadrants``    -- the MNHack7 four-region material sampled at element
                      centres (scripts/gen_field.py:29-37).
* ``lognormal``    -- ``k = exp(mu + sigma*G)`` with ``G`` a standardised
                      Gaussian random field of covariance ``exp(-r^2/L^2)``
                      on the periodic unit cube, synthesised by FFT filtering
                      of seeded white noise (scripts/gen_field.py:39-51, 96-106).
* ``layered``      -- x-slabs alternating between two conductivities
                      (scripts/gen_field.py:92-95).

The lognormal synthesis has to draw the same NumPy ``default_rng`` stream and
apply the same spectral filter in the same operation order as the reference
generator: the recorded fields of the reference's tests are only reproducible
bit for bit that way (the reference's ln32 seed-7 field has
``kmin = 0.02095277986074454``, ``kmax = 22.153757807186913``).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

__all__ = ["FieldSpec", "make_field", "write_field", "read_field", "generate"]


@dataclass
class FieldSpec:
    """Parameters of one material field (names follow the generator's flags)."""

    n: int
    model: str = "homogeneous"
    k: float = 1.0
    k2: float = 100.0
    period: int = 4
    rhoc: float = 1.0
    mu: float = 0.0
    sigma: float = 1.0
    rhoc_sigma: float = 0.0
    L: float = 0.125
    upscale: int = 1
    seed: int = 1
    extra: dict = field(default_factory=dict)


def _standard_gaussian_field(n: int, corr_len: float, seed: int) -> np.ndarray:
    """Unit-variance periodic Gaussian field with covariance exp(-r^2/L^2).

    The power spectrum of ``exp(-r^2/L^2)`` is proportional to
    ``exp(-|k|^2 L^2 / 4)``; filtering white noise by its square root in
    Fourier space and standardising gives the field.
    """
    noise = np.random.default_rng(seed).standard_normal((n, n, n))
    wave = 2 * np.pi * np.fft.fftfreq(n, d=1.0 / n)
    kx, ky, kz = np.meshgrid(wave, wave, wave, indexing="ij")
    k_sq = kx**2 + ky**2 + kz**2
    spectrum = np.exp(-k_sq * corr_len**2 / 4.0)
    g = np.fft.ifftn(np.fft.fftn(noise) * np.sqrt(spectrum)).real
    g -= g.mean()
    g /= g.std()
    return g


def _block_mean(fine: np.ndarray, r: int, harmonic: bool) -> np.ndarray:
    """Average r^3 blocks: harmonic (k, series bound) or arithmetic (rho*c)."""
    n = fine.shape[0] // r
    blocks = fine.reshape(n, r, n, r, n, r).transpose(0, 2, 4, 1, 3, 5).reshape(n, n, n, -1)
    if harmonic:
        return 1.0 / (1.0 / blocks).mean(-1)
    return blocks.mean(-1)


def _quadrant_material(n: int):
    h = 1.0 / n
    centre = (np.arange(n) + 0.5) * h
    X, Y, Z = np.meshgrid(centre, centre, centre, indexing="ij")
    k = np.full(X.shape, 400.0)
    rhoc = np.full(X.shape, 0.5 * 2.5)
    low_z = Z < 0.5
    region = (X < 0.5) & (Y < 0.5) & low_z
    k[region] = 100.0
    rhoc[region] = 1.0 * 1.0
    region = (X >= 0.5) & (Y < 0.5) & low_z
    k[region] = 200.0
    rhoc[region] = 0.8 * 1.5
    region = (X < 0.5) & (Y >= 0.5) & low_z
    k[region] = 300.0
    rhoc[region] = 0.6 * 2.0
    return k, rhoc


def make_field(spec: FieldSpec):
    """Return ``(k, rhoc, meta)`` with k, rhoc float64 arrays of shape (n, n, n)."""
    n = int(spec.n)
    meta = {
        "n": n, "model": spec.model, "k": spec.k, "k2": spec.k2, "period": spec.period,
        "rhoc": spec.rhoc, "mu": spec.mu, "sigma": spec.sigma, "rhoc_sigma": spec.rhoc_sigma,
        "L": spec.L, "upscale": spec.upscale, "seed": spec.seed,
    }
    meta.update(spec.extra)
    if spec.model == "homogeneous":
        k = np.full((n, n, n), spec.k)
        rhoc = np.full((n, n, n), spec.rhoc)
    elif spec.model == "quadrants":
        k, rhoc = _quadrant_material(n)
    elif spec.model == "layered":
        ix = np.arange(n)[:, None, None]
        k = np.where((ix // spec.period) % 2 == 0, spec.k, spec.k2) * np.ones((n, n, n))
        rhoc = np.full((n, n, n), spec.rhoc)
    elif spec.model == "lognormal":
        nf = n * spec.upscale
        g = _standard_gaussian_field(nf, spec.L, spec.seed)
        k_fine = np.exp(spec.mu + spec.sigma * g)
        rhoc_fine = np.exp(np.log(spec.rhoc) + spec.rhoc_sigma * g)
        if spec.upscale > 1:
            k = _block_mean(k_fine, spec.upscale, harmonic=True)
            rhoc = _block_mean(rhoc_fine, spec.upscale, harmonic=False)
            meta["upscale_rule"] = {"k": "harmonic", "rhoc": "arithmetic"}
        else:
            k, rhoc = k_fine, rhoc_fine
        meta["L_over_h"] = spec.L * n
    else:
        raise ValueError(f"unknown material model {spec.model!r}")
    k = np.ascontiguousarray(k, dtype=np.float64)
    rhoc = np.ascontiguousarray(rhoc, dtype=np.float64)
    meta.update(kmin=float(k.min()), kmax=float(k.max()), contrast=float(k.max() / k.min()),
                rhocmin=float(rhoc.min()), rhocmax=float(rhoc.max()), n_elements=int(n**3))
    return k, rhoc, meta


def write_field(prefix: str, k: np.ndarray, rhoc: np.ndarray, meta: Optional[dict] = None) -> None:
    """Write ``<prefix>_k.bin``, ``<prefix>_rhoc.bin`` (and ``_meta.json``)."""
    d = os.path.dirname(prefix)
    if d:
        os.makedirs(d, exist_ok=True)
    np.ascontiguousarray(k, dtype=np.float64).ravel(order="C").tofile(f"{prefix}_k.bin")
    np.ascontiguousarray(rhoc, dtype=np.float64).ravel(order="C").tofile(f"{prefix}_rhoc.bin")
    if meta is not None:
        m = dict(meta)
        m.setdefault("out", prefix)
        with open(f"{prefix}_meta.json", "w") as f:
            json.dump(m, f, indent=2)


def read_field(prefix: str, n: int):
    """Read a field pair written in the solver's input format."""
    k = np.fromfile(f"{prefix}_k.bin", dtype=np.float64)
    rhoc = np.fromfile(f"{prefix}_rhoc.bin", dtype=np.float64)
    if k.size < n**3 or rhoc.size < n**3:
        raise ValueError(f"field {prefix} holds fewer than {n**3} values")
    return k[: n**3].reshape(n, n, n), rhoc[: n**3].reshape(n, n, n)


def generate(prefix: str, n: int, model: str, **kw) -> dict:
    """Make and write one field; returns its meta dict."""
    spec = FieldSpec(n=n, model=model, **kw)
    k, rhoc, meta = make_field(spec)
    meta["out"] = prefix
    write_field(prefix, k, rhoc, meta)
    return meta


def _main(argv=None):
    import argparse

    p = argparse.ArgumentParser(description="Write a material field in the solver's input format.")
    p.add_argument("--n", type=int, required=True)
    p.add_argument("--model", choices=["homogeneous", "quadrants", "lognormal", "layered"], required=True)
    p.add_argument("--out", required=True)
    p.add_argument("--k", type=float, default=1.0)
    p.add_argument("--k2", type=float, default=100.0)
    p.add_argument("--period", type=int, default=4)
    p.add_argument("--rhoc", type=float, default=1.0)
    p.add_argument("--mu", type=float, default=0.0)
    p.add_argument("--sigma", type=float, default=1.0)
    p.add_argument("--rhoc-sigma", type=float, default=0.0)
    p.add_argument("--L", type=float, default=0.125)
    p.add_argument("--upscale", type=int, default=1)
    p.add_argument("--seed", type=int, default=1)
    a = p.parse_args(argv)
    meta = generate(a.out, a.n, a.model, k=a.k, k2=a.k2, period=a.period, rhoc=a.rhoc, mu=a.mu,
                    sigma=a.sigma, rhoc_sigma=a.rhoc_sigma, L=a.L, upscale=a.upscale, seed=a.seed)
    print(f"{a.model}: n={a.n}  k in [{meta['kmin']:.4g}, {meta['kmax']:.4g}] "
          f"(contrast {meta['contrast']:.3g})  rhoc in [{meta['rhocmin']:.4g}, {meta['rhocmax']:.4g}]"
          f"  -> {a.out}_{{k,rhoc}}.bin")


if __name__ == "__main__":
    _main()
