"""Generates the golden fixtures of tests/golden/ from independent references.

The reference project ships no golden vectors and cannot be built here, so
the fixtures pin the oracle's building blocks against independent
implementations of the same mathematics:

* fft_packed.npz   numpy.fft.rfft of seeded real lines, mapped to the
                   reference's packed layout (mod_fft.cc:79-86)
* eigen.npz        2(cos(2 pi i/n) - 1) in the reference's packed order
                   (mod_fft.cc:196-222), evaluated with numpy
* mesh.npz         the tanh / sin stretched dzf of mod_mesh.cc:95-125,
                   evaluated with numpy
* trid.npz         Neumann tridiagonal systems built from the reference's
                   coefficient formulas (mod_poisson_solver.cc:35-98) and
                   solved with scipy.linalg.solve_banded
* init_noise.npz   the project's noise generator (minstd 48271 mod 2^31-1,
                   jumped ahead by the cell index) evaluated with Python ints

Run: python tests/golden/make_golden.py   (writes next to this script)
"""
from __future__ import annotations

import os

import numpy as np
import scipy.linalg

HERE = os.path.dirname(os.path.abspath(__file__))
LENGTHS = [2, 4, 6, 8, 12, 16, 24, 48, 64, 96, 128, 192, 256, 384, 768]


def packed_rfft(x):
    n = x.size
    X = np.fft.rfft(x)
    out = np.zeros(n)
    out[0] = X[0].real
    out[1] = X[n // 2].real
    for m in range(1, n // 2):
        out[2 * m] = X[m].real
        out[2 * m + 1] = X[m].imag
    return out


def packed_eigen(n):
    aux = 2.0 * (np.cos(2.0 * np.pi * np.arange(n) / n) - 1.0)
    lam = np.empty(n)
    lam[0] = aux[0]
    lam[1] = aux[n // 2]
    for i in range(2, n):
        lam[i] = aux[i // 2]
    return lam


def mesh_dzf(nz, lz, ratio, func):
    z0 = np.arange(1, nz + 1) / nz
    if func == 0:
        zf = 0.5 * (1.0 + np.tanh((z0 - 0.5) * ratio) / np.tanh(ratio / 2.0))
    else:
        zf = 0.5 * (1.0 + np.sin((z0 - 0.5) * ratio * np.pi) / np.sin(ratio * np.pi / 2.0))
    zf = np.concatenate([[0.0], zf])
    d = np.empty(nz + 2)
    d[1:nz + 1] = lz * np.diff(zf)
    d[0] = d[1]
    d[nz + 1] = d[nz]
    return d


def trid_coeffs(dzf):
    nz = dzf.size - 2
    k = np.arange(nz)
    a = 2.0 / (dzf[k + 1] * (dzf[k] + dzf[k + 1]))
    c = 2.0 / (dzf[k + 1] * (dzf[k + 2] + dzf[k + 1]))
    b = -a - c
    b[0] += a[0]
    a[0] = 0.0
    b[nz - 1] += c[nz - 1]
    c[nz - 1] = 0.0
    return a, b, c


def noise(seed, offset):
    m, a = 2147483647, 48271
    x = seed % m or 1
    x = (x * pow(a, offset + 1, m)) % m
    return (x - 1) / (m - 1)


def main():
    rng = np.random.default_rng(20241203)
    lines = {}
    for n in LENGTHS:
        x = rng.standard_normal(n)
        lines[f"x{n}"] = x
        lines[f"X{n}"] = packed_rfft(x)
    np.savez_compressed(os.path.join(HERE, "fft_packed.npz"), **lines)

    np.savez_compressed(os.path.join(HERE, "eigen.npz"),
                        **{f"n{n}": packed_eigen(n) for n in LENGTHS if n >= 2})

    meshes = {}
    for nz, ratio, func in [(64, 1.5, 0), (128, 3.0, 0), (256, 1.8, 0), (48, 1.2, 1)]:
        meshes[f"nz{nz}_r{ratio}_f{func}"] = mesh_dzf(nz, 2.0, ratio, func)
    np.savez_compressed(os.path.join(HERE, "mesh.npz"), **meshes)

    tri = {}
    dzf = meshes["nz64_r1.5_f0"]
    a, b0, c = trid_coeffs(dzf)
    for lam in [-1.0, -37.5, -4000.0]:
        b = b0 + lam
        rhs = rng.standard_normal(64)
        ab = np.zeros((3, 64))
        ab[0, 1:] = c[:-1]
        ab[1, :] = b
        ab[2, :-1] = a[1:]
        sol = scipy.linalg.solve_banded((1, 1), ab, rhs)
        tri[f"lam{lam}_rhs"] = rhs
        tri[f"lam{lam}_sol"] = sol
    tri["dzf"] = dzf
    np.savez_compressed(os.path.join(HERE, "trid.npz"), **tri)

    offs = np.array([0, 1, 2, 1000, 524287, 75497471], dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "init_noise.npz"), offsets=offs,
                        **{f"seed{s}": np.array([noise(s, int(o)) for o in offs])
                           for s in (123, 456, 789)})


if __name__ == "__main__":
    main()
