"""Synthetic inputs of the benchmark configurations (seeded), built with the
product's host set-up (ifdda.objects) so GPU tests and the bench share them.

C1  sphere eps 2.25, R = 100 nm, nnnr = 16 (d = 12.5 nm, 2176 dipoles inside),
    lambda 632.8 nm, normal incidence x-polarised (pp = 1), RR, GPBICG1,
    tol 1e-4, inside-only (inverserig / produitfftmatvect3), FFT grid 32^3.
C2  GRF cube 64^3, d = 10 nm, mean 2.25, std 0.1, lc = 50 nm, seed ng,
    theta 20 deg p-polarised, full box, FFT grid 128^3.
"""
import math

import numpy as np

from ifdda import objects

LAMBDA_C1 = 632.8e-9
P0 = 1.0


def c1(nnnr=16, methode="RR"):
    k0 = 2 * math.pi / LAMBDA_C1
    ob = objects.sphere(100e-9, 2.25 + 0j, nnnr, k0, methode, na=-1)
    E0, _ = objects.irradiance(P0, 10 * LAMBDA_C1)
    return ob, k0, E0


def c2(n=64, ng=7):
    k0 = 2 * math.pi / LAMBDA_C1
    ob = objects.inhomocuboid(n, n, n, 10e-9, 2.25 + 0j, 50e-9, 0.1, ng, k0, "RR")
    E0, _ = objects.irradiance(P0, 10 * LAMBDA_C1)
    return ob, k0, E0


def c3_disk(nrhs_pairs=64, seed=3, na=0.9, k0=1.0):
    """(kx, ky) uniform on the disk |k_par| <= na k0."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r = na * k0 * np.sqrt(rng.uniform(0, 1, nrhs_pairs))
    t = rng.uniform(0, 2 * np.pi, nrhs_pairs)
    return r * np.cos(t), r * np.sin(t)


def random_field(n3, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n3) + 1j * rng.standard_normal(n3)


def rel(a, b):
    # in FP64, whatever the inputs' precision (FP32 squares can overflow)
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
