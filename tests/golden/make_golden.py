"""Generates the golden fixtures of tests/golden/ with the CPU oracle.

The reference itself cannot be run here (no Fortran compiler), so these
vectors are the oracle's outputs on small seeded inputs; they freeze the
oracle (tests/test_golden.py checks it still reproduces them) and give the
GPU tests expected values that do not need the oracle at run time.

    python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "if-dda_b200"))

import oracle  # noqa: E402
from ifdda import objects  # noqa: E402


def green_and_matvec():
    nx, ny, nz = 5, 4, 3
    d, k0 = 13e-9, 2 * math.pi / 520e-9
    G = oracle.greencalculfft(nx, ny, nz, d, k0)
    rng = np.random.default_rng(2024)
    N = nx * ny * nz
    x = rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)
    b = rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)
    y = oracle.matvec(G, nx, ny, nz, x, b)
    np.savez_compressed(os.path.join(HERE, "green_matvec_5x4x3.npz"), dims=np.array([nx, ny, nz]), d=d, k0=k0,
                        G=G, x=x, b=b, y=y)


# every methodeit branch of the reference's driver (cdmlib/inverserigopt.f)
METHODS = ("GPBICG1", "QMRBICGSTAB1", "QMRBICGSTAB2", "GPBICG2", "GPBICGsafe", "GPBICGplus", "GPBICGAR",
           "BICGSTARPLUS", "TFQMR", "CG", "BICGSTAB", "GPBICOR", "CORS", "QMRCLA")


def sphere_solves():
    lam = 632.8e-9
    k0 = 2 * math.pi / lam
    ob = objects.sphere(100e-9, 2.25 + 0j, 8, k0, "RR", na=-1)
    E0, _ = objects.irradiance(1.0, 10 * lam)
    ff0 = oracle.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    G = oracle.greencalculfft(8, 8, 8, ob.aretecube, k0)
    out = dict(tabdip=ob.tabdip, alpha=ob.alpha, eps=ob.eps, xs=ob.xs, ys=ob.ys, zs=ob.zs, ff0=ff0, k0=k0,
               E0=E0, d=ob.aretecube, methods=np.array(METHODS))
    for meth in METHODS:
        r = oracle.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, tabdip=ob.tabdip)
        out[meth + "_FFloc"] = r["FFloc"]
        out[meth + "_FF"] = r["FF"]
        out[meth + "_counts"] = np.array([r["nloop"], r["ncompte"]])
        out[meth + "_tol1"] = r["tol1"]
    r = oracle.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4, tabdip=ob.tabdip)
    out["macro"] = oracle.local_macro_all(ob.nbsphere, ob.nmax, ob.epsilon, r["FFloc"], ob.aretecube, k0)
    out["cext_cabs"] = np.array(oracle.cross_sections(ff0, r["FF"], r["FFloc"], k0, E0 ** 2))
    np.savez_compressed(os.path.join(HERE, "sphere8_solves.npz"), **out)


def known_answers():
    n = 5
    mat = np.diag([1j * (q + 1) for q in range(n)])
    x, st, nl = oracle.gpbicg_dense(mat, np.full(n, 1j), np.zeros(n), 1e-3)
    mie = oracle.mie(2.25, 100e-9, 632.8e-9)
    np.savez_compressed(os.path.join(HERE, "known_answers.npz"), kat_x=x, kat_status=st, kat_nloop=nl,
                        mie_c1=np.array(mie), sunif29=oracle.sunif_sequence(29, 64))


if __name__ == "__main__":
    green_and_matvec()
    sphere_solves()
    known_answers()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
