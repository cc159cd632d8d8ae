"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py).

CPU: the oracle and the product's host set-up still reproduce them.
GPU: the sm_100a path reproduces them without running the oracle.
"""
import math
import os

import numpy as np
import pytest

from cases import rel

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name)))


def test_oracle_reproduces_green_and_matvec(orc):
    g = load("green_matvec_5x4x3.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    G = orc.greencalculfft(nx, ny, nz, float(g["d"]), float(g["k0"]))
    assert rel(G, g["G"]) < 1e-14
    assert rel(orc.matvec(G, nx, ny, nz, g["x"], g["b"]), g["y"]) < 1e-14


def test_oracle_reproduces_sphere_solves(orc):
    from ifdda import objects
    s = load("sphere8_solves.npz")
    k0 = float(s["k0"])
    ob = objects.sphere(100e-9, 2.25 + 0j, 8, k0, "RR", na=-1)
    assert np.array_equal(ob.tabdip, s["tabdip"]) and rel(ob.alpha, s["alpha"]) < 1e-15
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    assert len(s["methods"]) == 14
    for meth in s["methods"]:
        meth = str(meth)
        r = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, s["ff0"], meth, 1e-4, tabdip=ob.tabdip)
        assert [r["nloop"], r["ncompte"]] == list(s[meth + "_counts"])
        assert rel(r["FFloc"], s[meth + "_FFloc"]) < 1e-12


def test_known_answers(orc):
    k = load("known_answers.npz")
    x, st, nl = orc.gpbicg_dense(np.diag([1j * (q + 1) for q in range(5)]), np.full(5, 1j), np.zeros(5), 1e-3)
    assert st == int(k["kat_status"]) == 1 and nl == int(k["kat_nloop"])
    assert np.allclose(x, k["kat_x"], rtol=1e-14)
    assert np.allclose(orc.mie(2.25, 100e-9, 632.8e-9), k["mie_c1"], rtol=1e-14)
    assert np.array_equal(orc.sunif_sequence(29, 64), k["sunif29"])


@pytest.mark.gpu
def test_gpu_reproduces_golden(gctx):
    from ifdda import objects
    g = load("green_matvec_5x4x3.npz")
    nx, ny, nz = (int(v) for v in g["dims"])
    gs = gctx.green(nx, ny, nz, float(g["d"]), float(g["k0"]))
    G = gs.export()
    for c in range(6):
        assert np.abs(G[c] - g["G"][c]).max() <= 1e-11 * np.abs(g["G"][c]).max()
    assert rel(gs.matvec(g["x"], g["b"]), g["y"]) < 1e-11
    gs.close()
    s = load("sphere8_solves.npz")
    k0 = float(s["k0"])
    ob = objects.sphere(100e-9, 2.25 + 0j, 8, k0, "RR", na=-1)
    gs = gctx.green(8, 8, 8, ob.aretecube, k0)
    for meth in s["methods"]:
        meth = str(meth)
        r = gs.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, s["ff0"], meth, 1e-4, tabdip=ob.tabdip)
        assert r.nstop == 0
        assert [int(r.nloop[0]), int(r.ncompte[0])] == list(s[meth + "_counts"])
        assert rel(r.FFloc, s[meth + "_FFloc"]) < 1e-7
        assert rel(r.FF, s[meth + "_FF"]) < 1e-7
    r = gs.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, s["ff0"], "GPBICG1", 1e-4, tabdip=ob.tabdip)
    em = gctx.local_macro(ob.nbsphere, ob.nmax, ob.epsilon, r.FFloc, ob.aretecube, k0)
    assert rel(em, s["macro"]) < 1e-7
    ce, ca = gctx.cross_sections(s["ff0"], r.FF, r.FFloc, k0, float(s["E0"]) ** 2)
    assert abs(ce - s["cext_cabs"][0]) <= 1e-7 * abs(s["cext_cabs"][0])
    gs.close()
