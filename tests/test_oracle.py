"""CPU tests: the oracle pinned against independent answers, and the
product's host set-up checked against the oracle."""
import math

import numpy as np
import pytest

from cases import c1, rel, random_field


def test_fft_sign_and_normalisation(orc):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((6, 10, 12)) + 1j * rng.standard_normal((6, 10, 12))
    # sign +1 is numpy's unnormalised inverse transform, sign -1 its forward one
    assert rel(orc.fft3d(a, +1), np.fft.ifftn(a) * a.size) < 1e-14
    assert rel(orc.fft3d(a, -1), np.fft.fftn(a)) < 1e-14


@pytest.mark.parametrize("shape", [(7, 1, 1), (3, 5, 2), (16, 9, 25), (13, 11, 7)])
def test_fft_any_length(orc, shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert rel(orc.fft3d(a, +1), np.fft.ifftn(a) * a.size) < 1e-13


def test_propa_espace_libre_symmetry(orc):
    k0 = 2 * math.pi / 500e-9
    t = orc.propa_espace_libre((1e-8, -2e-8, 3e-8), (0, 0, 0), k0)
    assert np.allclose(t, t.T, rtol=0, atol=1e-12 * abs(t).max())
    t2 = orc.propa_espace_libre((-1e-8, 2e-8, -3e-8), (0, 0, 0), k0)
    assert np.allclose(t, t2)  # even in r
    assert np.all(orc.propa_espace_libre((0, 0, 0), (0, 0, 0), k0) == 0)


@pytest.mark.parametrize("dims,inside", [((4, 3, 2), False), ((5, 5, 5), False), ((6, 6, 6), True)])
def test_fft_matvec_equals_direct_sum(orc, dims, inside):
    """Pins the circulant embedding, wrap, zero planes and 1/ntotal scaling."""
    nx, ny, nz = dims
    k0 = 2 * math.pi / 600e-9
    d = 15e-9
    G = orc.greencalculfft(nx, ny, nz, d, k0)
    N = nx * ny * nz
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = (a.transpose(2, 1, 0).ravel() for a in (i, j, k))
    tab = np.arange(1, N + 1, dtype=np.int32)
    if inside:
        keep = ((i - 2.5) ** 2 + (j - 2.5) ** 2 + (k - 2.5) ** 2) < 7.0
        tab = np.zeros(N, np.int32)
        tab[keep] = np.arange(1, keep.sum() + 1)
        i, j, k = i[keep], j[keep], k[keep]
    nb = len(i)
    x = random_field(3 * nb, 5)
    b = random_field(3 * nb, 6)
    y = orc.matvec(G, nx, ny, nz, x, b, tabdip=tab if inside else None)
    yd = orc.matvec_direct(i * d, j * d, k * d, k0, x, b)
    assert rel(y, yd) < 1e-12


def test_green_parity_octant(orc):
    """Every FFTTENSOR component is even or odd along each axis, so the GPU
    keeps only q <= n per axis."""
    nx, ny, nz = 5, 4, 3
    G = orc.greencalculfft(nx, ny, nz, 10e-9, 2 * math.pi / 500e-9)
    par = {0: (1, 1, 1), 1: (-1, -1, 1), 2: (-1, 1, -1), 3: (1, 1, 1), 4: (1, -1, -1), 5: (1, 1, 1)}
    for c, (px, py, pz) in par.items():
        g = G[c]  # (Z, Y, X)
        m = np.roll(g[::-1, ::-1, ::-1], 1, axis=(0, 1, 2))  # q -> (L - q) mod L on every axis
        assert rel(m * (px * py * pz), g) < 1e-12
        mx = np.roll(g[:, :, ::-1], 1, axis=2)
        assert rel(mx * px, g) < 1e-12


def test_gpbicg_self_test_kat(orc):
    """The reference's own GPBICG self-test (cdmlib/gpbicg.f:1-79): diag(i*k) x = i."""
    n = 5
    mat = np.diag([1j * (q + 1) for q in range(n)])
    x, st, _ = orc.gpbicg_dense(mat, np.full(n, 1j), np.zeros(n), 1e-3)
    assert st == 1
    # GPBICG's own stop test: relative 2-norm residual <= tol (gpbicg.f:282-296)
    assert np.linalg.norm(mat @ x - np.full(n, 1j)) / np.linalg.norm(np.full(n, 1j)) <= 1e-3
    assert np.allclose(x, 1.0 / np.arange(1, n + 1), rtol=2e-3)


def test_mie_known_answer(orc):
    """Small-sphere limit: Cext -> Rayleigh absorption/scattering."""
    eps = 2.25 + 0.1j
    a = 5e-9
    lam = 600e-9
    ce, cs, ca = orc.mie(eps, a, lam)
    k = 2 * math.pi / lam
    al = 4 * math.pi * a ** 3 * (eps - 1) / (eps + 2)
    cabs_r = k * al.imag
    csca_r = k ** 4 / (6 * math.pi) * abs(al) ** 2
    # size parameter x = 0.05: corrections to the dipole limit are O(x^2)
    assert abs(ca - cabs_r) / cabs_r < 5e-3
    assert abs(cs - csca_r) / csca_r < 5e-3
    assert abs(ce - (ca + cs)) / ce < 1e-12


def test_c1_solution_and_mie(orc):
    ob, k0, E0 = c1()
    assert ob.nbsphere == 2176 and abs(ob.aretecube - 12.5e-9) < 1e-20
    G = orc.greencalculfft(16, 16, 16, ob.aretecube, k0)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    r = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4, tabdip=ob.tabdip)
    assert r["nstop"] == 0 and r["tol1"] < 1e-4
    assert r["ncompte"] == 2 * r["nloop"] + 2
    ce, ca = orc.cross_sections(ff0, r["FF"], r["FFloc"], k0, E0 ** 2)
    me, _, _ = orc.mie(2.25, 100e-9, 632.8e-9)
    assert abs(ce - me) / me < 0.06  # DDA discretisation error at 16 layers


@pytest.mark.parametrize("meth", ["QMRBICGSTAB1", "QMRBICGSTAB2"])
def test_qmr_agrees_with_gpbicg(orc, meth):
    ob, k0, E0 = c1(nnnr=8)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    a = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-10, tabdip=ob.tabdip)
    b = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-10, tabdip=ob.tabdip)
    assert b["nstop"] == 0 and b["ncompte"] == 2 * b["nloop"] + 2
    assert rel(b["FFloc"], a["FFloc"]) < 1e-8


@pytest.mark.parametrize("meth", ["BICGSTAB", "CG", "TFQMR", "GPBICGsafe", "GPBICG2", "GPBICGplus", "GPBICGAR",
                                  "BICGSTARPLUS", "CORS", "GPBICOR"])
def test_other_methods_agree_with_gpbicg(orc, meth):
    """The other Krylov methods restated (pimzbicgstab.f, zcg.f, tfqmr.f,
    gpbicgsafe.f, gpbicg2.f, gpbicgplus.f, gpbicgar.f): on the homogeneous
    sphere (A complex symmetric) they reach the GPBICG solution; their
    counters follow the reference drivers (BiCGSTAB and the GPBiCG family: 2 +
    2 nloop mat-vecs, CG and TFQMR: nloop + 2), and BiCGSTAB's tol1 is divided
    by the squared norm of the initial residual as in the reference."""
    ob, k0, E0 = c1(nnnr=8)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    a = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-10, tabdip=ob.tabdip)
    b = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-10, tabdip=ob.tabdip)
    assert b["nstop"] == 0, b["infostr"]
    if meth in ("CG", "TFQMR"):
        assert b["ncompte"] == b["nloop"] + 2 and b["tol1"] < 1e-9
        assert rel(b["FFloc"], a["FFloc"]) < 1e-8
    elif meth in ("GPBICGsafe", "GPBICG2", "GPBICGplus", "GPBICGAR", "BICGSTARPLUS", "CORS", "GPBICOR"):
        assert b["ncompte"] == 2 * b["nloop"] + 2 and b["tol1"] < 1e-10
        assert rel(b["FFloc"], a["FFloc"]) < 1e-8
    else:
        assert b["ncompte"] == 2 * b["nloop"] + 2
        assert rel(b["FFloc"], a["FFloc"]) < 1e-4  # stops at ||r||^2/||r0||^2 <= tol/10
        # tol1 = ||A E - FF0|| / ||r0||^2: with r0 = FF0 - A FF0 its scale is 1/|E|
        assert 0 < b["tol1"] < 1e-10


def _nonsymmetric_pola(ob, seed=11):
    pol = ob.polarisa.copy()
    rng = np.random.default_rng(seed)
    nb, nmax = ob.nbsphere, ob.nmax
    for a in range(3):
        for b in range(3):
            pol[np.arange(nb) + nmax * (a + 3 * b)] += 0.1 * ob.alpha * (rng.standard_normal(nb) +
                                                                       1j * rng.standard_normal(nb))
    return pol


def test_transpose_product_identity(orc):
    """The QMRCLA branch's A^T (inverserigopt.f:555-584) with a full
    non-symmetric polarisability: u^T (A v) = (A^T u)^T v without
    conjugation, and A^T u = u - alpha^T G u written out with numpy."""
    ob, k0, E0 = c1(nnnr=6)
    G = orc.greencalculfft(6, 6, 6, ob.aretecube, k0)
    pol = _nonsymmetric_pola(ob)
    nb, nmax = ob.nbsphere, ob.nmax
    rng = np.random.default_rng(3)
    u, v = (rng.standard_normal(3 * nb) + 1j * rng.standard_normal(3 * nb) for _ in range(2))

    def alpha(x, transpose):
        y = np.zeros_like(x)
        for a in range(3):
            for b in range(3):
                t = pol[np.arange(nb) + nmax * ((b + 3 * a) if transpose else (a + 3 * b))]
                y[a::3] += t * x[b::3]
        return y

    av = orc.matvec(G, 6, 6, 6, alpha(v, False), v, tabdip=ob.tabdip)
    atu = orc.apply_transpose(G, 6, 6, 6, nb, pol, nmax, u, ob.tabdip)
    assert abs(u @ av - atu @ v) <= 1e-12 * abs(u @ av)
    want = u + alpha(orc.matvec(G, 6, 6, 6, u, np.zeros_like(u), tabdip=ob.tabdip), True)
    assert rel(atu, want) < 1e-13


@pytest.mark.parametrize("aniso", [False, True])
def test_qmrcla_agrees_with_gpbicg(orc, aniso):
    """QMRCLA (qmrpim.f, PIMZQMR) reaches the GPBICG solution, with or
    without a non-symmetric tensor; its driver counts nloop = ITNO and
    2 ITNO + 3 mat-vecs (A x0, A^T r0, two a pass, and the final residual)."""
    ob, k0, E0 = c1(nnnr=8)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    pol = _nonsymmetric_pola(ob) if aniso else ob.polarisa
    a = orc.inverserig(G, 8, 8, 8, ob.nbsphere, pol, ob.nmax, ff0, "GPBICG1", 1e-10, tabdip=ob.tabdip)
    b = orc.inverserig(G, 8, 8, 8, ob.nbsphere, pol, ob.nmax, ff0, "QMRCLA", 1e-10, tabdip=ob.tabdip)
    assert b["nstop"] == 0, b["infostr"]
    assert b["ncompte"] == 2 * b["nloop"] + 3
    assert b["tol1"] < 1e-10
    assert rel(b["FFloc"], a["FFloc"]) < 1e-8


@pytest.mark.parametrize("name,works", [("CG", True), ("CGX", False), ("BICGSTAB", True), ("GPBICGAR2", True),
                                        ("TFQMR", True), ("BICGSTARPLUS", True), ("QMRCLA", True),
                                        ("QMRCLAX", True),
                                        ("GPBICGsafe", True), ("GPBICG2", True),
                                        ("CORS", True), ("CORSX", False), ("GPBICOR", True)])
def test_method_prefixes(orc, name, works):
    """methodeit is matched by prefix in the reference's order: 'GPBICGAR2'
    meets the 'GPBICGAR' test first (and runs GPBICGAR), 'CGX' is not 'CG'
    (blank padded)."""
    ob, k0, E0 = c1(nnnr=4)
    G = orc.greencalculfft(4, 4, 4, ob.aretecube, k0)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    r = orc.inverserig(G, 4, 4, 4, ob.nbsphere, ob.polarisa, ob.nmax, ff0, name, 1e-4, tabdip=ob.tabdip)
    if works:
        assert r["nstop"] == 0
    else:
        assert r["nstop"] == 1 and r["infostr"].strip() == "Iterative method not correct!"


def test_unknown_method_message(orc):
    ob, k0, E0 = c1(nnnr=4)
    G = orc.greencalculfft(4, 4, 4, ob.aretecube, k0)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    r = orc.inverserig(G, 4, 4, 4, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "NOSUCHMETHOD", 1e-4, tabdip=ob.tabdip)
    assert r["nstop"] == 1 and r["infostr"].strip() == "Iterative method not correct!"


def test_zero_rhs_breakdown(orc):
    ob, k0, _ = c1(nnnr=4)
    G = orc.greencalculfft(4, 4, 4, ob.aretecube, k0)
    r = orc.inverserig(G, 4, 4, 4, ob.nbsphere, ob.polarisa, ob.nmax, np.zeros(3 * ob.nbsphere), "GPBICG1", 1e-4,
                       tabdip=ob.tabdip)
    assert r["nstop"] == 1 and r["infostr"].strip() == "Problem to solve Ax=b!"


def test_local_macro_roundtrip(orc):
    ob, k0, E0 = c1(nnnr=6)
    loc = random_field(3 * ob.nbsphere, 2)
    em = orc.local_macro_all(ob.nbsphere, ob.nmax, ob.epsilon, loc, ob.aretecube, k0)
    # nsens = -1 recovers Eloc: Eloc = M Em / 3 with M = eps + 2 - i c (eps - 1)
    c = k0 ** 3 * ob.aretecube ** 3 / 2 / math.pi
    e = ob.eps.repeat(3)
    back = (e + 2 - 1j * c * (e - 1)) * em / 3
    assert rel(back, loc) < 1e-13


# ---- product host set-up vs oracle -------------------------------------
def test_objects_sphere_matches_oracle(orc):
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    for na in (-1, 0):
        a = objects.sphere(100e-9, 2.25, 10, k0, "RR", na=na)
        b = orc.object_sphere(100e-9, 2.25, 10, na, k0, "RR")
        assert a.nbsphere == b.nbsphere
        assert np.array_equal(a.tabdip, b.tabdip)
        assert np.array_equal(a.xs, b.xs) and np.array_equal(a.zs, b.zs)
        assert rel(a.polarisa, b.polarisa) < 1e-15
        assert rel(a.epsilon, b.epsilon) < 1e-15


@pytest.mark.parametrize("meth", ["CM", "RR", "GB", "LA", "LR"])
def test_poladiff_matches_oracle(orc, meth):
    from ifdda import objects
    k0 = 2 * math.pi / 500e-9
    for eps in (2.25, 3.0 + 0.01j, 12 + 1j):
        a = objects.poladiff(10e-9, eps, k0, meth)
        b = orc.poladiff(10e-9, eps, k0, meth)
        assert abs(a - b) <= 1e-14 * abs(b)


def test_sunif_matches_oracle(orc):
    from ifdda import objects
    assert np.array_equal(objects.sunif_sequence(29, 1000), orc.sunif_sequence(29, 1000))


def test_grf_cuboid_matches_oracle(orc):
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    a = objects.inhomocuboid(16, 12, 10, 10e-9, 2.25, 50e-9, 0.1, 3, k0, "RR")
    b = orc.object_inhomocuboid(16, 12, 10, 10e-9, 2.25, 50e-9, 0.1, 3, k0, "RR")
    assert rel(a.epsilon, b.epsilon) < 1e-14
    assert rel(a.polarisa, b.polarisa) < 1e-13


def test_grf_statistics():
    """mean eps 2.25 and std close to hc for the C2 configuration"""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.inhomocuboid(64, 64, 64, 10e-9, 2.25, 50e-9, 0.1, 7, k0, "RR")
    e = ob.eps.real
    assert abs(e.mean() - 2.25) < 0.02
    assert 0.03 < e.std() < 0.2


def test_concentric_matches_oracle(orc):
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    for na in (-1, 0):
        a = objects.concentric([0.9e-6, 1.9e-6], [3.0 + 0.01j, 2.0], 12, k0, "RR", na=na)
        b = orc.object_concentric([0.9e-6, 1.9e-6], [3.0 + 0.01j, 2.0], 12, na, k0, "RR")
        assert a.nbsphere == b.nbsphere and np.array_equal(a.tabdip, b.tabdip)
        assert rel(a.polarisa, b.polarisa) < 1e-15


def test_cube_matches_oracle(orc):
    from ifdda import objects
    k0 = 2 * math.pi / 500e-9
    a = objects.cube(200e-9, 2.0 + 0.3j, 8, k0, "CM")
    b = orc.object_cube(200e-9, 2.0 + 0.3j, 8, k0, "CM")
    assert np.array_equal(a.xs, b.xs) and rel(a.polarisa, b.polarisa) < 1e-15


def test_integrated_green_tensor_properties(orc):
    """propaesplibreintsim.f restated: zero at the origin, the plain tensor
    beyond lim wavelengths, symmetric, off-diagonal terms zero where the
    points share a coordinate, and close to the plain tensor a few cells
    away (the cube average of a smooth field)."""
    k0, d = 2 * math.pi / 600e-9, 10e-9
    assert np.all(orc.propaesplibreintsim(0, 0, 0, 0, 0, 0, k0, d) == 0)
    far = orc.propaesplibreintsim(0, 0, 0, 0, 0, 70 * d, k0, d)  # 700 nm > one wavelength
    assert np.array_equal(far, orc.propaesplibreintsim(0, 0, 0, 0, 0, 70 * d, k0, d, lim=0.0))
    t = orc.propaesplibreintsim(0, 0, 0, d, 2 * d, 0, k0, d)
    assert np.allclose(t, t.T, rtol=0, atol=1e-12 * np.abs(t).max())
    assert t[0, 2] == 0 and t[1, 2] == 0 and t[0, 1] != 0
    plain = orc.propaesplibreintsim(0, 0, 0, 4 * d, 3 * d, 2 * d, k0, d, lim=0.0)
    avg = orc.propaesplibreintsim(0, 0, 0, 4 * d, 3 * d, 2 * d, k0, d)
    assert rel(avg, plain) < 0.02


def test_quad_spectrum_without_quad_is_the_plain_one(orc):
    k0, d = 2 * math.pi / 550e-9, 11e-9
    a = orc.greencalculquadfft(4, 3, 2, 0, d, k0)
    b = orc.greencalculfft(4, 3, 2, d, k0)
    assert np.array_equal(a, b)
    c = orc.greencalculquadfft(4, 3, 2, 1, d, k0)
    assert not np.array_equal(c, b) and rel(c, b) < 0.5


# ---- anisotropic permittivity (polaepstens.f, trope = 'ani') -------------
EPSANI = np.array([[2.25, 0.1j, 0.0], [-0.1j, 2.5 + 0.02j, 0.05], [0.0, 0.05, 3.0]])


@pytest.mark.parametrize("meth", ["CM", "RR"])
def test_polaepstens_matches_oracle(orc, meth):
    from ifdda import objects
    k0 = 2 * math.pi / 500e-9
    for dis in (0, 1):
        a = objects.polaepstens(10e-9, EPSANI, k0, meth, dis=dis)
        b = orc.polaepstens(10e-9, EPSANI, k0, meth, dis=dis)
        assert rel(a, b) < 1e-14
        # inv = -1 returns the inverse tensor
        ai = orc.polaepstens(10e-9, EPSANI, k0, meth, dis=dis, inv=-1)
        assert rel(ai @ b, np.eye(3)) < 1e-12
        assert rel(objects.polaepstens(10e-9, EPSANI, k0, meth, dis=dis, inv=-1), ai) < 1e-13


@pytest.mark.parametrize("meth", ["CM", "RR"])
def test_polaepstens_of_a_scalar_is_poladiff(orc, meth):
    """eps * I gives poladiff's value on the diagonal and zeros elsewhere."""
    k0 = 2 * math.pi / 500e-9
    for eps in (2.25, 3.0 + 0.01j, 12 + 1j):
        t = orc.polaepstens(10e-9, eps * np.eye(3), k0, meth)
        p = orc.poladiff(10e-9, eps, k0, meth)
        assert np.allclose(t, p * np.eye(3), rtol=1e-13, atol=1e-13 * abs(p))


def test_polaepstens_rejects_other_methods(orc):
    from ifdda import objects
    k0 = 2 * math.pi / 500e-9
    for meth in ("LA", "GB", "PS"):
        with pytest.raises(ValueError):
            orc.polaepstens(10e-9, EPSANI, k0, meth)
        with pytest.raises(ValueError):
            objects.polaepstens(10e-9, EPSANI, k0, meth)


def test_anisotropic_objects_match_oracle(orc):
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    for na in (-1, 0):
        a = objects.sphere(100e-9, 0, 10, k0, "RR", na=na, epsani=EPSANI)
        b = orc.object_sphere(100e-9, 0, 10, na, k0, "RR", epsani=EPSANI)
        assert a.nbsphere == b.nbsphere and np.array_equal(a.tabdip, b.tabdip)
        assert np.array_equal(a.xs, b.xs) and np.array_equal(a.zs, b.zs)
        assert rel(a.polarisa, b.polarisa) < 1e-15
        assert rel(a.epsilon, b.epsilon) < 1e-15
    a = objects.cube(200e-9, 0, 8, k0, "CM", epsani=EPSANI)
    b = orc.object_cube(200e-9, 0, 8, k0, "CM", epsani=EPSANI)
    assert rel(a.polarisa, b.polarisa) < 1e-15 and rel(a.epsilon, b.epsilon) < 1e-15
    with pytest.raises(ValueError, match="anisotrope with PS"):
        objects.sphere(100e-9, 0, 10, k0, "PS", epsani=EPSANI)
    with pytest.raises(ValueError):
        orc.object_sphere(100e-9, 0, 10, -1, k0, "PS", epsani=EPSANI)


# ---- wide near field (cdmlib.f:1967-2492) ----------------------------------
def test_wide_near_field_reproduces_the_local_field(orc):
    """On the object's own sites the wide field E0 + G p is the solve's local
    field (the linear system itself), to the solve's residual; off the
    object it is the incident wave plus the scattered one, and the
    macroscopic field there equals the local one (eps = 1)."""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.sphere(100e-9, 2.25 + 0.1j, 6, k0, "RR", na=0)
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 0.3, 0, 30.0, 40.0)
    G = orc.greencalculfft(6, 6, 6, ob.aretecube, k0)
    ref = orc.inverserig(G, 6, 6, 6, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-11)
    assert ref["nstop"] == 0
    w = orc.nearfield_wide(6, 6, 6, 2, 3, 1, ob.aretecube, k0, 632.8e-9, 0, ob.nbsphere, ob.nmax, ob.xs, ob.ys,
                           ob.zs, ref["FF"], ff0, ob.epsilon, E0, 30.0, 40.0, 0.3)
    nxw, nyw, nzw = 10, 12, 8
    assert len(w["xswf"]) == nxw * nyw * nzw
    # object sites: offsets (2, 3, 1) in the enlarged box
    sites = [(k + 1) * nxw * nyw + (j + 3) * nxw + (i + 2) for k in range(6) for j in range(6) for i in range(6)]
    loc = w["local"].reshape(-1, 3)[sites].reshape(-1)
    assert rel(loc, ref["FFloc"]) < 1e-9
    assert np.allclose(w["xswf"][sites], ob.xs, rtol=0, atol=1e-15)
    em = orc.local_macro_all(ob.nbsphere, ob.nmax, ob.epsilon, ref["FFloc"], ob.aretecube, k0)
    assert rel(w["macro"].reshape(-1, 3)[sites].reshape(-1), em) < 1e-9
    off = np.setdiff1d(np.arange(nxw * nyw * nzw), sites)
    assert rel(w["macro"].reshape(-1, 3)[off], w["local"].reshape(-1, 3)[off]) < 1e-14
    inc = orc.incident(w["xswf"][off], w["yswf"][off], w["zswf"][off], k0, E0, 0.3, 0, 30.0, 40.0)
    assert np.array_equal(w["incident"].reshape(-1, 3)[off].reshape(-1), inc)


# ---- far field by direct summation (cdmlib.f:2784-2880) --------------------
def test_farfield_csca_matches_mie_and_optical_theorem(orc):
    """Config 1 sphere: the integrated Cscai is Mie's scattering cross
    section within the DDA error, equals Cext - Cabs of the same solve (the
    optical theorem, to the quadrature error), and g lies in (0, 1)."""
    ob, k0, E0 = c1(16)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    G = orc.greencalculfft(16, 16, 16, ob.aretecube, k0)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-8, tabdip=ob.tabdip)
    ff = orc.farfield_csca(ob.xs, ob.ys, ob.zs, ref["FF"], k0, E0 ** 2, 0.0, 0.0, 36, 72)
    _, mie_sca, _ = orc.mie(2.25, 100e-9, 632.8e-9)
    assert abs(ff["Cscai"] - mie_sca) / mie_sca < 0.1
    ce, ca = orc.cross_sections(ff0, ref["FF"], ref["FFloc"], k0, E0 ** 2)
    assert abs(ff["Cscai"] - (ce - ca)) / (ce - ca) < 0.02
    assert 0.0 < ff["gasym"] < 1.0
    assert ff["thetafield"][-1] == 180.0 and ff["phifield"][71] == 355.0
    with pytest.raises(ValueError):
        orc.farfield_csca(ob.xs, ob.ys, ob.zs, ref["FF"], k0, E0 ** 2, 0.0, 0.0, 10, 72)


def test_farfield_fft_converges_to_the_direct_sum(orc):
    """The pupil-grid integration (computegcfft2d.f) approaches the direct
    summation's Cscai as nfft2d grows (its 1/kz edge makes small grids
    coarse); full box as cdmlib.f:630 requires."""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.sphere(100e-9, 2.25 + 0j, 8, k0, "RR", na=0)
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    sol = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-8)
    a = orc.farfield_csca(ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 0.0, 0.0, 36, 72)
    b = orc.farfield_fft(8, 8, 8, ob.aretecube, ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 0.0, 0.0, 1024, 36, 72)
    assert abs(b["Cscai"] - a["Cscai"]) / a["Cscai"] < 0.01
    assert abs(b["gasym"] - a["gasym"]) < 0.01
    with pytest.raises(ValueError, match="In FFT Poynting nfft2d too small"):
        orc.farfield_fft(8, 8, 8, ob.aretecube, ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 0.0, 0.0, 16, 36, 72)


def test_anisotropic_concentric_and_arbitrary(orc):
    """trope = 'ani' for the concentric spheres (one tensor per shell,
    objectsphereconcentric.f:128-146) and the arbitrary object (one tensor per
    dipole, objectarbitrary.f:130-151): the geometry of the isotropic builders,
    every dipole's tensors from the oracle's polaepstens."""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    shells = [EPSANI, EPSANI.T + 0.5 * np.eye(3)]
    for na in (-1, 0):
        a = objects.concentric([0.9e-6, 1.9e-6], [3.0, 2.0], 12, k0, "RR", na=na, epsanis=shells)
        iso = objects.concentric([0.9e-6, 1.9e-6], [3.0, 2.0], 12, k0, "RR", na=na)
        assert a.nbsphere == iso.nbsphere and np.array_equal(a.tabdip, iso.tabdip)
        pol = a.polarisa.reshape(3, 3, a.nmax)   # [b][a][n]
        eps = a.epsilon.reshape(3, 3, a.nmax)
        ref = [orc.polaepstens(a.aretecube, e, k0, "RR") for e in shells]
        isoe = iso.epsilon.reshape(3, 3, iso.nmax)[0, 0, : a.nbsphere]
        for n in range(a.nbsphere):
            e = isoe[n]
            if e == 1.0:  # vacuum site of the full box
                assert np.array_equal(pol[:, :, n], np.zeros((3, 3)))
                assert np.array_equal(eps[:, :, n], np.eye(3))
                continue
            s = 0 if e == 3.0 else 1
            assert np.allclose(pol[:, :, n].T, ref[s], rtol=1e-13, atol=1e-13 * abs(ref[s]).max())
            assert np.array_equal(eps[:, :, n].T, shells[s])
    rng = np.random.default_rng(5)
    nx = ny = nz = 4
    N = nx * ny * nz
    t = rng.uniform(1.5, 3.0, (N, 3, 3)) + 0.01j * rng.uniform(0, 1, (N, 3, 3))
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    x, y, z = (v.transpose(2, 1, 0).reshape(-1) * 10e-9 for v in (i, j, k))
    ob = objects.arbitrary(nx, ny, nz, 10e-9, x, y, z, np.ones(N), k0, "CM", epsani_site=t)
    pol = ob.polarisa.reshape(3, 3, N)
    for n in range(N):
        r = orc.polaepstens(10e-9, t[n], k0, "CM")
        assert np.allclose(pol[:, :, n].T, r, rtol=1e-13, atol=1e-13 * abs(r).max())
