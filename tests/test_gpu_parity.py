"""GPU parity of the sm_100a path against the FP64 oracle, through the C-ABI.

Tolerances: FP64 kernels agree with the oracle to 1e-11 relative (different
FFT factorisations round differently); FP32 mat-vecs to 2e-5; a converged
solve reproduces the oracle's iteration and mat-vec counts exactly and its
local field to 1e-7 relative (Krylov amplifies the 1e-15 FFT differences).
"""
import math

import numpy as np
import pytest

from cases import c1, rel, random_field

pytestmark = pytest.mark.gpu

SIZES = [(4, 3, 2), (5, 6, 3), (8, 8, 8), (12, 10, 8), (16, 16, 16), (24, 20, 12)]


@pytest.mark.parametrize("dims", SIZES)
def test_green_spectrum_matches_oracle(gctx, orc, dims):
    nx, ny, nz = dims
    d, k0 = 11e-9, 2 * math.pi / 550e-9
    g = gctx.green(nx, ny, nz, d, k0)
    got = g.export()
    ref = orc.greencalculfft(nx, ny, nz, d, k0)
    for c in range(6):
        assert np.abs(got[c] - ref[c]).max() <= 1e-11 * np.abs(ref[c]).max(), c
    g.close()


def test_green_recompute_matches_a_new_spectrum(gctx, orc):
    """ifdda_green_recompute (greencalculfft called again into the arrays the
    caller holds, cdmlib.f:1529-1531): the spectrum at a new spacing and
    wavelength matches the oracle's, and a solve after it (on workspaces and
    captured loops made for the old spectrum) equals a fresh handle's solve
    bit for bit."""
    ob, k0, E0, ff0, _ = _c1_inputs(orc, nnnr=10)
    g = gctx.green(10, 10, 10, ob.aretecube, k0)
    g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip)
    d2, k2 = 0.9 * ob.aretecube, 1.1 * k0
    g.recompute(d2, k2)
    ref = orc.greencalculfft(10, 10, 10, d2, k2)
    got = g.export()
    for c in range(6):
        assert np.abs(got[c] - ref[c]).max() <= 1e-11 * np.abs(ref[c]).max(), c
    for prec in (0, 1):
        r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip, precision=prec)
        fresh = gctx.green(10, 10, 10, d2, k2)
        f = fresh.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip,
                             precision=prec)
        fresh.close()
        assert r.nstop == f.nstop == 0
        assert np.array_equal(r.FFloc, f.FFloc) and int(r.ncompte[0]) == int(f.ncompte[0])
    g.close()


def test_tile_chooser_shapes_match_the_oracle(gctx, orc):
    """Every combination of the two tile shapes of zconv and of the y passes
    matches the oracle's mat-vec (they agree to rounding: the compiler may
    contract multiply-adds differently per shape), the chooser times both
    on first use and keeps one per grid, and the choice it reports is the
    one the next mat-vec uses."""
    from ifdda import IFDDA_FP32, IFDDA_FP64
    nx, ny, nz = 40, 32, 48  # FFT lengths 80, 64, 96: two shapes on every axis
    d, k0 = 10e-9, 2 * math.pi / 500e-9
    N = nx * ny * nz
    x, b = random_field(3 * N, 7), random_field(3 * N, 8)
    g = gctx.green(nx, ny, nz, d, k0)
    ref = orc.matvec(orc.greencalculfft(nx, ny, nz, d, k0), nx, ny, nz, x, b)
    for prec, tol in ((IFDDA_FP64, 1e-11), (IFDDA_FP32, 2e-5)):
        assert g.tiles(prec)[:2] == (-1, -1)
        outs = {}
        for zv, yv in ((0, 0), (1, 1), (0, 1), (1, 0)):
            g.set_tiles(prec, zv, yv)
            assert g.tiles(prec)[:2] == (zv, yv)
            outs[(zv, yv)] = g.matvec(x, b, precision=prec)
            assert rel(outs[(zv, yv)], ref) < tol
        g.set_tiles(prec, -1, -1)
        got = g.matvec(x, b, precision=prec)
        zv, yv, t = g.tiles(prec)
        assert zv in (0, 1) and yv in (0, 1) and min(t) > 0
        assert np.array_equal(got, outs[(zv, yv)])
    import ifdda
    with pytest.raises(ifdda.IfddaError):
        gctx.green(4, 4, 4, d, k0).set_tiles(IFDDA_FP64, 1, 0)  # length 8 has one shape
    g.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_batch_equals_single_bitwise_on_a_tiled_grid(gctx, orc, prec):
    """On a grid whose kernels have two tile shapes (lengths 96, 64, 80), a
    right-hand side solved alone and inside a batch of three gives the same
    bits: the shape is chosen per grid, not per batch size."""
    from ifdda import objects
    k0 = 2 * math.pi / 600e-9
    ob = objects.inhomocuboid(48, 32, 40, 10e-9, 2.25 + 0j, 40e-9, 0.1, 3, k0, "RR")
    E0, _ = objects.irradiance(1.0, 10 * 600e-9)
    ff0 = np.stack([orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, pp, 0, th, 0.0)
                    for th, pp in ((0.0, 1.0), (25.0, 0.0), (40.0, 1.0))])
    g = gctx.green(48, 32, 40, ob.aretecube, k0)
    batch = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-5, precision=prec)
    alone = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0[1], "GPBICG1", 1e-5, precision=prec)
    assert batch.nstop == alone.nstop == 0
    assert np.array_equal(alone.FFloc, batch.FFloc[1]) and int(alone.ncompte[0]) == int(batch.ncompte[1])
    g.close()


@pytest.mark.parametrize("dims", SIZES)
@pytest.mark.parametrize("inside", [False, True])
def test_matvec_fp64_matches_oracle(gctx, orc, dims, inside):
    nx, ny, nz = dims
    d, k0 = 9e-9, 2 * math.pi / 480e-9
    N = nx * ny * nz
    tab = None
    nb = N
    if inside:
        rng = np.random.default_rng(nx * 100 + ny)
        occ = rng.uniform(size=N) < 0.6
        tab = np.zeros(N, np.int32)
        tab[occ] = np.arange(1, occ.sum() + 1)
        nb = int(occ.sum())
    x = random_field(3 * nb, 1)
    b = random_field(3 * nb, 2)
    g = gctx.green(nx, ny, nz, d, k0)
    got = g.matvec(x, b, tabdip=tab)
    G = orc.greencalculfft(nx, ny, nz, d, k0)
    ref = orc.matvec(G, nx, ny, nz, x, b, tabdip=tab)
    assert rel(got, ref) < 1e-11
    from ifdda import IFDDA_FP32
    got32 = g.matvec(x, b, tabdip=tab, precision=IFDDA_FP32)
    assert rel(got32, ref) < 2e-5
    g.close()


def _c1_inputs(orc, nnnr=16):
    ob, k0, E0 = c1(nnnr)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    G = orc.greencalculfft(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
    return ob, k0, E0, ff0, G


@pytest.mark.parametrize("meth", ["GPBICG1", "QMRBICGSTAB1", "QMRBICGSTAB2"])
def test_c1_solve_fp64_matches_oracle(gctx, orc, meth):
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, tabdip=ob.tabdip)
    g = gctx.green(16, 16, 16, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, tabdip=ob.tabdip)
    assert r.nstop == ref["nstop"] == 0
    assert int(r.nloop[0]) == ref["nloop"]
    assert int(r.ncompte[0]) == ref["ncompte"]
    assert abs(r.tol1[0] - ref["tol1"]) <= 1e-6 * ref["tol1"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    assert rel(r.FF, ref["FF"]) < 1e-7
    g.close()


@pytest.mark.parametrize("meth", ["GPBICG1", "QMRBICGSTAB1"])
def test_full_box_solve_matches_oracle(gctx, orc, meth):
    """Sphere in its full box (na = 0, inverserigopt), vacuum sites alpha = 0."""
    from ifdda import objects
    k0 = 2 * math.pi / 500e-9
    ob = objects.sphere(120e-9, 3.0 + 0.2j, 12, k0, "RR", na=0)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, 1.0, 0.3, 0, 30.0, 40.0)
    G = orc.greencalculfft(12, 12, 12, ob.aretecube, k0)
    ref = orc.inverserig(G, 12, 12, 12, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-6)
    g = gctx.green(12, 12, 12, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-6)
    assert r.nstop == 0 and int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    g.close()


def _grf(orc, n):
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.inhomocuboid(n, n, n, 10e-9, 2.25 + 0j, 50e-9, 0.1, 7, k0, "RR")
    E0, _ = objects.irradiance(1.0, 10 * 632.8e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 20.0, 0.0)
    return ob, k0, ff0, orc.greencalculfft(n, n, n, ob.aretecube, k0)


@pytest.mark.parametrize("n,nlim", [(40, 0), (48, 10)])
def test_qmr_on_grf_cube_matches_oracle(gctx, orc, n, nlim):
    """Full-box GRF cube (the config-2 object at reduced size).  At 40^3 QMR
    converges; at 48^3 it stalls and is stopped at nlim iterations, where both
    paths report "Converge do not reach!" with the same iterate."""
    ob, k0, ff0, G = _grf(orc, n)
    for meth in ("QMRBICGSTAB1", "QMRBICGSTAB2"):
        ref = orc.inverserig(G, n, n, n, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, nlim=nlim)
        g = gctx.green(n, n, n, ob.aretecube, k0)
        r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, maxit=nlim)
        # the C-ABI adds cdmlib's own check tol1 >= tolinit (cdmlib.f:1586-1591)
        want = (1, "Converge do not reach!") if ref["tol1"] >= 1e-4 else (ref["nstop"], ref["infostr"].strip())
        assert (r.nstop, r.infostr.strip()) == want
        assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
        # each mat-vec agrees to 1e-11; a stalled recurrence stopped at nlim
        # amplifies that rounding (FMA contraction differs between builds), so
        # the unconverged iterate is held to 1e-6 and a converged one to 1e-7
        assert rel(r.FFloc, ref["FFloc"]) < (1e-7 if ref["tol1"] < 1e-4 else 1e-6)
        g.close()


def test_gpbicg_iteration_limit_matches_oracle(gctx, orc):
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-9, tabdip=ob.tabdip,
                         nlim=2)
    g = gctx.green(16, 16, 16, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-9, tabdip=ob.tabdip, maxit=2)
    assert ref["nstop"] == 0 and ref["tol1"] >= 1e-9  # inverserig itself does not test tol1
    assert r.nstop == 1 and r.infostr.strip() == "Converge do not reach!"
    assert int(r.nloop[0]) == ref["nloop"] == 4 and int(r.ncompte[0]) == ref["ncompte"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-9
    g.close()


@pytest.mark.parametrize("meth", ["GPBICG1", "QMRBICGSTAB1", "QMRBICGSTAB2", "GPBICG2", "GPBICGsafe", "GPBICGplus",
                                  "GPBICGAR", "BICGSTARPLUS", "TFQMR", "CG", "BICGSTAB", "GPBICOR", "CORS",
                                  "QMRCLA"])
def test_iteration_limit_every_method_matches_oracle(gctx, orc, meth):
    """Each method stopped by an iteration limit of 3 at tol 1e-12 ends as
    its branch of the reference's driver does: the current iterate with the
    counters of the passes made (then cdmlib's "Converge do not reach!"), or
    STATUS = -1 and "Problem to solve Ax=b!" (CG, BiCGSTAB, QMRCLA)."""
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-12, tabdip=ob.tabdip,
                         nlim=3)
    g = gctx.green(16, 16, 16, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-12, tabdip=ob.tabdip, maxit=3)
    if ref["nstop"] == 0:
        assert ref["tol1"] >= 1e-12
        assert (r.nstop, r.infostr.strip()) == (1, "Converge do not reach!")
        assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
        assert rel(r.FFloc, ref["FFloc"]) < 1e-9
    else:
        assert (r.nstop, r.infostr.strip()) == (ref["nstop"], ref["infostr"].strip())
    g.close()


@pytest.mark.parametrize("meth", ["GPBICG1", "QMRBICGSTAB1", "QMRBICGSTAB2", "GPBICG2", "GPBICGsafe", "GPBICGplus",
                                  "GPBICGAR", "BICGSTARPLUS", "CG", "BICGSTAB", "GPBICOR", "CORS", "QMRCLA"])
def test_zero_rhs_every_method_matches_oracle(gctx, orc, meth):
    """FF0 = 0 makes every method break down at its first test (NORM = 0 or
    a zero inner product): nstop = 1, "Problem to solve Ax=b!", the same
    counters.  (TFQMR is left out: its stopping test divides by NORM and the
    reference's loop never ends.)"""
    ob, k0, E0, ff0, _ = _c1_inputs(orc, nnnr=8)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    zero = np.zeros(3 * ob.nbsphere, dtype=np.complex128)
    ref = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, zero, meth, 1e-4, tabdip=ob.tabdip)
    g = gctx.green(8, 8, 8, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, zero, meth, 1e-4, tabdip=ob.tabdip)
    assert (r.nstop, r.infostr.strip()) == (ref["nstop"], ref["infostr"].strip()) == (1, "Problem to solve Ax=b!")
    g.close()


@pytest.mark.parametrize("dims", [(7, 5, 3), (15, 9, 11), (256, 2, 3), (200, 3, 2), (300, 2, 2), (320, 3, 2),
                                  (2, 300, 2), (3, 2, 320), (2, 256, 3), (3, 2, 200), (2, 320, 3), (2, 3, 300)])
def test_padded_lattice_matvec_matches_oracle(gctx, orc, dims):
    """A lattice side n whose 2n is not a compiled FFT length (14, 30, 18, 22,
    400, 600 here) runs on the smallest larger compiled box, the lattice at its
    corner: the mat-vec of the caller's lattice, full box and through a
    Tabdip, matches the oracle's on the caller's own 2n grid.  The long side
    sits on x, on y and on z in turn, so the x passes, the y passes and the z
    convolution each run at the lengths 512 (256 and 200 -> 512) and 640
    (300 and 320 -> 640)."""
    nx, ny, nz = dims
    d, k0 = 10e-9, 2 * math.pi / 600e-9
    G = orc.greencalculfft(nx, ny, nz, d, k0)
    rng = np.random.default_rng(5)
    N = nx * ny * nz
    x = rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)
    b = rng.standard_normal(3 * N) + 1j * rng.standard_normal(3 * N)
    g = gctx.green(nx, ny, nz, d, k0)
    assert rel(g.matvec(x, b), orc.matvec(G, nx, ny, nz, x, b)) < 1e-11
    occ = rng.random(N) < 0.6
    tab = np.zeros(N, np.int32)
    tab[occ] = np.arange(1, occ.sum() + 1)
    nd = int(occ.sum())
    xt, bt = x[:3 * nd], b[:3 * nd]
    assert rel(g.matvec(xt, bt, tabdip=tab), orc.matvec(G, nx, ny, nz, xt, bt, tabdip=tab)) < 1e-11
    assert rel(g.matvec(x, b, precision=2), orc.matvec(G, nx, ny, nz, x, b)) < 2e-5
    compiled = {2, 4, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256, 320, 384, 512, 640}
    if any(2 * n not in compiled for n in dims):
        with pytest.raises(Exception, match="padded"):
            g.export()
    g.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_padded_lattice_solve_matches_oracle(gctx, orc, prec):
    """Solves on lattices whose 2n is not compiled: the 15^3 sphere through
    its Tabdip, the full-box 15^3 GRF cube and a 200 x 3 x 2 GRF rod."""
    ob, k0, E0, ff0, G = _c1_inputs(orc, nnnr=15)
    ref = orc.inverserig(G, 15, 15, 15, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip)
    g = gctx.green(15, 15, 15, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip, precision=prec)
    assert r.nstop == ref["nstop"] == 0, r.infostr
    if prec == 0:
        assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
        assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    else:
        assert r.tol1[0] < 1e-6 and rel(r.FFloc, ref["FFloc"]) < 1e-4
    g.close()
    from ifdda import objects
    # the GRF cube, and a 200 x 3 x 2 GRF rod (its 400 runs on 512)
    for dims, meth in (((15, 15, 15), "QMRBICGSTAB1"), ((200, 3, 2), "GPBICG1")):
        ob = objects.inhomocuboid(*dims, 10e-9, 2.25 + 0j, 50e-9, 0.1, 7, k0, "RR")
        E0, _ = objects.irradiance(1.0, 10 * 632.8e-9)
        ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 20.0, 0.0)
        G = orc.greencalculfft(*dims, ob.aretecube, k0)
        ref = orc.inverserig(G, *dims, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-6)
        g = gctx.green(*dims, ob.aretecube, k0)
        r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-6, precision=prec)
        assert r.nstop == ref["nstop"] == 0, r.infostr
        if prec == 0:
            assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
            assert rel(r.FFloc, ref["FFloc"]) < 1e-7
        else:
            assert r.tol1[0] < 1e-6 and rel(r.FFloc, ref["FFloc"]) < 1e-4
        g.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_zero_rhs_inside_a_batch(gctx, orc, prec):
    """A zero right-hand side inside a batch stops at once ("Problem to solve
    Ax=b!", the batch's nstop), and the others give what they give alone."""
    ob, k0, E0, _, _ = _c1_inputs(orc, nnnr=10)
    angles = [(0.0, 0.0, 1.0), (20.0, 10.0, 0.0), (35.0, 70.0, 1.0)]
    ff0 = np.stack([orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, pp, 0, t, p) for t, p, pp in angles])
    ff0[1] = 0
    g = gctx.green(10, 10, 10, ob.aretecube, k0)
    rb = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-5, tabdip=ob.tabdip, precision=prec)
    assert rb.nstop == 1 and rb.infostr.strip() == "Problem to solve Ax=b!"
    for q in (0, 2):
        rs = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0[q], "GPBICG1", 1e-5, tabdip=ob.tabdip,
                          precision=prec)
        assert rs.nstop == 0
        assert np.array_equal(rs.FFloc, rb.FFloc[q])
        assert rs.nloop[0] == rb.nloop[q] and rs.ncompte[0] == rb.ncompte[q]
    g.close()


@pytest.mark.parametrize("meth", ["GPBICG2", "GPBICGsafe", "GPBICGplus", "GPBICGAR", "BICGSTARPLUS", "TFQMR", "CG",
                                  "BICGSTAB", "QMRBICGSTAB2", "GPBICOR", "CORS"])
def test_anisotropic_every_method_matches_oracle(gctx, orc, meth):
    """The full-tensor mat-vec under each of the other methods (a
    non-symmetric 3x3 polarisability per dipole): same counters, local field
    within 1e-7."""
    ob, k0, E0, ff0, G = _c1_inputs(orc, nnnr=10)
    nb, nmax = ob.nbsphere, ob.nmax
    pol = ob.polarisa.copy()
    rng = np.random.default_rng(11)
    for a in range(3):
        for b in range(3):
            pol[np.arange(nb) + nmax * (a + 3 * b)] += 0.1 * ob.alpha * (rng.standard_normal(nb) +
                                                                       1j * rng.standard_normal(nb))
    ref = orc.inverserig(G, 10, 10, 10, nb, pol, nmax, ff0, meth, 1e-6, tabdip=ob.tabdip)
    assert ref["nstop"] == 0, ref["infostr"]
    g = gctx.green(10, 10, 10, ob.aretecube, k0)
    r = g.inverserig(nb, pol, nmax, ff0, meth, 1e-6, tabdip=ob.tabdip)
    assert r.nstop == 0, r.infostr
    assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    g.close()


def test_mixed_precision_meets_fp64_residual(gctx, orc):
    from ifdda import IFDDA_MIXED
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    tight = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-10,
                           tabdip=ob.tabdip)
    g = gctx.green(16, 16, 16, ob.aretecube, k0)
    for meth in ("GPBICG1", "QMRBICGSTAB1"):
        r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, tabdip=ob.tabdip, precision=IFDDA_MIXED)
        assert r.nstop == 0, r.infostr
        assert r.tol1[0] < 1e-4
        # local-field error of a 1e-4 solve against the converged FP64 field
        assert rel(r.FFloc, tight["FFloc"]) < 1e-3
    g.close()


@pytest.mark.parametrize("meth", ["GPBICG1", "GPBICG2", "GPBICGsafe", "GPBICGplus", "GPBICGAR", "BICGSTARPLUS",
                                  "TFQMR", "CG", "BICGSTAB", "QMRBICGSTAB1", "QMRBICGSTAB2", "GPBICOR", "CORS",
                                  "QMRCLA"])
def test_batch_equals_single_bitwise(gctx, orc, meth):
    """A right-hand side gives bit-identical results alone and inside a batch
    (fixed-order reductions, per-RHS scalars), whatever the method: the
    right-hand sides of a batch stop at different iterations."""
    ob, k0, E0, _, _ = _c1_inputs(orc, nnnr=10)
    angles = [(0.0, 0.0, 1.0), (20.0, 10.0, 0.0), (35.0, 70.0, 1.0), (10.0, 200.0, 0.5)]
    ff0 = np.stack([orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, pp, 0, t, p) for t, p, pp in angles])
    g = gctx.green(10, 10, 10, ob.aretecube, k0)
    for prec in (0, 1):
        rb = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-5, tabdip=ob.tabdip,
                          precision=prec)
        assert rb.nstop == 0, rb.infostr
        for q in range(len(angles)):
            rs = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0[q], meth, 1e-5, tabdip=ob.tabdip,
                              precision=prec)
            assert np.array_equal(rs.FFloc, rb.FFloc[q])
            assert rs.nloop[0] == rb.nloop[q] and rs.ncompte[0] == rb.ncompte[q]
    g.close()


def test_post_step_matches_oracle(gctx, orc):
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4, tabdip=ob.tabdip)
    em_ref = orc.local_macro_all(ob.nbsphere, ob.nmax, ob.epsilon, ref["FFloc"], ob.aretecube, k0)
    em = gctx.local_macro(ob.nbsphere, ob.nmax, ob.epsilon, ref["FFloc"], ob.aretecube, k0)
    assert rel(em, em_ref) < 1e-13
    ce_r, ca_r = orc.cross_sections(ff0, ref["FF"], ref["FFloc"], k0, E0 ** 2)
    ce, ca = gctx.cross_sections(ff0, ref["FF"], ref["FFloc"], k0, E0 ** 2)
    assert abs(ce - ce_r) <= 1e-12 * abs(ce_r)
    assert abs(ca - ca_r) <= 1e-9 * abs(ce_r)


def test_planewaves_match_oracle(gctx, orc):
    ob, k0, E0, _, _ = _c1_inputs(orc, nnnr=8)
    beams = [(0, 0.0, 0.0, 1.0), (0, 25.0, -40.0, 0.3), (1, 0.3 * k0, -0.4 * k0, 0.0), (1, 0.0, 0.0, 1.0),
             (1, 0.1 * k0, 0.7 * k0, 0.6)]
    got = gctx.planewaves(ob.xs, ob.ys, ob.zs, k0, E0, [b[0] for b in beams], [b[1] for b in beams],
                          [b[2] for b in beams], [b[3] for b in beams])
    for q, (bm, a1, a2, pp) in enumerate(beams):
        ref = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, pp, bm, a1, a2)
        assert rel(got[q], ref) < 1e-13


def test_error_paths(gctx, orc):
    ob, k0, E0, ff0, _ = _c1_inputs(orc, nnnr=6)
    g = gctx.green(6, 6, 6, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "NOSUCHMETHOD", 1e-4, tabdip=ob.tabdip)
    assert r.nstop == 1 and r.infostr.strip() == "Iterative method not correct!"
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, np.zeros_like(ff0), "GPBICG1", 1e-4, tabdip=ob.tabdip)
    assert r.nstop == 1 and r.infostr.strip() == "Problem to solve Ax=b!"
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1.0, tabdip=ob.tabdip)
    assert r.nstop == 1
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4, tabdip=ob.tabdip, nstop_in=-1)
    assert r.nstop == -1 and r.infostr.strip() == "Calculation cancelled during iterative method"
    # unsupported FFT length: 2*7 = 14 has no compiled kernel
    import ifdda
    # a side above 320 has no compiled FFT length to pad to (2 n <= 640)
    with pytest.raises(ifdda.IfddaError):
        gctx.green(321, 2, 2, 10e-9, k0)
    # a mat-vec precision other than FP32 / FP64 is an error, not a silent FP64
    x = np.zeros(3 * ob.nbsphere, np.complex128)
    for prec in (1, 3, -1):
        with pytest.raises(ifdda.IfddaError, match="precision"):
            g.matvec(x, x.copy(), tabdip=ob.tabdip, precision=prec)
    g.close()


def test_cdmlib_driver_config1_matches_oracle(orc):
    """Config 1 through the cdmlib-style entry (reference option names and
    units) against the oracle pipeline; Cext within the DDA error of Mie."""
    from ifdda.cdmlib import cdmlib
    out = cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25 + 0j, nnnr=16, tolinit=1e-4,
                 methodeit="GPBICG1", polarizability="RR", nproche=0, theta=0.0, phi=0.0, pp=1.0, P0=1.0,
                 w0=6328.0)
    assert out["nstop"] == 0 and out["nbsphere"] == 2176
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4, tabdip=ob.tabdip)
    assert rel(out["localfield"], ref["FFloc"]) < 1e-7
    em = orc.local_macro_all(ob.nbsphere, ob.nmax, ob.epsilon, ref["FFloc"], ob.aretecube, k0)
    assert rel(out["macroscopicfield"][0], em) < 1e-7
    ce, ca = orc.cross_sections(ff0, ref["FF"], ref["FFloc"], k0, E0 ** 2)
    assert abs(out["Cext"][0] - ce) <= 1e-7 * ce
    mie_ext, _, _ = orc.mie(2.25, 100e-9, 632.8e-9)
    assert abs(out["Cext"][0] - mie_ext) / mie_ext < 0.06


@pytest.mark.parametrize("nproche", [0, 1])
def test_cdmlib_anisotropic_sphere_matches_oracle(orc, nproche):
    """trope = 'ani' (polaepstens.f, objectsphere.f:128-135): every dipole
    carries the full 3x3 tensor; inside-only (nproche 0) and full box
    (nproche 1) against the oracle pipeline with the oracle's own object."""
    from ifdda.cdmlib import cdmlib
    ani = np.array([[2.25, 0.1j, 0.0], [-0.1j, 2.5 + 0.02j, 0.05], [0.0, 0.05, 3.0]])
    out = cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25, nnnr=16, tolinit=1e-6,
                 methodeit="GPBICG1", polarizability="RR", trope="ani", epsani=ani, nproche=nproche, theta=20.0,
                 phi=30.0, pp=0.5, P0=1.0, w0=6328.0)
    assert out["nstop"] == 0, out["infostr"]
    k0 = 2 * math.pi / 632.8e-9
    na = -1 if nproche == 0 else 0
    ob = orc.object_sphere(100e-9, 0, 16, na, k0, "RR", epsani=ani)
    assert out["nbsphere"] == ob.nbsphere
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 0.5, 0, 20.0, 30.0)
    G = orc.greencalculfft(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6,
                         tabdip=ob.tabdip if na == -1 else None)
    assert ref["nstop"] == 0
    assert rel(out["localfield"], ref["FFloc"]) < 1e-9
    assert rel(out["FF"], ref["FF"]) < 1e-9
    em = orc.local_macro_all(ob.nbsphere, ob.nmax, ob.epsilon, ref["FFloc"], ob.aretecube, k0)
    assert rel(out["macroscopicfield"][0], em) < 1e-9
    ce, ca = orc.cross_sections(ff0, ref["FF"], ref["FFloc"], k0, E0 ** 2)
    assert abs(out["Cext"][0] - ce) <= 1e-9 * abs(ce)
    assert abs(out["Cabs"][0] - ca) <= 1e-8 * abs(ce)


def test_context_closed_before_its_spectrum():
    """A context destroyed while a spectrum made on it is alive (finalisers
    run in any order) is released by the spectrum's own destroy; neither
    call may fail or touch freed memory."""
    import ifdda
    ctx = ifdda.Context(0)
    g = ctx.green(4, 4, 4, 10e-9, 1e7)
    h = g.h
    ctx.close()
    assert g.lib.ifdda_green_destroy(h) == 0
    g.h = None
    ctx2 = ifdda.Context(0)
    g2 = ctx2.green(4, 4, 4, 10e-9, 1e7)
    g2.close()
    ctx2.close()


@pytest.mark.parametrize("meth,prec", [("GPBICG1", 0), ("QMRBICGSTAB1", 0), ("GPBICG1", 1), ("QMRCLA", 0),
                                       ("QMRCLA", 1)])
def test_anisotropic_polarisability_matches_oracle(gctx, orc, meth, prec):
    """A full 3x3 polarisability per dipole (polarisa(n,a,b) with off-diagonal
    terms) takes the mat-vec's full-tensor path and the unfused GPBiCG steps;
    QMRCLA's transposed product then needs alpha^T, not alpha."""
    ob, k0, E0, ff0, G = _c1_inputs(orc, nnnr=10)
    nb, nmax = ob.nbsphere, ob.nmax
    pol = ob.polarisa.copy()
    rng = np.random.default_rng(11)
    for a in range(3):
        for b in range(3):
            pol[np.arange(nb) + nmax * (a + 3 * b)] += 0.1 * ob.alpha * (rng.standard_normal(nb) +
                                                                       1j * rng.standard_normal(nb))
    ref = orc.inverserig(G, 10, 10, 10, nb, pol, nmax, ff0, meth, 1e-6, tabdip=ob.tabdip)
    assert ref["nstop"] == 0
    g = gctx.green(10, 10, 10, ob.aretecube, k0)
    r = g.inverserig(nb, pol, nmax, ff0, meth, 1e-6, tabdip=ob.tabdip, precision=prec)
    assert r.nstop == 0, r.infostr
    if prec == 0:
        assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
        assert rel(r.FFloc, ref["FFloc"]) < 1e-7
        assert rel(r.FF, ref["FF"]) < 1e-7
    else:
        assert r.tol1[0] < 1e-6
        assert rel(r.FFloc, ref["FFloc"]) < 1e-4
    g.close()


def test_anisotropy_only_in_the_tail_matches_oracle(gctx, orc):
    """The host entry checks the first dipoles before it starts and scans the
    rest while an isotropic solve runs; a tensor that is anisotropic only
    beyond that head must still give the full-tensor result."""
    ob, k0, E0, ff0, G = _c1_inputs(orc, nnnr=24)
    nb, nmax = ob.nbsphere, ob.nmax
    assert nb > 5000
    pol = ob.polarisa.copy()
    tail = np.arange(5000, nb)
    pol[tail + nmax * (0 + 3 * 1)] += 0.05 * ob.alpha[tail]
    pol[tail + nmax * (1 + 3 * 0)] += 0.05 * ob.alpha[tail]
    ref = orc.inverserig(G, 24, 24, 24, nb, pol, nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip)
    g = gctx.green(24, 24, 24, ob.aretecube, k0)
    r = g.inverserig(nb, pol, nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip)
    assert r.nstop == ref["nstop"] == 0
    assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    g.close()


@pytest.mark.parametrize("meth", ["BICGSTAB", "CG", "TFQMR", "GPBICGsafe", "GPBICG2", "GPBICGplus", "GPBICGAR",
                                  "BICGSTARPLUS", "CORS", "GPBICOR", "QMRCLA"])
def test_other_methods_match_oracle(gctx, orc, meth):
    """The reference's other Krylov methods (pimzbicgstab.f, zcg.f, tfqmr.f,
    gpbicgsafe.f, gpbicg2.f, gpbicgplus.f, gpbicgar.f, qmrpim.f) on the sphere
    (inside-only, Tabdip) and on a full-box GRF cube: identical counters,
    local field within 1e-7, the method's tol1."""
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-5, tabdip=ob.tabdip)
    assert ref["nstop"] == 0, ref["infostr"]
    g = gctx.green(16, 16, 16, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-5, tabdip=ob.tabdip)
    assert r.nstop == 0, r.infostr
    assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
    assert abs(r.tol1[0] - ref["tol1"]) <= 1e-6 * ref["tol1"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7 and rel(r.FF, ref["FF"]) < 1e-7
    g.close()
    ob, k0, ff0, G = _grf(orc, 16)
    ref = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-5)
    g = gctx.green(16, 16, 16, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-5)
    assert (r.nstop, int(r.nloop[0]), int(r.ncompte[0])) == (ref["nstop"], ref["nloop"], ref["ncompte"])
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    g.close()


@pytest.mark.parametrize("meth", ["BICGSTAB", "CG", "TFQMR", "GPBICGsafe", "GPBICG2", "QMRCLA"])
def test_other_methods_mixed_precision(gctx, orc, meth):
    from ifdda import IFDDA_MIXED
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    tight = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-10,
                           tabdip=ob.tabdip)
    g = gctx.green(16, 16, 16, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, tabdip=ob.tabdip, precision=IFDDA_MIXED)
    assert r.nstop == 0, r.infostr
    assert r.tol1[0] < 1e-4
    assert rel(r.FFloc, tight["FFloc"]) < 1e-3
    g.close()


@pytest.mark.parametrize("nquad", [1, 2])
def test_integrated_green_spectrum_matches_oracle(gctx, orc, nquad):
    """Spectrum with the cube-averaged tensor inside nquad (calculgreenquadfft.f)."""
    nx, ny, nz = 6, 5, 4
    d, k0 = 11e-9, 2 * math.pi / 550e-9
    g = gctx.green(nx, ny, nz, d, k0, nquad=nquad)
    got = g.export()
    ref = orc.greencalculquadfft(nx, ny, nz, nquad, d, k0)
    for c in range(6):
        assert np.abs(got[c] - ref[c]).max() <= 1e-11 * np.abs(ref[c]).max(), c
    g.close()


def test_solve_with_integrated_green_matches_oracle(gctx, orc):
    ob, k0, E0, ff0, _ = _c1_inputs(orc, nnnr=10)
    G = orc.greencalculquadfft(10, 10, 10, 2, ob.aretecube, k0)
    ref = orc.inverserig(G, 10, 10, 10, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip)
    g = gctx.green(10, 10, 10, ob.aretecube, k0, nquad=2)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip)
    assert r.nstop == ref["nstop"] == 0
    assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    g.close()


@pytest.mark.parametrize("margins,nquad", [((4, 2, 4), 0), ((4, 2, 4), 1), ((3, 2, 5), 0)])
def test_wide_near_field_matches_oracle(gctx, orc, margins, nquad):
    """ifdda_nearfield_wide against the oracle's restatement on the same
    solved dipole moments (cdmlib.f:1967-2492); margins (3, 2, 5) give a 14 x
    12 x 18 box, whose 28 and 36 are padded to compiled lengths."""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.sphere(100e-9, 2.25 + 0.1j, 8, k0, "RR", na=0)
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 0.3, 0, 30.0, 40.0)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    sol = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-8)
    mx, my, mz = margins
    ref = orc.nearfield_wide(8, 8, 8, mx, my, mz, ob.aretecube, k0, 632.8e-9, nquad, ob.nbsphere, ob.nmax, ob.xs,
                             ob.ys, ob.zs, sol["FF"], ff0, ob.epsilon, E0, 30.0, 40.0, 0.3)
    got = gctx.nearfield_wide(8, 8, 8, mx, my, mz, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, sol["FF"], ff0, ob.epsilon,
                              ob.nmax, E0, 30.0, 40.0, 0.3, nquad=nquad)
    for key in ("xswf", "yswf", "zswf"):
        assert np.array_equal(got[key], ref[key]), key
    assert rel(got["incident"], ref["incident"]) < 1e-13
    assert rel(got["local"], ref["local"]) < 1e-11
    assert rel(got["macro"], ref["macro"]) < 1e-11


def test_cdmlib_wide_near_field(orc):
    """nproche = 2: full-box solve, then the wide field; on the object's sites
    the wide local field is the solve's."""
    from ifdda.cdmlib import cdmlib
    out = cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25 + 0j, nnnr=8, tolinit=1e-8,
                 methodeit="GPBICG1", nproche=2, nxmp=4, nymp=4, nzmp=4, theta=10.0, phi=0.0, pp=1.0, P0=1.0,
                 w0=6328.0)
    assert out["nstop"] == 0, out["infostr"]
    assert out["nbsphere"] == 512 and len(out["xswf"]) == 16 ** 3
    sites = [(k + 4) * 256 + (j + 4) * 16 + (i + 4) for k in range(8) for j in range(8) for i in range(8)]
    loc = out["localfield_wf"][0].reshape(-1, 3)[sites].reshape(-1)
    assert rel(loc, out["localfield"][0] if out["localfield"].ndim > 1 else out["localfield"]) < 1e-6


def test_farfield_csca_matches_oracle(gctx, orc):
    """ifdda_farfield_csca against the oracle's direct sum on the same dipole
    moments (cdmlib.f:2784-2880): Poynting per direction, Cscai, gasym."""
    ob, k0, E0, ff0, G = _c1_inputs(orc)
    sol = orc.inverserig(G, 16, 16, 16, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6, tabdip=ob.tabdip)
    ref = orc.farfield_csca(ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 20.0, 30.0, 30, 60)
    got = gctx.farfield_csca(ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 20.0, 30.0, 30, 60)
    assert np.array_equal(got["thetafield"], ref["thetafield"]) and np.array_equal(got["phifield"], ref["phifield"])
    assert rel(got["poyntingfield"], ref["poyntingfield"]) < 1e-12
    assert abs(got["Cscai"] - ref["Cscai"]) <= 1e-12 * ref["Cscai"]
    assert abs(got["gasym"] - ref["gasym"]) <= 1e-11 * abs(ref["gasym"])
    with pytest.raises(ifdda_error()):
        gctx.farfield_csca(ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 0.0, 0.0, 10, 60)


def ifdda_error():
    import ifdda
    return ifdda.IfddaError


def test_cdmlib_scattering_cross_section(orc):
    """nsectionsca = 1 through the cdmlib entry: Cscai agrees with Cext - Cabs
    (optical theorem) and with Mie within the DDA error."""
    from ifdda.cdmlib import cdmlib
    out = cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25 + 0j, nnnr=16, tolinit=1e-8,
                 methodeit="GPBICG1", nproche=0, P0=1.0, w0=6328.0, nsectionsca=1, ntheta=36, nphi=72)
    assert out["nstop"] == 0, out["infostr"]
    assert abs(out["Cscai"][0] - out["Csca"][0]) / out["Csca"][0] < 0.02
    _, mie_sca, _ = orc.mie(2.25, 100e-9, 632.8e-9)
    assert abs(out["Cscai"][0] - mie_sca) / mie_sca < 0.1
    assert out["poyntingfield"].shape == (1, 37 * 72)


@pytest.mark.parametrize("nfft2d", [128, 100])
def test_farfield_fft_matches_oracle(gctx, orc, nfft2d):
    """ifdda_farfield_fft against the oracle's 2-D FFT restatement
    (diffractefft2d.f, computegcfft2d.f, the Poynting interpolation); any
    nfft2d, the device evaluating the pupil frequencies only."""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.sphere(100e-9, 2.25 + 0.1j, 8, k0, "RR", na=0)
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 0.4, 0, 20.0, 30.0)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    sol = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-6)
    ref = orc.farfield_fft(8, 8, 8, ob.aretecube, ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 20.0, 30.0, nfft2d,
                           30, 60)
    got = gctx.farfield_fft(8, 8, 8, ob.aretecube, ob.xs, ob.ys, ob.zs, sol["FF"], k0, E0 ** 2, 20.0, 30.0, nfft2d,
                            30, 60)
    assert got["imaxk0"] == ref["imaxk0"]
    assert rel(got["kpos"], ref["kpos"]) < 1e-11 and rel(got["kneg"], ref["kneg"]) < 1e-11
    assert abs(got["Cscai"] - ref["Cscai"]) <= 1e-11 * ref["Cscai"]
    assert abs(got["gasym"] - ref["gasym"]) <= 1e-10 * abs(ref["gasym"])
    ok = np.isfinite(ref["poyntingfield"])
    assert np.array_equal(ok, np.isfinite(got["poyntingfield"]))
    assert rel(got["poyntingfield"][ok], ref["poyntingfield"][ok]) < 1e-10


def test_cdmlib_anisotropic_concentric_matches_oracle(orc):
    """trope = 'ani' on the concentric spheres (one tensor per shell): the
    solve with per-dipole tensors against the oracle's solve of the same
    object (its tensors checked against polaepstens in the CPU tests)."""
    from ifdda import objects
    from ifdda.cdmlib import cdmlib
    shells = [np.array([[2.25, 0.1j, 0.0], [-0.1j, 2.5 + 0.02j, 0.05], [0.0, 0.05, 3.0]]), 1.8 * np.eye(3)]
    out = cdmlib(wavelength=632.8, object="concentricsphere", rayons=[60.0, 120.0], epss=[2.0, 2.0], nnnr=12,
                 tolinit=1e-8, methodeit="GPBICG1", trope="ani", epsanis=shells, nproche=0, P0=1.0, w0=6328.0)
    assert out["nstop"] == 0, out["infostr"]
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.concentric([60e-9, 120e-9], [2.0, 2.0], 12, k0, "RR", na=-1, epsanis=shells)
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 0.0, 0.0)
    G = orc.greencalculfft(12, 12, 12, ob.aretecube, k0)
    ref = orc.inverserig(G, 12, 12, 12, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-8, tabdip=ob.tabdip)
    assert rel(out["localfield"], ref["FFloc"]) < 1e-9
    em = orc.local_macro_all(ob.nbsphere, ob.nmax, ob.epsilon, ref["FFloc"], ob.aretecube, k0)
    assert rel(out["macroscopicfield"][0], em) < 1e-9
