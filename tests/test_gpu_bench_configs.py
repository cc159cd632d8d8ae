"""GPU parity at the benchmark configurations' own grids, through the C-ABI.

The kernels are templates on the FFT length of each axis, so the instances the
benchmark runs (lengths 128 for the 64^3 cube, 192/192/128 for the 96x96x64
ellipsoid lattice, 384 for the 192^3 object) are held to the oracle here, not
only the small-grid instances of test_gpu_parity.py:

* mat-vec (produitfftmatvectopt.f:3-121 / produitfftmatvect3.f:2-127) at each
  grid, FP64 within 1e-11 and FP32 within 2e-5 relative of the oracle, and a
  batch of right-hand sides in one launch sequence against the oracle per
  right-hand side;
* the complete FP64 GPBICG1 solve of the 64^3 GRF cube against the oracle's
  inverserig (inverserigopt.f:30-107): the same nloop and ncompte, the local
  field within 1e-7;
* the mixed-precision solve (FP32 inner, FP64 refinement to a true residual of
  1e-4) against a converged FP64 solve (true residual 1e-10; the FP64 drop-in
  is the oracle-held path above): local-field error at most 1e-4 relative, on
  the 64^3 cube and on 8 right-hand sides of the ellipsoid sweep.
"""
import math

import numpy as np
import pytest

from cases import c2, c3_disk, rel

pytestmark = pytest.mark.gpu


def _field(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


@pytest.mark.parametrize("dims", [(64, 64, 64), (96, 96, 64), (192, 192, 192)])
def test_matvec_at_bench_grid_matches_oracle(gctx, orc, dims):
    nx, ny, nz = dims
    N = nx * ny * nz
    d, k0 = 10e-9, 2 * math.pi / 500e-9
    x, b = _field(3 * N, 1), _field(3 * N, 2)
    G6 = orc.greencalculfft(nx, ny, nz, d, k0)
    ref = orc.matvec(G6, nx, ny, nz, x, b)
    g = gctx.green(nx, ny, nz, d, k0)
    assert rel(g.matvec(x, b), ref) < 1e-11
    assert rel(g.matvec(x, b, precision=2), ref) < 2e-5
    if dims == (64, 64, 64):
        # the inside-only path (Tabdip) on the same grid
        rng = np.random.default_rng(3)
        occ = rng.random(N) < 0.5
        tab = np.zeros(N, np.int32)
        tab[occ] = np.arange(1, occ.sum() + 1)
        nd = int(occ.sum())
        reft = orc.matvec(G6, nx, ny, nz, x[:3 * nd], b[:3 * nd], tabdip=tab)
        assert rel(g.matvec(x[:3 * nd], b[:3 * nd], tabdip=tab), reft) < 1e-11
        assert rel(g.matvec(x[:3 * nd], b[:3 * nd], tabdip=tab, precision=2), reft) < 2e-5
    del G6
    g.close()


def test_batched_matvec_at_c3_grid_matches_oracle(gctx, orc):
    """Four right-hand sides in one launch sequence (blockIdx.z = right-hand
    side) on the 192 x 192 x 128 grid, FP64 and FP32, each against the oracle."""
    import torch
    nx, ny, nz, R = 96, 96, 64, 4
    N = nx * ny * nz
    d, k0 = 10e-9, 2 * math.pi / 500e-9
    xs = np.stack([_field(3 * N, 10 + r) for r in range(R)])
    bs = np.stack([_field(3 * N, 20 + r) for r in range(R)])
    G6 = orc.greencalculfft(nx, ny, nz, d, k0)
    refs = [orc.matvec(G6, nx, ny, nz, xs[r], bs[r]) for r in range(R)]
    del G6
    g = gctx.green(nx, ny, nz, d, k0)
    for prec, dt, tol in ((0, torch.complex128, 1e-11), (2, torch.complex64, 2e-5)):
        x = torch.from_numpy(xs).to(dt).cuda()
        y = torch.from_numpy(bs).to(dt).cuda()
        g.matvec_device(R, N, x.data_ptr(), y.data_ptr(), precision=prec)
        gctx.synchronize()
        got = y.cpu().numpy()
        for r in range(R):
            assert rel(got[r], refs[r]) < tol, (prec, r)
    g.close()


def _c2_inputs(orc):
    ob, k0, E0 = c2()
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 1.0, 0, 20.0, 0.0)
    return ob, k0, E0, ff0


def test_c2_fp64_solve_matches_oracle(gctx, orc):
    """The FP64 drop-in on the benchmark's own 64^3 GRF cube: GPBICG1 to 1e-4,
    full box, the same counters as the oracle and the local field within 1e-7."""
    ob, k0, E0, ff0 = _c2_inputs(orc)
    G6 = orc.greencalculfft(64, 64, 64, ob.aretecube, k0)
    ref = orc.inverserig(G6, 64, 64, 64, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4)
    del G6
    g = gctx.green(64, 64, 64, ob.aretecube, k0)
    r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4)
    assert r.nstop == ref["nstop"] == 0, r.infostr
    assert int(r.nloop[0]) == ref["nloop"] and int(r.ncompte[0]) == ref["ncompte"]
    assert abs(r.tol1[0] - ref["tol1"]) <= 1e-6 * ref["tol1"]
    assert rel(r.FFloc, ref["FFloc"]) < 1e-7
    assert rel(r.FF, ref["FF"]) < 1e-7
    g.close()


def _mixed_vs_converged(g, ob, ff0, meth="GPBICG1"):
    from ifdda import IFDDA_FP64, IFDDA_MIXED
    conv = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-10, precision=IFDDA_FP64)
    assert conv.nstop == 0 and np.all(conv.tol1 <= 1e-10), conv.infostr
    mix = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0, meth, 1e-4, precision=IFDDA_MIXED)
    assert mix.nstop == 0 and np.all(mix.tol1 <= 1e-4), mix.infostr
    loc_c = conv.FFloc.reshape(-1, 3 * ob.nbsphere)
    loc_m = mix.FFloc.reshape(-1, 3 * ob.nbsphere)
    return max(rel(loc_m[r], loc_c[r]) for r in range(loc_c.shape[0]))


def test_c2_mixed_solve_within_1e4_of_converged(gctx, orc):
    ob, k0, E0, ff0 = _c2_inputs(orc)
    g = gctx.green(64, 64, 64, ob.aretecube, k0)
    assert _mixed_vs_converged(g, ob, ff0) <= 1e-4
    g.close()


def test_c3_mixed_solves_within_1e4_of_converged(gctx, orc):
    """Eight right-hand sides of the 128-incidence ellipsoid sweep (s and p of
    the first four (kx, ky) of the seeded NA 0.9 disk) solved as one batch."""
    from ifdda import objects
    lam = 500e-9
    k0 = 2 * math.pi / lam
    ob = objects.ellipsoid_lattice(96, 96, 64, 10e-9, 400e-9, 300e-9, 200e-9, 2.0, 2.6, 33, k0, "RR")
    E0, _ = objects.irradiance(1.0, 10 * lam)
    kx, ky = c3_disk(64, seed=3, k0=k0)
    ff0 = np.stack([orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, pp, 1, float(kx[i]), float(ky[i]))
                    for i in range(4) for pp in (0.0, 1.0)])
    g = gctx.green(96, 96, 64, ob.aretecube, k0)
    assert _mixed_vs_converged(g, ob, ff0) <= 1e-4
    g.close()
