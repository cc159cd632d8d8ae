"""GPU: the continuous-batching server gives each request the same result
alone and inside a concurrent mix (own context per slot, fixed-order
reductions), every request converges to the FP64 true residual, small
requests match the oracle's solve of the same object, and the HBM footprint
the admission uses covers what a request really holds on the device."""
import numpy as np
import pytest

from cases import rel

pytestmark = pytest.mark.gpu


def test_results_identical_alone_and_in_the_mix():
    from ifdda import IFDDA_MIXED
    from ifdda import serve
    reqs = serve.make_stream(8, rate=1000.0, seed=9, edges=(16, 24, 32), max_inc=4)
    alone = serve.Server(slots=1, precision=IFDDA_MIXED)
    ra = alone.run(reqs, realtime=False)
    alone.close()
    mix = serve.Server(slots=4, precision=IFDDA_MIXED)
    rm = mix.run(reqs, realtime=True)
    mix.close()
    assert len(ra) == len(rm) == len(reqs)
    assert len({r.slot for r in rm}) > 1  # the mix really ran on several slots
    for a, b in zip(ra, rm):
        assert a.rid == b.rid and a.nstop == b.nstop == 0
        assert np.array_equal(a.FFloc, b.FFloc)
        assert np.array_equal(a.nloop, b.nloop)
        assert np.all(b.tol1 < 1e-4)
    # least-work-first admission serves the same results in another order
    sjf = serve.Server(slots=2, precision=IFDDA_MIXED, policy="sjf")
    rs = sjf.run(reqs, realtime=True)
    sjf.close()
    for a, b in zip(ra, rs):
        assert a.rid == b.rid and b.nstop == 0
        assert np.array_equal(a.FFloc, b.FFloc)


@pytest.mark.parametrize("prec", [0, 1])
def test_ragged_serving_identical_alone_and_in_batches(prec):
    """Ragged serving: requests of several sizes batched per box (sides 12,
    16, 24 and 32, each on its own box), each request alone (batches of one
    object) against the mix (up to 8 objects per ragged batch): bit for bit
    the same fields and counters.  (A request padded into a larger box runs
    longer FFTs, so it agrees with its own-box result to the solver's
    tolerance, not bit for bit; the mix here pads nothing.)"""
    from ifdda import serve
    reqs = serve.make_stream(12, rate=1000.0, seed=13, edges=(12, 16, 24, 32), max_inc=3)
    alone = serve.Server(slots=1, precision=prec, ragged=True, max_objects=1)
    ra = alone.run(reqs, realtime=False)
    alone.close()
    mix = serve.Server(slots=2, precision=prec, ragged=True, max_objects=8)
    rm = mix.run(reqs, realtime=False)
    mix.close()
    assert len(ra) == len(rm) == len(reqs)
    groups = {}
    for r in rm:
        groups.setdefault((r.slot, r.start), []).append(r.rid)
    assert max(len(v) for v in groups.values()) > 1  # some batch held several objects
    for a, b in zip(ra, rm):
        assert a.rid == b.rid and a.nstop == b.nstop == 0, (a.infostr, b.infostr)
        assert np.array_equal(a.FFloc, b.FFloc)
        assert np.array_equal(a.ncompte, b.ncompte)
        assert np.all(b.tol1 < 1e-4)


@pytest.mark.parametrize("prec", [0, 1])
def test_served_requests_match_the_oracle(orc, prec):
    """Three small requests (sphere and cube, several incidences) served in a
    mix; each right-hand side's local field against the oracle's inverserig
    of the same object and incident field.  FP64 requests reproduce the
    oracle's counters and field (1e-7); for mixed ones the oracle's own
    operator (the produitfftmatvect3 restatement) confirms the true residual
    ||E - G alpha E - E0|| / ||E0|| <= 1e-4."""
    from ifdda import objects, serve
    reqs = serve.make_stream(3, rate=1000.0, seed=21, edges=(12, 16), max_inc=3)
    srv = serve.Server(slots=2, precision=prec)
    res = srv.run(reqs, realtime=False)
    srv.close()
    for req, r in zip(reqs, res):
        ob, k0 = serve.build_object(req)
        E0, _ = objects.irradiance(1.0, 10 * req.wavelength)
        G6 = orc.greencalculfft(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
        floc = np.asarray(r.FFloc).reshape(len(req.incidences), -1)
        for q, (a, b, pp) in enumerate(req.incidences):
            ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, pp, 1, a * k0, b * k0)
            ref = orc.inverserig(G6, ob.nx, ob.ny, ob.nz, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-4,
                                 tabdip=ob.tabdip_or_none)
            assert ref["nstop"] == 0 and r.nstop == 0
            if prec == 0:
                assert int(np.atleast_1d(r.ncompte)[q]) == ref["ncompte"]
                assert rel(floc[q], ref["FFloc"]) < 1e-7
            else:
                E = floc[q]
                p = np.repeat(ob.alpha, 3) * E  # isotropic: FF = alpha E per dipole
                AE = orc.matvec(G6, ob.nx, ob.ny, ob.nz, p, E, tabdip=ob.tabdip_or_none)
                assert np.linalg.norm(AE - ff0) / np.linalg.norm(ff0) <= 1e-4


def _pool():
    from cuda.bindings import driver
    assert driver.cuInit(0)[0] == driver.CUresult.CUDA_SUCCESS
    err, d = driver.cuDeviceGet(0)
    err, pool = driver.cuDeviceGetDefaultMemPool(d)
    assert err == driver.CUresult.CUDA_SUCCESS
    return driver, pool


@pytest.mark.parametrize("prec", [0, 1])
def test_footprint_covers_the_device_memory_of_a_request(prec):
    """footprint_bytes (the admission's estimate) against what one request
    really holds over its Green build and solve: the high-water mark of the
    device memory pool, from which the library takes every workspace, plus
    the peak of the request's own device inputs and outputs (torch).  The
    estimate is an upper bound, and no more than 3x the real use."""
    import torch
    from ifdda import serve
    driver, pool = _pool()
    A = driver.CUmemPool_attribute
    for n, ninc in ((24, 4), (48, 8)):
        req = serve.Request(rid=0, shape="cube", n=n, d=10e-9, eps=2.5 + 0.1j, wavelength=600e-9,
                            incidences=[(0.1 * i, 0.05 * i, float(i % 2)) for i in range(ninc)])
        slot = serve._Slot(0, 0, cache_size=1)
        slot.ctx.synchronize()
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats(0)
        tbase = torch.cuda.memory_allocated(0)
        base = int(driver.cuMemPoolGetAttribute(pool, A.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)[1])
        assert driver.cuMemPoolSetAttribute(pool, A.CU_MEMPOOL_ATTR_USED_MEM_HIGH, driver.cuuint64_t(0))[0] == \
            driver.CUresult.CUDA_SUCCESS
        r, hit = serve.solve_request(slot, req, prec)
        slot.ctx.synchronize()
        high = int(driver.cuMemPoolGetAttribute(pool, A.CU_MEMPOOL_ATTR_USED_MEM_HIGH)[1])
        tpeak = torch.cuda.max_memory_allocated(0) - tbase
        slot.close()
        assert r["nstop"] == 0 and not hit
        used = high - base + tpeak
        fp = serve.footprint_bytes(n, ninc, prec)
        assert used <= fp <= 3 * used, (n, ninc, used, fp)


def test_admission_respects_the_hbm_budget():
    from ifdda import IFDDA_MIXED
    from ifdda import serve
    reqs = serve.make_stream(6, rate=1000.0, seed=5, edges=(24, 32), max_inc=2)
    # a budget below every footprint admits one request at a time (the server
    # always admits a request when nothing else is in flight)
    srv = serve.Server(slots=3, precision=IFDDA_MIXED, hbm_budget=1.0)
    res = srv.run(reqs, realtime=False)
    srv.close()
    spans = sorted((r.start, r.end) for r in res)
    for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
        assert s1 >= e0 - 1e-3  # never two requests in flight
