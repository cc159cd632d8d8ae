"""GPU: the continuous-batching server gives each request the same result
alone and inside a concurrent mix (own context per slot, fixed-order
reductions), and every request converges to the FP64 true residual."""
import numpy as np
import pytest

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
