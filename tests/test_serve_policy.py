"""CPU: the serving admission policies pick the request the way they say
(fifo: the oldest; sjf: the least work among the arrived ones, the oldest
once it has waited the cap), and the policy is validated."""
import pytest

from ifdda import serve


def _req(rid, n, ninc, arrival):
    return serve.Request(rid=rid, shape="cube", n=n, d=10e-9, eps=2.0 + 0j, wavelength=600e-9,
                         incidences=[(0.0, 0.0, 1.0)] * ninc, arrival=arrival)


def test_fifo_takes_the_oldest():
    q = [_req(0, 96, 32, 0.0), _req(1, 16, 1, 0.1)]
    assert serve.pick_next(q, 1.0, "fifo", 5.0).rid == 0


def test_sjf_takes_the_least_work_among_arrived():
    q = [_req(0, 96, 32, 0.0), _req(1, 32, 4, 0.1), _req(2, 16, 2, 0.2), _req(3, 16, 1, 9.0)]
    # request 3 has the least work but has not arrived at t = 1
    assert serve.pick_next(q, 1.0, "sjf", 5.0).rid == 2
    # equal work: the earlier one
    q2 = [_req(0, 96, 32, 0.0), _req(1, 16, 2, 0.1), _req(2, 16, 2, 0.2)]
    assert serve.pick_next(q2, 1.0, "sjf", 5.0).rid == 1


def test_sjf_serves_the_oldest_after_the_wait_cap():
    q = [_req(0, 96, 32, 0.0), _req(1, 16, 1, 0.1)]
    assert serve.pick_next(q, 4.9, "sjf", 5.0).rid == 1
    assert serve.pick_next(q, 5.0, "sjf", 5.0).rid == 0


def test_policy_is_validated():
    with pytest.raises(ValueError):
        serve.Server(slots=1, policy="lifo")
    with pytest.raises(ValueError):
        serve.Server(slots=1, policy="sjf", ragged=True)


def test_readback_pool_reuses_buffers_when_arrays_are_freed():
    import gc
    pool = serve._PinnedPool(pin=False)  # host tensors: the logic without a GPU
    a = pool.array_view((3, 1000))[1]
    b = pool.array_view((2, 10))[1]
    assert a.shape == (3, 1000) and b.shape == (2, 10) and pool.free == []
    a[:] = 1.0
    big = a.ctypes.data
    v = a[1:]  # a view keeps the buffer out of the pool
    del a
    gc.collect()
    assert pool.free == []
    del v
    gc.collect()
    assert len(pool.free) == 1  # a's buffer is back
    c = pool.array_view((5, 5))[1]  # the smallest free buffer that fits
    assert c.ctypes.data == big and pool.free == []
    pool.prewarm(pool.GRAIN + 1, 2)
    assert len(pool.free) == 2 and all(f.numel() == 2 * pool.GRAIN for f in pool.free)
    del b, c
    gc.collect()
    assert len(pool.free) == 4
