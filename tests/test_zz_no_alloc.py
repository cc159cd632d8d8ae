"""GPU: the allocation-free mat-vec (ifdda_matvec_noalloc) against the
allocating one (ifdda_matvec_device) and against the FP64 oracle.

Callers that cannot allocate device memory while they run (a real-time loop
avoiding cudaMalloc's device-wide synchronisation, a framework whose caching
allocator owns the GPU memory, an application whose memory budget is spoken
for) use the entry point whose scratch is a fixed array inside the library.
Both entry points run the same kernels, so the results must agree within the
FP64/FP32 tolerances of the parity tests (1e-11 / 2e-5 relative), and both
match the oracle's produitfftmatvectopt / produitfftmatvect3 restatement to
the same tolerances.  Three calls in a row check that the shared array left by
one call does not change the next, and that the second and third calls
allocate nothing: the device's default memory pool (where the library's other
entry points grow their workspaces) and the device's free memory are
unchanged across them.  The 7 x 5 x 3 lattice runs on the padded 8 x 5 x 3
box (14 is not a compiled FFT length), so the padded Tabdip and the padded
scratch size are exercised too.  This file is named to be collected last and
creates its own context, so it passes alone in a fresh process and after the
other tests.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    # in FP64: without a polarisability the values reach ~1e25, whose squares
    # overflow a single-precision norm
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _pool_used(dev):
    """Bytes in use in the device's default memory pool (driver API)."""
    from cuda.bindings import driver
    err, = driver.cuInit(0)
    assert err == driver.CUresult.CUDA_SUCCESS
    err, d = driver.cuDeviceGet(dev)
    assert err == driver.CUresult.CUDA_SUCCESS
    err, pool = driver.cuDeviceGetDefaultMemPool(d)
    assert err == driver.CUresult.CUDA_SUCCESS
    err, used = driver.cuMemPoolGetAttribute(pool, driver.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)
    assert err == driver.CUresult.CUDA_SUCCESS
    return int(used)


@pytest.mark.parametrize("dims,inside", [((16, 12, 10), False), ((16, 12, 10), True), ((7, 5, 3), False),
                                         ((7, 5, 3), True)])
def test_noalloc_matches_allocating_matvec_and_oracle(orc, dims, inside):
    import torch

    import ifdda
    from ifdda import IFDDA_FP32, IFDDA_FP64

    nx, ny, nz = dims
    N = nx * ny * nz
    d, k0 = 12e-9, 2 * math.pi / 550e-9
    ctx = ifdda.Context(0)
    g = ctx.green(nx, ny, nz, d, k0)
    G6 = orc.greencalculfft(nx, ny, nz, d, k0)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(11)
    nd = N
    tab_h, tab = None, None
    if inside:
        occ = rng.uniform(size=N) < 0.5
        tab_h = np.zeros(N, np.int32)
        tab_h[occ] = np.arange(1, occ.sum() + 1)
        nd = int(occ.sum())
        tab = torch.from_numpy(tab_h).to(dev)
    x_h = rng.standard_normal(3 * nd) + 1j * rng.standard_normal(3 * nd)
    b_h = rng.standard_normal(3 * nd) + 1j * rng.standard_normal(3 * nd)
    ref_orc = orc.matvec(G6, nx, ny, nz, x_h, b_h, tabdip=tab_h)
    tab_arg = C.c_void_p(tab.data_ptr()) if tab is not None else None
    for prec, dt, tol in ((IFDDA_FP64, torch.complex128, 1e-11), (IFDDA_FP32, torch.complex64, 2e-5)):
        x = torch.from_numpy(x_h).to(dt).to(dev)
        b = torch.from_numpy(b_h).to(dt).to(dev)
        ref = b.clone()
        g.matvec_device(1, nd, x.data_ptr(), ref.data_ptr(), tabdip_ptr=tab.data_ptr() if tab is not None else None,
                        precision=prec)
        ctx.synchronize()
        ref_h = ref.cpu().numpy()
        assert _rel(ref_h, ref_orc) <= tol
        # every output buffer exists before the first call, so nothing but
        # the library could allocate between the calls measured below
        ys = [b.clone() for _ in range(3)]
        torch.cuda.synchronize()
        mem = []
        for y in ys:
            rc = ctx.lib.ifdda_matvec_noalloc(g.h, prec, nd, tab_arg, C.c_void_p(x.data_ptr()),
                                              C.c_void_p(y.data_ptr()))
            assert rc == 0, ctx.last_error()
            ctx.synchronize()
            mem.append((_pool_used(0), torch.cuda.mem_get_info(0)[0]))
            got = y.cpu().numpy()
            assert _rel(got, ref_h) <= tol
            assert _rel(got, ref_orc) <= tol
        assert mem[1] == mem[0] and mem[2] == mem[0], mem
    g.close()
    ctx.close()


def test_noalloc_rejects_grids_beyond_its_scratch_and_bad_precision():
    import torch

    import ifdda
    from ifdda import IFDDA_FP64, IFDDA_MIXED

    ctx = ifdda.Context(0)
    g = ctx.green(48, 48, 48, 10e-9, 2 * math.pi / 600e-9)  # 18 * 48^3 * 16 B = 31.9 MB > 16 MiB
    N = 48 ** 3
    x = torch.zeros(3 * N, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    rc = ctx.lib.ifdda_matvec_noalloc(g.h, IFDDA_FP64, N, None, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()))
    assert rc == 1
    assert "scratch" in ctx.last_error()
    g.close()
    g = ctx.green(8, 8, 8, 10e-9, 2 * math.pi / 600e-9)
    for prec in (IFDDA_MIXED, 7, -1):
        rc = ctx.lib.ifdda_matvec_noalloc(g.h, prec, 512, None, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()))
        assert rc == 1
        assert "precision" in ctx.last_error()
    g.close()
    ctx.close()
