"""GPU: the allocation-free mat-vec (ifdda_matvec_noalloc) against the
allocating one (ifdda_matvec_device).

Callers that cannot allocate device memory while they run (a real-time loop
avoiding cudaMalloc's device-wide synchronisation, a framework whose caching
allocator owns the GPU memory, an application whose memory budget is spoken
for) use the entry point whose scratch is a fixed array inside the library.  Both entry points run the
same kernels, so the results must agree within the FP64/FP32 tolerances of the
parity tests (1e-11 / 2e-5 relative); two calls in a row check that the shared
array left by the first call does not change the second.  This file is named
to be collected last and creates its own context, so it passes alone in a
fresh process and after the other tests.
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


@pytest.mark.parametrize("inside", [False, True])
def test_noalloc_matches_allocating_matvec(inside):
    import torch

    import ifdda
    from ifdda import IFDDA_FP32, IFDDA_FP64

    nx, ny, nz = 16, 12, 10
    N = nx * ny * nz
    ctx = ifdda.Context(0)
    g = ctx.green(nx, ny, nz, 12e-9, 2 * math.pi / 550e-9)
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(11)
    nd = N
    tab = None
    if inside:
        occ = rng.uniform(size=N) < 0.5
        tab_h = np.zeros(N, np.int32)
        tab_h[occ] = np.arange(1, occ.sum() + 1)
        nd = int(occ.sum())
        tab = torch.from_numpy(tab_h).to(dev)
    for prec, dt, tol in ((IFDDA_FP64, torch.complex128, 1e-11), (IFDDA_FP32, torch.complex64, 2e-5)):
        x = torch.from_numpy(rng.standard_normal(3 * nd) + 1j * rng.standard_normal(3 * nd)).to(dt).to(dev)
        b = torch.from_numpy(rng.standard_normal(3 * nd) + 1j * rng.standard_normal(3 * nd)).to(dt).to(dev)
        ref = b.clone()
        g.matvec_device(1, nd, x.data_ptr(), ref.data_ptr(), tabdip_ptr=tab.data_ptr() if tab is not None else None,
                        precision=prec)
        ctx.synchronize()
        ref_h = ref.cpu().numpy()
        for _ in range(2):
            y = b.clone()
            torch.cuda.synchronize()
            rc = ctx.lib.ifdda_matvec_noalloc(g.h, prec, nd, C.c_void_p(tab.data_ptr()) if tab is not None else None,
                                              C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()))
            assert rc == 0, ctx.last_error()
            ctx.synchronize()
            assert _rel(y.cpu().numpy(), ref_h) <= tol
    g.close()
    ctx.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    import ifdda
    from ifdda import IFDDA_FP64

    ctx = ifdda.Context(0)
    g = ctx.green(48, 48, 48, 10e-9, 2 * math.pi / 600e-9)  # 18 * 48^3 * 16 B = 31.9 MB > 16 MiB
    N = 48 ** 3
    x = torch.zeros(3 * N, dtype=torch.complex128, device="cuda")
    y = torch.zeros_like(x)
    rc = ctx.lib.ifdda_matvec_noalloc(g.h, IFDDA_FP64, N, None, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()))
    assert rc == 1
    assert "scratch" in ctx.last_error()
    g.close()
    ctx.close()
