"""CPU tests of host-side logic: the cdmlib-style driver's input checks and
the bench's replica timing over two gloo ranks."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cdmlib_driver_rejects_like_the_reference():
    """Input checks of cdmlib/cdmlib.f:462-471 and :994-999 (no GPU needed:
    they run before any device work)."""
    from ifdda.cdmlib import cdmlib
    assert cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25, nnnr=8,
                  tolinit=1e-13)["infostr"] == "Tolerance for the iterative method too small!"
    assert cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25, nnnr=8,
                  tolinit=0.9)["infostr"] == "Tolerance  for the iterative method too large!"
    assert cdmlib(wavelength=632.8, object="sphere", rayon=1000.0, eps=2.25, nnnr=4)["infostr"] == \
        "Meshsize larger than lambda/4!"
    assert cdmlib(wavelength=632.8, object="sphere", rayon=0.0, eps=2.25, nnnr=8)["nstop"] == 1
    assert cdmlib(wavelength=632.8, object="torus", nnnr=8)["nstop"] == 1
    assert cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25, nnnr=8, nlocal=0, nmacro=0,
                  nsection=0)["infostr"] == "No calculation requested!"
    # anisotropic objects (cdmlib.f:597-611)
    ani = [[2.25, 0, 0], [0, 2.5, 0], [0, 0, 3.0]]
    assert cdmlib(wavelength=632.8, object="sphere", rayon=100.0, nnnr=8, trope="ani",
                  epsani=np.zeros((3, 3)))["infostr"] == "No relative permittivity given"
    assert cdmlib(wavelength=632.8, object="sphere", rayon=100.0, nnnr=8, trope="ani", epsani=ani,
                  polarizability="LA")["infostr"] == "Polarizability should be CM or RR with anisotropy"
    assert cdmlib(wavelength=632.8, object="inhomocuboid2", nnnr=8, trope="ani", epsani=ani)["nstop"] == 1
    assert cdmlib(wavelength=632.8, object="concentricsphere", rayons=[90.0, 190.0], epss=[3.0, 2.0], nnnr=8,
                  trope="ani", epsani=ani)["infostr"] == "epsanis: one 3x3 tensor per sphere"
    assert cdmlib(wavelength=632.8, object="arbitrary", nx=2, ny=2, nz=2, aretecube=10.0,
                  positions=np.zeros((8, 3)), trope="ani", epsani=ani)["infostr"] == \
        "epsani_site: one 3x3 tensor per dipole"
    assert cdmlib(wavelength=632.8, object="sphere", rayon=1000.0, eps=2.25, nnnr=4, trope="ani",
                  epsani=ani)["infostr"] == "Meshsize larger than lambda/4!"
    # microscope options (cdmlib.f:365-389)
    sph = dict(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25, nnnr=8, nlentille=1)
    assert cdmlib(numaper=1.5, **sph)["infostr"] == "Problem with numerical aperture!"
    assert cdmlib(gross=0.5, **sph)["infostr"] == "Problem with manification!"
    assert cdmlib(theta=95.0, **sph)["infostr"] == "Illumination on the wrong side with the options"
    assert cdmlib(ntypemic=3, **sph)["nstop"] == 1
    assert cdmlib(nquicklens=2, **sph)["nstop"] == 1
    # scattering cross section by integration (cdmlib.f:394-400, :2789-2793)
    sph = dict(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25, nnnr=8, nsectionsca=1)
    assert cdmlib(theta=50.0, **sph)["infostr"] == "Angle too strong: Imprecise calculation with FFT"
    assert cdmlib(ntheta=10, **sph)["infostr"] == "ntheta and nphi too small!"


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ws, r, local = bench.dist_setup()
    bench.barrier(ws)
    t = bench.max_over_ranks(10.0 + 5.0 * rank, ws)
    q.put((r, ws, t))
    dist.destroy_process_group()


def test_replica_timing_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert res == [(0, 2, 15.0), (1, 2, 15.0)]


def test_product_path_fails_loudly_without_a_gpu():
    """No CPU fallback: without a CUDA device the library's context creation
    fails (and frees what it made) and the host API raises."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import ifdda
    for _ in range(3):
        with pytest.raises(ifdda.IfddaError):
            ifdda.Context(0)
