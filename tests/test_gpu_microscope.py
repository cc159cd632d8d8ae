"""GPU: the microscopes (bright field, microsbf.f; dark field and phase,
microsdf.f) with the FFT lens, through the C-ABI, against the oracle's
restatement, which solves the illuminations one by one and forms the image
with full 2-D FFTs as the reference does.

The solves converge to the same iteration counts, so the dipole moments agree
to ~1e-10 and the images, sums of squared FFT outputs, to the same order; the
test allows 1e-8 (relative, per image component).  Incidence lists and axes
come from the same double arithmetic on the host and must be identical."""
import math

import numpy as np
import pytest

from cases import rel

pytestmark = pytest.mark.gpu


def _object(nnnr=8):
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.sphere(100e-9, 2.25 + 0j, nnnr, k0, "RR", na=0)  # full box
    return ob, k0


def _compare(r, ref, tol=1e-8):
    assert r.nstop == 0 and ref["nstop"] == 0, (r.infostr, ref["infostr"])
    assert np.array_equal(r.kxinc, ref["kxinc"]) and np.array_equal(r.kyinc, ref["kyinc"])
    assert np.array_equal(r.xy, ref["xy"]) and np.array_equal(r.kxy, ref["kxy"])
    assert r.nloop == ref["nloop"] and r.ncompte == ref["ncompte"]
    for c in range(6):
        assert rel(r.image[c], ref["image"][c]) < tol, c


@pytest.mark.parametrize("ntypemic,nfft2d,nside", [(1, 64, 0), (1, 128, 0), (2, 64, 0), (1, 64, 1), (2, 64, 1),
                                                  (1, 768, 0)])
def test_microscope_matches_oracle(gctx, orc, ntypemic, nfft2d, nside):
    ob, k0 = _object()
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    ref = orc.microscope(ntypemic, G, 8, 8, 8, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6,
                         0.9, 0.5, nfft2d, 100.0, 50e-9, 1.0, 6328e-9, nside=nside)
    g = gctx.green(8, 8, 8, ob.aretecube, k0)
    r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, ntypemic=ntypemic, nfft2d=nfft2d,
                     numaper=0.9, numaperinc=0.5, gross=100.0, zlens=50e-9, P0=1.0, w0=6328e-9, nside=nside)
    _compare(r, ref)
    # the image carries the object: the scattered intensity is not zero
    assert r.image[0].max() > 0
    if nside == 0:
        assert r.image[3].max() > r.image[0].max()
    else:  # reflection: no image with the incident wave (microssansinc.f)
        assert not r.image[3:].any()
    g.close()


def test_microscope_on_a_padded_lattice_matches_oracle(gctx, orc):
    """A 7^3 full-box sphere: 2 x 7 = 14 is not a compiled FFT length, so the
    solves run on the 8^3 box through a padded Tabdip while the FFT lens
    reads the caller's 7^3 lattice."""
    ob, k0 = _object(nnnr=7)
    G = orc.greencalculfft(7, 7, 7, ob.aretecube, k0)
    ref = orc.microscope(1, G, 7, 7, 7, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6,
                         0.9, 0.5, 64, 100.0, 50e-9, 1.0, 6328e-9)
    g = gctx.green(7, 7, 7, ob.aretecube, k0)
    r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, ntypemic=1, nfft2d=64, numaper=0.9,
                     numaperinc=0.5, gross=100.0, zlens=50e-9, P0=1.0, w0=6328e-9)
    _compare(r, ref)
    g.close()


@pytest.mark.parametrize("ntypemic,nside,inside", [(1, 0, True), (2, 0, False), (1, 1, True)])
def test_microscope_direct_lens_matches_oracle(gctx, orc, ntypemic, nside, inside):
    """nquicklens = 0: the lens's far field by direct summation over the
    dipoles, on the inside-only object or the full box (microsbf.f:139-157,
    627-666)."""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.sphere(100e-9, 2.25 + 0j, 8, k0, "RR", na=-1 if inside else 0)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    tab = ob.tabdip if inside else None
    ref = orc.microscope(ntypemic, G, 8, 8, 8, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6,
                         0.9, 0.5, 64, 100.0, 50e-9, 1.0, 6328e-9, nside=nside, nquicklens=0, tabdip=tab)
    g = gctx.green(8, 8, 8, ob.aretecube, k0)
    r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, ntypemic=ntypemic, nfft2d=64, numaper=0.9,
                     numaperinc=0.5, gross=100.0, zlens=50e-9, P0=1.0, w0=6328e-9, nside=nside, nquicklens=0,
                     tabdip=tab)
    _compare(r, ref)
    assert r.image[0].max() > 0
    g.close()


def test_microscope_batches_agree(gctx, orc):
    """Illuminations split over batches of 3 give the image of one batch."""
    ob, k0 = _object()
    g = gctx.green(8, 8, 8, ob.aretecube, k0)
    kw = dict(ntypemic=1, nfft2d=64, numaper=0.9, numaperinc=0.5, gross=100.0, zlens=0.0, P0=1.0, w0=6328e-9)
    a = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, batch=3, **kw)
    b = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, batch=0, **kw)
    assert a.nstop == 0 and b.nstop == 0
    for c in range(6):
        assert rel(a.image[c], b.image[c]) < 1e-12
    g.close()


def test_microscope_reports_the_references_errors(gctx, orc):
    ob, k0 = _object()
    g = gctx.green(8, 8, 8, ob.aretecube, k0)
    kw = dict(nfft2d=64, numaper=0.9, gross=100.0, zlens=0.0, P0=1.0, w0=6328e-9)
    r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, numaperinc=1.0, **kw)
    assert r.nstop == 1 and r.infostr.strip() == "NA inc strictly between 0 and 1"
    # a pupil grid too coarse for the condenser (dkx >= NA_inc k0)
    r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, numaperinc=0.1, **kw)
    ref = orc.microscope(1, orc.greencalculfft(8, 8, 8, ob.aretecube, k0), 8, 8, 8, ob.aretecube, k0, ob.xs, ob.ys,
                         ob.zs, ob.polarisa, "GPBICG1", 1e-6, 0.9, 0.1, 64, 100.0, 0.0, 1.0, 6328e-9)
    assert r.nstop == ref["nstop"] == 1 and r.infostr.strip() == ref["infostr"].strip()
    # nfft2d outside the compiled lengths
    r = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6, ntypemic=1, nfft2d=96, numaper=0.9,
                     numaperinc=0.5)
    assert r.nstop == 1 and "nfft2d not supported" in r.infostr
    g.close()


def test_cdmlib_microscope_matches_oracle(orc):
    """nlentille = 1 through the cdmlib-style entry: the object is put in its
    full box (cdmlib.f:631) and the images follow the normal-incidence
    solve; zlens in nm as the reference takes it."""
    from ifdda.cdmlib import cdmlib
    out = cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25 + 0j, nnnr=8, tolinit=1e-6,
                 methodeit="GPBICG1", polarizability="RR", nproche=0, P0=1.0, w0=6328.0, nlentille=1, ntypemic=2,
                 nfft2d=64, numaper=0.9, numaperinc=0.5, gross=100.0, zlens=50.0)
    assert out["nstop"] == 0, out["infostr"]
    assert out["nbsphere"] == 512  # full box
    ob, k0 = _object()
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    ref = orc.microscope(2, G, 8, 8, 8, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, ob.polarisa, "GPBICG1", 1e-6,
                         0.9, 0.5, 64, 100.0, 50e-9, 1.0, 6328e-9)
    for c, name in enumerate(("Eimagex", "Eimagey", "Eimagez", "Eimageincx", "Eimageincy", "Eimageincz")):
        assert rel(out[name], ref["image"][c]) < 1e-8, name


@pytest.mark.parametrize("nside,nfft2d", [(0, 64), (1, 64), (0, 128), (0, 768)])
def test_holography_matches_oracle(gctx, orc, nside, nfft2d):
    """ntypemic = 0 (cdmlib.f:4075-4660): the complex image fields of one
    oblique plane-wave solve, and the pupil fields, against the oracle's
    restatement with full 2-D FFTs."""
    ob, k0 = _object()
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 0.3, 0, 10.0, 30.0)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    sol = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-8)
    args = (8, 8, 8, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, sol["FF"], E0, 10.0, 30.0, 0.3)
    ref = orc.holography(*args, nfft2d, 0.9, 100.0, 50e-9, nside=nside)
    got = gctx.holography(*args, nfft2d=nfft2d, numaper=0.9, gross=100.0, zlens=50e-9, nside=nside)
    assert got["nstop"] == ref["nstop"] == 0, (got["infostr"], ref["infostr"])
    assert got["imaxk0"] == ref["imaxk0"]
    assert np.array_equal(got["xy"], ref["xy"]) and np.array_equal(got["kxy"], ref["kxy"])
    for c in range(3 if nside else 6):
        assert rel(got["image"][c], ref["image"][c]) < 1e-10, c
        assert rel(got["fourier"][c], ref["fourier"][c]) < 1e-10, c
    if nside:
        assert not got["image"][3:].any()
    else:  # the incident wave dominates the image with it
        assert np.abs(got["image"][3]).max() > np.abs(got["image"][0]).max()


def test_cdmlib_holography_matches_oracle(orc):
    """ntypemic = 0 through the cdmlib entry (the reference's test1 driver
    runs this microscope): full box, then the holographic images of the
    solve's plane wave."""
    from ifdda.cdmlib import cdmlib
    out = cdmlib(wavelength=632.8, object="sphere", rayon=100.0, eps=2.25 + 0j, nnnr=8, tolinit=1e-8,
                 methodeit="GPBICG1", nproche=0, theta=10.0, phi=30.0, pp=0.3, P0=1.0, w0=6328.0, nlentille=1,
                 ntypemic=0, nfft2d=64, numaper=0.9, gross=100.0, zlens=50.0)
    assert out["nstop"] == 0, out["infostr"]
    assert out["nbsphere"] == 512
    ob, k0 = _object()
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ref = orc.holography(8, 8, 8, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, out["FF"], E0, 10.0, 30.0, 0.3, 64, 0.9,
                         100.0, 50e-9)
    for c, name in enumerate(("Eimagex", "Eimagey", "Eimagez", "Eimageincx", "Eimageincy", "Eimageincz")):
        assert rel(out[name], ref["image"][c]) < 1e-10, name


@pytest.mark.parametrize("nside,inside", [(0, True), (1, False)])
def test_holography_direct_lens_matches_oracle(gctx, orc, nside, inside):
    """Holography without the FFT lens (cdmlib.f:3803-4074): the finer pupil
    grid and the far field by direct summation, on the inside-only object or
    the full box."""
    from ifdda import objects
    k0 = 2 * math.pi / 632.8e-9
    ob = objects.sphere(100e-9, 2.25 + 0j, 8, k0, "RR", na=-1 if inside else 0)
    E0, _ = orc.irradiance(1.0, 6328e-9)
    ff0 = orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, 0.3, 0, 10.0, 30.0)
    G = orc.greencalculfft(8, 8, 8, ob.aretecube, k0)
    sol = orc.inverserig(G, 8, 8, 8, ob.nbsphere, ob.polarisa, ob.nmax, ff0, "GPBICG1", 1e-8,
                         tabdip=ob.tabdip_or_none)
    args = (8, 8, 8, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, sol["FF"], E0, 10.0, 30.0, 0.3)
    ref = orc.holography(*args, 64, 0.9, 100.0, 50e-9, nside=nside, nquicklens=0)
    got = gctx.holography(*args, nfft2d=64, numaper=0.9, gross=100.0, zlens=50e-9, nside=nside, nquicklens=0)
    assert got["nstop"] == ref["nstop"] == 0, (got["infostr"], ref["infostr"])
    assert got["imaxk0"] == ref["imaxk0"] > 20
    assert np.array_equal(got["xy"], ref["xy"])
    for c in range(3 if nside else 6):
        assert rel(got["image"][c], ref["image"][c]) < 1e-10, c
        assert rel(got["fourier"][c], ref["fourier"][c]) < 1e-10, c
