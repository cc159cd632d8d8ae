"""ctypes wrapper of the CPU oracle (``oracle/_build/libifdda_oracle.so``).

TEST INFRASTRUCTURE ONLY.  The oracle is an FP64 C restatement of IF-DDA's
FFT-accelerated dipole solve (see ``ifdda_oracle.c`` for the reference
file:line each function follows).  Only the tests, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` import this module; the product path
never does.

Parity status: pinned by numpy.fft, a dense direct sum, the reference's own
GPBICG self-test (cdmlib/gpbicg.f:1-79) and the Mie series; unpinned with
respect to outputs of the reference itself (it cannot be compiled here).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libifdda_oracle.so")
_lib = None

c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)


def build() -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.orc_sunif.restype = C.c_double
        _lib.orc_num_threads.restype = C.c_int
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _z(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(C.c_int(n))


def num_threads() -> int:
    return lib().orc_num_threads()


def fft3d(v: np.ndarray, isign: int) -> np.ndarray:
    """fftsingletonz3d on an array shaped (n3, n2, n1) (x fastest)."""
    a = _z(v).copy()
    n3, n2, n1 = a.shape
    lib().orc_fft3d(_p(a), C.c_int(n1), C.c_int(n2), C.c_int(n3), C.c_int(isign))
    return a


def propa_espace_libre(r, r0, k0) -> np.ndarray:
    out = np.zeros(9, np.complex128)
    lib().orc_propa_espace_libre(*(C.c_double(float(v)) for v in r),
                                 *(C.c_double(float(v)) for v in r0),
                                 C.c_double(k0), _p(out))
    return out.reshape(3, 3, order="F")


def greencalculfft(nx, ny, nz, d, k0) -> np.ndarray:
    """Returns G6 shaped (6, 2nz, 2ny, 2nx): xx, xy, xz, yy, yz, zz."""
    M = 8 * nx * ny * nz
    g = np.zeros(6 * M, np.complex128)
    lib().orc_greencalculfft(C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_double(d),
                             C.c_double(k0), _p(g))
    return g.reshape(6, 2 * nz, 2 * ny, 2 * nx)


def greencalculquadfft(nx, ny, nz, nquad, d, k0) -> np.ndarray:
    """greencalculfft with the cube-averaged tensor at offsets within nquad."""
    M = 8 * nx * ny * nz
    g = np.zeros(6 * M, np.complex128)
    lib().orc_greencalculquadfft(C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_int(nquad), C.c_double(d),
                                 C.c_double(k0), _p(g))
    return g.reshape(6, 2 * nz, 2 * ny, 2 * nx)


def propaesplibreintsim(x, y, z, x0, y0, z0, k0, d, lim=1.0) -> np.ndarray:
    """Cube-averaged tensor, 3x3 (row a, column b)."""
    out = np.zeros(9, np.complex128)
    lib().orc_propaesplibreintsim(C.c_double(x), C.c_double(y), C.c_double(z), C.c_double(x0), C.c_double(y0),
                                  C.c_double(z0), C.c_double(k0), C.c_double(d), C.c_double(lim), _p(out))
    return out.reshape(3, 3).T


def matvec(G6, nx, ny, nz, FFX, FFB, tabdip=None) -> np.ndarray:
    """FFB - (1/M) IFFT(G~ FFT(pad FFX)); returns the new FFB."""
    g = _z(G6)
    x = _z(FFX)
    b = _z(FFB).copy()
    if tabdip is None:
        lib().orc_matvec_opt(_p(g), C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(x), _p(b))
    else:
        t = np.ascontiguousarray(tabdip, dtype=np.int32)
        lib().orc_matvec3(_p(g), C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(t), _p(x), _p(b))
    return b


def apply_transpose(G6, nx, ny, nz, nbsphere, polarisa, nmax, FFX, tabdip) -> np.ndarray:
    """A^T FFX with A = I - G alpha (the QMRCLA product, inverserigopt.f:555-584)."""
    g = _z(G6)
    x = _z(FFX)
    out = np.zeros(3 * nbsphere, dtype=np.complex128)
    t = np.ascontiguousarray(tabdip, dtype=np.int32)
    lib().orc_apply_transpose(_p(g), C.c_int(nx), C.c_int(ny), C.c_int(nz), _p(t), C.c_int(nbsphere), C.c_int(nmax),
                              _p(_z(polarisa)), _p(x), _p(out))
    return out


def matvec_direct(xs, ys, zs, k0, FFX, FFB) -> np.ndarray:
    xs = np.ascontiguousarray(xs, np.float64)
    ys = np.ascontiguousarray(ys, np.float64)
    zs = np.ascontiguousarray(zs, np.float64)
    x = _z(FFX)
    b = _z(FFB).copy()
    lib().orc_matvec_direct(C.c_int(len(xs)), _p(xs), _p(ys), _p(zs), C.c_double(k0), _p(x), _p(b))
    return b


_CANCEL = C.CFUNCTYPE(C.c_int, C.c_int)


def inverserig(G6, nx, ny, nz, nbsphere, polarisa, nmax, FF0, methodeit, tol,
               tabdip=None, max_matvecs=None, nlim=0):
    """Solver driver (inverserig / inverserigopt).  Returns a dict with
    FF, FFloc, tol1, nloop, ncompte, nstop, infostr.  ``max_matvecs`` stops
    the solve after that many mat-vecs (the bounded CPU-baseline sample);
    ``nlim`` > 0 replaces the reference's iteration limit of 10000."""
    g = _z(G6)
    pol = _z(polarisa)
    ff0 = _z(FF0)
    n3 = 3 * nbsphere
    FF = np.zeros(n3, np.complex128)
    FFloc = np.zeros(n3, np.complex128)
    tol1 = C.c_double(0)
    nloop = C.c_int(0)
    ncompte = C.c_int(0)
    nstop = C.c_int(0)
    info = C.create_string_buffer(b" " * 64, 65)
    tab = None if tabdip is None else np.ascontiguousarray(tabdip, dtype=np.int32)
    cb = None
    if max_matvecs is not None:
        lim = int(max_matvecs)
        cb = _CANCEL(lambda n: 1 if n >= lim else 0)
    lib().orc_inverserig(_p(g), C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_int(nbsphere),
                         _p(tab) if tab is not None else None, _p(pol), C.c_int(nmax), _p(ff0),
                         methodeit.encode(), C.c_double(tol), _p(FF), _p(FFloc),
                         C.byref(tol1), C.byref(nloop), C.byref(ncompte), C.byref(nstop),
                         info, cb, C.c_int(nlim))
    return dict(FF=FF, FFloc=FFloc, tol1=tol1.value, nloop=nloop.value,
                ncompte=ncompte.value, nstop=nstop.value,
                infostr=info.raw[:64].decode(errors="replace"))


def gpbicg_dense(mat, b, x0, tol, maxit=100):
    mat = np.asfortranarray(mat, dtype=np.complex128)
    b = _z(b)
    x = _z(x0).copy()
    nloop = C.c_int(0)
    st = lib().orc_gpbicg_dense(C.c_int(len(b)), _p(mat), _p(b), _p(x), C.c_double(tol),
                                C.c_int(maxit), C.byref(nloop))
    return x, st, nloop.value


def poladiff(rayon, eps, k0, methode, eps0=1.0, dddis=1) -> complex:
    """poladiff (cdmlib/polarisabilite.f:1-62) for one dipole."""
    return _poladiff_shim(rayon, complex(eps), eps0, k0, dddis, methode)


class _ZC(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def _poladiff_shim(rayon, eps, eps0, k0, dddis, methode):
    f = lib().orc_poladiff
    f.argtypes = [C.c_double, _ZC, C.c_double, C.c_double, C.c_int, C.c_char_p, C.c_void_p]
    f.restype = C.c_int
    out = np.zeros(1, np.complex128)
    rc = f(rayon, _ZC(eps.real, eps.imag), eps0, k0, dddis, methode.encode(), _p(out))
    if rc:
        raise ValueError("poladiff: bad method or dddis")
    return complex(out[0])


def local_macro_all(nbsphere, nmax, epsilon, FFloc, d, k0) -> np.ndarray:
    eps = _z(epsilon)
    loc = _z(FFloc)
    Em = np.zeros(3 * nbsphere, np.complex128)
    rc = lib().orc_macro_all(C.c_int(nbsphere), C.c_int(nmax), _p(eps), _p(loc),
                             C.c_double(d), C.c_double(k0), _p(Em))
    if rc:
        raise ValueError("local_macro: singular matrix")
    return Em


def irradiance(P0, w0):
    E0 = C.c_double(0)
    irra = C.c_double(0)
    lib().orc_irradiance(C.c_double(P0), C.c_double(w0), C.byref(E0), C.byref(irra))
    return E0.value, irra.value


def incident(xs, ys, zs, k0, E0, pp, beam, a1, a2) -> np.ndarray:
    """beam 0: ondeplane(theta=a1, phi=a2 in degrees); 1: ondeplanekxky(kx=a1, ky=a2)."""
    f = lib().orc_incident
    f.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, _ZC, C.c_double,
                  C.c_int, C.c_double, C.c_double, C.c_void_p]
    xs = np.ascontiguousarray(xs, np.float64)
    ys = np.ascontiguousarray(ys, np.float64)
    zs = np.ascontiguousarray(zs, np.float64)
    out = np.zeros(3 * len(xs), np.complex128)
    E0 = complex(E0)
    rc = f(len(xs), _p(xs), _p(ys), _p(zs), k0, _ZC(E0.real, E0.imag), pp, beam, a1, a2, _p(out))
    if rc:
        raise ValueError("problem in plance incident wave")
    return out


def cross_sections(FF0, FF, FFloc, k0, I0):
    Ce = C.c_double(0)
    Ca = C.c_double(0)
    n = len(FF0) // 3
    lib().orc_cross_sections(C.c_int(n), _p(_z(FF0)), _p(_z(FF)), _p(_z(FFloc)), C.c_double(k0),
                             C.c_double(I0), C.byref(Ce), C.byref(Ca))
    return Ce.value, Ca.value


def mie(eps, radius, wavelength):
    f = lib().orc_mie
    f.argtypes = [_ZC, C.c_double, C.c_double, c_double_p, c_double_p, c_double_p]
    a, b, c = C.c_double(0), C.c_double(0), C.c_double(0)
    e = complex(eps)
    f(_ZC(e.real, e.imag), radius, wavelength, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


def sunif_sequence(ir: int, n: int) -> np.ndarray:
    st = C.c_double(0)
    irr = C.c_int(ir)
    return np.array([lib().orc_sunif(C.byref(irr), C.byref(st)) for _ in range(n)])


class DipoleObject(dict):
    """Result of an object builder: nx, ny, nz, aretecube, nbsphere, ndipole,
    xs, ys, zs, tabdip, polarisa (nmax,3,3 column-major), epsilon, nmax."""

    def __getattr__(self, k):
        return self[k]


def _alloc(nmax):
    return (np.zeros(nmax), np.zeros(nmax), np.zeros(nmax), np.zeros(nmax, np.int32),
            np.zeros(9 * nmax, np.complex128), np.zeros(9 * nmax, np.complex128))


def _pack(nx, ny, nz, d, nb, nd, xs, ys, zs, tab, pol, eps, nmax):
    return DipoleObject(nx=nx, ny=ny, nz=nz, aretecube=d, nbsphere=nb, ndipole=nd,
                        xs=xs[:nb].copy(), ys=ys[:nb].copy(), zs=zs[:nb].copy(), tabdip=tab,
                        polarisa=pol, epsilon=eps, nmax=nmax)


def polaepstens(rayon, epsani, k0, methode, eps0=1.0, dis=1, inv=1) -> np.ndarray:
    """polaepstens (cdmlib/polaepstens.f:1-122): 3x3 polarisability of a cube
    of anisotropic permittivity epsani (3x3, [row, column])."""
    e = _z(np.asarray(epsani, np.complex128).T.ravel())  # column-major
    out = np.zeros(9, np.complex128)
    f = lib().orc_polaepstens
    f.argtypes = [C.c_double, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_char_p, C.c_int, C.c_void_p]
    f.restype = C.c_int
    if f(rayon, _p(e), eps0, k0, dis, methode.encode(), inv, _p(out)):
        raise ValueError("polaepstens: bad method, dis or singular matrix")
    return out.reshape(3, 3).T.copy()


def object_sphere(rayon, eps, nnnr, na, k0, methode, epsani=None):
    nmax = nnnr ** 3
    xs, ys, zs, tab, pol, ep = _alloc(nmax)
    nb, nd, d = C.c_int(0), C.c_int(0), C.c_double(0)
    if epsani is not None:
        ea = _z(np.asarray(epsani, np.complex128).T.ravel())
        rc = lib().orc_object_sphere_ani(C.c_double(rayon), _p(ea), C.c_int(nnnr), C.c_int(na), C.c_double(k0),
                                         methode.encode(), C.c_int(nmax), _p(xs), _p(ys), _p(zs), _p(tab),
                                         _p(pol), _p(ep), C.byref(nb), C.byref(nd), C.byref(d))
        if rc:
            raise ValueError("object sphere")
        return _pack(nnnr, nnnr, nnnr, d.value, nb.value, nd.value, xs, ys, zs, tab, pol, ep, nmax)
    f = lib().orc_object_sphere
    f.argtypes = [C.c_double, _ZC, C.c_int, C.c_int, C.c_double, C.c_char_p, C.c_int] + \
        [C.c_void_p] * 6 + [c_int_p, c_int_p, c_double_p]
    e = complex(eps)
    rc = f(rayon, _ZC(e.real, e.imag), nnnr, na, k0, methode.encode(), nmax, _p(xs), _p(ys),
           _p(zs), _p(tab), _p(pol), _p(ep), C.byref(nb), C.byref(nd), C.byref(d))
    if rc:
        raise ValueError("object sphere")
    return _pack(nnnr, nnnr, nnnr, d.value, nb.value, nd.value, xs, ys, zs, tab, pol, ep, nmax)


def object_cube(side, eps, nnnr, k0, methode, epsani=None):
    nmax = nnnr ** 3
    xs, ys, zs, tab, pol, ep = _alloc(nmax)
    nb, nd, d = C.c_int(0), C.c_int(0), C.c_double(0)
    if epsani is not None:
        ea = _z(np.asarray(epsani, np.complex128).T.ravel())
        rc = lib().orc_object_cube_ani(C.c_double(side), _p(ea), C.c_int(nnnr), C.c_double(k0), methode.encode(),
                                       C.c_int(nmax), _p(xs), _p(ys), _p(zs), _p(tab), _p(pol), _p(ep),
                                       C.byref(nb), C.byref(nd), C.byref(d))
        if rc:
            raise ValueError("object cube")
        return _pack(nnnr, nnnr, nnnr, d.value, nb.value, nd.value, xs, ys, zs, tab, pol, ep, nmax)
    f = lib().orc_object_cube
    f.argtypes = [C.c_double, _ZC, C.c_int, C.c_double, C.c_char_p, C.c_int] + \
        [C.c_void_p] * 6 + [c_int_p, c_int_p, c_double_p]
    e = complex(eps)
    rc = f(side, _ZC(e.real, e.imag), nnnr, k0, methode.encode(), nmax, _p(xs), _p(ys), _p(zs),
           _p(tab), _p(pol), _p(ep), C.byref(nb), C.byref(nd), C.byref(d))
    if rc:
        raise ValueError("object cube")
    return _pack(nnnr, nnnr, nnnr, d.value, nb.value, nd.value, xs, ys, zs, tab, pol, ep, nmax)


def object_inhomocuboid(nx, ny, nz, d, eps, lc, hc, ng, k0, methode):
    nmax = nx * ny * nz
    xs, ys, zs, tab, pol, ep = _alloc(nmax)
    nb, nd = C.c_int(0), C.c_int(0)
    f = lib().orc_object_inhomocuboid
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _ZC, C.c_double, C.c_double, C.c_int,
                  C.c_double, C.c_char_p, C.c_int] + [C.c_void_p] * 6 + [c_int_p, c_int_p]
    e = complex(eps)
    rc = f(nx, ny, nz, d, _ZC(e.real, e.imag), lc, hc, ng, k0, methode.encode(), nmax, _p(xs),
           _p(ys), _p(zs), _p(tab), _p(pol), _p(ep), C.byref(nb), C.byref(nd))
    if rc:
        raise ValueError("object inhomocuboid")
    return _pack(nx, ny, nz, d, nb.value, nd.value, xs, ys, zs, tab, pol, ep, nmax)


def object_concentric(rayons, epss, nnnr, na, k0, methode):
    nmax = nnnr ** 3
    xs, ys, zs, tab, pol, ep = _alloc(nmax)
    nb, nd, d = C.c_int(0), C.c_int(0), C.c_double(0)
    r = np.ascontiguousarray(rayons, np.float64)
    e = _z(epss)
    rc = lib().orc_object_concentric(C.c_int(len(r)), _p(r), _p(e), C.c_int(nnnr), C.c_int(na),
                                     C.c_double(k0), methode.encode(), C.c_int(nmax), _p(xs),
                                     _p(ys), _p(zs), _p(tab), _p(pol), _p(ep), C.byref(nb),
                                     C.byref(nd), C.byref(d))
    if rc:
        raise ValueError("object concentric")
    return _pack(nnnr, nnnr, nnnr, d.value, nb.value, nd.value, xs, ys, zs, tab, pol, ep, nmax)


def object_arbitrary(nx, ny, nz, d, px, py, pz, eps_site, k0, methode):
    nmax = nx * ny * nz
    xs, ys, zs, tab, pol, ep = _alloc(nmax)
    nb, nd = C.c_int(0), C.c_int(0)
    px = np.ascontiguousarray(px, np.float64)
    py = np.ascontiguousarray(py, np.float64)
    pz = np.ascontiguousarray(pz, np.float64)
    es = _z(eps_site)
    rc = lib().orc_object_arbitrary(C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_double(d), _p(px),
                                    _p(py), _p(pz), _p(es), C.c_double(k0), methode.encode(),
                                    C.c_int(nmax), _p(xs), _p(ys), _p(zs), _p(tab), _p(pol),
                                    _p(ep), C.byref(nb), C.byref(nd))
    if rc:
        raise ValueError("object arbitrary")
    return _pack(nx, ny, nz, d, nb.value, nd.value, xs, ys, zs, tab, pol, ep, nmax)


def microscope(ntypemic, G6, nx, ny, nz, d, k0, xs, ys, zs, polarisa, methodeit, tol, numaper, numaperinc, nfft2d,
               gross, zlens, P0, w0, nside=0, nquicklens=1, tabdip=None):
    """Bright-field (ntypemic 1, cdmlib/microsbf.f) or dark-field/phase
    (ntypemic 2, cdmlib/microsdf.f) microscope in transmission with the FFT
    lens, full box.  numaper is the objective's NA (multiplied by k0 here as
    cdmlib.f:3674 does); zlens in metres; nside 0 transmission, 1 reflection
    (microsbfneg / microsdfneg, cdmlib/microssansinc.f: no incident image);
    nquicklens 0: the lens's far field by direct summation, any object
    (tabdip for inside-only dipoles), 1: the FFT lens on the full box.  Returns a dict with image (6, n, n)
    [x, y, z, incx, incy, incz; row v, column u], xy, kxy, kxinc/kyinc (in
    units of k0), the last solve's tol1/nloop/ncompte, nstop, infostr."""
    n = int(nfft2d)
    img = np.zeros(6 * n * n, np.float64)
    xy = np.zeros(n, np.float64)
    kxy = np.zeros(n, np.float64)
    cap = 100000
    kxi = np.zeros(cap, np.float64)
    kyi = np.zeros(cap, np.float64)
    ninc = C.c_int(cap)
    tol1, nloop, ncompte = C.c_double(0), C.c_int(0), C.c_int(0)
    info = C.create_string_buffer(b" " * 64, 65)
    f = lib().orc_microscope
    f.restype = C.c_int
    tab = None if tabdip is None else np.ascontiguousarray(tabdip, np.int32)
    nstop = f(C.c_int(ntypemic), C.c_int(nside), C.c_int(nquicklens), _p(_z(G6)), C.c_int(nx), C.c_int(ny),
              C.c_int(nz), C.c_double(d), C.c_double(k0), C.c_int(len(xs)), _p(tab) if tab is not None else None,
              _p(np.ascontiguousarray(xs, np.float64)), _p(np.ascontiguousarray(ys, np.float64)),
              _p(np.ascontiguousarray(zs, np.float64)), _p(_z(polarisa)), methodeit.encode(), C.c_double(tol),
              C.c_double(numaper * k0), C.c_double(numaperinc), C.c_int(n), C.c_double(gross), C.c_double(zlens),
              C.c_double(P0), C.c_double(w0), _p(img), _p(xy), _p(kxy), C.byref(ninc), _p(kxi), _p(kyi),
              C.byref(tol1), C.byref(nloop), C.byref(ncompte), info)
    m = ninc.value
    return dict(image=img.reshape(6, n, n), xy=xy, kxy=kxy, kxinc=kxi[:m].copy(), kyinc=kyi[:m].copy(),
                tol1=tol1.value, nloop=nloop.value, ncompte=ncompte.value, nstop=nstop,
                infostr=info.raw[:64].decode(errors="replace"))


def nearfield_wide(nx, ny, nz, nxmp, nymp, nzmp, d, k0, lam, nquad, nbsphere, nmax, xs, ys, zs, FF, FF0, epsilon,
                   E0, theta, phi, pp):
    """Wide near field (cdmlib/cdmlib.f:1967-2492): returns dict with xswf,
    yswf, zswf, incident, local, macro on the enlarged box."""
    nw = (nx + 2 * nxmp) * (ny + 2 * nymp) * (nz + 2 * nzmp)
    px, py, pz = (np.zeros(nw) for _ in range(3))
    inc, loc, mac = (np.zeros(3 * nw, np.complex128) for _ in range(3))
    f = lib().orc_nearfield_wide
    f.argtypes = [C.c_int] * 6 + [C.c_double] * 3 + [C.c_int] * 3 + [C.c_void_p] * 6 + [_ZC] + \
        [C.c_double] * 3 + [C.c_void_p] * 6
    f.restype = C.c_int
    e0 = complex(E0)
    rc = f(nx, ny, nz, nxmp, nymp, nzmp, d, k0, lam, nquad, nbsphere, nmax,
           _p(np.ascontiguousarray(xs, np.float64)), _p(np.ascontiguousarray(ys, np.float64)),
           _p(np.ascontiguousarray(zs, np.float64)), _p(_z(FF)), _p(_z(FF0)), _p(_z(epsilon)),
           _ZC(e0.real, e0.imag), theta, phi, pp, _p(px), _p(py), _p(pz), _p(inc), _p(loc), _p(mac))
    if rc:
        raise ValueError("nearfield_wide: singular local-macro matrix")
    return dict(xswf=px, yswf=py, zswf=pz, incident=inc, local=loc, macro=mac)


def farfield_csca(xs, ys, zs, FF, k0, I0, theta, phi, ntheta, nphi):
    """Cscai, gasym and the Poynting vector by direct summation
    (cdmlib/cdmlib.f:2784-2880)."""
    nd = (ntheta + 1) * nphi
    pf, tf, phf = np.zeros(nd), np.zeros(nd), np.zeros(nd)
    cs, g = C.c_double(0), C.c_double(0)
    f = lib().orc_farfield_csca
    f.argtypes = [C.c_int] + [C.c_void_p] * 4 + [C.c_double] * 4 + [C.c_int] * 2 + [C.c_void_p] * 5
    f.restype = C.c_int
    xs = np.ascontiguousarray(xs, np.float64)
    if f(len(xs), _p(xs), _p(np.ascontiguousarray(ys, np.float64)), _p(np.ascontiguousarray(zs, np.float64)),
         _p(_z(FF)), k0, I0, theta, phi, ntheta, nphi, C.byref(cs), C.byref(g), _p(pf), _p(tf), _p(phf)):
        raise ValueError("ntheta and nphi too small!")
    return dict(Cscai=cs.value, gasym=g.value, poyntingfield=pf, thetafield=tf, phifield=phf)


def farfield_fft(nx, ny, nz, d, xs, ys, zs, FF, k0, I0, theta, phi, nfft2d, ntheta, nphi):
    """Cscai, gasym and the Poynting vector from the pupil-grid far field
    (diffractefft2d.f, computegcfft2d.f, cdmlib.f:2990-3075)."""
    nd = (ntheta + 1) * nphi
    pf, tf, phf = np.zeros(nd), np.zeros(nd), np.zeros(nd)
    kmax = nfft2d * nfft2d
    kp, kn = np.zeros(kmax), np.zeros(kmax)
    cs, g, imax = C.c_double(0), C.c_double(0), C.c_int(0)
    info = C.create_string_buffer(b" " * 64, 65)
    f = lib().orc_farfield_fft
    f.argtypes = [C.c_int] * 3 + [C.c_double] + [C.c_void_p] * 4 + [C.c_double] * 4 + [C.c_int] * 3 + \
        [C.c_void_p] * 5 + [C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p]
    f.restype = C.c_int
    rc = f(nx, ny, nz, d, _p(np.ascontiguousarray(xs, np.float64)), _p(np.ascontiguousarray(ys, np.float64)),
           _p(np.ascontiguousarray(zs, np.float64)), _p(_z(FF)), k0, I0, theta, phi, nfft2d, ntheta, nphi,
           C.byref(cs), C.byref(g), _p(pf), _p(tf), _p(phf), C.byref(imax), _p(kp), _p(kn), info)
    if rc:
        raise ValueError(info.raw[:64].decode().strip())
    S = 2 * imax.value + 1
    return dict(Cscai=cs.value, gasym=g.value, poyntingfield=pf, thetafield=tf, phifield=phf, imaxk0=imax.value,
                kpos=kp[:S * S].copy(), kneg=kn[:S * S].copy())


def holography(nx, ny, nz, d, k0, xs, ys, zs, FF, E0, theta, phi, pp, nfft2d, numaper, gross, zlens, nside=0,
               nquicklens=1):
    """Holographic microscope with the FFT lens after one plane-wave solve
    (cdmlib.f:4075-4660): complex image fields (6, n, n) [x, y, z, then with
    the incident wave], the pupil fields (6, S, S), xy, kxy, imaxk0."""
    n = int(nfft2d)
    img = np.zeros(6 * n * n, np.complex128)
    four = np.zeros(6 * n * n, np.complex128)
    xy, kxy = np.zeros(n), np.zeros(n)
    imax = C.c_int(0)
    info = C.create_string_buffer(b" " * 64, 65)
    f = lib().orc_holography
    f.argtypes = [C.c_int] * 3 + [C.c_double] * 2 + [C.c_int] + [C.c_void_p] * 4 + [_ZC] + [C.c_double] * 3 + \
        [C.c_int] + [C.c_double] * 3 + [C.c_int] * 2 + [C.c_void_p] * 5 + [C.c_char_p]
    f.restype = C.c_int
    e0 = complex(E0)
    rc = f(nx, ny, nz, d, k0, len(xs), _p(np.ascontiguousarray(xs, np.float64)), _p(np.ascontiguousarray(ys, np.float64)),
           _p(np.ascontiguousarray(zs, np.float64)), _p(_z(FF)), _ZC(e0.real, e0.imag), theta, phi, pp, n, numaper,
           gross, zlens, nside, nquicklens, _p(img), _p(four), _p(xy), _p(kxy), C.byref(imax), info)
    S = 2 * imax.value + 1
    return dict(nstop=rc, infostr=info.raw[:64].decode(errors="replace"), image=img.reshape(6, n, n),
                fourier=four[:6 * S * S].reshape(6, S, S), xy=xy, kxy=kxy, imaxk0=imax.value)
