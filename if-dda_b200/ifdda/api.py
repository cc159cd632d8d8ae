"""Object interface over the C-ABI (numpy in, numpy out).

Errors follow the reference's nstop/infostr convention: a failing solve
returns nstop = 1 and the reference's message in ``infostr`` ("Problem to
solve Ax=b!", "Converge do not reach!", "Iterative method not correct!");
a failing library call (bad argument, CUDA error) raises IfddaError.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import IFDDA_FP32, IFDDA_FP64, IFDDA_MIXED, DComplex, MicroscopeOptions, SolveOptions


class IfddaError(RuntimeError):
    pass


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _zc(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.complex128)


@dataclass
class SolveResult:
    FF: np.ndarray            # dipole moments polarisa . E
    FFloc: np.ndarray         # local field E
    tol1: np.ndarray          # true residual per right-hand side
    nloop: np.ndarray
    ncompte: np.ndarray
    nstop: int
    infostr: str
    extra: dict = field(default_factory=dict)


@dataclass
class MicroscopeResult:
    image: np.ndarray   # (6, n, n): |E| of x, y, z, then with the incident wave
    xy: np.ndarray      # image positions (m)
    kxy: np.ndarray     # pupil kx / k0
    kxinc: np.ndarray   # incidences of one polarisation, units of k0
    kyinc: np.ndarray
    tol1: float         # last solve
    nloop: int
    ncompte: int
    nstop: int
    infostr: str


class Context:
    """One CUDA device and stream (ifdda_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = _capi.load()
        h = C.c_void_p()
        if self.lib.ifdda_ctx_create(int(device), C.byref(h)) != 0:
            raise IfddaError(f"ifdda_ctx_create failed for device {device}")
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.ifdda_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def last_error(self) -> str:
        return (self.lib.ifdda_ctx_last_error(self.h) or b"").decode()

    def stream(self) -> int:
        return self.lib.ifdda_ctx_stream(self.h) or 0

    def synchronize(self):
        self._check(self.lib.ifdda_ctx_synchronize(self.h))

    def _check(self, rc):
        if rc != 0:
            raise IfddaError(self.last_error() or f"ifdda call failed ({rc})")

    def green(self, nx, ny, nz, aretecube, k0, nquad=0) -> "GreenSpectrum":
        return GreenSpectrum(self, nx, ny, nz, aretecube, k0, nquad)

    def green_box(self, nx, ny, nz, box, aretecube, k0) -> "GreenSpectrum":
        """Spectrum of an nx x ny x nz lattice on the larger box `box` (bx,
        by, bz): the form every object of a ragged batch needs."""
        return GreenSpectrum(self, nx, ny, nz, aretecube, k0, 0, box=box)

    def inverserig_ragged(self, items, methodeit="GPBICG1", tol=1e-4, precision=IFDDA_FP64, maxit=0):
        """Ragged batch: items = [(green, nbsphere, nmax, tabdip or None,
        polarisa, FF0 (nrhs_i, 3 nbsphere))], every green from green_box on
        one box.  Returns (per item (FF, FFloc), tol1, nloop, ncompte, nstop,
        infostr) with the counters of every right-hand side in item order."""
        n = len(items)
        keep = []
        ff0s, ffs, locs = [], [], []
        for g, nb, nmax, tab, pol, ff0 in items:
            f = _zc(ff0).reshape(-1, 3 * nb)
            ff0s.append(f)
            ffs.append(np.zeros_like(f))
            locs.append(np.zeros_like(f))
        R = sum(f.shape[0] for f in ff0s)
        arr = lambda t, vals: (t * n)(*vals)
        greens = arr(C.c_void_p, [it[0].h for it in items])
        nrhs = arr(C.c_int, [f.shape[0] for f in ff0s])
        nbs = arr(C.c_int, [int(it[1]) for it in items])
        nmaxs = arr(C.c_int, [int(it[2]) for it in items])
        tabs_np = [None if it[3] is None else np.ascontiguousarray(it[3], np.int32) for it in items]
        pols_np = [_zc(it[4]) for it in items]
        keep += tabs_np + pols_np
        tabs = arr(C.c_void_p, [None if t is None else t.ctypes.data for t in tabs_np])
        pols = arr(C.c_void_p, [p.ctypes.data for p in pols_np])
        p_ff0 = arr(C.c_void_p, [f.ctypes.data for f in ff0s])
        p_ff = arr(C.c_void_p, [f.ctypes.data for f in ffs])
        p_loc = arr(C.c_void_p, [f.ctypes.data for f in locs])
        tol1 = np.zeros(R)
        nloop = np.zeros(R, np.int32)
        ncompte = np.zeros(R, np.int32)
        nstop = C.c_int(0)
        info = C.create_string_buffer(b" " * 64, 65)
        opt = SolveOptions(precision, 0, 0, 0.0, maxit)
        rc = self.lib.ifdda_inverserig_ragged(n, greens, nrhs, nbs, nmaxs, tabs, pols, p_ff0, methodeit.encode(),
                                              float(tol), p_ff, p_loc, _p(tol1), _p(nloop), _p(ncompte),
                                              C.byref(nstop), info, C.byref(opt))
        infostr = info.raw[:64].decode(errors="replace")
        if rc == 1 and nstop.value == 0:
            raise IfddaError(self.last_error() or infostr.strip())
        return list(zip(ffs, locs)), tol1, nloop, ncompte, nstop.value, infostr

    # -- post-step ------------------------------------------------------
    def local_macro(self, nbsphere, nmax, epsilon, FFloc, aretecube, k0) -> np.ndarray:
        eps = _zc(epsilon)
        loc = _zc(FFloc)
        em = np.zeros(3 * nbsphere, np.complex128)
        self._check(self.lib.ifdda_local_macro(self.h, nbsphere, nmax, _p(eps), _p(loc), aretecube, k0, _p(em)))
        return em

    def cross_sections(self, FF0, FF, FFloc, k0, I0):
        a, b, c = _zc(FF0), _zc(FF), _zc(FFloc)
        ce, ca = C.c_double(0), C.c_double(0)
        self._check(self.lib.ifdda_cross_sections(self.h, len(a) // 3, _p(a), _p(b), _p(c), k0, I0, C.byref(ce),
                                                  C.byref(ca)))
        return ce.value, ca.value

    def holography(self, nx, ny, nz, aretecube, k0, xs, ys, zs, FF, E0, theta, phi, pp, nfft2d=128, numaper=0.9,
                   gross=100.0, zlens=0.0, nside=0, nquicklens=1) -> dict:
        """Holographic microscope with the FFT lens after one plane-wave solve
        (cdmlib.f:4075-4660): complex image fields (6, n, n) [x, y, z, then
        with the incident wave], pupil fields (6, S, S), xy, kxy, imaxk0,
        nstop, infostr."""
        n = int(nfft2d)
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        zs = np.ascontiguousarray(zs, np.float64)
        ff = _zc(FF)
        img = np.zeros((6, n, n), np.complex128)
        imax_est = max(int(round(k0 * n * aretecube / (2 * math.pi))) + 2, n // 2)
        four = np.zeros(6 * (2 * imax_est + 1) ** 2, np.complex128)
        xy, kxy = np.zeros(n), np.zeros(n)
        im = C.c_int(0)
        info = C.create_string_buffer(b" " * 64, 65)
        e0 = complex(E0)
        rc = self.lib.ifdda_holography(self.h, nx, ny, nz, aretecube, k0, len(xs), _p(xs), _p(ys), _p(zs), _p(ff),
                                       DComplex(e0.real, e0.imag), theta, phi, pp, n, numaper, gross, zlens, nside,
                                       nquicklens, _p(img), _p(four), _p(xy), _p(kxy), C.byref(im), info)
        S = 2 * im.value + 1
        return dict(nstop=rc, infostr=info.raw[:64].decode(errors="replace"), image=img,
                    fourier=four[:6 * S * S].reshape(6, S, S), xy=xy, kxy=kxy, imaxk0=im.value)

    def farfield_csca(self, xs, ys, zs, FF, k0, I0, theta, phi, ntheta, nphi) -> dict:
        """Cscai, gasym and the far-field Poynting vector by direct summation
        over (ntheta+1) x nphi directions (cdmlib.f:2784-2880)."""
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        zs = np.ascontiguousarray(zs, np.float64)
        ff = _zc(FF)
        nd = (ntheta + 1) * nphi
        pf, tf, phf = np.zeros(nd), np.zeros(nd), np.zeros(nd)
        cs, g = C.c_double(0), C.c_double(0)
        self._check(self.lib.ifdda_farfield_csca(self.h, len(xs), _p(xs), _p(ys), _p(zs), _p(ff), k0, I0, theta, phi,
                                                 ntheta, nphi, C.byref(cs), C.byref(g), _p(pf), _p(tf), _p(phf)))
        return dict(Cscai=cs.value, gasym=g.value, poyntingfield=pf, thetafield=tf, phifield=phf)

    def farfield_fft(self, nx, ny, nz, aretecube, xs, ys, zs, FF, k0, I0, theta, phi, nfft2d, ntheta, nphi) -> dict:
        """Cscai, gasym and the Poynting vector from the far field on the
        pupil grid of nfft2d (diffractefft2d.f, computegcfft2d.f,
        cdmlib.f:2990-3075); FF on the full box."""
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        zs = np.ascontiguousarray(zs, np.float64)
        ff = _zc(FF)
        nd = (ntheta + 1) * nphi
        pf, tf, phf = np.zeros(nd), np.zeros(nd), np.zeros(nd)
        imax = int(round(k0 * nfft2d * aretecube / (2 * math.pi))) + 2
        S = 2 * imax + 1
        kp, kn = np.zeros(S * S), np.zeros(S * S)
        cs, g, im = C.c_double(0), C.c_double(0), C.c_int(0)
        self._check(self.lib.ifdda_farfield_fft(self.h, nx, ny, nz, aretecube, _p(xs), _p(ys), _p(zs), _p(ff), k0, I0,
                                                theta, phi, nfft2d, ntheta, nphi, C.byref(cs), C.byref(g), _p(pf),
                                                _p(tf), _p(phf), C.byref(im), _p(kp), _p(kn)))
        S = 2 * im.value + 1
        return dict(Cscai=cs.value, gasym=g.value, poyntingfield=pf, thetafield=tf, phifield=phf, imaxk0=im.value,
                    kpos=kp[:S * S].copy(), kneg=kn[:S * S].copy())

    def nearfield_wide(self, nx, ny, nz, nxmp, nymp, nzmp, aretecube, k0, xs, ys, zs, FF, FF0, epsilon, nmax, E0,
                       theta, phi, pp, nquad=0) -> dict:
        """Wide near field (cdmlib.f:1967-2492) around a solved object:
        positions xswf/yswf/zswf and the incident, local and macroscopic
        fields (3 per site) on the box enlarged by nxmp, nymp, nzmp layers."""
        nw = (nx + 2 * nxmp) * (ny + 2 * nymp) * (nz + 2 * nzmp)
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        zs = np.ascontiguousarray(zs, np.float64)
        px, py, pz = (np.zeros(nw) for _ in range(3))
        inc, loc, mac = (np.zeros(3 * nw, np.complex128) for _ in range(3))
        e0 = complex(E0)
        ff, ff0, eps = _zc(FF), _zc(FF0), _zc(epsilon)
        self._check(self.lib.ifdda_nearfield_wide(self.h, nx, ny, nz, nxmp, nymp, nzmp, aretecube, k0, nquad,
                                                  len(xs), nmax, _p(xs), _p(ys), _p(zs), _p(ff), _p(ff0), _p(eps),
                                                  DComplex(e0.real, e0.imag), theta, phi, pp, _p(px), _p(py),
                                                  _p(pz), _p(inc), _p(loc), _p(mac)))
        return dict(xswf=px, yswf=py, zswf=pz, incident=inc, local=loc, macro=mac)

    def planewaves_device(self, nbsphere, xs_ptr, ys_ptr, zs_ptr, k0, E0, beam, a1, a2, pp, out_ptr):
        """planewaves with device positions and a device result (pointers,
        e.g. torch data_ptr()); beam, a1, a2, pp are host sequences."""
        beam = np.ascontiguousarray(np.atleast_1d(beam), np.int32)
        a1 = np.ascontiguousarray(np.atleast_1d(a1), np.float64)
        a2 = np.ascontiguousarray(np.atleast_1d(a2), np.float64)
        pp = np.ascontiguousarray(np.atleast_1d(pp), np.float64)
        e0 = complex(E0)
        self._check(self.lib.ifdda_incident_planewaves_device(
            self.h, int(nbsphere), C.c_void_p(xs_ptr), C.c_void_p(ys_ptr), C.c_void_p(zs_ptr), k0,
            DComplex(e0.real, e0.imag), len(beam), _p(beam), _p(a1), _p(a2), _p(pp), C.c_void_p(out_ptr)))

    def inverserig_ragged_device(self, items, methodeit="GPBICG1", tol=1e-4, precision=IFDDA_FP64, maxit=0):
        """Ragged batch on device pointers: items = [(green, nbsphere, nmax,
        tabdip_ptr or None, polarisa_ptr, FF0_ptr, FF_ptr, FFloc_ptr, nrhs)].
        Returns (tol1, nloop, ncompte, nstop, infostr), counters per
        right-hand side in item order."""
        n = len(items)
        arr = lambda t, vals: (t * n)(*vals)
        greens = arr(C.c_void_p, [it[0].h for it in items])
        nbs = arr(C.c_int, [int(it[1]) for it in items])
        nmaxs = arr(C.c_int, [int(it[2]) for it in items])
        tabs = arr(C.c_void_p, [it[3] for it in items])
        pols = arr(C.c_void_p, [it[4] for it in items])
        p_ff0 = arr(C.c_void_p, [it[5] for it in items])
        p_ff = arr(C.c_void_p, [it[6] for it in items])
        p_loc = arr(C.c_void_p, [it[7] for it in items])
        nrhs = arr(C.c_int, [int(it[8]) for it in items])
        R = sum(int(it[8]) for it in items)
        tol1 = np.zeros(R)
        nloop = np.zeros(R, np.int32)
        ncompte = np.zeros(R, np.int32)
        nstop = C.c_int(0)
        info = C.create_string_buffer(b" " * 64, 65)
        opt = SolveOptions(precision, 0, 0, 0.0, maxit)
        rc = self.lib.ifdda_inverserig_ragged_device(n, greens, nrhs, nbs, nmaxs, tabs, pols, p_ff0,
                                                     methodeit.encode(), float(tol), p_ff, p_loc, _p(tol1),
                                                     _p(nloop), _p(ncompte), C.byref(nstop), info, C.byref(opt))
        infostr = info.raw[:64].decode(errors="replace")
        if rc == 1 and nstop.value == 0:
            raise IfddaError(self.last_error() or infostr.strip())
        return tol1, nloop, ncompte, nstop.value, infostr

    def planewaves(self, xs, ys, zs, k0, E0, beam, a1, a2, pp) -> np.ndarray:
        """FF0 for a batch of plane waves: beam 0 = ondeplane(theta, phi deg),
        1 = ondeplanekxky(kx, ky).  Returns (nrhs, 3*nbsphere)."""
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        zs = np.ascontiguousarray(zs, np.float64)
        beam = np.ascontiguousarray(np.atleast_1d(beam), np.int32)
        a1 = np.ascontiguousarray(np.atleast_1d(a1), np.float64)
        a2 = np.ascontiguousarray(np.atleast_1d(a2), np.float64)
        pp = np.ascontiguousarray(np.atleast_1d(pp), np.float64)
        nrhs = len(beam)
        out = np.zeros((nrhs, 3 * len(xs)), np.complex128)
        e0 = complex(E0)
        self._check(self.lib.ifdda_incident_planewaves(self.h, len(xs), _p(xs), _p(ys), _p(zs), k0,
                                                       DComplex(e0.real, e0.imag), nrhs, _p(beam), _p(a1),
                                                       _p(a2), _p(pp), _p(out)))
        return out


class GreenSpectrum:
    """Device-resident Green spectrum of one lattice (greencalculfft) plus the
    solver workspace that uses it."""

    def __init__(self, ctx: Context, nx, ny, nz, aretecube, k0, nquad=0, box=None):
        self.ctx = ctx
        self.lib = ctx.lib
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.aretecube, self.k0 = float(aretecube), float(k0)
        self.nquad = int(nquad)
        h = C.c_void_p()
        if box is not None:
            bx, by, bz = (int(v) for v in box)
            rc = self.lib.ifdda_green_create_box(ctx.h, self.nx, self.ny, self.nz, bx, by, bz, self.aretecube,
                                                 self.k0, C.byref(h))
        else:
            rc = self.lib.ifdda_green_create_nquad(ctx.h, self.nx, self.ny, self.nz, self.aretecube, self.k0,
                                                   self.nquad, C.byref(h))
        if rc != 0:
            raise IfddaError(ctx.last_error() or "ifdda_green_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ifdda_green_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def recompute(self, aretecube, k0):
        """Recompute the spectrum in place for another spacing / wavenumber
        (greencalculfft called again into the same FFTTENSOR arrays)."""
        self.ctx._check(self.lib.ifdda_green_recompute(self.h, float(aretecube), float(k0)))
        self.aretecube, self.k0 = float(aretecube), float(k0)

    def tiles(self, precision):
        """The tile chooser's (zconv shape, y-pass shape, times ms) for this
        grid and precision; shapes are -1 before the first mat-vec."""
        zv, yv = C.c_int(0), C.c_int(0)
        t = (C.c_float * 4)()
        self.ctx._check(self.lib.ifdda_green_tiles(self.h, precision, C.byref(zv), C.byref(yv), t))
        return zv.value, yv.value, list(t)

    def set_tiles(self, precision, zconv_variant, ypass_variant):
        self.ctx._check(self.lib.ifdda_green_set_tiles(self.h, precision, zconv_variant, ypass_variant))

    def release_workspace(self):
        """Free the solver / mat-vec workspaces; the spectrum stays."""
        self.ctx._check(self.lib.ifdda_green_release_workspace(self.h))

    @property
    def ntotal(self):
        return 8 * self.nx * self.ny * self.nz

    def export(self) -> np.ndarray:
        """The six FFTTENSOR arrays, shape (6, 2nz, 2ny, 2nx)."""
        M = self.ntotal
        out = np.zeros((6, M), np.complex128)
        self.ctx._check(self.lib.ifdda_green_export(self.h, *[_p(out[c]) for c in range(6)]))
        return out.reshape(6, 2 * self.nz, 2 * self.ny, 2 * self.nx)

    def matvec(self, FFX, FFB, tabdip=None, precision=IFDDA_FP64) -> np.ndarray:
        """FFB - (1/ntotal) IFFT(G~ FFT(pad FFX)): produitfftmatvectopt (tabdip
        None) or produitfftmatvect3.  Returns the new FFB."""
        x = _zc(FFX)
        b = _zc(FFB).copy()
        nd = len(x) // 3
        tab = None if tabdip is None else np.ascontiguousarray(tabdip, np.int32)
        self.ctx._check(self.lib.ifdda_matvec(self.h, precision, nd, _p(tab) if tab is not None else None, _p(x),
                                              _p(b)))
        return b

    def matvec_device(self, nrhs, ndip, FFX_ptr, FFB_ptr, tabdip_ptr=None, precision=IFDDA_FP64):
        """In-place FFB -= conv(FFX) on device pointers (asynchronous on the
        context's stream)."""
        self.ctx._check(self.lib.ifdda_matvec_device(self.h, precision, nrhs, ndip,
                                                     C.c_void_p(tabdip_ptr) if tabdip_ptr else None,
                                                     C.c_void_p(FFX_ptr), C.c_void_p(FFB_ptr)))

    def inverserig(self, nbsphere, polarisa, nmax, FF0, methodeit="GPBICG1", tol=1e-4, tabdip=None,
                   precision=IFDDA_FP64, check_every=0, max_outer=0, inner_floor=0.0, nstop_in=0,
                   maxit=0, out=None) -> SolveResult:
        """Rigorous solve (inverserig / inverserigopt) for one or a batch of
        right-hand sides.  FF0: (3*nbsphere,) or (nrhs, 3*nbsphere).

        out: optional (FF, FFloc) pair of C-contiguous complex128 arrays of
        FF0's shape that receive the fields (e.g. pinned buffers reused from
        call to call, like the reference's own FF / FFloc arrays); new arrays
        are allocated otherwise."""
        ff0 = _zc(FF0)
        single = ff0.ndim == 1
        ff0 = ff0.reshape(-1, 3 * nbsphere)
        nrhs = ff0.shape[0]
        pol = _zc(polarisa)
        if out is None:
            FF = np.zeros_like(ff0)
            FFloc = np.zeros_like(ff0)
        else:
            FF, FFloc = out
            for a in (FF, FFloc):
                if a.dtype != np.complex128 or not a.flags.c_contiguous or a.size != ff0.size:
                    raise ValueError("out arrays must be C-contiguous complex128 of FF0's size")
            FF = FF.reshape(ff0.shape)
            FFloc = FFloc.reshape(ff0.shape)
        tol1 = np.zeros(nrhs)
        nloop = np.zeros(nrhs, np.int32)
        ncompte = np.zeros(nrhs, np.int32)
        nstop = C.c_int(nstop_in)
        info = C.create_string_buffer(b" " * 64, 65)
        opt = SolveOptions(precision, check_every, max_outer, inner_floor, maxit)
        tab = None if tabdip is None else np.ascontiguousarray(tabdip, np.int32)
        self.lib.ifdda_inverserig_batch(self.h, nrhs, nbsphere, nmax, _p(tab) if tab is not None else None,
                                        _p(pol), _p(ff0), methodeit.encode(), tol, _p(FF), _p(FFloc), _p(tol1),
                                        _p(nloop), _p(ncompte), C.byref(nstop), info, C.byref(opt))
        r = SolveResult(FF=FF[0] if single else FF, FFloc=FFloc[0] if single else FFloc, tol1=tol1, nloop=nloop,
                        ncompte=ncompte, nstop=nstop.value, infostr=info.raw[:64].decode(errors="replace"))
        return r

    def microscope(self, xs, ys, zs, polarisa, methodeit="GPBICG1", tol=1e-4, ntypemic=1, nfft2d=128, numaper=0.9,
                   numaperinc=0.5, gross=100.0, zlens=0.0, P0=1.0, w0=1e-6, batch=0, precision=IFDDA_FP64, nside=0,
                   nquicklens=1, tabdip=None):
        """Bright-field (ntypemic 1, microsbf) or dark-field / phase
        (ntypemic 2, microsdf) microscope in transmission with the FFT lens,
        on the full box of this spectrum (nquicklens 1, the FFT lens) or on any
        object (nquicklens 0, the lens's far field by direct summation;
        tabdip for inside-only dipoles).  zlens and w0 in metres; nside 0
        transmission, 1 reflection (no image with the incident wave).  Returns a
        MicroscopeResult: image (6, n, n) = |E| of the x, y, z image fields
        and of the same with the incident wave (row v, column u), xy, kxy,
        kxinc / kyinc (units of k0), the last solve's counters, nstop, infostr."""
        n = int(nfft2d)
        xs = np.ascontiguousarray(xs, np.float64)
        ys = np.ascontiguousarray(ys, np.float64)
        zs = np.ascontiguousarray(zs, np.float64)
        tab = None if tabdip is None else np.ascontiguousarray(tabdip, np.int32)
        pol = _zc(polarisa)
        img = np.zeros((6, n, n), np.float64)
        xy = np.zeros(n)
        kxy = np.zeros(n)
        cap = 4 * (n + 8) ** 2
        kxi = np.zeros(cap)
        kyi = np.zeros(cap)
        ninc = C.c_int(cap)
        tol1 = C.c_double(0)
        nloop, ncompte, nstop = C.c_int(0), C.c_int(0), C.c_int(0)
        info = C.create_string_buffer(b" " * 64, 65)
        mo = MicroscopeOptions(int(ntypemic), n, float(numaper), float(numaperinc), float(gross), float(zlens),
                               float(P0), float(w0), int(batch), int(nside), int(nquicklens))
        opt = SolveOptions(precision, 0, 0, 0.0, 0)
        self.lib.ifdda_microscope(self.h, len(xs), _p(tab) if tab is not None else None, _p(xs), _p(ys), _p(zs),
                                  _p(pol), methodeit.encode(), tol, C.byref(mo),
                                  _p(img), _p(xy), _p(kxy), C.byref(ninc), _p(kxi), _p(kyi), C.byref(tol1),
                                  C.byref(nloop), C.byref(ncompte), C.byref(nstop), info, C.byref(opt))
        m = min(ninc.value, cap)
        return MicroscopeResult(image=img, xy=xy, kxy=kxy, kxinc=kxi[:m].copy(), kyinc=kyi[:m].copy(),
                                tol1=tol1.value, nloop=nloop.value, ncompte=ncompte.value, nstop=nstop.value,
                                infostr=info.raw[:64].decode(errors="replace"))

    def inverserig_device(self, nrhs, nbsphere, nmax, tabdip_ptr, polarisa_ptr, FF0_ptr, FF_ptr, FFloc_ptr,
                          methodeit="GPBICG1", tol=1e-4, precision=IFDDA_FP64, check_every=0, max_outer=0,
                          inner_floor=0.0, maxit=0):
        """Batched solve on device pointers (ints, e.g. torch data_ptr())."""
        tol1 = np.zeros(nrhs)
        nloop = np.zeros(nrhs, np.int32)
        ncompte = np.zeros(nrhs, np.int32)
        nstop = C.c_int(0)
        info = C.create_string_buffer(b" " * 64, 65)
        opt = SolveOptions(precision, check_every, max_outer, inner_floor, maxit)
        self.lib.ifdda_inverserig_batch_device(self.h, nrhs, nbsphere, nmax, C.c_void_p(tabdip_ptr or 0) if tabdip_ptr else None,
                                               C.c_void_p(polarisa_ptr), C.c_void_p(FF0_ptr), methodeit.encode(),
                                               tol, C.c_void_p(FF_ptr), C.c_void_p(FFloc_ptr), _p(tol1), _p(nloop),
                                               _p(ncompte), C.byref(nstop), info, C.byref(opt))
        return dict(tol1=tol1, nloop=nloop, ncompte=ncompte, nstop=nstop.value,
                    infostr=info.raw[:64].decode(errors="replace"))
