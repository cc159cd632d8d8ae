"""Host-side object set-up: lattice, Tabdip, polarisability, permittivity.

One-time host work that cdmlib does before the solve (cdmlib/cdmlib.f:661-805),
restated with numpy so the GPU path gets its inputs without the oracle:
  poladiff          cdmlib/polarisabilite.f:1-62
  polaepstens       cdmlib/polaepstens.f:1-122 (anisotropic permittivity tensor)
  sphere            cdmlib/objectsphere.f:94-195          (na = -1 or 0; trope 'ani')
  cube              cdmlib/objectcube.f:60-130            (trope 'ani')
  inhomocuboid      cdmlib/objectparainhomonxnynz.f:85-237 (+ SUNIF, cdmlib/random.f:19-56)
  concentric        cdmlib/objectsphereconcentric.f:76-230 (trope 'ani': a tensor per shell)
  arbitrary         cdmlib/objectarbitrary.f:81-157 (arrays instead of a file;
                    trope 'ani': a tensor per dipole)
All lengths are in metres (the reference multiplies its nm inputs by 1e-9).
A DipoleObject carries the reference's arrays: xs, ys, zs (nbsphere),
tabdip (nx*ny*nz, 1-based, 0 = empty), polarisa and epsilon as (nmax,3,3)
column-major flattened, plus ``alpha`` and ``eps`` (one isotropic value per
dipole) or, for an anisotropic object, ``alpha_t`` and ``eps_t`` (the 3x3
tensors every dipole of the object shares, or one per dipole).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class DipoleObject:
    nx: int
    ny: int
    nz: int
    aretecube: float
    nbsphere: int
    ndipole: int
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    tabdip: np.ndarray
    alpha: np.ndarray   # isotropic polarisability per dipole
    eps: np.ndarray     # isotropic permittivity per dipole
    inside_only: bool
    # anisotropic object: the 3x3 polarisability / permittivity (row a, column
    # b) shared by all its dipoles, or one per dipole (nbsphere, 3, 3)
    alpha_t: np.ndarray = None
    eps_t: np.ndarray = None
    # full box with an anisotropic object: which sites hold a dipole of it
    occupied: np.ndarray = None

    @property
    def nmax(self) -> int:
        return self.nx * self.ny * self.nz

    def _tensor(self, diag: np.ndarray, full: np.ndarray = None, vacuum: complex = 0.0) -> np.ndarray:
        n = self.nmax
        t = np.zeros((3, 3, n), np.complex128)
        if full is None:
            for a in range(3):
                t[a, a, : self.nbsphere] = diag
        else:
            on = np.ones(self.nbsphere, bool) if self.occupied is None else self.occupied
            for a in range(3):
                for b in range(3):
                    v = full[:, a, b] if full.ndim == 3 else full[a, b]
                    t[a, b, : self.nbsphere] = np.where(on, v, vacuum if a == b else 0.0)
        # (nmax,3,3) column-major: (n,a,b) at n + nmax*(a + 3b)  ->  t[b, a, n]
        return np.ascontiguousarray(t.transpose(1, 0, 2)).reshape(-1)

    @property
    def polarisa(self) -> np.ndarray:
        return self._tensor(self.alpha, self.alpha_t, 0.0)

    @property
    def epsilon(self) -> np.ndarray:
        return self._tensor(self.eps, self.eps_t, 1.0)

    @property
    def tabdip_or_none(self):
        """tabdip for the inside-only path (inverserig), None for the full box."""
        return self.tabdip if self.inside_only else None


def poladiff(aretecube: float, eps, k0: float, methode: str, eps0: float = 1.0, dddis: int = 1) -> np.ndarray:
    """Per-dipole polarisability (polarisabilite.f:1-62), vectorised over eps."""
    eps = np.asarray(eps, np.complex128)
    pi = math.acos(-1.0)
    rapport = (eps - eps0) / (eps + 2.0 * eps0)
    indice = math.sqrt(eps0)
    k03 = k0 ** 3 * indice ** 3
    rayon = aretecube
    maille = 0.0
    if dddis == 0:
        volume = rayon ** 3
    elif dddis == 1:
        maille = rayon
        rayon = rayon * (0.75 / pi) ** (1.0 / 3.0)
        volume = rayon * rayon * rayon
    else:
        raise ValueError("dddis must be 0 or 1")
    pola = rapport * volume
    m = methode[:2]
    if m == "CM":
        return pola * eps0
    if m in ("RR", "PS"):
        return eps0 * pola / (1.0 - 2.0 / 3.0 * 1j * k03 * pola)
    if m == "GB":
        return pola / (1.0 - 2.0 / 3.0 * 1j * k03 * pola - k0 * k0 * pola * indice * indice / rayon)
    if m == "LA":
        return pola / (1.0 - 2.0 * rapport * ((1.0 - 1j * k0 * indice * rayon) * np.exp(1j * k0 * indice * rayon) - 1.0))
    if m == "LR":
        sldr = 1.0 / 5.0
        return eps0 * pola / (1.0 + pola * ((-1.8915316 + eps / eps0 * 0.1648469 - eps / eps0 * 1.7700004 * sldr)
                                            * k0 * k0 * indice * indice / maille
                                            - 2.0 / 3.0 * 1j * k03 * indice ** 3))
    raise ValueError(f"incorrect method {methode!r}")


def polaepstens(aretecube: float, epsani, k0: float, methode: str, eps0: float = 1.0, dis: int = 1,
                inv: int = 1) -> np.ndarray:
    """Polarisability tensor of a cube of anisotropic permittivity epsani (3x3)
    (polaepstens.f:1-122): alpha0 = V (eps - eps0 I) (eps + 2 eps0 I)^-1,
    CM: alpha0 eps0, RR: (I - 2/3 i k^3 alpha0)^-1 alpha0 eps0; inv = -1
    returns the inverse.  Only CM and RR exist for a tensor.  epsani may
    also be a stack (..., 3, 3), one tensor per dipole."""
    e = np.asarray(epsani, np.complex128)
    e = e.reshape(3, 3) if e.size == 9 else e.reshape(-1, 3, 3)
    pi = math.acos(-1.0)
    k03 = k0 ** 3 * math.sqrt(eps0) ** 3
    if dis == 0:
        volume = aretecube ** 3
    elif dis == 1:
        volume = (aretecube * (0.75 / pi) ** (1.0 / 3.0)) ** 3
    else:
        raise ValueError("Bad value of dis")
    eye = np.eye(3)
    a0 = (e - eps0 * eye) @ np.linalg.inv(e + 2.0 * eps0 * eye) * volume
    m = methode[:2]
    if m == "CM":
        a = a0 * eps0
    elif m == "RR":
        a = np.linalg.inv(eye - 2.0 / 3.0 * 1j * k03 * a0) @ a0 * eps0
    else:
        raise ValueError(f"incorrect method for the polarizability {methode!r}")
    return np.linalg.inv(a) if inv == -1 else a


def _lattice(n1, n2, n3):
    k, j, i = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
    return i.ravel(), j.ravel(), k.ravel()


def _finish_ani(nx, ny, nz, d, x, y, z, keep, epsani, k0, methode, inside_only) -> DipoleObject:
    """Anisotropic object (trope = 'ani'): every dipole gets polaepstens of
    its permittivity with dis = 1 (objectsphere.f:129-135); 'PS' is refused
    there.  epsani: one 3x3 tensor for the object, or one per lattice site
    (nx*ny*nz, 3, 3)."""
    if methode[:2] == "PS":
        raise ValueError("anisotrope with PS")
    e = np.asarray(epsani, np.complex128)
    N = nx * ny * nz
    if e.size != 9:
        e = e.reshape(N, 3, 3)
        if inside_only:
            tab = np.zeros(N, np.int32)
            idx = np.nonzero(keep)[0]
            tab[idx] = np.arange(1, len(idx) + 1, dtype=np.int32)
            es = e[idx].copy()
            at = polaepstens(d, es, k0, methode, dis=1)
            return DipoleObject(nx, ny, nz, d, len(idx), N, x[idx].copy(), y[idx].copy(), z[idx].copy(), tab,
                                at[:, 0, 0].copy(), es[:, 0, 0].copy(), True, at, es)
        es = np.where(keep[:, None, None], e, np.eye(3))
        at = polaepstens(d, es, k0, methode, dis=1)
        tab = np.arange(1, N + 1, dtype=np.int32)
        return DipoleObject(nx, ny, nz, d, N, N, x.copy(), y.copy(), z.copy(), tab,
                            np.where(keep, at[:, 0, 0], 0.0), np.where(keep, es[:, 0, 0], 1.0 + 0j), False, at, es,
                            keep.copy())
    e = e.reshape(3, 3)
    at = polaepstens(d, e, k0, methode, dis=1)
    if inside_only:
        tab = np.zeros(N, np.int32)
        idx = np.nonzero(keep)[0]
        tab[idx] = np.arange(1, len(idx) + 1, dtype=np.int32)
        nb = len(idx)
        return DipoleObject(nx, ny, nz, d, nb, N, x[idx].copy(), y[idx].copy(), z[idx].copy(), tab,
                            np.full(nb, at[0, 0]), np.full(nb, e[0, 0]), True, at, e)
    tab = np.arange(1, N + 1, dtype=np.int32)
    return DipoleObject(nx, ny, nz, d, N, N, x.copy(), y.copy(), z.copy(), tab, np.where(keep, at[0, 0], 0.0),
                        np.where(keep, e[0, 0], 1.0 + 0j), False, at, e, keep.copy())


def _finish(nx, ny, nz, d, x, y, z, keep, eps_site, k0, methode, inside_only) -> DipoleObject:
    """keep: per lattice site, True for a dipole with permittivity eps_site."""
    N = nx * ny * nz
    eps_site = np.broadcast_to(np.asarray(eps_site, np.complex128), (N,))
    alpha_site = poladiff(d, eps_site, k0, methode)
    if inside_only:
        tab = np.zeros(N, np.int32)
        idx = np.nonzero(keep)[0]
        tab[idx] = np.arange(1, len(idx) + 1, dtype=np.int32)
        return DipoleObject(nx, ny, nz, d, len(idx), N, x[idx].copy(), y[idx].copy(), z[idx].copy(), tab,
                            alpha_site[idx].copy(), eps_site[idx].copy(), True)
    tab = np.arange(1, N + 1, dtype=np.int32)
    alpha = np.where(keep, alpha_site, 0.0).astype(np.complex128)
    eps = np.where(keep, eps_site, 1.0 + 0j).astype(np.complex128)
    return DipoleObject(nx, ny, nz, d, N, N, x.copy(), y.copy(), z.copy(), tab, alpha, eps, False)


def sphere(rayon, eps, nnnr, k0, methode="RR", na=-1, epsani=None) -> DipoleObject:
    """objetsphere: d = 2R/nnnr, dipole where |r| < R (objectsphere.f:94-113);
    epsani (3x3) makes it anisotropic (trope = 'ani')."""
    if rayon == 0.0:
        raise ValueError("object sphere: radius=0!")
    d = 2.0 * rayon / nnnr
    i, j, k = _lattice(nnnr, nnnr, nnnr)
    x = -rayon + d * (i + 1 - 0.5)
    y = -rayon + d * (j + 1 - 0.5)
    z = -rayon + d * (k + 1 - 0.5)
    keep = np.sqrt(x * x + y * y + z * z) < rayon
    if epsani is not None:
        return _finish_ani(nnnr, nnnr, nnnr, d, x, y, z, keep, epsani, k0, methode, na == -1)
    return _finish(nnnr, nnnr, nnnr, d, x, y, z, keep, eps, k0, methode, na == -1)


def cube(side, eps, nnnr, k0, methode="RR", epsani=None) -> DipoleObject:
    """objetcube: full box, d = side/nnnr (objectcube.f:91-117); epsani (3x3)
    makes it anisotropic."""
    if side == 0.0:
        raise ValueError("object cube: side=0!")
    d = side / nnnr
    xc = (side + d) / 2.0
    i, j, k = _lattice(nnnr, nnnr, nnnr)
    x = (i + 1) * d - xc
    y = (j + 1) * d - xc
    z = (k + 1) * d - xc
    keep = np.ones(nnnr ** 3, bool)
    if epsani is not None:
        return _finish_ani(nnnr, nnnr, nnnr, d, x, y, z, keep, epsani, k0, methode, False)
    return _finish(nnnr, nnnr, nnnr, d, x, y, z, keep, eps, k0, methode, False)


def sunif_sequence(ir: int, n: int) -> np.ndarray:
    """SUNIF (random.f:19-56): R <- frac(R * 41475557), R0 = float(IR)/2^28,
    each value rounded to single precision."""
    factor, two28 = 41475557.0, 268435456.0
    out = np.empty(n)
    r = float(np.float32(ir)) / two28
    for q in range(n):
        r = math.fmod(r * factor, 1.0)
        out[q] = float(np.float32(r))
    return out


def inhomocuboid(nx, ny, nz, d, eps, lc, hc, ng, k0, methode="RR") -> DipoleObject:
    """objetparainhomonxnynz: Gaussian random field of std hc and correlation
    length lc by spectral synthesis (objectparainhomonxnynz.f:146-197)."""
    if lc <= 0.0:
        raise ValueError("coherence length equal to zero")
    if hc <= 0.0:
        raise ValueError("standard deviation equal to zero")
    pi = math.acos(-1.0)
    N = nx * ny * nz
    dkx, dky, dkz = 2 * pi / (nx * d), 2 * pi / (ny * d), 2 * pi / (nz * d)
    coeff1 = 0.125 * hc * hc * lc ** 3 / (pi * math.sqrt(pi))
    coeff2 = lc * lc
    coeff3 = 4.0 * dkx * dky * dkz
    i, j, k = _lattice(nx, ny, nz)  # i fastest (k in the reference loop), 0-based
    kx = np.where(i + 1 <= nx // 2 + 1, i, i - nx) * dkx
    ky = np.where(j + 1 <= ny // 2 + 1, j, j - ny) * dky
    kz = np.where(k + 1 <= nz // 2 + 1, k, k - nz) * dkz
    spec = coeff1 * np.exp(-0.25 * coeff2 * (kx * kx + ky * ky + kz * kz))
    phase = 2.0 * pi * sunif_sequence(4 * ng + 1, N)
    v = np.sqrt(spec * coeff3) * np.exp(1j * phase)
    nk = np.arange(1, N + 1)
    zero = (nk == 1) | ((nk >= nx // 2 + 2) & (nk <= nx)) | ((nk >= (ny // 2 + 1) * nx + 1) & (nk <= nx * ny)) | \
        ((nk >= (nz // 2 + 1) * nx * ny + 1) & (nk <= N))
    v[zero] = 0.0
    # fftsingletonz3d(+1): unnormalised exp(+i) transform
    f = np.fft.ifftn(v.reshape(nz, ny, nx)) * N
    eps_site = f.real.ravel() + complex(eps)
    sx, sy, sz = d * nx, d * ny, d * nz
    x = -sx / 2 + d * (i + 0.5)
    y = -sy / 2 + d * (j + 0.5)
    z = -sz / 2 + d * (k + 0.5)
    return _finish(nx, ny, nz, d, x, y, z, np.ones(N, bool), eps_site, k0, methode, False)


def concentric(rayons, epss, nnnr, k0, methode="RR", na=-1, epsanis=None) -> DipoleObject:
    """objetsphereconcentric: d = 2 r_out / nnnr; shell l holds r in
    [r_{l-1}, r_l] (objectsphereconcentric.f:112-167); epsanis (one 3x3 per
    shell) makes it anisotropic (trope = 'ani', objectsphereconcentric.f:
    128-146)."""
    rayons = list(rayons)
    if rayons[0] == 0.0:
        raise ValueError("spheres concentrics: 1st rayon=0")
    for a, b in zip(rayons, rayons[1:]):
        if b - a <= 0:
            raise ValueError("spheres concentrics: rayons non croissants")
    ns = len(rayons)
    d = 2.0 * rayons[-1] / nnnr
    centre = d * nnnr / 2.0
    i, j, k = _lattice(nnnr, nnnr, nnnr)
    x = i * d + d / 2 - centre
    y = j * d + d / 2 - centre
    z = k * d + d / 2 - centre
    ray = np.sqrt(x * x + y * y + z * z)
    shell = np.zeros(len(ray), np.int64)
    shell[ray <= rayons[0]] = 1
    for l in range(2, ns + 1):
        sel = (ray > rayons[0]) & (ray <= rayons[l - 1]) & (ray >= rayons[l - 2])
        shell[sel] = l
    keep = shell > 0
    if epsanis is not None:
        ea = np.asarray(epsanis, np.complex128).reshape(ns, 3, 3)
        e_site = np.where(keep[:, None, None], ea[np.maximum(shell - 1, 0)], np.eye(3))
        return _finish_ani(nnnr, nnnr, nnnr, d, x, y, z, keep, e_site, k0, methode, na == -1)
    epss = np.asarray(epss, np.complex128)
    eps_site = np.where(keep, epss[np.maximum(shell - 1, 0)], 1.0)
    return _finish(nnnr, nnnr, nnnr, d, x, y, z, keep, eps_site, k0, methode, na == -1)


def arbitrary(nx, ny, nz, d, x, y, z, eps_site, k0, methode="RR", epsani_site=None) -> DipoleObject:
    """objetarbitrary without the file: every lattice site is a dipole of its
    own isotropic permittivity (vacuum sites have eps = 1, alpha = 0), or of
    its own 3x3 tensor epsani_site (nx*ny*nz, 3, 3) (trope = 'ani',
    objectarbitrary.f:130-151)."""
    N = nx * ny * nz
    if epsani_site is not None:
        return _finish_ani(nx, ny, nz, d, np.asarray(x, float), np.asarray(y, float), np.asarray(z, float),
                           np.ones(N, bool), np.asarray(epsani_site, np.complex128).reshape(N, 3, 3), k0, methode,
                           False)
    eps_site = np.asarray(eps_site, np.complex128).reshape(N)
    return _finish(nx, ny, nz, d, np.asarray(x, float), np.asarray(y, float), np.asarray(z, float),
                   np.ones(N, bool), eps_site, k0, methode, False)


def ellipsoid_lattice(nx, ny, nz, d, a, b, c, eps_lo, eps_hi, seed, k0, methode="RR") -> DipoleObject:
    """Inhomogeneous ellipsoid (semi-axes a, b, c) centred in an explicit
    nx*ny*nz lattice of spacing d, eps uniform in [eps_lo, eps_hi] per dipole
    inside (numpy Generator(seed)), vacuum outside, built as an arbitrary
    object (full box)."""
    i, j, k = _lattice(nx, ny, nz)
    x = (i + 0.5) * d - nx * d / 2
    y = (j + 0.5) * d - ny * d / 2
    z = (k + 0.5) * d - nz * d / 2
    inside = (x / a) ** 2 + (y / b) ** 2 + (z / c) ** 2 <= 1.0
    rng = np.random.Generator(np.random.PCG64(seed))
    e = rng.uniform(eps_lo, eps_hi, size=nx * ny * nz)
    eps_site = np.where(inside, e, 1.0).astype(np.complex128)
    return arbitrary(nx, ny, nz, d, x, y, z, eps_site, k0, methode)


def irradiance(P0: float, w0: float):
    """E0 and irradiance of a plane wave of power P0 over a waist w0 (irradiance.f:6-20)."""
    pi = math.acos(-1.0)
    c = 299792458.0
    eps0 = 1.0 / (c * c * 4.0 * pi * 1e-7)
    irra = P0 / (w0 * w0 * pi)
    return math.sqrt(2.0 * irra / c / eps0), irra
