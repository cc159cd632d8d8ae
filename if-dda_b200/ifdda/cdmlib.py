"""cdmlib -- host-side mirror of the reference's entry point for the rigorous
solve (cdmlib/cdmlib.f:3-60, C prototype cdmlib/cdmlib.h:5-71), on the GPU.

It takes the reference's option names and units (lengths in nm, angles in
degrees, eps as complex), runs the same sequence as cdmlib.f --
validation (:317-471), object (:661-805), padded grid (:1141-1148), incident
field (:1172-1187), Green spectrum (:1518-1546), solve (:1555-1597), local and
macroscopic fields (:2497-2655), cross sections (:2717-2778) -- and returns
the reference's outputs in a dict together with nstop/infostr.  Only the
options on the rigorous-solve path are implemented (trope 'iso' for every
object here, trope 'ani' for the sphere, the cube (epsani), the concentric
spheres (epsanis, one tensor per shell) and the arbitrary object (epsani_site,
one per dipole), plane waves, nrig = 0,
0 <= nquad <= 16), and the bright-field and dark-field microscopes in
transmission or reflection with or without the FFT lens (nlentille = 1,
ntypemic 1 or 2, nside 0 or 1, nquicklens 0 or 1, cdmlib.f:3660-3800), the
holographic microscope (ntypemic 0, cdmlib.f:3803-4660), the wide near field (nproche >= 2) and
the scattering cross section / asymmetry factor / Poynting vector
(nsectionsca = 1, by direct summation or, with nquickdiffracte = 1, from the
far field on the nfft2d pupil grid); anything else returns nstop = 1 with a
message.
"""
from __future__ import annotations

import math

import numpy as np

from . import objects
from .api import Context, IfddaError

_SUPPORTED_OBJECTS = ("sphere", "cube", "inhomocuboid2", "concentricsphere", "arbitrary")


def _fail(msg, **extra):
    d = dict(nstop=1, infostr=msg)
    d.update(extra)
    return d


def cdmlib(*, wavelength, object, eps=None, nnnr=None, rayon=None, side=None, rayons=None, epss=None,
           nx=None, ny=None, nz=None, aretecube=None, epsani=None, epsanis=None, epsani_site=None, lc=None, hc=None, ng=0, positions=None, eps_site=None,
           beam="pwavelinear", theta=0.0, phi=0.0, pp=1.0, incidences=None, P0=1.0, w0=None,
           tolinit=1e-4, methodeit="GPBICG1", polarizability="RR", trope="iso", nproche=0, nrig=0, nquad=0,
           nlocal=1, nmacro=1, nsection=1, precision=0, nlentille=0, ntypemic=1, nside=0, nquicklens=1,
           nfft2d=128, numaper=0.9, numaperinc=0.5, gross=100.0, zlens=0.0, microscope_batch=0, nxmp=0, nymp=0,
           nzmp=0, nsectionsca=0, nquickdiffracte=0, ntheta=36, nphi=72,
           ctx: Context | None = None, device=0):
    """Rigorous solve of one object for one plane wave (theta, phi, pp) or a
    batch of them (incidences = [(theta, phi, pp), ...]).  nproche follows the
    GUI convention: 0 -> dipoles inside the object only (inverserig), 1 ->
    the full box (inverserigopt), >= 2 -> the full box and the wide near
    field on the box enlarged by nxmp, nymp, nzmp layers (incidentfield_wf,
    localfield_wf, macroscopicfield_wf, xswf, yswf, zswf).  precision: 0 plain FP64, 1 FP32 inner
    iterations with FP64 refinement.  nlentille = 1 adds the microscope's
    images (Eimagex..z, Eimageincx..z as |E| on nfft2d^2 pixels, xy, kxy,
    kxinc/kyinc); zlens in nm."""
    lam = wavelength * 1e-9
    if trope not in ("iso", "ani"):
        return _fail(f"trope {trope!r} is neither 'iso' nor 'ani'")
    if trope == "ani":
        # cdmlib.f:597-611 (the first object's tensor: epsanimulti(:,:,1))
        first = epsani if epsani is not None else (epsanis[0] if epsanis is not None else epsani_site)
        if first is None or float(np.sum(np.abs(np.asarray(first, np.complex128)))) == 0.0:
            return _fail("No relative permittivity given")
        if polarizability not in ("RR", "CM"):
            return _fail("Polarizability should be CM or RR with anisotropy")
        if object not in ("sphere", "cube", "concentricsphere", "arbitrary"):
            return _fail(f"anisotropic {object!r} not handled by the GPU drop-in")
        if object == "concentricsphere" and (epsanis is None or rayons is None or len(epsanis) != len(rayons)):
            return _fail("epsanis: one 3x3 tensor per sphere")
        if object == "arbitrary" and epsani_site is None:
            return _fail("epsani_site: one 3x3 tensor per dipole")
    if nrig != 0:
        return _fail("only the rigorous solve (nrig = 0) is handled by the GPU drop-in")
    if not 0 <= nquad <= 16:
        return _fail("nquad must be in [0, 16]")
    if beam != "pwavelinear":
        return _fail("Cross section only with plane wave" if nsection else "only plane waves are handled")
    if tolinit < 1e-12:
        return _fail("Tolerance for the iterative method too small!")
    if tolinit > 0.5:
        return _fail("Tolerance  for the iterative method too large!")
    if object not in _SUPPORTED_OBJECTS:
        return _fail(f"object {object!r} not handled by the GPU drop-in")
    if nsectionsca:
        # cdmlib.f:394-400
        if abs(theta) >= 45.0:
            return _fail("Angle too strong: Imprecise calculation with FFT")
        if ntheta <= 10 or nphi <= 20:
            return _fail("ntheta and nphi too small!")
    if nquickdiffracte:
        nproche = max(nproche, 1)  # the FFT far field needs the full box (cdmlib.f:630)
    if nlentille:
        # cdmlib.f:365-389
        if not 0.0 < numaper <= 1.0:
            return _fail("Problem with numerical aperture!")
        if abs(gross) < 1.0:
            return _fail("Problem with manification!")
        if abs(theta) >= 90.0:
            return _fail("Illumination on the wrong side with the options")
        if ntypemic not in (0, 1, 2) or nside not in (0, 1) or nquicklens not in (0, 1):
            return _fail("ntypemic 0, 1 or 2, nside 0 or 1, nquicklens 0 or 1")
        if nquicklens:
            nproche = max(nproche, 1)  # the FFT lens needs the full box (cdmlib.f:631)
    if not (nlocal or nmacro or nsection):
        return _fail("No calculation requested!")
    k0 = 2 * math.pi / lam
    inside = nproche - 1 == -1  # cdmlib.f:627 decrements the GUI value
    wide = nproche - 1 >= 1     # cdmlib.f:636-640: nprochefft, solved on the full box
    # ---- object (cdmlib.f:661-805) -------------------------------------
    try:
        ani = epsani if trope == "ani" else None
        e_iso = complex(eps) if eps is not None else 0j
        if object == "sphere":
            ob = objects.sphere(rayon * 1e-9, e_iso, nnnr, k0, polarizability, na=-1 if inside else 0, epsani=ani)
        elif object == "cube":
            ob = objects.cube(side * 1e-9, e_iso, nnnr, k0, polarizability, epsani=ani)
        elif object == "inhomocuboid2":
            ob = objects.inhomocuboid(nx, ny, nz, aretecube * 1e-9, complex(eps), lc * 1e-9, hc, ng, k0,
                                      polarizability)
        elif object == "concentricsphere":
            ob = objects.concentric([r * 1e-9 for r in rayons], epss, nnnr, k0, polarizability,
                                    na=-1 if inside else 0, epsanis=epsanis if trope == "ani" else None)
        else:
            pos = np.asarray(positions, float) * 1e-9
            ob = objects.arbitrary(nx, ny, nz, aretecube * 1e-9, pos[:, 0], pos[:, 1], pos[:, 2],
                                   eps_site if eps_site is not None else np.ones(len(pos)), k0, polarizability,
                                   epsani_site=epsani_site if trope == "ani" else None)
    except ValueError as e:
        return _fail(str(e))
    if ob.nbsphere == 0:
        return _fail("No dipole in the object!")
    # mesh size check (cdmlib.f:994-999); for an anisotropic object the
    # reference tests the scalar eps argument, so none given passes
    if trope == "ani":
        eps_max = abs(np.sqrt(complex(eps))) if eps is not None else 0.0
    else:
        eps_max = np.max(np.abs(np.sqrt(ob.eps))) if len(ob.eps) else 1.0
    if eps_max > 0 and ob.aretecube > 2.5 * lam / 10.0 / eps_max:
        return _fail("Meshsize larger than lambda/4!")
    own = ctx is None
    ctx = ctx or Context(device)
    try:
        # ---- incident field (cdmlib.f:1172-1187, irradiance.f) -----------
        E0, irra = objects.irradiance(P0, (w0 if w0 is not None else 10 * wavelength) * 1e-9)
        inc = incidences if incidences is not None else [(theta, phi, pp)]
        ff0 = ctx.planewaves(ob.xs, ob.ys, ob.zs, k0, E0, [0] * len(inc), [t for t, _, _ in inc],
                             [p for _, p, _ in inc], [q for _, _, q in inc])
        # ---- Green spectrum and solve (cdmlib.f:1518-1597) ---------------
        try:
            g = ctx.green(ob.nx, ob.ny, ob.nz, ob.aretecube, k0, nquad)
        except IfddaError as e:
            return _fail(str(e)[:64])
        r = g.inverserig(ob.nbsphere, ob.polarisa, ob.nmax, ff0 if len(inc) > 1 else ff0[0], methodeit, tolinit,
                         tabdip=ob.tabdip_or_none, precision=precision)
        out = dict(nstop=r.nstop, infostr=r.infostr, nbsphere=ob.nbsphere, ndipole=ob.ndipole,
                   aretecube=ob.aretecube, k0=k0, irra=irra, E0=E0, tol1=r.tol1, nloop=r.nloop,
                   ncompte=r.ncompte, incidentfield=ff0, FF=r.FF, localfield=r.FFloc, xs=ob.xs, ys=ob.ys,
                   zs=ob.zs)
        if r.nstop == 0 and nlentille and ntypemic == 0:
            # ---- holographic microscope (cdmlib.f:4075-4660) ---------------
            FFs = np.atleast_2d(r.FF)
            t, p, s = inc[0]
            h = ctx.holography(ob.nx, ob.ny, ob.nz, ob.aretecube, k0, ob.xs, ob.ys, ob.zs, FFs[0], E0, t, p, s,
                               nfft2d=nfft2d, numaper=numaper, gross=gross, zlens=zlens * 1e-9, nside=nside,
                               nquicklens=nquicklens)
            if h["nstop"] != 0:
                g.close()
                out.update(nstop=h["nstop"], infostr=h["infostr"])
                return out
            for c, name in enumerate(("Eimagex", "Eimagey", "Eimagez", "Eimageincx", "Eimageincy", "Eimageincz")):
                out[name] = h["image"][c]
            for c, name in enumerate(("Efourierx", "Efouriery", "Efourierz", "Efourierincx", "Efourierincy",
                                      "Efourierincz")):
                out[name] = h["fourier"][c]
            out.update(xy=h["xy"], kxy=h["kxy"])
        elif r.nstop == 0 and nlentille:
            # ---- microscope (cdmlib.f:3660-3800) ---------------------------
            m = g.microscope(ob.xs, ob.ys, ob.zs, ob.polarisa, methodeit, tolinit, ntypemic=ntypemic,
                             nfft2d=nfft2d, numaper=numaper, numaperinc=numaperinc, gross=gross,
                             zlens=zlens * 1e-9, P0=P0, w0=(w0 if w0 is not None else 10 * wavelength) * 1e-9,
                             batch=microscope_batch, precision=precision, nside=nside, nquicklens=nquicklens,
                             tabdip=ob.tabdip_or_none)
            if m.nstop != 0:
                g.close()
                out.update(nstop=m.nstop, infostr=m.infostr)
                return out
            for c, name in enumerate(("Eimagex", "Eimagey", "Eimagez", "Eimageincx", "Eimageincy", "Eimageincz")):
                out[name] = m.image[c]
            out.update(xy=m.xy, kxy=m.kxy, kxinc=m.kxinc, kyinc=m.kyinc)
        g.close()
        if r.nstop != 0:
            return out
        FF = np.atleast_2d(r.FF)
        FFloc = np.atleast_2d(r.FFloc)
        if wide:
            # ---- wide near field (cdmlib.f:1967-2492) ----------------------
            wf = [ctx.nearfield_wide(ob.nx, ob.ny, ob.nz, nxmp, nymp, nzmp, ob.aretecube, k0, ob.xs, ob.ys, ob.zs,
                                     FF[q], ff0[q], ob.epsilon, ob.nmax, E0, t, p, s, nquad)
                  for q, (t, p, s) in enumerate(inc)]
            out.update(xswf=wf[0]["xswf"], yswf=wf[0]["yswf"], zswf=wf[0]["zswf"],
                       incidentfield_wf=np.stack([w["incident"] for w in wf]),
                       localfield_wf=np.stack([w["local"] for w in wf]),
                       macroscopicfield_wf=np.stack([w["macro"] for w in wf]))
        # ---- macroscopic field (cdmlib.f:2595-2655) ----------------------
        if nmacro:
            out["macroscopicfield"] = np.stack([ctx.local_macro(ob.nbsphere, ob.nmax, ob.epsilon, FFloc[q],
                                                                ob.aretecube, k0) for q in range(len(inc))])
        # ---- Csca, g and Poynting by direct summation (cdmlib.f:2784-2880)
        if nsectionsca:
            if nquickdiffracte:
                sc = [ctx.farfield_fft(ob.nx, ob.ny, ob.nz, ob.aretecube, ob.xs, ob.ys, ob.zs, FF[q], k0,
                                       abs(E0) ** 2, t, p, nfft2d, ntheta, nphi) for q, (t, p, _) in enumerate(inc)]
            else:
                sc = [ctx.farfield_csca(ob.xs, ob.ys, ob.zs, FF[q], k0, abs(E0) ** 2, t, p, ntheta, nphi)
                      for q, (t, p, _) in enumerate(inc)]
            out.update(Cscai=np.array([s["Cscai"] for s in sc]), gasym=np.array([s["gasym"] for s in sc]),
                       poyntingfield=np.stack([s["poyntingfield"] for s in sc]), thetafield=sc[0]["thetafield"],
                       phifield=sc[0]["phifield"])
        # ---- cross sections (cdmlib.f:2717-2778) -------------------------
        if nsection:
            cs = [ctx.cross_sections(ff0[q], FF[q], FFloc[q], k0, abs(E0) ** 2) for q in range(len(inc))]
            cext = np.array([c[0] for c in cs])
            cabs = np.array([c[1] for c in cs])
            csca = cext - cabs
            cabs = np.where(cabs <= cext * 1e-12, 0.0, cabs)
            out.update(Cext=cext, Cabs=cabs, Csca=csca)
        return out
    finally:
        if own:
            ctx.close()
