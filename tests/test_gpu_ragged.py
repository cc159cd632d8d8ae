"""GPU: ragged batches -- objects of uneven lattices, spacings and wavelengths
solved together (ifdda_inverserig_ragged) on one common box.

Each object's spectrum is made on the common box (ifdda_green_create_box),
its lattice at the corner; the batch runs one launch sequence per iteration
for every right-hand side of every object.  Checks: FP64 right-hand sides
reproduce their solo solve on the same box (same iteration and mat-vec
counts, local field within 1e-9) and the oracle's solve of the object on its
own lattice (same counts, 1e-7); mixed-precision right-hand sides reach the
FP64 true residual and agree with their solo mixed solve to 1e-3; and an
object solved as a ragged batch of its own gives the same bits as inside the
batch (its vectors are laid out on the box, whatever the other objects).
"""
import math

import numpy as np
import pytest

from cases import rel

pytestmark = pytest.mark.gpu

BOX = (16, 16, 16)


def _objects():
    from ifdda import objects
    out = []
    lam = 560e-9
    k0 = 2 * math.pi / lam
    ob = objects.sphere(70e-9, 2.8 + 0.2j, 12, k0, "RR", na=-1)  # inside-only, 12^3 lattice
    out.append((ob, k0, [(0, 0.0, 0.0, 1.0), (0, 30.0, 10.0, 0.0)]))
    lam = 700e-9
    k0 = 2 * math.pi / lam
    ob = objects.cube(150e-9, 1.9 + 0.05j, 16, k0, "RR")  # full box 16^3
    out.append((ob, k0, [(0, 10.0, 0.0, 0.0)]))
    lam = 450e-9
    k0 = 2 * math.pi / lam
    ob = objects.inhomocuboid(10, 14, 8, 9e-9, 2.25 + 0j, 40e-9, 0.1, 5, k0, "RR")  # full box 10x14x8
    out.append((ob, k0, [(0, 0.0, 0.0, 1.0), (0, 20.0, 45.0, 1.0), (0, 50.0, 90.0, 0.0)]))
    return out


def _items(gctx, orc):
    from ifdda import objects
    items, greens, ff0s = [], [], []
    for ob, k0, beams in _objects():
        E0, _ = objects.irradiance(1.0, 10 * 2 * math.pi / k0)
        ff0 = np.stack([orc.incident(ob.xs, ob.ys, ob.zs, k0, E0, pp, bm, a1, a2) for bm, a1, a2, pp in beams])
        g = gctx.green_box(ob.nx, ob.ny, ob.nz, BOX, ob.aretecube, k0)
        greens.append(g)
        ff0s.append(ff0)
        items.append((g, ob.nbsphere, ob.nmax, ob.tabdip_or_none, ob.polarisa, ff0))
    return items, greens, ff0s


@pytest.mark.parametrize("prec", [0, 1])
def test_ragged_batch_matches_solo_solves(gctx, orc, prec):
    items, greens, ff0s = _items(gctx, orc)
    tol = 1e-6 if prec == 0 else 1e-4
    fields, tol1, nloop, ncompte, nstop, info = gctx.inverserig_ragged(items, "GPBICG1", tol, precision=prec)
    assert nstop == 0, info
    r0 = 0
    for (g, nb, nmax, tab, pol, ff0), (FF, FFloc) in zip(items, fields):
        solo = g.inverserig(nb, pol, nmax, ff0, "GPBICG1", tol, tabdip=tab, precision=prec)
        assert solo.nstop == 0
        loc_s = solo.FFloc.reshape(ff0.shape)
        for q in range(ff0.shape[0]):
            assert tol1[r0 + q] < tol
            if prec == 0:
                assert nloop[r0 + q] == int(solo.nloop[q]) and ncompte[r0 + q] == int(solo.ncompte[q])
                assert rel(FFloc[q], loc_s[q]) < 1e-9
            else:
                assert rel(FFloc[q], loc_s[q]) < 1e-3
        # FF = alpha E
        assert rel(FF, np.repeat(pol[:nb], 3)[None, :] * FFloc) < 1e-14
        # alone as a batch of one: bit for bit
        f1, t1, nl1, nc1, ns1, _ = gctx.inverserig_ragged([(g, nb, nmax, tab, pol, ff0)], "GPBICG1", tol,
                                                          precision=prec)
        assert ns1 == 0 and np.array_equal(f1[0][1], FFloc) and np.array_equal(nc1, ncompte[r0:r0 + len(nc1)])
        r0 += ff0.shape[0]
    for g in greens:
        g.close()


def test_ragged_batch_matches_the_oracle(gctx, orc):
    """The sphere (inside-only) and the GRF cuboid of the batch against the
    oracle's inverserig on each object's own 2n grid, FP64."""
    items, greens, ff0s = _items(gctx, orc)
    fields, tol1, nloop, ncompte, nstop, info = gctx.inverserig_ragged(items, "GPBICG1", 1e-6, precision=0)
    assert nstop == 0, info
    starts = np.cumsum([0] + [f.shape[0] for f in ff0s])
    objs = _objects()
    for i in (0, 2):
        ob, k0, _ = objs[i]
        G6 = orc.greencalculfft(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
        for q in range(ff0s[i].shape[0]):
            ref = orc.inverserig(G6, ob.nx, ob.ny, ob.nz, ob.nbsphere, ob.polarisa, ob.nmax, ff0s[i][q], "GPBICG1",
                                 1e-6, tabdip=ob.tabdip_or_none)
            assert ref["nstop"] == 0
            assert ncompte[starts[i] + q] == ref["ncompte"] and nloop[starts[i] + q] == ref["nloop"]
            assert rel(fields[i][1][q], ref["FFloc"]) < 1e-7
    for g in greens:
        g.close()


def test_ragged_batch_rejects_mismatched_boxes(gctx):
    import ifdda
    from ifdda import objects
    k0 = 2 * math.pi / 600e-9
    ob = objects.cube(100e-9, 2.0 + 0j, 8, k0, "RR")
    ga = gctx.green_box(8, 8, 8, (16, 16, 16), ob.aretecube, k0)
    gb = gctx.green_box(8, 8, 8, (8, 8, 8), ob.aretecube, k0)
    ff0 = np.ones((1, 3 * ob.nbsphere), np.complex128)
    with pytest.raises(ifdda.IfddaError, match="box"):
        gctx.inverserig_ragged([(ga, ob.nbsphere, ob.nmax, None, ob.polarisa, ff0),
                                (gb, ob.nbsphere, ob.nmax, None, ob.polarisa, ff0)])
    with pytest.raises(ifdda.IfddaError, match="box"):
        gctx.green_box(8, 8, 8, (6, 8, 8), ob.aretecube, k0)
    ga.close()
    gb.close()


def test_ragged_device_entry_matches_host_entry(gctx, orc):
    """ifdda_inverserig_ragged_device (every per-object array on the device,
    the polarisability compacted there) gives the host entry's bits, and
    ifdda_incident_planewaves_device the host planewaves' bits."""
    import torch
    items, greens, ff0s = _items(gctx, orc)
    fields, tol1, nloop, ncompte, nstop, info = gctx.inverserig_ragged(items, "GPBICG1", 1e-4, precision=1)
    assert nstop == 0, info
    keep, ditems = [], []
    for (g, nb, nmax, tab, pol, ff0) in items:
        t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in
             (("pol", pol), ("ff0", ff0)) }
        t["tab"] = torch.from_numpy(np.ascontiguousarray(tab, np.int32)).cuda() if tab is not None else None
        t["ff"] = torch.empty_like(t["ff0"])
        t["loc"] = torch.empty_like(t["ff0"])
        keep.append(t)
        ditems.append((g, nb, nmax, t["tab"].data_ptr() if t["tab"] is not None else None, t["pol"].data_ptr(),
                       t["ff0"].data_ptr(), t["ff"].data_ptr(), t["loc"].data_ptr(), ff0.shape[0]))
    d1, dl, dc, ds, dinfo = gctx.inverserig_ragged_device(ditems, "GPBICG1", 1e-4, precision=1)
    assert ds == 0, dinfo
    assert np.array_equal(d1, tol1) and np.array_equal(dc, ncompte) and np.array_equal(dl, nloop)
    for t, (FF, FFloc) in zip(keep, fields):
        assert np.array_equal(t["loc"].cpu().numpy(), FFloc) and np.array_equal(t["ff"].cpu().numpy(), FF)
    # incident fields built on the device
    from ifdda import objects
    ob, k0, _ = _objects()[0]
    E0, _ = objects.irradiance(1.0, 10 * 2 * math.pi / k0)
    kx, ky, pp = [0.1 * k0, -0.3 * k0], [0.2 * k0, 0.0], [0.0, 1.0]
    host = gctx.planewaves(ob.xs, ob.ys, ob.zs, k0, E0, [1, 1], kx, ky, pp)
    xs, ys, zs = (torch.from_numpy(np.ascontiguousarray(v, np.float64)).cuda() for v in (ob.xs, ob.ys, ob.zs))
    out = torch.empty(host.shape, dtype=torch.complex128, device="cuda")
    gctx.planewaves_device(ob.nbsphere, xs.data_ptr(), ys.data_ptr(), zs.data_ptr(), k0, E0, [1, 1], kx, ky, pp,
                           out.data_ptr())
    assert np.array_equal(out.cpu().numpy(), host)
    for g in greens:
        g.close()
