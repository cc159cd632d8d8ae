// Amplitude of the plane wave of ondeplanekxky (cdmlib/ondeplanekxky.f:1-60)
// at the origin: polarisation pp (0 = s, 1 = p) for the transverse wave
// vector (kx, ky).  Shared by the incident-field kernel and the microscope's
// lens, which adds the specular wave of the illumination.
#pragma once
#include "cplx.cuh"

namespace ifdda {

__device__ __forceinline__ void kxky_amplitude(double k0, double2 E0, double pp, double kx, double ky, double2& ex,
                                               double2& ey, double2& ez, double& kz) {
    const double p = sqrt(pp), s = sqrt(1.0 - pp);
    kz = sqrt(k0 * k0 - kx * kx - ky * ky);
    const double2 E0s = make_double2(E0.x * s, E0.y * s), E0p = make_double2(E0.x * p, E0.y * p);
    if (kz >= 0.99999 * k0) {
        ex = E0p;
        ey = E0s;
        ez = make_double2(0, 0);
    } else {
        const double kp = sqrt(kx * kx + ky * ky);
        const double nsx = -ky / kp, nsy = kx / kp;
        double npx = kz * nsy, npy = -kz * nsx, npz = -kx * nsy + ky * nsx;
        const double np = sqrt(npx * npx + npy * npy + npz * npz);
        npx /= np;
        npy /= np;
        npz /= np;
        ex = make_double2(E0s.x * nsx + E0p.x * npx, E0s.y * nsx + E0p.y * npx);
        ey = make_double2(E0s.x * nsy + E0p.x * npy, E0s.y * nsy + E0p.y * npy);
        ez = make_double2(E0p.x * npz, E0p.y * npz);
    }
}

}  // namespace ifdda
