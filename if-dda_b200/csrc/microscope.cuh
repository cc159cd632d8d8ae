// Microscope image formation with the FFT lens (device launchers).
//   far field : cdmlib/diffractefft2dlens.f:1-181 (nside = +1)
//   lens      : cdmlib/microsbf.f:689-795, cdmlib/microsdf.f:668-766
//   image     : cdmlib/fouriertoimage.f:1-128 and the |E|^2 sums of
//               cdmlib/microsbf.f:800-826 / microsdf.f:771-790
#pragma once
#include "engine.cuh"

// image sides n (nfft2d) the lens transforms are compiled for: the powers of
// two and the reference's option list up to 4096 (cdm/cdmOptions.cpp:35 also
// offers 768, 1536, 3072)
#define IFDDA_IMG_LENGTHS(X) X(32) X(64) X(128) X(256) X(512) X(768) X(1024) X(1536) X(2048) X(3072) X(4096)

namespace ifdda {

bool image_length_supported(int n);

// The FFT lens of one object on an n x n pupil grid: frequencies
// (i dkx, j dky) for |i|, |j| <= imax (S = 2 imax + 1 per axis).
struct MicGeom {
    int nx, ny, nz;
    int n;
    int imax;
    int ntypemic;     // 1 bright field, 2 dark field and phase
    double k0, dkx, dky;
    double numaper;   // numerical aperture of the objective times k0
    double var1, var2;  // phase origin of the lattice (diffractefft2dlens.f:45-46)
    double zlens, gross;
    double dside;       // +1 transmission (kz > 0), -1 reflection (kz < 0)
    __host__ __device__ int S() const { return 2 * imax + 1; }
};

// Far field Ed (nb x S x S x 3, entry ((b S + jrow) S + irow) 3 + c) of the
// dipole moments FF (nb vectors of 3 nx ny nz, full box).  zplane: z of each
// lattice plane; tw: exp(+2 pi i m / n), m < n; Q: nb nz ny S 3 scratch.
// both_sides: the lens-free far field of diffractefft2d.f on the kz > 0
// side, then the kz < 0 side (2 nb S S 3 values), instead of the lens's.
void mic_farfield_dev(const MicGeom& m, int nb, const double2* FF, const double* zplane, const double2* tw,
                      double2* Q, double2* Ed, cudaStream_t st, bool both_sides = false);
// The same far field by direct summation over nd dipoles at (xs, ys, zs)
// (nquicklens = 0); part holds nb S^2 mic_direct_chunks(nd) 3 values.
int mic_direct_chunks(long nd);
void mic_direct_dev(const MicGeom& m, int nb, int nd, const double* xs, const double* ys, const double* zs,
                    const double2* FF, double2* part, double2* Ed, cudaStream_t st);
// Fourier-plane fields F (nb x 6 x S x S: x, y, z, then with the incident
// wave) after the lens: focus phase, the specular wave at grid point
// (ik[b], jk[b]) with polarisation pp[b], and the rotation by the lens.
void mic_lens_dev(const MicGeom& m, int nb, const double2* Ed, const int* ik, const int* jk, const double* pp,
                  double2 E0, double2* F, cudaStream_t st);
// Adds sum_b |image|^2 of the six fields to img (6 x n x n, pixel u + n v);
// T: nb 6 S n scratch.  Returns false for an n that is not compiled.
bool mic_image_dev(const MicGeom& m, int nb, const double2* F, const double2* tw, double2* T, double* img,
                   cudaStream_t st);
// Holographic image of one incidence: the lens of cdmlib.f:4380-4560 on the
// far field Ed (S x S x 3), the incident wave at (ik, jk) on the transmission
// side, then the complex image cimg (6 x n x n, pixel u + n v); four receives
// the pupil fields (6 x S x S); F (6 S S) and T (6 S n) are scratch.  slow:
// the lens without FFT (Ed by direct summation, points inside the aperture).
bool mic_holo_dev(const MicGeom& m, const double2* Ed, int ik, int jk, double pp, double2 E0, bool slow,
                  double2* F, double2* four, const double2* tw, double2* T, double2* cimg, cudaStream_t st);
// img = sqrt(img), cnt values
void mic_sqrt_dev(long cnt, double* img, cudaStream_t st);

}  // namespace ifdda
