/*
 * ifdda_gpu.h -- C-ABI of libifdda_gpu.so, the sm_100a drop-in for the
 * FFT-accelerated dipole solve of IF-DDA's cdmlib.
 *
 * Conventions are the reference's (cdmlib/cdmlib.h, cdmlib/cdmlib.f):
 *   - double complex = { double re, im } (ifdda_dcmplx);
 *   - field vectors are AoS: dipole n (0-based) at 3n+{0,1,2};
 *   - lattice site (i,j,k) (0-based) has index i + nx*j + nx*ny*k;
 *   - tabdip[site] is the 1-based dipole number, 0 for an empty site;
 *   - polarisa / epsilon are column-major (nmax,3,3): (n,a,b) at n + nmax*(a + 3*b);
 *   - infostr is a Fortran character(64): space padded, not NUL terminated.
 * Every entry point returns the reference's nstop convention: 0 success,
 * 1 error (infostr or ifdda_ctx_last_error says why), -1 cancelled.
 * Nothing here aborts the process (unlike cdmlib/local-macro.f:41-48).
 */
#ifndef IFDDA_GPU_H
#define IFDDA_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define IFDDA_GPU_ABI_VERSION 1

typedef struct {
    double re, im;
} ifdda_dcmplx;

typedef struct ifdda_ctx ifdda_ctx;     /* one device + one CUDA stream */
typedef struct ifdda_green ifdda_green; /* device-resident Green spectrum + solver workspace */

/* arithmetic of a solve */
enum { IFDDA_FP64 = 0, IFDDA_MIXED = 1, IFDDA_FP32 = 2 };

typedef struct {
    int precision;      /* IFDDA_FP64 (plain drop-in) or IFDDA_MIXED (FP32 inner, FP64 refinement) */
    int check_every;    /* iterations launched between status polls; 0 = 4 */
    int max_outer;      /* refinement steps of IFDDA_MIXED; 0 = 12 */
    double inner_floor; /* smallest relative tolerance asked of an FP32 inner solve; 0 = 1e-6 */
    int maxit;          /* iteration limit; 0 = 10000, the reference's nlim (cdmlib/inverserigopt.f:30) */
} ifdda_solve_options;

int ifdda_abi_version(void);

/* Context: device ordinal, owns a CUDA stream for its work and a second
   one on which ifdda_inverserig / ifdda_inverserig_batch move host data
   while earlier work still runs (a call that returns host results has
   finished with both).  No counterpart in the reference (which has no
   device); cdmlib's FFTW plan set-up (cdmlib/cdmlib.f:1150-1165) is the
   closest analogue. */
int ifdda_ctx_create(int device, ifdda_ctx** out);
/* Releases the context.  If spectra made on it are still alive, the release
   waits until the last of them is destroyed (they keep using its stream);
   no new spectrum can be made on it meanwhile. */
int ifdda_ctx_destroy(ifdda_ctx* ctx);
const char* ifdda_ctx_last_error(const ifdda_ctx* ctx);
int ifdda_ctx_synchronize(ifdda_ctx* ctx);
/* the context's CUDA stream, as a cudaStream_t cast to void* */
void* ifdda_ctx_stream(ifdda_ctx* ctx);

/* Green spectrum.  Replaces greencalculfft (cdmlib/calculgreenfft.f:1-104,
   called at cdmlib/cdmlib.f:1529-1531) with nquad = 0: the six components of
   the free-space dyadic on the (2nx,2ny,2nz) circulant grid, FFT sign +1.
   aretecube in metres, k0 in 1/m.  The spectrum stays on the device.
   Every side from 1 to 320 is accepted, as the reference accepts any
   (cdmlib/primefactor.f only warns).  2n in {2,4,6,8,10,12,16,20,24,32,40,
   48,64,80,96,128,160,192,256,320,384,512,640} is computed as is; any other side n
   is padded to the smallest n' > n with 2n' in that set.  The lattice then
   sits at the corner of the larger box, and the mat-vecs and solves map the
   caller's sites onto it.  The results are those of the caller's lattice, up
   to the rounding of a longer FFT. */
int ifdda_green_create(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, double k0, ifdda_green** out);
/* The same with the integrated Green tensor (nquad = 1..16, 0 = plain):
   replaces greencalculquadfft (cdmlib/calculgreenquadfft.f, called at
   cdmlib/cdmlib.f:1532-1536 when nquad != 0) with propaesplibreintsim
   (cdmlib/propaesplibreintsim.f): at lattice offsets i^2+j^2+k^2 <= nquad^2
   the tensor averaged over the source cube (Simpson rule, 128 steps per axis),
   zero at the origin, the plain tensor beyond one wavelength. */
int ifdda_green_create_nquad(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, double k0, int nquad,
                             ifdda_green** out);
/* Spectrum of an nx x ny x nz lattice computed on a given larger box
   bx x by x bz (each side at least the lattice's, 2b a compiled FFT length),
   the lattice at the box's corner: greencalculfft on the box.  Spectra of
   different lattices, spacings and wavelengths made on one box can be solved
   together by ifdda_inverserig_ragged.  No counterpart in the reference,
   which solves one object per cdmlib call. */
int ifdda_green_create_box(ifdda_ctx* ctx, int nx, int ny, int nz, int bx, int by, int bz, double aretecube,
                           double k0, ifdda_green** out);
/* Tile chooser.  The zconv and y-pass kernels are compiled with two tile
   shapes for FFT lengths of 64 and more; before the first mat-vec of a
   precision on a grid, the library times both on that grid (best of three
   launches with CUDA events) and keeps shape 1 if it is at least 5% faster,
   for every later mat-vec of that precision on that grid and device, by
   every spectrum and batch size: a right-hand side runs the same kernels
   alone and in a batch.  The two shapes agree to rounding (the compiler may
   contract multiply-adds differently), not always bit for bit.
   ifdda_green_tiles reports the choice for g's grid (-1: not made yet) and,
   if times_ms is not NULL, the four times measured (zconv shapes 0, 1, y
   passes 0, 1; 0 where not timed).  ifdda_green_set_tiles imposes a choice
   (-1: choose again at the next mat-vec).  No counterpart in the reference
   (whose FFT has no tiles). */
int ifdda_green_tiles(ifdda_green* g, int precision, int* zconv_variant, int* ypass_variant, float* times_ms);
int ifdda_green_set_tiles(ifdda_green* g, int precision, int zconv_variant, int ypass_variant);
/* Recomputes g's spectrum in place for another lattice spacing and
   wavenumber (same lattice sides, nquad and padding): the call cdmlib makes
   at cdmlib/cdmlib.f:1529-1531 on every run, writing greencalculfft's result
   into the FFTTENSOR arrays it already holds.  g's solver workspaces (and the
   CUDA graphs captured on them) stay valid, so a solve that follows starts
   without re-allocation.  Returns after the spectrum is complete. */
int ifdda_green_recompute(ifdda_green* g, double aretecube, double k0);
int ifdda_green_destroy(ifdda_green* g);
/* Frees the solver and mat-vec workspaces held by g (they are re-created on
   the next solve); the spectrum stays.  For callers that cache many spectra.
   No counterpart in the reference. */
int ifdda_green_release_workspace(ifdda_green* g);
/* Writes the six FFTTENSOR arrays (xx,xy,xz,yy,yz,zz, 8*nx*ny*nz each, x
   fastest) exactly as greencalculfft leaves them.  Returns 1 for a padded
   lattice, whose spectrum is on another grid. */
int ifdda_green_export(ifdda_green* g, ifdda_dcmplx* xx, ifdda_dcmplx* xy, ifdda_dcmplx* xz, ifdda_dcmplx* yy,
                       ifdda_dcmplx* yz, ifdda_dcmplx* zz);

/* Mat-vec FFB <- FFB - (1/ntotal) IFFT(G~ . FFT(pad FFX)).  Replaces
   produitfftmatvectopt (cdmlib/produitfftmatvectopt.f:3-121, tabdip == NULL,
   ndip = nx*ny*nz) and produitfftmatvect3 (cdmlib/produitfftmatvect3.f:2-127,
   tabdip != NULL, ndip = dipole count).  precision: IFDDA_FP64 or IFDDA_FP32;
   any other value returns 1. */
int ifdda_matvec(ifdda_green* g, int precision, int ndip, const int* tabdip, const ifdda_dcmplx* FFX,
                 ifdda_dcmplx* FFB);

/* Same operation on nrhs vectors already in device memory, in place on
   FFB_dev: complex128 vectors for IFDDA_FP64, complex64 for IFDDA_FP32
   (3*ndip per right-hand side, contiguous).  Asynchronous on the context's
   stream.  Any other precision returns 1. */
int ifdda_matvec_device(ifdda_green* g, int precision, int nrhs, int ndip, const int* tabdip_dev,
                        const void* FFX_dev, void* FFB_dev);

/* Same operation as ifdda_matvec_device for one right-hand side, for callers
   that cannot allocate device memory while they run: a real-time loop that
   must avoid the device-wide synchronisation of cudaMalloc/cudaFree, a
   framework whose own caching allocator owns the GPU memory, or a host
   application that has handed its whole memory budget to another library.  It has no counterpart in the reference (whose
   buffers are static Fortran arrays).  The mat-vec scratch lives in one fixed
   16 MiB device array inside the library (held by every GPU that loads it
   until the process exits), so 18*nx'*ny'*nz' complex values of the chosen
   precision must fit in 16 MiB, where nx', ny', nz' are the sides the
   spectrum was computed on: the caller's sides, or the larger padded ones
   when a side n has 2n outside the compiled FFT lengths (e.g. 32^3 sites fit
   in FP64 and 40^3 in FP32, 48^3 does not fit in FP64; 33^3 runs on the 40^3
   box).  Larger grids, and a precision other than IFDDA_FP32 / IFDDA_FP64,
   return 1 with the reason in ifdda_ctx_last_error.  The first
   call on a device looks up the array's device address; make that first call
   before any stream capture.  All calls share the array: calls whose kernels
   overlap on the GPU race.  The spectrum comes from ifdda_green_create, made
   beforehand. */
int ifdda_matvec_noalloc(ifdda_green* g, int precision, int ndip, const int* tabdip_dev, const void* FFX_dev,
                         void* FFB_dev);

/* Rigorous solve.  Replaces inverserigopt (cdmlib/inverserigopt.f:1-1085,
   tabdip == NULL) and inverserig (cdmlib/inverserig.f:1-1090, tabdip != NULL),
   called at cdmlib/cdmlib.f:1565-1581: initial guess FF0, methodeit
   "GPBICG1" | "QMRBICGSTAB1" | "QMRBICGSTAB2" | "BICGSTAB" (pimzbicgstab.f)
   | "CG" (zcg.f) | "TFQMR" (tfqmr.f) | "GPBICGsafe" (gpbicgsafe.f) | "GPBICG2"
   (gpbicg2.f) | "GPBICGplus" (gpbicgplus.f) | "GPBICGAR" (gpbicgar.f; also
   "GPBICGAR2", as in the reference) | "BICGSTARPLUS" (bicgstarplus.f) |
   "GPBICOR" (gpbicor.f) | "CORS" (cors.f) | "QMRCLA" (qmrpim.f, with
   products by A^T = I - alpha^T G), matched by prefix in the reference's
   order; any other string answers nstop = 1, "Iterative method not
   correct!".  On return FFloc = E (local field), FF = polarisa . E (dipole
   moments), tol1 = ||A E - FF0|| / NORM in FP64 with the method's NORM
   (||FF0||; for BICGSTAB the squared norm of the initial residual, as the
   reference computes it), nloop iterations, ncompte mat-vecs.  *nstop is read during the
   solve: a value of -1 written by another thread cancels it, as in the
   reference (cdm/cdmRunWidget.cpp:156).  A converged tol1 >= tol is reported
   as nstop = 1 "Converge do not reach!" (cdmlib/cdmlib.f:1586-1591).
   opt may be NULL (plain FP64). */
int ifdda_inverserig(ifdda_green* g, int nbsphere, int nmax, const int* tabdip, const ifdda_dcmplx* polarisa,
                     const ifdda_dcmplx* FF0, const char* methodeit, double tol, ifdda_dcmplx* FF,
                     ifdda_dcmplx* FFloc, double* tol1, int* nloop, int* ncompte, int* nstop, char* infostr,
                     const ifdda_solve_options* opt);

/* Batched solve of nrhs right-hand sides sharing the object (the serial
   incidence loop of cdmlib/microsbf.f:214-280 as one launch sequence).
   FF0, FF, FFloc hold nrhs vectors of 3*nbsphere; tol1, nloop, ncompte hold
   nrhs entries; nstop/infostr report the first failing right-hand side. */
int ifdda_inverserig_batch(ifdda_green* g, int nrhs, int nbsphere, int nmax, const int* tabdip,
                           const ifdda_dcmplx* polarisa, const ifdda_dcmplx* FF0, const char* methodeit, double tol,
                           ifdda_dcmplx* FF, ifdda_dcmplx* FFloc, double* tol1, int* nloop, int* ncompte,
                           int* nstop, char* infostr, const ifdda_solve_options* opt);

/* Same as ifdda_inverserig_batch with every array already in device memory
   of the context's device (inputs resident in HBM).  polarisa_dev is the
   (nmax,3,3) tensor; tabdip_dev may be NULL. */
int ifdda_inverserig_batch_device(ifdda_green* g, int nrhs, int nbsphere, int nmax, const int* tabdip_dev,
                                  const ifdda_dcmplx* polarisa_dev, const ifdda_dcmplx* FF0_dev,
                                  const char* methodeit, double tol, ifdda_dcmplx* FF_dev, ifdda_dcmplx* FFloc_dev,
                                  double* tol1, int* nloop, int* ncompte, int* nstop, char* infostr,
                                  const ifdda_solve_options* opt);

/* Ragged batch: nobj objects of uneven lattices, spacings and wavelengths,
   object i with nrhs[i] right-hand sides, solved together in one launch
   sequence per iteration (what the reference does as one cdmlib call per
   object, cdmlib/cdmlib.f:1565-1581, each a serial incidence loop as in
   cdmlib/microsbf.f:214-280).  greens[i] is object i's spectrum, every one
   made by ifdda_green_create_box on the same box and context; the first
   one's workspaces hold the batch.  Object i: nbsphere[i] dipoles, nmax[i],
   tabdip[i] on its own lattice (tabdip may be NULL, or tabdip[i] NULL for a
   full box), polarisa[i] (nmax[i],3,3) isotropic, FF0[i] / FF[i] / FFloc[i]
   nrhs[i] vectors of 3*nbsphere[i].  tol1, nloop, ncompte hold one entry per
   right-hand side, objects in order; nstop / infostr report the first
   failing one.  Every right-hand side is laid out on the box's sites, so its
   result does not depend on the other objects of the batch: bit for bit the
   same alone (nobj = 1) and in any batch on that box, and the solo solve's
   (ifdda_inverserig) up to rounding.  QMRCLA and anisotropic tensors return
   1. */
int ifdda_inverserig_ragged(int nobj, ifdda_green* const* greens, const int* nrhs, const int* nbsphere,
                            const int* nmax, const int* const* tabdip, const ifdda_dcmplx* const* polarisa,
                            const ifdda_dcmplx* const* FF0, const char* methodeit, double tol, ifdda_dcmplx* const* FF,
                            ifdda_dcmplx* const* FFloc, double* tol1, int* nloop, int* ncompte, int* nstop,
                            char* infostr, const ifdda_solve_options* opt);

/* The same with every per-object array in device memory of the context's
   device (tabdip_dev[i] may be NULL): the polarisability is checked for
   isotropy and compacted on the device.  For a request loop that builds its
   incident fields on the device (ifdda_incident_planewaves_device) and reads
   back only what a request returns. */
int ifdda_inverserig_ragged_device(int nobj, ifdda_green* const* greens, const int* nrhs, const int* nbsphere,
                                   const int* nmax, const int* const* tabdip_dev,
                                   const ifdda_dcmplx* const* polarisa_dev, const ifdda_dcmplx* const* FF0_dev,
                                   const char* methodeit, double tol, ifdda_dcmplx* const* FF_dev,
                                   ifdda_dcmplx* const* FFloc_dev, double* tol1, int* nloop, int* ncompte, int* nstop,
                                   char* infostr, const ifdda_solve_options* opt);

/* Local -> macroscopic field of every dipole (nsens = 1), replacing the loop
   of cdmlib/cdmlib.f:2595-2655 over local_macro (cdmlib/local-macro.f:3-71);
   the 3x3 inverse is evaluated in closed form on the device.  epsilon is
   (nmax,3,3); Em receives 3*nbsphere values. */
int ifdda_local_macro(ifdda_ctx* ctx, int nbsphere, int nmax, const ifdda_dcmplx* epsilon,
                      const ifdda_dcmplx* FFloc, double aretecube, double k0, ifdda_dcmplx* Em);

/* Extinction and absorption cross sections (cdmlib/cdmlib.f:2730-2746):
   Cext = 4 pi k0 / I0 sum Im(conj(FF0) . FF),
   Cabs = 4 pi k0 / I0 sum [Im(FF . conj(FFloc)) - 2/3 k0^3 |FF|^2]. */
int ifdda_cross_sections(ifdda_ctx* ctx, int nbsphere, const ifdda_dcmplx* FF0, const ifdda_dcmplx* FF,
                         const ifdda_dcmplx* FFloc, double k0, double I0, double* Cext, double* Cabs);

/* Incident plane waves for a batch of incidences (the OpenMP loops of
   cdmlib/cdmlib.f:1180-1187 over ondeplane, cdmlib/ondeplane.f:1-50, and of
   cdmlib/microsbf.f:245-253 over ondeplanekxky, cdmlib/ondeplanekxky.f:1-60).
   beam 0: a1 = theta, a2 = phi in degrees; beam 1: a1 = kx, a2 = ky in 1/m.
   Writes nrhs vectors of 3*nbsphere into FF0. */
int ifdda_incident_planewaves(ifdda_ctx* ctx, int nbsphere, const double* xs, const double* ys, const double* zs,
                              double k0, ifdda_dcmplx E0, int nrhs, const int* beam, const double* a1,
                              const double* a2, const double* pp, ifdda_dcmplx* FF0);

/* ifdda_incident_planewaves with the dipole positions (xs_dev, ys_dev,
   zs_dev) and the result FF0_dev in device memory of the context's device;
   beam, a1, a2, pp stay host arrays of nrhs entries. */
int ifdda_incident_planewaves_device(ifdda_ctx* ctx, int nbsphere, const double* xs_dev, const double* ys_dev,
                                     const double* zs_dev, double k0, ifdda_dcmplx E0, int nrhs, const int* beam,
                                     const double* a1, const double* a2, const double* pp, ifdda_dcmplx* FF0_dev);

/* Scattering cross section Cscai, asymmetry factor gasym and far-field
   Poynting vector by direct summation of the dipole moments FF over the
   (ntheta+1) x nphi directions (cdmlib/cdmlib.f:2784-2880, nsectionsca = 1,
   nquickdiffracte = 0); the |E|^2 of every direction on the device, the
   integration on the host in the reference's order.  theta, phi: incidence
   (deg) for gasym; I0 = |E0|^2.  poynting, thetafield, phifield ((ntheta+1)
   nphi values each, may be NULL): the reference's poyntingfield (W/sr) and its
   angles in degrees.  ntheta <= 10 or nphi <= 20: "ntheta and nphi too small!". */
int ifdda_farfield_csca(ifdda_ctx* ctx, int nbsphere, const double* xs, const double* ys, const double* zs,
                        const ifdda_dcmplx* FF, double k0, double I0, double theta, double phi, int ntheta, int nphi,
                        double* Cscai, double* gasym, double* poynting, double* thetafield, double* phifield);

/* The same quantities from the far field on the pupil grid (nsectionsca = 1,
   nquickdiffracte = 1): diffractefft2d (cdmlib/diffractefft2d.f:1-183) on
   both sides, evaluated on the device at the (2 imaxk0 + 1)^2 propagating
   frequencies (i dk, j dk), dk = 2 pi / (nfft2d aretecube), imaxk0 =
   nint(k0 / dk) + 1; Cscai and gasym by computegcfft2d
   (cdmlib/computegcfft2d.f:1-51); poynting on the (ntheta+1) x nphi grid by
   the reference's bilinear interpolation (cdmlib/cdmlib.f:2990-3075).  FF
   on the full nx*ny*nz box (cdmlib.f:630 forces it).  kpos / kneg ((2 imaxk0
   + 1)^2 values, index (i + imaxk0)(2 imaxk0 + 1) + j + imaxk0, may be NULL):
   the Poynting vector on the pupil grid for kz > 0 and kz < 0.  Any nfft2d up
   to 16384 (the sums are evaluated at the pupil frequencies only). */
int ifdda_farfield_fft(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, const double* xs, const double* ys,
                       const double* zs, const ifdda_dcmplx* FF, double k0, double I0, double theta, double phi,
                       int nfft2d, int ntheta, int nphi, double* Cscai, double* gasym, double* poynting,
                       double* thetafield, double* phifield, int* imaxk0, double* kpos, double* kneg);

/* Wide near field (cdmlib/cdmlib.f:1967-2492, nprochefft >= 1): the fields
   on the box enlarged by nxmp, nymp, nzmp layers on every side of the
   object's nx*ny*nz box, after a solve.  Its (nx+2nxmp)(ny+2nymp)(nz+2nzmp)
   = nw sites run in z, y, x order from the smallest object coordinate minus
   the layers; a site takes object dipole l (the next one in order) when
   their positions agree within lambda/1000 (comparaison.f).  The Green
   spectrum of the enlarged box is built (nquad as for ifdda_green_create_nquad),
   and one FP64 mat-vec gives E = E0 - A(-FF): incident receives E0 (FF0 at the
   object's dipoles, the plane wave ondeplane(theta, phi [deg], pp, E0)
   elsewhere), local the field, macro local_macro of it with the object's
   epsilon (nmax,3,3) and the identity elsewhere; 3*nw values each (may be
   NULL), positions in xswf, yswf, zswf (nw values, may be NULL). */
int ifdda_nearfield_wide(ifdda_ctx* ctx, int nx, int ny, int nz, int nxmp, int nymp, int nzmp, double aretecube,
                         double k0, int nquad, int nbsphere, int nmax, const double* xs, const double* ys,
                         const double* zs, const ifdda_dcmplx* FF, const ifdda_dcmplx* FF0,
                         const ifdda_dcmplx* epsilon, ifdda_dcmplx E0, double theta, double phi, double pp,
                         double* xswf, double* yswf, double* zswf, ifdda_dcmplx* incident, ifdda_dcmplx* local,
                         ifdda_dcmplx* macro);

/* Microscope options: the cdmlib arguments that the microscopes read
   (cdmlib/cdmlib.f:3660-3800 with nlentille = 1, nquicklens = 1). */
typedef struct {
    int ntypemic;      /* 1 bright field (microsbf.f), 2 dark field and phase (microsdf.f) */
    int nfft2d;        /* side n of the pupil and image grids: a power of two from 32 to
                          4096, or 768, 1536, 3072 (the reference's list up to 4096) */
    double numaper;    /* numerical aperture of the objective, (0, 1] */
    double numaperinc; /* numerical aperture of the condenser, < 1 */
    double gross;      /* magnification */
    double zlens;      /* focal-plane position in metres, as given (the side's sign is applied inside) */
    double P0, w0;     /* power (W) shared by all illuminations, waist (m) of irradiance.f */
    int batch;         /* illuminations solved together; 0 = 64 */
    int nside;         /* 0 transmission (microsbf / microsdf), 1 reflection (microsbfneg /
                          microsdfneg, cdmlib/microssansinc.f: no image with the incident wave) */
    int nquicklens;    /* 1 the FFT lens (full box), 0 the lens's far field by direct summation
                          over the dipoles (any object, microsbf.f:139-157, 627-666) */
} ifdda_microscope_options;

/* Bright-field or dark-field / phase microscope with the FFT lens, in
   transmission or reflection: replaces microsbf (cdmlib/microsbf.f:1-965),
   microsdf (cdmlib/microsdf.f:1-915) and their reflection forms microsbfneg /
   microsdfneg (cdmlib/microssansinc.f:1-1741), called at
   cdmlib/cdmlib.f:3735-3800, with
   diffractefft2dlens.f, fouriertoimage.f and deltakroutine.f inside.  With
   the FFT lens (nquicklens = 1) the object fills the full box of the
   spectrum g (nbsphere = nx*ny*nz, tabdip NULL: the reference forces it,
   cdmlib.f:631); with nquicklens = 0 tabdip may name inside-only dipoles as
   for ifdda_inverserig.  xs, ys, zs: nbsphere positions; polarisa: the
   (nx*ny*nz,3,3) tensor.  Every illumination
   (both polarisations, s first) is solved in batches of mo->batch through the
   batched solver, without the tol1 < tol check of cdmlib (microsbf does not
   make it).  image receives 6 * n * n values: sqrt(sum |E|^2) over the
   illuminations of the x, y, z image fields and of the same with the
   incident wave (Eimagex..z, Eimageincx..z), pixel u + n v.  xy and kxy
   (n values, may be NULL): image positions (m) and pupil kx / k0.  *ninc: on
   entry the room in kxinc / kyinc (may be 0 with NULL arrays), on return the
   number of incidences per polarisation; kxinc / kyinc receive them in
   units of k0.  tol1, nloop, ncompte: those of the last solve, as the
   reference leaves them.  Errors answer nstop = 1 with the reference's
   messages. */
int ifdda_microscope(ifdda_green* g, int nbsphere, const int* tabdip, const double* xs, const double* ys,
                     const double* zs, const ifdda_dcmplx* polarisa, const char* methodeit, double tol,
                     const ifdda_microscope_options* mo, double* image, double* xy, double* kxy, int* ninc,
                     double* kxinc, double* kyinc, double* tol1, int* nloop, int* ncompte, int* nstop,
                     char* infostr, const ifdda_solve_options* opt);

/* Holographic microscope (ntypemic = 0) with the FFT lens, after the solve of
   one plane wave (theta, phi in degrees, polarisation pp, amplitude E0):
   replaces cdmlib/cdmlib.f:4075-4660 with nenergie = 0, that is
   diffractefft2dlens (cdmlib/diffractefft2dlens.f:1-181) on the dipole
   moments FF of the full nx*ny*nz box, the incident wave in the pupil
   (cdmlib/diffractefft2dinc.f:75-91), the lens rotation and fouriertoimage
   (cdmlib/fouriertoimage.f, fouriertoimage2.f on the reflection side).
   numaper unitless, zlens in metres without the side's sign, nside 0
   transmission / 1 reflection.  nquicklens 0: the lens without FFT
   (cdmlib.f:3803-4074): a finer pupil grid (more than 20 points over k0),
   the far field by direct summation over the nbsphere dipoles (any object;
   FF and xs, ys, zs of those dipoles), only points inside the aperture; with
   nquicklens = 1 the object is the full box (nbsphere = nx*ny*nz).  image: 6 complex n*n fields (Eimagex..z,
   then Eimageincx..z, zero on the reflection side), pixel u + n v; fourier
   (may be NULL): the pupil fields Efourierx..z, Efourierincx..z before the
   rotation, 6 x (2 imaxk0 + 1)^2, row j, column i; xy, kxy (n values, may be
   NULL).  nfft2d: a power of two from 32 to 4096, or 768, 1536, 3072.  Returns 1 with the
   reference's message on an error. */
int ifdda_holography(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, double k0, int nbsphere,
                     const double* xs, const double* ys, const double* zs, const ifdda_dcmplx* FF, ifdda_dcmplx E0,
                     double theta, double phi, double pp, int nfft2d, double numaper, double gross, double zlens,
                     int nside, int nquicklens, ifdda_dcmplx* image, ifdda_dcmplx* fourier, double* xy,
                     double* kxy, int* imaxk0, char* infostr);

/* Diagnostics (no counterpart in the reference, whose only instrumentation
   is the wall/CPU-time printout of cdmlib/cdmlib.f:1956-1963 and the
   mat-vec count ncompte).
   ifdda_launch_count: kernels launched by this library since it was loaded.
   ifdda_timing_enable: bracket every launch of one mat-vec pass with CUDA
   events on its stream (pass 1 fwd_x, 2 fwd_y, 3 zconv, 4 inv_y, 5 inv_x;
   0 disables; precision IFDDA_FP64 / IFDDA_FP32 filters, -1 both).
   ifdda_timing_read: waits for the recorded events, returns the number of
   timed launches and their summed duration, and clears the record. */
unsigned long long ifdda_launch_count(void);
int ifdda_timing_enable(int pass, int precision);
int ifdda_timing_read(int* launches, double* total_ms);

#ifdef __cplusplus
}
#endif
#endif
