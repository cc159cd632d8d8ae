/*
 * ifdda_oracle.c -- CPU restatement (FP64, OpenMP) of IF-DDA's FFT-accelerated
 * discrete-dipole solve.  TEST INFRASTRUCTURE ONLY: the parity tests hold the
 * CUDA path to it, and it is the timed CPU baseline.  Nothing in the product links it.
 *
 * Parity status: the reference (Fortran 77/90) cannot be compiled where this was
 * written (no Fortran compiler, no FFTW3), and its own tests store no outputs.
 * The restatement is therefore pinned by
 *   - numpy.fft on the same data (FFT sign and normalisation convention),
 *   - a dense O(N^2) direct sum of propa_espace_libre (circulant embedding,
 *     wrap-around, zero planes, 1/ntotal scaling of the FFT mat-vec),
 *   - the reference's own GPBICG self-test (cdmlib/gpbicg.f:1-79, 5x5 diagonal
 *     system with known solution x_i = 1/i),
 *   - the Mie series for homogeneous spheres (the comparison cdmlib prints at
 *     cdmlib/cdmlib.f:2767-2773),
 * and not by outputs produced by the reference itself ("parity unpinned" with
 * respect to reference-generated vectors).
 *
 * Conventions kept from the reference (cdmlib/cdmlib.h, cdmlib/cdmlib.f):
 *   - field vectors are AoS, 3 complex per dipole, dipole n at 3n+{0,1,2};
 *   - the lattice index of site (i,j,k) (0-based) is i + nx*j + nx*ny*k;
 *   - polarisa/epsilon are column-major (nmax,3,3): element (n,a,b) at
 *     n + nmax*a + 3*nmax*b;
 *   - padded FFT grids are (2nx,2ny,2nz), x fastest;
 *   - the "forward" transform of G and x has sign +1 (exp(+i...)), the inverse
 *     sign -1, both unnormalised; 1/ntotal is applied once at the crop.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex zc;

/* ------------------------------------------------------------------------- */
/* Mixed-radix FFT (any length), recursive decimation in time.               */
/* Follows the contract of cdmlib/fftsingletonz.f:21-43 (fftsingletonz3d):    */
/* in-place 3-D transform as three strided 1-D passes, unnormalised,          */
/* exp(+i 2 pi jk/n) for isign >= 0 and exp(-i ...) otherwise                 */
/* (fftsingletonz.f:109-114).                                                */
/* ------------------------------------------------------------------------- */

typedef struct {
    int n;
    int nf;
    int fac[32];
    zc *w; /* w[j] = exp(+2 pi i j / n) */
} fft_plan;

static void plan_init(fft_plan *p, int n) {
    p->n = n;
    p->nf = 0;
    int m = n;
    /* radix 4 first, then 2, 3, 5, then any remaining prime */
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    for (int f = 3; m > 1; f += 2) {
        while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
    }
    p->w = (zc *)malloc(sizeof(zc) * (size_t)n);
    const double two_pi = 6.283185307179586476925286766559;
    for (int j = 0; j < n; j++) {
        double a = two_pi * (double)j / (double)n;
        p->w[j] = cos(a) + I * sin(a);
    }
}

static void plan_free(fft_plan *p) { free(p->w); }

/* out[0..n) = DFT of in[0], in[s], ..., sign sg (+1/-1) */
static void fft_rec(const fft_plan *p, const zc *in, int s, zc *out, int n,
                    int fi, int sg, zc *tmp) {
    if (n == 1) { out[0] = in[0]; return; }
    int r = p->fac[fi];
    int m = n / r;
    for (int q = 0; q < r; q++)
        fft_rec(p, in + (size_t)q * s, s * r, out + (size_t)q * m, m, fi + 1, sg, tmp);
    int stepn = p->n / n; /* w_n^j = W[j*stepn] */
    int stepr = p->n / r; /* w_r^j = W[j*stepr] */
    for (int k = 0; k < m; k++) {
        zc t[64];
        for (int q = 0; q < r; q++) {
            int e = (int)(((long)q * k * stepn) % p->n);
            zc w = p->w[e];
            if (sg < 0) w = conj(w);
            t[q] = out[(size_t)q * m + k] * w;
        }
        for (int o = 0; o < r; o++) {
            zc acc = 0;
            for (int q = 0; q < r; q++) {
                int e = (int)(((long)q * o * stepr) % p->n);
                zc w = p->w[e];
                if (sg < 0) w = conj(w);
                acc += t[q] * w;
            }
            tmp[o] = acc;
        }
        for (int o = 0; o < r; o++) out[(size_t)o * m + k] = tmp[o];
    }
}

/* one strided pass over all lines of dimension `axis` of an n1 x n2 x n3 array */
static void fft_axis(zc *v, int n1, int n2, int n3, int axis, int sg) {
    int n = axis == 0 ? n1 : (axis == 1 ? n2 : n3);
    if (n < 2) return;
    fft_plan p;
    plan_init(&p, n);
    long stride = axis == 0 ? 1 : (axis == 1 ? n1 : (long)n1 * n2);
    long nlines = (long)n1 * n2 * n3 / n;
#pragma omp parallel
    {
        zc *buf = (zc *)malloc(sizeof(zc) * (size_t)n * 2);
        zc tmp[64];
#pragma omp for schedule(static)
        for (long l = 0; l < nlines; l++) {
            long base;
            if (axis == 0) base = l * n1;
            else if (axis == 1) base = (l % n1) + (l / n1) * (long)n1 * n2;
            else base = l;
            for (int j = 0; j < n; j++) buf[j] = v[base + j * stride];
            fft_rec(&p, buf, 1, buf + n, n, 0, sg, tmp);
            for (int j = 0; j < n; j++) v[base + j * stride] = buf[n + j];
        }
        free(buf);
    }
    plan_free(&p);
}

/* fftsingletonz3d(vect,NX,NY,NZ,ISIGN): x, y, z passes for +1; z, y, x for -1 */
void orc_fft3d(zc *v, int n1, int n2, int n3, int isign) {
    if (isign >= 0) {
        fft_axis(v, n1, n2, n3, 0, +1);
        fft_axis(v, n1, n2, n3, 1, +1);
        fft_axis(v, n1, n2, n3, 2, +1);
    } else {
        fft_axis(v, n1, n2, n3, 2, -1);
        fft_axis(v, n1, n2, n3, 1, -1);
        fft_axis(v, n1, n2, n3, 0, -1);
    }
}

/* ------------------------------------------------------------------------- */
/* Free-space dyadic Green tensor: cdmlib/espace_libre.f:2-43                 */
/* T = [(3RR/R^2 - I)(1/R - i k0)/R^2 + (I - RR/R^2) k0^2/R] exp(i k0 R),     */
/* zero at R = 0.  out is column-major 3x3.                                   */
/* ------------------------------------------------------------------------- */
void orc_propa_espace_libre(double x, double y, double z, double x0, double y0,
                            double z0, double k0, zc *out) {
    double r[3] = {x - x0, y - y0, z - z0};
    double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    double rab = sqrt(r2);
    if (rab == 0.0) {
        for (int q = 0; q < 9; q++) out[q] = 0;
        return;
    }
    zc c1 = (1.0 / rab - I * k0) / r2;
    zc c2 = k0 * k0 / rab;
    zc e = cexp(I * k0 * rab);
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            double id = a == b ? 1.0 : 0.0;
            double rr = r[a] * r[b] / r2;
            out[a + 3 * b] = ((3.0 * rr - id) * c1 + (id - rr) * c2) * e;
        }
}

/* ------------------------------------------------------------------------- */
/* Green spectrum: cdmlib/calculgreenfft.f:1-104.                             */
/* G6 holds 6 arrays of M = 8 nx ny nz complex, in the order                  */
/* xx, xy, xz, yy, yz, zz, each with leading dims (2nx, 2ny), x fastest.      */
/* ------------------------------------------------------------------------- */
void orc_greencalculfft(int nx, int ny, int nz, double d, double k0, zc *G6) {
    int nx2 = 2 * nx, ny2 = 2 * ny, nz2 = 2 * nz;
    long M = (long)nx2 * ny2 * nz2;
#pragma omp parallel for schedule(static)
    for (long idx = 0; idx < M; idx++) {
        int ii = (int)(idx % nx2);
        int jj = (int)((idx / nx2) % ny2);
        int kk = (int)(idx / ((long)nx2 * ny2));
        if (ii == nx || jj == ny || kk == nz) {
            for (int c = 0; c < 6; c++) G6[c * M + idx] = 0;
            continue;
        }
        int i = ii > nx ? ii - nx2 : ii;
        int j = jj > ny ? jj - ny2 : jj;
        int k = kk > nz ? kk - nz2 : kk;
        zc t[9];
        orc_propa_espace_libre(0, 0, 0, i * d, j * d, k * d, k0, t);
        G6[0 * M + idx] = t[0 + 3 * 0];
        G6[1 * M + idx] = t[0 + 3 * 1];
        G6[2 * M + idx] = t[0 + 3 * 2];
        G6[3 * M + idx] = t[1 + 3 * 1];
        G6[4 * M + idx] = t[1 + 3 * 2];
        G6[5 * M + idx] = t[2 + 3 * 2];
    }
    for (int c = 0; c < 6; c++) orc_fft3d(G6 + c * M, nx2, ny2, nz2, +1);
}

/* ------------------------------------------------------------------------- */
/* Green tensor averaged over the source cube: cdmlib/propaesplibreintsim.f.  */
/* Zero when the points are closer than d/10, the plain tensor beyond lim    */
/* wavelengths, otherwise a Simpson rule with 128 steps per axis over the     */
/* cube of side d centred on (x,y,z); the off-diagonal terms are zeroed       */
/* along the axes on which the two points coincide (closer than d/10).        */
/* out is column-major 3x3.                                                   */
/* ------------------------------------------------------------------------- */
void orc_propaesplibreintsim(double x, double y, double z, double x0, double y0, double z0,
                             double k0, double d, double lim, zc *out) {
    const double pi = acos(-1.0), lambda = 2.0 * pi / k0, dm = d * 0.1;
    const double rab = sqrt((x - x0) * (x - x0) + (y - y0) * (y - y0) + (z - z0) * (z - z0));
    if (rab <= dm) {
        for (int q = 0; q < 9; q++) out[q] = 0;
        return;
    }
    if (rab >= lim * lambda) {
        orc_propa_espace_libre(x, y, z, x0, y0, z0, k0, out);
        return;
    }
    const int nstep = 128;
    double w[129];
    w[0] = w[nstep] = 1.0;
    for (int i = 1; i < nstep; i++) w[i] = i % 2 ? 4.0 : 2.0;
    const double pas = d / nstep, ax = x - d / 2, ay = y - d / 2, az = z - d / 2;
    double acc[12] = {0};
#pragma omp parallel for reduction(+ : acc[:12]) schedule(static)
    for (int i = 0; i <= nstep; i++)
        for (int j = 0; j <= nstep; j++)
            for (int k = 0; k <= nstep; k++) {
                zc t[9];
                orc_propa_espace_libre(ax + pas * i, ay + pas * j, az + pas * k, x0, y0, z0, k0, t);
                const double ww = w[i] * w[j] * w[k];
                const int qs[6] = {0, 3, 6, 4, 7, 8};  /* xx xy xz yy yz zz */
                for (int q = 0; q < 6; q++) {
                    acc[2 * q] += creal(t[qs[q]]) * ww;
                    acc[2 * q + 1] += cimag(t[qs[q]]) * ww;
                }
            }
    const double tmp = pas / 3.0 * pas / 3.0 * pas / 3.0 / d / d / d;
    const double fx = fabs(x - x0) <= dm ? 0.0 : 1.0, fy = fabs(y - y0) <= dm ? 0.0 : 1.0,
                 fz = fabs(z - z0) <= dm ? 0.0 : 1.0;
    zc v[6];
    for (int q = 0; q < 6; q++) v[q] = (acc[2 * q] + I * acc[2 * q + 1]) * tmp;
    v[1] *= fx * fy;
    v[2] *= fx * fz;
    v[4] *= fy * fz;
    out[0] = v[0];
    out[3] = out[1] = v[1];
    out[6] = out[2] = v[2];
    out[4] = v[3];
    out[7] = out[5] = v[4];
    out[8] = v[5];
}

/* Green spectrum with the integrated tensor at the offsets i^2+j^2+k^2 <=     */
/* nquad^2: cdmlib/calculgreenquadfft.f (lim = 1 wavelength).                 */
void orc_greencalculquadfft(int nx, int ny, int nz, int nquad, double d, double k0, zc *G6) {
    int nx2 = 2 * nx, ny2 = 2 * ny, nz2 = 2 * nz;
    long M = (long)nx2 * ny2 * nz2;
    for (long idx = 0; idx < M; idx++) {
        int ii = (int)(idx % nx2);
        int jj = (int)((idx / nx2) % ny2);
        int kk = (int)(idx / ((long)nx2 * ny2));
        if (ii == nx || jj == ny || kk == nz) {
            for (int c = 0; c < 6; c++) G6[c * M + idx] = 0;
            continue;
        }
        int i = ii > nx ? ii - nx2 : ii;
        int j = jj > ny ? jj - ny2 : jj;
        int k = kk > nz ? kk - nz2 : kk;
        zc t[9];
        if (nquad != 0 && i * i + j * j + k * k <= nquad * nquad)
            orc_propaesplibreintsim(0, 0, 0, i * d, j * d, k * d, k0, d, 1.0, t);
        else
            orc_propa_espace_libre(0, 0, 0, i * d, j * d, k * d, k0, t);
        G6[0 * M + idx] = t[0 + 3 * 0];
        G6[1 * M + idx] = t[0 + 3 * 1];
        G6[2 * M + idx] = t[0 + 3 * 2];
        G6[3 * M + idx] = t[1 + 3 * 1];
        G6[4 * M + idx] = t[1 + 3 * 2];
        G6[5 * M + idx] = t[2 + 3 * 2];
    }
    for (int c = 0; c < 6; c++) orc_fft3d(G6 + c * M, nx2, ny2, nz2, +1);
}

/* ------------------------------------------------------------------------- */
/* FFT mat-vec: FFB <- FFB - (1/M) IFFT(G~ . FFT(pad(FFX)))                   */
/* cdmlib/produitfftmatvectopt.f:3-121 (tabdip == NULL, full box) and         */
/* cdmlib/produitfftmatvect3.f:2-127 (tabdip != NULL: lattice site s holds    */
/* dipole tabdip[s]-1, 0 meaning empty).                                      */
/* ------------------------------------------------------------------------- */
static void matvec_core(const zc *G6, int nx, int ny, int nz, const int *tabdip,
                        const zc *FFX, zc *FFB) {
    int nx2 = 2 * nx, ny2 = 2 * ny, nz2 = 2 * nz;
    long M = (long)nx2 * ny2 * nz2;
    long nxy2 = (long)nx2 * ny2;
    long nxy = (long)nx * ny;
    double dntotal = (double)M;
    zc *v = (zc *)calloc((size_t)(3 * M), sizeof(zc));
    zc *vx = v, *vy = v + M, *vz = v + 2 * M;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                long site = i + (long)nx * j + nxy * k;
                long n = site;
                if (tabdip) {
                    if (tabdip[site] == 0) continue;
                    n = tabdip[site] - 1;
                }
                long ind = i + (long)nx2 * j + nxy2 * k;
                vx[ind] = FFX[3 * n + 0];
                vy[ind] = FFX[3 * n + 1];
                vz[ind] = FFX[3 * n + 2];
            }
    orc_fft3d(vx, nx2, ny2, nz2, +1);
    orc_fft3d(vy, nx2, ny2, nz2, +1);
    orc_fft3d(vz, nx2, ny2, nz2, +1);
    const zc *gxx = G6, *gxy = G6 + M, *gxz = G6 + 2 * M, *gyy = G6 + 3 * M,
             *gyz = G6 + 4 * M, *gzz = G6 + 5 * M;
#pragma omp parallel for schedule(static)
    for (long q = 0; q < M; q++) {
        zc a = vx[q], b = vy[q], c = vz[q];
        vx[q] = gxx[q] * a + gxy[q] * b + gxz[q] * c;
        vy[q] = gxy[q] * a + gyy[q] * b + gyz[q] * c;
        vz[q] = gxz[q] * a + gyz[q] * b + gzz[q] * c;
    }
    orc_fft3d(vx, nx2, ny2, nz2, -1);
    orc_fft3d(vy, nx2, ny2, nz2, -1);
    orc_fft3d(vz, nx2, ny2, nz2, -1);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                long site = i + (long)nx * j + nxy * k;
                long n = site;
                if (tabdip) {
                    if (tabdip[site] == 0) continue;
                    n = tabdip[site] - 1;
                }
                long ind = i + (long)nx2 * j + nxy2 * k;
                FFB[3 * n + 0] -= vx[ind] / dntotal;
                FFB[3 * n + 1] -= vy[ind] / dntotal;
                FFB[3 * n + 2] -= vz[ind] / dntotal;
            }
    free(v);
}

void orc_matvec_opt(const zc *G6, int nx, int ny, int nz, const zc *FFX, zc *FFB) {
    matvec_core(G6, nx, ny, nz, NULL, FFX, FFB);
}

void orc_matvec3(const zc *G6, int nx, int ny, int nz, const int *tabdip,
                 const zc *FFX, zc *FFB) {
    matvec_core(G6, nx, ny, nz, tabdip, FFX, FFB);
}

/* Dense direct sum of the same operator (no FFT):                            */
/* FFB_i -= sum_{j != i} T(r_i - r_j) FFX_j  over the dipoles (xs,ys,zs).      */
void orc_matvec_direct(int nd, const double *xs, const double *ys, const double *zs,
                       double k0, const zc *FFX, zc *FFB) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < nd; i++) {
        zc acc[3] = {0, 0, 0};
        for (int j = 0; j < nd; j++) {
            if (j == i) continue;
            zc t[9];
            orc_propa_espace_libre(xs[i], ys[i], zs[i], xs[j], ys[j], zs[j], k0, t);
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) acc[a] += t[a + 3 * b] * FFX[3 * j + b];
        }
        for (int a = 0; a < 3; a++) FFB[3 * i + a] -= acc[a];
    }
}

/* ------------------------------------------------------------------------- */
/* GPBICG reverse-communication state machine: cdmlib/gpbicg.f:81-338.        */
/* Work columns (0-based): 0 r0*, 1 p, 2 r, 3 y, 4 t, 5 Ap, 6 At, 7 u, 8 w,    */
/* 9 z, 10 x, 11 t(previous).  Same update order as the reference.            */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc alpha, beta, eta, dzeta, r0rn;
    double norm;
} gpbicg_state;

/* every2 = 1 is GPBICG2 (cdmlib/gpbicg2.f): the same iteration, but every
   even ITNO (not only the first) takes the zeta-only step (gpbicg2.f, label
   30: mod(ITNO,2) = 0). */
static void gpbicg(zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *itno,
                   int maxit, double tol, gpbicg_state *S, int *status, int *steperr, int every2) {
#define WK(c) (W + (size_t)(c) * n)
    zc *r0 = WK(0), *p = WK(1), *r = WK(2), *y = WK(3), *t = WK(4), *Ap = WK(5),
       *At = WK(6), *u = WK(7), *w = WK(8), *z = WK(9), *x = WK(10), *told = WK(11);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += creal(B[i] * conj(B[i]));
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10: {
    double rr = 0, ri = 0;
#pragma omp parallel for reduction(+ : rr, ri)
    for (long i = 0; i < n; i++) {
        p[i] = 0;
        r[i] = B[i] - xr[i];
        r0[i] = conj(r[i]);
        t[i] = 0;
        w[i] = 0;
        u[i] = 0;
        z[i] = 0;
        zc q = r0[i] * r[i];
        rr += creal(q);
        ri += cimag(q);
    }
    S->r0rn = rr + I * ri;
    S->beta = 0;
    *itno = -1;
}
L100:
    *itno += 1;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        p[i] = r[i] + S->beta * (p[i] - u[i]);
        xi[i] = p[i];
    }
    *nou = 2;
    return;
L20: {
    double cr = 0, ci = 0;
#pragma omp parallel for reduction(+ : cr, ci)
    for (long i = 0; i < n; i++) {
        Ap[i] = xr[i];
        zc q = r0[i] * Ap[i];
        cr += creal(q);
        ci += cimag(q);
    }
    zc c = cr + I * ci;
    if (c == 0) { *status = -1; *steperr = 1; return; }
    S->alpha = S->r0rn / c;
    zc al = S->alpha;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        y[i] = t[i] - r[i] + al * (Ap[i] - w[i]);
        told[i] = t[i];
        t[i] = r[i] - al * Ap[i];
        xi[i] = t[i];
    }
    *nou = 3;
    return;
}
L30: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) At[i] = xr[i];
    if (every2 ? *itno % 2 == 0 : *itno == 0) {
        double dr = 0, di = 0, cr = 0, ci = 0;
#pragma omp parallel for reduction(+ : dr, di, cr, ci)
        for (long i = 0; i < n; i++) {
            zc a = conj(At[i]) * t[i];
            zc b = conj(At[i]) * At[i];
            dr += creal(a); di += cimag(a);
            cr += creal(b); ci += cimag(b);
        }
        S->eta = 0;
        zc c = cr + I * ci;
        if (c == 0) { *status = -1; *steperr = 2; return; }
        S->dzeta = (dr + I * di) / c;
    } else {
        double s[10] = {0};
#pragma omp parallel for reduction(+ : s[:10])
        for (long i = 0; i < n; i++) {
            zc c1 = conj(At[i]) * At[i];
            zc c2 = conj(y[i]) * y[i];
            zc c3 = conj(At[i]) * y[i];
            zc c4 = conj(At[i]) * t[i];
            zc c5 = conj(y[i]) * t[i];
            s[0] += creal(c1); s[1] += cimag(c1);
            s[2] += creal(c2); s[3] += cimag(c2);
            s[4] += creal(c3); s[5] += cimag(c3);
            s[6] += creal(c4); s[7] += cimag(c4);
            s[8] += creal(c5); s[9] += cimag(c5);
        }
        zc c1 = s[0] + I * s[1], c2 = s[2] + I * s[3], c3 = s[4] + I * s[5],
           c4 = s[6] + I * s[7], c5 = s[8] + I * s[9];
        zc c = c1 * c2 - c3 * conj(c3);
        if (c == 0) { *status = -1; *steperr = 3; return; }
        S->dzeta = (c2 * c4 - c5 * c3) / c;
        S->eta = (c1 * c5 - conj(c3) * c4) / c;
    }
    double res = 0;
    zc dz = S->dzeta, et = S->eta, al = S->alpha, be = S->beta;
#pragma omp parallel for reduction(+ : res)
    for (long i = 0; i < n; i++) {
        u[i] = dz * Ap[i] + et * (told[i] - r[i] + be * u[i]);
        z[i] = dz * r[i] + et * z[i] - al * u[i];
        x[i] = x[i] + al * p[i] + z[i];
        r[i] = t[i] - et * y[i] - dz * At[i];
        res += creal(r[i] * conj(r[i]));
    }
    res = sqrt(res) / S->norm;
    if (res <= tol) {
        *status = 1;
#pragma omp parallel for
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *nou = 4;
        return;
    }
}
L40: {
    double cr = 0, ci = 0;
#pragma omp parallel for reduction(+ : cr, ci)
    for (long i = 0; i < n; i++) {
        zc q = r0[i] * r[i];
        cr += creal(q);
        ci += cimag(q);
    }
    zc c = cr + I * ci;
    if (S->r0rn == 0) { *status = -1; *steperr = 4; return; }
    S->beta = S->alpha * c / S->dzeta / S->r0rn;
    S->r0rn = c;
    zc be = S->beta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) w[i] = At[i] + be * Ap[i];
}
    if (*itno <= maxit) goto L100;
    *status = 1;
    *steperr = 0;
#pragma omp parallel for
    for (long i = 0; i < n; i++) xi[i] = x[i];
}

/* ------------------------------------------------------------------------- */
/* QMR-BiCGSTAB reverse-communication state machine: cdmlib/qmrbicgstab.f.    */
/* methode 1 or 2 selects the omega formula (qmrbicgstab.f:165-185).          */
/* Work columns: 0 r, 1 p, 2 v, 3 d, 4 rtilde0, 5 s, 6 xtilde, 7 dtilde, 8 t. */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc alpha, rho, omega, tau, taut, theta, thetat, eta, etat;
    double norm, residu;
} qmr_state;

static zc zsum(const zc *a, const zc *b, long n, int conja) {
    double sr = 0, si = 0;
#pragma omp parallel for reduction(+ : sr, si)
    for (long i = 0; i < n; i++) {
        zc q = (conja ? conj(a[i]) : a[i]) * b[i];
        sr += creal(q);
        si += cimag(q);
    }
    return sr + I * si;
}

static void qmrbicgstab(zc *x, zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W,
                        int *itno, int maxit, double tol, qmr_state *S, int methode,
                        int *status, int *steperr) {
#define WK(c) (W + (size_t)(c) * n)
    zc *r = WK(0), *p = WK(1), *v = WK(2), *d = WK(3), *rt = WK(4), *s = WK(5),
       *xt = WK(6), *dt = WK(7), *t = WK(8);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += creal(B[i] * conj(B[i]));
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        r[i] = B[i] - xr[i];
        p[i] = 0;
        v[i] = 0;
        d[i] = 0;
        rt[i] = r[i];
    }
    zc c = zsum(r, r, n, 1); /* sum r * conj(r) */
    S->rho = 1;
    S->alpha = 1;
    S->omega = 1;
    S->tau = csqrt(c);
    S->theta = 0;
    S->eta = 0;
    *itno = 0;
}
L100:
    *itno += 1;
    {
        zc rho0 = S->rho;
        S->rho = zsum(rt, r, n, 1);
        zc beta = S->rho * S->alpha / rho0 / S->omega;
        zc om = S->omega;
#pragma omp parallel for
        for (long i = 0; i < n; i++) {
            p[i] = r[i] + beta * (p[i] - om * v[i]);
            xi[i] = p[i];
        }
    }
    *nou = 2;
    return;
L20: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) v[i] = xr[i];
    zc a = zsum(rt, v, n, 1);
    if (cabs(a) == 0.0) { *status = -1; *steperr = 1; return; }
    S->alpha = S->rho / a;
    zc al = S->alpha;
#pragma omp parallel for
    for (long i = 0; i < n; i++) s[i] = r[i] - al * v[i];
    zc th = zsum(s, s, n, 1);
    if (cabs(S->tau) == 0.0) { *status = -1; *steperr = 2; return; }
    S->thetat = csqrt(th) / S->tau;
    zc c = 1.0 / csqrt(1.0 + S->thetat * S->thetat);
    S->taut = S->tau * S->thetat * c;
    S->etat = c * c * S->alpha;
    zc f = S->theta * S->theta * S->eta / S->alpha;
    zc et = S->etat;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        dt[i] = p[i] + f * d[i];
        xt[i] = x[i] + et * dt[i];
        xi[i] = s[i];
    }
    *nou = 3;
    return;
}
L30: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) t[i] = xr[i];
    zc om, ct;
    if (methode == 1) {
        om = zsum(t, t, n, 1);
        ct = zsum(s, t, n, 1);
    } else {
        om = zsum(s, t, n, 1);
        ct = zsum(s, s, n, 1);
    }
    if (cabs(om) == 0.0) { *status = -1; *steperr = 3; return; }
    S->omega = ct / om;
    zc omg = S->omega;
#pragma omp parallel for
    for (long i = 0; i < n; i++) r[i] = s[i] - omg * t[i];
    zc th = zsum(r, r, n, 1);
    if (cabs(S->taut) == 0.0) { *status = -1; *steperr = 4; return; }
    S->theta = csqrt(th) / S->taut;
    zc c = 1.0 / csqrt(1.0 + S->theta * S->theta);
    S->tau = S->taut * S->theta * c;
    S->eta = c * c * S->omega;
    if (cabs(S->omega) == 0.0) { *status = -1; *steperr = 5; return; }
    zc f = S->thetat * S->thetat * S->etat / S->omega;
    zc et = S->eta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        d[i] = s[i] + f * dt[i];
        x[i] = xt[i] + et * d[i];
    }
    S->residu = sqrt((double)(*itno + 1)) * cabs(S->tau) / S->norm;
    if (S->residu <= tol) {
        *status = 1;
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *nou = 4;
        return;
    }
}
L40:
    if (*itno <= maxit) goto L100;
    /* The reference passes the same variable as ITNO and MAXIT
       (inverserigopt.f:813-815), so it never leaves here; the restatement caps
       the loop at nlim iterations and ends like GPBICG does at MAXIT
       (gpbicg.f:327-336): status 1 with the current iterate. */
    *status = 1;
    *steperr = 0;
    for (long i = 0; i < n; i++) xi[i] = x[i];
    *nou = 4;
}

/* ------------------------------------------------------------------------- */
/* BiCGSTAB reverse-communication state machine: cdmlib/pimzbicgstab.f:1-216. */
/* x is the caller's solution array (FFLOC in the reference).  Work columns:  */
/* 0 r, 1 rtilde, 2 p, 4 s, 5 t, 6 v, 7 A x0.  The reference keeps NORM as the */
/* SQUARED norm of the initial residual, takes rho = r^H r (not rtilde^H r),  */
/* stops when ||r||^2 / NORM <= tol / 10 and reports ITNO > MAXIT as an error. */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc alpha, omega, rho;
    double norm;
} bicgstab_state;

static void bicgstab(zc *x, zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *itno,
                     int maxit, double tol, bicgstab_state *S, int *status, int *steperr) {
#define WK(c) (W + (size_t)(c) * n)
    zc *r = WK(0), *rt = WK(1), *p = WK(2), *s = WK(4), *t = WK(5), *v = WK(6), *ax0 = WK(7);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L100;
    *status = 0;
    *steperr = -1;
    for (long i = 0; i < n; i++) {
        r[i] = B[i];
        x[i] = xi[i];
    }
    *nou = 1;
    return;
L10: {
    double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
    for (long i = 0; i < n; i++) {
        ax0[i] = xr[i];
        r[i] = r[i] - ax0[i];
        nrm += creal(r[i] * conj(r[i]));
        rt[i] = r[i];
        p[i] = 0;
        v[i] = 0;
    }
    S->norm = nrm;
}
    S->rho = 1;
    S->alpha = 1;
    S->omega = 1;
    *itno = 0;
L100: {
    *itno += 1;
    const zc rho0 = S->rho;
    S->rho = zsum(r, r, n, 1);
    const zc kappa = rho0 * S->omega;
    if (cabs(kappa) == 0.0) {
        *status = -3;
        *steperr = 6;
        return;
    }
    const zc beta = S->rho * S->alpha / kappa, om = S->omega;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        const zc q = p[i] - om * v[i];
        p[i] = r[i] + beta * q;
        xi[i] = p[i];
    }
    *nou = 2;
    return;
}
L20: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) v[i] = xr[i];
    const zc xxi = zsum(rt, v, n, 1);
    if (cabs(xxi) == 0.0) {
        *status = -3;
        *steperr = 10;
        return;
    }
    S->alpha = S->rho / xxi;
    const zc al = S->alpha;
#pragma omp parallel for
    for (long i = 0; i < n; i++) s[i] = r[i] - al * v[i];
    const zc kappa = csqrt(zsum(s, s, n, 1));
    if (cabs(kappa) < 1e-15) {
        *status = -2;
        *steperr = 12;
        for (long i = 0; i < n; i++) x[i] = p[i];
        return;
    }
    for (long i = 0; i < n; i++) xi[i] = s[i];
    *nou = 3;
    return;
}
L30: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) t[i] = xr[i];
    const zc c1 = zsum(t, t, n, 1), c2 = zsum(t, s, n, 1);
    if (cabs(c1) == 0.0) {
        *status = -3;
        *steperr = 14;
        return;
    }
    S->omega = c2 / c1;
    const zc al = S->alpha, om = S->omega;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        x[i] = x[i] + al * p[i] + om * s[i];
        r[i] = s[i] - om * t[i];
    }
    const zc c = zsum(r, r, n, 1) / S->norm;
    if (*itno > maxit) {
        *status = -1;
        *itno = maxit;
        return;
    }
    if (cabs(c) <= tol / 10.0) {
        *status = 1;
        *nou = 4;
        return;
    }
    goto L100;
}
}

/* ------------------------------------------------------------------------- */
/* Conjugate gradient for complex-symmetric systems (dot products without     */
/* conjugation), reverse communication: cdmlib/zcg.f:1-179.  One mat-vec per  */
/* iteration: w = A p is carried by the recurrence w = A r + beta w.  Work    */
/* columns: 0 x, 1 r, 2 p, 3 s = A r, 4 w.  Where the reference stops the     */
/* program (xi = p^T A p = 0) the restatement returns status -3.              */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc rho0, xxi;
    double norm;
} cg_state;

static void zcg(zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *nloop, int maxit,
                double tol, cg_state *S, int *status) {
#define WK(c) (W + (size_t)(c) * n)
    zc *x = WK(0), *r = WK(1), *p = WK(2), *s = WK(3), *w = WK(4);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *nou = 1;
    *status = 0;
    for (long i = 0; i < n; i++) x[i] = xi[i];
    return;
L10: {
    double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
    for (long i = 0; i < n; i++) {
        r[i] = B[i] - xr[i];
        nrm += creal(B[i] * conj(B[i]));
        p[i] = r[i];
        xi[i] = p[i];
    }
    S->norm = sqrt(nrm);
    S->rho0 = zsum(r, r, n, 0);
    *nou = 2;
    return;
}
L20: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) w[i] = xr[i];
    S->xxi = zsum(p, w, n, 0);
    if (S->xxi == 0) {
        *status = -3;
        return;
    }
}
L50: {
    *nloop += 1;
    if (*nloop >= maxit) {
        *status = -4;
        *nou = 0;
        for (long i = 0; i < n; i++) xi[i] = x[i];
        return;
    }
    const zc al = S->rho0 / S->xxi;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        x[i] = x[i] + al * p[i];
        r[i] = r[i] - al * w[i];
    }
    const double tole = sqrt(cabs(zsum(r, r, n, 1))) / S->norm;
    if (tole <= tol) {
        *status = 1;
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *nou = 4;
        return;
    }
}
L40:
    *nou = 3;
    for (long i = 0; i < n; i++) xi[i] = r[i];
    return;
L30: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) s[i] = xr[i];
    const zc rho = zsum(r, r, n, 0), delta = zsum(r, s, n, 0);
    const zc beta = rho / S->rho0;
    S->rho0 = rho;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        p[i] = r[i] + beta * p[i];
        w[i] = s[i] + beta * w[i];
    }
    S->xxi = delta - beta * beta * S->xxi;
    goto L50;
}
}

/* ------------------------------------------------------------------------- */
/* TFQMR reverse-communication state machine: cdmlib/tfqmr.f:1-218.  x is the */
/* caller's solution array (FFloc).  Work columns: 0 u, 1 w, 2 r, 3 v, 4 d,   */
/* 5 rtilde, 6 u(next), 7 A u, 8 A u (previous).  Passes alternate: an even   */
/* pass forms alpha and the next u, an odd pass rho, beta and v.  Stop when   */
/* sqrt(ITNO+1) |tau| / NORM <= tol.  Past MAXIT the reference routine falls  */
/* off its end without a status and its driver loops for ever; the            */
/* restatement ends there with status 1 and the current iterate.             */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc alpha, beta, rho, tau, theta, eta;
    double norm;
} tfqmr_state;

static void tfqmr(zc *x, zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *itno, int maxit,
                  double tol, tfqmr_state *S, int *status, int *steperr) {
#define WK(c) (W + (size_t)(c) * n)
    zc *u = WK(0), *w = WK(1), *r = WK(2), *v = WK(3), *d = WK(4), *rt = WK(5), *u1 = WK(6),
       *au = WK(7), *aup = WK(8);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += creal(B[i] * conj(B[i]));
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10:
    *nou = 2;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        r[i] = B[i] - xr[i];
        w[i] = r[i];
        u[i] = r[i];
        xi[i] = u[i];
    }
    return;
L20:
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        v[i] = xr[i];
        d[i] = 0;
        au[i] = v[i];
        rt[i] = r[i];
    }
    S->rho = zsum(rt, r, n, 1);
    S->tau = S->norm;
    S->theta = 0;
    S->eta = 0;
    *itno = -1;
L100: {
    *itno += 1;
    if (*itno % 2 == 0) {
        S->alpha = S->rho / zsum(rt, v, n, 1);
        const zc al = S->alpha;
#pragma omp parallel for
        for (long i = 0; i < n; i++) u1[i] = u[i] - al * v[i];
    }
    const zc al = S->alpha, f = S->theta * S->theta / S->alpha * S->eta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        w[i] = w[i] - al * au[i];
        d[i] = u[i] + f * d[i];
    }
    S->theta = csqrt(zsum(w, w, n, 1)) / S->tau;
    const zc c = 1.0 / csqrt(1.0 + S->theta * S->theta);
    S->tau = S->tau * S->theta * c;
    S->eta = c * c * S->alpha;
    const zc et = S->eta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) x[i] = x[i] + et * d[i];
    if (sqrt((double)(*itno + 1)) * cabs(S->tau) / S->norm <= tol) {
        *status = 1;
        *nou = 4;
        return;
    }
}
L40:
    if (*itno % 2 == 1) {
        const zc rho0 = S->rho;
        S->rho = zsum(rt, w, n, 1);
        S->beta = S->rho / rho0;
        const zc be = S->beta;
#pragma omp parallel for
        for (long i = 0; i < n; i++) {
            u1[i] = w[i] + be * u[i];
            aup[i] = au[i];
        }
    }
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        xi[i] = u1[i];
        u[i] = u1[i];
    }
    *nou = 3;
    return;
L30:
    *nou = 3;
#pragma omp parallel for
    for (long i = 0; i < n; i++) au[i] = xr[i];
    if (*itno % 2 == 1) {
        const zc be = S->beta;
#pragma omp parallel for
        for (long i = 0; i < n; i++) v[i] = au[i] + be * (aup[i] + be * v[i]);
    }
    if (*itno <= maxit) goto L100;
    *status = 1;
    *steperr = 0;
    *nou = 4;
}

/* ------------------------------------------------------------------------- */
/* GPBiCGsafe reverse-communication state machine: cdmlib/gpbicgsafe.f.       */
/* The mat-vecs are A r and A u; A p is carried by Ap = Ar + beta (Ap - Au).  */
/* Work columns: 0 r0 (shadow), 1 p, 2 u, 3 r, 4 A u, 5 A r, 6 A p, 7 t,     */
/* 8 z, 9 y, 10 x.  Ends like GPBICG: status 1 past MAXIT with the iterate.   */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc alpha, beta, eta, dzeta, r0rn;
    double norm;
} gpsafe_state;

/* plus = 1 is GPBICGplus (cdmlib/gpbicgplus.f): the same iteration (it forms
   t and z before the second mat-vec instead of after), NORM summed as
   |b_i|^2 and zeta, eta written from the same five dot products in its own
   form. */
static void gpbicgsafe(zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *itno, int maxit,
                       double tol, gpsafe_state *S, int *status, int *steperr, int plus) {
#define WK(c) (W + (size_t)(c) * n)
    zc *r0 = WK(0), *p = WK(1), *u = WK(2), *r = WK(3), *au = WK(4), *ar = WK(5), *ap = WK(6), *t = WK(7),
       *z = WK(8), *y = WK(9), *x = WK(10);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += plus ? cabs(B[i]) * cabs(B[i]) : creal(B[i] * conj(B[i]));
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10:
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        r0[i] = B[i] - xr[i];
        p[i] = 0;
        u[i] = 0;
        z[i] = 0;
        ap[i] = 0;
        au[i] = 0;
        y[i] = 0;
        r[i] = r0[i];
    }
    S->r0rn = zsum(r0, r0, n, 1);
    S->beta = 0;
    *itno = -1;
L100: {
    *itno += 1;
    const zc be = S->beta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        p[i] = r[i] + be * (p[i] - u[i]);
        xi[i] = r[i];
    }
    *nou = 2;
    return;
}
L20: {
    const zc be = S->beta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        ar[i] = xr[i];
        ap[i] = ar[i] + be * (ap[i] - au[i]);
    }
    const zc c0 = zsum(r0, ap, n, 1);
    if (c0 == 0) {
        *status = -1;
        *steperr = 1;
        return;
    }
    S->alpha = S->r0rn / c0;
    if (*itno == 0) {
        S->eta = 0;
        const zc num = zsum(ar, r, n, 1), den = zsum(ar, ar, n, 1);
        if (den == 0) {
            *status = -1;
            *steperr = 2;
            return;
        }
        S->dzeta = num / den;
    } else {
        if (plus) {
            const zc c1 = zsum(y, y, n, 1), c2 = zsum(ar, ar, n, 1), c3 = zsum(ar, r, n, 1),
                     c4 = zsum(y, r, n, 1), c5 = zsum(y, ar, n, 1);
            const zc c = c1 * c2 - c5 * conj(c5);
            if (c == 0) {
                *status = -1;
                *steperr = 3;
                return;
            }
            S->dzeta = (c1 * c3 - c4 * conj(c5)) / c;
            S->eta = (c2 * c4 - c5 * c3) / c;
        } else {
            const zc c1 = zsum(y, y, n, 1), c2 = zsum(ar, r, n, 1), c3 = zsum(y, r, n, 1),
                     c4 = zsum(ar, y, n, 1), c5 = zsum(ar, ar, n, 1);
            const zc c = c5 * c1 - c4 * conj(c4);
            if (c == 0) {
                *status = -1;
                *steperr = 3;
                return;
            }
            S->dzeta = (c1 * c2 - c3 * c4) / c;
            S->eta = (c5 * c3 - conj(c4) * c2) / c;
        }
    }
    const zc dz = S->dzeta, et = S->eta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        u[i] = dz * ap[i] + et * (y[i] + be * u[i]);
        xi[i] = u[i];
    }
    *nou = 3;
    return;
}
L30: {
    const zc al = S->alpha, dz = S->dzeta, et = S->eta;
    double res = 0;
#pragma omp parallel for reduction(+ : res)
    for (long i = 0; i < n; i++) {
        au[i] = xr[i];
        t[i] = r[i] - al * ap[i];
        z[i] = dz * r[i] + et * z[i] - al * u[i];
        y[i] = dz * ar[i] + et * y[i] - al * au[i];
        x[i] = x[i] + al * p[i] + z[i];
        r[i] = t[i] - y[i];
        res += creal(r[i] * conj(r[i]));
    }
    if (sqrt(res) / S->norm <= tol) {
        *status = 1;
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *nou = 4;
        return;
    }
}
L40: {
    const zc c = zsum(r0, r, n, 1);
    if (S->r0rn == 0) {
        *status = -1;
        *steperr = 4;
        return;
    }
    S->beta = S->alpha * c / S->dzeta / S->r0rn;
    S->r0rn = c;
    if (*itno <= maxit) goto L100;
    *status = 1;
    for (long i = 0; i < n; i++) xi[i] = x[i];
    *nou = 4;
}
}

/* ------------------------------------------------------------------------- */
/* GPBiCG-AR (associate residual) reverse communication: cdmlib/gpbicgar.f.   */
/* Mat-vecs A u then A r; A p carried by Ap = Ar + beta (Ap - Au).  Work      */
/* columns: 0 r0 (shadow), 1 p, 2 r, 3 t, 4 z, 5 Ap, 6 Ar, 7 u, 8 y, 10 x,    */
/* 11 Au.  The reference never sets p, u, Ap, Au, t before the first pass     */
/* (they are multiplied by beta = 0 there); they start at zero here.          */
/* ------------------------------------------------------------------------- */
static void gpbicgar(zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *itno, int maxit,
                     double tol, gpsafe_state *S, int *status, int *steperr) {
#define WK(c) (W + (size_t)(c) * n)
    zc *r0 = WK(0), *p = WK(1), *r = WK(2), *t = WK(3), *z = WK(4), *ap = WK(5), *ar = WK(6), *u = WK(7),
       *y = WK(8), *x = WK(10), *au = WK(11);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 4) goto L40;
    if (*nou == 5) goto L50;
    if (*nou == 6) goto L60;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += creal(B[i] * conj(B[i]));
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10:
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        r0[i] = B[i] - xr[i];
        r[i] = r0[i];
        xi[i] = r0[i];
        p[i] = u[i] = ap[i] = au[i] = t[i] = z[i] = y[i] = 0;
    }
    S->r0rn = zsum(r0, r0, n, 1);
    *nou = 2;
    return;
L20:
    S->beta = 0;
#pragma omp parallel for
    for (long i = 0; i < n; i++) ar[i] = xr[i];
    *itno = -1;
L100: {
    *itno += 1;
    const zc be = S->beta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        p[i] = r[i] + be * (p[i] - u[i]);
        ap[i] = ar[i] + be * (ap[i] - au[i]);
    }
    const zc c0 = zsum(r0, ap, n, 1);
    if (cabs(c0) == 0.0) {
        *status = -1;
        *steperr = 1;
        return;
    }
    S->alpha = S->r0rn / c0;
    if (*itno != 0) {
        const zc c1 = zsum(y, y, n, 1), c2 = zsum(ar, r, n, 1), c3 = zsum(y, r, n, 1),
                 c4 = zsum(ar, y, n, 1), c5 = zsum(ar, ar, n, 1);
        const zc c = c5 * c1 - c4 * conj(c4);
        if (cabs(c) == 0.0) {
            *status = -1;
            *steperr = 3;
            return;
        }
        S->dzeta = (c1 * c2 - c3 * c4) / c;
        S->eta = (c5 * c3 - conj(c4) * c2) / c;
    } else {
        const zc den = zsum(ar, ar, n, 1), num = zsum(ar, r, n, 1);
        if (cabs(den) == 0.0) {
            *status = -1;
            *steperr = 2;
            return;
        }
        S->dzeta = num / den;
        S->eta = 0;
    }
    const zc dz = S->dzeta, et = S->eta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        u[i] = dz * ap[i] + et * (t[i] - r[i] + be * u[i]);
        xi[i] = u[i];
    }
    *nou = 4;
    return;
}
L40: {
    const zc al = S->alpha, dz = S->dzeta, et = S->eta;
    double res = 0;
#pragma omp parallel for reduction(+ : res)
    for (long i = 0; i < n; i++) {
        au[i] = xr[i];
        t[i] = r[i] - al * ap[i];
        z[i] = dz * r[i] + et * z[i] - al * u[i];
        y[i] = dz * ar[i] + et * y[i] - al * au[i];
        x[i] = x[i] + al * p[i] + z[i];
        r[i] = t[i] - y[i];
        res += creal(r[i] * conj(r[i]));
    }
    if (sqrt(res) / S->norm <= tol) {
        *status = 1;
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *nou = 6;
        return;
    }
}
L60:
    *nou = 5;
    for (long i = 0; i < n; i++) xi[i] = r[i];
    return;
L50: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) ar[i] = xr[i];
    const zc c = zsum(r0, r, n, 1);
    if (cabs(S->r0rn) == 0.0) {
        *status = -1;
        *steperr = 5;
        return;
    }
    if (cabs(S->dzeta) == 0.0) {
        *status = -1;
        *steperr = 6;
        return;
    }
    S->beta = S->alpha * c / S->dzeta / S->r0rn;
    S->r0rn = c;
    if (*itno <= maxit) goto L100;
    *status = 1;
    for (long i = 0; i < n; i++) xi[i] = x[i];
    *nou = 6;
}
}

/* ------------------------------------------------------------------------- */
/* BiCGStar-plus reverse communication: cdmlib/bicgstarplus.f (subroutine     */
/* GPBICGSTARPLUS).  The shadow vector is conj(r0) with unconjugated dots.    */
/* Work columns: 0 conj(r0), 1 A r, 2 r, 3 w4, 4 w5, 5 w6, 6 w7, 7 w8, 8 w9,  */
/* 9 A w4, 10 x, 11 w12.  On its first pass the reference adds into two       */
/* accumulators it never cleared (bicgstarplus.f, label 20); they start at 0  */
/* here.  Ends like GPBICG (status 1 with the iterate past MAXIT).            */
/* ------------------------------------------------------------------------- */
static void bicgstarplus(zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *itno, int maxit,
                         double tol, gpsafe_state *S, int *status, int *steperr) {
#define WK(c) (W + (size_t)(c) * n)
    zc *r0s = WK(0), *ar = WK(1), *r = WK(2), *w4 = WK(3), *w5 = WK(4), *w6 = WK(5), *w7 = WK(6), *w8 = WK(7),
       *w9 = WK(8), *aw4 = WK(9), *x = WK(10), *w12 = WK(11);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += creal(B[i] * conj(B[i]));
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10:
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        r[i] = B[i] - xr[i];
        r0s[i] = conj(r[i]);
        w8[i] = w4[i] = w9[i] = w5[i] = w12[i] = 0;
    }
    S->r0rn = zsum(r0s, r, n, 0);
    *itno = -1;
L100:
    *itno += 1;
    for (long i = 0; i < n; i++) xi[i] = r[i];
    *nou = 2;
    return;
L20: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) ar[i] = xr[i];
    if (*itno == 0) {
        S->eta = 0;
        S->beta = 0;
        const zc an = zsum(r0s, r, n, 0), zn = zsum(ar, r, n, 1), c1 = zsum(ar, ar, n, 1),
                 c2 = zsum(r0s, ar, n, 0);
        S->r0rn = an;
        if (c1 == 0) {
            *status = -1;
            *steperr = 2;
            return;
        }
        S->dzeta = zn / c1;
        if (c2 == 0) {
            *status = -1;
            *steperr = 3;
            return;
        }
        S->alpha = an / c2;
    } else {
        const zc c1 = zsum(r0s, r, n, 0), c2 = zsum(r0s, ar, n, 0), c3 = zsum(w5, w5, n, 1),
                 c4 = zsum(ar, r, n, 1), c5 = zsum(ar, w5, n, 1), c6 = zsum(w5, r, n, 1),
                 c7 = zsum(ar, ar, n, 1), c8 = zsum(r0s, w12, n, 0);
        if (S->dzeta == 0) {
            *status = -1;
            *steperr = 4;
            return;
        }
        if (S->r0rn == 0) {
            *status = -1;
            *steperr = 5;
            return;
        }
        S->beta = -S->alpha / S->dzeta * c1 / S->r0rn;
        const zc c = c2 - S->beta * c8;
        if (c == 0) {
            *status = -1;
            *steperr = 6;
            return;
        }
        S->alpha = c1 / c;
        const zc d = c7 * c3 - c5 * conj(c5);
        if (d == 0) {
            *status = -1;
            *steperr = 7;
            return;
        }
        S->dzeta = (c3 * c4 - c5 * c6) / d;
        S->eta = (c7 * c6 - conj(c5) * c4) / d;
        S->r0rn = c1;
    }
    const zc be = S->beta, dz = S->dzeta, et = S->eta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        w7[i] = ar[i] - be * w12[i];
        w6[i] = dz * r[i] + et * w9[i];
        w4[i] = dz * w7[i] + et * (w5[i] - be * w4[i]);
        xi[i] = w4[i];
    }
    *nou = 3;
    return;
}
L30: {
    const zc al = S->alpha, be = S->beta, dz = S->dzeta, et = S->eta;
    double res = 0;
#pragma omp parallel for reduction(+ : res)
    for (long i = 0; i < n; i++) {
        aw4[i] = xr[i];
        w8[i] = r[i] - be * w8[i] - w4[i];
        w12[i] = w7[i] - aw4[i];
        w9[i] = w6[i] - al * w4[i];
        const zc tmp = dz * ar[i] + et * w5[i];
        w5[i] = tmp - al * aw4[i];
        x[i] = x[i] + w6[i] + al * w8[i];
        r[i] = r[i] - tmp - al * w12[i];
        res += creal(r[i] * conj(r[i]));
    }
    if (sqrt(res) / S->norm <= tol) {
        *status = 1;
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *nou = 4;
        return;
    }
}
L40:
    if (*itno <= maxit) goto L100;
    *status = 1;
    *steperr = 0;
    for (long i = 0; i < n; i++) xi[i] = x[i];
    *nou = 4;
}

/* ------------------------------------------------------------------------- */
/* CORS reverse communication: cdmlib/cors.f.  Shadow conj(A r0) with         */
/* unconjugated dots; mat-vecs A r and A d.  Work columns: 0 shadow, 1 r,     */
/* 2 A r, 3 e, 4 h, 5 d, 6 f, 7 g, 8 q = A d, 9 x.  Past MAXIT the reference  */
/* returns work column 11, which it never writes; the restatement returns x.  */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc alpha, beta, rho, rhoa;
    double norm;
} cors_state;

static void cors(zc *xi, zc *xr, const zc *B, long n, int *nou, zc *W, int *itno, int maxit, double tol,
                 cors_state *S, int *status, int *steperr) {
#define WK(c) (W + (size_t)(c) * n)
    zc *rs = WK(0), *r = WK(1), *ar = WK(2), *e = WK(3), *h = WK(4), *d = WK(5), *f = WK(6), *g = WK(7),
       *q = WK(8), *x = WK(9);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += cabs(B[i]) * cabs(B[i]);
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10:
#pragma omp parallel for
    for (long i = 0; i < n; i++) r[i] = B[i] - xr[i];
    *itno = -1;
L100:
    *itno += 1;
    for (long i = 0; i < n; i++) xi[i] = r[i];
    *nou = 2;
    return;
L20:
    if (*itno == 0)
        for (long i = 0; i < n; i++) rs[i] = conj(xr[i]);
#pragma omp parallel for
    for (long i = 0; i < n; i++) ar[i] = xr[i];
    S->rho = zsum(rs, ar, n, 0);
    if (S->rho == 0) {
        *status = -1;
        *steperr = 1;
        return;
    }
    if (*itno == 0) {
        for (long i = 0; i < n; i++) {
            e[i] = r[i];
            h[i] = ar[i];
            d[i] = ar[i];
            xi[i] = d[i];
        }
    } else {
        S->beta = S->rho / S->rhoa;
        const zc be = S->beta;
#pragma omp parallel for
        for (long i = 0; i < n; i++) {
            e[i] = r[i] + be * f[i];
            h[i] = ar[i] + be * g[i];
            d[i] = h[i] + be * (g[i] + be * d[i]);
            xi[i] = d[i];
        }
    }
    *nou = 3;
    return;
L30: {
#pragma omp parallel for
    for (long i = 0; i < n; i++) q[i] = xr[i];
    const zc c = zsum(rs, q, n, 0);
    if (c == 0) {
        *status = -1;
        *steperr = 2;
        return;
    }
    S->alpha = S->rho / c;
    const zc al = S->alpha;
    double res = 0;
#pragma omp parallel for reduction(+ : res)
    for (long i = 0; i < n; i++) {
        f[i] = e[i] - al * d[i];
        g[i] = h[i] - al * q[i];
        x[i] = x[i] + al * (2.0 * e[i] - al * d[i]);
        r[i] = r[i] - al * (2.0 * h[i] - al * q[i]);
        res += cabs(r[i]) * cabs(r[i]);
    }
    if (sqrt(res) / S->norm <= tol) {
        *status = 1;
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *nou = 4;
        return;
    }
}
L40:
    S->rhoa = S->rho;
    if (*itno <= maxit) goto L100;
    *status = 1;
    for (long i = 0; i < n; i++) xi[i] = x[i];
    *nou = 4;
}

/* ------------------------------------------------------------------------- */
/* GPBiCOR reverse communication: cdmlib/gpbicor.f.  x is the caller's       */
/* solution array (FFloc).  ITNO counts from 1.  Work columns: 0 r0, 1 p,     */
/* 2 A r, 3 w4, 4 w5, 5 w6, 6 t, 7 w8, 8 w9, 9 r, 10 z, 11 w12, 12 q, 13 s.   */
/* The reference keeps q and s in the driver's xi and xr arrays (its driver   */
/* overwrites both after the return); past MAXIT it returns status 1 without */
/* setting the solution; the restatement returns x there.                    */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc alpha, beta, eta, dzeta, rho, rhoa;
    double norm;
} gpbicor_state;

static void gpbicor(zc *xi, zc *xr, const zc *B, zc *x, long n, int *nou, zc *W, int *itno, int maxit,
                    double tol, gpbicor_state *S, int *status, int *steperr) {
#define WK(c) (W + (size_t)(c) * n)
    zc *r0 = WK(0), *p = WK(1), *ar = WK(2), *w4 = WK(3), *w5 = WK(4), *w6 = WK(5), *t = WK(6), *w8 = WK(7),
       *w9 = WK(8), *r = WK(9), *z = WK(10), *w12 = WK(11), *q = WK(12), *s = WK(13);
#undef WK
    if (*nou == 1) goto L10;
    if (*nou == 2) goto L20;
    if (*nou == 3) goto L30;
    if (*nou == 4) goto L40;
    *status = 0;
    *steperr = -1;
    {
        double nrm = 0;
#pragma omp parallel for reduction(+ : nrm)
        for (long i = 0; i < n; i++) {
            x[i] = xi[i];
            nrm += creal(B[i] * conj(B[i]));
        }
        S->norm = sqrt(nrm);
    }
    *nou = 1;
    return;
L10:
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        r0[i] = B[i] - xr[i];
        r[i] = r0[i];
        z[i] = 0;
    }
    *itno = 0;
L100:
    *itno += 1;
    for (long i = 0; i < n; i++) xi[i] = r[i];
    *nou = 2;
    return;
L20:
#pragma omp parallel for
    for (long i = 0; i < n; i++) ar[i] = xr[i];
    S->rho = zsum(r0, ar, n, 1);
    if (S->rho == 0) {
        *status = -1;
        *steperr = 1;
        return;
    }
    if (*itno == 1) {
        S->beta = 0;
        for (long i = 0; i < n; i++) {
            p[i] = r0[i];
            w4[i] = ar[i];
            w12[i] = w5[i] = w8[i] = w9[i] = w6[i] = 0;
            xi[i] = w4[i];
        }
    } else {
        S->beta = S->rho / S->rhoa * S->alpha / S->dzeta;
        const zc be = S->beta;
#pragma omp parallel for
        for (long i = 0; i < n; i++) {
            w5[i] = w6[i] + be * w4[i];
            p[i] = r[i] + be * (p[i] - w8[i]);
            w4[i] = ar[i] + be * (w4[i] - w9[i]);
            xi[i] = w4[i];
        }
    }
    *nou = 3;
    return;
L30: {
    const zc c = zsum(r0, xr, n, 1);
    if (c == 0) {
        *status = -1;
        *steperr = 2;
        return;
    }
    S->alpha = S->rho / c;
    const zc al = S->alpha;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        q[i] = w12[i] - r[i] + al * (w4[i] - w5[i]);
        t[i] = r[i] - al * w4[i];
        s[i] = ar[i] - al * xr[i];
    }
    if (*itno == 1) {
        S->eta = 0;
        const zc num = zsum(s, t, n, 1), den = zsum(s, s, n, 1);
        if (den == 0) {
            *status = -1;
            *steperr = 3;
            return;
        }
        S->dzeta = num / den;
    } else {
        const zc c1 = zsum(s, s, n, 1), c2 = zsum(q, t, n, 1), c3 = zsum(q, s, n, 1), c4 = zsum(s, t, n, 1),
                 c5 = zsum(q, q, n, 1);
        const zc cc = c1 * c5 - c3 * conj(c3);
        if (cc == 0) {
            *status = -1;
            *steperr = 4;
            return;
        }
        S->eta = (c1 * c2 - c3 * c4) / cc;
        S->dzeta = (c5 * c4 - c2 * conj(c3)) / cc;
    }
    const zc be = S->beta, dz = S->dzeta, et = S->eta;
#pragma omp parallel for
    for (long i = 0; i < n; i++) {
        w8[i] = dz * w4[i] + et * (w12[i] - r[i] + be * w8[i]);
        w9[i] = dz * (ar[i] - s[i]) / al + et * (w6[i] - ar[i] + be * w9[i]);
        z[i] = dz * r[i] + et * z[i] - al * w8[i];
    }
    double res = 0;
#pragma omp parallel for reduction(+ : res)
    for (long i = 0; i < n; i++) {
        r[i] = t[i] - et * q[i] - dz * s[i];
        res += creal(r[i] * conj(r[i]));
        x[i] = x[i] + al * p[i] + z[i];
        w6[i] = s[i];
        w12[i] = t[i];
    }
    if (sqrt(res) / S->norm <= tol) {
        for (long i = 0; i < n; i++) xi[i] = x[i];
        *status = 1;
        *nou = 4;
        return;
    }
}
L40:
    S->rhoa = S->rho;
    if (*itno <= maxit) goto L100;
    *status = 1;
    for (long i = 0; i < n; i++) xi[i] = x[i];
    *nou = 4;
}

/* ------------------------------------------------------------------------- */
/* Solver driver: cdmlib/inverserigopt.f:1-107 (GPBICG1), :811-942             */
/* (QMRBICGSTAB1/2) and cdmlib/inverserig.f (tabdip != NULL).                  */
/* Returns nstop; infostr receives the reference's messages (space padded to   */
/* 64 characters like a Fortran character(64)).                               */
/* ------------------------------------------------------------------------- */
static void set_info(char *infostr, const char *msg) {
    size_t L = strlen(msg);
    memset(infostr, ' ', 64);
    memcpy(infostr, msg, L > 64 ? 64 : L);
}

static void apply_pola(long nbs, long nmax, const zc *pol, const zc *xr, zc *xi) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nbs; i++) {
        for (int a = 0; a < 3; a++) {
            zc acc = 0;
            for (int b = 0; b < 3; b++) acc += pol[i + nmax * a + 3 * nmax * b] * xr[3 * i + b];
            xi[3 * i + a] = acc;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* QMR without look-ahead, PIMZQMR (cdmlib/qmrpim.f:1-270), behind methodeit  */
/* 'QMRCLA'.  Reverse communication: on return *nt = 1 asks for A xi, *nt = 2 */
/* for A^T xi (inverserigopt.f:528-584).  W columns 1..9 (0-based here).      */
/* xs is the solution (the reference passes FFloc).                           */
/* ------------------------------------------------------------------------- */
typedef struct {
    zc lambda, kappa, theta, gamma, ksi, rho, eps, mu, tau, dots1, dots2, dots3, dots4;
    double norm;
} qmrcla_state;

static void qmrcla(zc *xs, zc *xi, const zc *xr, const zc *B, long n, int *nou, int *nt, zc *W,
                   int *itno, int maxit, double tol, qmrcla_state *s, int *status, int *steperr) {
#define WC(c) (W + (size_t)(c - 1) * n)
    zc *w1 = WC(1), *w2 = WC(2), *w3 = WC(3), *w4 = WC(4), *w5 = WC(5), *w6 = WC(6), *w7 = WC(7),
       *w8 = WC(8), *w9 = WC(9);
#undef WC
    switch (*nou) {
    case 0: {
        s->lambda = 1.0;
        s->kappa = -1.0;
        s->theta = -1.0;
        double nrm = 0;
        for (long i = 0; i < n; i++) {
            nrm += creal(B[i] * conj(B[i]));
            xs[i] = xi[i];
        }
        s->norm = sqrt(nrm);
        *status = 0;
        *steperr = -1;
        *itno = 0;
        *nou = 1;
        *nt = 1;
        return;
    }
    case 1: {
        zc d1 = 0, d2 = 0, d3 = 0;
        for (long i = 0; i < n; i++) {
            w3[i] = xr[i];
            w1[i] = B[i] - w3[i];
            w7[i] = w1[i];
            w8[i] = w1[i];
            w2[i] = w4[i] = w5[i] = w6[i] = 0;
            d1 += w7[i] * conj(w7[i]);
            d2 += w8[i] * conj(w8[i]);
            d3 += w7[i] * w8[i];
            xi[i] = w8[i];
        }
        s->dots1 = d1; s->dots2 = d2; s->dots3 = d3;
        *nt = 2;
        *nou = 2;
        return;
    }
    case 2: {
        zc d4 = 0;
        for (long i = 0; i < n; i++) {
            w9[i] = xr[i];
            d4 += w7[i] * w9[i];
        }
        s->dots4 = d4;
        s->gamma = csqrt(s->dots1);
        s->ksi = csqrt(s->dots2);
        s->rho = s->dots3;
        s->eps = s->dots4;
        s->mu = 0;
        if (cabs(s->rho) == 0.0) {
            *itno = 0;
            *status = -3;
            *steperr = 5;
            return;
        }
        s->tau = s->eps / s->rho;
        goto label100;
    }
    case 3: {
        zc d1 = 0, d2 = 0, d3 = 0;
        for (long i = 0; i < n; i++) {
            w3[i] = xr[i];
            w7[i] = w3[i] - s->tau / s->gamma * w7[i];
            w8[i] = w4[i] - s->tau / s->ksi * w8[i];
            d1 += w7[i] * conj(w7[i]);
            d2 += w8[i] * conj(w8[i]);
            d3 += w7[i] * w8[i];
            xi[i] = w8[i];
        }
        s->dots1 = d1; s->dots2 = d2; s->dots3 = d3;
        *nt = 2;
        *nou = 4;
        return;
    }
    case 4: {
        zc d4 = 0;
        for (long i = 0; i < n; i++) {
            w9[i] = xr[i];
            d4 += w7[i] * w9[i];
        }
        s->dots4 = d4;
        zc gamma0 = s->gamma, ksi0 = s->ksi, rho0 = s->rho;
        s->gamma = csqrt(s->dots1);
        s->ksi = csqrt(s->dots2);
        s->rho = s->dots3;
        s->eps = s->dots4;
        zc den = s->gamma * s->tau * rho0;
        if (cabs(den) == 0.0) { *status = -3; *steperr = 12; return; }
        s->mu = (gamma0 * ksi0 * s->rho) / den;
        if (cabs(s->rho) == 0.0) { *status = -3; *steperr = 13; return; }
        zc tau0 = s->tau;
        s->tau = s->eps / s->rho - s->gamma * s->mu;
        double abstau02 = pow(cabs(tau0), 2.0), absgamma2 = pow(cabs(s->gamma), 2.0);
        den = s->lambda * abstau02 + absgamma2;
        if (cabs(den) == 0.0) { *status = -3; *steperr = 14; return; }
        s->theta = (abstau02 * (1.0 - s->lambda)) / den;
        zc kappa0 = s->kappa;
        s->kappa = -(gamma0 * conj(tau0) * kappa0) / den;
        zc lambda0 = s->lambda;
        s->lambda = lambda0 * abstau02 / den;
        zc tmp1 = 0;
        for (long i = 0; i < n; i++) {
            w5[i] = s->theta * w5[i] + s->kappa * w2[i];
            w6[i] = s->theta * w6[i] + s->kappa * w3[i];
            xs[i] = xs[i] + w5[i];
            w1[i] = w1[i] - w6[i];
            tmp1 += w1[i] * conj(w1[i]);
        }
        double tole = sqrt(cabs(tmp1)) / s->norm;
        if (tole <= tol) {
            *nou = 5;
            *status = 1;
            return;
        }
        if (*itno > maxit) {
            *status = -1;
            *itno = maxit;
        }
        goto label100;
    }
    default:
        goto label100;
    }
label100:
    *itno += 1;
    if (cabs(s->gamma) == 0.0) { *status = -3; *steperr = 6; return; }
    if (cabs(s->ksi) == 0.0) { *status = -3; *steperr = 7; return; }
    for (long i = 0; i < n; i++) {
        w2[i] = w7[i] / s->gamma - s->mu * w2[i];
        w4[i] = (w9[i] - s->gamma * s->mu * w4[i]) / s->ksi;
        xi[i] = w2[i];
    }
    *nt = 1;
    *nou = 3;
}

/* A^T xi for the QMRCLA branch (inverserigopt.f:555-584): xr = 0 - G xi,
   then xr = alpha^T xr + xi (G is symmetric, so A^T = I - alpha^T G) */
static void apply_transpose(const zc *G6, int nx, int ny, int nz, const int *tabdip, long nbs, long nmax,
                            const zc *pol, const zc *xi, zc *xr) {
    long n3 = 3 * nbs;
    memset(xr, 0, sizeof(zc) * n3);
    matvec_core(G6, nx, ny, nz, tabdip, xi, xr);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nbs; i++) {
        zc t[3];
        for (int a = 0; a < 3; a++) {
            zc acc = 0;
            for (int b = 0; b < 3; b++) acc += pol[i + nmax * b + 3 * nmax * a] * xr[3 * i + b];
            t[a] = acc;
        }
        for (int a = 0; a < 3; a++) xr[3 * i + a] = t[a] + xi[3 * i + a];
    }
}

/* The transposed product on its own, for the tests of its identity
   u^T (A v) = (A^T u)^T v */
void orc_apply_transpose(const zc *G6, int nx, int ny, int nz, const int *tabdip, int nbs, int nmax,
                         const zc *pol, const zc *xi, zc *xr) {
    apply_transpose(G6, nx, ny, nz, tabdip, nbs, nmax, pol, xi, xr);
}

/* An optional callback lets the CPU baseline stop after a bounded number of
   mat-vecs; it is NULL in the parity tests. */
typedef int (*orc_cancel_fn)(int ncompte);

int orc_inverserig(const zc *G6, int nx, int ny, int nz, int nbsphere, const int *tabdip,
                   const zc *polarisa, int nmax, const zc *FF0, const char *methodeit,
                   double tol, zc *FF, zc *FFloc, double *tol1, int *nloop, int *ncompte,
                   int *nstop, char *infostr, orc_cancel_fn cancel, int nlim_in) {
    long n3 = 3L * nbsphere;
    /* nlim = 10000 in the reference (inverserigopt.f:30); tests may lower it */
    int nlim = nlim_in > 0 ? nlim_in : 10000;
    int nou = 0, nstat = 0, steperr = 0;
    zc *xi = (zc *)malloc(sizeof(zc) * n3);
    zc *xr = (zc *)malloc(sizeof(zc) * n3);
    zc *W = (zc *)calloc((size_t)n3 * 16, sizeof(zc)); /* GPBiCOR uses 14 columns */
    memcpy(xi, FF0, sizeof(zc) * n3);
    *nstop = 0;
    *ncompte = 0;
    *nloop = 0;
    *tol1 = 0;
    char meth[13];
    memset(meth, ' ', 12);
    meth[12] = 0;
    memcpy(meth, methodeit, strnlen(methodeit, 12));
    /* the reference's elseif chain (inverserigopt.f:42-1009) compares prefixes
       of the blank-padded character(12) methodeit, in this order */
    int kind = 0;
    if (strncmp(meth, "GPBICG1", 7) == 0) kind = 1;
    else if (strncmp(meth, "GPBICG2", 7) == 0) kind = 8;
    else if (strncmp(meth, "GPBICGsafe", 10) == 0) kind = 7;
    else if (strncmp(meth, "GPBICGplus", 10) == 0) kind = 9;
    else if (strncmp(meth, "GPBICGAR", 8) == 0) kind = 10;  /* 'GPBICGAR2' too: (1:8) is tested first */
    else if (strncmp(meth, "BICGSTARPLUS", 12) == 0) kind = 11;
    else if (strncmp(meth, "QMRCLA", 6) == 0) kind = 14;
    else if (strncmp(meth, "TFQMR", 5) == 0) kind = 6;
    else if (strncmp(meth, "CG   ", 5) == 0) kind = 5;
    else if (strncmp(meth, "BICGSTAB", 8) == 0) kind = 4;
    else if (strncmp(meth, "QMRBICGSTAB1", 12) == 0) kind = 2;
    else if (strncmp(meth, "QMRBICGSTAB2", 12) == 0) kind = 3;
    else if (strncmp(meth, "GPBICOR", 7) == 0) kind = 13;
    else if (strncmp(meth, "CORS   ", 7) == 0) kind = 12;
    if (kind == 0) {
        *nstop = 1;
        set_info(infostr, "Iterative method not correct!");
        free(xi); free(xr); free(W);
        return *nstop;
    }
    gpbicg_state gs;
    qmr_state qs;
    bicgstab_state bs;
    cg_state cs;
    tfqmr_state ts;
    gpsafe_state ss;
    cors_state rs;
    gpbicor_state os;
    qmrcla_state ls;
    int nt = 1;
    memset(&ls, 0, sizeof ls);
    memset(&rs, 0, sizeof rs);
    memset(&os, 0, sizeof os);
    memset(&ts, 0, sizeof ts);
    memset(&ss, 0, sizeof ss);
    memset(&gs, 0, sizeof gs);
    memset(&qs, 0, sizeof qs);
    memset(&bs, 0, sizeof bs);
    memset(&cs, 0, sizeof cs);
    double norm = 0;
    /* GPBICG and CG return the solution in xi; QMR-BiCGSTAB and BiCGSTAB in
       FFloc (the X argument), which the driver copies back to xi */
    const int x_in_floc = kind == 2 || kind == 3 || kind == 4 || kind == 6;
    for (;;) {
        if (kind == 1 || kind == 8)
            gpbicg(xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &gs, &nstat, &steperr, kind == 8);
        else if (kind == 4)
            bicgstab(FFloc, xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &bs, &nstat, &steperr);
        else if (kind == 5)
            zcg(xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &cs, &nstat);
        else if (kind == 6)
            tfqmr(FFloc, xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &ts, &nstat, &steperr);
        else if (kind == 12)
            cors(xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &rs, &nstat, &steperr);
        else if (kind == 13)
            gpbicor(xi, xr, FF0, FFloc, n3, &nou, W, nloop, nlim, tol, &os, &nstat, &steperr);
        else if (kind == 11)
            bicgstarplus(xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &ss, &nstat, &steperr);
        else if (kind == 10)
            gpbicgar(xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &ss, &nstat, &steperr);
        else if (kind == 7 || kind == 9)
            gpbicgsafe(xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &ss, &nstat, &steperr, kind == 9);
        else if (kind == 14)
            qmrcla(FFloc, xi, xr, FF0, n3, &nou, &nt, W, nloop, nlim, tol, &ls, &nstat, &steperr);
        else
            qmrbicgstab(FFloc, xi, xr, FF0, n3, &nou, W, nloop, nlim, tol, &qs,
                        kind == 2 ? 1 : 2, &nstat, &steperr);
        norm = kind == 1 || kind == 8 ? gs.norm : kind == 4 ? bs.norm : kind == 5 ? cs.norm : kind == 6 ? ts.norm
             : kind == 12 ? rs.norm : kind == 13 ? os.norm : kind == 14 ? ls.norm : kind >= 7 ? ss.norm : qs.norm;
        if (nstat < 0) {
            *nstop = 1;
            /* the TFQMR branch prints it without '!' (inverserigopt.f:609) */
            set_info(infostr, kind == 6 ? "Problem to solve Ax=b" : "Problem to solve Ax=b!");
            free(xi); free(xr); free(W);
            return *nstop;
        }
        *ncompte += 1;
        if (kind == 14) {
            /* inverserigopt.f:516-584: the solution is in FFloc; nt = 1 asks
               for A xi (xi becomes alpha xi), nt = 2 for A^T xi */
            if (nstat == 1) {
                memcpy(xi, FFloc, sizeof(zc) * n3);
                nt = 1;
            }
            if (nt == 1) {
                memcpy(xr, xi, sizeof(zc) * n3);
                apply_pola(nbsphere, nmax, polarisa, xr, xi);
                matvec_core(G6, nx, ny, nz, tabdip, xi, xr);
            } else {
                apply_transpose(G6, nx, ny, nz, tabdip, nbsphere, nmax, polarisa, xi, xr);
            }
        } else if (!x_in_floc) {
            memcpy(xr, xi, sizeof(zc) * n3);
            if (nstat == 1) memcpy(FFloc, xi, sizeof(zc) * n3);
        } else {
            if (nstat == 1) memcpy(xi, FFloc, sizeof(zc) * n3);
            memcpy(xr, xi, sizeof(zc) * n3);
        }
        if (kind != 14) {
            apply_pola(nbsphere, nmax, polarisa, xr, xi);
            matvec_core(G6, nx, ny, nz, tabdip, xi, xr);
        }
        if (cancel && cancel(*ncompte)) {
            *nstop = -1;
            set_info(infostr, "Calculation cancelled during iterative method");
            free(xi); free(xr); free(W);
            return *nstop;
        }
        if (nstat == 1) break;
    }
    double t = 0;
    for (long i = 0; i < n3; i++) {
        xr[i] -= FF0[i];
        FF[i] = xi[i];
        t += creal(xr[i] * conj(xr[i]));
    }
    *tol1 = sqrt(t) / norm;
    /* the GPBICOR and QMRCLA branches do not */
    if (kind == 1 || (kind >= 6 && kind != 13 && kind != 14)) *nloop += 1;
    free(xi); free(xr); free(W);
    return *nstop;
}

/* GPBICG driven on a dense matrix (the commented self-test of gpbicg.f:1-79) */
int orc_gpbicg_dense(int ndim, const zc *mat /* column-major ndim x ndim */, const zc *b,
                     zc *x, double tol, int maxit, int *nloop) {
    zc *xi = (zc *)calloc(ndim, sizeof(zc)), *xr = (zc *)calloc(ndim, sizeof(zc));
    zc *W = (zc *)calloc((size_t)ndim * 12, sizeof(zc));
    memcpy(xi, x, sizeof(zc) * ndim);
    int nou = 0, st = 0, se = 0, itno = 0;
    gpbicg_state S;
    memset(&S, 0, sizeof S);
    for (;;) {
        gpbicg(xi, xr, b, ndim, &nou, W, &itno, maxit, tol, &S, &st, &se, 0);
        if (st < 0) break;
        for (int i = 0; i < ndim; i++) {
            zc acc = 0;
            for (int j = 0; j < ndim; j++) acc += mat[i + (size_t)ndim * j] * xi[j];
            xr[i] = acc;
        }
        if (st == 1) break;
    }
    memcpy(x, xi, sizeof(zc) * ndim);
    *nloop = itno;
    free(xi); free(xr); free(W);
    return st;
}

/* ------------------------------------------------------------------------- */
/* Polarisability: cdmlib/polarisabilite.f:1-62 (poladiff).                   */
/* methode: "CM", "RR", "PS", "GB", "LA", "LR".  Returns 0, or 1 on an        */
/* unknown method or dddis (the reference stops the process there).           */
/* ------------------------------------------------------------------------- */
int orc_poladiff(double rayon1, zc eps, double eps0, double k0, int dddis,
                 const char *methode, zc *out) {
    const double pi = acos(-1.0);
    zc rapport = (eps - eps0) / (eps + 2.0 * eps0);
    double indice = sqrt(eps0);
    double k03 = k0 * k0 * k0 * indice * indice * indice;
    double rayon = rayon1, maille = 0, volume;
    if (dddis == 0) volume = rayon * rayon * rayon;
    else if (dddis == 1) {
        maille = rayon;
        rayon = rayon * pow(0.75 / pi, 1.0 / 3.0);
        volume = rayon * rayon * rayon;
    } else return 1;
    zc pola = rapport * volume;
    if (!strncmp(methode, "CM", 2)) *out = pola * eps0;
    else if (!strncmp(methode, "RR", 2) || !strncmp(methode, "PS", 2))
        *out = eps0 * pola / (1.0 - 2.0 / 3.0 * I * k03 * pola);
    else if (!strncmp(methode, "GB", 2))
        *out = pola / (1.0 - 2.0 / 3.0 * I * k03 * pola - k0 * k0 * pola * indice * indice / rayon);
    else if (!strncmp(methode, "LA", 2))
        *out = pola / (1.0 - 2.0 * rapport *
                                 ((1.0 - I * k0 * indice * rayon) * cexp(I * k0 * indice * rayon) - 1.0));
    else if (!strncmp(methode, "LR", 2)) {
        double sldr = 1.0 / 5.0;
        *out = eps0 * pola /
               (1.0 + pola * ((-1.8915316 + eps / eps0 * 0.1648469 - eps / eps0 * 1.7700004 * sldr) *
                                  k0 * k0 * indice * indice / maille -
                              2.0 / 3.0 * I * k03 * indice * indice * indice));
    } else return 1;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Local -> macroscopic field: cdmlib/local-macro.f:3-71 (nsens = +1 or -1).   */
/* The 3x3 inverse is done by cofactors instead of LINPACK zgefa/zgedi.       */
/* eps is column-major 3x3.  Returns 1 for a singular matrix or bad nsens.    */
/* ------------------------------------------------------------------------- */
static int inv33(const zc *m, zc *o) {
#define A(i, j) m[(i) + 3 * (j)]
    zc c00 = A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1);
    zc c01 = A(1, 2) * A(2, 0) - A(1, 0) * A(2, 2);
    zc c02 = A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0);
    zc det = A(0, 0) * c00 + A(0, 1) * c01 + A(0, 2) * c02;
    if (det == 0) return 1;
    o[0 + 3 * 0] = c00 / det;
    o[1 + 3 * 0] = c01 / det;
    o[2 + 3 * 0] = c02 / det;
    o[0 + 3 * 1] = (A(0, 2) * A(2, 1) - A(0, 1) * A(2, 2)) / det;
    o[1 + 3 * 1] = (A(0, 0) * A(2, 2) - A(0, 2) * A(2, 0)) / det;
    o[2 + 3 * 1] = (A(0, 1) * A(2, 0) - A(0, 0) * A(2, 1)) / det;
    o[0 + 3 * 2] = (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1)) / det;
    o[1 + 3 * 2] = (A(0, 2) * A(1, 0) - A(0, 0) * A(1, 2)) / det;
    o[2 + 3 * 2] = (A(0, 0) * A(1, 1) - A(0, 1) * A(1, 0)) / det;
#undef A
    return 0;
}

int orc_local_macro(zc *Eloc, zc *Em, const zc *eps, double d, double k0, int nsens) {
    const double pi = acos(-1.0);
    double cst = k0 * k0 * k0 * d * d * d / 2.0 / pi;
    zc m[9];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            zc e = eps[a + 3 * b];
            zc m0 = e + (a == b ? 2.0 : 0.0);
            zc m1 = e - (a == b ? 1.0 : 0.0);
            m[a + 3 * b] = m0 - I * cst * m1;
        }
    if (nsens == 1) {
        zc mi[9];
        if (inv33(m, mi)) return 1;
        for (int a = 0; a < 3; a++) {
            zc acc = 0;
            for (int b = 0; b < 3; b++) acc += mi[a + 3 * b] * Eloc[b];
            Em[a] = acc * 3.0;
        }
    } else if (nsens == -1) {
        for (int a = 0; a < 3; a++) {
            zc acc = 0;
            for (int b = 0; b < 3; b++) acc += m[a + 3 * b] * Em[b];
            Eloc[a] = acc / 3.0;
        }
    } else return 1;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Anisotropic polarisability: cdmlib/polaepstens.f:1-122.  eps is a          */
/* column-major 3x3 permittivity; alpha0 = V (eps - eps0 I)(eps + 2 eps0 I)^-1 */
/* (:33-62), CM: alpha0 eps0 (:64-69), RR: (I - 2/3 i k^3 alpha0)^-1 alpha0    */
/* eps0 (:70-99); inv = -1 inverts the result (:106-118).  Returns 1 on an    */
/* unknown method, a bad dis or a singular matrix (the reference stops).      */
/* ------------------------------------------------------------------------- */
int orc_polaepstens(double rayon1, const zc *eps, double eps0, double k0, int dis,
                    const char *methode, int inv, zc *out) {
    const double pi = acos(-1.0);
    double indice = sqrt(eps0);
    double k03 = k0 * k0 * k0 * indice * indice * indice;
    double rayon = rayon1, volume;
    if (dis == 0) volume = rayon * rayon * rayon;
    else if (dis == 1) {
        rayon = rayon * pow(0.75 / pi, 1.0 / 3.0);
        volume = rayon * rayon * rayon;
    } else return 1;
    zc m[9], m1[9], mi[9], a0[9], r[9];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            m[a + 3 * b] = eps[a + 3 * b] + (a == b ? 2.0 * eps0 : 0.0);
            m1[a + 3 * b] = eps[a + 3 * b] - (a == b ? eps0 : 0.0);
        }
    if (inv33(m, mi)) return 1;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            zc acc = 0;
            for (int c = 0; c < 3; c++) acc += m1[a + 3 * c] * mi[c + 3 * b];
            a0[a + 3 * b] = acc * volume;
        }
    if (!strncmp(methode, "CM", 2)) {
        for (int q = 0; q < 9; q++) r[q] = a0[q] * eps0;
    } else if (!strncmp(methode, "RR", 2)) {
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                m[a + 3 * b] = -2.0 / 3.0 * I * k03 * a0[a + 3 * b] + (a == b ? 1.0 : 0.0);
        if (inv33(m, mi)) return 1;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                zc acc = 0;
                for (int c = 0; c < 3; c++) acc += mi[a + 3 * c] * a0[c + 3 * b] * eps0;
                r[a + 3 * b] = acc;
            }
    } else return 1;
    if (inv == -1) return inv33(r, out);
    for (int q = 0; q < 9; q++) out[q] = r[q];
    return 0;
}

/* macroscopic field of every dipole (cdmlib/cdmlib.f:2595-2655), eps in the
   (nmax,3,3) column-major layout */
int orc_macro_all(int nbsphere, int nmax, const zc *epsilon, const zc *FFloc, double d,
                  double k0, zc *Em) {
    int bad = 0;
#pragma omp parallel for reduction(| : bad)
    for (int i = 0; i < nbsphere; i++) {
        zc e[9], loc[3];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) e[a + 3 * b] = epsilon[i + (long)nmax * a + 3L * nmax * b];
        for (int a = 0; a < 3; a++) loc[a] = FFloc[3L * i + a];
        bad |= orc_local_macro(loc, Em + 3L * i, e, d, k0, 1);
    }
    return bad;
}

/* ------------------------------------------------------------------------- */
/* Incident plane waves: cdmlib/ondeplane.f:1-50, cdmlib/ondeplanekxky.f:1-60, */
/* cdmlib/irradiance.f:6-20.  Angles in degrees as in ondeplane.              */
/* ------------------------------------------------------------------------- */
void orc_irradiance(double P0, double w0, double *E0, double *irra) {
    const double pi = acos(-1.0);
    double c = 299792458.0;
    double eps0 = 1.0 / (c * c * 4.0 * pi * 1e-7);
    double surf = w0 * w0 * pi;
    *irra = P0 / surf;
    *E0 = sqrt(2.0 * (*irra) / c / eps0);
}

int orc_ondeplane(double x, double y, double z, double k0, zc E0, double pp, double thetat,
                  double phit, zc *E) {
    const double pi = acos(-1.0);
    if (pp < 0.0 || pp > 1.0) return -1;
    double theta = thetat * pi / 180.0, phi = phit * pi / 180.0;
    double p = sqrt(pp), s = sqrt(1.0 - pp);
    double sg = copysign(1.0, theta);
    zc E0s = E0 * s * sg, E0p = E0 * p * sg;
    double kx = k0 * sin(theta) * cos(phi), ky = k0 * sin(theta) * sin(phi), kz = k0 * cos(theta);
    zc Ey = E0s * cos(phi) + E0p * cos(theta) * sin(phi);
    zc Ex = -E0s * sin(phi) + E0p * cos(theta) * cos(phi);
    zc Ez = -E0p * sin(theta);
    zc e = cexp(I * (x * kx + y * ky + z * kz));
    E[0] = Ex * e;
    E[1] = Ey * e;
    E[2] = Ez * e;
    return 0;
}

int orc_ondeplanekxky(double x, double y, double z, double k0, zc E0, double pp, double kx,
                      double ky, zc *E) {
    if (pp < 0.0 || pp > 1.0) return -1;
    double p = sqrt(pp), s = sqrt(1.0 - pp);
    zc E0s = E0 * s, E0p = E0 * p;
    double kz = sqrt(k0 * k0 - kx * kx - ky * ky);
    zc Ex, Ey, Ez;
    if (kz >= 0.99999 * k0) {
        Ex = E0p;
        Ey = E0s;
        Ez = 0;
    } else {
        double kp = sqrt(kx * kx + ky * ky);
        double nsx = -ky / kp, nsy = kx / kp;
        double npx = kz * nsy, npy = -kz * nsx, npz = -kx * nsy + ky * nsx;
        double np = sqrt(npx * npx + npy * npy + npz * npz);
        npx /= np; npy /= np; npz /= np;
        Ex = E0s * nsx + E0p * npx;
        Ey = E0s * nsy + E0p * npy;
        Ez = E0p * npz;
    }
    zc e = cexp(I * (x * kx + y * ky + z * kz));
    E[0] = Ex * e;
    E[1] = Ey * e;
    E[2] = Ez * e;
    return 0;
}

/* FF0 for all dipoles: beam 0 = ondeplane(theta,phi), 1 = ondeplanekxky(kx,ky) */
int orc_incident(int nbsphere, const double *xs, const double *ys, const double *zs, double k0,
                 zc E0, double pp, int beam, double a1, double a2, zc *FF0) {
    int bad = 0;
#pragma omp parallel for reduction(| : bad)
    for (int i = 0; i < nbsphere; i++) {
        int r = beam == 0 ? orc_ondeplane(xs[i], ys[i], zs[i], k0, E0, pp, a1, a2, FF0 + 3L * i)
                          : orc_ondeplanekxky(xs[i], ys[i], zs[i], k0, E0, pp, a1, a2, FF0 + 3L * i);
        bad |= (r != 0);
    }
    return bad;
}

/* ------------------------------------------------------------------------- */
/* Cross sections: cdmlib/cdmlib.f:2730-2746.                                  */
/* ------------------------------------------------------------------------- */
void orc_cross_sections(int nbsphere, const zc *FF0, const zc *FF, const zc *FFloc, double k0,
                        double I0, double *Cext, double *Cabs) {
    const double pi = acos(-1.0);
    double k03 = k0 * k0 * k0;
    double ce = 0, ca = 0;
#pragma omp parallel for reduction(+ : ce, ca)
    for (long i = 0; i < nbsphere; i++) {
        zc s1 = 0, s2 = 0;
        double s3 = 0;
        for (int a = 0; a < 3; a++) {
            long q = 3 * i + a;
            s1 += conj(FF0[q]) * FF[q];
            s2 += FF[q] * conj(FFloc[q]);
            s3 += creal(FF[q] * conj(FF[q]));
        }
        ce += cimag(s1);
        ca += cimag(s2) - 2.0 / 3.0 * k03 * s3;
    }
    *Cext = 4.0 * pi * k0 * ce / I0;
    *Cabs = 4.0 * pi * k0 * ca / I0;
}

/* ------------------------------------------------------------------------- */
/* Mie series for a homogeneous sphere (Bohren & Huffman 1983, appendix A:     */
/* logarithmic derivative by downward recurrence, Riccati-Bessel functions by */
/* upward recurrence).  The reference calls it through CALLBHMIE              */
/* (cdmlib/module_mie.f:1) with refmed = 1 and m = sqrt(eps).  Radius and     */
/* wavelength in metres; cross sections in m^2.                               */
/* ------------------------------------------------------------------------- */
int orc_mie(zc eps, double radius, double wavelength, double *qcext, double *qcsca,
            double *qcabs) {
    const double pi = acos(-1.0);
    zc m = csqrt(eps);
    double x = 2.0 * pi * radius / wavelength;
    zc y = m * x;
    double xstop = x + 4.0 * cbrt(x) + 2.0;
    int nstop = (int)xstop;
    double ymod = cabs(y);
    int nmx = (int)fmax(xstop, ymod) + 15;
    if (nmx > 200000) return 1;
    zc *D = (zc *)calloc((size_t)nmx + 1, sizeof(zc));
    D[nmx] = 0;
    for (int n = nmx; n >= 1; n--) {
        zc en = n / y;
        D[n - 1] = en - 1.0 / (D[n] + en);
    }
    double psi0 = cos(x), psi1 = sin(x);
    double chi0 = -sin(x), chi1 = cos(x);
    zc xi1 = psi1 - I * chi1;
    double qsca = 0, qext = 0;
    for (int n = 1; n <= nstop; n++) {
        double fn = (2.0 * n + 1.0);
        double psi = (2.0 * n - 1.0) * psi1 / x - psi0;
        double chi = (2.0 * n - 1.0) * chi1 / x - chi0;
        zc xi = psi - I * chi;
        zc da = D[n] / m + n / x;
        zc db = D[n] * m + n / x;
        zc an = (da * psi - psi1) / (da * xi - xi1);
        zc bn = (db * psi - psi1) / (db * xi - xi1);
        qsca += fn * (creal(an) * creal(an) + cimag(an) * cimag(an) + creal(bn) * creal(bn) +
                      cimag(bn) * cimag(bn));
        qext += fn * creal(an + bn);
        psi0 = psi1; psi1 = psi;
        chi0 = chi1; chi1 = chi;
        xi1 = psi1 - I * chi1;
    }
    free(D);
    qsca *= 2.0 / (x * x);
    qext *= 2.0 / (x * x);
    double g = pi * radius * radius;
    *qcext = qext * g;
    *qcsca = qsca * g;
    *qcabs = (qext - qsca) * g;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* SUNIF: multiplicative congruential uniform generator, cdmlib/random.f:19-56 */
/* (Ahrens, Dieter & Grube 1970).  R := frac(R * 41475557); first call seeds   */
/* R = float(IR) / 2^28 and sets IR = -1; the returned value is rounded to    */
/* single precision like SNGL.  The state is kept per call site in *state.    */
/* ------------------------------------------------------------------------- */
double orc_sunif(int *ir, double *state) {
    const double factor = 41475557.0, two28 = 268435456.0;
    if (*ir >= 0) {
        *state = (double)(float)(*ir) / two28;
        *state = fmod(*state * factor, 1.0);
        *ir = -1;
        return (double)(float)(*state);
    }
    *state = fmod(*state * factor, 1.0);
    return (double)(float)(*state);
}

/* ------------------------------------------------------------------------- */
/* Object builders (host set-up restated for input generation).               */
/* All lengths in metres (the reference converts nm inputs by 1e-9 first).    */
/* tabdip has nx*ny*nz entries, 1-based dipole numbers, 0 = empty.            */
/* polarisa/epsilon: (nmax,3,3) column-major, nmax >= nx*ny*nz.               */
/* ------------------------------------------------------------------------- */
static void set_iso(zc *pol, zc *eps, long nmax, long n, zc a, zc e) {
    for (int q = 0; q < 3; q++) {
        pol[n + nmax * q + 3 * nmax * q] = a;
        eps[n + nmax * q + 3 * nmax * q] = e;
    }
}

/* one dipole of an anisotropic object: epsilon(n,:,:) = epsani,
   polarisa(n,:,:) = polaeps (objectsphere.f:128-135) */
static void set_full(zc *pol, zc *eps, long nmax, long n, const zc *a9, const zc *e9) {
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            pol[n + nmax * a + 3 * nmax * b] = a9[a + 3 * b];
            eps[n + nmax * a + 3 * nmax * b] = e9[a + 3 * b];
        }
}

/* a dipole of the object: isotropic (epsani NULL) or anisotropic */
static void set_obj(zc *pol, zc *eps, long nmax, long n, zc a, zc e, const zc *a9, const zc *epsani) {
    if (epsani) set_full(pol, eps, nmax, n, a9, epsani);
    else set_iso(pol, eps, nmax, n, a, e);
}

/* objetsphere (cdmlib/objectsphere.f:94-195), na = -1 (inside only) or 0;
   epsani (column-major 3x3) non-NULL for trope = 'ani', where 'PS' is refused
   (:64-67) and every dipole gets polaepstens with dis = 1, inv = 1 */
static int sphere_impl(double rayon, zc eps, const zc *epsani, int nnnr, int na, double k0,
                       const char *methode, int nmax, double *xs, double *ys, double *zs,
                       int *tabdip, zc *pol, zc *epsilon, int *nbsphere, int *ndipole,
                       double *aretecube) {
    if (rayon == 0.0) return 1;
    if (epsani && !strncmp(methode, "PS", 2)) return 1;
    long cap = (long)nmax;
    memset(pol, 0, sizeof(zc) * 9 * cap);
    memset(epsilon, 0, sizeof(zc) * 9 * cap);
    double d = 2.0 * rayon / nnnr;
    *aretecube = d;
    int nb = 0, nd = 0;
    zc a = 0, a9[9];
    if (epsani) {
        if (orc_polaepstens(d, epsani, 1.0, k0, 1, methode, 1, a9)) return 1;
    } else if (orc_poladiff(d, eps, 1.0, k0, 1, methode, &a)) return 1;
    for (int i = 1; i <= nnnr; i++)
        for (int j = 1; j <= nnnr; j++)
            for (int k = 1; k <= nnnr; k++) {
                double x = -rayon + d * (k - 0.5);
                double y = -rayon + d * (j - 0.5);
                double z = -rayon + d * (i - 0.5);
                nd++;
                tabdip[nd - 1] = 0;
                int inside = sqrt(x * x + y * y + z * z) < rayon;
                if (na == -1) {
                    if (!inside) continue;
                    nb++;
                    tabdip[nd - 1] = nb;
                    xs[nb - 1] = x; ys[nb - 1] = y; zs[nb - 1] = z;
                    set_obj(pol, epsilon, cap, nb - 1, a, eps, a9, epsani);
                } else {
                    nb++;
                    tabdip[nd - 1] = nb;
                    xs[nb - 1] = x; ys[nb - 1] = y; zs[nb - 1] = z;
                    if (inside) set_obj(pol, epsilon, cap, nb - 1, a, eps, a9, epsani);
                    else set_iso(pol, epsilon, cap, nb - 1, 0, 1.0);
                }
            }
    *nbsphere = nb;
    *ndipole = nd;
    return 0;
}

int orc_object_sphere(double rayon, zc eps, int nnnr, int na, double k0, const char *methode,
                      int nmax, double *xs, double *ys, double *zs, int *tabdip, zc *pol,
                      zc *epsilon, int *nbsphere, int *ndipole, double *aretecube) {
    return sphere_impl(rayon, eps, NULL, nnnr, na, k0, methode, nmax, xs, ys, zs, tabdip, pol,
                       epsilon, nbsphere, ndipole, aretecube);
}

int orc_object_sphere_ani(double rayon, const zc *epsani, int nnnr, int na, double k0,
                          const char *methode, int nmax, double *xs, double *ys, double *zs,
                          int *tabdip, zc *pol, zc *epsilon, int *nbsphere, int *ndipole,
                          double *aretecube) {
    return sphere_impl(rayon, 0, epsani, nnnr, na, k0, methode, nmax, xs, ys, zs, tabdip, pol,
                       epsilon, nbsphere, ndipole, aretecube);
}

/* objetcube (cdmlib/objectcube.f:60-130): full box of nnnr^3 dipoles;
   epsani non-NULL for trope = 'ani' (:118-135) */
static int cube_impl(double side, zc eps, const zc *epsani, int nnnr, double k0,
                     const char *methode, int nmax, double *xs, double *ys, double *zs,
                     int *tabdip, zc *pol, zc *epsilon, int *nbsphere, int *ndipole,
                     double *aretecube) {
    if (side == 0.0) return 1;
    long cap = nmax;
    memset(pol, 0, sizeof(zc) * 9 * cap);
    memset(epsilon, 0, sizeof(zc) * 9 * cap);
    double d = side / nnnr;
    *aretecube = d;
    double xc = (side + d) / 2.0;
    zc a = 0, a9[9];
    if (epsani) {
        if (orc_polaepstens(d, epsani, 1.0, k0, 1, methode, 1, a9)) return 1;
    } else if (orc_poladiff(d, eps, 1.0, k0, 1, methode, &a)) return 1;
    int nb = 0;
    for (int i = 1; i <= nnnr; i++)
        for (int j = 1; j <= nnnr; j++)
            for (int k = 1; k <= nnnr; k++) {
                nb++;
                tabdip[nb - 1] = nb;
                xs[nb - 1] = k * d - xc;
                ys[nb - 1] = j * d - xc;
                zs[nb - 1] = i * d - xc;
                set_obj(pol, epsilon, cap, nb - 1, a, eps, a9, epsani);
            }
    *nbsphere = nb;
    *ndipole = nb;
    return 0;
}

int orc_object_cube(double side, zc eps, int nnnr, double k0, const char *methode, int nmax,
                    double *xs, double *ys, double *zs, int *tabdip, zc *pol, zc *epsilon,
                    int *nbsphere, int *ndipole, double *aretecube) {
    return cube_impl(side, eps, NULL, nnnr, k0, methode, nmax, xs, ys, zs, tabdip, pol, epsilon,
                     nbsphere, ndipole, aretecube);
}

int orc_object_cube_ani(double side, const zc *epsani, int nnnr, double k0, const char *methode,
                        int nmax, double *xs, double *ys, double *zs, int *tabdip, zc *pol,
                        zc *epsilon, int *nbsphere, int *ndipole, double *aretecube) {
    return cube_impl(side, 0, epsani, nnnr, k0, methode, nmax, xs, ys, zs, tabdip, pol, epsilon,
                     nbsphere, ndipole, aretecube);
}

/* objetparainhomonxnynz (cdmlib/objectparainhomonxnynz.f:85-237): cuboid with
   a Gaussian-random-field permittivity built by spectral synthesis with SUNIF
   phases seeded by 4*ng+1.  d and lc in metres; hc = standard deviation. */
int orc_object_inhomocuboid(int nx, int ny, int nz, double d, zc eps, double lc, double hc,
                            int ng, double k0, const char *methode, int nmax, double *xs,
                            double *ys, double *zs, int *tabdip, zc *pol, zc *epsilon,
                            int *nbsphere, int *ndipole) {
    if (lc <= 0.0 || hc <= 0.0) return 1;
    const double pi = acos(-1.0);
    long cap = nmax;
    long N = (long)nx * ny * nz;
    memset(pol, 0, sizeof(zc) * 9 * cap);
    memset(epsilon, 0, sizeof(zc) * 9 * cap);
    zc *epsb = (zc *)calloc((size_t)N, sizeof(zc));
    double lx = nx * d, ly = ny * d, lz = nz * d;
    double dkx = 2 * pi / lx, dky = 2 * pi / ly, dkz = 2 * pi / lz;
    double coeff1 = 0.125 * hc * hc * lc * lc * lc / (pi * sqrt(pi));
    double coeff2 = lc * lc;
    double coeff3 = 4.0 * dkx * dky * dkz;
    int ngraine = 4 * ng + 1;
    double rstate = 0;
    long nk = 0;
    for (int i = 1; i <= nz; i++)
        for (int j = 1; j <= ny; j++)
            for (int k = 1; k <= nx; k++) {
                nk++;
                double kx = (k <= nx / 2 + 1) ? (k - 1) * dkx : (k - 1 - nx) * dkx;
                double ky = (j <= ny / 2 + 1) ? (j - 1) * dky : (j - 1 - ny) * dky;
                double kz = (i <= nz / 2 + 1) ? (i - 1) * dkz : (i - 1 - nz) * dkz;
                double spec = coeff1 * exp(-0.25 * coeff2 * (kx * kx + ky * ky + kz * kz));
                double phase = 2.0 * pi * orc_sunif(&ngraine, &rstate);
                zc v = sqrt(spec * coeff3) * cexp(I * phase);
                if (nk == 1) v = 0;
                if (nk >= nx / 2 + 2 && nk <= nx) v = 0;
                if (nk >= (long)(ny / 2 + 1) * nx + 1 && nk <= (long)nx * ny) v = 0;
                if (nk >= (long)(nz / 2 + 1) * nx * ny + 1 && nk <= N) v = 0;
                epsb[nk - 1] = v;
            }
    orc_fft3d(epsb, nx, ny, nz, +1);
    for (long q = 0; q < N; q++) epsb[q] = creal(epsb[q]) + eps;
    double sx = d * nx, sy = d * ny, sz = d * nz;
    int nb = 0;
    for (int i = 1; i <= nz; i++)
        for (int j = 1; j <= ny; j++)
            for (int k = 1; k <= nx; k++) {
                nb++;
                tabdip[nb - 1] = nb;
                xs[nb - 1] = -sx / 2 + d * (k - 0.5);
                ys[nb - 1] = -sy / 2 + d * (j - 0.5);
                zs[nb - 1] = -sz / 2 + d * (i - 0.5);
                zc e = epsb[nb - 1];
                zc a;
                if (orc_poladiff(d, e, 1.0, k0, 1, methode, &a)) { free(epsb); return 1; }
                set_iso(pol, epsilon, cap, nb - 1, a, e);
            }
    free(epsb);
    *nbsphere = nb;
    *ndipole = nb;
    return 0;
}

/* objetsphereconcentric (cdmlib/objectsphereconcentric.f:76-230), na -1 or 0.
   rayons increasing, in metres; d = 2 rayons[ns-1] / nnnr. */
int orc_object_concentric(int ns, const double *rayons, const zc *epss, int nnnr, int na,
                          double k0, const char *methode, int nmax, double *xs, double *ys,
                          double *zs, int *tabdip, zc *pol, zc *epsilon, int *nbsphere,
                          int *ndipole, double *aretecube) {
    if (rayons[0] == 0.0) return 1;
    for (int s = 1; s < ns; s++)
        if (rayons[s] - rayons[s - 1] <= 0.0) return 1;
    long cap = nmax;
    memset(pol, 0, sizeof(zc) * 9 * cap);
    memset(epsilon, 0, sizeof(zc) * 9 * cap);
    double d = 2.0 * rayons[ns - 1] / nnnr;
    *aretecube = d;
    double centre = d * nnnr / 2.0;
    zc *alph = (zc *)malloc(sizeof(zc) * ns);
    for (int s = 0; s < ns; s++)
        if (orc_poladiff(d, epss[s], 1.0, k0, 1, methode, &alph[s])) { free(alph); return 1; }
    int nb = 0, nd = 0;
    for (int i = 1; i <= nnnr; i++)
        for (int j = 1; j <= nnnr; j++)
            for (int k = 1; k <= nnnr; k++) {
                double x = (k - 1) * d + d / 2 - centre;
                double y = (j - 1) * d + d / 2 - centre;
                double z = (i - 1) * d + d / 2 - centre;
                double ray = sqrt(x * x + y * y + z * z);
                nd++;
                tabdip[nd - 1] = 0;
                int is = 0;
                if (ray <= rayons[0]) is = 1;
                else
                    for (int l = 2; l <= ns; l++)
                        if (ray <= rayons[l - 1] && ray >= rayons[l - 2]) is = l;
                if (na == -1) {
                    if (!is) continue;
                    nb++;
                    tabdip[nd - 1] = nb;
                    xs[nb - 1] = x; ys[nb - 1] = y; zs[nb - 1] = z;
                    set_iso(pol, epsilon, cap, nb - 1, alph[is - 1], epss[is - 1]);
                } else {
                    nb++;
                    tabdip[nd - 1] = nb;
                    xs[nb - 1] = x; ys[nb - 1] = y; zs[nb - 1] = z;
                    if (is) set_iso(pol, epsilon, cap, nb - 1, alph[is - 1], epss[is - 1]);
                    else set_iso(pol, epsilon, cap, nb - 1, 0, 1.0);
                }
            }
    free(alph);
    *nbsphere = nb;
    *ndipole = nd;
    return 0;
}

/* objetarbitrary (cdmlib/objectarbitrary.f:81-157) without the file: the
   caller gives the lattice positions and one isotropic eps per site. */
int orc_object_arbitrary(int nx, int ny, int nz, double d, const double *px, const double *py,
                         const double *pz, const zc *eps_site, double k0, const char *methode,
                         int nmax, double *xs, double *ys, double *zs, int *tabdip, zc *pol,
                         zc *epsilon, int *nbsphere, int *ndipole) {
    long cap = nmax;
    long N = (long)nx * ny * nz;
    memset(pol, 0, sizeof(zc) * 9 * cap);
    memset(epsilon, 0, sizeof(zc) * 9 * cap);
    int bad = 0;
#pragma omp parallel for reduction(| : bad)
    for (long n = 0; n < N; n++) {
        tabdip[n] = (int)n + 1;
        xs[n] = px[n]; ys[n] = py[n]; zs[n] = pz[n];
        zc a;
        bad |= orc_poladiff(d, eps_site[n], 1.0, k0, 1, methode, &a);
        set_iso(pol, epsilon, cap, n, a, eps_site[n]);
    }
    *nbsphere = (int)N;
    *ndipole = (int)N;
    return bad;
}

/* ------------------------------------------------------------------------- */
/* Far field by direct summation: cdmlib/cdmlib.f:2784-2880 (nsectionsca = 1, */
/* nquickdiffracte = 0): Poynting vector on (ntheta+1) x nphi directions,      */
/* Cscai and the asymmetry factor gasym.  Returns 1 for too few directions.  */
/* ------------------------------------------------------------------------- */
int orc_farfield_csca(int nbsphere, const double *xs, const double *ys, const double *zs,
                      const zc *FF, double k0, double I0, double theta, double phi, int ntheta,
                      int nphi, double *Cscai, double *gasym, double *poynting, double *thetafield,
                      double *phifield) {
    if (ntheta <= 10 || nphi <= 20) return 1;
    const double pi = acos(-1.0), c = 299792458.0, quatpieps0 = 1.0 / (c * c * 1e-7);
    double deltatheta = pi / (double)ntheta, deltaphi = 2.0 * pi / (double)nphi;
    double k03 = k0 * k0 * k0;
    double cs = 0.0, g = 0.0;
    int cnt = 0;
    for (int itheta = 0; itheta <= ntheta; itheta++) {
        double thetas = deltatheta * (double)itheta;
        for (int iphi = 0; iphi < nphi; iphi++, cnt++) {
            double phis = deltaphi * (double)iphi;
            double n0 = sin(thetas) * cos(phis), n1 = sin(thetas) * sin(phis), n2 = cos(thetas);
            zc Ex = 0, Ey = 0, Ez = 0;
            for (int i = 0; i < nbsphere; i++) {
                zc ctmp = cexp(-I * k0 * (n0 * xs[i] + n1 * ys[i] + n2 * zs[i]));
                zc ctmp1 = n0 * FF[3 * i] + n1 * FF[3 * i + 1] + n2 * FF[3 * i + 2];
                Ex += ctmp * (FF[3 * i] - ctmp1 * n0);
                Ey += ctmp * (FF[3 * i + 1] - ctmp1 * n1);
                Ez += ctmp * (FF[3 * i + 2] - ctmp1 * n2);
            }
            double Emod = creal(Ex * conj(Ex) + Ey * conj(Ey) + Ez * conj(Ez));
            poynting[cnt] = Emod * k0 * k0 * k0 * k0 * c / 8 / pi * quatpieps0;
            thetafield[cnt] = thetas * 180.0 / pi;
            phifield[cnt] = phis * 180.0 / pi;
            cs = cs + deltaphi * deltatheta * sin(thetas) * Emod;
            g = g + deltaphi * deltatheta * sin(thetas) * Emod *
                        (n0 * sin(theta * pi / 180.0) * cos(phi * pi / 180.0) +
                         n1 * sin(theta * pi / 180.0) * sin(phi * pi / 180.0) +
                         n2 * cos(theta * pi / 180.0));
        }
    }
    *gasym = g / cs;
    *Cscai = cs * k03 * k0 / I0;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Wide near field: cdmlib/cdmlib.f:1967-2492 (nprochefft >= 1, nrig = 0,     */
/* plane wave).  The box enlarged by nxmp, nymp, nzmp layers, the object's    */
/* dipoles matched to its sites in order with comparaison.f:41-50 (within     */
/* lambda/1000), xi = -FF there, xr = FF0 there and ondeplane elsewhere, the  */
/* Green spectrum of the enlarged box, one mat-vec xr -= G xi, then           */
/* local_macro with epsilon (identity off the object).  Outputs 3*nw values.  */
/* ------------------------------------------------------------------------- */
int orc_nearfield_wide(int nx, int ny, int nz, int nxmp, int nymp, int nzmp, double d, double k0,
                       double lambda, int nquad, int nbsphere, int nmax, const double *xs,
                       const double *ys, const double *zs, const zc *FF, const zc *FF0,
                       const zc *epsilon, zc E0, double theta, double phi, double pp, double *xswf,
                       double *yswf, double *zswf, zc *incident, zc *local, zc *macro) {
    int nxw = nx + 2 * nxmp, nyw = ny + 2 * nymp, nzw = nz + 2 * nzmp;
    long nw = (long)nxw * nyw * nzw;
    double xmin = 1e300, ymin = 1e300, zmin = 1e300;
    for (int i = 0; i < nbsphere; i++) {
        xmin = fmin(xmin, xs[i]);
        ymin = fmin(ymin, ys[i]);
        zmin = fmin(zmin, zs[i]);
    }
    double err = lambda / 1000.0;
    zc *xi = (zc *)calloc(3 * nw, sizeof(zc));
    zc *xr = (zc *)calloc(3 * nw, sizeof(zc));
    zc *eps = (zc *)calloc(9 * nw, sizeof(zc));
    for (long s = 0; s < nw; s++)
        for (int a = 0; a < 3; a++) eps[s + nw * (a + 3 * a)] = 1.0;
    long l = 0, s = 0;
    for (int i = 1; i <= nzw; i++)
        for (int j = 1; j <= nyw; j++)
            for (int k = 1; k <= nxw; k++, s++) {
                double x = xmin + (double)(k - nxmp - 1) * d;
                double y = ymin + (double)(j - nymp - 1) * d;
                double z = zmin + (double)(i - nzmp - 1) * d;
                xswf[s] = x;
                yswf[s] = y;
                zswf[s] = z;
                if (l < nbsphere && x >= xs[l] - err && x <= xs[l] + err && y >= ys[l] - err &&
                    y <= ys[l] + err && z >= zs[l] - err && z <= zs[l] + err) {
                    for (int a = 0; a < 3; a++) {
                        xi[3 * s + a] = -FF[3 * l + a];
                        xr[3 * s + a] = FF0[3 * l + a];
                        for (int b = 0; b < 3; b++)
                            eps[s + nw * (a + 3 * b)] = epsilon[l + (long)nmax * (a + 3 * b)];
                    }
                    l++;
                } else {
                    orc_ondeplane(x, y, z, k0, E0, pp, theta, phi, xr + 3 * s);
                }
            }
    memcpy(incident, xr, sizeof(zc) * 3 * nw);
    zc *G6 = (zc *)malloc(sizeof(zc) * 6 * 8 * nw);
    if (nquad > 0) orc_greencalculquadfft(nxw, nyw, nzw, nquad, d, k0, G6);
    else orc_greencalculfft(nxw, nyw, nzw, d, k0, G6);
    orc_matvec_opt(G6, nxw, nyw, nzw, xi, xr);
    free(G6);
    memcpy(local, xr, sizeof(zc) * 3 * nw);
    int bad = 0;
    for (long q = 0; q < nw; q++) {
        zc e[9], loc[3];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) e[a + 3 * b] = eps[q + nw * (a + 3 * b)];
        for (int a = 0; a < 3; a++) loc[a] = xr[3 * q + a];
        bad |= orc_local_macro(loc, macro + 3 * q, e, d, k0, 1);
    }
    free(xi);
    free(xr);
    free(eps);
    return bad;
}

/* ------------------------------------------------------------------------- */
/* Microscopes in transmission with the FFT lens (nquicklens = 1, nside = +1): */
/* bright field cdmlib/microsbf.f (ntypemic = 1) and dark field / phase       */
/* cdmlib/microsdf.f (ntypemic = 2) over the rigorous full-box solve; far     */
/* field cdmlib/diffractefft2dlens.f, image cdmlib/fouriertoimage.f, grid     */
/* index cdmlib/deltakroutine.f.  numaper is the objective's NA times k0, as  */
/* cdmlib.f:3674 passes it.  image: 6 arrays of n*n (x, y, z, then the same   */
/* with the incident field), pixel u + n v, each sqrt(sum |E|^2) over the     */
/* incidences and both polarisations.  Returns nstop.                        */
/* ------------------------------------------------------------------------- */

/* deltakroutine.f:1-17: nearest grid index, truncated when outside na */
static void orc_deltakroutine(double kxinc, double kyinc, double dkx, double dky, double na, int *i,
                              int *j) {
    *i = (int)lround(kxinc / dkx);
    *j = (int)lround(kyinc / dky);
    double kx = dkx * *i, ky = dky * *j;
    if (kx * kx + ky * ky <= na * na) return;
    *i = (int)(kxinc / dkx);
    *j = (int)(kyinc / dky);
}

/* slot of 1-based index i in the FFT array (tabfft2, diffractefft2dlens.f:48-56) */
static int orc_tabfft2(int i, int n) {
    int n2 = n / 2;
    return (i - n2 - 1 >= 0) ? i - n2 : n2 + i;
}

/* diffractefft2dlens.f:1-181 (nside = +1).  Ediff: (2 imax + 1)^2 x 3 with
   entry ((jj * S + ii) * 3 + c), ii = imax + i, jj = imax + j. */
static int orc_diffractefft2dlens(int nx, int ny, int nz, int n, double k0, const double *xs,
                                  const double *ys, const double *zs, double d, const zc *FF,
                                  double numaper, double dside, int *imax_out, zc **Ediff_out,
                                  char *infostr) {
    const double pi = acos(-1.0);
    double dkx = 2.0 * pi / ((double)n * d), dky = dkx;
    if (n > 16384) { set_info(infostr, "nfft2d too large"); return 1; }
    if (dkx >= numaper) { set_info(infostr, "In FFT lens nfft2d too small"); return 1; }
    int n2 = n / 2;
    double var1 = (xs[0] + (double)n2 * d) * dkx;
    double var2 = (ys[0] + (double)n2 * d) * dky;
    int imax = (int)lround(k0 / dkx) + 1;
    if (2 * imax + 1 > n) {
        set_info(infostr, "In FFT diffraction for lens nfft2d too small!");
        return 1;
    }
    if (2 * imax + 1 < 7) { set_info(infostr, "In FFT diffract nfft2d too small"); return 1; }
    int S = 2 * imax + 1;
    zc *Ed = (zc *)calloc((size_t)S * S * 3, sizeof(zc));
    zc *E = (zc *)malloc(sizeof(zc) * 3 * (size_t)n * n);
    for (int k = 1; k <= nz; k++) {
        memset(E, 0, sizeof(zc) * 3 * (size_t)n * n);
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j <= ny; j++) {
                long kk = i + (long)nx * (j - 1) + (long)nx * ny * (k - 1);
                long ind = (orc_tabfft2(i, n) - 1) + (long)n * (orc_tabfft2(j, n) - 1);
                for (int c = 0; c < 3; c++) E[c * (size_t)n * n + ind] = FF[3 * (kk - 1) + c];
            }
        for (int c = 0; c < 3; c++) orc_fft3d(E + c * (size_t)n * n, n, n, 1, -1);
        long kk = 1 + (long)nx * ny * (k - 1);
        for (int i = -imax; i <= imax; i++)
            for (int j = -imax; j <= imax; j++) {
                double kx = (double)i * dkx, ky = (double)j * dky;
                if (kx * kx + ky * ky < numaper * numaper) {
                    double kz = sqrt(k0 * k0 - kx * kx - ky * ky);
                    long ind = (orc_tabfft2(i + n2 + 1, n) - 1) +
                               (long)n * (orc_tabfft2(j + n2 + 1, n) - 1);
                    zc ex = E[ind], ey = E[(size_t)n * n + ind], ez = E[2 * (size_t)n * n + ind];
                    zc ctmp = (kx * ex + ky * ey + kz * dside * ez) / k0;
                    zc ctmp1 = cexp(-I * dside * kz * zs[kk - 1]) * cexp(-I * (var1 * i + var2 * j)) /
                               (-2.0 * pi * I * kz);
                    zc *o = Ed + ((size_t)(imax + j) * S + (imax + i)) * 3;
                    o[0] += (ex - kx * ctmp / k0) * ctmp1;
                    o[1] += (ey - ky * ctmp / k0) * ctmp1;
                    o[2] += (ez - kz * dside * ctmp / k0) * ctmp1;
                }
            }
    }
    for (size_t q = 0; q < (size_t)S * S * 3; q++) Ed[q] = Ed[q] * k0 * k0;
    free(E);
    *imax_out = imax;
    *Ediff_out = Ed;
    return 0;
}

/* fouriertoimage.f:1-128: 2-D FFT (sign -1) of the six arrays, centred
   (fftshift) and scaled by dkx dky / gross */
static void orc_fouriertoimage(double dkx, double dky, double gross, zc *F, int n) {
    int n2 = n / 2;
    double tmp = dkx * dky / gross;
    for (int c = 0; c < 6; c++) orc_fft3d(F + c * (size_t)n * n, n, n, 1, -1);
    for (int c = 0; c < 6; c++) {
        zc *a = F + c * (size_t)n * n;
        for (int i = -n2; i <= n2 - 1; i++)
            for (int j = -n2; j <= -1; j++) {
                int ix = i >= 0 ? i + 1 : n + i + 1, iy = j >= 0 ? j + 1 : n + j + 1;
                long ind = (ix - 1) + (long)n * (iy - 1);
                long kk = (i + n2) + (long)n * (j + n2);
                zc t = a[kk];
                a[kk] = a[ind] * tmp;
                a[ind] = t * tmp;
            }
    }
}

/* the lens's far field by direct summation over the dipoles (nquicklens = 0,
   microsbf.f:627-666): inside dsqrt(kx^2 + ky^2) <= numaper, Ed =
   k0^2 / (-2 pi i kz) sum exp(-i k0 n.r) (p - n (n.p)), n = (kx, ky, dside kz) / k0 */
static void orc_lens_direct(int nb, const double *xs, const double *ys, const double *zs, const zc *FF,
                            double k0, double numaper, double dside, int imax, double dkx, zc *Ed) {
    const double pi = acos(-1.0);
    int S = 2 * imax + 1;
    for (int i = -imax; i <= imax; i++) {
        double kx = dkx * (double)i;
        for (int j = -imax; j <= imax; j++) {
            double ky = dkx * (double)j;
            zc *o = Ed + ((size_t)(imax + j) * S + (imax + i)) * 3;
            o[0] = o[1] = o[2] = 0;
            if (!(sqrt(kx * kx + ky * ky) <= numaper)) continue;
            double kz = sqrt(k0 * k0 - kx * kx - ky * ky);
            double n0 = kx / k0, n1 = ky / k0, n2 = sqrt(1.0 - n0 * n0 - n1 * n1) * dside;
            zc Ex = 0, Ey = 0, Ez = 0;
            for (int q = 0; q < nb; q++) {
                zc ctmp = cexp(-I * k0 * (n0 * xs[q] + n1 * ys[q] + n2 * zs[q]));
                zc ctmp1 = n0 * FF[3 * q] + n1 * FF[3 * q + 1] + n2 * FF[3 * q + 2];
                Ex += ctmp * (FF[3 * q] - ctmp1 * n0);
                Ey += ctmp * (FF[3 * q + 1] - ctmp1 * n1);
                Ez += ctmp * (FF[3 * q + 2] - ctmp1 * n2);
            }
            zc ct = -2.0 * pi * I * kz;
            o[0] = Ex * k0 * k0 / ct;
            o[1] = Ey * k0 * k0 / ct;
            o[2] = Ez * k0 * k0 / ct;
        }
    }
}

int orc_microscope(int ntypemic, int nside, int nquicklens, const zc *G6, int nx, int ny, int nz,
                   double d, double k0, int nbsphere, const int *tabdip, const double *xs,
                   const double *ys, const double *zs, const zc *pol,
                   const char *methodeit, double tol, double numaper, double numaperinc, int n,
                   double gross, double zlens, double P0, double w0, double *image, double *xy,
                   double *kxy, int *ninc, double *kxinc_out, double *kyinc_out, double *tol1,
                   int *nloop, int *ncompte, char *infostr) {
    const double pi = acos(-1.0);
    int N = nbsphere, nmax = nx * ny * nz;
    long n3 = 3L * N;
    int n2 = n / 2;
    double numaperk = k0 * numaperinc;
    /* cdmlib.f:237-238, 389: nside 0 (transmission) -> +1, 1 (reflection,
       microsbfneg / microsdfneg of microssansinc.f) -> -1; zlens takes the sign */
    double dside = nside == 1 ? -1.0 : 1.0;
    zlens = zlens * dside;
    set_info(infostr, "");
    if (numaperinc >= 1.0 || numaper <= 0.0) {
        set_info(infostr, "NA inc strictly between 0 and 1");
        return 1;
    }
    double xmax = -1e300, xmin = 1e300, ymax = -1e300, ymin = 1e300;
    for (int i = 0; i < N; i++) {
        xmax = fmax(xmax, xs[i]); xmin = fmin(xmin, xs[i]);
        ymax = fmax(ymax, ys[i]); ymin = fmin(ymin, ys[i]);
    }
    double deltakm = pi / fmax(xmax - xmin, ymax - ymin);
    double dkx = 2.0 * pi / (d * (double)n), dky;
    double deltak;
    int imaxinc, imaxk0 = 0;
    if (nquicklens == 1) {
        if (dkx >= numaperk) {
            set_info(infostr, "In FFT lens nfft2d too small:Increase size of FFT 1");
            return 1;
        }
        int imul = (int)(deltakm / dkx);
        if (imul == 0) {
            set_info(infostr, "In FFT lens nfft2d too small:Increase size of FFT 2");
            return 1;
        }
        for (;;) {
            deltak = dkx * (double)imul;
            imaxinc = (int)lround(k0 / deltak) + 1;
            if (imaxinc > 3) break;
            imul--;
            if (imul == 0) {
                set_info(infostr, "In FFT lens nfft2d too small:Increase size of FFT 3");
                return 1;
            }
        }
    } else {
        /* microsbf.f:139-157: halve the pupil step until more than 5 points
           cover k0, then the incidence step from the object's size */
        for (int k = 0;; k++) {
            dkx = 2.0 * pi / ((double)n * d) / (double)(1 << k);
            imaxk0 = (int)lround(k0 / dkx) + 1;
            if (imaxk0 > 5) break;
        }
        for (int k = 0;; k++) {
            deltak = dkx * round(deltakm / dkx) / (double)(1 << k);
            imaxinc = (int)lround(k0 / deltak) + 1;
            if (imaxinc > 2) break;
        }
        if (2 * imaxk0 + 1 > n) {
            set_info(infostr, "In FFT lens nfft2d too small");
            return 1;
        }
    }
    dky = dkx;
    /* incidence list of one polarisation */
    int cap = 0, cnt = 0;
    double *kxi = NULL, *kyi = NULL;
    if (ntypemic == 1) {
        int m = imaxinc;
        cap = (2 * m + 1) * (2 * m + 1);
        kxi = (double *)malloc(sizeof(double) * cap);
        kyi = (double *)malloc(sizeof(double) * cap);
        for (int id = -m; id <= m; id++)
            for (int jd = -m; jd <= m; jd++) {
                double kx = id * deltak, ky = jd * deltak;
                if (kx * kx + ky * ky <= numaperk * numaperk) { kxi[cnt] = kx; kyi[cnt] = ky; cnt++; }
            }
        if (n > 16384) { set_info(infostr, "nfft2d too large"); free(kxi); free(kyi); return 1; }
        if (deltak >= numaperk) {
            set_info(infostr, "In FFT lens nfft2d too small");
            free(kxi); free(kyi);
            return 1;
        }
    } else if (ntypemic == 2) {
        double deltatheta = deltak / k0 * numaperinc;
        int m = (int)(2.0 * pi / deltatheta) + 1;
        if (m < 8) m = 8;
        kxi = (double *)malloc(sizeof(double) * m);
        kyi = (double *)malloc(sizeof(double) * m);
        for (int id = 0; id < m; id++) {
            double phi = (double)id * 2.0 * pi / (double)m;
            kxi[cnt] = cos(phi) * k0 * numaperinc;
            kyi[cnt] = sin(phi) * k0 * numaperinc;
            cnt++;
        }
    } else {
        set_info(infostr, "ntypemic must be 1 or 2");
        return 1;
    }
    int cap_out = *ninc;
    *ninc = cnt;
    for (int q = 0; q < cnt && q < cap_out; q++) {
        if (kxinc_out) kxinc_out[q] = kxi[q] / k0;
        if (kyinc_out) kyinc_out[q] = kyi[q] / k0;
    }
    double E0r, irra;
    orc_irradiance(P0 / (double)(2 * cnt), w0, &E0r, &irra);
    zc E0 = E0r;
    memset(image, 0, sizeof(double) * 6 * (size_t)n * n);
    zc *FF0 = (zc *)malloc(sizeof(zc) * n3), *FF = (zc *)malloc(sizeof(zc) * n3),
       *FFloc = (zc *)malloc(sizeof(zc) * n3);
    zc *F = (zc *)malloc(sizeof(zc) * 6 * (size_t)n * n);
    int nstop = 0, imax = 0;
    for (int ipol = 1; ipol <= 2 && !nstop; ipol++) {
        double pp = ipol == 1 ? 0.0 : 1.0;
        for (int q = 0; q < cnt && !nstop; q++) {
            double kxinc = kxi[q], kyinc = kyi[q];
            for (int i = 0; i < N; i++) orc_ondeplanekxky(xs[i], ys[i], zs[i], k0, E0, pp, kxinc, kyinc, FF0 + 3L * i);
            orc_inverserig(G6, nx, ny, nz, N, tabdip, pol, nmax, FF0, methodeit, tol, FF, FFloc, tol1, nloop,
                           ncompte, &nstop, infostr, NULL, 0);
            if (nstop == 1) break;
            zc *Ed = NULL;
            if (nquicklens == 0) {
                imax = imaxk0;
                Ed = (zc *)malloc(sizeof(zc) * (size_t)(2 * imax + 1) * (2 * imax + 1) * 3);
                orc_lens_direct(N, xs, ys, zs, FF, k0, numaper, dside, imax, dkx, Ed);
            } else if (orc_diffractefft2dlens(nx, ny, nz, n, k0, xs, ys, zs, d, FF, numaper, dside, &imax, &Ed,
                                              infostr)) {
                nstop = 1;
                break;
            }
            int S = 2 * imax + 1;
            memset(F, 0, sizeof(zc) * 6 * (size_t)n * n);
            int ik, jk;
            if (ntypemic == 1) orc_deltakroutine(kxinc, kyinc, deltak, deltak, k0, &ik, &jk);
            else orc_deltakroutine(kxinc, kyinc, dkx, dky, k0, &ik, &jk);
            double dkxy = dkx * dky;
            for (int i = -imax; i <= imax; i++)
                for (int j = -imax; j <= imax; j++) {
                    int ix = i >= 0 ? i + 1 : n + i + 1, iy = j >= 0 ? j + 1 : n + j + 1;
                    long ind = (ix - 1) + (long)n * (iy - 1);
                    double kx = dkx * i, ky = dky * j, tmp = kx * kx + ky * ky;
                    if (!(tmp <= numaper * numaper)) continue;
                    double kz = sqrt(k0 * k0 - tmp);
                    zc zf = cexp(I * kz * zlens);
                    zc *e = Ed + ((size_t)(imax + j) * S + (imax + i)) * 3;
                    zc f[6];
                    for (int c = 0; c < 3; c++) f[c] = f[c + 3] = e[c] * zf;
                    /* the reflection side forms no image with the incident wave */
                    if (dside < 0)
                        for (int c = 3; c < 6; c++) f[c] = 0;
                    if (dside > 0 && i == ik && j == jk) {
                        zc Ei[3];
                        orc_ondeplanekxky(0.0, 0.0, 0.0, k0, E0, pp, kx, ky, Ei);
                        if (ntypemic == 1) {
                            /* microsbf.f: z divided by deltaky alone, as the reference does */
                            f[3] += Ei[0] / dkxy * zf;
                            f[4] += Ei[1] / dkxy * zf;
                            f[5] += Ei[2] / dky * zf;
                        } else {
                            for (int c = 0; c < 3; c++) f[3 + c] += Ei[c] / dkx / dky * zf * I;
                        }
                    }
                    if (tmp != 0.0) {
                        double u[3], v[3];
                        u[0] = kx / k0; u[1] = ky / k0;
                        u[2] = sqrt(1.0 - u[0] * u[0] - u[1] * u[1]) * dside;
                        v[0] = -kx / k0 / gross; v[1] = -ky / k0 / gross;
                        v[2] = sqrt(1.0 - v[0] * v[0] - v[1] * v[1]) * dside;
                        double u1 = u[1] * v[2] - u[2] * v[1];
                        double u2 = -u[0] * v[2] + u[2] * v[0];
                        double cs = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
                        double sn = sqrt(u1 * u1 + u2 * u2);
                        u1 = u1 / sn;
                        u2 = u2 / sn;
                        double t = sqrt(u[2] / v[2]);
                        for (int h = 3; h >= 0; h -= 3) {
                            zc X = f[h], Y = f[h + 1], Z = f[h + 2];
                            zc tx = (u1 * u1 + (1.0 - u1 * u1) * cs) * X + u1 * u2 * (1.0 - cs) * Y + u2 * sn * Z;
                            zc ty = u1 * u2 * (1.0 - cs) * X + (u2 * u2 + (1.0 - u2 * u2) * cs) * Y - u1 * sn * Z;
                            zc tz = -u2 * sn * X + u1 * sn * Y + cs * Z;
                            f[h] = tx * t;
                            f[h + 1] = ty * t;
                            f[h + 2] = tz * t;
                        }
                    }
                    for (int c = 0; c < 6; c++) F[c * (size_t)n * n + ind] = f[c];
                }
            free(Ed);
            orc_fouriertoimage(dkx, dky, gross, F, n);
            for (size_t p = 0; p < 6 * (size_t)n * n; p++)
                image[p] += creal(F[p] * conj(F[p]));
        }
    }
    free(FF0); free(FF); free(FFloc); free(F); free(kxi); free(kyi);
    if (nstop) return nstop;
    for (size_t p = 0; p < 6 * (size_t)n * n; p++) image[p] = sqrt(image[p]);
    double deltax = 2.0 * pi / (double)n / dkx;
    for (int i = -n2; i <= n2 - 1; i++) {
        xy[i + n2] = deltax * (double)i * gross;
        kxy[i + n2] = dkx * (double)i / k0;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Far field on the pupil grid: diffractefft2d.f:1-183 (both sides, full box), */
/* computegcfft2d.f:1-51 (Cscai, gasym) and the Poynting interpolation of     */
/* cdmlib.f:2990-3075 (nsectionsca = 1, nquickdiffracte = 1).                 */
/* ------------------------------------------------------------------------- */
int orc_farfield_fft(int nx, int ny, int nz, double d, const double *xs, const double *ys,
                     const double *zs, const zc *FF, double k0, double I0, double theta, double phi,
                     int n, int ntheta, int nphi, double *Cscai, double *gasym, double *poynting,
                     double *thetafield, double *phifield, int *imax_out, double *kpos, double *kneg,
                     char *infostr) {
    const double pi = acos(-1.0), c = 299792458.0, quatpieps0 = 1.0 / (c * c * 1e-7);
    double dkx = 2.0 * pi / ((double)n * d), dky = dkx;
    int n2 = n / 2;
    double var1 = (xs[0] + (double)n2 * d) * dkx, var2 = (ys[0] + (double)n2 * d) * dky;
    if (n > 16384) { set_info(infostr, "nfft2d too large"); return 1; }
    if (dkx >= k0) { set_info(infostr, "In FFT Poynting nfft2d too small"); return 1; }
    int imax = (int)lround(k0 / dkx) + 1, S = 2 * imax + 1;
    if (S > n || S < 7) { set_info(infostr, "In FFT diffract nfft2d too small"); return 1; }
    if (ntheta <= 10 || nphi <= 20) { set_info(infostr, "ntheta and nphi too small!"); return 1; }
    zc *Ep = (zc *)calloc((size_t)S * S * 3, sizeof(zc)), *En = (zc *)calloc((size_t)S * S * 3, sizeof(zc));
    zc *E = (zc *)malloc(sizeof(zc) * 3 * (size_t)n * n);
    for (int k = 1; k <= nz; k++) {
        memset(E, 0, sizeof(zc) * 3 * (size_t)n * n);
        for (int i = 1; i <= nx; i++)
            for (int j = 1; j <= ny; j++) {
                long kk = i + (long)nx * (j - 1) + (long)nx * ny * (k - 1);
                long ind = (orc_tabfft2(i, n) - 1) + (long)n * (orc_tabfft2(j, n) - 1);
                for (int q = 0; q < 3; q++) E[q * (size_t)n * n + ind] = FF[3 * (kk - 1) + q];
            }
        for (int q = 0; q < 3; q++) orc_fft3d(E + q * (size_t)n * n, n, n, 1, -1);
        long kk = 1 + (long)nx * ny * (k - 1);
        for (int i = -imax; i <= imax; i++)
            for (int j = -imax; j <= imax; j++) {
                double kx = (double)i * dkx, ky = (double)j * dky;
                if (!(k0 * k0 - kx * kx - ky * ky > 0.0)) continue;
                double kz = sqrt(k0 * k0 - kx * kx - ky * ky);
                long ind = (orc_tabfft2(i + n2 + 1, n) - 1) + (long)n * (orc_tabfft2(j + n2 + 1, n) - 1);
                zc ex = E[ind], ey = E[(size_t)n * n + ind], ez = E[2 * (size_t)n * n + ind];
                zc ph = cexp(-I * (var1 * i + var2 * j));
                zc ctmp = (kx * ex + ky * ey + kz * ez) / k0;
                zc ctmp1 = cexp(-I * kz * zs[kk - 1]) * ph;
                zc *o = Ep + ((size_t)(imax + j) * S + (imax + i)) * 3;
                o[0] += (ex - kx * ctmp / k0) * ctmp1;
                o[1] += (ey - ky * ctmp / k0) * ctmp1;
                o[2] += (ez - kz * ctmp / k0) * ctmp1;
                ctmp = (kx * ex + ky * ey - kz * ez) / k0;
                ctmp1 = cexp(I * kz * zs[kk - 1]) * ph;
                o = En + ((size_t)(imax + j) * S + (imax + i)) * 3;
                o[0] += (ex - kx * ctmp / k0) * ctmp1;
                o[1] += (ey - ky * ctmp / k0) * ctmp1;
                o[2] += (ez + kz * ctmp / k0) * ctmp1;
            }
    }
    free(E);
#define EMOD(A, i, j)                                                                           \
    (cabs((A)[((size_t)(imax + (j)) * S + (imax + (i))) * 3]) *                                 \
         cabs((A)[((size_t)(imax + (j)) * S + (imax + (i))) * 3]) +                             \
     cabs((A)[((size_t)(imax + (j)) * S + (imax + (i))) * 3 + 1]) *                             \
         cabs((A)[((size_t)(imax + (j)) * S + (imax + (i))) * 3 + 1]) +                         \
     cabs((A)[((size_t)(imax + (j)) * S + (imax + (i))) * 3 + 2]) *                             \
         cabs((A)[((size_t)(imax + (j)) * S + (imax + (i))) * 3 + 2]))
    double sth = sin(theta * pi / 180.0), cph = cos(phi * pi / 180.0), sph = sin(phi * pi / 180.0),
           cth = cos(theta * pi / 180.0);
    double cs = 0.0, g = 0.0;
    int k = 0;
    for (int i = -imax; i <= imax; i++)
        for (int j = -imax; j <= imax; j++, k++) {
            double kx = (double)i * dkx, ky = (double)j * dky;
            kpos[k] = 0.0;
            kneg[k] = 0.0;
            if (!(k0 * k0 - kx * kx - ky * ky > 0.0)) continue;
            double kz = sqrt(k0 * k0 - kx * kx - ky * ky);
            double e = EMOD(Ep, i, j);
            kpos[k] = e * k0 * k0 * k0 * k0 * c / 8 / pi * quatpieps0;
            cs = cs + dkx * dky * e / kz;
            g = g + dkx * dky * e / kz * (kx * sth * cph + ky * sth * sph + kz * cth) / k0;
            e = EMOD(En, i, j);
            kneg[k] = e * k0 * k0 * k0 * k0 * c / 8 / pi * quatpieps0;
            cs = cs + dkx * dky * e / kz;
            g = g + dkx * dky * e / kz * (kx * sth * cph + ky * sth * sph - kz * cth) / k0;
        }
    *gasym = g / cs;
    *Cscai = cs * (k0 * k0 * k0) / I0;
    *imax_out = imax;
    double deltatheta = pi / (double)ntheta, deltaphi = 2.0 * pi / (double)nphi;
    int cnt = 0;
    for (int itheta = 0; itheta <= ntheta; itheta++) {
        double thetas = deltatheta * (double)itheta;
        for (int iphi = 0; iphi < nphi; iphi++, cnt++) {
            double phis = deltaphi * (double)iphi;
            thetafield[cnt] = thetas * 180.0 / pi;
            phifield[cnt] = phis * 180.0 / pi;
            double kx = k0 * sin(thetas) * cos(phis), ky = k0 * sin(thetas) * sin(phis);
            int i2 = -imax, j2 = -imax;
            for (int i = -imax; i <= imax; i++)
                if (kx >= i * dkx) i2 = i;
            for (int j = -imax; j <= imax; j++)
                if (ky >= j * dkx) j2 = j;
            zc *A = thetas <= pi / 2.0 ? Ep : En;
            double e11 = EMOD(A, i2, j2), e22 = EMOD(A, i2 + 1, j2 + 1), e21 = EMOD(A, i2 + 1, j2),
                   e12 = EMOD(A, i2, j2 + 1);
            int test = (e11 == 0.0) + (e22 == 0.0) + (e21 == 0.0) + (e12 == 0.0);
            double e;
            if (test == 0)
                e = (e21 - e11) * (kx - dkx * i2) / dkx + (e12 - e11) * (ky - dkx * j2) / dkx +
                    (e11 + e22 - e12 - e21) * (kx - dkx * i2) / dkx * (ky - dkx * j2) / dkx + e11;
            else
                e = (e11 + e12 + e21 + e22) / (double)(4 - test);
            poynting[cnt] = e * k0 * k0 * k0 * k0 * c / 8.0 / pi * quatpieps0;
        }
    }
#undef EMOD
    free(Ep);
    free(En);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Holographic microscope (ntypemic = 0) with the FFT lens, after the solve of */
/* one plane wave (cdmlib.f:4075-4660 with nenergie = 0 and the lens far      */
/* field computed afresh): diffractefft2dlens, the incident wave in the pupil */
/* (diffractefft2dinc.f:75-91 for 'pwavelinear': E / dk^2 at the grid point   */
/* of deltakroutine), the lens rotation, then fouriertoimage (fouriertoimage2 */
/* on the reflection side).  nside 0 transmission, 1 reflection.  image: 6    */
/* complex arrays of n*n (x, y, z, then with the incident wave; the latter    */
/* stay zero on the reflection side); fourier: 6 arrays of (2 imax + 1)^2     */
/* (row j, column i), the pupil fields before the rotation.  Returns nstop.  */
/* ------------------------------------------------------------------------- */
int orc_holography(int nx, int ny, int nz, double d, double k0, int nb, const double *xs,
                   const double *ys, const double *zs, const zc *FF, zc E0, double theta,
                   double phi, double pp, int n, double numaper, double gross, double zlens,
                   int nside, int nquicklens, zc *image, zc *fourier, double *xy, double *kxy,
                   int *imax_out, char *infostr) {
    const double pi = acos(-1.0);
    double dside = nside == 1 ? -1.0 : 1.0;
    zlens = zlens * dside;
    numaper = numaper * k0;
    set_info(infostr, "");
    int imax = 0;
    zc *Ed = NULL;
    double dkx = 2.0 * pi / ((double)n * d), dky;
    if (nquicklens == 1) {
        if (orc_diffractefft2dlens(nx, ny, nz, n, k0, xs, ys, zs, d, FF, numaper, dside, &imax, &Ed,
                                   infostr))
            return 1;
    } else {
        /* cdmlib.f:3818-3826: halve the pupil step until more than 20
           points cover k0; the far field by direct summation */
        for (int k = 0;; k++) {
            dkx = 2.0 * pi / ((double)n * d) / (double)(1 << k);
            imax = (int)lround(k0 / dkx) + 1;
            if (imax > 20) break;
        }
        if (2 * imax + 1 > n) {
            set_info(infostr, "In FFT lens nfft2d too small");
            return 1;
        }
        Ed = (zc *)malloc(sizeof(zc) * (size_t)(2 * imax + 1) * (2 * imax + 1) * 3);
        orc_lens_direct(nb, xs, ys, zs, FF, k0, numaper, dside, imax, dkx, Ed);
    }
    int S = 2 * imax + 1, n2 = n / 2;
    dky = dkx;
    /* the incident wave on the pupil grid (transmission only) */
    zc *Ei = (zc *)calloc((size_t)S * S * 3, sizeof(zc));
    if (dside > 0) {
        if (dkx >= numaper) {
            set_info(infostr, "In FFT lens inc nfft2d too small");
            free(Ed); free(Ei);
            return 1;
        }
        double kxinc = sin(theta * pi / 180.0) * cos(phi * pi / 180.0) * k0;
        double kyinc = sin(theta * pi / 180.0) * sin(phi * pi / 180.0) * k0;
        int ik, jk;
        orc_deltakroutine(kxinc, kyinc, dkx, dky, k0, &ik, &jk);
        double kx = dkx * (double)ik, ky = dkx * (double)jk;
        zc E[3];
        orc_ondeplanekxky(0.0, 0.0, 0.0, k0, E0, pp, kx, ky, E);
        zc *o = Ei + ((size_t)(imax + jk) * S + (imax + ik)) * 3;
        for (int c = 0; c < 3; c++) o[c] = E[c] / dkx / dkx;
    }
    zc *F = (zc *)calloc(6 * (size_t)n * n, sizeof(zc));
    if (fourier) memset(fourier, 0, sizeof(zc) * 6 * (size_t)S * S);
    for (int i = -imax; i <= imax; i++)
        for (int j = -imax; j <= imax; j++) {
            int ix = i >= 0 ? i + 1 : n + i + 1, iy = j >= 0 ? j + 1 : n + j + 1;
            long ind = (ix - 1) + (long)n * (iy - 1);
            double kx = dkx * (double)i, ky = dkx * (double)j;
            double kz;
            if (nquicklens == 1) {
                kz = k0 * k0 - kx * kx - ky * ky;
                if (!(kz >= 0.0)) continue;
                kz = sqrt(kz);
            } else {
                /* cdmlib.f:3885-3916: the objective's aperture */
                if (!(sqrt(kx * kx + ky * ky) <= numaper)) continue;
                kz = sqrt(k0 * k0 - kx * kx - ky * ky);
            }
            zc zf = cexp(I * kz * zlens);
            zc *e = Ed + ((size_t)(imax + j) * S + (imax + i)) * 3;
            zc *ei = Ei + ((size_t)(imax + j) * S + (imax + i)) * 3;
            zc f[6];
            for (int c = 0; c < 3; c++) {
                f[c] = e[c] * zf;
                if (dside < 0) f[c + 3] = 0;
                else f[c + 3] = nquicklens == 1 ? (e[c] + ei[c]) * zf : f[c] + ei[c] * zf;
            }
            if (fourier)
                for (int c = 0; c < 6; c++) fourier[(size_t)c * S * S + (size_t)(imax + j) * S + (imax + i)] = f[c];
            double u[3], v[3];
            u[0] = kx / k0; u[1] = ky / k0; u[2] = sqrt(1.0 - u[0] * u[0] - u[1] * u[1]) * dside;
            v[0] = -kx / k0 / gross; v[1] = -ky / k0 / gross;
            v[2] = sqrt(1.0 - v[0] * v[0] - v[1] * v[1]) * dside;
            double u1 = u[1] * v[2] - u[2] * v[1];
            double u2 = -u[0] * v[2] + u[2] * v[0];
            double cs = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
            double sn = sqrt(u1 * u1 + u2 * u2);
            if (sn == 0.0) {
                for (int c = 0; c < 6; c++) F[(size_t)c * n * n + ind] = f[c];
                continue;
            }
            u1 = u1 / sn;
            u2 = u2 / sn;
            double t = sqrt(u[2] / v[2]);
            for (int h = 0; h < 6; h += 3) {
                zc X = f[h], Y = f[h + 1], Z = f[h + 2];
                F[(size_t)h * n * n + ind] =
                    ((u1 * u1 + (1.0 - u1 * u1) * cs) * X + u1 * u2 * (1.0 - cs) * Y + u2 * sn * Z) * t;
                F[(size_t)(h + 1) * n * n + ind] =
                    (u1 * u2 * (1.0 - cs) * X + (u2 * u2 + (1.0 - u2 * u2) * cs) * Y - u1 * sn * Z) * t;
                F[(size_t)(h + 2) * n * n + ind] = (-u2 * sn * X + u1 * sn * Y + cs * Z) * t;
            }
        }
    free(Ed);
    free(Ei);
    orc_fouriertoimage(dkx, dky, gross, F, n);
    memcpy(image, F, sizeof(zc) * 6 * (size_t)n * n);
    free(F);
    double deltax = 2.0 * pi / (double)n / dkx;
    for (int i = -n2; i <= n2 - 1; i++) {
        xy[i + n2] = deltax * (double)i * gross;
        kxy[i + n2] = dkx * (double)i / k0;
    }
    *imax_out = imax;
    return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
