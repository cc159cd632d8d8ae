// Microscope image formation with the FFT lens, for a batch of solved
// incidences (cdmlib/microsbf.f, cdmlib/microsdf.f with nquicklens = 1 and
// nside = +1).
//
// The reference pads every lattice plane to an n x n array, runs a 2-D FFT
// per plane and keeps the (2 imax + 1)^2 frequencies inside the pupil
// (diffractefft2dlens.f:86-150).  Here the same sums are evaluated only at
// those frequencies, as two separable DFTs: along x for every (plane, row)
// (k_mic_xdft) and along y, summed over the planes with the reference's
// projection and phase factors (k_mic_far).  The DFT phases are exact roots
// of unity from the table exp(+2 pi i m / n), indexed by the integer product
// of frequency and slot, so the values are the FFT's to rounding.
//
// The image (fouriertoimage.f) is a 2-D FFT of the pupil field: the rows
// (k_mic_rows) transform only the S rows that hold the pupil, the columns
// (k_mic_cols) then transform every column and add |E|^2 of all incidences
// of the batch in registers before one update of the image sums.  Both use
// the shared-memory Stockham engine of the mat-vec (fft_tile.cuh).
#include <algorithm>
#include "microscope.cuh"
#include "fft_tile.cuh"
#include "planewave.cuh"
#include "reduce.cuh"

namespace ifdda {

namespace {

// slot p (0 <= p < n) of a transform along one axis -> row of the pupil
// (frequency p or p - n), or -1 outside |frequency| <= imax
__device__ __forceinline__ int pupil_row(int p, int imax, int n) {
    return p <= imax ? p + imax : (p >= n - imax ? p - n + imax : -1);
}

__device__ __forceinline__ int posmod(long a, int n) {
    const long r = a % n;
    return (int)(r < 0 ? r + n : r);
}

// x-DFT of every (incidence, plane, row): Q[b][k][y][irow][c] =
// sum_x FF[b][x, y, k][c] exp(-2 pi i (irow - imax)(x - n/2) / n)
__global__ void __launch_bounds__(256) k_mic_xdft(const MicGeom m, int nb, const double2* __restrict__ FF,
                                                   const double2* __restrict__ tw, double2* __restrict__ Q) {
    const int S = m.S();
    const long total = (long)nb * m.nz * m.ny * S;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int irow = (int)(t % S);
    long r = t / S;
    const int y = (int)(r % m.ny);
    r /= m.ny;
    const int k = (int)(r % m.nz);
    const int b = (int)(r / m.nz);
    const int n = m.n, i = irow - m.imax;
    const int step = posmod(i, n);
    int ph = posmod((long)i * (-(n / 2)), n);
    const long N = (long)m.nx * m.ny * m.nz;
    const double2* p = FF + (long)b * 3 * N + 3L * ((long)m.nx * y + (long)m.nx * m.ny * k);
    double2 a0 = make_double2(0, 0), a1 = a0, a2 = a0;
    for (int x = 0; x < m.nx; x++) {
        const double2 w = cconj(tw[ph]);
        a0 = cadd(a0, cmul(p[3 * x], w));
        a1 = cadd(a1, cmul(p[3 * x + 1], w));
        a2 = cadd(a2, cmul(p[3 * x + 2], w));
        ph += step;
        if (ph >= n) ph -= n;
    }
    double2* q = Q + ((((long)b * m.nz + k) * m.ny + y) * S + irow) * 3;
    q[0] = a0;
    q[1] = a1;
    q[2] = a2;
}

// y-DFT of plane k at pupil column irow: P_c = sum_y Q[b][k][y][irow][c]
// exp(-2 pi i j (y - n/2) / n), with ph0 / step the phase index of y = 0 and
// its increment
__device__ __forceinline__ void ydft_plane(const MicGeom& m, const double2* __restrict__ Q, const double2* __restrict__ tw,
                                           int b, int k, int irow, int ph0, int step, double2& p0, double2& p1,
                                           double2& p2) {
    const int S = m.S(), n = m.n;
    const double2* q = Q + (((long)b * m.nz + k) * m.ny * S + irow) * 3;
    p0 = make_double2(0, 0);
    p1 = p0;
    p2 = p0;
    int ph = ph0;
    for (int y = 0; y < m.ny; y++) {
        const double2 w = cconj(tw[ph]);
        const double2* qy = q + (long)y * S * 3;
        p0 = cadd(p0, cmul(qy[0], w));
        p1 = cadd(p1, cmul(qy[1], w));
        p2 = cadd(p2, cmul(qy[2], w));
        ph += step;
        if (ph >= n) ph -= n;
    }
}

// y-DFT and the sum over planes (diffractefft2dlens.f:121-150): inside the
// pupil (kx^2 + ky^2 < numaper^2)
//   Ed_c = k0^2 sum_k (P_c - k_c (k.P) / k0^2) exp(-i kz z_k)
//          exp(-i (var1 i + var2 j)) / (-2 pi i kz)
// with the products and sums of the pupil test and of kz rounded one by one
// as the reference evaluates them.
__global__ void __launch_bounds__(256) k_mic_far(const MicGeom m, int nb, const double2* __restrict__ Q,
                                                  const double* __restrict__ zplane, const double2* __restrict__ tw,
                                                  double2* __restrict__ Ed) {
    const int S = m.S();
    const long total = (long)nb * S * S;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int irow = (int)(t % S);
    const int jrow = (int)((t / S) % S);
    const int b = (int)(t / ((long)S * S));
    const int i = irow - m.imax, j = jrow - m.imax, n = m.n;
    const double kx = (double)i * m.dkx, ky = (double)j * m.dky;
    double2 o0 = make_double2(0, 0), o1 = o0, o2 = o0;
    if (__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)) < __dmul_rn(m.numaper, m.numaper)) {
        const double kz = sqrt(__dsub_rn(__dsub_rn(__dmul_rn(m.k0, m.k0), __dmul_rn(kx, kx)), __dmul_rn(ky, ky)));
        double sn, cs;
        sincos(-__dadd_rn(__dmul_rn(m.var1, (double)i), __dmul_rn(m.var2, (double)j)), &sn, &cs);
        const double2 exy = make_double2(cs, sn);
        const double2 den = make_double2(0.0, -2.0 * 3.14159265358979323846 * kz);
        const int step = posmod(j, n), ph0 = posmod((long)j * (-(n / 2)), n);
        for (int k = 0; k < m.nz; k++) {
            double2 p0, p1, p2;
            ydft_plane(m, Q, tw, b, k, irow, ph0, step, p0, p1, p2);
            // ctmp = (kx P_x + ky P_y + kz dside P_z) / k0, on the side dside
            const double kzs = kz * m.dside;
            const double2 ct = make_double2((kx * p0.x + ky * p1.x + kzs * p2.x) / m.k0,
                                            (kx * p0.y + ky * p1.y + kzs * p2.y) / m.k0);
            sincos(-kzs * zplane[k], &sn, &cs);
            const double2 c1 = zdiv(cmul(make_double2(cs, sn), exy), den);
            o0 = cadd(o0, cmul(csub(p0, make_double2(kx * ct.x / m.k0, kx * ct.y / m.k0)), c1));
            o1 = cadd(o1, cmul(csub(p1, make_double2(ky * ct.x / m.k0, ky * ct.y / m.k0)), c1));
            o2 = cadd(o2, cmul(csub(p2, make_double2(kzs * ct.x / m.k0, kzs * ct.y / m.k0)), c1));
        }
        const double k02 = m.k0 * m.k0;
        o0 = cscale(o0, k02);
        o1 = cscale(o1, k02);
        o2 = cscale(o2, k02);
    }
    double2* e = Ed + (((long)b * S + jrow) * S + irow) * 3;
    e[0] = o0;
    e[1] = o1;
    e[2] = o2;
}

// Far field on both sides without a lens (diffractefft2d.f:104-170): for
// every propagating wave (k0^2 - kx^2 - ky^2 > 0) the sums over planes
//   E+_c = sum_k (P_c - k+_c (k+.P) / k0^2) exp(-i kz z_k) exp(-i (var1 i + var2 j))
//   E-_c = sum_k (P_c - k-_c (k-.P) / k0^2) exp(+i kz z_k) exp(-i (var1 i + var2 j))
// with k+- = (kx, ky, +-kz); Ed holds E+ for all nb, then E-.
__global__ void __launch_bounds__(256) k_mic_far2(const MicGeom m, int nb, const double2* __restrict__ Q,
                                                   const double* __restrict__ zplane, const double2* __restrict__ tw,
                                                   double2* __restrict__ Ed) {
    const int S = m.S();
    const long total = (long)nb * S * S;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int irow = (int)(t % S);
    const int jrow = (int)((t / S) % S);
    const int b = (int)(t / ((long)S * S));
    const int i = irow - m.imax, j = jrow - m.imax, n = m.n;
    const double kx = (double)i * m.dkx, ky = (double)j * m.dky;
    double2 a0 = make_double2(0, 0), a1 = a0, a2 = a0, c0 = a0, c1 = a0, c2 = a0;
    const double kz2 = __dsub_rn(__dsub_rn(__dmul_rn(m.k0, m.k0), __dmul_rn(kx, kx)), __dmul_rn(ky, ky));
    if (kz2 > 0.0) {
        const double kz = sqrt(kz2);
        double sn, cs;
        sincos(-__dadd_rn(__dmul_rn(m.var1, (double)i), __dmul_rn(m.var2, (double)j)), &sn, &cs);
        const double2 exy = make_double2(cs, sn);
        const int step = posmod(j, n), ph0 = posmod((long)j * (-(n / 2)), n);
        for (int k = 0; k < m.nz; k++) {
            double2 p0, p1, p2;
            ydft_plane(m, Q, tw, b, k, irow, ph0, step, p0, p1, p2);
            sincos(kz * zplane[k], &sn, &cs);
            const double2 up = cmul(make_double2(cs, -sn), exy), dn = cmul(make_double2(cs, sn), exy);
            const double2 tp = make_double2((kx * p0.x + ky * p1.x + kz * p2.x) / m.k0,
                                            (kx * p0.y + ky * p1.y + kz * p2.y) / m.k0);
            const double2 tn = make_double2((kx * p0.x + ky * p1.x - kz * p2.x) / m.k0,
                                            (kx * p0.y + ky * p1.y - kz * p2.y) / m.k0);
            a0 = cadd(a0, cmul(csub(p0, make_double2(kx * tp.x / m.k0, kx * tp.y / m.k0)), up));
            a1 = cadd(a1, cmul(csub(p1, make_double2(ky * tp.x / m.k0, ky * tp.y / m.k0)), up));
            a2 = cadd(a2, cmul(csub(p2, make_double2(kz * tp.x / m.k0, kz * tp.y / m.k0)), up));
            c0 = cadd(c0, cmul(csub(p0, make_double2(kx * tn.x / m.k0, kx * tn.y / m.k0)), dn));
            c1 = cadd(c1, cmul(csub(p1, make_double2(ky * tn.x / m.k0, ky * tn.y / m.k0)), dn));
            c2 = cadd(c2, cmul(cadd(p2, make_double2(kz * tn.x / m.k0, kz * tn.y / m.k0)), dn));
        }
    }
    double2* e = Ed + (((long)b * S + jrow) * S + irow) * 3;
    e[0] = a0;
    e[1] = a1;
    e[2] = a2;
    double2* f = e + (long)nb * S * S * 3;
    f[0] = c0;
    f[1] = c1;
    f[2] = c2;
}

// The lens's far field by direct summation over the dipoles (nquicklens = 0,
// microsbf.f:627-666): pupil point (i, j) inside sqrt(kx^2 + ky^2) <=
// numaper, n = (kx, ky, dside kz) / k0, E = sum exp(-i k0 n.r)(p - n (n.p)).
// Stage 1: block (point, chunk, incidence) sums its dipoles; stage 2 adds
// the chunks in order and applies k0^2 / (-2 pi i kz).
constexpr int MD_NT = 256;
__device__ __forceinline__ bool direct_point(const MicGeom& m, int irow, int jrow, double& kx, double& ky) {
    kx = m.dkx * (double)(irow - m.imax);
    ky = m.dkx * (double)(jrow - m.imax);
    return sqrt(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky))) <= m.numaper;
}
__global__ void __launch_bounds__(MD_NT) k_mic_direct_part(const MicGeom m, int nd, const double* __restrict__ xs,
                                                           const double* __restrict__ ys,
                                                           const double* __restrict__ zs,
                                                           const double2* __restrict__ FF, int nchunk,
                                                           double2* __restrict__ part) {
    const int S = m.S(), pt = blockIdx.x, ch = blockIdx.y, b = blockIdx.z;
    const int irow = pt % S, jrow = pt / S;
    double kx, ky;
    double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    if (direct_point(m, irow, jrow, kx, ky)) {
        const double n0 = kx / m.k0, n1 = ky / m.k0;
        const double n2 = sqrt(__dsub_rn(__dsub_rn(1.0, __dmul_rn(n0, n0)), __dmul_rn(n1, n1))) * m.dside;
        const long per = ((long)nd + nchunk - 1) / nchunk;
        const long i0 = (long)ch * per, i1 = min((long)nd, i0 + per);
        const double2* p = FF + (long)b * 3 * nd;
        for (long i = i0 + threadIdx.x; i < i1; i += MD_NT) {
            double sn, cs;
            sincos(-m.k0 * (n0 * xs[i] + n1 * ys[i] + n2 * zs[i]), &sn, &cs);
            const double2 e = make_double2(cs, sn);
            const double2 p0 = p[3 * i], p1 = p[3 * i + 1], p2 = p[3 * i + 2];
            const double2 np = make_double2(n0 * p0.x + n1 * p1.x + n2 * p2.x, n0 * p0.y + n1 * p1.y + n2 * p2.y);
            acc[0] = cadd(acc[0], cmul(e, make_double2(p0.x - np.x * n0, p0.y - np.y * n0)));
            acc[1] = cadd(acc[1], cmul(e, make_double2(p1.x - np.x * n1, p1.y - np.y * n1)));
            acc[2] = cadd(acc[2], cmul(e, make_double2(p2.x - np.x * n2, p2.y - np.y * n2)));
        }
    }
    __shared__ double2 scratch[3 * 32];
    block_sum<MD_NT, 3>(acc, scratch);
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; c++) part[(((long)b * S * S + pt) * nchunk + ch) * 3 + c] = acc[c];
}
__global__ void k_mic_direct_final(const MicGeom m, int nb, int nchunk, const double2* __restrict__ part,
                                   double2* __restrict__ Ed) {
    const int S = m.S();
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nb * S * S) return;
    const int pt = (int)(t % ((long)S * S)), b = (int)(t / ((long)S * S));
    const int irow = pt % S, jrow = pt / S;
    double kx, ky;
    double2 e[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    if (direct_point(m, irow, jrow, kx, ky)) {
        const double kz = sqrt(__dsub_rn(__dsub_rn(__dmul_rn(m.k0, m.k0), __dmul_rn(kx, kx)), __dmul_rn(ky, ky)));
        const double2 den = make_double2(0.0, -2.0 * 3.14159265358979323846 * kz);
        for (int ch = 0; ch < nchunk; ch++)
            for (int c = 0; c < 3; c++) e[c] = cadd(e[c], part[(((long)b * S * S + pt) * nchunk + ch) * 3 + c]);
        const double k02 = m.k0 * m.k0;
        for (int c = 0; c < 3; c++) e[c] = zdiv(cscale(e[c], k02), den);
    }
    double2* o = Ed + (((long)b * S + jrow) * S + irow) * 3;
    for (int c = 0; c < 3; c++) o[c] = e[c];
}

// The lens (microsbf.f:699-795, microsdf.f:677-766): focus phase
// exp(i kz zlens) inside the pupil (kx^2 + ky^2 <= numaper^2), the specular
// incident wave added at its grid point, and the rotation of the field from
// the pupil to the image side with the magnification gross.
__global__ void __launch_bounds__(256) k_mic_lens(const MicGeom m, int nb, const double2* __restrict__ Ed,
                                                   const int* __restrict__ ik, const int* __restrict__ jk,
                                                   const double* __restrict__ pp, double2 E0,
                                                   double2* __restrict__ F) {
    const int S = m.S();
    const long total = (long)nb * S * S;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const int irow = (int)(t % S);
    const int jrow = (int)((t / S) % S);
    const int b = (int)(t / ((long)S * S));
    const int i = irow - m.imax, j = jrow - m.imax;
    const double kx = m.dkx * (double)i, ky = m.dky * (double)j;
    const double tmp = __dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky));
    double2 f[6];
    for (int c = 0; c < 6; c++) f[c] = make_double2(0, 0);
    if (tmp <= __dmul_rn(m.numaper, m.numaper)) {
        const double kz = sqrt(__dsub_rn(__dmul_rn(m.k0, m.k0), tmp));
        double sn, cs;
        sincos(kz * m.zlens, &sn, &cs);
        const double2 zf = make_double2(cs, sn);
        const double2* e = Ed + (((long)b * S + jrow) * S + irow) * 3;
        for (int c = 0; c < 3; c++) f[c] = cmul(e[c], zf);
        // the reflection side (microssansinc.f) forms no image with the
        // incident wave: those three fields stay zero
        if (m.dside > 0)
            for (int c = 0; c < 3; c++) f[c + 3] = f[c];
        if (m.dside > 0 && i == ik[b] && j == jk[b]) {
            double2 ex, ey, ez;
            double kzi;
            kxky_amplitude(m.k0, E0, pp[b], kx, ky, ex, ey, ez, kzi);
            if (m.ntypemic == 1) {
                // microsbf.f:733-741: x and y over dkx dky, z over dky alone,
                // as the reference writes it
                const double dkxy = m.dkx * m.dky;
                f[3] = cadd(f[3], cmul(make_double2(ex.x / dkxy, ex.y / dkxy), zf));
                f[4] = cadd(f[4], cmul(make_double2(ey.x / dkxy, ey.y / dkxy), zf));
                f[5] = cadd(f[5], cmul(make_double2(ez.x / m.dky, ez.y / m.dky), zf));
            } else {
                // microsdf.f:707-717: phase plate, i / (dkx dky)
                const double2 a[3] = {ex, ey, ez};
                for (int c = 0; c < 3; c++) {
                    const double2 v = cmul(make_double2(a[c].x / m.dkx / m.dky, a[c].y / m.dkx / m.dky), zf);
                    f[3 + c] = cadd(f[3 + c], make_double2(-v.y, v.x));
                }
            }
        }
        if (tmp != 0.0) {
            const double u0 = kx / m.k0, u1v = ky / m.k0;
            const double u2v = sqrt(__dsub_rn(__dsub_rn(1.0, __dmul_rn(u0, u0)), __dmul_rn(u1v, u1v))) * m.dside;
            const double v0 = -kx / m.k0 / m.gross, v1 = -ky / m.k0 / m.gross;
            const double v2 = sqrt(__dsub_rn(__dsub_rn(1.0, __dmul_rn(v0, v0)), __dmul_rn(v1, v1))) * m.dside;
            double a1 = __dsub_rn(__dmul_rn(u1v, v2), __dmul_rn(u2v, v1));
            double a2 = __dadd_rn(__dmul_rn(-u0, v2), __dmul_rn(u2v, v0));
            const double co = __dadd_rn(__dadd_rn(__dmul_rn(u0, v0), __dmul_rn(u1v, v1)), __dmul_rn(u2v, v2));
            const double si = sqrt(__dadd_rn(__dmul_rn(a1, a1), __dmul_rn(a2, a2)));
            a1 = a1 / si;
            a2 = a2 / si;
            const double tt = sqrt(u2v / v2);
            const double r00 = a1 * a1 + (1.0 - a1 * a1) * co, r01 = a1 * a2 * (1.0 - co), r02 = a2 * si;
            const double r11 = a2 * a2 + (1.0 - a2 * a2) * co, r12 = -a1 * si;
            const double r20 = -a2 * si, r21 = a1 * si;
            for (int h = 0; h < 6; h += 3) {
                const double2 X = f[h], Y = f[h + 1], Z = f[h + 2];
                const double2 tx = cadd(cadd(cscale(X, r00), cscale(Y, r01)), cscale(Z, r02));
                const double2 ty = cadd(cadd(cscale(X, r01), cscale(Y, r11)), cscale(Z, r12));
                const double2 tz = cadd(cadd(cscale(X, r20), cscale(Y, r21)), cscale(Z, co));
                f[h] = cscale(tx, tt);
                f[h + 1] = cscale(ty, tt);
                f[h + 2] = cscale(tz, tt);
            }
        }
    }
    for (int c = 0; c < 6; c++) F[((((long)b * 6 + c) * S) + jrow) * S + irow] = f[c];
}

template <int L> struct ImgTiles {
    static constexpr int NT = 256;
    // lines per block: about 4096 points of shared memory (64 KB), at most 32
    // lines, a power of two so that it divides every compiled L
    static constexpr int NB = clamp_pow2(4096 / L, 1, 32);
    static_assert(L % NB == 0, "column blocks must tile the image");
    static constexpr size_t smem = (size_t)(NB * L + L) * sizeof(double2);
};

// rows: line = (b 6 + c) S + jrow of the pupil field, transformed along x
struct RowSrc {
    static constexpr bool GLOBAL = true, HALF = false;
    const double2* F;
    int line0, nlines, S, imax, n;
    template <class C> __device__ C load(int b, int p) const {
        const int line = line0 + b, irow = pupil_row(p, imax, n);
        if (line >= nlines || irow < 0) return mk(0.0, 0.0);
        return F[(long)line * S + irow];
    }
};
struct RowDst {
    static constexpr bool GLOBAL = true, HALF = false;
    double2* T;
    int line0, nlines, n;
    template <class C> __device__ void store(int b, int o, C v) const {
        const int line = line0 + b;
        if (line < nlines) T[(long)line * n + o] = v;
    }
};

template <int L>
__global__ void __launch_bounds__(ImgTiles<L>::NT) k_mic_rows(const MicGeom m, int nlines,
                                                              const double2* __restrict__ F,
                                                              const double2* __restrict__ tw, double2* __restrict__ T) {
    using TT = ImgTiles<L>;
    extern __shared__ double2 sm[];
    double2* tws = sm + TT::NB * L;
    load_twiddles<double2, L, TT::NT>(tws, tw);
    const int line0 = blockIdx.x * TT::NB;
    const RowSrc src{F, line0, nlines, m.S(), m.imax, L};
    const RowDst dst{T, line0, nlines, L};
    fft_tile<double2, L, TT::NB, TT::NT, -1, Layout<1, L, false>, RowSrc, RowDst>(sm, tws, src, dst);
}

// columns x0 .. x0 + NB - 1 of one incidence's rows, transformed along y
struct ColSrc {
    static constexpr bool GLOBAL = true, HALF = false;
    const double2* T;  // rows of (b, c): S x n
    int x0, imax, n;
    template <class C> __device__ C load(int b, int p) const {
        const int jrow = pupil_row(p, imax, n);
        if (jrow < 0) return mk(0.0, 0.0);
        return T[(long)jrow * n + x0 + b];
    }
};

// img[c][v][u] += sum_b |dkx dky / gross E_b(slot (u - n/2, v - n/2))|^2
template <int L>
__global__ void __launch_bounds__(ImgTiles<L>::NT) k_mic_cols(const MicGeom m, int nb, const double2* __restrict__ T,
                                                              const double2* __restrict__ tw, double* __restrict__ img) {
    using TT = ImgTiles<L>;
    using Lay = Layout<TT::NB, 1, true>;
    constexpr int NB = TT::NB, NT = TT::NT, PER = (L * NB + NT - 1) / NT;
    extern __shared__ double2 sm[];
    double2* tws = sm + NB * L;
    load_twiddles<double2, L, NT>(tws, tw);
    const int x0 = blockIdx.x * NB, c = blockIdx.y, S = m.S();
    const double sc = m.dkx * m.dky / m.gross;
    double acc[PER];
#pragma unroll
    for (int q = 0; q < PER; q++) acc[q] = 0.0;
    for (int b = 0; b < nb; b++) {
        const ColSrc src{T + ((long)b * 6 + c) * S * L, x0, m.imax, L};
        fft_tile<double2, L, NB, NT, -1, Lay, ColSrc, SmemIO>(sm, tws, src);
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int idx = threadIdx.x + q * NT;
            if (PER * NT == L * NB || idx < L * NB) {
                const double2 v = sm[Lay::addr(idx / NB, idx % NB)];
                const double vx = v.x * sc, vy = v.y * sc;
                acc[q] += vx * vx + vy * vy;
            }
        }
        __syncthreads();  // the next transform overwrites the tile
    }
    const int n2 = L / 2;
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int idx = threadIdx.x + q * NT;
        if (PER * NT == L * NB || idx < L * NB) {
            const int u = (x0 + idx % NB + n2) % L, v = (idx / NB + n2) % L;
            double* o = img + ((long)c * L + v) * L + u;
            *o += acc[q];
        }
    }
}

// Holographic image: the complex field of one incidence, transformed along
// y, centred and scaled by dkx dky / gross (fouriertoimage.f:37-95),
// written to cimg[c][v][u]
template <int L>
__global__ void __launch_bounds__(ImgTiles<L>::NT) k_mic_cols_field(const MicGeom m, const double2* __restrict__ T,
                                                                    const double2* __restrict__ tw,
                                                                    double2* __restrict__ cimg) {
    using TT = ImgTiles<L>;
    using Lay = Layout<TT::NB, 1, true>;
    constexpr int NB = TT::NB, NT = TT::NT, PER = (L * NB + NT - 1) / NT;
    extern __shared__ double2 sm[];
    double2* tws = sm + NB * L;
    load_twiddles<double2, L, NT>(tws, tw);
    const int x0 = blockIdx.x * NB, c = blockIdx.y, S = m.S();
    const double sc = m.dkx * m.dky / m.gross;
    const ColSrc src{T + (long)c * S * L, x0, m.imax, L};
    fft_tile<double2, L, NB, NT, -1, Lay, ColSrc, SmemIO>(sm, tws, src);
    const int n2 = L / 2;
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int idx = threadIdx.x + q * NT;
        if (PER * NT == L * NB || idx < L * NB) {
            const double2 v = sm[Lay::addr(idx / NB, idx % NB)];
            const int u = (x0 + idx % NB + n2) % L, w = (idx / NB + n2) % L;
            cimg[((long)c * L + w) * L + u] = make_double2(v.x * sc, v.y * sc);
        }
    }
}

template <int L> void launch_image_field(const MicGeom& m, const double2* F, const double2* tw, double2* T,
                                         double2* cimg, cudaStream_t st) {
    using TT = ImgTiles<L>;
    IFDDA_CUDA(cudaFuncSetAttribute(k_mic_rows<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT::smem));
    IFDDA_CUDA(
        cudaFuncSetAttribute(k_mic_cols_field<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT::smem));
    const int nlines = 6 * m.S();
    count_launch();
    k_mic_rows<L><<<(nlines + TT::NB - 1) / TT::NB, TT::NT, TT::smem, st>>>(m, nlines, F, tw, T);
    IFDDA_CUDA(cudaGetLastError());
    count_launch();
    k_mic_cols_field<L><<<dim3(L / TT::NB, 6), TT::NT, TT::smem, st>>>(m, T, tw, cimg);
    IFDDA_CUDA(cudaGetLastError());
}

// The holographic microscope's lens (cdmlib.f:4380-4560): every pupil point
// with k0^2 - kx^2 - ky^2 >= 0 gets the focus phase; on the transmission side
// the field with the incident wave adds E_inc / dkx^2 at the grid point (ik,
// jk) (diffractefft2dinc.f:75-91); then the rotation by the lens, skipped
// where its axis vanishes (the centre).  four: the pupil fields before the
// rotation (6 x S x S); F: after it, as the image transform reads them.
// slow: the lens without FFT (cdmlib.f:3885-3960): only points inside the
// objective's aperture, and the field with the incident wave formed as
// E zf + E_inc zf.
__global__ void __launch_bounds__(256) k_mic_holo(const MicGeom m, const double2* __restrict__ Ed, int ik, int jk,
                                                   double pp, double2 E0, int slow, double2* __restrict__ F,
                                                   double2* __restrict__ four) {
    const int S = m.S();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= S * S) return;
    const int irow = t % S, jrow = t / S, i = irow - m.imax, j = jrow - m.imax;
    const double kx = m.dkx * (double)i, ky = m.dkx * (double)j;
    const double kz2 = __dsub_rn(__dsub_rn(__dmul_rn(m.k0, m.k0), __dmul_rn(kx, kx)), __dmul_rn(ky, ky));
    const bool in = slow ? sqrt(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky))) <= m.numaper : kz2 >= 0.0;
    double2 f[6], g[6];
    for (int c = 0; c < 6; c++) f[c] = g[c] = make_double2(0, 0);
    if (in) {
        const double kz = sqrt(kz2);
        double sn, cs;
        sincos(kz * m.zlens, &sn, &cs);
        const double2 zf = make_double2(cs, sn);
        const double2* e = Ed + ((long)jrow * S + irow) * 3;
        double2 inc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
        if (m.dside > 0 && i == ik && j == jk) {
            double2 ex, ey, ez;
            double kzi;
            kxky_amplitude(m.k0, E0, pp, kx, ky, ex, ey, ez, kzi);
            const double2 a[3] = {ex, ey, ez};
            for (int c = 0; c < 3; c++) inc[c] = make_double2(a[c].x / m.dkx / m.dkx, a[c].y / m.dkx / m.dkx);
        }
        for (int c = 0; c < 3; c++) {
            f[c] = cmul(e[c], zf);
            if (m.dside > 0) f[c + 3] = slow ? cadd(f[c], cmul(inc[c], zf)) : cmul(cadd(e[c], inc[c]), zf);
        }
        const double u0 = kx / m.k0, u1v = ky / m.k0;
        const double u2v = sqrt(__dsub_rn(__dsub_rn(1.0, __dmul_rn(u0, u0)), __dmul_rn(u1v, u1v))) * m.dside;
        const double v0 = -kx / m.k0 / m.gross, v1 = -ky / m.k0 / m.gross;
        const double v2 = sqrt(__dsub_rn(__dsub_rn(1.0, __dmul_rn(v0, v0)), __dmul_rn(v1, v1))) * m.dside;
        double a1 = __dsub_rn(__dmul_rn(u1v, v2), __dmul_rn(u2v, v1));
        double a2 = __dadd_rn(__dmul_rn(-u0, v2), __dmul_rn(u2v, v0));
        const double co = __dadd_rn(__dadd_rn(__dmul_rn(u0, v0), __dmul_rn(u1v, v1)), __dmul_rn(u2v, v2));
        const double si = sqrt(__dadd_rn(__dmul_rn(a1, a1), __dmul_rn(a2, a2)));
        if (si == 0.0) {
            for (int c = 0; c < 6; c++) g[c] = f[c];
        } else {
            a1 = a1 / si;
            a2 = a2 / si;
            const double tt = sqrt(u2v / v2);
            const double r00 = a1 * a1 + (1.0 - a1 * a1) * co, r01 = a1 * a2 * (1.0 - co), r02 = a2 * si;
            const double r11 = a2 * a2 + (1.0 - a2 * a2) * co, r12 = -a1 * si;
            const double r20 = -a2 * si, r21 = a1 * si;
            for (int h = 0; h < 6; h += 3) {
                const double2 X = f[h], Y = f[h + 1], Z = f[h + 2];
                g[h] = cscale(cadd(cadd(cscale(X, r00), cscale(Y, r01)), cscale(Z, r02)), tt);
                g[h + 1] = cscale(cadd(cadd(cscale(X, r01), cscale(Y, r11)), cscale(Z, r12)), tt);
                g[h + 2] = cscale(cadd(cadd(cscale(X, r20), cscale(Y, r21)), cscale(Z, co)), tt);
            }
        }
    }
    for (int c = 0; c < 6; c++) {
        four[((long)c * S + jrow) * S + irow] = f[c];
        F[((long)c * S + jrow) * S + irow] = g[c];
    }
}

__global__ void k_mic_sqrt(long cnt, double* __restrict__ img) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (long)gridDim.x * blockDim.x)
        img[i] = sqrt(img[i]);
}

template <int L> void launch_image(const MicGeom& m, int nb, const double2* F, const double2* tw, double2* T,
                                   double* img, cudaStream_t st) {
    using TT = ImgTiles<L>;
    IFDDA_CUDA(cudaFuncSetAttribute(k_mic_rows<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT::smem));
    IFDDA_CUDA(cudaFuncSetAttribute(k_mic_cols<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TT::smem));
    const int nlines = nb * 6 * m.S();
    count_launch();
    k_mic_rows<L><<<(nlines + TT::NB - 1) / TT::NB, TT::NT, TT::smem, st>>>(m, nlines, F, tw, T);
    IFDDA_CUDA(cudaGetLastError());
    count_launch();
    k_mic_cols<L><<<dim3(L / TT::NB, 6), TT::NT, TT::smem, st>>>(m, nb, T, tw, img);
    IFDDA_CUDA(cudaGetLastError());
}

}  // namespace

bool image_length_supported(int n) {
    switch (n) {
#define IFDDA_CASE_IMG(L) case L:
        IFDDA_IMG_LENGTHS(IFDDA_CASE_IMG)
#undef IFDDA_CASE_IMG
        return true;
        default:
            return false;
    }
}

void mic_farfield_dev(const MicGeom& m, int nb, const double2* FF, const double* zplane, const double2* tw,
                      double2* Q, double2* Ed, cudaStream_t st, bool both_sides) {
    const long nq = (long)nb * m.nz * m.ny * m.S(), ne = (long)nb * m.S() * m.S();
    count_launch();
    k_mic_xdft<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(m, nb, FF, tw, Q);
    IFDDA_CUDA(cudaGetLastError());
    count_launch();
    if (both_sides) k_mic_far2<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(m, nb, Q, zplane, tw, Ed);
    else k_mic_far<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(m, nb, Q, zplane, tw, Ed);
    IFDDA_CUDA(cudaGetLastError());
}

int mic_direct_chunks(long nd) { return (int)std::max(1L, std::min(64L, (nd + 4095) / 4096)); }

void mic_direct_dev(const MicGeom& m, int nb, int nd, const double* xs, const double* ys, const double* zs,
                    const double2* FF, double2* part, double2* Ed, cudaStream_t st) {
    const int S = m.S(), nchunk = mic_direct_chunks(nd);
    count_launch();
    k_mic_direct_part<<<dim3(S * S, nchunk, nb), MD_NT, 0, st>>>(m, nd, xs, ys, zs, FF, nchunk, part);
    IFDDA_CUDA(cudaGetLastError());
    const long ne = (long)nb * S * S;
    count_launch();
    k_mic_direct_final<<<(unsigned)((ne + 127) / 128), 128, 0, st>>>(m, nb, nchunk, part, Ed);
    IFDDA_CUDA(cudaGetLastError());
}

void mic_lens_dev(const MicGeom& m, int nb, const double2* Ed, const int* ik, const int* jk, const double* pp,
                  double2 E0, double2* F, cudaStream_t st) {
    const long ne = (long)nb * m.S() * m.S();
    count_launch();
    k_mic_lens<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(m, nb, Ed, ik, jk, pp, E0, F);
    IFDDA_CUDA(cudaGetLastError());
}

bool mic_image_dev(const MicGeom& m, int nb, const double2* F, const double2* tw, double2* T, double* img,
                   cudaStream_t st) {
    switch (m.n) {
#define IFDDA_CASE_IMG(L) \
    case L: launch_image<L>(m, nb, F, tw, T, img, st); return true;
        IFDDA_IMG_LENGTHS(IFDDA_CASE_IMG)
#undef IFDDA_CASE_IMG
        default:
            return false;
    }
}

bool mic_holo_dev(const MicGeom& m, const double2* Ed, int ik, int jk, double pp, double2 E0, bool slow,
                  double2* F, double2* four, const double2* tw, double2* T, double2* cimg, cudaStream_t st) {
    const int S = m.S();
    count_launch();
    k_mic_holo<<<(S * S + 255) / 256, 256, 0, st>>>(m, Ed, ik, jk, pp, E0, slow ? 1 : 0, F, four);
    IFDDA_CUDA(cudaGetLastError());
    switch (m.n) {
#define IFDDA_CASE_IMG(L) \
    case L: launch_image_field<L>(m, F, tw, T, cimg, st); return true;
        IFDDA_IMG_LENGTHS(IFDDA_CASE_IMG)
#undef IFDDA_CASE_IMG
        default:
            return false;
    }
}

void mic_sqrt_dev(long cnt, double* img, cudaStream_t st) {
    const int grid = (int)std::max(1L, std::min<long>((cnt + 255) / 256, 148L * 8));
    count_launch();
    k_mic_sqrt<<<grid, 256, 0, st>>>(cnt, img);
    IFDDA_CUDA(cudaGetLastError());
}

}  // namespace ifdda
