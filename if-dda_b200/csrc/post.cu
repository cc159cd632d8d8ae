// Post-step and incident-field kernels.
//   local_macro  : cdmlib/local-macro.f:3-71 over every dipole (cdmlib/cdmlib.f:2595-2655)
//   cross sections: cdmlib/cdmlib.f:2730-2746
//   plane waves  : cdmlib/ondeplane.f:1-50, cdmlib/ondeplanekxky.f:1-60
#include "post.cuh"
#include "krylov_kernels.cuh"
#include "planewave.cuh"

namespace ifdda {

// closed-form 3x3 complex inverse by cofactors; returns false when singular
__device__ __forceinline__ bool inv33(const double2 (&m)[9], double2 (&o)[9]) {
#define A(i, j) m[(i) + 3 * (j)]
    const double2 c00 = zsub(zmul(A(1, 1), A(2, 2)), zmul(A(1, 2), A(2, 1)));
    const double2 c01 = zsub(zmul(A(1, 2), A(2, 0)), zmul(A(1, 0), A(2, 2)));
    const double2 c02 = zsub(zmul(A(1, 0), A(2, 1)), zmul(A(1, 1), A(2, 0)));
    const double2 det = zadd(zadd(zmul(A(0, 0), c00), zmul(A(0, 1), c01)), zmul(A(0, 2), c02));
    if (zisnull(det)) return false;
    const double2 cof[9] = {
        c00,
        c01,
        c02,
        zsub(zmul(A(0, 2), A(2, 1)), zmul(A(0, 1), A(2, 2))),
        zsub(zmul(A(0, 0), A(2, 2)), zmul(A(0, 2), A(2, 0))),
        zsub(zmul(A(0, 1), A(2, 0)), zmul(A(0, 0), A(2, 1))),
        zsub(zmul(A(0, 1), A(1, 2)), zmul(A(0, 2), A(1, 1))),
        zsub(zmul(A(0, 2), A(1, 0)), zmul(A(0, 0), A(1, 2))),
        zsub(zmul(A(0, 0), A(1, 1)), zmul(A(0, 1), A(1, 0))),
    };
#undef A
    // cof[] is listed column by column of the inverse: (0,0),(1,0),(2,0),(0,1),...
    for (int q = 0; q < 9; q++) o[q] = zdiv(cof[q], det);
    return true;
}

__global__ void k_local_macro(int nb, long nmax, const double2* __restrict__ eps, const double2* __restrict__ loc,
                              double cst, double2* __restrict__ em, int* __restrict__ bad) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (long)gridDim.x * blockDim.x) {
        double2 m[9], mi[9];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                const double2 e = eps[i + nmax * (a + 3 * b)];
                const double d0 = a == b ? 2.0 : 0.0, d1 = a == b ? 1.0 : 0.0;
                // eps + 2I - i cst (eps - I)
                const double2 m1 = make_double2(e.x - d1, e.y);
                m[a + 3 * b] = make_double2(e.x + d0 + cst * m1.y, e.y - cst * m1.x);
            }
        if (!inv33(m, mi)) {
            atomicOr(bad, 1);
            continue;
        }
        for (int a = 0; a < 3; a++) {
            double2 acc = make_double2(0, 0);
            for (int b = 0; b < 3; b++) acc = zadd(acc, zmul(mi[a + 3 * b], loc[3 * i + b]));
            em[3 * i + a] = make_double2(3.0 * acc.x, 3.0 * acc.y);
        }
    }
}

struct CrossOp {
    const double2* ff0;
    const double2* ff;
    const double2* loc;
    double k03;
    KState* stt;
    __device__ void elem(const KState&, int, long i, double2* acc) const {
        // i runs over 3*nb components
        const double2 e0 = ff0[i], p = ff[i], l = loc[i];
        acc[0].x += zconjmul(e0, p).y;                              // Im(conj(E0) p)
        acc[1].x += zmul(p, zconj(l)).y - 2.0 / 3.0 * k03 * (p.x * p.x + p.y * p.y);
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.alpha = a[0];
        s.beta = a[1];
    }
};

void local_macro_dev(int nb, long nmax, const double2* eps, const double2* loc, double d, double k0, double2* em,
                     int* bad_dev, cudaStream_t st) {
    const double pi = 3.14159265358979323846;
    const double cst = k0 * k0 * k0 * d * d * d / 2.0 / pi;
    const int grid = (int)std::max(1L, std::min<long>((nb + 255) / 256, 148L * 8));
    count_launch();
    k_local_macro<<<grid, 256, 0, st>>>(nb, nmax, eps, loc, cst, em, bad_dev);
    IFDDA_CUDA(cudaGetLastError());
}

void cross_sections_dev(int nb, const double2* ff0, const double2* ff, const double2* loc, double k0,
                        double2* partials, unsigned* tickets, KState* stt, int* zstatus, cudaStream_t st) {
    const long n3 = 3L * nb;
    const int nblk = reduction_blocks(n3);
    RedSlots rs{partials, tickets, nblk};
    count_launch();
    k_vec<2, CrossOp><<<dim3(nblk, 1), KNT, 0, st>>>(CrossOp{ff0, ff, loc, k0 * k0 * k0, stt}, n3, nblk, rs, zstatus);
    IFDDA_CUDA(cudaGetLastError());
}

// one incidence per blockIdx.y; beam 0 ondeplane(theta, phi [deg]); 1 ondeplanekxky(kx, ky)
__global__ void k_planewaves(int nb, const double* __restrict__ xs, const double* __restrict__ ys,
                             const double* __restrict__ zs, double k0, double2 E0, const int* __restrict__ beam,
                             const double* __restrict__ a1, const double* __restrict__ a2,
                             const double* __restrict__ pp, double2* __restrict__ out, int* __restrict__ bad) {
    const int r = blockIdx.y;
    const double ppr = pp[r];
    if (ppr < 0.0 || ppr > 1.0) {
        if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(bad, 1);
        return;
    }
    const double p = sqrt(ppr), s = sqrt(1.0 - ppr);
    double kx, ky, kz;
    double2 ex, ey, ez;
    if (beam[r] == 0) {
        const double pi = 3.14159265358979323846;
        const double th = a1[r] * pi / 180.0, ph = a2[r] * pi / 180.0;
        const double sg = copysign(1.0, th);
        const double2 E0s = make_double2(E0.x * s * sg, E0.y * s * sg), E0p = make_double2(E0.x * p * sg, E0.y * p * sg);
        kx = k0 * sin(th) * cos(ph);
        ky = k0 * sin(th) * sin(ph);
        kz = k0 * cos(th);
        ey = make_double2(E0s.x * cos(ph) + E0p.x * cos(th) * sin(ph), E0s.y * cos(ph) + E0p.y * cos(th) * sin(ph));
        ex = make_double2(-E0s.x * sin(ph) + E0p.x * cos(th) * cos(ph), -E0s.y * sin(ph) + E0p.y * cos(th) * cos(ph));
        ez = make_double2(-E0p.x * sin(th), -E0p.y * sin(th));
    } else {
        kx = a1[r];
        ky = a2[r];
        kxky_amplitude(k0, E0, ppr, kx, ky, ex, ey, ez, kz);
    }
    double2* o = out + (long)r * 3 * nb;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (long)gridDim.x * blockDim.x) {
        double sn, cs;
        sincos(xs[i] * kx + ys[i] * ky + zs[i] * kz, &sn, &cs);
        const double2 e = make_double2(cs, sn);
        o[3 * i] = zmul(ex, e);
        o[3 * i + 1] = zmul(ey, e);
        o[3 * i + 2] = zmul(ez, e);
    }
}

void planewaves_dev(int nb, const double* xs, const double* ys, const double* zs, double k0, double2 E0, int nrhs,
                    const int* beam, const double* a1, const double* a2, const double* pp, double2* out, int* bad,
                    cudaStream_t st) {
    const int gx = (int)std::max(1L, std::min<long>((nb + 255) / 256, 148L * 4));
    count_launch();
    k_planewaves<<<dim3(gx, nrhs), 256, 0, st>>>(nb, xs, ys, zs, k0, E0, beam, a1, a2, pp, out, bad);
    IFDDA_CUDA(cudaGetLastError());
}

// Far field by direct summation (cdmlib.f:2803-2836): for direction n(theta,
// phi) of the (ntheta+1) x nphi grid, E = sum_i exp(-i k0 n.r_i)(p_i -
// n (n.p_i)).  Stage 1: block (direction, chunk) sums its dipoles; stage 2:
// one thread per direction adds the chunks in order and returns |E|^2.
constexpr int FF_NT = 256;
__global__ void __launch_bounds__(FF_NT) k_farfield_part(int nb, const double* __restrict__ xs,
                                                         const double* __restrict__ ys, const double* __restrict__ zs,
                                                         const double2* __restrict__ ff, double k0, int ntheta,
                                                         int nphi, int nchunk, double2* __restrict__ part) {
    const int dir = blockIdx.x, ch = blockIdx.y;
    const double pi = 3.14159265358979323846;
    const int itheta = dir / nphi, iphi = dir % nphi;
    const double th = pi / (double)ntheta * (double)itheta, ph = 2.0 * pi / (double)nphi * (double)iphi;
    const double n0 = sin(th) * cos(ph), n1 = sin(th) * sin(ph), n2 = cos(th);
    const long per = ((long)nb + nchunk - 1) / nchunk;
    const long i0 = (long)ch * per, i1 = min((long)nb, i0 + per);
    double2 acc[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (long i = i0 + threadIdx.x; i < i1; i += FF_NT) {
        double sn, cs;
        sincos(-k0 * (n0 * xs[i] + n1 * ys[i] + n2 * zs[i]), &sn, &cs);
        const double2 e = make_double2(cs, sn);
        const double2 p0 = ff[3 * i], p1 = ff[3 * i + 1], p2 = ff[3 * i + 2];
        const double2 np = make_double2(n0 * p0.x + n1 * p1.x + n2 * p2.x, n0 * p0.y + n1 * p1.y + n2 * p2.y);
        acc[0] = zadd(acc[0], zmul(e, make_double2(p0.x - np.x * n0, p0.y - np.y * n0)));
        acc[1] = zadd(acc[1], zmul(e, make_double2(p1.x - np.x * n1, p1.y - np.y * n1)));
        acc[2] = zadd(acc[2], zmul(e, make_double2(p2.x - np.x * n2, p2.y - np.y * n2)));
    }
    __shared__ double2 scratch[3 * 32];
    block_sum<FF_NT, 3>(acc, scratch);
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; c++) part[((long)dir * nchunk + ch) * 3 + c] = acc[c];
}

__global__ void k_farfield_final(int ndir, int nchunk, const double2* __restrict__ part, double* __restrict__ emod) {
    const int dir = blockIdx.x * blockDim.x + threadIdx.x;
    if (dir >= ndir) return;
    double2 e[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int ch = 0; ch < nchunk; ch++)
        for (int c = 0; c < 3; c++) e[c] = zadd(e[c], part[((long)dir * nchunk + ch) * 3 + c]);
    emod[dir] = (e[0].x * e[0].x + e[0].y * e[0].y) + (e[1].x * e[1].x + e[1].y * e[1].y) +
                (e[2].x * e[2].x + e[2].y * e[2].y);
}

int farfield_chunks(long nb) { return (int)std::max(1L, std::min(256L, (nb + 4095) / 4096)); }

void farfield_dev(int nb, const double* xs, const double* ys, const double* zs, const double2* ff, double k0,
                  int ntheta, int nphi, double2* part, double* emod, cudaStream_t st) {
    const int ndir = (ntheta + 1) * nphi, nchunk = farfield_chunks(nb);
    count_launch();
    k_farfield_part<<<dim3(ndir, nchunk), FF_NT, 0, st>>>(nb, xs, ys, zs, ff, k0, ntheta, nphi, nchunk, part);
    IFDDA_CUDA(cudaGetLastError());
    count_launch();
    k_farfield_final<<<(ndir + 127) / 128, 128, 0, st>>>(ndir, nchunk, part, emod);
    IFDDA_CUDA(cudaGetLastError());
}

// Sites of the enlarged box of the wide near field (cdmlib.f:2142-2216):
// site s holding object dipole l = map[s] takes its incident field, -FF as
// the source of the mat-vec and its permittivity; the other sites keep the
// incident wave already in xr, no source and the identity.
__global__ void k_wide_fill(long nw, const int* __restrict__ map, const double2* __restrict__ ff,
                            const double2* __restrict__ ff0, const double2* __restrict__ eps, long nmax,
                            double2* __restrict__ xr, double2* __restrict__ xi, double2* __restrict__ epsw) {
    for (long s = (long)blockIdx.x * blockDim.x + threadIdx.x; s < nw; s += (long)gridDim.x * blockDim.x) {
        const int l = map[s];
        for (int a = 0; a < 3; a++) {
            if (l >= 0) {
                xr[3 * s + a] = ff0[3L * l + a];
                xi[3 * s + a] = make_double2(-ff[3L * l + a].x, -ff[3L * l + a].y);
            } else {
                xi[3 * s + a] = make_double2(0, 0);
            }
            for (int b = 0; b < 3; b++)
                epsw[s + nw * (a + 3 * b)] = l >= 0 ? eps[l + nmax * (a + 3 * b)] : make_double2(a == b ? 1.0 : 0.0, 0.0);
        }
    }
}

void wide_fill_dev(long nw, const int* map, const double2* ff, const double2* ff0, const double2* eps, long nmax,
                   double2* xr, double2* xi, double2* epsw, cudaStream_t st) {
    const int grid = (int)std::max(1L, std::min<long>((nw + 255) / 256, 148L * 8));
    count_launch();
    k_wide_fill<<<grid, 256, 0, st>>>(nw, map, ff, ff0, eps, nmax, xr, xi, epsw);
    IFDDA_CUDA(cudaGetLastError());
}

// Compacts an isotropic (nmax,3,3) polarisability to one value per dipole;
// sets *aniso when any tensor is not a multiple of the identity.
__global__ void k_pola_compact(const double2* __restrict__ pol, long nb, long nmax, double2* __restrict__ alpha,
                               int* __restrict__ aniso) {
    int bad = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (long)gridDim.x * blockDim.x) {
        const double2 d0 = pol[i];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                const double2 v = pol[i + nmax * (a + 3 * b)];
                if (a == b) bad |= (v.x != d0.x || v.y != d0.y);
                else bad |= (v.x != 0.0 || v.y != 0.0);
            }
        alpha[i] = d0;
    }
    if (bad) atomicOr(aniso, 1);
}

void pola_compact_dev(const double2* pol, long nb, long nmax, double2* alpha, int* aniso, cudaStream_t st) {
    const int grid = (int)std::max(1L, std::min<long>((nb + 255) / 256, 148L * 8));
    count_launch();
    k_pola_compact<<<grid, 256, 0, st>>>(pol, nb, nmax, alpha, aniso);
    IFDDA_CUDA(cudaGetLastError());
}

}  // namespace ifdda
