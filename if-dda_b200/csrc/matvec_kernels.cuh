// FFT mat-vec y = b - (1/M) F^-1[ G~ . F(pad(alpha x)) ]  on sm_100a.
//
// Replaces cdmlib/produitfftmatvectopt.f:3-121 (full box) and
// cdmlib/produitfftmatvect3.f:2-127 (Tabdip indirection), with the driver's
// `xi = polarisa . xr` step (cdmlib/inverserigopt.f:68-80) fused into the first
// pass.  The padded grid (X,Y,Z) = (2nx,2ny,2nz) is never materialised in full:
//
//   pass 1  fwd_x : read AoS x (3 per site) and alpha, FFT along x of the nx
//                   nonzeros padded to X              -> B1[r][c][k<nz][j<ny][X]
//   pass 2  fwd_y : FFT along y of the ny nonzeros     -> B2[r][c][k<nz][Y][X]
//   pass 3  zconv : FFT along z of the nz nonzeros, 3x3 symmetric multiply by
//                   the parity-compressed G~, inverse FFT along z, keep k<nz
//                                                     -> B2 (in place)
//   pass 4  inv_y : inverse FFT along y, keep j<ny     -> B1
//   pass 5  inv_x : inverse FFT along x, keep i<nx, y = b - v/M (AoS), with
//                   optional fused dot products for the Krylov scalars.
//
// The compressed spectrum: G(r) on the circulant grid is even (xx,yy,zz) or odd
// (xy in x,y; xz in x,z; yz in y,z) under q -> (L - q) mod L along each axis
// (zero planes at nx,ny,nz, cdmlib/calculgreenfft.f:29-35), so its DFT has the
// same parity and only q in [0, L/2] per axis is stored:
//   Gc[c6][qz][qy][qx], dims (nz+1, ny+1, nx+1), c6 = xx,xy,xz,yy,yz,zz.
#pragma once
#include "fft_tile.cuh"
#include "reduce.cuh"

namespace ifdda {

struct MvGeom {
    int nx, ny, nz;     // lattice
    int X, Y, Z;        // padded FFT grid
    long N;             // nx*ny*nz
    long b1_rhs;        // elements of B1 per right-hand side: 3*nz*ny*X
    long b2_rhs;        // elements of B2 per right-hand side: 3*nz*Y*X
    long gc_comp;       // elements of one compressed G~ component
};

// polarisability modes
enum { ALPHA_NONE = 0, ALPHA_ISO = 1, ALPHA_FULL = 2 };

template <class T> struct MvArgs {
    using C = cplx<T>;
    MvGeom g;
    const C* x;          // input vectors, AoS, per rhs stride xstride
    const C* b;          // subtrahend vectors (may alias y)
    C* y;                // output vectors
    long xstride;        // complex elements between right-hand sides
    int amode;
    const C* alpha;      // ISO: alpha[d]; FULL: alpha[d + nmax*(a + 3*b)]
    long nmax;
    const int* tabdip;   // lattice -> 1-based dipole (null: identity)
    C* B1;
    C* B2;
    const C* Gc;         // compressed spectrum
    const C* twx;
    const C* twy;
    const C* twz;
    const int* status;   // per rhs: nonzero -> skip (solve finished)
    T inv_m;             // 1 / (X Y Z)
};

template <class T, int L> struct MvTiles {
    static constexpr int S = (int)sizeof(cplx<T>);
    static constexpr int TLX = clamp_pow2(49152 / (L * 3 * S), 1, 16);
    static constexpr int TLY = clamp_pow2(49152 / (L * S), 2, 32);
    static constexpr int TLZ = clamp_pow2(98304 / (L * 3 * S), 1, 16);
    static constexpr int NT = 256;
    static constexpr int LSX = (3 * TLX) | 1;
    static constexpr size_t smem_x = (size_t)L * S + (size_t)L * LSX * S;
    static constexpr size_t smem_y = (size_t)L * S + (size_t)L * TLY * S;
    static constexpr size_t smem_z = (size_t)L * S + (size_t)L * 3 * TLZ * S;
};

template <class C> __device__ __forceinline__ C* smem_base() {
    extern __shared__ __align__(16) unsigned char ifdda_smem[];
    return reinterpret_cast<C*>(ifdda_smem);
}

template <class T>
__device__ __forceinline__ void apply_alpha(const MvArgs<T>& a, long d, cplx<T>& v0, cplx<T>& v1,
                                            cplx<T>& v2) {
    using C = cplx<T>;
    if (a.amode == ALPHA_ISO) {
        C al = a.alpha[d];
        v0 = cmul(al, v0);
        v1 = cmul(al, v1);
        v2 = cmul(al, v2);
    } else if (a.amode == ALPHA_FULL) {
        const long n = a.nmax;
        C w[3] = {v0, v1, v2};
        C o[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            C acc = czero<C>();
#pragma unroll
            for (int c = 0; c < 3; c++) acc = cadd(acc, cmul(a.alpha[d + n * (r + 3 * c)], w[c]));
            o[r] = acc;
        }
        v0 = o[0];
        v1 = o[1];
        v2 = o[2];
    }
}

// ---- pass 1 -------------------------------------------------------------
template <class T, int L, bool TAB>
__global__ void __launch_bounds__(MvTiles<T, L>::NT) k_fwd_x(const MvArgs<T> a) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLX, NB = 3 * TL, LS = TT::LSX, NT = TT::NT;
    const int rhs = blockIdx.z;
    if (a.status && a.status[rhs]) return;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int j0 = blockIdx.x * TL, k = blockIdx.y;
    const int nl = min(TL, ny - j0);
    load_twiddles<C, L, NT>(tw, a.twx);
    const long site0 = (long)k * nx * ny + (long)j0 * nx;
    const C* x = a.x + rhs * a.xstride;
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int jl = e / L, p = e - jl * L;
        C v0 = czero<C>(), v1 = v0, v2 = v0;
        if (jl < nl && p < nx) {
            const long site = site0 + (long)jl * nx + p;
            long d = site;
            bool occ = true;
            if (TAB) {
                const int t = a.tabdip[site];
                occ = t != 0;
                d = (long)t - 1;
            }
            if (occ) {
                v0 = x[3 * d];
                v1 = x[3 * d + 1];
                v2 = x[3 * d + 2];
                apply_alpha<T>(a, d, v0, v1, v2);
            }
        }
        sm[p * LS + jl] = v0;
        sm[p * LS + TL + jl] = v1;
        sm[p * LS + 2 * TL + jl] = v2;
    }
    __syncthreads();
    tile_fft<C, L, NB, LS, NT, +1>(sm, tw);
    C* B1 = a.B1 + rhs * a.g.b1_rhs;
    for (int e = threadIdx.x; e < NB * L; e += NT) {
        const int bl = e / L, p = e - bl * L;
        const int c = bl / TL, jl = bl - c * TL;
        if (jl < nl) B1[(((long)c * nz + k) * ny + j0 + jl) * L + p] = sm[p * LS + bl];
    }
}

// ---- pass 2 and 4 ---------------------------------------------------------
// DIR=+1: B1 (ny rows) -> B2 (Y rows);  DIR=-1: B2 (Y rows) -> B1 (ny rows)
template <class T, int L, int DIR>
__global__ void __launch_bounds__(MvTiles<T, L>::NT) k_pass_y(const MvArgs<T> a) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLY, NT = TT::NT;
    const int rhs = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3);
    if (a.status && a.status[rhs]) return;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int X = a.g.X, ny = a.g.ny, nz = a.g.nz;
    const int i0 = blockIdx.x * TL, k = blockIdx.y;
    load_twiddles<C, L, NT>(tw, a.twy);
    const int rows_in = DIR > 0 ? ny : L;
    const int rows_out = DIR > 0 ? L : ny;
    const C* src = DIR > 0 ? a.B1 + rhs * a.g.b1_rhs : a.B2 + rhs * a.g.b2_rhs;
    C* dst = DIR > 0 ? a.B2 + rhs * a.g.b2_rhs : a.B1 + rhs * a.g.b1_rhs;
    const long rin0 = ((long)c * nz + k) * rows_in;
    const long rout0 = ((long)c * nz + k) * rows_out;
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int p = e / TL, il = e - p * TL;
        const int i = i0 + il;
        C v = czero<C>();
        if (p < rows_in && i < X) v = src[(rin0 + p) * X + i];
        sm[e] = v;
    }
    __syncthreads();
    tile_fft<C, L, TL, TL, NT, DIR>(sm, tw);
    for (int e = threadIdx.x; e < TL * rows_out; e += NT) {
        const int p = e / TL, il = e - p * TL;
        const int i = i0 + il;
        if (i < X) dst[(rout0 + p) * X + i] = sm[e];
    }
}

// ---- pass 3 -----------------------------------------------------------------
template <class T, int L>
__global__ void __launch_bounds__(MvTiles<T, L>::NT) k_zconv(const MvArgs<T> a) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLZ, NB = 3 * TL, NT = TT::NT;
    const int rhs = blockIdx.z;
    if (a.status && a.status[rhs]) return;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz, X = a.g.X, Y = a.g.Y;
    const int i0 = blockIdx.x * TL;
    const int qy = blockIdx.y;
    load_twiddles<C, L, NT>(tw, a.twz);
    C* B2 = a.B2 + rhs * a.g.b2_rhs;
    for (int e = threadIdx.x; e < NB * L; e += NT) {
        const int p = e / NB, bl = e - p * NB;
        const int c = bl / TL, il = bl - c * TL;
        const int i = i0 + il;
        C v = czero<C>();
        if (p < nz && i < X) v = B2[(((long)c * nz + p) * Y + qy) * X + i];
        sm[e] = v;
    }
    __syncthreads();
    tile_fft<C, L, NB, NB, NT, +1>(sm, tw);
    // 3x3 symmetric multiply with the compressed spectrum
    const int qyc = qy <= ny ? qy : Y - qy;
    const T sy = qy <= ny ? (T)1 : (T)-1;
    const long gcs = a.g.gc_comp;
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int p = e / TL, il = e - p * TL;
        const int i = i0 + il;
        if (i >= X) continue;
        const int qxc = i <= nx ? i : X - i;
        const T sx = i <= nx ? (T)1 : (T)-1;
        const int qzc = p <= nz ? p : L - p;
        const T sz = p <= nz ? (T)1 : (T)-1;
        const long gi = ((long)qzc * (ny + 1) + qyc) * (nx + 1) + qxc;
        const C gxx = a.Gc[gi];
        const C gxy = cscale(a.Gc[gcs + gi], sx * sy);
        const C gxz = cscale(a.Gc[2 * gcs + gi], sx * sz);
        const C gyy = a.Gc[3 * gcs + gi];
        const C gyz = cscale(a.Gc[4 * gcs + gi], sy * sz);
        const C gzz = a.Gc[5 * gcs + gi];
        C* row = sm + p * NB + il;
        const C vx = row[0], vy = row[TL], vz = row[2 * TL];
        row[0] = cadd(cadd(cmul(gxx, vx), cmul(gxy, vy)), cmul(gxz, vz));
        row[TL] = cadd(cadd(cmul(gxy, vx), cmul(gyy, vy)), cmul(gyz, vz));
        row[2 * TL] = cadd(cadd(cmul(gxz, vx), cmul(gyz, vy)), cmul(gzz, vz));
    }
    __syncthreads();
    tile_fft<C, L, NB, NB, NT, -1>(sm, tw);
    for (int e = threadIdx.x; e < NB * nz; e += NT) {
        const int p = e / NB, bl = e - p * NB;
        const int c = bl / TL, il = bl - c * TL;
        const int i = i0 + il;
        if (i < X) B2[(((long)c * nz + p) * Y + qy) * X + i] = sm[e];
    }
}

// ---- pass 5 -----------------------------------------------------------------
// Epi: epilogue policy with up to Epi::NDOT fused dot products
//   sum_site conj(U) V, U and V chosen per dot among {y (the result), ext[k]}.
template <class T, int L, bool TAB, class Epi>
__global__ void __launch_bounds__(MvTiles<T, L>::NT) k_inv_x(const MvArgs<T> a, const Epi epi) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLX, NB = 3 * TL, LS = TT::LSX, NT = TT::NT;
    const int rhs = blockIdx.z;
    const bool skip = a.status && a.status[rhs];
    double2 acc[Epi::NDOT > 0 ? Epi::NDOT : 1];
#pragma unroll
    for (int q = 0; q < (Epi::NDOT > 0 ? Epi::NDOT : 1); q++) acc[q] = make_double2(0, 0);
    if (!skip) {
        C* tw = smem_base<C>();
        C* sm = tw + L;
        const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
        const int j0 = blockIdx.x * TL, k = blockIdx.y;
        const int nl = min(TL, ny - j0);
        load_twiddles<C, L, NT>(tw, a.twx);
        const C* B1 = a.B1 + rhs * a.g.b1_rhs;
        for (int e = threadIdx.x; e < NB * L; e += NT) {
            const int bl = e / L, p = e - bl * L;
            const int c = bl / TL, jl = bl - c * TL;
            C v = czero<C>();
            if (jl < nl) v = B1[(((long)c * nz + k) * ny + j0 + jl) * L + p];
            sm[p * LS + bl] = v;
        }
        __syncthreads();
        tile_fft<C, L, NB, LS, NT, -1>(sm, tw);
        const long site0 = (long)k * nx * ny + (long)j0 * nx;
        const C* bv = a.b + rhs * a.xstride;
        C* yv = a.y + rhs * a.xstride;
        for (int s = threadIdx.x; s < nl * nx; s += NT) {
            const int jl = s / nx, p = s - jl * nx;
            const long site = site0 + s;
            long d = site;
            if (TAB) {
                const int t = a.tabdip[site];
                if (t == 0) continue;
                d = (long)t - 1;
            }
            C o[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const C v = sm[p * LS + c * TL + jl];
                o[c] = csub(bv[3 * d + c], cscale(v, a.inv_m));
                yv[3 * d + c] = o[c];
            }
            epi.template accumulate<C>(rhs, 3 * d, o, acc);
        }
    }
    if constexpr (Epi::NDOT > 0) epi.finish(rhs, acc, skip);
}

struct EpiNone {
    static constexpr int NDOT = 0;
    template <class C> __device__ __forceinline__ void accumulate(int, long, const C*, double2*) const {}
    __device__ __forceinline__ void finish(int, double2*, bool) const {}
};

}  // namespace ifdda
