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
//   pass 5  inv_x : inverse FFT along x, keep i<nx, y = b - v/M (AoS)
//
// Every pass loads its lines straight into the registers of the first FFT
// pass (the zero half of the padding is never read) and stores from the
// registers of the last one (the cropped half is never written); shared memory
// holds the tile between the inner FFT passes only.
//
// The compressed spectrum: G(r) on the circulant grid is even (xx,yy,zz) or odd
// (xy in x,y; xz in x,z; yz in y,z) under q -> (L - q) mod L along each axis
// (zero planes at nx,ny,nz, cdmlib/calculgreenfft.f:29-35), so its DFT has the
// same parity and only q in [0, L/2] per axis is stored:
//   Gc[c6][qz][qy][qx], dims (nz+1, ny+1, nx+1), c6 = xx,xy,xz,yy,yz,zz.
// zconv treats the mirror rows qy and Y-qy in one block, so each compressed
// value read serves both.
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

// Tile shapes: lines per block and threads per block for each pass.
template <class T, int L> struct MvTiles {
    static constexpr int S = (int)sizeof(cplx<T>);
    static constexpr int SMEM_X = 16384, SMEM_Y = 16384, SMEM_Z = 24576 * (S / 8);
    static constexpr int TLX = clamp_pow2(SMEM_X / (3 * (L + 1) * S), 1, 16);
    static constexpr int TLY = clamp_pow2(SMEM_Y / (L * S), 32 / S > 2 ? 32 / S : 2, 32);
    static constexpr int TLZ = clamp_pow2(SMEM_Z / (6 * L * S), 32 / S > 2 ? 32 / S : 2, 16);
    static constexpr int NBX = 3 * TLX, NBY = TLY, NBZ = 6 * TLZ;
    static constexpr int LP = L + 1;  // padded line stride of the x-pass tile
    static constexpr int PSY = NBY + 1, PSZ = NBZ + 1;  // padded point strides (odd) of the y and z tiles
    // one butterfly of the widest radix per thread
    static constexpr int nthreads(int nb) {
        int t = nb * L / max_radix(L);
        t = (t + 31) / 32 * 32;
        return t < 64 ? 64 : (t > 256 ? 256 : t);
    }
    static constexpr int NTX = nthreads(NBX), NTY = nthreads(NBY), NTZ = nthreads(NBZ);
    static constexpr size_t smem_x = (size_t)L * S + (size_t)NBX * LP * S;
    static constexpr size_t smem_y = (size_t)L * S + (size_t)L * PSY * S;
    // twiddles, the data tile, then the compressed spectrum of the block:
    // 6 components x (L/2 + 1) z planes x TLZ columns
    static constexpr size_t smem_z = (size_t)L * S + (size_t)L * PSZ * S + (size_t)6 * (L / 2 + 1) * TLZ * S;
};

// asynchronous global -> shared copy of one complex element (8 or 16 bytes)
template <class C> __device__ __forceinline__ void cp_async_elem(C* dst_smem, const C* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"((int)sizeof(C)));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <class C> __device__ __forceinline__ C* smem_base() {
    extern __shared__ __align__(16) unsigned char ifdda_smem[];
    return reinterpret_cast<C*>(ifdda_smem);
}

// ---- pass 1 ---------------------------------------------------------------
template <class T, bool TAB> struct FwdXLoad {
    static constexpr bool GLOBAL = true, HALF = true;  // points p >= nx are the padding
    const MvArgs<T>* a;
    const cplx<T>* x;
    long site0;
    int nl, tl;
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const int c = b / tl, jl = b - c * tl;
        if (jl >= nl) return czero<C>();
        const long site = site0 + (long)jl * a->g.nx + p;
        long d = site;
        if (TAB) {
            const int t = a->tabdip[site];
            if (t == 0) return czero<C>();
            d = (long)t - 1;
        }
        if (a->amode == ALPHA_ISO) return cmul(a->alpha[d], x[3 * d + c]);
        if (a->amode == ALPHA_FULL) {
            C acc = czero<C>();
#pragma unroll
            for (int q = 0; q < 3; q++) acc = cadd(acc, cmul(a->alpha[d + a->nmax * (c + 3 * q)], x[3 * d + q]));
            return acc;
        }
        return x[3 * d + c];
    }
};

// B1 rows of one x-pass tile: line b = c * TL + jl is row ((c * nz + k) * ny + j0 + jl)
template <class T, int L, int TL> struct B1RowIO {
    static constexpr bool GLOBAL = true, HALF = false;
    cplx<T>* B1;
    int nl, nz, ny, k, j0;
    template <class C> __device__ __forceinline__ long at(int b, int p) const {
        const int c = b / TL, jl = b - c * TL;
        return jl < nl ? (((long)c * nz + k) * ny + j0 + jl) * L + p : -1;
    }
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const long o = at<C>(b, p);
        if (o >= 0) B1[o] = v;
    }
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const long o = at<C>(b, p);
        return o >= 0 ? B1[o] : czero<C>();
    }
};

template <class T, int L, bool TAB>
__global__ void __launch_bounds__(MvTiles<T, L>::NTX) k_fwd_x(const MvArgs<T> a) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLX, NB = TT::NBX, NT = TT::NTX;
    const int rhs = blockIdx.z;
    if (a.status && a.status[rhs]) return;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int j0 = blockIdx.x * TL, k = blockIdx.y;
    const int nl = min(TL, ny - j0);
    load_twiddles<C, L, NT>(tw, a.twx);
    FwdXLoad<T, TAB> src{&a, a.x + rhs * a.xstride, (long)k * nx * ny + (long)j0 * nx, nl, TL};
    B1RowIO<T, L, TL> dst{a.B1 + rhs * a.g.b1_rhs, nl, nz, ny, k, j0};
    fft_tile<C, L, NB, NT, +1, Layout<1, TT::LP, false>>(sm, tw, src, dst);
}

// ---- pass 2 and 4 ---------------------------------------------------------
// DIR=+1: B1 (ny rows) -> B2 (Y rows);  DIR=-1: B2 (Y rows) -> B1 (ny rows)
template <class T, int DIR> struct YLoad {
    static constexpr bool GLOBAL = true, HALF = DIR > 0;  // forward: rows >= ny are padding
    const cplx<T>* src;
    int X, i0;
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const int i = i0 + b;
        return i < X ? src[(long)p * X + i] : czero<C>();
    }
};
template <class T, int DIR> struct YStore {
    static constexpr bool GLOBAL = true, HALF = DIR < 0;  // inverse: keep rows < ny
    cplx<T>* dst;
    int X, i0;
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const int i = i0 + b;
        if (i < X) dst[(long)p * X + i] = v;
    }
};

template <class T, int L, int DIR>
__global__ void __launch_bounds__(MvTiles<T, L>::NTY) k_pass_y(const MvArgs<T> a) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLY, NT = TT::NTY;
    const int rhs = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3);
    if (a.status && a.status[rhs]) return;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int X = a.g.X, ny = a.g.ny, nz = a.g.nz;
    const int i0 = blockIdx.x * TL, k = blockIdx.y;
    load_twiddles<C, L, NT>(tw, a.twy);
    const int rows_in = DIR > 0 ? ny : L;
    const int rows_out = DIR > 0 ? L : ny;
    const C* srcb = DIR > 0 ? a.B1 + rhs * a.g.b1_rhs : a.B2 + rhs * a.g.b2_rhs;
    C* dstb = DIR > 0 ? a.B2 + rhs * a.g.b2_rhs : a.B1 + rhs * a.g.b1_rhs;
    YLoad<T, DIR> src{srcb + ((long)c * nz + k) * rows_in * X, X, i0};
    YStore<T, DIR> dst{dstb + ((long)c * nz + k) * rows_out * X, X, i0};
    fft_tile<C, L, TL, NT, DIR, Layout<TT::PSY, 1, true>>(sm, tw, src, dst);
}

// ---- pass 3 -----------------------------------------------------------------
// lines b = (h * 3 + c) * TL + il: h = 0 row qy, h = 1 the mirror row Y - qy
template <class T> struct ZLoad {
    static constexpr bool GLOBAL = true, HALF = true;  // rows >= nz are padding
    const cplx<T>* B2;
    long rs;  // elements between z rows (Y * X)
    long comp;  // elements between components (nz * Y * X)
    long row0, row1;
    int X, i0, tl, two;
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const int hc = b / tl, il = b - hc * tl;
        const int h = hc / 3, c = hc - 3 * h;
        const int i = i0 + il;
        if (i >= X || h >= two) return czero<C>();
        return B2[c * comp + (long)p * rs + (h ? row1 : row0) + i];
    }
};
template <class T> struct ZStore {
    static constexpr bool GLOBAL = true, HALF = true;  // keep z rows < nz
    cplx<T>* B2;
    long rs, comp, row0, row1;
    int X, i0, tl, two;
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const int hc = b / tl, il = b - hc * tl;
        const int h = hc / 3, c = hc - 3 * h;
        const int i = i0 + il;
        if (i < X && h < two) B2[c * comp + (long)p * rs + (h ? row1 : row0) + i] = v;
    }
};

template <class T, int L>
__global__ void __launch_bounds__(MvTiles<T, L>::NTZ) k_zconv(const MvArgs<T> a) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLZ, NB = TT::NBZ, NT = TT::NTZ;
    const int rhs = blockIdx.z;
    if (a.status && a.status[rhs]) return;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz, X = a.g.X, Y = a.g.Y;
    const int i0 = blockIdx.x * TL;
    const int qy = blockIdx.y;                       // 0 .. ny
    const int two = (qy > 0 && qy < ny) ? 2 : 1;     // rows qy and Y - qy
    load_twiddles<C, L, NT>(tw, a.twz);
    // start copying this block's slice of the compressed spectrum (qy fixed,
    // every qz, the TL columns qx(i)) into shared memory; it lands while the
    // forward z transform runs
    constexpr int PS = TT::PSZ;
    C* gs = sm + L * PS;
    constexpr int NQ = L / 2 + 1;
    const long gcs = a.g.gc_comp;
    for (int e = threadIdx.x; e < 6 * NQ * TL; e += NT) {
        const int il = e % TL, cq = e / TL;
        const int c6 = cq / NQ, qz = cq - c6 * NQ;
        const int i = min(i0 + il, X - 1);
        const int qxc = i <= nx ? i : X - i;
        const C* src = a.Gc + c6 * gcs + ((long)qz * (ny + 1) + qy) * (nx + 1) + qxc;
        cp_async_elem(gs + e, src);
    }
    cp_async_commit();
    C* B2 = a.B2 + rhs * a.g.b2_rhs;
    const long rs = (long)Y * X, comp = (long)nz * Y * X;
    const long row0 = (long)qy * X, row1 = (long)(Y - qy) * X;
    fft_tile<C, L, NB, NT, +1, Layout<PS, 1, true>>(sm, tw, ZLoad<T>{B2, rs, comp, row0, row1, X, i0, TL, two},
                                                    SmemIO{});
    cp_async_wait_all();
    __syncthreads();
    // 3x3 symmetric multiply with the compressed spectrum; the mirror row
    // uses the same values with the sign of the y-odd components flipped
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int p = e / TL, il = e - p * TL;
        const int i = i0 + il;
        if (i >= X) continue;
        const T sx = i <= nx ? (T)1 : (T)-1;
        const int qzc = p <= nz ? p : L - p;
        const T sz = p <= nz ? (T)1 : (T)-1;
        const C* gq = gs + qzc * TL + il;
        const C gxx = gq[0];
        const C gxy = cscale(gq[NQ * TL], sx);
        const C gxz = cscale(gq[2 * NQ * TL], sx * sz);
        const C gyy = gq[3 * NQ * TL];
        const C gyz = cscale(gq[4 * NQ * TL], sz);
        const C gzz = gq[5 * NQ * TL];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (h >= two) break;
            const T sy = h ? (T)-1 : (T)1;
            const C hxy = cscale(gxy, sy), hyz = cscale(gyz, sy);
            C* row = sm + p * PS + h * 3 * TL + il;
            const C vx = row[0], vy = row[TL], vz = row[2 * TL];
            row[0] = cadd(cadd(cmul(gxx, vx), cmul(hxy, vy)), cmul(gxz, vz));
            row[TL] = cadd(cadd(cmul(hxy, vx), cmul(gyy, vy)), cmul(hyz, vz));
            row[2 * TL] = cadd(cadd(cmul(gxz, vx), cmul(hyz, vy)), cmul(gzz, vz));
        }
    }
    __syncthreads();
    fft_tile<C, L, NB, NT, -1, Layout<PS, 1, true>>(sm, tw, SmemIO{},
                                                    ZStore<T>{B2, rs, comp, row0, row1, X, i0, TL, two});
}

// ---- pass 5 -----------------------------------------------------------------
template <class T, bool TAB> struct InvXStore {
    static constexpr bool GLOBAL = true, HALF = true;  // keep points < nx
    const MvArgs<T>* a;
    const cplx<T>* bv;
    cplx<T>* yv;
    long site0;
    int nl, tl;
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const int c = b / tl, jl = b - c * tl;
        if (jl >= nl) return;
        const long site = site0 + (long)jl * a->g.nx + p;
        long d = site;
        if (TAB) {
            const int t = a->tabdip[site];
            if (t == 0) return;
            d = (long)t - 1;
        }
        yv[3 * d + c] = csub(bv[3 * d + c], cscale(v, a->inv_m));
    }
};

template <class T, int L, bool TAB, class Epi>
__global__ void __launch_bounds__(MvTiles<T, L>::NTX) k_inv_x(const MvArgs<T> a, const Epi epi) {
    using C = cplx<T>;
    using TT = MvTiles<T, L>;
    constexpr int TL = TT::TLX, NB = TT::NBX, NT = TT::NTX;
    const int rhs = blockIdx.z;
    if (a.status && a.status[rhs]) return;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int j0 = blockIdx.x * TL, k = blockIdx.y;
    const int nl = min(TL, ny - j0);
    load_twiddles<C, L, NT>(tw, a.twx);
    B1RowIO<T, L, TL> src{a.B1 + rhs * a.g.b1_rhs, nl, nz, ny, k, j0};
    InvXStore<T, TAB> dst{&a, a.b + rhs * a.xstride, a.y + rhs * a.xstride, (long)k * nx * ny + (long)j0 * nx, nl,
                          TL};
    fft_tile<C, L, NB, NT, -1, Layout<1, TT::LP, false>>(sm, tw, src, dst);
    (void)epi;
}

struct EpiNone {};

}  // namespace ifdda
