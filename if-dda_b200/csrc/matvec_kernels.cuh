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
    int zvar, yvar;      // tile variants of zconv and of the y passes (MvTiles V)
    // Ragged batch (objects of different lattices, spacings and wavelengths
    // on one common box): per right-hand side, its object's spectrum and the
    // offsets of its polarisability (dipoles) and Tabdip (box sites) in the
    // concatenated alpha / tabdip arrays.  Null: one object for every rhs.
    const C* const* gc_r;
    const long* alpha_off;
    const long* tab_off;
    __device__ __forceinline__ const int* tab_of(int rhs) const { return tab_off ? tabdip + tab_off[rhs] : tabdip; }
    __device__ __forceinline__ const C* alpha_of(int rhs) const { return alpha_off ? alpha + alpha_off[rhs] : alpha; }
};

// Tile shapes: lines per block, threads per block and the register cap of
// each pass.  The rules come from a sweep of every pass over tile widths,
// thread counts and register caps on B200 at the 128^3 (FP32, FP64),
// 192x192x128 (8 right-hand sides) and 384^3 grids:
//  * x passes: latency-bound at small grids (every shape within 5%); a cap of
//    80 (FP32) / 96 (FP64) registers helps the larger grids;
//  * y passes: 16 columns per block (64 contiguous bytes per row in FP32) at
//    every length, about 30% faster than narrower tiles at 192 and 384;
//  * zconv: as many columns as fit in ~80 KB (FP32) / ~160 KB (FP64) of
//    shared memory, so that two blocks (FP32) share an SM, and a register
//    cap near 72 (FP32) / 168 (FP64) to keep more blocks resident.
//
// Variant V = 1 (compiled for lengths of 64 and more, where the grid is large
// enough for the choice to matter) halves the zconv and y tiles; the tile
// chooser (tune_tiles) times both on the caller's grid and keeps one per
// grid.  The two agree to rounding (the compiler may contract multiply-adds
// differently in the two instances).
constexpr int tile_variants(int L) { return L >= 64 ? 2 : 1; }
template <class T, int L, int V = 0> struct MvTiles {
    static constexpr int S = (int)sizeof(cplx<T>);
    static constexpr int SMEM_X = 16384;
    static constexpr int TLX = clamp_pow2(SMEM_X / (3 * (L + 1) * S), 1, 16);
    static constexpr int TLY = V ? 8 : 16;
    static constexpr int NBX = 3 * TLX, NBY = TLY;
    // x tile: points contiguous with one pad word every 16, line pitch = 8 (mod 16)
    static constexpr int lpitch() {
        int p = L + L / 16 + 1;
        while (p % 16 != 8) p++;
        return p;
    }
    static constexpr int LP = lpitch();
    // one butterfly of the widest radix per thread
    static constexpr int nthreads(int nb, int policy = 0) {
        int t = nb * L / max_radix(L, policy);
        t = (t + 31) / 32 * 32;
        return t < 64 ? 64 : (t > 512 ? 512 : t);
    }
    // blocks per SM asked of the compiler so that it keeps to about cap registers
    static constexpr int minblocks(int nt, int cap) {
        int m = 65536 / (nt * cap);
        if (m * nt > 2048) m = 2048 / nt;
        return m < 1 ? 1 : (m > 32 ? 32 : m);
    }
    // z tile: shared memory of TL columns of mr mirror rows (twiddles, data
    // tile with one pad point every 16, the block's slice of the compressed
    // spectrum)
    static constexpr size_t zbytes(int tl, int mr = 2) {
        return (size_t)L * S + (size_t)(L + (L >> 4)) * 3 * mr * tl * S + (size_t)6 * (L / 2 + 1) * tl * S;
    }
    // zconv's FFT plan in FP32: two passes (a 32- or 16-point first pass)
    // where that saves a pass over the usual plan (lengths 96, 160, 192, 256,
    // 384), at about 120 registers a thread; FP64 keeps the usual plan (its
    // 12-point middle for three components would not fit the registers)
    static constexpr int ZP = (S == 8 && plan_len(L, 1) > 0 && plan_len(L, 1) < plan_len(L, 0)) ? 1 : 0;
    // With the two-pass plan the tile is wider (up to ~120 KB, 32-byte rows
    // at 384), one block per SM.  Variant 1 takes one of the two mirror rows
    // per block (MRZ = 1) and as many columns as fit (up to ~160 KB with the
    // two-pass plan, 64-byte rows at 384; up to 112 KB otherwise, so that two
    // blocks share an SM in FP64 too): wider rows, whose DRAM accesses are
    // less scattered, the spectrum slice then read by the two blocks of a row
    // pair back to back (L2 serves the second).  The tile chooser times the
    // two.
    static constexpr int MRZ = V ? 1 : 2;
    static constexpr int ztile() {
        const size_t budget = MRZ == 1 ? (size_t)(ZP ? 160 : 112) * 1024 : (size_t)(ZP ? 120 : 80) * 1024 * (S / 8);
        int tl = 16;
        while (tl > 1 && zbytes(tl, MRZ) > budget) tl /= 2;
        return tl;
    }
    static constexpr int TLZ = ztile(), NBZ = 3 * MRZ * TLZ;
    // L2 prefetch size of the column reads of zconv and the y passes (rows of
    // TLZ or TLY columns, 32 to 128 bytes, that neighbouring blocks read at
    // the same time): 256-byte DRAM bursts, 4-5% faster at 192^2 x 128 and 384^3
    static constexpr int ZPF = 256;
    // y tile: odd point stride; z tile: point stride NBZ with one pad point every 16
    static constexpr int PSY = NBY + 1, PSZ = NBZ;
    using LayX = Layout<1, LP, false, 4>;
    using LayY = Layout<PSY, 1, true>;
    using LayZ = Layout<PSZ, 1, true, 4>;
    static constexpr int NTX = nthreads(NBX), NTY = nthreads(NBY), NTZ = nthreads(NBZ, ZP);
    static constexpr int MINBX = minblocks(NTX, S == 8 ? 80 : 96);
    static constexpr int MINBY = minblocks(NTY, S == 8 ? 80 : 112);
    static constexpr int MINBZ = minblocks(NTZ, S == 8 ? (ZP ? 128 : 72) : 168);
    static constexpr size_t smem_x = (size_t)L * S + (size_t)NBX * LP * S;
    static constexpr size_t smem_y = (size_t)L * S + (size_t)L * PSY * S;
    static constexpr size_t smem_z = (size_t)L * S + (size_t)LayZ::span(L) * PSZ * S +
                                     (size_t)6 * (L / 2 + 1) * TLZ * S;
    static_assert(zbytes(TLZ, MRZ) == smem_z, "z tile size rule and layout disagree");
};

// asynchronous global -> shared copy of one complex element (8 or 16 bytes);
// PF = 256 asks L2 to fetch the 256 bytes around it from DRAM
template <int PF = 0, class C> __device__ __forceinline__ void cp_async_elem(C* dst_smem, const C* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
    if constexpr (PF == 256)
        asm volatile("cp.async.ca.shared.global.L2::256B [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"((int)sizeof(C)));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"((int)sizeof(C)));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

template <class C> __device__ __forceinline__ C* smem_base() {
    extern __shared__ __align__(16) unsigned char ifdda_smem[];
    return reinterpret_cast<C*>(ifdda_smem);
}

// ---- pass 1 ---------------------------------------------------------------
// The mat-vec input: Pre::value(e) returns element e = 3 d + c of the vector
// to multiply.  PreNone reads it; a solver's Pre may instead form it from its
// own vectors (storing the result) and accumulate ND dot products, which the
// x pass leaves as per-block partial sums.  value() is called exactly once per
// element, except with a full polarisability tensor (three calls per
// element), which only PreNone supports.
template <class T> struct PreNone {
    static constexpr int ND = 0;
    const cplx<T>* x;
    double2 acc[1];
    __device__ __forceinline__ void bind(const MvArgs<T>& a, int rhs) { x = a.x + rhs * a.xstride; }
    template <class C> __device__ __forceinline__ C value(int e) { return __ldg(x + e); }
};

// Element offsets inside one right-hand side's vectors and scratch fit in 32
// bits for every compiled FFT length (at most 3 * 192^3 dipole components,
// 3 * 192 * 384^2 grid points), so the pass functors index with int from
// per-block base pointers; the fields they need are copied by value.
template <class T, bool TAB, class Pre> struct FwdXLoad {
    static constexpr bool GLOBAL = true, HALF = true;  // points p >= nx are the padding
    const int* tab;
    const cplx<T>* alpha;
    int amode, nmax, nx;
    mutable Pre pre;
    int site0, nl, tl;
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const int c = b / tl, jl = b - c * tl;
        if (jl >= nl) return czero<C>();
        const int site = site0 + jl * nx + p;
        int d = site;
        if (TAB) {
            const int t = __ldg(tab + site);
            if (t == 0) return czero<C>();
            d = t - 1;
        }
        if (amode == ALPHA_ISO) return cmul(__ldg(alpha + d), pre.template value<C>(3 * d + c));
        if (amode == ALPHA_FULL) {
            C acc = czero<C>();
#pragma unroll
            for (int q = 0; q < 3; q++)
                acc = cadd(acc, cmul(__ldg(alpha + d + nmax * (c + 3 * q)), pre.template value<C>(3 * d + q)));
            return acc;
        }
        return pre.template value<C>(3 * d + c);
    }
};

// B1 rows of one x-pass tile: line b = c * TL + jl is row ((c * nz + k) * ny + j0 + jl)
template <class T, int L, int TL> struct B1RowIO {
    static constexpr bool GLOBAL = true, HALF = false;
    cplx<T>* base;  // row (c = 0, k, j0) of this right-hand side
    int nl, cstride;  // valid rows, elements between components (nz ny L)
    template <class C> __device__ __forceinline__ int at(int b, int p) const {
        const int c = b / TL, jl = b - c * TL;
        return jl < nl ? c * cstride + jl * L + p : -1;
    }
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const int o = at<C>(b, p);
        if (o >= 0) base[o] = v;
    }
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const int o = at<C>(b, p);
        return o >= 0 ? base[o] : czero<C>();
    }
};

template <class T, int L, bool TAB, class TT = MvTiles<T, L>, class Pre = PreNone<T>>
__global__ void __launch_bounds__(TT::NTX, TT::MINBX) k_fwd_x(const MvArgs<T> a, const Pre pre, const MvRed red) {
    using C = cplx<T>;
    constexpr int TL = TT::TLX, NB = TT::NBX, NT = TT::NTX;
    const int rhs = blockIdx.z;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int j0 = blockIdx.x * TL, k = blockIdx.y;
    const int nl = min(TL, ny - j0);
    load_twiddles<C, L, NT>(tw, a.twx);
    pdl_trigger();
    pdl_wait();
    if (a.status && a.status[rhs]) return;
    FwdXLoad<T, TAB, Pre> src{a.tab_of(rhs), a.alpha_of(rhs), a.amode, (int)a.nmax, nx, pre, k * nx * ny + j0 * nx,
                              nl, TL};
    src.pre.bind(a, rhs);
    B1RowIO<T, L, TL> dst{a.B1 + rhs * a.g.b1_rhs + ((long)k * ny + j0) * L, nl, nz * ny * L};
    fft_tile<C, L, NB, NT, +1, typename TT::LayX>(sm, tw, src, dst);
    if constexpr (Pre::ND > 0)
        block_partial<NT, Pre::ND>(src.pre.acc,
                                   red.ppart + (((long)rhs * gridDim.y + k) * red.gxs + blockIdx.x) * Pre::ND);
}

// ---- pass 2 and 4 ---------------------------------------------------------
// DIR=+1: B1 (ny rows) -> B2 (Y rows);  DIR=-1: B2 (Y rows) -> B1 (ny rows)
template <class T, int DIR, int PF = 0> struct YLoad {
    static constexpr bool GLOBAL = true, HALF = DIR > 0;  // forward: rows >= ny are padding
    const cplx<T>* src;
    int X, i0;
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const int i = i0 + b;
        return i < X ? ld_l2pf<PF>(src + p * X + i) : czero<C>();
    }
};
template <class T, int DIR> struct YStore {
    static constexpr bool GLOBAL = true, HALF = DIR < 0;  // inverse: keep rows < ny
    cplx<T>* dst;
    int X, i0;
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const int i = i0 + b;
        if (i < X) dst[p * X + i] = v;
    }
};

template <class T, int L, int DIR, class TT = MvTiles<T, L>>
__global__ void __launch_bounds__(TT::NTY, TT::MINBY) k_pass_y(const MvArgs<T> a) {
    using C = cplx<T>;
    constexpr int TL = TT::TLY, NT = TT::NTY;
    const int rhs = blockIdx.z / 3, c = blockIdx.z - 3 * (blockIdx.z / 3);
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int X = a.g.X, ny = a.g.ny, nz = a.g.nz;
    const int i0 = blockIdx.x * TL, k = blockIdx.y;
    load_twiddles<C, L, NT>(tw, a.twy);
    pdl_trigger();
    pdl_wait();
    if (a.status && a.status[rhs]) return;
    const int rows_in = DIR > 0 ? ny : L;
    const int rows_out = DIR > 0 ? L : ny;
    const C* srcb = DIR > 0 ? a.B1 + rhs * a.g.b1_rhs : a.B2 + rhs * a.g.b2_rhs;
    C* dstb = DIR > 0 ? a.B2 + rhs * a.g.b2_rhs : a.B1 + rhs * a.g.b1_rhs;
    YLoad<T, DIR, TT::ZPF> src{srcb + ((long)c * nz + k) * rows_in * X, X, i0};
    YStore<T, DIR> dst{dstb + ((long)c * nz + k) * rows_out * X, X, i0};
    fft_tile<C, L, TL, NT, DIR, typename TT::LayY>(sm, tw, src, dst);
}

// ---- pass 3 -----------------------------------------------------------------
// lines b = (h * 3 + c) * TL + il: h = 0 row qy, h = 1 the mirror row Y - qy
template <class T, int TL, int PF = 0> struct ZLoad {
    static constexpr bool GLOBAL = true, HALF = true;  // rows >= nz are padding
    const cplx<T>* base;  // B2 of this right-hand side, column i0 of row qy
    int rs;    // elements between z rows (Y * X)
    int comp;  // elements between components (nz * Y * X)
    int drow;  // row Y - qy minus row qy
    int nv, two;  // valid columns, rows in the block (1 or 2)
    template <class C> __device__ __forceinline__ C load(int b, int p) const {
        const int hc = b / TL, il = b - hc * TL;
        const int h = hc / 3, c = hc - 3 * h;
        if (il >= nv || h >= two) return czero<C>();
        return ld_l2pf<PF>(base + c * comp + p * rs + h * drow + il);
    }
};
template <class T, int TL> struct ZStore {
    static constexpr bool GLOBAL = true, HALF = true;  // keep z rows < nz
    cplx<T>* base;
    int rs, comp, drow, nv, two;
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const int hc = b / TL, il = b - hc * TL;
        const int h = hc / 3, c = hc - 3 * h;
        if (il < nv && h < two) base[c * comp + p * rs + h * drow + il] = v;
    }
};

// Group g of the fused zconv middle -> (column il, butterfly j, mirror row h):
// order 0 takes il fastest, then j, then h; order 1 il, then h, then j.
__host__ __device__ constexpr void zmid_map(int order, int g, int TL, int NJ, int& il, int& j, int& h) {
    il = g % TL;
    if (order == 0) {
        j = (g / TL) % NJ;
        h = g / (TL * NJ);
    } else {
        h = (g / TL) % 2;
        j = g / (2 * TL);
    }
}

// Shared-memory cost of the middle's reads (points j + r NJ) and writes
// (points j RK + r) under a group order, for the first warps of a block: each
// request of 32 lanes is served in phases of 128 bytes (16 lanes of 8-byte or
// 8 lanes of 16-byte elements), and a phase costs the largest number of
// distinct addresses that share a bank group.  Used at compile time to pick
// the order without bank conflicts.
template <class LZ> constexpr int zmid_cost(int order, int TL, int NJ, int RK, int NG, int S) {
    const int per = 128 / S;
    int total = 0;
    for (int w = 0; w < 4 && w * 32 < NG; w++)
        for (int pass = 0; pass < 2; pass++)
            for (int r = 0; r < RK; r++)
                for (int ph = 0; ph < 32 / per; ph++) {
                    int addr[16] = {};
                    int n = 0;
                    for (int l = 0; l < per; l++) {
                        const int g = w * 32 + ph * per + l;
                        if (g >= NG) continue;
                        int il = 0, j = 0, h = 0;
                        zmid_map(order, g, TL, NJ, il, j, h);
                        const int p = pass == 0 ? j + r * NJ : j * RK + r;
                        addr[n++] = LZ::pidx(p) * LZ::PS + h * 3 * TL + il;
                    }
                    int worst = 0;
                    for (int a = 0; a < n; a++) {
                        int cnt = 0;
                        for (int q = 0; q < n; q++) {
                            if (addr[q] % per != addr[a] % per) continue;
                            bool dup = false;
                            for (int z = 0; z < q; z++) dup = dup || addr[z] == addr[q];
                            if (!dup) cnt++;
                        }
                        worst = cnt > worst ? cnt : worst;
                    }
                    total += worst;
                }
    return total;
}

// Forward z transform (passes 0 .. n-2 of the plan), then in registers: the
// last forward pass, the 3x3 multiply and the first pass of the inverse
// transform run on the reversed plan, so the inverse starts from the values
// the forward one ended with (its pass 0 reads exactly the points
// j + r L/R the forward last pass produced), then inverse passes 1 .. n-1.
// Grid (right-hand side, column tile, mirror-row pair): the right-hand side
// varies fastest, so the blocks that read one slice of the spectrum run
// together and a batch takes that slice from HBM once (L2 serves the rest).
// (A loop over right-hand sides inside the block, keeping the slice in shared
// memory, needs about twice the registers and spills.)
template <class T, int L, class TT = MvTiles<T, L>>
__global__ void __launch_bounds__(TT::NTZ, TT::MINBZ) k_zconv(const MvArgs<T> a) {
    using C = cplx<T>;
    using LZ = typename TT::LayZ;
    constexpr int TL = TT::TLZ, NB = TT::NBZ, NT = TT::NTZ;
    constexpr int ZP = TT::ZP;
    constexpr int NP = plan_len(L, ZP);
    constexpr int RK = plan_radix(L, NP - 1, ZP);  // last forward radix = first inverse radix
    constexpr int NJ = L / RK;                 // butterflies per line in that pass
    constexpr int MR = TT::MRZ;                // mirror rows per block
    constexpr int NG = MR * TL * NJ;           // (row half, column, butterfly) groups
    constexpr int PERM = (NG + NT - 1) / NT;
    constexpr int S = (int)sizeof(C);
    constexpr int ORDER =
        MR == 2 && zmid_cost<LZ>(1, TL, NJ, RK, NG, S) < zmid_cost<LZ>(0, TL, NJ, RK, NG, S) ? 1 : 0;
    constexpr int NQ = L / 2 + 1;
    // with one mirror row per block, blockIdx.x = 2 rhs + hm: hm = 1 takes
    // row Y - qy (which exists for 0 < qy < ny only)
    const int rhs = MR == 2 ? (int)blockIdx.x : (int)blockIdx.x >> 1;
    const int hm = MR == 2 ? 0 : (int)blockIdx.x & 1;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    C* gs = sm + LZ::span(L) * TT::PSZ;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz, X = a.g.X, Y = a.g.Y;
    const int i0 = blockIdx.y * TL;
    const int qy = blockIdx.z;                    // 0 .. ny
    const bool pair = qy > 0 && qy < ny;
    if (hm && !pair) return;
    const int two = MR == 2 && pair ? 2 : 1;      // rows qy and Y - qy in the block
    const int row = hm ? Y - qy : qy;             // the block's first row
    load_twiddles<C, L, NT>(tw, a.twz);
    const C* gbase = (a.gc_r ? a.gc_r[rhs] : a.Gc) + qy * (nx + 1);
    // this block's slice of the compressed spectrum (qy fixed, every qz, the
    // TL columns qx(i)) is copied into shared memory while the forward
    // transform runs
    {
        static_assert(NT % TL == 0, "a thread keeps one column of the slice");
        const int il = threadIdx.x % TL;
        const int i = min(i0 + il, X - 1);
        const int qxc = i <= nx ? i : X - i;
        const C* gsrc = gbase + qxc;
        const int gcs = (int)a.g.gc_comp, qzs = (ny + 1) * (nx + 1);
        for (int cq = threadIdx.x / TL; cq < 6 * NQ; cq += NT / TL) {
            const int c6 = cq / NQ, qz = cq - c6 * NQ;
            cp_async_elem<TT::ZPF>(gs + cq * TL + il, gsrc + c6 * gcs + qz * qzs);
        }
    }
    cp_async_commit();
    // the spectrum and the twiddles are constant: only B2 waits for the y pass
    pdl_trigger();
    pdl_wait();
    if (a.status && a.status[rhs]) {
        cp_async_wait_all();
        return;
    }
    C* B2 = a.B2 + rhs * a.g.b2_rhs + (long)row * X + i0;
    const int rs = Y * X, comp = nz * Y * X, drow = (Y - 2 * qy) * X, nv = min(TL, X - i0);
    const ZLoad<T, TL, TT::ZPF> zload{B2, rs, comp, drow, nv, two};
    const ZStore<T, TL> zstore{B2, rs, comp, drow, nv, two};
    if constexpr (NP > 1)
        stockham_range<C, L, NB, NT, +1, LZ, false, NP - 1, 0, 1, ZLoad<T, TL, TT::ZPF>, SmemIO, ZP>(sm, tw, zload,
                                                                                                    SmemIO{});
    cp_async_wait_all();
    __syncthreads();
    // ---- fused middle: read, transform, multiply, transform (registers) ----
    C v[PERM][3][RK];
#pragma unroll
    for (int q = 0; q < PERM; q++) {
        const int g = threadIdx.x + q * NT;
        if (!(PERM * NT == NG || g < NG)) continue;
        int il, j, h;
        zmid_map(ORDER, g, TL, NJ, il, j, h);
        const int i = i0 + il;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int b = (h * 3 + c) * TL + il;
#pragma unroll
            for (int r = 0; r < RK; r++) {
                const int p = j + r * NJ;
                if constexpr (NP == 1) {
                    v[q][c][r] = (2 * p >= L) ? czero<C>() : zload.template load<C>(b, p);
                } else if constexpr (read_split<LZ>(NJ, RK)) {
                    v[q][c][r] = sm[LZ::addr(j, b) + LZ::pidx(r * NJ) * LZ::PS];
                } else {
                    v[q][c][r] = sm[LZ::addr(p, b)];
                }
            }
            if constexpr (NJ > 1) {
                // forward last pass: Ns = NJ, k = j, twiddle w^(j r)
#pragma unroll
                for (int r = 1; r < RK; r++) v[q][c][r] = cmul(v[q][c][r], tw[j * r]);
            }
            Dft<RK, +1, C>::run(v[q][c]);
        }
        if (h < two && i < X) {
            const T sx = i <= nx ? (T)1 : (T)-1;
            const T sy = (h | hm) ? (T)-1 : (T)1;
#pragma unroll
            for (int r = 0; r < RK; r++) {
                const int p = j + r * NJ;  // spectral index of this output
                const int qzc = 2 * p <= L ? p : L - p;  // nz = L / 2
                const T sz = 2 * p <= L ? (T)1 : (T)-1;
                C g6[6];
                const C* gq = gs + qzc * TL + il;
#pragma unroll
                for (int c6 = 0; c6 < 6; c6++) g6[c6] = gq[c6 * NQ * TL];
                const C gxx = g6[0];
                const C gxy = cscale(g6[1], sx * sy);
                const C gxz = cscale(g6[2], sx * sz);
                const C gyy = g6[3];
                const C gyz = cscale(g6[4], sy * sz);
                const C gzz = g6[5];
                const C vx = v[q][0][r], vy = v[q][1][r], vz = v[q][2][r];
                v[q][0][r] = cadd(cadd(cmul(gxx, vx), cmul(gxy, vy)), cmul(gxz, vz));
                v[q][1][r] = cadd(cadd(cmul(gxy, vx), cmul(gyy, vy)), cmul(gyz, vz));
                v[q][2][r] = cadd(cadd(cmul(gxz, vx), cmul(gyz, vy)), cmul(gzz, vz));
            }
        }
        // inverse pass 0 of the reversed plan: Ns = 1, inputs j + r NJ, no twiddles
#pragma unroll
        for (int c = 0; c < 3; c++) Dft<RK, -1, C>::run(v[q][c]);
    }
    if constexpr (NP > 1) __syncthreads();  // every read of the tile is done
#pragma unroll
    for (int q = 0; q < PERM; q++) {
        const int g = threadIdx.x + q * NT;
        if (!(PERM * NT == NG || g < NG)) continue;
        int il, j, h;
        zmid_map(ORDER, g, TL, NJ, il, j, h);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const int b = (h * 3 + c) * TL + il;
#pragma unroll
            for (int r = 0; r < RK; r++) {
                const int o = j * RK + r;
                if constexpr (NP == 1) {
                    if (2 * o < L) zstore.template store<C>(b, o, v[q][c][r]);
                } else if constexpr (write_split<LZ>(NJ, 1, RK)) {
                    sm[LZ::addr(j * RK, b) + LZ::pidx(r) * LZ::PS] = v[q][c][r];
                } else {
                    sm[LZ::addr(o, b)] = v[q][c][r];
                }
            }
        }
    }
    if constexpr (NP > 1) {
        __syncthreads();
        stockham_range<C, L, NB, NT, -1, LZ, true, NP, 1, RK, SmemIO, ZStore<T, TL>, ZP>(sm, tw, SmemIO{}, zstore);
    }
}

// ---- pass 5 -----------------------------------------------------------------
// The mat-vec output: Epi::elem(e, y) sees every stored element y of the
// result (e = 3 d + c) and may accumulate ND dot products; the last block of
// the grid then holds them, with the NDP partials of the first x pass, and
// calls Epi::finish.
struct EpiNone {
    static constexpr int ND = 0, NDP = 0;
    double2 acc[1];
    template <class T> __device__ __forceinline__ void bind(const MvArgs<T>&, int) {}
    template <class C> __device__ __forceinline__ void elem(int, C) {}
    __device__ __forceinline__ void finish(int, const double2*) {}
};

template <class T, bool TAB, class Epi> struct InvXStore {
    static constexpr bool GLOBAL = true, HALF = true;  // keep points < nx
    const int* tab;
    const cplx<T>* bv;
    cplx<T>* yv;
    T inv_m;
    int nx, site0, nl, tl;
    mutable Epi epi;
    template <class C> __device__ __forceinline__ void store(int b, int p, C v) const {
        const int c = b / tl, jl = b - c * tl;
        if (jl >= nl) return;
        const int site = site0 + jl * nx + p;
        int d = site;
        if (TAB) {
            const int t = __ldg(tab + site);
            if (t == 0) return;
            d = t - 1;
        }
        // b is read at an element before this thread writes y there (b may be y)
        const C y = csub(__ldg(bv + 3 * d + c), cscale(v, inv_m));
        yv[3 * d + c] = y;
        epi.elem(3 * d + c, y);
    }
};

template <class T, int L, bool TAB, class Epi, class TT = MvTiles<T, L>>
__global__ void __launch_bounds__(TT::NTX, TT::MINBX) k_inv_x(const MvArgs<T> a, const Epi epi, const MvRed red) {
    using C = cplx<T>;
    constexpr int TL = TT::TLX, NB = TT::NBX, NT = TT::NTX;
    const int rhs = blockIdx.z;
    C* tw = smem_base<C>();
    C* sm = tw + L;
    const int nx = a.g.nx, ny = a.g.ny, nz = a.g.nz;
    const int j0 = blockIdx.x * TL, k = blockIdx.y;
    const int nl = min(TL, ny - j0);
    load_twiddles<C, L, NT>(tw, a.twx);
    pdl_trigger();
    pdl_wait();
    if (a.status && a.status[rhs]) return;
    B1RowIO<T, L, TL> src{a.B1 + rhs * a.g.b1_rhs + ((long)k * ny + j0) * L, nl, nz * ny * L};
    InvXStore<T, TAB, Epi> dst{a.tab_of(rhs), a.b + rhs * a.xstride, a.y + rhs * a.xstride, a.inv_m, nx,
                               k * nx * ny + j0 * nx, nl, TL, epi};
    dst.epi.bind(a, rhs);
    fft_tile<C, L, NB, NT, -1, typename TT::LayX>(sm, tw, src, dst);
    if constexpr (Epi::ND > 0) {
        double2 tot[Epi::ND + Epi::NDP];
        if (reduce_rows<NT, Epi::ND, Epi::NDP>(dst.epi.acc, tot, rhs, blockIdx.x, k, gridDim.x, gridDim.y, red) &&
            threadIdx.x == 0)
            dst.epi.finish(rhs, tot);
    }
}

}  // namespace ifdda
