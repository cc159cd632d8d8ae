// Shared-memory Stockham FFT on a tile of NB independent lines of length L.
//
// Layout in shared memory: point p of line b sits at sm[p * LS + b] (lines
// fastest), so a warp touching consecutive lines at one point reads
// consecutive words.  Each pass of radix R combines R sub-transforms of length
// Ns into one of length Ns * R (autosort Stockham, natural-order output):
//     v[r] = x[j + r L/R] * w^(DIR * (j mod Ns) * r * L / (Ns R)),  r < R
//     v    = DFT_R(v, DIR)
//     x[(j / Ns) Ns R + (j mod Ns) + r Ns] = v[r]
// Every thread keeps its butterflies in registers across a barrier, so the
// transform runs in place.  DIR = +1 is exp(+i 2 pi jk / L) (the reference's
// "forward" convention for G and x, cdmlib/calculgreenfft.f:16,76-99), DIR = -1
// the inverse; both unnormalised.  L may be any product of 2, 3 and 5.
#pragma once
#include "cplx.cuh"

namespace ifdda {

// radix used for the pass that starts at sub-length Ns
__host__ __device__ constexpr int pick_radix(int rem) {
    return rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2 : rem % 3 == 0 ? 3 : rem % 5 == 0 ? 5 : 0;
}
__host__ __device__ constexpr int num_passes(int L) {
    int n = 0;
    for (int rem = L; rem > 1; rem /= pick_radix(rem)) {
        if (pick_radix(rem) == 0) return -1;
        n++;
    }
    return n;
}
__host__ __device__ constexpr bool smooth235(int L) {
    if (L < 1) return false;
    while (L % 2 == 0) L /= 2;
    while (L % 3 == 0) L /= 3;
    while (L % 5 == 0) L /= 5;
    return L == 1;
}

__host__ __device__ constexpr int clamp_pow2(int v, int lo, int hi) {
    int p = 1;
    while (p * 2 <= v && p * 2 <= hi) p *= 2;
    return p < lo ? lo : p;
}

// Exact mathematical constants used by the radix-3/5/8 butterflies.
#define IFDDA_SQRT3_2 0.86602540378443864676372317075294
#define IFDDA_SQRT1_2 0.70710678118654752440084436210485
#define IFDDA_C1_5 0.30901699437494742410229341718282   // cos(2 pi / 5)
#define IFDDA_C2_5 -0.80901699437494742410229341718282  // cos(4 pi / 5)
#define IFDDA_S1_5 0.95105651629515357211643933337938   // sin(2 pi / 5)
#define IFDDA_S2_5 0.58778525229247312916870595463907   // sin(4 pi / 5)

template <int R, int DIR, class C> struct Dft;

template <int DIR, class C> struct Dft<2, DIR, C> {
    __device__ __forceinline__ static void run(C* v) {
        C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int DIR, class C> struct Dft<4, DIR, C> {
    __device__ __forceinline__ static void run(C* v) {
        C s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        C s13 = cadd(v[1], v[3]), d13 = cmul_i<DIR>(csub(v[1], v[3]));
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    }
};

template <int DIR, class C> struct Dft<8, DIR, C> {
    __device__ __forceinline__ static void run(C* v) {
        using T = decltype(C().x);
        C e[4] = {v[0], v[2], v[4], v[6]};
        C o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, DIR, C>::run(e);
        Dft<4, DIR, C>::run(o);
        const T h = (T)IFDDA_SQRT1_2;
        // w^1 = (1 + DIR i)/sqrt2, w^2 = DIR i, w^3 = (-1 + DIR i)/sqrt2
        C o1 = cscale(cadd(o[1], cmul_i<DIR>(o[1])), h);
        C o2 = cmul_i<DIR>(o[2]);
        C o3 = cscale(csub(cmul_i<DIR>(o[3]), o[3]), h);
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

template <int DIR, class C> struct Dft<3, DIR, C> {
    __device__ __forceinline__ static void run(C* v) {
        using T = decltype(C().x);
        C t1 = cadd(v[1], v[2]);
        C t2 = csub(v[0], cscale(t1, (T)0.5));
        C t3 = cmul_i<DIR>(cscale(csub(v[1], v[2]), (T)IFDDA_SQRT3_2));
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    }
};

template <int DIR, class C> struct Dft<5, DIR, C> {
    __device__ __forceinline__ static void run(C* v) {
        using T = decltype(C().x);
        const T c1 = (T)IFDDA_C1_5, c2 = (T)IFDDA_C2_5, s1 = (T)IFDDA_S1_5, s2 = (T)IFDDA_S2_5;
        C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        C a1 = cadd(v[0], cadd(cscale(t1, c1), cscale(t2, c2)));
        C a2 = cadd(v[0], cadd(cscale(t1, c2), cscale(t2, c1)));
        C b1 = cmul_i<DIR>(cadd(cscale(t3, s1), cscale(t4, s2)));
        C b2 = cmul_i<DIR>(csub(cscale(t3, s2), cscale(t4, s1)));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, b1);
        v[4] = csub(a1, b1);
        v[2] = cadd(a2, b2);
        v[3] = csub(a2, b2);
    }
};

// One Stockham pass.  tw[j] = exp(+2 pi i j / L) in shared memory.
template <class C, int L, int Ns, int NB, int LS, int NT, int DIR>
__device__ __forceinline__ void stockham_pass(C* sm, const C* tw) {
    constexpr int R = pick_radix(L / Ns);
    constexpr int NBF = NB * (L / R);
    constexpr int PER = (NBF + NT - 1) / NT;
    constexpr int TSTEP = L / (Ns * R);
    C v[PER][R];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int u = threadIdx.x + q * NT;
        if (PER * NT == NBF || u < NBF) {
            const int b = u % NB, j = u / NB;
#pragma unroll
            for (int r = 0; r < R; r++) v[q][r] = sm[(j + r * (L / R)) * LS + b];
            if (Ns > 1) {
                const int k = j % Ns;
#pragma unroll
                for (int r = 1; r < R; r++) {
                    C w = tw[k * r * TSTEP];
                    if (DIR < 0) w = cconj(w);
                    v[q][r] = cmul(v[q][r], w);
                }
            }
            Dft<R, DIR, C>::run(v[q]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int u = threadIdx.x + q * NT;
        if (PER * NT == NBF || u < NBF) {
            const int b = u % NB, j = u / NB;
            const int k = j % Ns;
            const int d = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) sm[(d + r * Ns) * LS + b] = v[q][r];
        }
    }
    __syncthreads();
}

template <class C, int L, int Ns, int NB, int LS, int NT, int DIR>
__device__ __forceinline__ void stockham_chain(C* sm, const C* tw) {
    if constexpr (Ns < L) {
        stockham_pass<C, L, Ns, NB, LS, NT, DIR>(sm, tw);
        stockham_chain<C, L, Ns * pick_radix(L / Ns), NB, LS, NT, DIR>(sm, tw);
    }
}

// Full transform of the tile; callers __syncthreads() before (data in place)
// and may read the result right after.
template <class C, int L, int NB, int LS, int NT, int DIR>
__device__ __forceinline__ void tile_fft(C* sm, const C* tw) {
    static_assert(smooth235(L), "FFT length must be a product of 2, 3 and 5");
    stockham_chain<C, L, 1, NB, LS, NT, DIR>(sm, tw);
}

// copy the twiddle table for length L into shared memory
template <class C, int L, int NT>
__device__ __forceinline__ void load_twiddles(C* tws, const C* __restrict__ twg) {
    for (int j = threadIdx.x; j < L; j += NT) tws[j] = twg[j];
}

}  // namespace ifdda
