// Shared-memory Stockham FFT on a tile of NB independent lines of length L.
//
// Each pass of radix R combines R sub-transforms of length Ns into one of
// length Ns * R (autosort Stockham, natural-order output):
//     v[r] = x[j + r L/R] * w^(DIR * (j mod Ns) * r * L / (Ns R)),  r < R
//     v    = DFT_R(v, DIR)
//     x[(j / Ns) Ns R + (j mod Ns) + r Ns] = v[r]
// Every thread keeps its butterflies in registers across a barrier, so the
// transform runs in place.  DIR = +1 is exp(+i 2 pi jk / L) (the reference's
// "forward" convention for G and x, cdmlib/calculgreenfft.f:16,76-99), DIR = -1
// the inverse; both unnormalised.  L may be any product of 2, 3 and 5.
//
// The first pass may read its inputs straight from global memory (Src::GLOBAL)
// and the last pass may write straight to global memory (Dst::GLOBAL), so a
// transform costs one shared-memory round trip less at each end.  With
// Src::HALF the upper half of the input is known to be zero (the padding of
// the circulant embedding) and is neither loaded nor stored; with Dst::HALF
// only the first half of the output is written (the crop).
//
// Shared-memory layout: point p of line b at sm[p * PS + b * BS].  With
// BFAST the butterflies of consecutive threads belong to consecutive lines
// (use with BS = 1: lines contiguous in global memory, e.g. the y and z axes);
// otherwise consecutive threads take consecutive points of one line (PS = 1,
// e.g. the x axis).
#pragma once
#include "cplx.cuh"

namespace ifdda {

// radices 8, 4, 2, 3, 5 in that order of preference
__host__ __device__ constexpr int pick_radix_basic(int rem) {
    return rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2 : rem % 3 == 0 ? 3 : rem % 5 == 0 ? 5 : 0;
}
__host__ __device__ constexpr int passes_basic(int rem) {
    int n = 0;
    while (rem > 1) {
        const int r = pick_radix_basic(rem);
        if (r == 0) return 1000;
        rem /= r;
        n++;
    }
    return n;
}
// radix of the pass that has `rem` = L / Ns points left to combine: the
// first pass takes 16 where that saves a whole pass (one shared-memory round
// trip less; the first pass needs no table twiddles), otherwise 8, 4, 2, 3, 5
__host__ __device__ constexpr int pick_radix(int rem, bool first = false) {
    return (first && rem % 16 == 0 && 1 + passes_basic(rem / 16) < passes_basic(rem)) ? 16 : pick_radix_basic(rem);
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
// Radices with a register butterfly (Dft<R> below).
__host__ __device__ constexpr bool has_dft(int r) {
    return r == 2 || r == 3 || r == 4 || r == 5 || r == 8 || r == 12 || r == 16 || r == 32;
}
// Plan policy 1 (two passes): a first radix of 32 or 16 and one more radix of
// at most 12, where such a pair exists; otherwise policy 0.  It halves the
// shared-memory round trips of a three-pass length (160, 192, 256, 384) for
// a kernel that can afford the registers of a 32-point butterfly.
__host__ __device__ constexpr int two_pass_first(int L) {
    return (L % 32 == 0 && has_dft(L / 32) && L / 32 <= 12) ? 32
         : (L % 16 == 0 && has_dft(L / 16) && L / 16 <= 12) ? 16 : 0;
}
__host__ __device__ constexpr int pick_radix_p(int L, int rem, bool first, int policy) {
    if (policy == 1 && two_pass_first(L)) return first ? two_pass_first(L) : rem;
    return pick_radix(rem, first);
}
// The plan of L: radix of pass q (0-based) and number of passes.  A plan
// runs forward (q = 0 .. n-1) or reversed; any order of the radices is a
// valid Stockham transform, and the reversed plan lets an inverse transform
// start from the registers the forward transform ended with.
__host__ __device__ constexpr int plan_len(int L, int policy = 0) {
    int n = 0;
    bool first = true;
    for (int rem = L; rem > 1;) {
        const int r = pick_radix_p(L, rem, first, policy);
        if (r == 0) return -1;
        rem /= r;
        first = false;
        n++;
    }
    return n;
}
__host__ __device__ constexpr int plan_radix(int L, int q, int policy = 0) {
    int rem = L;
    bool first = true;
    for (int i = 0; i < q; i++) {
        rem /= pick_radix_p(L, rem, first, policy);
        first = false;
    }
    return pick_radix_p(L, rem, first, policy);
}
__host__ __device__ constexpr int plan_radix_dir(int L, int q, bool rev, int policy = 0) {
    return rev ? plan_radix(L, plan_len(L, policy) - 1 - q, policy) : plan_radix(L, q, policy);
}

// largest radix used by the plan of L (sets the register footprint)
__host__ __device__ constexpr int max_radix(int L, int policy = 0) {
    int m = 1;
    bool first = true;
    for (int rem = L; rem > 1;) {
        const int r = pick_radix_p(L, rem, first, policy);
        if (r == 0) return 0;
        m = r > m ? r : m;
        rem /= r;
        first = false;
    }
    return m;
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

// 16 points as 4 x 4: DFT4 over the stride-4 subsequences, the inner twiddles
// w16^(n2 k1), then DFT4 across them; X[k1 + 4 k2]
#define IFDDA_COS_PI8 0.92387953251128675612818318939679  // cos(pi / 8)
#define IFDDA_SIN_PI8 0.38268343236508977172845998403040  // sin(pi / 8)
template <int DIR, class C> struct Dft<16, DIR, C> {
    __device__ __forceinline__ static void run(C* v) {
        using T = decltype(C().x);
        C a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) {
            C t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
            Dft<4, DIR, C>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++) a[n2][k1] = t[k1];
        }
        const T c = (T)IFDDA_COS_PI8, s = (T)IFDDA_SIN_PI8, h = (T)IFDDA_SQRT1_2;
        const T ds = DIR > 0 ? s : -s, dc = DIR > 0 ? c : -c, dh = DIR > 0 ? h : -h;
        // w^1 = c + i DIR s, w^2 = (1 + i DIR)/sqrt2, w^3 = s + i DIR c,
        // w^4 = i DIR, w^6 = (-1 + i DIR)/sqrt2, w^9 = -w^1
        const C w1 = mk(c, ds), w2 = mk(h, dh), w3 = mk(s, dc), w6 = mk(-h, dh), w9 = mk(-c, -ds);
        a[1][1] = cmul(a[1][1], w1);
        a[1][2] = cmul(a[1][2], w2);
        a[1][3] = cmul(a[1][3], w3);
        a[2][1] = cmul(a[2][1], w2);
        a[2][2] = cmul_i<DIR>(a[2][2]);
        a[2][3] = cmul(a[2][3], w6);
        a[3][1] = cmul(a[3][1], w3);
        a[3][2] = cmul(a[3][2], w6);
        a[3][3] = cmul(a[3][3], w9);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            C t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
            Dft<4, DIR, C>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[k2];
        }
    }
};

// 32 points as 2 x 16: DFT16 over the even and the odd points, the twiddles
// w32^k on the odd half, then DFT2 across; X[k] and X[k + 16]
#define IFDDA_COS_PI16 0.98078528040323044912618223613424   // cos(pi / 16)
#define IFDDA_SIN_PI16 0.19509032201612826784828486847702   // sin(pi / 16)
#define IFDDA_COS_3PI16 0.83146961230254523707878837761791  // cos(3 pi / 16)
#define IFDDA_SIN_3PI16 0.55557023301960222474283081394853  // sin(3 pi / 16)
template <int DIR, class C> struct Dft<32, DIR, C> {
    __device__ __forceinline__ static void run(C* v) {
        using T = decltype(C().x);
        C e[16], o[16];
#pragma unroll
        for (int n = 0; n < 16; n++) {
            e[n] = v[2 * n];
            o[n] = v[2 * n + 1];
        }
        Dft<16, DIR, C>::run(e);
        Dft<16, DIR, C>::run(o);
        // cos and sin of k pi / 16, k = 0..8 (k pi / 16 for k > 8 by symmetry)
        const T cs[9] = {(T)1, (T)IFDDA_COS_PI16, (T)IFDDA_COS_PI8, (T)IFDDA_COS_3PI16, (T)IFDDA_SQRT1_2,
                         (T)IFDDA_SIN_3PI16, (T)IFDDA_SIN_PI8, (T)IFDDA_SIN_PI16, (T)0};
#pragma unroll
        for (int k = 0; k < 16; k++) {
            // w32^k = cos(k pi/16) + i DIR sin(k pi/16)
            const T c = k <= 8 ? cs[k] : -cs[16 - k];
            const T sn = k <= 8 ? cs[8 - k] : cs[k - 8];
            const C w = mk(c, DIR > 0 ? sn : -sn);
            const C t = k == 0 ? o[0] : cmul(o[k], w);
            v[k] = cadd(e[k], t);
            v[k + 16] = csub(e[k], t);
        }
    }
};

// 12 points as 4 x 3: DFT3 over the stride-4 subsequences, the twiddles
// w12^(n2 k1), then DFT4 across them; X[k1 + 3 k2]
template <int DIR, class C> struct Dft<12, DIR, C> {
    __device__ __forceinline__ static void run(C* v);
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

template <int DIR, class C> __device__ __forceinline__ void Dft<12, DIR, C>::run(C* v) {
    using T = decltype(C().x);
    C a[4][3];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
        C t[3] = {v[n2], v[4 + n2], v[8 + n2]};
        Dft<3, DIR, C>::run(t);
#pragma unroll
        for (int k1 = 0; k1 < 3; k1++) a[n2][k1] = t[k1];
    }
    // w12^1 = (sqrt3/2, DIR/2), w12^2 = (1/2, DIR sqrt3/2), w12^4 = (-1/2, DIR sqrt3/2)
    const T h = (T)0.5, r3 = (T)IFDDA_SQRT3_2;
    const C w1 = mk(r3, DIR > 0 ? h : -h), w2 = mk(h, DIR > 0 ? r3 : -r3), w4 = mk(-h, DIR > 0 ? r3 : -r3);
    a[1][1] = cmul(a[1][1], w1);
    a[1][2] = cmul(a[1][2], w2);
    a[2][1] = cmul(a[2][1], w2);
    a[2][2] = cmul(a[2][2], w4);
    a[3][1] = cmul_i<DIR>(a[3][1]);  // w12^3
    a[3][2] = cscale(a[3][2], (T)-1);  // w12^6
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
        C t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
        Dft<4, DIR, C>::run(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) v[k1 + 3 * k2] = t[k2];
    }
}

// Source / destination that is the shared-memory tile itself.
struct SmemIO {
    static constexpr bool GLOBAL = false;
    static constexpr bool HALF = false;
    template <class C> __device__ C load(int, int) const { return C(); }
    template <class C> __device__ void store(int, int, C) const {}
};

// PADSH > 0 inserts one padding word every 2^PADSH points, so the strided
// writes of a radix-R pass (points j*R + r of consecutive j) spread over the
// shared-memory banks.
template <int PS_, int BS_, bool BFAST_, int PADSH_ = 0> struct Layout {
    static constexpr int PS = PS_, BS = BS_, PADSH = PADSH_;
    static constexpr bool BFAST = BFAST_;
    // padded position of point p
    __host__ __device__ static constexpr int pidx(int p) { return PADSH ? p + (p >> PADSH) : p; }
    __device__ __forceinline__ static int addr(int p, int b) { return pidx(p) * PS + b * BS; }
    // points spanned by a line of length L (padding included)
    static constexpr int span(int L) { return PADSH ? L + (L >> PADSH) : L; }
};

// True when the padded positions of a butterfly's points j + r NJ (j < NJ,
// r < R) are pidx(j) + pidx(r NJ): the shared-memory address of every point
// is then the thread's base address plus a compile-time offset.
template <class Lay> constexpr bool read_split(int NJ, int R) {
    for (int j = 0; j < NJ; j++)
        for (int r = 0; r < R; r++)
            if (Lay::pidx(j + r * NJ) - Lay::pidx(j) != Lay::pidx(r * NJ)) return false;
    return true;
}
// The same for the outputs d + r Ns, d = (j / Ns) Ns R + j mod Ns, of a pass.
template <class Lay> constexpr bool write_split(int NJ, int Ns, int R) {
    for (int j = 0; j < NJ; j++) {
        const int d = (j / Ns) * Ns * R + j % Ns;
        for (int r = 0; r < R; r++)
            if (Lay::pidx(d + r * Ns) - Lay::pidx(d) != Lay::pidx(r * Ns)) return false;
    }
    return true;
}

// One Stockham pass.  tw[j] = exp(+2 pi i j / L) in shared memory.
template <class C, int L, int R, int Ns, int NB, int NT, int DIR, class Lay, class Src, class Dst>
__device__ __forceinline__ void stockham_pass(C* sm, const C* tw, const Src& src, const Dst& dst) {
    constexpr int NJ = L / R;
    constexpr int NBF = NB * NJ;
    constexpr int PER = (NBF + NT - 1) / NT;
    constexpr int TSTEP = L / (Ns * R);
    constexpr bool FIRST = Ns == 1, LAST = Ns * R == L;
    constexpr bool GIN = FIRST && Src::GLOBAL, GOUT = LAST && Dst::GLOBAL;
    constexpr bool RSPLIT = read_split<Lay>(NJ, R), WSPLIT = write_split<Lay>(NJ, Ns, R);
    C v[PER][R];
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int u = threadIdx.x + q * NT;
        if (PER * NT == NBF || u < NBF) {
            const int b = Lay::BFAST ? u % NB : u / NJ;
            const int j = Lay::BFAST ? u / NB : u % NJ;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int p = j + r * NJ;
                if (GIN) {
                    // zero upper half: for an even radix p >= L/2 exactly when r >= R/2
                    const bool zero = Src::HALF && (R % 2 == 0 ? 2 * r >= R : 2 * p >= L);
                    v[q][r] = zero ? mk(decltype(C().x)(0), decltype(C().x)(0)) : src.template load<C>(b, p);
                } else if constexpr (RSPLIT) {
                    v[q][r] = sm[Lay::addr(j, b) + Lay::pidx(r * NJ) * Lay::PS];
                } else {
                    v[q][r] = sm[Lay::addr(p, b)];
                }
            }
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
    if (!GIN) __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; q++) {
        const int u = threadIdx.x + q * NT;
        if (PER * NT == NBF || u < NBF) {
            const int b = Lay::BFAST ? u % NB : u / NJ;
            const int j = Lay::BFAST ? u / NB : u % NJ;
            const int k = j % Ns;
            const int d = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int o = d + r * Ns;
                if (GOUT) {
                    // last pass: o = j + r L/R; for an even radix o < L/2 exactly when r < R/2
                    const bool keep = !Dst::HALF || (R % 2 == 0 ? 2 * r < R : 2 * o < L);
                    if (keep) dst.template store<C>(b, o, v[q][r]);
                } else if constexpr (WSPLIT) {
                    sm[Lay::addr(d, b) + Lay::pidx(r * Ns) * Lay::PS] = v[q][r];
                } else {
                    sm[Lay::addr(o, b)] = v[q][r];
                }
            }
        }
    }
    if (!GOUT) __syncthreads();
}

// Passes q in [q, Q1) of the plan (reversed when REV); Ns is the product of
// the radices of the passes before q.
template <class C, int L, int NB, int NT, int DIR, class Lay, bool REV, int Q1, int q, int Ns, class Src, class Dst,
          int PLAN = 0>
__device__ __forceinline__ void stockham_range(C* sm, const C* tw, const Src& src, const Dst& dst) {
    if constexpr (q < Q1) {
        constexpr int R = plan_radix_dir(L, q, REV, PLAN);
        stockham_pass<C, L, R, Ns, NB, NT, DIR, Lay, Src, Dst>(sm, tw, src, dst);
        stockham_range<C, L, NB, NT, DIR, Lay, REV, Q1, q + 1, Ns * R, Src, Dst, PLAN>(sm, tw, src, dst);
    }
}

// Transform NB lines.  When the source is shared memory the caller must have
// synchronised after filling it; when the destination is shared memory the
// result may be read right after the call (the last pass ends in a barrier).
// The twiddle table must be resident before the second pass (the first pass
// uses none), so a caller may start filling it together with the first pass.
template <class C, int L, int NB, int NT, int DIR, class Lay, class Src = SmemIO, class Dst = SmemIO>
__device__ __forceinline__ void fft_tile(C* sm, const C* tw, const Src& src = Src(), const Dst& dst = Dst()) {
    static_assert(smooth235(L), "FFT length must be a product of 2, 3 and 5");
    stockham_range<C, L, NB, NT, DIR, Lay, false, plan_len(L), 0, 1, Src, Dst>(sm, tw, src, dst);
}

// shared-memory to shared-memory transform with lines fastest (LS >= NB)
template <class C, int L, int NB, int LS, int NT, int DIR>
__device__ __forceinline__ void tile_fft(C* sm, const C* tw) {
    fft_tile<C, L, NB, NT, DIR, Layout<LS, 1, true>>(sm, tw);
}

// copy the twiddle table for length L into shared memory
template <class C, int L, int NT>
__device__ __forceinline__ void load_twiddles(C* tws, const C* __restrict__ twg) {
    for (int j = threadIdx.x; j < L; j += NT) tws[j] = twg[j];
}

}  // namespace ifdda
