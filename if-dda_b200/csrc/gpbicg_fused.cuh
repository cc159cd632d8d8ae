// GPBiCG steps folded into the x passes of its two mat-vecs.
//
// One GPBiCG iteration (cdmlib/gpbicg.f:158-327) is, unfused, GpP, A p,
// GpAlpha, GpYT, A t, GpZeta, GpUpdate (krylov_kernels.cuh).  The vector
// updates that feed a mat-vec are done by its first x pass as it reads its
// input, and the dot products of a mat-vec's result by its last x pass as it
// writes it, so an iteration is A p, A t, GpUpdate: four kernels and four
// passes over the vectors fewer.  Every element is visited once by each x
// pass (isotropic or no polarisability; a full tensor keeps the unfused
// form), the arithmetic per element is that of the unfused ops, and the dot
// products are reduced in a fixed order over the x-pass grid, so results stay
// deterministic and independent of the batch.
#pragma once
#include "krylov_kernels.cuh"
#include "matvec_kernels.cuh"

namespace ifdda {

// label 100 (gpbicg.f:158-170) with label 40's w (gpbicg.f:318-324):
// p = r + beta (p - u); after the first iteration w = At + beta Ap.  The
// mat-vec input is the new p.
template <class T> struct PreGpP {
    static constexpr int ND = 0;
    Slots<T> V;
    const KState* S;
    cplx<T>*p, *w;
    const cplx<T>*r, *u, *at, *ap;
    double2 beta;
    bool upd_w;
    double2 acc[1];
    __device__ __forceinline__ void bind(const MvArgs<T>&, int rhs) {
        p = V.v(G_P, rhs);
        w = V.v(G_W, rhs);
        r = V.v(G_R, rhs);
        u = V.v(G_U, rhs);
        at = V.v(G_AT, rhs);
        ap = V.v(G_AP, rhs);
        beta = S[rhs].beta;
        upd_w = S[rhs].itno > 0;
    }
    template <class C> __device__ __forceinline__ C value(int e) {
        const C pc = from_d<C>(zadd(ldg(r, e), zmul(beta, zsub(ldg(p, e), ldg(u, e)))));
        p[e] = pc;
        if (upd_w) st(w, e, zadd(ldg(at, e), zmul(beta, ldg(ap, e))));
        return pc;
    }
};

// gpbicg.f:173-190 on the result Ap: r0^H Ap, then alpha = r0rn / r0^H Ap.
template <class T> struct EpiGpAlpha {
    static constexpr int ND = 1, NDP = 0;
    Slots<T> V;
    KState* S;
    int* status;
    const cplx<T>* r0;
    double2 acc[1];
    template <class U> __device__ __forceinline__ void bind(const MvArgs<U>&, int rhs) {
        r0 = V.v(G_R0, rhs);
        acc[0] = make_double2(0, 0);
    }
    template <class C> __device__ __forceinline__ void elem(int e, C y) {
        acc[0] = zadd(acc[0], zconjmul(ldg(r0, e), to_d(y)));
    }
    __device__ __forceinline__ void finish(int rhs, const double2* tot) {
        GpAlpha<T>{V, S}.finish(rhs, S[rhs], status[rhs], tot);
    }
};

// gpbicg.f:193-203 and the dots of gpbicg.f:236-243 that need y and t:
// y = t_old - r + alpha (Ap - w), t = r - alpha Ap, y^H y, y^H t.  The
// mat-vec input is the new t.
template <class T> struct PreGpYT {
    static constexpr int ND = 2;
    Slots<T> V;
    const KState* S;
    int tcur, tnew;
    const cplx<T>*t, *r, *ap, *w;
    cplx<T>*y, *tn;
    double2 alpha;
    double2 acc[2];
    __device__ __forceinline__ void bind(const MvArgs<T>&, int rhs) {
        t = V.v(tcur, rhs);
        r = V.v(G_R, rhs);
        ap = V.v(G_AP, rhs);
        w = V.v(G_W, rhs);
        y = V.v(G_Y, rhs);
        tn = V.v(tnew, rhs);
        alpha = S[rhs].alpha;
        acc[0] = acc[1] = make_double2(0, 0);
    }
    template <class C> __device__ __forceinline__ C value(int e) {
        const double2 rr = ldg(r, e), apv = ldg(ap, e);
        const double2 yv = zadd(zsub(ldg(t, e), rr), zmul(alpha, zsub(apv, ldg(w, e))));
        const double2 tv = zsub(rr, zmul(alpha, apv));
        st(y, e, yv);
        const C tc = from_d<C>(tv);
        tn[e] = tc;
        acc[0] = zadd(acc[0], zconjmul(yv, yv));
        acc[1] = zadd(acc[1], zconjmul(yv, tv));
        return tc;
    }
};

// label 30 (gpbicg.f:212-264) on the result At: At^H At, At^H y, At^H t, with
// y^H y and y^H t from the first x pass, then zeta and eta.
template <class T> struct EpiGpZeta {
    static constexpr int ND = 3, NDP = 2;
    Slots<T> V;
    KState* S;
    int* status;
    int tnew;
    int every2;  // GPBICG2 (see GpZeta)
    const cplx<T>*y, *t;
    double2 acc[3];
    template <class U> __device__ __forceinline__ void bind(const MvArgs<U>&, int rhs) {
        y = V.v(G_Y, rhs);
        t = V.v(tnew, rhs);
        acc[0] = acc[1] = acc[2] = make_double2(0, 0);
    }
    template <class C> __device__ __forceinline__ void elem(int e, C atc) {
        const double2 a = to_d(atc);
        acc[0] = zadd(acc[0], zconjmul(a, a));
        acc[1] = zadd(acc[1], zconjmul(a, ldg(y, e)));
        acc[2] = zadd(acc[2], zconjmul(a, ldg(t, e)));
    }
    __device__ __forceinline__ void finish(int rhs, const double2* tot) {
        KState& s = S[rhs];
        s.c2 = tot[3];
        s.c5 = tot[4];
        GpZeta<T>{V, S, tnew, every2}.finish(rhs, s, status[rhs], tot);
    }
};

}  // namespace ifdda
