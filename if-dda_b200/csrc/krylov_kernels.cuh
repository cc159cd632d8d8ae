// Device-resident Krylov solvers: GPBiCG (cdmlib/gpbicg.f:81-338) and
// QMR-BiCGSTAB (cdmlib/qmrbicgstab.f:1-253), batched over right-hand sides.
//
// The reference runs each solver as a reverse-communication state machine
// that returns to its driver for every mat-vec (cdmlib/inverserigopt.f:42-107).
// Here the same update sequence is split into a few fused vector kernels
// around the two mat-vecs of an iteration; every dot product is a
// deterministic two-stage reduction whose last block evaluates the scalar
// recurrence (alpha, zeta/eta, beta, omega, tau ...) on the device and writes
// the per-RHS status (0 running, 1 done, -1 breakdown, with STEPERR as the
// reference numbers it).  Kernels of a finished right-hand side return at
// once, so the host may launch iterations ahead and check the status only now
// and then.  Vectors may be FP32 or FP64 complex; scalars and sums are FP64.
#pragma once
#include "matvec_kernels.cuh"  // ALPHA_* modes of the transposed product
#include "reduce.cuh"

namespace ifdda {

struct KState {
    // GPBiCG
    double2 alpha, beta, eta, dzeta, r0rn, c2, c5;
    // QMR-BiCGSTAB
    double2 rho, omega, tau, taut, theta, thetat, etaq, etat, f1, qbeta;
    // CORS, GPBiCOR: rho of the previous iteration
    double2 rhoa;
    double norm, residu, tol;
    int itno, steperr, maxit, conv;
    int atmax;  // TFQMR, GPBiCGAR: stopped past MAXIT, after the pass's last product
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 zconjmul(double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 zsqrt(double2 z) {
    // principal square root
    const double r = hypot(z.x, z.y);
    if (r == 0.0) return make_double2(0, 0);
    if (z.x >= 0) {
        const double t = sqrt(0.5 * (r + z.x));
        return make_double2(t, z.y / (2 * t));
    }
    const double t = sqrt(0.5 * (r - z.x));
    return make_double2(fabs(z.y) / (2 * t), copysign(t, z.y));
}

// vector slots of one solver workspace: slot s of rhs r at base + (s*nrhs + r)*n3
template <class T> struct Slots {
    cplx<T>* base;
    long n3;
    int nrhs;
    __host__ __device__ __forceinline__ cplx<T>* v(int s, int r) const { return base + ((long)s * nrhs + r) * n3; }
};

template <class C> __device__ __forceinline__ double2 ld(const C* p, long i) { return to_d(p[i]); }
// The same through the read-only path.  For vectors that a kernel reads at an
// element before (or without) writing that element from the same thread: the
// loads may then be issued ahead of the stores to other elements, instead of
// waiting behind them for want of alias information.
template <class C> __device__ __forceinline__ double2 ldg(const C* p, long i) { return to_d(__ldg(p + i)); }
template <class C> __device__ __forceinline__ void st(C* p, long i, double2 v) { p[i] = from_d<C>(v); }

constexpr int KNT = 256;

// Generic fused vector kernel: op.elem() per element, then ND sums reduced and
// handed to op.finish() in one block.
template <int ND, class Op>
__global__ void __launch_bounds__(KNT) k_vec(const Op op, long n3, int nblk, RedSlots rs, int* __restrict__ status) {
    const int rhs = blockIdx.y;
    pdl_trigger();
    pdl_wait();
    if (status[rhs]) return;
    double2 acc[ND > 0 ? ND : 1];
#pragma unroll
    for (int m = 0; m < (ND > 0 ? ND : 1); m++) acc[m] = make_double2(0, 0);
    const KState s = op.stt[rhs];
    for (long i = (long)blockIdx.x * KNT + threadIdx.x; i < n3; i += (long)nblk * KNT) op.elem(s, rhs, i, acc);
    if constexpr (ND > 0) {
        if (reduce_across_blocks<KNT, ND>(acc, rhs, blockIdx.x, nblk, rs) && threadIdx.x == 0)
            op.finish(rhs, op.stt[rhs], status[rhs], acc);
    }
}

// ---------------------------------------------------------------- GPBiCG ----
// slots: 0 r0, 1 p, 2 r, 3 y, 4/5 t (two buffers, alternate), 6 Ap, 7 At,
//        8 u, 9 w, 10 z, 11 x, 12 xr (mat-vec out), 13 b
enum { G_R0 = 0, G_P, G_R, G_Y, G_TA, G_TB, G_AP, G_AT, G_U, G_W, G_Z, G_X, G_XR, G_B, G_NSLOT };

// start: x = b (initial guess FF0, inverserigopt.f:34-40) or 0; NORM = ||b|| (gpbicg.f:116-127)
template <class T> struct GpStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(G_B, r), i);
        st(V.v(G_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(G_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
        (void)status;
    }
};

// label 10 (gpbicg.f:132-150): r = b - A x0, r0 = r, p = t = w = u = z = 0
template <class T> struct GpInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = zsub(ld(V.v(G_B, r), i), ld(V.v(G_XR, r), i));
        const double2 z = make_double2(0, 0);
        st(V.v(G_R, r), i, rr);
        st(V.v(G_R0, r), i, rr);
        st(V.v(G_P, r), i, z);
        st(V.v(G_TA, r), i, z);
        st(V.v(G_W, r), i, z);
        st(V.v(G_U, r), i, z);
        st(V.v(G_Z, r), i, z);
        acc[0] = zadd(acc[0], zconjmul(rr, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.r0rn = a[0];
        s.beta = make_double2(0, 0);
        s.itno = 0;
    }
};

// label 100 (gpbicg.f:158-170), preceded by label 40's w update (gpbicg.f:318-324)
template <class T> struct GpP {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 p = ld(V.v(G_P, r), i), u = ld(V.v(G_U, r), i), rr = ld(V.v(G_R, r), i);
        st(V.v(G_P, r), i, zadd(rr, zmul(s.beta, zsub(p, u))));
        if (s.itno > 0) st(V.v(G_W, r), i, zadd(ld(V.v(G_AT, r), i), zmul(s.beta, ld(V.v(G_AP, r), i))));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 20 (gpbicg.f:173-190): alpha = r0rn / (r0^H Ap)
template <class T> struct GpAlpha {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(G_R0, r), i), ld(V.v(G_AP, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zisnull(a[0])) {
            status = -1;
            s.steperr = 1;
            return;
        }
        s.alpha = zdiv(s.r0rn, a[0]);
    }
};

// gpbicg.f:193-203: y = t - r + alpha (Ap - w), t_old = t, t = r - alpha Ap;
// also the two dots of gpbicg.f:236-243 that need only y and t
template <class T> struct GpYT {
    Slots<T> V;
    KState* stt;
    int tcur, tnew;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 t = ld(V.v(tcur, r), i), rr = ld(V.v(G_R, r), i), ap = ld(V.v(G_AP, r), i),
                      w = ld(V.v(G_W, r), i);
        const double2 y = zadd(zsub(t, rr), zmul(s.alpha, zsub(ap, w)));
        const double2 tn = zsub(rr, zmul(s.alpha, ap));
        st(V.v(G_Y, r), i, y);
        st(V.v(tnew, r), i, tn);
        acc[0] = zadd(acc[0], zconjmul(y, y));
        acc[1] = zadd(acc[1], zconjmul(y, tn));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.c2 = a[0];
        s.c5 = a[1];
    }
};

// label 30 coefficients (gpbicg.f:212-264).  every2: GPBICG2
// (cdmlib/gpbicg2.f), which takes the zeta-only step on every even ITNO, not
// only the first (its label 30 tests mod(ITNO,2) = 0).
template <class T> struct GpZeta {
    Slots<T> V;
    KState* stt;
    int tnew;
    int every2;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 at = ld(V.v(G_AT, r), i), y = ld(V.v(G_Y, r), i), t = ld(V.v(tnew, r), i);
        acc[0] = zadd(acc[0], zconjmul(at, at));
        acc[1] = zadd(acc[1], zconjmul(at, y));
        acc[2] = zadd(acc[2], zconjmul(at, t));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        const double2 c1 = a[0], c3 = a[1], c4 = a[2], c2 = s.c2, c5 = s.c5;
        if (every2 ? s.itno % 2 == 0 : s.itno == 0) {
            s.eta = make_double2(0, 0);
            if (zisnull(c1)) {
                status = -1;
                s.steperr = 2;
                return;
            }
            s.dzeta = zdiv(c4, c1);
        } else {
            const double2 c = zsub(zmul(c1, c2), zmul(c3, zconj(c3)));
            if (zisnull(c)) {
                status = -1;
                s.steperr = 3;
                return;
            }
            s.dzeta = zdiv(zsub(zmul(c2, c4), zmul(c5, c3)), c);
            s.eta = zdiv(zsub(zmul(c1, c5), zmul(zconj(c3), c4)), c);
        }
    }
};

// gpbicg.f:268-296 and label 40 (gpbicg.f:300-327): u, z, x, r, residual, beta
template <class T> struct GpUpdate {
    Slots<T> V;
    KState* stt;
    int tcur, tnew;  // tcur = t_old after GpYT
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 ap = ldg(V.v(G_AP, r), i), told = ldg(V.v(tcur, r), i), rr = ldg(V.v(G_R, r), i);
        const double2 u0 = ldg(V.v(G_U, r), i), z0 = ldg(V.v(G_Z, r), i);
        const double2 u = zadd(zmul(s.dzeta, ap), zmul(s.eta, zadd(zsub(told, rr), zmul(s.beta, u0))));
        const double2 z = zsub(zadd(zmul(s.dzeta, rr), zmul(s.eta, z0)), zmul(s.alpha, u));
        const double2 x = zadd(zadd(ldg(V.v(G_X, r), i), zmul(s.alpha, ldg(V.v(G_P, r), i))), z);
        const double2 rn = zsub(zsub(ldg(V.v(tnew, r), i), zmul(s.eta, ldg(V.v(G_Y, r), i))),
                                zmul(s.dzeta, ldg(V.v(G_AT, r), i)));
        st(V.v(G_U, r), i, u);
        st(V.v(G_Z, r), i, z);
        st(V.v(G_X, r), i, x);
        st(V.v(G_R, r), i, rn);
        acc[0].x += rn.x * rn.x + rn.y * rn.y;
        acc[1] = zadd(acc[1], zconjmul(ldg(V.v(G_R0, r), i), rn));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
            return;
        }
        if (zisnull(s.r0rn)) {
            status = -1;
            s.steperr = 4;
            return;
        }
        s.beta = zdiv(zdiv(zmul(s.alpha, a[1]), s.dzeta), s.r0rn);
        s.r0rn = a[1];
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            status = 1;
            s.steperr = 0;
        }
    }
};

// ---------------------------------------------------------- QMR-BiCGSTAB ----
// slots: 0 r, 1 p, 2 v, 3 d, 4 rtilde, 5 s, 6 t, 7 x, 8 xr, 9 b
enum { Q_R = 0, Q_P, Q_V, Q_D, Q_RT, Q_S, Q_T, Q_X, Q_XR, Q_B, Q_NSLOT };

template <class T> struct QStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(Q_B, r), i);
        st(V.v(Q_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(Q_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
        s.conv = 0;
    }
};

// label 10 (qmrbicgstab.f:49-71) and the rho/beta of the first label 100
template <class T> struct QInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = zsub(ld(V.v(Q_B, r), i), ld(V.v(Q_XR, r), i));
        const double2 z = make_double2(0, 0);
        st(V.v(Q_R, r), i, rr);
        st(V.v(Q_P, r), i, z);
        st(V.v(Q_V, r), i, z);
        st(V.v(Q_D, r), i, z);
        st(V.v(Q_RT, r), i, rr);
        acc[0] = zadd(acc[0], zconjmul(rr, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        const double2 one = make_double2(1, 0);
        s.alpha = one;
        s.omega = one;
        s.tau = zsqrt(a[0]);
        s.theta = make_double2(0, 0);
        s.etaq = make_double2(0, 0);
        // first pass of label 100: rho0 = 1, rho = rtilde^H r = r^H r
        s.rho = a[0];
        s.qbeta = zdiv(zmul(s.rho, s.alpha), s.omega);
        s.itno = 1;
    }
};

// p = r + beta (p - omega v)   (qmrbicgstab.f:88-97)
template <class T> struct QP {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 p = ld(V.v(Q_P, r), i), v = ld(V.v(Q_V, r), i), rr = ld(V.v(Q_R, r), i);
        st(V.v(Q_P, r), i, zadd(rr, zmul(s.qbeta, zsub(p, zmul(s.omega, v)))));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 20 (qmrbicgstab.f:101-115): alpha = rho / (rtilde^H v)
template <class T> struct QAlpha {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(Q_RT, r), i), ld(V.v(Q_V, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zabs(a[0]) == 0.0) {
            status = -1;
            s.steperr = 1;
            return;
        }
        s.alpha = zdiv(s.rho, a[0]);
    }
};

// qmrbicgstab.f:118-151: s = r - alpha v, thetat, c, taut, etat
template <class T> struct QS {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 sv = zsub(ld(V.v(Q_R, r), i), zmul(s.alpha, ld(V.v(Q_V, r), i)));
        st(V.v(Q_S, r), i, sv);
        acc[0] = zadd(acc[0], zconjmul(sv, sv));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zabs(s.tau) == 0.0) {
            status = -1;
            s.steperr = 2;
            return;
        }
        const double2 one = make_double2(1, 0);
        s.thetat = zdiv(zsqrt(a[0]), s.tau);
        const double2 c = zdiv(one, zsqrt(zadd(one, zmul(s.thetat, s.thetat))));
        s.taut = zmul(zmul(s.tau, s.thetat), c);
        s.etat = zmul(zmul(c, c), s.alpha);
        // dtilde = p + (theta^2 eta / alpha) d  (qmrbicgstab.f:146)
        s.f1 = zdiv(zmul(zmul(s.theta, s.theta), s.etaq), s.alpha);
    }
};

// label 30 (qmrbicgstab.f:155-185): omega
template <class T> struct QOmega {
    Slots<T> V;
    KState* stt;
    int methode;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 t = ld(V.v(Q_T, r), i), sv = ld(V.v(Q_S, r), i);
        if (methode == 1) {
            acc[0] = zadd(acc[0], zconjmul(t, t));
            acc[1] = zadd(acc[1], zconjmul(sv, t));
        } else {
            acc[0] = zadd(acc[0], zconjmul(sv, t));
            acc[1] = zadd(acc[1], zconjmul(sv, sv));
        }
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zabs(a[0]) == 0.0) {
            status = -1;
            s.steperr = 3;
            return;
        }
        s.omega = zdiv(a[1], a[0]);
    }
};

// qmrbicgstab.f:192-226: r = s - omega t, theta, c, tau, eta, and the next
// iteration's rho and beta (label 100) from the new r
template <class T> struct QR {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 rn = zsub(ld(V.v(Q_S, r), i), zmul(s.omega, ld(V.v(Q_T, r), i)));
        st(V.v(Q_R, r), i, rn);
        acc[0] = zadd(acc[0], zconjmul(rn, rn));
        acc[1] = zadd(acc[1], zconjmul(ld(V.v(Q_RT, r), i), rn));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zabs(s.taut) == 0.0) {
            status = -1;
            s.steperr = 4;
            return;
        }
        const double2 one = make_double2(1, 0);
        s.theta = zdiv(zsqrt(a[0]), s.taut);
        const double2 c = zdiv(one, zsqrt(zadd(one, zmul(s.theta, s.theta))));
        s.tau = zmul(zmul(s.taut, s.theta), c);
        s.etaq = zmul(zmul(c, c), s.omega);
        if (zabs(s.omega) == 0.0) {
            status = -1;
            s.steperr = 5;
            return;
        }
        s.residu = sqrt((double)(s.itno + 1)) * zabs(s.tau) / s.norm;
        s.conv = s.residu <= s.tol ? 1 : 0;
        // next label 100: rho0 = rho, rho = rtilde^H r, beta = rho alpha / rho0 / omega
        const double2 rho0 = s.rho;
        s.rho = a[1];
        s.qbeta = zdiv(zdiv(zmul(s.rho, s.alpha), rho0), s.omega);
    }
};

// qmrbicgstab.f:146-148 and 209-213 (dtilde, xtilde recomputed on the fly):
//   dt = p + f1 d, xt = x + etat dt, d = s + (thetat^2 etat / omega) dt, x = xt + eta d
// then the stop test (qmrbicgstab.f:216-224) or the next iteration.
template <class T> struct QX {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 f2 = zdiv(zmul(zmul(s.thetat, s.thetat), s.etat), s.omega);
        const double2 dt = zadd(ld(V.v(Q_P, r), i), zmul(s.f1, ld(V.v(Q_D, r), i)));
        const double2 xt = zadd(ld(V.v(Q_X, r), i), zmul(s.etat, dt));
        const double2 d = zadd(ld(V.v(Q_S, r), i), zmul(f2, dt));
        st(V.v(Q_D, r), i, d);
        st(V.v(Q_X, r), i, zadd(xt, zmul(s.etaq, d)));
        (void)acc;
    }
    __device__ void finish(int, KState& s, int& status, const double2*) const {
        if (s.conv) {
            status = 1;
            s.steperr = 0;
            return;
        }
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            status = 1;
            s.steperr = 0;
        }
    }
};

// -------------------------------------------------------------- BiCGSTAB ----
// cdmlib/pimzbicgstab.f:1-216 as the reference writes it: NORM is the SQUARED
// norm of the initial residual, rho = r^H r, the loop stops when
// ||r||^2 / NORM <= tol / 10, and ITNO > MAXIT, a zero denominator or
// ||s|| < 1e-15 (soft breakdown: x = p, done by the host) end it with an
// error status.  KState: alpha, beta, omega, rho; itno = ITNO.
// slots: 0 r, 1 rtilde, 2 p, 3 v = A p, 4 s, 5 t = A s, 6 x, 7 xr (mat-vec out), 8 b
enum { B_R = 0, B_RT, B_P, B_V, B_S, B_T, B_X, B_XR, B_B, B_NSLOT };

// x = x0 (FF0) or 0 (pimzbicgstab.f:40-47)
template <class T> struct BStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2*) const {
        st(V.v(B_X, r), i, zero_guess ? make_double2(0, 0) : ld(V.v(B_B, r), i));
        if (zero_guess) st(V.v(B_XR, r), i, make_double2(0, 0));
    }
    __device__ void finish(int, KState& s, int&, const double2*) const {
        s.steperr = -1;
        s.itno = 0;
    }
};

// label 10 (pimzbicgstab.f:52-72) and the first pass of label 100
// (:76-97): r = b - A x0, rtilde = r, p = v = 0, NORM = ||r||^2,
// rho = alpha = omega = 1, then ITNO = 1, rho = r^H r, beta = rho
template <class T> struct BInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = zsub(ld(V.v(B_B, r), i), ld(V.v(B_XR, r), i));
        const double2 z = make_double2(0, 0);
        st(V.v(B_R, r), i, rr);
        st(V.v(B_RT, r), i, rr);
        st(V.v(B_P, r), i, z);
        st(V.v(B_V, r), i, z);
        acc[0].x += rr.x * rr.x + rr.y * rr.y;
        acc[1] = zadd(acc[1], zconjmul(rr, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = a[0].x;
        s.alpha = make_double2(1, 0);
        s.omega = make_double2(1, 0);
        s.itno = 1;
        s.rho = a[1];
        s.beta = s.rho;  // rho alpha / (rho0 omega) with rho0 = alpha = omega = 1
    }
};

// pimzbicgstab.f:100-110: p = r + beta (p - omega v)
template <class T> struct BP {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 q = zsub(ld(V.v(B_P, r), i), zmul(s.omega, ld(V.v(B_V, r), i)));
        st(V.v(B_P, r), i, zadd(ld(V.v(B_R, r), i), zmul(s.beta, q)));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 20 (pimzbicgstab.f:114-131): xi = rtilde^H v, alpha = rho / xi
template <class T> struct BXi {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(B_RT, r), i), ld(V.v(B_V, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zisnull(a[0])) {
            status = -1;
            s.steperr = 10;
            return;
        }
        s.alpha = zdiv(s.rho, a[0]);
    }
};

// pimzbicgstab.f:133-157: s = r - alpha v, soft breakdown when ||s|| < 1e-15
template <class T> struct BS {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 sv = zsub(ld(V.v(B_R, r), i), zmul(s.alpha, ld(V.v(B_V, r), i)));
        st(V.v(B_S, r), i, sv);
        acc[0] = zadd(acc[0], zconjmul(sv, sv));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        const double2 k = zsqrt(a[0]);
        if (hypot(k.x, k.y) < 1e-15) {
            status = -1;
            s.steperr = 12;
        }
    }
};

// label 30 (pimzbicgstab.f:169-186): omega = t^H s / t^H t
template <class T> struct BOmega {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 t = ld(V.v(B_T, r), i);
        acc[0] = zadd(acc[0], zconjmul(t, t));
        acc[1] = zadd(acc[1], zconjmul(t, ld(V.v(B_S, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zisnull(a[0])) {
            status = -1;
            s.steperr = 14;
            return;
        }
        s.omega = zdiv(a[1], a[0]);
    }
};

// pimzbicgstab.f:188-211: x += alpha p + omega s, r = s - omega t, the stop
// test, then the next pass of label 100: rho0 = rho, rho = r^H r,
// beta = rho alpha / (rho0 omega)
template <class T> struct BUpdate {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 sv = ld(V.v(B_S, r), i);
        st(V.v(B_X, r), i,
           zadd(zadd(ld(V.v(B_X, r), i), zmul(s.alpha, ld(V.v(B_P, r), i))), zmul(s.omega, sv)));
        const double2 rn = zsub(sv, zmul(s.omega, ld(V.v(B_T, r), i)));
        st(V.v(B_R, r), i, rn);
        acc[0] = zadd(acc[0], zconjmul(rn, rn));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        const double2 c = make_double2(a[0].x / s.norm, a[0].y / s.norm);
        s.residu = hypot(c.x, c.y);
        if (s.itno > s.maxit) {
            status = -1;
            s.steperr = 0;
            s.itno = s.maxit;
            return;
        }
        if (hypot(c.x, c.y) <= s.tol / 10.0) {
            status = 1;
            s.steperr = 0;
            return;
        }
        s.itno += 1;
        const double2 rho0 = s.rho;
        s.rho = a[0];
        const double2 kappa = zmul(rho0, s.omega);
        if (zisnull(kappa)) {
            status = -1;
            s.steperr = 6;
            return;
        }
        s.beta = zdiv(zmul(s.rho, s.alpha), kappa);
    }
};

// ---------------------------------------------------------------- ZCG ----
// Conjugate gradient for complex-symmetric systems (unconjugated dot
// products), cdmlib/zcg.f:1-179: one mat-vec per iteration, w = A p carried
// by w = A r + beta w.  NORM = ||b||; the loop stops when ||r|| / NORM <= tol;
// NLOOP >= MAXIT and p^T A p = 0 (where the reference stops the program) end
// it with an error status.  KState: alpha, beta, rho = rho0, c2 = xi;
// itno = NLOOP.
// slots: 0 x, 1 r, 2 p, 3 s = A r, 4 w, 5 xr (mat-vec out), 6 b
enum { C_X = 0, C_R, C_P, C_S, C_W, C_XR, C_B, C_NSLOT };

template <class T> struct CStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2*) const {
        st(V.v(C_X, r), i, zero_guess ? make_double2(0, 0) : ld(V.v(C_B, r), i));
        if (zero_guess) st(V.v(C_XR, r), i, make_double2(0, 0));
    }
    __device__ void finish(int, KState& s, int&, const double2*) const {
        s.steperr = -1;
        s.itno = 0;
    }
};

// label 10 (zcg.f:45-64): r = b - A x0, p = r, NORM = ||b||, rho0 = r^T r
template <class T> struct CInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(C_B, r), i);
        const double2 rr = zsub(b, ld(V.v(C_XR, r), i));
        st(V.v(C_R, r), i, rr);
        st(V.v(C_P, r), i, rr);
        acc[0].x += b.x * b.x + b.y * b.y;
        acc[1] = zadd(acc[1], zmul(rr, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.rho = a[1];
        s.itno = 0;
    }
};

// next pass of label 50 (zcg.f:74-85): NLOOP += 1, the iteration limit, alpha
__device__ __forceinline__ void cg_next(KState& s, int& status) {
    s.itno += 1;
    if (s.itno >= s.maxit) {
        status = -1;
        s.steperr = 0;
        return;
    }
    s.alpha = zdiv(s.rho, s.c2);
}

// label 20 (zcg.f:66-73): xi = p^T w with w = A p, then label 50
template <class T> struct CXi {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zmul(ld(V.v(C_P, r), i), ld(V.v(C_W, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.c2 = a[0];
        if (a[0].x == 0.0 && a[0].y == 0.0) {
            status = -1;
            s.steperr = 3;
            return;
        }
        cg_next(s, status);
    }
};

// zcg.f:154-157 (after the first iteration: p = r + beta p, w = s + beta w),
// then zcg.f:89-110: x += alpha p, r -= alpha w, stop when ||r||/NORM <= tol
template <class T> struct CUpdate {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        double2 p = ld(V.v(C_P, r), i), w = ld(V.v(C_W, r), i);
        const double2 rr = ld(V.v(C_R, r), i);
        if (s.itno > 1) {
            p = zadd(rr, zmul(s.beta, p));
            w = zadd(ld(V.v(C_S, r), i), zmul(s.beta, w));
            st(V.v(C_P, r), i, p);
            st(V.v(C_W, r), i, w);
        }
        st(V.v(C_X, r), i, zadd(ld(V.v(C_X, r), i), zmul(s.alpha, p)));
        const double2 rn = zsub(rr, zmul(s.alpha, w));
        st(V.v(C_R, r), i, rn);
        acc[0].x += rn.x * rn.x + rn.y * rn.y;
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
        }
    }
};

// label 30 (zcg.f:139-160): rho = r^T r, delta = r^T s, beta = rho / rho0,
// xi = delta - beta^2 xi, then label 50
template <class T> struct CBeta {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = ld(V.v(C_R, r), i);
        acc[0] = zadd(acc[0], zmul(rr, rr));
        acc[1] = zadd(acc[1], zmul(rr, ld(V.v(C_S, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.beta = zdiv(a[0], s.rho);
        s.rho = a[0];
        s.c2 = zsub(a[1], zmul(zmul(s.beta, s.beta), s.c2));
        cg_next(s, status);
    }
};

// ------------------------------------------------------------ GPBiCGsafe ----
// cdmlib/gpbicgsafe.f: the mat-vecs are A r and A u; A p is carried by
// Ap = Ar + beta (Ap - Au); zeta and eta come from five dot products.  Ends
// like GPBICG (status 1 with the iterate past MAXIT).  KState: alpha, beta,
// eta, dzeta, r0rn; itno = ITNO.
// slots: 0 r0 (shadow), 1 p, 2 u, 3 r, 4 A u, 5 A r, 6 A p, 7 z, 8 y, 9 x,
//        10 xr (mat-vec out), 11 b
enum { S_R0 = 0, S_P, S_U, S_R, S_AU, S_AR, S_AP, S_Z, S_Y, S_X, S_XR, S_B, S_NSLOT };

template <class T> struct SfStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(S_B, r), i);
        st(V.v(S_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(S_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
    }
};

// label 10: r0 = r = b - A x0, p = u = z = Ap = Au = y = 0, R0RN = r0^H r0
template <class T> struct SfInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = zsub(ld(V.v(S_B, r), i), ld(V.v(S_XR, r), i));
        const double2 z = make_double2(0, 0);
        st(V.v(S_R0, r), i, rr);
        st(V.v(S_R, r), i, rr);
        st(V.v(S_P, r), i, z);
        st(V.v(S_U, r), i, z);
        st(V.v(S_Z, r), i, z);
        st(V.v(S_AP, r), i, z);
        st(V.v(S_AU, r), i, z);
        st(V.v(S_Y, r), i, z);
        acc[0] = zadd(acc[0], zconjmul(rr, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.r0rn = a[0];
        s.beta = make_double2(0, 0);
        s.itno = 0;
    }
};

// label 100: p = r + beta (p - u); then A r
template <class T> struct SfP {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 p = ld(V.v(S_P, r), i), u = ld(V.v(S_U, r), i);
        st(V.v(S_P, r), i, zadd(ld(V.v(S_R, r), i), zmul(s.beta, zsub(p, u))));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 20: Ap = Ar + beta (Ap - Au), alpha = R0RN / r0^H Ap, zeta and eta
// (first iteration: zeta = Ar^H r / Ar^H Ar, eta = 0).  plus: GPBICGplus
// (cdmlib/gpbicgplus.f), the same iteration with zeta and eta written from
// the same five dot products in its own form.
template <class T> struct SfAlpha {
    Slots<T> V;
    KState* stt;
    int plus;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 ar = ld(V.v(S_AR, r), i), y = ld(V.v(S_Y, r), i), rr = ld(V.v(S_R, r), i);
        const double2 ap = zadd(ar, zmul(s.beta, zsub(ld(V.v(S_AP, r), i), ld(V.v(S_AU, r), i))));
        st(V.v(S_AP, r), i, ap);
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(S_R0, r), i), ap));
        acc[1] = zadd(acc[1], zconjmul(y, y));
        acc[2] = zadd(acc[2], zconjmul(ar, rr));
        acc[3] = zadd(acc[3], zconjmul(y, rr));
        acc[4] = zadd(acc[4], zconjmul(ar, y));
        acc[5] = zadd(acc[5], zconjmul(ar, ar));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zisnull(a[0])) {
            status = -1;
            s.steperr = 1;
            return;
        }
        s.alpha = zdiv(s.r0rn, a[0]);
        const double2 c1 = a[1], c2 = a[2], c3 = a[3], c4 = a[4], c5 = a[5];
        if (s.itno == 0) {
            s.eta = make_double2(0, 0);
            if (zisnull(c5)) {
                status = -1;
                s.steperr = 2;
                return;
            }
            s.dzeta = zdiv(c2, c5);
        } else if (plus) {
            // gpbicgplus.f names: y^H y, Ar^H Ar, Ar^H r, y^H r, y^H Ar
            const double2 p1 = c1, p2 = c5, p3 = c2, p4 = c3, p5 = zconj(c4);
            const double2 c = zsub(zmul(p1, p2), zmul(p5, zconj(p5)));
            if (zisnull(c)) {
                status = -1;
                s.steperr = 3;
                return;
            }
            s.dzeta = zdiv(zsub(zmul(p1, p3), zmul(p4, zconj(p5))), c);
            s.eta = zdiv(zsub(zmul(p2, p4), zmul(p5, p3)), c);
        } else {
            const double2 c = zsub(zmul(c5, c1), zmul(c4, zconj(c4)));
            if (zisnull(c)) {
                status = -1;
                s.steperr = 3;
                return;
            }
            s.dzeta = zdiv(zsub(zmul(c1, c2), zmul(c3, c4)), c);
            s.eta = zdiv(zsub(zmul(c5, c3), zmul(zconj(c4), c2)), c);
        }
    }
};

// u = zeta Ap + eta (y + beta u); then A u
template <class T> struct SfU {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 u = ld(V.v(S_U, r), i);
        st(V.v(S_U, r), i,
           zadd(zmul(s.dzeta, ld(V.v(S_AP, r), i)), zmul(s.eta, zadd(ld(V.v(S_Y, r), i), zmul(s.beta, u)))));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 30 and 40: t = r - alpha Ap, z, y, x += alpha p + z, r = t - y, the
// stop test on ||r|| / NORM, beta = alpha r0^H r / zeta / R0RN
template <class T> struct SfUpdate {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 rr = ld(V.v(S_R, r), i);
        const double2 t = zsub(rr, zmul(s.alpha, ld(V.v(S_AP, r), i)));
        const double2 z = zsub(zadd(zmul(s.dzeta, rr), zmul(s.eta, ld(V.v(S_Z, r), i))), zmul(s.alpha, ld(V.v(S_U, r), i)));
        const double2 y = zsub(zadd(zmul(s.dzeta, ld(V.v(S_AR, r), i)), zmul(s.eta, ld(V.v(S_Y, r), i))),
                               zmul(s.alpha, ld(V.v(S_AU, r), i)));
        st(V.v(S_Z, r), i, z);
        st(V.v(S_Y, r), i, y);
        st(V.v(S_X, r), i, zadd(zadd(ld(V.v(S_X, r), i), zmul(s.alpha, ld(V.v(S_P, r), i))), z));
        const double2 rn = zsub(t, y);
        st(V.v(S_R, r), i, rn);
        acc[0].x += rn.x * rn.x + rn.y * rn.y;
        acc[1] = zadd(acc[1], zconjmul(ld(V.v(S_R0, r), i), rn));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
            return;
        }
        if (zisnull(s.r0rn)) {
            status = -1;
            s.steperr = 4;
            return;
        }
        s.beta = zdiv(zdiv(zmul(s.alpha, a[1]), s.dzeta), s.r0rn);
        s.r0rn = a[1];
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            status = 1;
            s.steperr = 0;
        }
    }
};

// -------------------------------------------------------------- GPBiCG-AR ----
// cdmlib/gpbicgar.f (associate residual): mat-vecs A u then A r, A p carried
// by Ap = Ar + beta (Ap - Au), zeta and eta from the same five dot products as
// GPBiCGsafe (SfAlpha), u = zeta Ap + eta (t - r + beta u).  'GPBICGAR2'
// lands here too (the reference tests the 8-character prefix first).
// slots: 0 r0, 1 p, 2 r, 3 t, 4 z, 5 A p, 6 A r, 7 u, 8 y, 9 x, 10 A u,
//        11 xr (mat-vec out), 12 b
enum { A_R0 = 0, A_P, A_R, A_T, A_Z, A_AP, A_AR, A_U, A_Y, A_X, A_AU, A_XR, A_B, A_NSLOT };

template <class T> struct ArStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(A_B, r), i);
        st(V.v(A_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(A_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
        s.atmax = 0;
    }
};

// label 10: r0 = r = b - A x0, R0RN = r0^H r0 (the other vectors start at 0);
// then A r, and label 20: beta = 0
template <class T> struct ArInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = zsub(ld(V.v(A_B, r), i), ld(V.v(A_XR, r), i));
        const double2 z = make_double2(0, 0);
        st(V.v(A_R0, r), i, rr);
        st(V.v(A_R, r), i, rr);
        st(V.v(A_P, r), i, z);
        st(V.v(A_U, r), i, z);
        st(V.v(A_AP, r), i, z);
        st(V.v(A_AU, r), i, z);
        st(V.v(A_T, r), i, z);
        st(V.v(A_Z, r), i, z);
        st(V.v(A_Y, r), i, z);
        acc[0] = zadd(acc[0], zconjmul(rr, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.r0rn = a[0];
        s.beta = make_double2(0, 0);
        s.itno = 0;
    }
};

// label 100: p = r + beta (p - u), Ap = Ar + beta (Ap - Au), alpha, zeta, eta
template <class T> struct ArAlpha {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 ar = ld(V.v(A_AR, r), i), y = ld(V.v(A_Y, r), i), rr = ld(V.v(A_R, r), i);
        st(V.v(A_P, r), i, zadd(rr, zmul(s.beta, zsub(ld(V.v(A_P, r), i), ld(V.v(A_U, r), i)))));
        const double2 ap = zadd(ar, zmul(s.beta, zsub(ld(V.v(A_AP, r), i), ld(V.v(A_AU, r), i))));
        st(V.v(A_AP, r), i, ap);
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(A_R0, r), i), ap));
        acc[1] = zadd(acc[1], zconjmul(y, y));
        acc[2] = zadd(acc[2], zconjmul(ar, rr));
        acc[3] = zadd(acc[3], zconjmul(y, rr));
        acc[4] = zadd(acc[4], zconjmul(ar, y));
        acc[5] = zadd(acc[5], zconjmul(ar, ar));
    }
    __device__ void finish(int rhs, KState& s, int& status, const double2* a) const {
        SfAlpha<T>{V, stt, 0}.finish(rhs, s, status, a);
    }
};

// u = zeta Ap + eta (t - r + beta u); then A u
template <class T> struct ArU {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 q = zadd(zsub(ld(V.v(A_T, r), i), ld(V.v(A_R, r), i)), zmul(s.beta, ld(V.v(A_U, r), i)));
        st(V.v(A_U, r), i, zadd(zmul(s.dzeta, ld(V.v(A_AP, r), i)), zmul(s.eta, q)));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 40: t, z, y, x, r = t - y and the stop test; then A r
template <class T> struct ArUpdate {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 rr = ld(V.v(A_R, r), i);
        const double2 t = zsub(rr, zmul(s.alpha, ld(V.v(A_AP, r), i)));
        const double2 z = zsub(zadd(zmul(s.dzeta, rr), zmul(s.eta, ld(V.v(A_Z, r), i))), zmul(s.alpha, ld(V.v(A_U, r), i)));
        const double2 y = zsub(zadd(zmul(s.dzeta, ld(V.v(A_AR, r), i)), zmul(s.eta, ld(V.v(A_Y, r), i))),
                               zmul(s.alpha, ld(V.v(A_AU, r), i)));
        st(V.v(A_T, r), i, t);
        st(V.v(A_Z, r), i, z);
        st(V.v(A_Y, r), i, y);
        st(V.v(A_X, r), i, zadd(zadd(ld(V.v(A_X, r), i), zmul(s.alpha, ld(V.v(A_P, r), i))), z));
        const double2 rn = zsub(t, y);
        st(V.v(A_R, r), i, rn);
        acc[0].x += rn.x * rn.x + rn.y * rn.y;
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
        }
    }
};

// label 50: beta = alpha r0^H r / zeta / R0RN, the iteration limit
template <class T> struct ArBeta {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(A_R0, r), i), ld(V.v(A_R, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (zisnull(s.r0rn)) {
            status = -1;
            s.steperr = 5;
            return;
        }
        if (zisnull(s.dzeta)) {
            status = -1;
            s.steperr = 6;
            return;
        }
        s.beta = zdiv(zdiv(zmul(s.alpha, a[0]), s.dzeta), s.r0rn);
        s.r0rn = a[0];
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            // past MAXIT (gpbicgar.f:360) after the pass's A r: one product
            // more than a pass that converges at label 40
            status = 1;
            s.steperr = 0;
            s.atmax = 1;
        }
    }
};

// ---------------------------------------------------------- BiCGStar-plus ----
// cdmlib/bicgstarplus.f (subroutine GPBICGSTARPLUS): shadow conj(r0) with
// unconjugated dots, mat-vecs A r and A w4, eight dot products per
// iteration.  The reference's first pass adds into two accumulators it never
// cleared; they start at zero here.  Ends like GPBICG past MAXIT.
// slots: 0 conj(r0), 1 A r, 2 r, 3 w4, 4 w5, 5 w6, 6 w7, 7 w8, 8 w9,
//        9 A w4, 10 x, 11 w12, 12 xr (mat-vec out), 13 b
enum { P_R0S = 0, P_AR, P_R, P_W4, P_W5, P_W6, P_W7, P_W8, P_W9, P_AW4, P_X, P_W12, P_XR, P_B, P_NSLOT };

template <class T> struct PsStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(P_B, r), i);
        st(V.v(P_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(P_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
    }
};

// label 10: r = b - A x0, shadow conj(r), w4 = w5 = w8 = w9 = w12 = 0
template <class T> struct PsInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = zsub(ld(V.v(P_B, r), i), ld(V.v(P_XR, r), i));
        const double2 z = make_double2(0, 0), rs = zconj(rr);
        st(V.v(P_R, r), i, rr);
        st(V.v(P_R0S, r), i, rs);
        st(V.v(P_W4, r), i, z);
        st(V.v(P_W5, r), i, z);
        st(V.v(P_W8, r), i, z);
        st(V.v(P_W9, r), i, z);
        st(V.v(P_W12, r), i, z);
        acc[0] = zadd(acc[0], zmul(rs, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.r0rn = a[0];
        s.itno = 0;
    }
};

// label 20: the eight dot products, beta, alpha, zeta, eta
template <class T> struct PsCoef {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rs = ld(V.v(P_R0S, r), i), rr = ld(V.v(P_R, r), i), ar = ld(V.v(P_AR, r), i),
                      w5 = ld(V.v(P_W5, r), i);
        acc[0] = zadd(acc[0], zmul(rs, rr));
        acc[1] = zadd(acc[1], zmul(rs, ar));
        acc[2] = zadd(acc[2], zconjmul(w5, w5));
        acc[3] = zadd(acc[3], zconjmul(ar, rr));
        acc[4] = zadd(acc[4], zconjmul(ar, w5));
        acc[5] = zadd(acc[5], zconjmul(w5, rr));
        acc[6] = zadd(acc[6], zconjmul(ar, ar));
        acc[7] = zadd(acc[7], zmul(rs, ld(V.v(P_W12, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        const double2 c1 = a[0], c2 = a[1], c3 = a[2], c4 = a[3], c5 = a[4], c6 = a[5], c7 = a[6], c8 = a[7];
        if (s.itno == 0) {
            s.eta = make_double2(0, 0);
            s.beta = make_double2(0, 0);
            s.r0rn = c1;
            if (zisnull(c7)) {
                status = -1;
                s.steperr = 2;
                return;
            }
            s.dzeta = zdiv(c4, c7);
            if (zisnull(c2)) {
                status = -1;
                s.steperr = 3;
                return;
            }
            s.alpha = zdiv(c1, c2);
            return;
        }
        if (zisnull(s.dzeta)) {
            status = -1;
            s.steperr = 4;
            return;
        }
        if (zisnull(s.r0rn)) {
            status = -1;
            s.steperr = 5;
            return;
        }
        s.beta = zdiv(zmul(zdiv(make_double2(-s.alpha.x, -s.alpha.y), s.dzeta), c1), s.r0rn);
        const double2 c = zsub(c2, zmul(s.beta, c8));
        if (zisnull(c)) {
            status = -1;
            s.steperr = 6;
            return;
        }
        s.alpha = zdiv(c1, c);
        const double2 d = zsub(zmul(c7, c3), zmul(c5, zconj(c5)));
        if (zisnull(d)) {
            status = -1;
            s.steperr = 7;
            return;
        }
        s.dzeta = zdiv(zsub(zmul(c3, c4), zmul(c5, c6)), d);
        s.eta = zdiv(zsub(zmul(c7, c6), zmul(zconj(c5), c4)), d);
        s.r0rn = c1;
    }
};

// w7 = Ar - beta w12, w6 = zeta r + eta w9, w4 = zeta w7 + eta (w5 - beta w4); then A w4
template <class T> struct PsW {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 w7 = zsub(ld(V.v(P_AR, r), i), zmul(s.beta, ld(V.v(P_W12, r), i)));
        st(V.v(P_W7, r), i, w7);
        st(V.v(P_W6, r), i, zadd(zmul(s.dzeta, ld(V.v(P_R, r), i)), zmul(s.eta, ld(V.v(P_W9, r), i))));
        const double2 q = zsub(ld(V.v(P_W5, r), i), zmul(s.beta, ld(V.v(P_W4, r), i)));
        st(V.v(P_W4, r), i, zadd(zmul(s.dzeta, w7), zmul(s.eta, q)));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 30 and 40: w8, w12, w9, w5, x, r, the stop test, the iteration limit
template <class T> struct PsUpdate {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 rr = ld(V.v(P_R, r), i), w4 = ld(V.v(P_W4, r), i), aw4 = ld(V.v(P_AW4, r), i),
                      w6 = ld(V.v(P_W6, r), i);
        const double2 w8 = zsub(zsub(rr, zmul(s.beta, ld(V.v(P_W8, r), i))), w4);
        const double2 w12 = zsub(ld(V.v(P_W7, r), i), aw4);
        st(V.v(P_W8, r), i, w8);
        st(V.v(P_W12, r), i, w12);
        st(V.v(P_W9, r), i, zsub(w6, zmul(s.alpha, w4)));
        const double2 tmp = zadd(zmul(s.dzeta, ld(V.v(P_AR, r), i)), zmul(s.eta, ld(V.v(P_W5, r), i)));
        st(V.v(P_W5, r), i, zsub(tmp, zmul(s.alpha, aw4)));
        st(V.v(P_X, r), i, zadd(zadd(ld(V.v(P_X, r), i), w6), zmul(s.alpha, w8)));
        const double2 rn = zsub(zsub(rr, tmp), zmul(s.alpha, w12));
        st(V.v(P_R, r), i, rn);
        acc[0].x += rn.x * rn.x + rn.y * rn.y;
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
            return;
        }
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            status = 1;
            s.steperr = 0;
        }
    }
};

// ------------------------------------------------------------------- CORS ----
// cdmlib/cors.f: shadow conj(A r0) with unconjugated dots, mat-vecs A r and
// A d.  Past MAXIT the reference returns a work column it never writes;
// here x.  KState: alpha, beta, rho, rhoa; itno = ITNO (from 0).
// slots: 0 shadow, 1 r, 2 A r, 3 e, 4 h, 5 d, 6 f, 7 g, 8 q = A d, 9 x,
//        10 xr (mat-vec out), 11 b
enum { R_RS = 0, R_R, R_AR, R_E, R_H, R_D, R_F, R_G, R_Q, R_X, R_XR, R_B, R_NSLOT };

// x = x0 (or 0), NORM summed as |b_i|^2 (cors.f)
template <class T> struct CsStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(R_B, r), i);
        st(V.v(R_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(R_XR, r), i, make_double2(0, 0));
        const double a = hypot(b.x, b.y);
        acc[0].x += a * a;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
    }
};

// label 10: r = b - A x0
template <class T> struct CsInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2*) const {
        st(V.v(R_R, r), i, zsub(ld(V.v(R_B, r), i), ld(V.v(R_XR, r), i)));
    }
    __device__ void finish(int, KState& s, int&, const double2*) const { s.itno = 0; }
};

// label 20: (first pass) shadow = conj(A r); rho = shadow^T A r; beta
template <class T> struct CsRho {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 ar = ld(V.v(R_AR, r), i);
        double2 rs;
        if (s.itno == 0) {
            rs = zconj(ar);
            st(V.v(R_RS, r), i, rs);
        } else {
            rs = ld(V.v(R_RS, r), i);
        }
        acc[0] = zadd(acc[0], zmul(rs, ar));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.rho = a[0];
        if (a[0].x == 0.0 && a[0].y == 0.0) {
            status = -1;
            s.steperr = 1;
            return;
        }
        if (s.itno != 0) s.beta = zdiv(s.rho, s.rhoa);
    }
};

// e, h, d (first pass: e = r, h = d = A r); then A d
template <class T> struct CsD {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 rr = ld(V.v(R_R, r), i), ar = ld(V.v(R_AR, r), i);
        if (s.itno == 0) {
            st(V.v(R_E, r), i, rr);
            st(V.v(R_H, r), i, ar);
            st(V.v(R_D, r), i, ar);
        } else {
            const double2 g = ld(V.v(R_G, r), i);
            st(V.v(R_E, r), i, zadd(rr, zmul(s.beta, ld(V.v(R_F, r), i))));
            const double2 h = zadd(ar, zmul(s.beta, g));
            st(V.v(R_H, r), i, h);
            st(V.v(R_D, r), i, zadd(h, zmul(s.beta, zadd(g, zmul(s.beta, ld(V.v(R_D, r), i))))));
        }
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 30: alpha = rho / shadow^T q
template <class T> struct CsAlpha {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zmul(ld(V.v(R_RS, r), i), ld(V.v(R_Q, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (a[0].x == 0.0 && a[0].y == 0.0) {
            status = -1;
            s.steperr = 2;
            return;
        }
        s.alpha = zdiv(s.rho, a[0]);
    }
};

// f, g, x += alpha (2 e - alpha d), r -= alpha (2 h - alpha q), the stop
// test (||r|| summed as |r_i|^2), label 40
template <class T> struct CsUpdate {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 e = ld(V.v(R_E, r), i), d = ld(V.v(R_D, r), i), h = ld(V.v(R_H, r), i),
                      q = ld(V.v(R_Q, r), i);
        st(V.v(R_F, r), i, zsub(e, zmul(s.alpha, d)));
        st(V.v(R_G, r), i, zsub(h, zmul(s.alpha, q)));
        const double2 two = make_double2(2, 0);
        st(V.v(R_X, r), i, zadd(ld(V.v(R_X, r), i), zmul(s.alpha, zsub(zmul(two, e), zmul(s.alpha, d)))));
        const double2 rn = zsub(ld(V.v(R_R, r), i), zmul(s.alpha, zsub(zmul(two, h), zmul(s.alpha, q))));
        st(V.v(R_R, r), i, rn);
        const double a = hypot(rn.x, rn.y);
        acc[0].x += a * a;
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
            return;
        }
        s.rhoa = s.rho;
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            status = 1;
            s.steperr = 0;
        }
    }
};

// ---------------------------------------------------------------- GPBiCOR ----
// cdmlib/gpbicor.f: mat-vecs A r and A w4; ITNO counts from 1 and its driver
// reports it as is.  Past MAXIT the reference sets no solution; here x.
// KState: alpha, beta, eta, dzeta, rho, rhoa; itno = ITNO.
// slots: 0 r0, 1 p, 2 A r, 3 w4, 4 w5, 5 w6, 6 t, 7 w8, 8 w9, 9 r, 10 z,
//        11 w12, 12 q, 13 s, 14 A w4, 15 x, 16 xr (mat-vec out), 17 b
enum { O_R0 = 0, O_P, O_AR, O_W4, O_W5, O_W6, O_T, O_W8, O_W9, O_R, O_Z, O_W12, O_Q, O_S, O_AW4, O_X, O_XR, O_B,
       O_NSLOT };

template <class T> struct OStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(O_B, r), i);
        st(V.v(O_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(O_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 1;
        s.steperr = -1;
    }
};

// label 10: r0 = r = b - A x0, z = 0
template <class T> struct OInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2*) const {
        const double2 rr = zsub(ld(V.v(O_B, r), i), ld(V.v(O_XR, r), i));
        st(V.v(O_R0, r), i, rr);
        st(V.v(O_R, r), i, rr);
        st(V.v(O_Z, r), i, make_double2(0, 0));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 20: rho = r0^H A r, beta = rho / rhoa alpha / zeta (0 on the first pass)
template <class T> struct ORho {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(O_R0, r), i), ld(V.v(O_AR, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.rho = a[0];
        if (a[0].x == 0.0 && a[0].y == 0.0) {
            status = -1;
            s.steperr = 1;
            return;
        }
        s.beta = s.itno == 1 ? make_double2(0, 0) : zdiv(zmul(zdiv(s.rho, s.rhoa), s.alpha), s.dzeta);
    }
};

// p, w4, w5 (first pass: p = r0, w4 = A r, the rest 0); then A w4
template <class T> struct OP {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 ar = ld(V.v(O_AR, r), i);
        if (s.itno == 1) {
            const double2 z = make_double2(0, 0);
            st(V.v(O_P, r), i, ld(V.v(O_R0, r), i));
            st(V.v(O_W4, r), i, ar);
            st(V.v(O_W12, r), i, z);
            st(V.v(O_W5, r), i, z);
            st(V.v(O_W8, r), i, z);
            st(V.v(O_W9, r), i, z);
            st(V.v(O_W6, r), i, z);
        } else {
            const double2 w4 = ld(V.v(O_W4, r), i);
            st(V.v(O_W5, r), i, zadd(ld(V.v(O_W6, r), i), zmul(s.beta, w4)));
            st(V.v(O_P, r), i,
               zadd(ld(V.v(O_R, r), i), zmul(s.beta, zsub(ld(V.v(O_P, r), i), ld(V.v(O_W8, r), i)))));
            st(V.v(O_W4, r), i, zadd(ar, zmul(s.beta, zsub(w4, ld(V.v(O_W9, r), i)))));
        }
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 30: alpha = rho / r0^H A w4
template <class T> struct OAlpha {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(O_R0, r), i), ld(V.v(O_AW4, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (a[0].x == 0.0 && a[0].y == 0.0) {
            status = -1;
            s.steperr = 2;
            return;
        }
        s.alpha = zdiv(s.rho, a[0]);
    }
};

// q, t, s and the five dot products of zeta and eta
template <class T> struct OZeta {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 rr = ld(V.v(O_R, r), i), w4 = ld(V.v(O_W4, r), i);
        const double2 q = zadd(zsub(ld(V.v(O_W12, r), i), rr), zmul(s.alpha, zsub(w4, ld(V.v(O_W5, r), i))));
        const double2 t = zsub(rr, zmul(s.alpha, w4));
        const double2 sv = zsub(ld(V.v(O_AR, r), i), zmul(s.alpha, ld(V.v(O_AW4, r), i)));
        st(V.v(O_Q, r), i, q);
        st(V.v(O_T, r), i, t);
        st(V.v(O_S, r), i, sv);
        acc[0] = zadd(acc[0], zconjmul(sv, sv));
        acc[1] = zadd(acc[1], zconjmul(q, t));
        acc[2] = zadd(acc[2], zconjmul(q, sv));
        acc[3] = zadd(acc[3], zconjmul(sv, t));
        acc[4] = zadd(acc[4], zconjmul(q, q));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        const double2 c1 = a[0], c2 = a[1], c3 = a[2], c4 = a[3], c5 = a[4];
        if (s.itno == 1) {
            s.eta = make_double2(0, 0);
            if (c1.x == 0.0 && c1.y == 0.0) {
                status = -1;
                s.steperr = 3;
                return;
            }
            s.dzeta = zdiv(c4, c1);
            return;
        }
        const double2 c = zsub(zmul(c1, c5), zmul(c3, zconj(c3)));
        if (c.x == 0.0 && c.y == 0.0) {
            status = -1;
            s.steperr = 4;
            return;
        }
        s.eta = zdiv(zsub(zmul(c1, c2), zmul(c3, c4)), c);
        s.dzeta = zdiv(zsub(zmul(c5, c4), zmul(c2, zconj(c3))), c);
    }
};

// w8, w9, z, r = t - eta q - zeta s, x += alpha p + z, w6 = s, w12 = t;
// the stop test, label 40
template <class T> struct OUpdate {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 rr = ld(V.v(O_R, r), i), w4 = ld(V.v(O_W4, r), i), w12 = ld(V.v(O_W12, r), i),
                      ar = ld(V.v(O_AR, r), i), sv = ld(V.v(O_S, r), i), t = ld(V.v(O_T, r), i);
        const double2 w8 = zadd(zmul(s.dzeta, w4), zmul(s.eta, zadd(zsub(w12, rr), zmul(s.beta, ld(V.v(O_W8, r), i)))));
        const double2 w9 = zadd(zdiv(zmul(s.dzeta, zsub(ar, sv)), s.alpha),
                                zmul(s.eta, zadd(zsub(ld(V.v(O_W6, r), i), ar), zmul(s.beta, ld(V.v(O_W9, r), i)))));
        const double2 z = zsub(zadd(zmul(s.dzeta, rr), zmul(s.eta, ld(V.v(O_Z, r), i))), zmul(s.alpha, w8));
        st(V.v(O_W8, r), i, w8);
        st(V.v(O_W9, r), i, w9);
        st(V.v(O_Z, r), i, z);
        const double2 rn = zsub(zsub(t, zmul(s.eta, ld(V.v(O_Q, r), i))), zmul(s.dzeta, sv));
        st(V.v(O_R, r), i, rn);
        acc[0].x += rn.x * rn.x + rn.y * rn.y;
        st(V.v(O_X, r), i, zadd(zadd(ld(V.v(O_X, r), i), zmul(s.alpha, ld(V.v(O_P, r), i))), z));
        st(V.v(O_W6, r), i, sv);
        st(V.v(O_W12, r), i, t);
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
            return;
        }
        s.rhoa = s.rho;
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            status = 1;
            s.steperr = 0;
        }
    }
};

// ----------------------------------------------------------------- TFQMR ----
// cdmlib/tfqmr.f:1-218: passes alternate, an even pass forms alpha and the
// next u, an odd one rho, beta and v; stop when sqrt(ITNO+1) |tau| / NORM <=
// tol.  Past MAXIT the reference routine returns no status (its driver loops
// for ever); here the solve ends there with the current iterate.  KState:
// alpha, beta, rho, tau, theta, etaq = eta, conv; itno = ITNO.
// slots: 0 u, 1 w, 2 r, 3 v, 4 d, 5 rtilde, 6 u next, 7 A u, 8 A u previous,
//        9 x, 10 xr (mat-vec out), 11 b
enum { T_U = 0, T_W, T_R, T_V, T_D, T_RT, T_U1, T_AU, T_AUP, T_X, T_XR, T_B, T_NSLOT };

// tfqmr.f:45-53: x = x0 (or 0), NORM = ||b||
template <class T> struct TStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(T_B, r), i);
        st(V.v(T_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(T_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
        s.conv = 0;
        s.atmax = 0;
    }
};

// label 10 (tfqmr.f:57-64): r = w = u = b - A x0
template <class T> struct TInit1 {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2*) const {
        const double2 rr = zsub(ld(V.v(T_B, r), i), ld(V.v(T_XR, r), i));
        st(V.v(T_R, r), i, rr);
        st(V.v(T_W, r), i, rr);
        st(V.v(T_U, r), i, rr);
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 20 (tfqmr.f:66-82): v = A u, d = 0, rtilde = r, rho = rtilde^H r,
// tau = NORM, theta = eta = 0, ITNO = 0
template <class T> struct TInit2 {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 rr = ld(V.v(T_R, r), i);
        st(V.v(T_AU, r), i, ld(V.v(T_V, r), i));
        st(V.v(T_D, r), i, make_double2(0, 0));
        st(V.v(T_RT, r), i, rr);
        acc[0] = zadd(acc[0], zconjmul(rr, rr));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.rho = a[0];
        s.tau = make_double2(s.norm, 0);
        s.theta = make_double2(0, 0);
        s.etaq = make_double2(0, 0);
        s.itno = 0;
        s.conv = 0;
    }
};

// tfqmr.f:88-96 (even pass): alpha = rho / rtilde^H v
template <class T> struct TAlpha {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zconjmul(ld(V.v(T_RT, r), i), ld(V.v(T_V, r), i)));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const { s.alpha = zdiv(s.rho, a[0]); }
};

// tfqmr.f:97-125: (even) u next = u - alpha v; w -= alpha A u,
// d = u + theta^2 / alpha eta d; theta, c, tau, eta; the stop test
template <class T, bool EVEN> struct TW {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 u = ld(V.v(T_U, r), i);
        if (EVEN) st(V.v(T_U1, r), i, zsub(u, zmul(s.alpha, ld(V.v(T_V, r), i))));
        const double2 wn = zsub(ld(V.v(T_W, r), i), zmul(s.alpha, ld(V.v(T_AU, r), i)));
        const double2 f = zmul(zdiv(zmul(s.theta, s.theta), s.alpha), s.etaq);
        st(V.v(T_W, r), i, wn);
        st(V.v(T_D, r), i, zadd(u, zmul(f, ld(V.v(T_D, r), i))));
        acc[0] = zadd(acc[0], zconjmul(wn, wn));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.theta = zdiv(zsqrt(a[0]), s.tau);
        const double2 c = zdiv(make_double2(1, 0), zsqrt(zadd(make_double2(1, 0), zmul(s.theta, s.theta))));
        s.tau = zmul(zmul(s.tau, s.theta), c);
        s.etaq = zmul(zmul(c, c), s.alpha);
        if (sqrt((double)(s.itno + 1)) * hypot(s.tau.x, s.tau.y) / s.norm <= s.tol) s.conv = 1;
    }
};

// tfqmr.f:127-149: x += eta d; converged -> stop; (odd) rho = rtilde^H w,
// beta = rho / rho0
template <class T, bool ODD> struct TX {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        st(V.v(T_X, r), i, zadd(ld(V.v(T_X, r), i), zmul(s.etaq, ld(V.v(T_D, r), i))));
        if (ODD) acc[0] = zadd(acc[0], zconjmul(ld(V.v(T_RT, r), i), ld(V.v(T_W, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        if (s.conv) {
            status = 1;
            s.steperr = 0;
            return;
        }
        if (ODD) {
            const double2 rho0 = s.rho;
            s.rho = a[0];
            s.beta = zdiv(s.rho, rho0);
        }
    }
};

// tfqmr.f:150-163: (odd) u next = w + beta u, A u previous = A u; u = u next
template <class T, bool ODD> struct TU {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        if (ODD) {
            const double2 un = zadd(ld(V.v(T_W, r), i), zmul(s.beta, ld(V.v(T_U, r), i)));
            st(V.v(T_U, r), i, un);
            st(V.v(T_AUP, r), i, ld(V.v(T_AU, r), i));
        } else {
            st(V.v(T_U, r), i, ld(V.v(T_U1, r), i));
        }
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 30 (tfqmr.f:166-177): (odd) v = A u + beta (A u previous + beta v);
// next pass, or the end past MAXIT
template <class T, bool ODD> struct TV {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        if (ODD) {
            const double2 v = ld(V.v(T_V, r), i);
            st(V.v(T_V, r), i,
               zadd(ld(V.v(T_AU, r), i), zmul(s.beta, zadd(ld(V.v(T_AUP, r), i), zmul(s.beta, v)))));
        }
    }
    __device__ void finish(int, KState& s, int& status, const double2*) const {
        if (s.itno <= s.maxit) {
            s.itno += 1;
        } else {
            // past MAXIT after the pass's A u (tfqmr.f:216): one product more
            // than a pass that converges
            status = 1;
            s.steperr = 0;
            s.atmax = 1;
        }
    }
};

// ---------------------------------------------------------------- QMRCLA ----
// QMR without look-ahead (PIMZQMR, cdmlib/qmrpim.f:1-270), with products by
// A and by A^T.  Slots: w1 .. w9 are the reference's WRK columns 1 .. 9, T the
// scratch of the transposed product.  State: lambda = alpha, kappa = beta,
// theta, gamma = dzeta, ksi = eta, rho, epsilon = omega, mu = etaq, tau, the
// dot products DOTS1..3 in c2, c5, f1.
enum { L_X = 0, L_W1, L_W2, L_W3, L_W4, L_W5, L_W6, L_W7, L_W8, L_W9, L_T, L_XR, L_B, L_NSLOT };

// label 10 (qmrpim.f:45-64): NORM = ||b||, x = x0
template <class T> struct LStart {
    Slots<T> V;
    KState* stt;
    int zero_guess;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 b = ld(V.v(L_B, r), i);
        st(V.v(L_X, r), i, zero_guess ? make_double2(0, 0) : b);
        if (zero_guess) st(V.v(L_XR, r), i, make_double2(0, 0));
        acc[0].x += b.x * b.x + b.y * b.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.alpha = make_double2(1, 0);
        s.beta = make_double2(-1, 0);
        s.theta = make_double2(-1, 0);
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        s.steperr = -1;
    }
};

// label 20 (:68-92): w3 = A x0, w1 = w7 = w8 = b - A x0, w2 = w4 = w5 = w6 = 0;
// DOTS1 = w7^H w7, DOTS2 = w8^H w8, DOTS3 = w7^T w8
template <class T> struct LInit {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 w3 = ld(V.v(L_XR, r), i), w1 = zsub(ld(V.v(L_B, r), i), w3);
        st(V.v(L_W3, r), i, w3);
        st(V.v(L_W1, r), i, w1);
        st(V.v(L_W7, r), i, w1);
        st(V.v(L_W8, r), i, w1);
        const double2 z = make_double2(0, 0);
        st(V.v(L_W2, r), i, z);
        st(V.v(L_W4, r), i, z);
        st(V.v(L_W5, r), i, z);
        st(V.v(L_W6, r), i, z);
        acc[0] = zadd(acc[0], zconjmul(w1, w1));
        acc[1] = zadd(acc[1], zconjmul(w1, w1));
        acc[2] = zadd(acc[2], zmul(w1, w1));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.c2 = a[0];
        s.c5 = a[1];
        s.f1 = a[2];
    }
};

// The transposed product's second half (inverserigopt.f:570-583): slot T
// holds x - G x, and out = alpha^T (T - x) + x (A^T = I - alpha^T G, G being
// symmetric)
template <class T> struct LTrans {
    Slots<T> V;
    KState* stt;
    int sin, sout;
    int amode;
    const cplx<T>* alpha;
    long nmax;
    __device__ void elem(const KState&, int r, long i, double2*) const {
        const long d = i / 3;
        const int c = (int)(i - 3 * d);
        const cplx<T>* t = V.v(L_T, r);
        const cplx<T>* x = V.v(sin, r);
        const double2 xi = ld(x, i);
        double2 acc;
        if (amode == ALPHA_ISO) {
            acc = zmul(to_d(alpha[d]), zsub(ld(t, i), xi));
        } else if (amode == ALPHA_FULL) {
            acc = make_double2(0, 0);
            for (int b = 0; b < 3; b++)
                acc = zadd(acc, zmul(to_d(alpha[d + nmax * (b + 3 * c)]), zsub(ld(t, 3 * d + b), ld(x, 3 * d + b))));
        } else {
            acc = zsub(ld(t, i), xi);
        }
        st(V.v(sout, r), i, zadd(acc, xi));
    }
    __device__ void finish(int, KState&, int&, const double2*) const {}
};

// label 30 (:96-121): DOTS4 = w7^T w9 (w9 = A^T w8), then gamma, ksi, rho,
// epsilon, mu = 0, tau
template <class T> struct LInit2 {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zmul(ld(V.v(L_W7, r), i), ld(V.v(L_W9, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.dzeta = zsqrt(s.c2);
        s.eta = zsqrt(s.c5);
        s.rho = s.f1;
        s.omega = a[0];
        s.etaq = make_double2(0, 0);
        if (zisnull(s.rho)) {
            s.itno = 0;
            s.steperr = 5;
            status = -1;
            return;
        }
        s.tau = zdiv(s.omega, s.rho);
        // the checks that open label 100
        if (zisnull(s.dzeta)) {
            s.steperr = 6;
            status = -1;
        } else if (zisnull(s.eta)) {
            s.steperr = 7;
            status = -1;
        }
    }
};

// label 100 (:122-146): ITNO + 1, the zero checks, w2 = w7 / gamma - mu w2,
// w4 = (w9 - gamma mu w4) / ksi (A w2 follows).  The checks of this pass are
// made by the previous pass's finish (or LInit2's) on the new values, so the
// pass itself only updates; its single sum is unused.
template <class T> struct LA {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2*) const {
        const double2 w2 = zsub(zdiv(ld(V.v(L_W7, r), i), s.dzeta), zmul(s.etaq, ld(V.v(L_W2, r), i)));
        const double2 w4 = zdiv(zsub(ld(V.v(L_W9, r), i), zmul(zmul(s.dzeta, s.etaq), ld(V.v(L_W4, r), i))), s.eta);
        st(V.v(L_W2, r), i, w2);
        st(V.v(L_W4, r), i, w4);
    }
    __device__ void finish(int, KState& s, int&, const double2*) const { s.itno += 1; }
};

// label 40 (:148-166): w3 = A w2, w7 = w3 - tau / gamma w7, w8 = w4 - tau /
// ksi w8, the three dots (A^T w8 follows)
template <class T> struct LB {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 w7 = zsub(ld(V.v(L_W3, r), i), zmul(zdiv(s.tau, s.dzeta), ld(V.v(L_W7, r), i)));
        const double2 w8 = zsub(ld(V.v(L_W4, r), i), zmul(zdiv(s.tau, s.eta), ld(V.v(L_W8, r), i)));
        st(V.v(L_W7, r), i, w7);
        st(V.v(L_W8, r), i, w8);
        acc[0] = zadd(acc[0], zconjmul(w7, w7));
        acc[1] = zadd(acc[1], zconjmul(w8, w8));
        acc[2] = zadd(acc[2], zmul(w7, w8));
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const {
        s.c2 = a[0];
        s.c5 = a[1];
        s.f1 = a[2];
    }
};

// label 50, first half (:176-215): DOTS4 = w7^T w9, then gamma, ksi, rho,
// epsilon, mu, tau, theta, kappa, lambda with the breakdown checks 12-14
template <class T> struct LC {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        acc[0] = zadd(acc[0], zmul(ld(V.v(L_W7, r), i), ld(V.v(L_W9, r), i)));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        const double2 gamma0 = s.dzeta, ksi0 = s.eta, rho0 = s.rho;
        s.dzeta = zsqrt(s.c2);
        s.eta = zsqrt(s.c5);
        s.rho = s.f1;
        s.omega = a[0];
        double2 den = zmul(zmul(s.dzeta, s.tau), rho0);
        if (zisnull(den)) {
            s.steperr = 12;
            status = -1;
            return;
        }
        s.etaq = zdiv(zmul(zmul(gamma0, ksi0), s.rho), den);
        if (zisnull(s.rho)) {
            s.steperr = 13;
            status = -1;
            return;
        }
        const double2 tau0 = s.tau;
        s.tau = zsub(zdiv(s.omega, s.rho), zmul(s.dzeta, s.etaq));
        const double at = hypot(tau0.x, tau0.y), ag = hypot(s.dzeta.x, s.dzeta.y);
        const double abstau02 = at * at, absgamma2 = ag * ag;
        den = make_double2(s.alpha.x * abstau02 + absgamma2, s.alpha.y * abstau02);
        if (zisnull(den)) {
            s.steperr = 14;
            status = -1;
            return;
        }
        s.theta = zdiv(make_double2(abstau02 * (1.0 - s.alpha.x), -abstau02 * s.alpha.y), den);
        const double2 kappa0 = s.beta;
        const double2 k = zmul(zmul(gamma0, zconj(tau0)), kappa0);
        s.beta = zdiv(make_double2(-k.x, -k.y), den);
        s.alpha = zdiv(make_double2(s.alpha.x * abstau02, s.alpha.y * abstau02), den);
    }
};

// label 50, second half (:217-240): w5 = theta w5 + kappa w2, w6 = theta w6 +
// kappa w3, x += w5, w1 -= w6; stop when ||w1|| / NORM <= tol; past the
// iteration limit the reference fails (STATUS = -1)
template <class T> struct LD {
    Slots<T> V;
    KState* stt;
    __device__ void elem(const KState& s, int r, long i, double2* acc) const {
        const double2 w5 = zadd(zmul(s.theta, ld(V.v(L_W5, r), i)), zmul(s.beta, ld(V.v(L_W2, r), i)));
        const double2 w6 = zadd(zmul(s.theta, ld(V.v(L_W6, r), i)), zmul(s.beta, ld(V.v(L_W3, r), i)));
        st(V.v(L_W5, r), i, w5);
        st(V.v(L_W6, r), i, w6);
        st(V.v(L_X, r), i, zadd(ld(V.v(L_X, r), i), w5));
        const double2 w1 = zsub(ld(V.v(L_W1, r), i), w6);
        st(V.v(L_W1, r), i, w1);
        acc[0].x += w1.x * w1.x + w1.y * w1.y;
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(fabs(a[0].x)) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            s.steperr = 0;
            return;
        }
        if (s.itno > s.maxit) {
            // STATUS = -1, ITNO = MAXIT, then label 100 counts one more
            s.itno = s.maxit + 1;
            s.steperr = 0;
            status = -1;
            return;
        }
        // the checks that open label 100 for the next pass
        if (zisnull(s.dzeta)) {
            s.steperr = 6;
            status = -1;
        } else if (zisnull(s.eta)) {
            s.steperr = 7;
            status = -1;
        }
    }
};

// ------------------------------------------------------------ shared ------
// y = alpha . x (polarisability, cdmlib/inverserigopt.f:68-80) on FP64 vectors
__global__ void k_apply_alpha(const double2* __restrict__ x, double2* __restrict__ y, long nd, int nrhs, long stride,
                              int amode, const double2* __restrict__ alpha, long nmax);

}  // namespace ifdda
