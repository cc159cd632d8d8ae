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
#include "reduce.cuh"

namespace ifdda {

struct KState {
    // GPBiCG
    double2 alpha, beta, eta, dzeta, r0rn, c2, c5;
    // QMR-BiCGSTAB
    double2 rho, omega, tau, taut, theta, thetat, etaq, etat, f1, qbeta;
    double norm, residu, tol;
    int itno, steperr, maxit, conv;
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

// label 30 coefficients (gpbicg.f:212-264)
template <class T> struct GpZeta {
    Slots<T> V;
    KState* stt;
    int tnew;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const double2 at = ld(V.v(G_AT, r), i), y = ld(V.v(G_Y, r), i), t = ld(V.v(tnew, r), i);
        acc[0] = zadd(acc[0], zconjmul(at, at));
        acc[1] = zadd(acc[1], zconjmul(at, y));
        acc[2] = zadd(acc[2], zconjmul(at, t));
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        const double2 c1 = a[0], c3 = a[1], c4 = a[2], c2 = s.c2, c5 = s.c5;
        if (s.itno == 0) {
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
        const double2 ap = ld(V.v(G_AP, r), i), told = ld(V.v(tcur, r), i), rr = ld(V.v(G_R, r), i);
        const double2 u0 = ld(V.v(G_U, r), i), z0 = ld(V.v(G_Z, r), i);
        const double2 u = zadd(zmul(s.dzeta, ap), zmul(s.eta, zadd(zsub(told, rr), zmul(s.beta, u0))));
        const double2 z = zsub(zadd(zmul(s.dzeta, rr), zmul(s.eta, z0)), zmul(s.alpha, u));
        const double2 x = zadd(zadd(ld(V.v(G_X, r), i), zmul(s.alpha, ld(V.v(G_P, r), i))), z);
        const double2 rn = zsub(zsub(ld(V.v(tnew, r), i), zmul(s.eta, ld(V.v(G_Y, r), i))),
                                zmul(s.dzeta, ld(V.v(G_AT, r), i)));
        st(V.v(G_U, r), i, u);
        st(V.v(G_Z, r), i, z);
        st(V.v(G_X, r), i, x);
        st(V.v(G_R, r), i, rn);
        acc[0].x += rn.x * rn.x + rn.y * rn.y;
        acc[1] = zadd(acc[1], zconjmul(ld(V.v(G_R0, r), i), rn));
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

// ------------------------------------------------------------ shared ------
// y = alpha . x (polarisability, cdmlib/inverserigopt.f:68-80) on FP64 vectors
__global__ void k_apply_alpha(const double2* __restrict__ x, double2* __restrict__ y, long nd, int nrhs, long stride,
                              int amode, const double2* __restrict__ alpha, long nmax);

}  // namespace ifdda
