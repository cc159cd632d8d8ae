// Host orchestration of the device Krylov solvers and of the mixed-precision
// (FP32 inner / FP64 outer) iterative refinement.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <utility>
#include <vector>
#include "gpbicg_fused.cuh"
#include "solver.cuh"

namespace ifdda {

// ---------------------------------------------------------------- kernels --
__global__ void k_apply_alpha(const double2* __restrict__ x, double2* __restrict__ y, long nd, int nrhs, long stride,
                              int amode, const double2* __restrict__ alpha, long nmax) {
    const long tot = nd * nrhs;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        const long r = q / nd, d = q - r * nd;
        const double2* xv = x + r * stride + 3 * d;
        double2* yv = y + r * stride + 3 * d;
        const double2 v[3] = {xv[0], xv[1], xv[2]};
        for (int a = 0; a < 3; a++) {
            double2 acc = make_double2(0, 0);
            if (amode == ALPHA_ISO) acc = zmul(alpha[d], v[a]);
            else if (amode == ALPHA_FULL)
                for (int b = 0; b < 3; b++) acc = zadd(acc, zmul(alpha[d + nmax * (a + 3 * b)], v[b]));
            else acc = v[a];
            yv[a] = acc;
        }
    }
}

// outer residual of the refinement: r = b - A x (A x in ax), relative norm, and
// the FP32 right-hand side of the next inner solve
struct ResidualOp {
    const double2* b;
    const double2* ax;
    float2* b32;
    long n3;
    KState* stt;     // outer state: norm, residu, tol
    KState* inner;   // inner state: tol set here
    int* inner_status;
    double inner_floor;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const long o = (long)r * n3 + i;
        const double2 rv = zsub(b[o], ax[o]);
        b32[o] = make_float2((float)rv.x, (float)rv.y);
        acc[0].x += rv.x * rv.x + rv.y * rv.y;
    }
    __device__ void finish(int r, KState& s, int& status, const double2* a) const {
        s.residu = sqrt(a[0].x) / s.norm;
        if (s.residu <= s.tol) {
            status = 1;
            inner_status[r] = 1;
            return;
        }
        // ask the inner solve to bring the true residual to a fifth of tol,
        // but for no more than FP32 vectors can deliver: the solve then stops
        // with a residual well below tol, and its local field within tol of
        // the converged field (a residual just under tol leaves an error of
        // about tol times the operator's condition)
        inner[r].tol = fmax(0.2 * s.tol / s.residu, inner_floor);
        inner[r].maxit = s.maxit;
        inner_status[r] = 0;
        s.itno += 1;
    }
};

// Fresh solver state for nrhs right-hand sides, set on the device: a copy
// from pageable host memory would wait for the stream first
__global__ void k_init_state(KState* __restrict__ s, int* __restrict__ status, int nrhs, double tol, int maxit) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrhs) return;
    KState k{};
    k.tol = tol;
    k.maxit = maxit;
    s[r] = k;
    if (status) status[r] = 0;
}
static void init_state(KState* s, int* status, int nrhs, double tol, int maxit, cudaStream_t st) {
    count_launch();
    k_init_state<<<(nrhs + 127) / 128, 128, 0, st>>>(s, status, nrhs, tol, maxit);
    IFDDA_CUDA(cudaGetLastError());
}

struct NormOp {  // ||b|| of the outer problem, x = b
    const double2* b;
    double2* x;
    long n3;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const long o = (long)r * n3 + i;
        const double2 v = b[o];
        x[o] = v;
        acc[0].x += v.x * v.x + v.y * v.y;
    }
    __device__ void finish(int, KState& s, int& status, const double2* a) const {
        s.norm = sqrt(a[0].x);
        s.itno = 0;
        // b = 0: every method's first test fails on it (NORM = 0), so the
        // right-hand side stops here instead of refining a 0/0 residual
        if (s.norm == 0.0) status = -1;
    }
};

struct TrueResOp {  // tol1 = ||A x - b|| / NORM (cdmlib/inverserigopt.f:92-102)
    const double2* b;
    const double2* ax;
    long n3;
    KState* stt;
    __device__ void elem(const KState&, int r, long i, double2* acc) const {
        const long o = (long)r * n3 + i;
        const double2 rv = zsub(ax[o], b[o]);
        acc[0].x += rv.x * rv.x + rv.y * rv.y;
    }
    __device__ void finish(int, KState& s, int&, const double2* a) const { s.residu = sqrt(a[0].x) / s.norm; }
};

template <class T>
__global__ void k_axpy_outer(double2* __restrict__ x, const cplx<T>* __restrict__ d, long n3, int nrhs,
                             const int* __restrict__ ostatus) {
    const long tot = n3 * nrhs;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        const long r = q / n3;
        if (ostatus[r]) continue;
        const double2 v = to_d(d[q]);
        x[q] = make_double2(x[q].x + v.x, x[q].y + v.y);
    }
}

template <class T> __global__ void k_cast(const double2* __restrict__ a, cplx<T>* __restrict__ b, long n) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        b[q] = from_d<cplx<T>>(a[q]);
}

template <class T> __global__ void k_uncast(const cplx<T>* __restrict__ a, double2* __restrict__ b, long n) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        b[q] = to_d(a[q]);
}

static inline int grid_for(long n, int nt = 256) { return (int)std::max<long>(1, std::min<long>((n + nt - 1) / nt, 148L * 16)); }

void apply_alpha_dev(const double2* x, double2* y, long nd, int nrhs, long stride, int amode, const double2* alpha,
                     long nmax, cudaStream_t st) {
    count_launch();
    k_apply_alpha<<<grid_for(nd * nrhs), 256, 0, st>>>(x, y, nd, nrhs, stride, amode, alpha, nmax);
    IFDDA_CUDA(cudaGetLastError());
}

template <class T> void cast_dev(const double2* a, cplx<T>* b, long n, cudaStream_t st) {
    count_launch();
    k_cast<T><<<grid_for(n), 256, 0, st>>>(a, b, n);
    IFDDA_CUDA(cudaGetLastError());
}
template void cast_dev<float>(const double2*, float2*, long, cudaStream_t);
template void cast_dev<double>(const double2*, double2*, long, cudaStream_t);

// ------------------------------------------------------------- solver ----
namespace {
std::mutex g_retired_mu;
std::vector<std::pair<int, cudaGraphExec_t>> g_retired;  // (device, executable)

void destroy_execs(const std::vector<std::pair<int, cudaGraphExec_t>>& v) {
    if (v.empty()) return;
    int prev = -1;
    cudaGetDevice(&prev);
    for (const auto& [dev, e] : v) {
        cudaSetDevice(dev);
        cudaGraphExecDestroy(e);
    }
    if (prev >= 0) cudaSetDevice(prev);
}
}  // namespace

void retire_graph_exec(cudaGraphExec_t exec) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<std::pair<int, cudaGraphExec_t>> now;
    {
        std::lock_guard<std::mutex> lk(g_retired_mu);
        g_retired.emplace_back(dev, exec);
        if (g_retired.size() >= 256) now.swap(g_retired);
    }
    destroy_execs(now);
}

void destroy_retired_graph_execs() {
    std::vector<std::pair<int, cudaGraphExec_t>> now;
    {
        std::lock_guard<std::mutex> lk(g_retired_mu);
        now.swap(g_retired);
    }
    destroy_execs(now);
}

int reduction_blocks(long n3) { return (int)std::max<long>(1, std::min<long>((n3 + KNT * 2 - 1) / (KNT * 2), 2048)); }

template <class T> void KrylovWork<T>::ensure(int method, int nrhs_, long n3_) {
    static const int nslots[] = {0,       G_NSLOT, Q_NSLOT, 0,       B_NSLOT, C_NSLOT, T_NSLOT,
                                 S_NSLOT, A_NSLOT, P_NSLOT, R_NSLOT, O_NSLOT, L_NSLOT};
    nslot = nslots[method_family(method)];
    nrhs = nrhs_;
    n3 = n3_;
    nblk = reduction_blocks(n3);
    vecs.ensure((size_t)nslot * nrhs * n3);
    st.ensure(nrhs);
    status.ensure(nrhs);
    zstatus.ensure(nrhs);
    partials.ensure((size_t)nrhs * nblk * 8);  // up to 8 sums per reduction
    tickets.ensure(nrhs);
    hstatus.resize(nrhs);
}

template <class T> Slots<T> KrylovWork<T>::slots() const { return Slots<T>{vecs.p, n3, nrhs}; }

// Reduction buffers of the fused mat-vecs: x-pass grids have at most ny x nz
// blocks per right-hand side; up to 2 partial sums per block from the first
// x pass, 3 from the last, 5 per row.
template <class T> MvRed KrylovWork<T>::mv_red(int ny, int nz) {
    const long rows = (long)nrhs * nz;
    const long np = rows * ny * 2, ne = rows * ny * 3, nr = rows * 5;
    mvpart.ensure((size_t)(np + ne + nr));
    mvtk.ensure((size_t)(rows + nrhs));
    MvRed r;
    r.ppart = mvpart.p;
    r.epart = mvpart.p + np;
    r.rpart = mvpart.p + np + ne;
    r.t1 = mvtk.p;
    r.t2 = mvtk.p + rows;
    r.gxs = ny;
    return r;
}

// Condition of the device-side iteration loop: run another body while some
// right-hand side is still iterating and fewer than `chunk` bodies have run
// in this launch.  One thread; status was written by the body's last kernel.
__global__ void k_loop_ctl(cudaGraphConditionalHandle h, const int* __restrict__ status, int nrhs, int* count,
                           int chunk) {
    if (threadIdx.x != 0) return;
    const int c = *count + 1;
    *count = c;
    bool run = false;
    if (c < chunk)
        for (int r = 0; r < nrhs && !run; r++) run = status[r] == 0;
    cudaGraphSetConditional(h, run ? 1u : 0u);
}

template <int ND, class Op>
static void vec_launch(const Op& op, long n3, int nblk, int nrhs, const RedSlots& rs, int* status, cudaStream_t st) {
    count_launch();
    launch_pdl(k_vec<ND, Op>, dim3(nblk, nrhs), dim3(KNT), 0, st, op, n3, nblk, rs, status);
}

template <class T>
static void mv_solver(Green& G, const SolveSpec& sp, KrylovWork<T>& W, int sx, int sy, const int* status,
                      cudaStream_t st) {
    Slots<T> V = W.slots();
    const cplx<T>* x = V.base + (long)sx * W.nrhs * W.n3;
    cplx<T>* y = V.base + (long)sy * W.nrhs * W.n3;
    MvArgs<T> a = mv_args<T>(G, W.nrhs, x, x, y, W.n3, sp.amode, (const cplx<T>*)sp.alpha, sp.nmax, sp.tabdip, status);
    set_ragged(a, sp);
    if (!matvec_launch<T>(a, W.nrhs, sp.tabdip != nullptr, st))
        throw EngineError{1, "FFT size not supported by the compiled kernels"};
}

// y = A^T x for the QMRCLA branch (cdmlib/inverserigopt.f:555-584): the
// scratch slot T gets x - G x from a mat-vec without the polarisability,
// then y = alpha^T (T - x) + x.  No memset, so the pass stays a pair of
// kernel nodes inside the captured loop body.
template <class T>
static void mv_transpose(Green& G, const SolveSpec& sp, KrylovWork<T>& W, int sx, int sy, int* status,
                         const RedSlots& rs, cudaStream_t st) {
    Slots<T> V = W.slots();
    MvArgs<T> a = mv_args<T>(G, W.nrhs, V.v(sx, 0), V.v(sx, 0), V.v(L_T, 0), W.n3, ALPHA_NONE, nullptr, 0, sp.tabdip,
                             status);
    set_ragged(a, sp);
    if (!matvec_launch<T>(a, W.nrhs, sp.tabdip != nullptr, st))
        throw EngineError{1, "FFT size not supported by the compiled kernels"};
    vec_launch<0>(LTrans<T>{V, W.st.p, sx, sy, sp.amode, (const cplx<T>*)sp.alpha, sp.nmax}, W.n3, W.nblk, W.nrhs, rs,
                  status, st);
}

template <class T> static bool poll(KrylovWork<T>& W, const SolveSpec& sp, cudaStream_t st, bool& cancelled) {
    IFDDA_CUDA(cudaMemcpyAsync(W.hstatus.data(), W.status.p, W.nrhs * sizeof(int), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    if (sp.cancel && *sp.cancel == -1) {
        cancelled = true;
        return true;
    }
    for (int r = 0; r < W.nrhs; r++)
        if (W.hstatus[r] == 0) return false;
    return true;
}

// Runs the Krylov loop on slot B (right-hand sides) into slot X.  The state
// (tol, maxit) must be set for each right-hand side before the call when
// sp.preset_state is true; otherwise tol/maxit come from sp.
template <class T> bool krylov_run(Green& G, const SolveSpec& sp, KrylovWork<T>& W, cudaStream_t st) {
    Slots<T> V = W.slots();
    const long n3 = W.n3;
    const int nrhs = W.nrhs, nblk = W.nblk;
    RedSlots rs{W.partials.p, W.tickets.p, nblk};
    if (!sp.preset_state) init_state(W.st.p, W.status.p, nrhs, sp.tol, sp.maxit, st);
    IFDDA_CUDA(cudaMemsetAsync(W.tickets.p, 0, nrhs * sizeof(unsigned), st));
    int* status = W.status.p;
    KState* S = W.st.p;
    bool cancelled = false;
    // GPBiCG with its vector steps folded into the mat-vecs (one element per
    // x-pass visit needs an isotropic or absent polarisability)
    // GPBICG2 (method 8) is GPBiCG with the zeta-only step on every even iteration
    const bool gp = sp.method == 1 || sp.method == 8;
    const int every2 = sp.method == 8 ? 1 : 0;
    const bool fused = gp && sp.fuse && sp.amode != ALPHA_FULL;
    MvRed red{};
    if (fused) {
        red = W.mv_red(G.g.ny, G.g.nz);
        IFDDA_CUDA(cudaMemsetAsync(W.mvtk.p, 0, W.mvtk.n * sizeof(unsigned), st));
    }
    const bool tab = sp.tabdip != nullptr;
    const cplx<T>* alpha = (const cplx<T>*)sp.alpha;
    // poll at an even number of iterations so a two-iteration graph fits
    const int every = std::max(2, (sp.check_every + 1) / 2 * 2);
    const int methode = sp.method == 3 ? 2 : 1;
    // one iteration; for GPBiCG `par` selects which t buffer is current
    auto iteration = [&](int par) {
        if (fused) {
            const int tcur = par ? G_TB : G_TA, tnew = par ? G_TA : G_TB;
            MvArgs<T> a1 = mv_args<T>(G, nrhs, V.v(G_P, 0), V.v(G_P, 0), V.v(G_AP, 0), n3, sp.amode, alpha,
                                      sp.nmax, sp.tabdip, status);
            MvArgs<T> a2 = mv_args<T>(G, nrhs, V.v(tnew, 0), V.v(tnew, 0), V.v(G_AT, 0), n3, sp.amode, alpha,
                                      sp.nmax, sp.tabdip, status);
            set_ragged(a1, sp);
            set_ragged(a2, sp);
            if (!matvec_launch_fused<T>(a1, PreGpP<T>{V, S}, EpiGpAlpha<T>{V, S, status}, red, nrhs, tab, st) ||
                !matvec_launch_fused<T>(a2, PreGpYT<T>{V, S, tcur, tnew}, EpiGpZeta<T>{V, S, status, tnew, every2}, red, nrhs,
                                        tab, st))
                throw EngineError{1, "FFT size not supported by the compiled kernels"};
            vec_launch<2>(GpUpdate<T>{V, S, tcur, tnew}, n3, nblk, nrhs, rs, status, st);
        } else if (gp) {
            const int tcur = par ? G_TB : G_TA, tnew = par ? G_TA : G_TB;
            vec_launch<0>(GpP<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, G_P, G_AP, status, st);
            vec_launch<1>(GpAlpha<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<2>(GpYT<T>{V, S, tcur, tnew}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, tnew, G_AT, status, st);
            vec_launch<3>(GpZeta<T>{V, S, tnew, every2}, n3, nblk, nrhs, rs, status, st);
            vec_launch<2>(GpUpdate<T>{V, S, tcur, tnew}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 4) {
            vec_launch<0>(BP<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, B_P, B_V, status, st);
            vec_launch<1>(BXi<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<1>(BS<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, B_S, B_T, status, st);
            vec_launch<2>(BOmega<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<1>(BUpdate<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 12) {
            mv_solver<T>(G, sp, W, R_R, R_AR, status, st);
            vec_launch<1>(CsRho<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<0>(CsD<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, R_D, R_Q, status, st);
            vec_launch<1>(CsAlpha<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<1>(CsUpdate<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 13) {
            mv_solver<T>(G, sp, W, O_R, O_AR, status, st);
            vec_launch<1>(ORho<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<0>(OP<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, O_W4, O_AW4, status, st);
            vec_launch<1>(OAlpha<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<5>(OZeta<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<1>(OUpdate<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 11) {
            mv_solver<T>(G, sp, W, P_R, P_AR, status, st);
            vec_launch<8>(PsCoef<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<0>(PsW<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, P_W4, P_AW4, status, st);
            vec_launch<1>(PsUpdate<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 10) {
            vec_launch<6>(ArAlpha<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<0>(ArU<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, A_U, A_AU, status, st);
            vec_launch<1>(ArUpdate<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, A_R, A_AR, status, st);
            vec_launch<1>(ArBeta<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 7 || sp.method == 9) {
            vec_launch<0>(SfP<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, S_R, S_AR, status, st);
            vec_launch<6>(SfAlpha<T>{V, S, sp.method == 9 ? 1 : 0}, n3, nblk, nrhs, rs, status, st);
            vec_launch<0>(SfU<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, S_U, S_AU, status, st);
            vec_launch<2>(SfUpdate<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 6) {
            if (par == 0) {
                vec_launch<1>(TAlpha<T>{V, S}, n3, nblk, nrhs, rs, status, st);
                vec_launch<1>(TW<T, true>{V, S}, n3, nblk, nrhs, rs, status, st);
                vec_launch<1>(TX<T, false>{V, S}, n3, nblk, nrhs, rs, status, st);
                vec_launch<0>(TU<T, false>{V, S}, n3, nblk, nrhs, rs, status, st);
                mv_solver<T>(G, sp, W, T_U, T_AU, status, st);
                vec_launch<1>(TV<T, false>{V, S}, n3, nblk, nrhs, rs, status, st);
            } else {
                vec_launch<1>(TW<T, false>{V, S}, n3, nblk, nrhs, rs, status, st);
                vec_launch<1>(TX<T, true>{V, S}, n3, nblk, nrhs, rs, status, st);
                vec_launch<0>(TU<T, true>{V, S}, n3, nblk, nrhs, rs, status, st);
                mv_solver<T>(G, sp, W, T_U, T_AU, status, st);
                vec_launch<1>(TV<T, true>{V, S}, n3, nblk, nrhs, rs, status, st);
            }
        } else if (sp.method == 14) {
            vec_launch<1>(LA<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, L_W2, L_W3, status, st);
            vec_launch<3>(LB<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_transpose<T>(G, sp, W, L_W8, L_W9, status, rs, st);
            vec_launch<1>(LC<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<1>(LD<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else if (sp.method == 5) {
            vec_launch<1>(CUpdate<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, C_R, C_S, status, st);
            vec_launch<2>(CBeta<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        } else {
            vec_launch<0>(QP<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, Q_P, Q_V, status, st);
            vec_launch<1>(QAlpha<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<1>(QS<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            mv_solver<T>(G, sp, W, Q_S, Q_T, status, st);
            vec_launch<2>(QOmega<T>{V, S, methode}, n3, nblk, nrhs, rs, status, st);
            vec_launch<2>(QR<T>{V, S}, n3, nblk, nrhs, rs, status, st);
            vec_launch<1>(QX<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        }
        IFDDA_CUDA(cudaGetLastError());
    };
    if (gp) {
        vec_launch<1>(GpStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, G_X, G_XR, status, st);
        vec_launch<1>(GpInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 4) {
        vec_launch<1>(BStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, B_X, B_XR, status, st);
        vec_launch<2>(BInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 12) {
        vec_launch<1>(CsStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, R_X, R_XR, status, st);
        vec_launch<1>(CsInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 13) {
        vec_launch<1>(OStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, O_X, O_XR, status, st);
        vec_launch<0>(OInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 11) {
        vec_launch<1>(PsStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, P_X, P_XR, status, st);
        vec_launch<1>(PsInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 10) {
        vec_launch<1>(ArStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, A_X, A_XR, status, st);
        vec_launch<1>(ArInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        mv_solver<T>(G, sp, W, A_R, A_AR, status, st);
    } else if (sp.method == 7 || sp.method == 9) {
        vec_launch<1>(SfStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, S_X, S_XR, status, st);
        vec_launch<1>(SfInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 6) {
        vec_launch<1>(TStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, T_X, T_XR, status, st);
        vec_launch<0>(TInit1<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        mv_solver<T>(G, sp, W, T_U, T_V, status, st);
        vec_launch<1>(TInit2<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 14) {
        vec_launch<1>(LStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, L_X, L_XR, status, st);
        vec_launch<3>(LInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        mv_transpose<T>(G, sp, W, L_W8, L_W9, status, rs, st);
        vec_launch<1>(LInit2<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else if (sp.method == 5) {
        vec_launch<1>(CStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, C_X, C_XR, status, st);
        vec_launch<2>(CInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
        mv_solver<T>(G, sp, W, C_P, C_W, status, st);
        vec_launch<1>(CXi<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    } else {
        vec_launch<1>(QStart<T>{V, S, sp.zero_guess}, n3, nblk, nrhs, rs, status, st);
        if (!sp.zero_guess) mv_solver<T>(G, sp, W, Q_X, Q_XR, status, st);
        vec_launch<1>(QInit<T>{V, S}, n3, nblk, nrhs, rs, status, st);
    }
    const bool graphs = sp.use_graphs && !timing_active();
    // the buffers and shapes a captured loop is bound to
    std::vector<const void*> key;
    if (graphs) {
        TileChoice tcur;
        const long tile_code = G.tile_choice<T>(tcur) ? 1 + tcur.zvar + 2 * tcur.yvar : 0;
        MvWork<T>& mw = G.work<T>();
        mw.ensure(G.g, nrhs);
        W.loopcount.ensure(1);
        key = {V.base, sp.alpha, sp.tabdip, G.gc<T>(), mw.B1.p, mw.B2.p, W.partials.p, W.tickets.p, status, S,
               W.mvpart.p, W.mvtk.p, W.loopcount.p, (const void*)(long)fused,
               (const void*)(long)sp.method, (const void*)(long)nrhs, (const void*)n3, (const void*)(long)sp.amode,
               (const void*)sp.nmax, (const void*)(long)nblk, sp.gc64_r, sp.gc32_r, sp.alpha_off, sp.tab_off,
               (const void*)(long)tile_code};
    }
    const bool cached = graphs && W.graph.exec && W.graph.key == key;
    // without a loop captured for these buffers, the first two iterations run
    // as plain launches (they also set the kernels' shared-memory limits
    // before any capture); with one, the device-side loop starts at once
    long it = 0;
    bool done = false;
    for (; it < 2 && !done && !cached; it++) {
        iteration((int)(it & 1));
        done = poll(W, sp, st, cancelled);
    }
    // Builds the device-side loop: [clear counter] -> while(cond) { two
    // iterations; k_loop_ctl }.  Returns false (nothing kept) if the driver
    // cannot build it; the caller then replays plain two-iteration graphs.
    constexpr int CHUNK = 32;  // bodies (2 iterations each) per launch, between host checks
    auto build_loop = [&]() -> bool {
        cudaGraph_t g = nullptr;
        if (cudaGraphCreate(&g, 0) != cudaSuccess) return false;
        bool ok = false;
        cudaGraphExec_t ex = nullptr;
        unsigned long long nk = 0;
        do {
            cudaGraphConditionalHandle h;
            if (cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) break;
            cudaMemsetParams mp = {};
            mp.dst = W.loopcount.p;
            mp.value = 0;
            mp.elementSize = sizeof(int);
            mp.width = 1;
            mp.height = 1;
            cudaGraphNode_t nm, nc;
            if (cudaGraphAddMemsetNode(&nm, g, nullptr, 0, &mp) != cudaSuccess) break;
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = h;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            if (cudaGraphAddNode(&nc, g, &nm, 1, &cp) != cudaSuccess) break;
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            if (cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
                cudaSuccess)
                break;
            const unsigned long long c0 = launch_counter().load();
            bool cap_ok = true;
            try {
                iteration(0);
                iteration(1);
                count_launch();
                k_loop_ctl<<<1, 32, 0, st>>>(h, status, nrhs, W.loopcount.p, CHUNK);
            } catch (...) {
                cap_ok = false;
            }
            nk = launch_counter().load() - c0;
            launch_counter().fetch_sub(nk);  // captured, not run
            cudaGraph_t out = nullptr;
            const cudaError_t ee = cudaStreamEndCapture(st, &out);
            if (!cap_ok || ee != cudaSuccess) break;
            if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
                ex = nullptr;
                break;
            }
            ok = true;
        } while (0);
        cudaGraphDestroy(g);
        if (!ok) {
            cudaGetLastError();
            return false;
        }
        W.graph.exec = ex;
        W.graph.kernels = nk;
        W.graph.loop = true;
        W.graph.chunk = CHUNK;
        return true;
    };
    if (!done && graphs) {
        if (!cached) {
            W.graph.reset();
            if (build_loop()) {
                W.graph.key = key;
            } else {
                const unsigned long long c0 = launch_counter().load();
                cudaGraph_t graph;
                IFDDA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                iteration(0);
                iteration(1);
                IFDDA_CUDA(cudaStreamEndCapture(st, &graph));
                const unsigned long long nk = launch_counter().load() - c0;
                launch_counter().fetch_sub(nk);  // captured, not run
                const cudaError_t e = cudaGraphInstantiate(&W.graph.exec, graph, 0);
                cudaGraphDestroy(graph);
                IFDDA_CUDA(e);
                W.graph.key = key;
                W.graph.kernels = nk;
            }
        }
    }
    while (!done) {
        if (graphs && W.graph.exec && W.graph.loop) {
            IFDDA_CUDA(cudaGraphLaunch(W.graph.exec, st));
            int bodies = 0;
            IFDDA_CUDA(cudaMemcpyAsync(&bodies, W.loopcount.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            done = poll(W, sp, st, cancelled);
            count_launch((unsigned)(W.graph.kernels * (unsigned long long)bodies));
            it += 2L * bodies;
            if (it > (long)sp.maxit + 4) break;
            continue;
        }
        for (int k = 0; k < every; k += 2) {
            if (graphs && W.graph.exec) {
                IFDDA_CUDA(cudaGraphLaunch(W.graph.exec, st));
                count_launch((unsigned)W.graph.kernels);
            } else {
                iteration(0);
                iteration(1);
            }
            it += 2;
        }
        done = poll(W, sp, st, cancelled);
        if (it > (long)sp.maxit + 4) break;
    }
    return !cancelled;
}

// Method codes (capi.cu method_code) -> the state machine and slot layout
// they run on: GPBICG2 runs on GPBiCG's (1), GPBICGplus on GPBiCGsafe's (7),
// QMRBICGSTAB2 on QMRBICGSTAB1's (2); GPBICGAR (8), BICGSTARPLUS (9), CORS
// (10) and GPBICOR (11) have their own.
int method_family(int method) {
    switch (method) {
    case 1:
    case 8: return 1;
    case 4: return 4;
    case 5: return 5;
    case 6: return 6;
    case 7:
    case 9: return 7;
    case 10: return 8;
    case 11: return 9;
    case 12: return 10;
    case 13: return 11;
    case 14: return 12;
    default: return 2;
    }
}

template <class T> int KrylovWork<T>::x_slot(int method) const {
    static const int s[] = {0, G_X, Q_X, 0, B_X, C_X, T_X, S_X, A_X, P_X, R_X, O_X, L_X};
    return s[method_family(method)];
}
template <class T> int KrylovWork<T>::b_slot(int method) const {
    static const int s[] = {0, G_B, Q_B, 0, B_B, C_B, T_B, S_B, A_B, P_B, R_B, O_B, L_B};
    return s[method_family(method)];
}
template <class T> int KrylovWork<T>::xr_slot(int method) const {
    static const int s[] = {0, G_XR, Q_XR, 0, B_XR, C_XR, T_XR, S_XR, A_XR, P_XR, R_XR, O_XR, L_XR};
    return s[method_family(method)];
}

// Mat-vecs and iterations the reference's driver counts for a solve that
// ended after `itno` passes of the method's loop (GPBICG: one pass less than
// the iterations it reports, cdmlib/inverserigopt.f:42-107; QMR-BiCGSTAB and
// BiCGSTAB: two mat-vecs per iteration plus the first and the residual one,
// :743-942; CG: one per iteration plus A x0, A p0 and the residual one,
// :676-742; TFQMR: one per pass plus A x0, A u0 and the residual one, and
// the driver adds one to ITNO, :603-675).  atmax: TFQMR or GPBiCGAR stopped
// past MAXIT, whose last pass made the product that a converging pass skips.
void method_counts(int method, int itno, int& nloop, int& ncompte, bool atmax = false) {
    if (method == 14) {
        // QMRCLA (:499-598): A x0, A^T r0, two products per pass and the
        // residual one; its branch does not add one to ITNO
        nloop = itno;
        ncompte = 2 * itno + 3;
    } else if (method == 1 || (method >= 7 && method != 13)) {
        // GPBICG1, GPBICGsafe (:174-237), GPBICG2 (:109-173), GPBICGplus
        // (:238-301), GPBICGAR (:302-366), BICGSTARPLUS (:431-498), CORS
        // (:1009-1072); GPBICOR (:943-1008) counts ITNO from 1 and its driver
        // does not add one, so it counts like QMR-BiCGSTAB
        nloop = itno + 1;
        ncompte = 1 + 2 * (itno + 1) + 1 + (method == 10 && atmax ? 1 : 0);
    } else if (method == 6) {
        nloop = itno + 1;
        ncompte = nloop + 2 + (atmax ? 1 : 0);
    } else if (method == 5) {
        nloop = itno;
        ncompte = itno + 2;
    } else {
        nloop = itno;
        ncompte = 2 + 2 * itno;
    }
}

template struct KrylovWork<float>;
template struct KrylovWork<double>;
template bool krylov_run<float>(Green&, const SolveSpec&, KrylovWork<float>&, cudaStream_t);
template bool krylov_run<double>(Green&, const SolveSpec&, KrylovWork<double>&, cudaStream_t);

// ------------------------------------------------------ public drivers ----
// Plain FP64 solve (the drop-in for inverserig/inverserigopt): the solution
// x, then A x and the true residual, all FP64.
void solve_fp64(Green& G, SolverWork& SW, const SolveSpec& sp, const double2* b_dev, double2* x_out, std::vector<SolveResult>& res,
                cudaStream_t st) {
    KrylovWork<double>& W = SW.kw64;
    tune_tiles<double>(G, sp.nrhs, st);
    W.ensure(sp.method, sp.nrhs, sp.n3);
    // a ragged batch pads shorter objects' vectors with entries no kernel
    // writes: they start at zero and stay zero
    if (sp.tab_off) IFDDA_CUDA(cudaMemsetAsync(W.vecs.p, 0, W.vecs.n * sizeof(double2), st));
    const long tot = (long)sp.nrhs * sp.n3;
    Slots<double> V = W.slots();
    const int bs = W.b_slot(sp.method), xs = W.x_slot(sp.method), xrs = W.xr_slot(sp.method);
    IFDDA_CUDA(cudaMemcpyAsync(V.v(bs, 0), b_dev, tot * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    const bool ok = krylov_run<double>(G, sp, W, st);
    res.assign(sp.nrhs, SolveResult{});
    // W.hstatus holds the statuses the loop's last poll read; they do not
    // change after it.  BiCGSTAB's soft breakdown returns x = p
    // (cdmlib/pimzbicgstab.f:145-156), which needs the state now; the other
    // methods read it once, with tol1, below.
    if (sp.method == 4) {
        std::vector<KState> hs(sp.nrhs);
        IFDDA_CUDA(cudaMemcpyAsync(hs.data(), W.st.p, sp.nrhs * sizeof(KState), cudaMemcpyDeviceToHost, st));
        IFDDA_CUDA(cudaStreamSynchronize(st));
        for (int r = 0; r < sp.nrhs; r++)
            if (W.hstatus[r] < 0 && hs[r].steperr == 12)
                IFDDA_CUDA(cudaMemcpyAsync(V.v(B_X, r), V.v(B_P, r), sp.n3 * sizeof(double2), cudaMemcpyDeviceToDevice,
                                           st));
    }
    // final A x and true residual, for every right-hand side that did not break down
    IFDDA_CUDA(cudaMemsetAsync(W.zstatus.p, 0, sp.nrhs * sizeof(int), st));
    {
        MvArgs<double> a = mv_args<double>(G, sp.nrhs, V.v(xs, 0), V.v(xs, 0), V.v(xrs, 0), sp.n3, sp.amode,
                                           (const double2*)sp.alpha, sp.nmax, sp.tabdip, W.zstatus.p);
        set_ragged(a, sp);
        if (!matvec_launch<double>(a, sp.nrhs, sp.tabdip != nullptr, st))
            throw EngineError{1, "FFT size not supported by the compiled kernels"};
        RedSlots rs{W.partials.p, W.tickets.p, W.nblk};
        vec_launch<1>(TrueResOp{V.v(bs, 0), V.v(xrs, 0), sp.n3, W.st.p}, sp.n3, W.nblk, sp.nrhs, rs, W.zstatus.p, st);
    }
    IFDDA_CUDA(cudaMemcpyAsync(x_out, V.v(xs, 0), tot * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    std::vector<KState> hf(sp.nrhs);
    IFDDA_CUDA(cudaMemcpyAsync(hf.data(), W.st.p, sp.nrhs * sizeof(KState), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    for (int r = 0; r < sp.nrhs; r++) {
        SolveResult& o = res[r];
        o.status = W.hstatus[r];
        o.steperr = hf[r].steperr;  // TrueResOp sets residu only
        o.cancelled = !ok;
        o.tol1 = hf[r].residu;
        method_counts(sp.method, hf[r].itno, o.nloop, o.ncompte, hf[r].atmax != 0);
        o.ncompte64 = o.ncompte;
        o.outer = 0;
    }
}

// Mixed precision: FP32 mat-vec and inner Krylov vectors (FP64 scalars)
// inside FP64 iterative refinement on the true residual.
void solve_mixed(Green& G, SolverWork& SW, const SolveSpec& sp, const double2* b_dev, double2* x_out, std::vector<SolveResult>& res,
                 cudaStream_t st) {
    const int nrhs = sp.nrhs;
    const long n3 = sp.n3, tot = (long)nrhs * n3;
    MixedWork& M = SW.mixed;
    M.x.ensure(tot);
    M.ax.ensure(tot);
    M.alpha32.ensure(sp.amode == ALPHA_FULL ? (size_t)9 * sp.nmax : (size_t)std::max<long>(1, sp.nmax));
    M.ost.ensure(nrhs);
    M.ostatus.ensure(nrhs);
    M.partials.ensure((size_t)nrhs * reduction_blocks(n3) * 4);
    M.tickets.ensure(nrhs);
    KrylovWork<float>& W = SW.kw32;
    tune_tiles<double>(G, nrhs, st);
    tune_tiles<float>(G, nrhs, st);
    W.ensure(sp.method, nrhs, n3);
    if (sp.tab_off) {  // ragged batch: padding entries start at zero (see solve_fp64)
        IFDDA_CUDA(cudaMemsetAsync(W.vecs.p, 0, W.vecs.n * sizeof(float2), st));
        IFDDA_CUDA(cudaMemsetAsync(M.ax.p, 0, tot * sizeof(double2), st));
    }
    const int nblk = reduction_blocks(n3);
    RedSlots rs{M.partials.p, M.tickets.p, nblk};
    // FP32 copy of the polarisability
    if (sp.amode != ALPHA_NONE) {
        const long na = sp.amode == ALPHA_FULL ? 9 * sp.nmax : sp.nmax;
        cast_dev<float>((const double2*)sp.alpha, M.alpha32.p, na, st);
    }
    init_state(M.ost.p, M.ostatus.p, nrhs, sp.tol, sp.maxit, st);
    IFDDA_CUDA(cudaMemsetAsync(M.tickets.p, 0, nrhs * sizeof(unsigned), st));
    // inner state defaults
    init_state(W.st.p, nullptr, nrhs, sp.tol, sp.maxit, st);
    vec_launch<1>(NormOp{b_dev, M.x.p, n3, M.ost.p}, n3, nblk, nrhs, rs, M.ostatus.p, st);
    Slots<float> V = W.slots();
    const int bs = W.b_slot(sp.method), xs = W.x_slot(sp.method);
    SolveSpec isp = sp;
    isp.zero_guess = 1;
    isp.preset_state = true;
    isp.alpha = M.alpha32.p;
    std::vector<int> ost(nrhs, 0), done_before(nrhs, 0);
    res.assign(nrhs, SolveResult{});
    std::vector<long> inner_iters(nrhs, 0), inner_mv(nrhs, 0), outer_mv(nrhs, 0), inner_runs(nrhs, 0);
    bool ok = true;
    int outer = 0;
    bool early = false;  // a copy of x to sp.early_loc has been issued
    // The inner solve's counters are read with the next outer status (one
    // wait instead of two): the residual step that runs between them changes
    // only the inner tol and maxit.  mask: the outer status before that solve.
    std::vector<KState> hs(nrhs);
    std::vector<int> mask(nrhs, 0);
    bool pending = false;
    auto account = [&]() {
        for (int r = 0; r < nrhs; r++) {
            if (mask[r]) continue;
            int its = 0, mvs = 0;
            method_counts(sp.method, hs[r].itno, its, mvs, hs[r].atmax != 0);
            inner_iters[r] += its;
            // zero initial guess: no A x0 (QMRCLA still forms A^T r0)
            if (sp.method == 5 || sp.method == 6) inner_mv[r] += its + 1;
            else if (sp.method == 14) inner_mv[r] += 2 * its + 1;
            else inner_mv[r] += 2 * its;
            if (hs[r].atmax && (sp.method == 6 || sp.method == 10)) inner_mv[r] += 1;
            inner_runs[r] += 1;
        }
        pending = false;
    };
    for (;; outer++) {
        MvArgs<double> a = mv_args<double>(G, nrhs, M.x.p, M.x.p, M.ax.p, n3, sp.amode, (const double2*)sp.alpha,
                                           sp.nmax, sp.tabdip, M.ostatus.p);
        set_ragged(a, sp);
        if (!matvec_launch<double>(a, nrhs, sp.tabdip != nullptr, st))
            throw EngineError{1, "FFT size not supported by the compiled kernels"};
        vec_launch<1>(ResidualOp{b_dev, M.ax.p, V.v(bs, 0), n3, M.ost.p, W.st.p, W.status.p, sp.inner_floor}, n3,
                      nblk, nrhs, rs, M.ostatus.p, st);
        IFDDA_CUDA(cudaMemcpyAsync(ost.data(), M.ostatus.p, nrhs * sizeof(int), cudaMemcpyDeviceToHost, st));
        if (pending)
            IFDDA_CUDA(cudaMemcpyAsync(hs.data(), W.st.p, nrhs * sizeof(KState), cudaMemcpyDeviceToHost, st));
        IFDDA_CUDA(cudaStreamSynchronize(st));
        if (pending) account();
        bool all = true;
        for (int r = 0; r < nrhs; r++) {
            if (!done_before[r]) outer_mv[r]++;
            done_before[r] = ost[r];
            if (!ost[r]) all = false;
        }
        if (all) break;
        if (outer >= sp.max_outer) break;
        if (sp.cancel && *sp.cancel == -1) {
            ok = false;
            break;
        }
        if (!krylov_run<float>(G, isp, W, st)) {
            // cancelled: the iterations and mat-vecs the partial inner run
            // made still count (read after the loop)
            ok = false;
            mask = ost;
            pending = true;
            break;
        }
        mask = ost;
        pending = true;
        // the previous step's copy to the host reads x: it must end first
        if (early) IFDDA_CUDA(cudaStreamWaitEvent(st, sp.loc_copied, 0));
        count_launch();
        k_axpy_outer<float><<<grid_for(tot), 256, 0, st>>>(M.x.p, V.v(xs, 0), n3, nrhs, M.ostatus.p);
        IFDDA_CUDA(cudaGetLastError());
        if (sp.early_loc) {
            IFDDA_CUDA(cudaEventRecord(sp.loc_ready, st));
            IFDDA_CUDA(cudaStreamWaitEvent(sp.early_stream, sp.loc_ready, 0));
            IFDDA_CUDA(cudaMemcpyAsync(sp.early_loc, M.x.p, tot * sizeof(double2), cudaMemcpyDeviceToHost,
                                       sp.early_stream));
            IFDDA_CUDA(cudaEventRecord(sp.loc_copied, sp.early_stream));
            early = true;
        }
    }
    // whatever follows on the solve stream comes after the last host copy
    if (early) IFDDA_CUDA(cudaStreamWaitEvent(st, sp.loc_copied, 0));
    if (pending) {
        IFDDA_CUDA(cudaMemcpyAsync(hs.data(), W.st.p, nrhs * sizeof(KState), cudaMemcpyDeviceToHost, st));
        IFDDA_CUDA(cudaStreamSynchronize(st));
        account();
    }
    std::vector<KState> hf(nrhs);
    IFDDA_CUDA(cudaMemcpyAsync(hf.data(), M.ost.p, nrhs * sizeof(KState), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaMemcpyAsync(x_out, M.x.p, tot * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    for (int r = 0; r < nrhs; r++) {
        SolveResult& o = res[r];
        o.status = ost[r] > 0 ? 1 : ost[r] < 0 ? -1 : 0;
        o.steperr = 0;
        o.cancelled = !ok;
        o.tol1 = hf[r].residu;
        o.nloop = (int)inner_iters[r];
        o.ncompte = (int)(inner_mv[r] + outer_mv[r]);
        o.ncompte64 = (int)outer_mv[r];
        o.outer = (int)inner_runs[r];
        // every step was followed by a copy, so the last one holds x
        o.loc_on_host = early;
    }
}

}  // namespace ifdda
