// Solver workspaces and entry points (host side).
#pragma once
#include "engine.cuh"
#include "krylov_kernels.cuh"

namespace ifdda {

struct SolveSpec {
    int method = 1;        // 1 GPBICG1, 2 QMRBICGSTAB1, 3 QMRBICGSTAB2
    int nrhs = 1;
    long n3 = 0;           // 3 * dipoles
    double tol = 1e-4;
    int maxit = 10000;     // nlim of cdmlib/inverserigopt.f:30
    int check_every = 4;   // iterations launched between status polls
    bool fuse = true;      // GPBiCG vector steps inside the mat-vec x passes (gpbicg_fused.cuh)
    bool use_graphs = true;  // replay captured iterations instead of launching kernels
    int zero_guess = 0;    // x0 = 0 instead of x0 = b
    bool preset_state = false;
    const int* tabdip = nullptr;  // device, lattice -> 1-based dipole, or null (full box)
    int amode = ALPHA_ISO;
    const void* alpha = nullptr;  // device polarisability (precision of the vectors)
    long nmax = 0;
    volatile int* cancel = nullptr;  // host word, -1 cancels (the reference's nstop)
    // mixed precision
    int max_outer = 12;
    double inner_floor = 1e-6;
    // ragged batch (objects of different lattices on one common box, see
    // MvArgs): per right-hand side spectra and offsets, device arrays; null
    // when every right-hand side belongs to one object
    const double2* const* gc64_r = nullptr;
    const float2* const* gc32_r = nullptr;
    const long* alpha_off = nullptr;
    const long* tab_off = nullptr;
    // mixed precision, optional: a page-locked host array (nrhs * n3, the
    // layout of the solution) that receives the solution after every outer
    // step, copied on early_stream while the solve checks the new residual;
    // the copy after the last step is the result.  loc_ready / loc_copied
    // order the copy after the step and the next step after the copy.
    double2* early_loc = nullptr;
    cudaStream_t early_stream = nullptr;
    cudaEvent_t loc_ready = nullptr, loc_copied = nullptr;
};

// a solver's mat-vec arguments carry the ragged-batch tables of its spec
inline void set_ragged(MvArgs<double>& a, const SolveSpec& sp) {
    a.gc_r = sp.gc64_r;
    a.alpha_off = sp.alpha_off;
    a.tab_off = sp.tab_off;
}
inline void set_ragged(MvArgs<float>& a, const SolveSpec& sp) {
    a.gc_r = sp.gc32_r;
    a.alpha_off = sp.alpha_off;
    a.tab_off = sp.tab_off;
}

struct SolveResult {
    int status = 0;     // 1 converged, 0 not converged, -1 breakdown
    int steperr = 0;
    bool cancelled = false;
    double tol1 = 0;    // true FP64 residual ||A x - b|| / ||b||
    int nloop = 0;      // iterations (inner iterations for mixed)
    int ncompte = 0;    // mat-vecs
    int ncompte64 = 0;  // of which FP64
    int outer = 0;      // refinement steps (mixed)
    bool loc_on_host = false;  // early_loc holds the returned solution
};

// Krylov iterations as one CUDA graph, reused while every pointer and size
// baked into its kernel arguments stays the same.  Two iterations make one
// body (the t buffers alternate, so two iterations bring the pointers back).
// With `loop` the body sits in a device-side while node that repeats it until
// every right-hand side has stopped or `chunk` bodies have run (a counter in
// device memory, cleared by the graph), so one launch replaces many host
// polls; otherwise one launch runs the body once.
// Graph executables are not destroyed where they are dropped but queued and
// destroyed in batches (every 256) or when a context is freed: destroying
// one while other threads' solves run on the device measured up to seconds
// per call with four serving threads on B200, against 0.3 ms alone.
void retire_graph_exec(cudaGraphExec_t exec);
void destroy_retired_graph_execs();

struct IterGraph {
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> key;
    unsigned long long kernels = 0;  // kernel launches per body
    bool loop = false;
    int chunk = 0;
    void reset() {
        if (exec) retire_graph_exec(exec);
        exec = nullptr;
        key.clear();
        loop = false;
    }
    ~IterGraph() { reset(); }
};

template <class T> struct KrylovWork {
    IterGraph graph;
    DevBuf<cplx<T>> vecs;
    DevBuf<KState> st;
    DevBuf<int> status, zstatus;
    DevBuf<double2> partials;
    DevBuf<unsigned> tickets;
    DevBuf<double2> mvpart;  // reductions of the fused mat-vecs (MvRed)
    DevBuf<unsigned> mvtk;
    DevBuf<int> loopcount;   // bodies run by the last device-side loop
    std::vector<int> hstatus;
    int nslot = 0, nrhs = 0, nblk = 1;
    long n3 = 0;
    void ensure(int method, int nrhs, long n3);
    MvRed mv_red(int ny, int nz);  // sized for x-pass grids of up to ny x nz blocks
    Slots<T> slots() const;
    int x_slot(int method) const;
    int b_slot(int method) const;
    int xr_slot(int method) const;
    void release() {
        graph.reset();
        vecs.release();
        st.release();
        status.release();
        zstatus.release();
        partials.release();
        tickets.release();
        mvpart.release();
        mvtk.release();
        loopcount.release();
        hstatus.clear();
        nrhs = 0;
        n3 = 0;
    }
};

struct MixedWork {
    DevBuf<double2> x, ax;
    DevBuf<float2> alpha32;
    DevBuf<KState> ost;
    DevBuf<int> ostatus;
    DevBuf<double2> partials;
    DevBuf<unsigned> tickets;
    void release() {
        x.release();
        ax.release();
        alpha32.release();
        ost.release();
        ostatus.release();
        partials.release();
        tickets.release();
    }
};

struct SolverWork {
    KrylovWork<double> kw64;
    KrylovWork<float> kw32;
    MixedWork mixed;
};

int reduction_blocks(long n3);
int method_family(int method);
template <class T> bool krylov_run(Green& G, const SolveSpec& sp, KrylovWork<T>& W, cudaStream_t st);
void solve_fp64(Green& G, SolverWork& SW, const SolveSpec& sp, const double2* b_dev, double2* x_out,
                std::vector<SolveResult>& res, cudaStream_t st);
void solve_mixed(Green& G, SolverWork& SW, const SolveSpec& sp, const double2* b_dev, double2* x_out,
                 std::vector<SolveResult>& res, cudaStream_t st);
void apply_alpha_dev(const double2* x, double2* y, long nd, int nrhs, long stride, int amode, const double2* alpha,
                     long nmax, cudaStream_t st);
template <class T> void cast_dev(const double2* a, cplx<T>* b, long n, cudaStream_t st);

}  // namespace ifdda
