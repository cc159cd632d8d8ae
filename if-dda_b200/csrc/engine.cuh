// Host-side engine types shared by the translation units of libifdda_gpu.so.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <atomic>
#include <mutex>
#include <unordered_map>
#include <map>
#include <utility>
#include "instrument.cuh"
#include "matvec_kernels.cuh"

// FFT lengths (padded grid edges 2n) with compiled kernels.  A lattice edge n
// whose 2n is not in this list runs on the smallest larger edge whose 2n is
// (green_build's pad), so every edge up to 320 is accepted, as the
// reference's own FFT accepts any length, warning above prime factor 5
// (cdmlib/primefactor.f).
#define IFDDA_FFT_LENGTHS(X) \
    X(2) X(4) X(6) X(8) X(10) X(12) X(16) X(20) X(24) X(32) X(40) X(48) X(64) X(80) X(96) X(128) X(160) X(192) X(256) X(320) X(384) \
        X(512) X(640)

namespace ifdda {

bool fft_length_supported(int L);

struct EngineError {
    int code;
    std::string msg;
};

#define IFDDA_CUDA(call)                                                                          \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            throw ::ifdda::EngineError{1, std::string("CUDA error: ") + cudaGetErrorString(e_) + \
                                              " at " + __FILE__ + ":" + std::to_string(__LINE__)}; \
    } while (0)

// Set the dynamic shared-memory limit of a kernel once per (kernel, device).
inline void ensure_smem_ptr(const void* kernel, size_t bytes) {
    static std::mutex mu;
    static std::unordered_map<const void*, uint64_t> done;
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    std::lock_guard<std::mutex> lk(mu);
    uint64_t& m = done[kernel];
    if (m & bit) return;
    if (bytes > 48 * 1024)
        IFDDA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    // prefer the largest shared-memory carveout: the tiles, not L1, hold the data
    IFDDA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared));
    m |= bit;
}
template <class K> inline void ensure_smem(K kernel, size_t bytes) { ensure_smem_ptr((const void*)kernel, bytes); }

// Launch with programmatic dependent launch allowed (see pdl_wait): the
// kernel's blocks may be scheduled during the previous kernel's last wave.
template <class... KP, class... A>
inline void launch_pdl(void (*kernel)(KP...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    IFDDA_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...));
}

// Stream on which DevBuf allocates and frees (stream-ordered, from the
// device's memory pool): the calling entry point sets it to its context's
// stream, so buffers are neither allocated nor freed with a device-wide
// synchronisation and a free is ordered after the work that used the buffer.
inline cudaStream_t& alloc_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}
struct AllocStreamScope {
    cudaStream_t prev;
    explicit AllocStreamScope(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~AllocStreamScope() { alloc_stream() = prev; }
};

template <class T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void ensure(size_t count) {
        if (count <= n) return;
        release();
        IFDDA_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), alloc_stream()));
        n = count;
    }
    void release() {
        if (p) cudaFreeAsync(p, alloc_stream());
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
};

// mat-vec scratch for one precision: B1 and B2 for up to `cap` right-hand sides
template <class T> struct MvWork {
    DevBuf<cplx<T>> B1, B2;
    void ensure(const MvGeom& g, int nrhs) {
        B1.ensure((size_t)g.b1_rhs * nrhs);
        B2.ensure((size_t)g.b2_rhs * nrhs);
    }
};

// Tile variants chosen by the tile chooser for one (precision, batch), with
// the times it measured (ms; 0 where a variant was not timed).
struct TileChoice {
    int zvar = 0, yvar = 0;
    float z_ms[2] = {0, 0}, y_ms[2] = {0, 0};
};

// Tile chooser results, one per (device, precision 0 FP64 / 1 FP32, grid
// X x Y x Z), shared by every spectrum on that grid and every batch size: a
// request stream of many spectra on few grids times each grid once, and a
// right-hand side runs the same kernels alone and in a batch (the shapes can
// differ in the last bits where the compiler contracts multiply-adds
// differently, so one grid keeps one shape).
bool tile_get(int dev, int prec, const MvGeom& g, TileChoice& out);
void tile_put(int dev, int prec, const MvGeom& g, const TileChoice& tc);
void tile_erase(int dev, int prec, const MvGeom& g);

// Green spectrum of one (lattice, spacing, wavenumber), device resident.
struct Green {
    int device = 0;
    MvGeom g{};
    // the caller's lattice; g is larger where 2 nx, 2 ny or 2 nz is not a
    // compiled FFT length, the lattice then sitting at the corner of g's
    int ux = 0, uy = 0, uz = 0;
    long uN = 0;
    bool padded() const { return ux != g.nx || uy != g.ny || uz != g.nz; }
    double d = 0, k0 = 0;
    int nquad = 0;
    DevBuf<double2> gc64;
    DevBuf<float2> gc32;
    DevBuf<double2> tw64[3];
    DevBuf<float2> tw32[3];
    MvWork<float> w32;
    MvWork<double> w64;
    // the tile chooser's result for this grid (shared with every spectrum on
    // the same grid and device) and precision T
    template <class T> bool tile_choice(TileChoice& out) const;
    template <class T> const cplx<T>* gc() const;
    template <class T> const cplx<T>* tw(int axis) const;
    template <class T> MvWork<T>& work();
};
template <> inline const float2* Green::gc<float>() const { return gc32.p; }
template <> inline const double2* Green::gc<double>() const { return gc64.p; }
template <> inline const float2* Green::tw<float>(int a) const { return tw32[a].p; }
template <> inline const double2* Green::tw<double>(int a) const { return tw64[a].p; }
template <> inline MvWork<float>& Green::work<float>() { return w32; }
template <> inline MvWork<double>& Green::work<double>() { return w64; }
template <class T> inline bool Green::tile_choice(TileChoice& out) const {
    return tile_get(device, sizeof(T) == 4 ? 1 : 0, g, out);
}

MvGeom make_geom(int nx, int ny, int nz);
// builds the spectrum (FP64, plus an FP32 copy) on `st`; throws EngineError
// nquad > 0: the cube-averaged tensor at offsets within nquad (calculgreenquadfft.f)
// pad: a lattice side n whose 2 n is not a compiled length is padded to the
// smallest n' > n whose 2 n' is (the spectrum of the larger box holds the same
// tensor at every offset between the caller's sites)
// box: explicit sides (bx, by, bz) of the grid's box, each at least the
// lattice's, instead of the padding rule (a ragged batch's common box)
void green_build(Green& G, int nx, int ny, int nz, double d, double k0, cudaStream_t st, int nquad = 0,
                 bool pad = false, const int* box = nullptr);
// the spectrum of G's lattice (and nquad, padding) for another spacing and
// wavenumber, into G's own buffers (its solver workspaces stay valid)
void green_recompute(Green& G, double d, double k0, cudaStream_t st);
// full FFTTENSOR arrays (6 x 8N) on the host, expanded from the compressed octant
void green_export(const Green& G, double2* const out[6], cudaStream_t st);

// The five mat-vec passes.  Returns false if a length has no compiled kernel.
template <class T> bool matvec_launch(const MvArgs<T>& a, int nrhs, bool tab, cudaStream_t st);
// The same with a solver's input functor in the first x pass and output
// functor in the last one (gpbicg_fused.cuh); red holds their reductions.
template <class T, class Pre, class Epi>
bool matvec_launch_fused(const MvArgs<T>& a, const Pre& pre, const Epi& epi, const MvRed& red, int nrhs, bool tab,
                         cudaStream_t st);

// fill MvArgs from a Green object and the caller's vectors
template <class T>
MvArgs<T> mv_args(Green& G, int nrhs, const cplx<T>* x, const cplx<T>* b, cplx<T>* y, long xstride, int amode,
                  const cplx<T>* alpha, long nmax, const int* tabdip, const int* status) {
    MvArgs<T> a{};
    a.g = G.g;
    a.x = x;
    a.b = b;
    a.y = y;
    a.xstride = xstride;
    a.amode = amode;
    a.alpha = alpha;
    a.nmax = nmax;
    a.tabdip = tabdip;
    MvWork<T>& w = G.work<T>();
    w.ensure(G.g, nrhs);
    a.B1 = w.B1.p;
    a.B2 = w.B2.p;
    a.Gc = G.gc<T>();
    a.twx = G.tw<T>(0);
    a.twy = G.tw<T>(1);
    a.twz = G.tw<T>(2);
    a.status = status;
    a.inv_m = (T)(1.0 / ((double)G.g.X * G.g.Y * G.g.Z));
    TileChoice tc;
    if (G.tile_choice<T>(tc)) {
        a.zvar = tc.zvar;
        a.yvar = tc.yvar;
    }
    return a;
}

// time the tile variants of T on G's grid once (with nrhs right-hand sides),
// see mv_impl.cuh
template <class T> void tune_tiles(Green& G, int nrhs, cudaStream_t st);

}  // namespace ifdda
