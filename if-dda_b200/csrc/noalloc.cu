// Mat-vec entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they solve: a real-time loop that
// must not hit the device-wide synchronisation cudaMalloc/cudaFree imply, a
// host framework whose own caching allocator owns the device memory and must
// not be bypassed, or an application that has handed its whole device memory
// budget to another library.  ifdda_matvec_device needs B1/B2
// scratch and grows it from the device memory pool on first use; this variant runs the
// same five mat-vec kernels with their scratch in one fixed device array of
// this file instead.
//
// The array (IFDDA_NOALLOC_SCRATCH_BYTES, 16 MiB) is a static __device__
// object: every GPU that loads libifdda_gpu.so holds it until the process
// exits.  Every call shares it and it keeps the last call's contents; no part
// needs to start at zero, because each pass writes every element the next
// pass reads.  Two calls whose kernels overlap on the GPU (different streams
// or different host threads on one device) race on the array.
#include <exception>
#include <mutex>
#include "capi_types.cuh"

#define IFDDA_NOALLOC_SCRATCH_BYTES (16u << 20)

static __device__ __align__(256) unsigned char ifdda_noalloc_scratch[IFDDA_NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_scratch_mu;
void* g_scratch_ptr[64] = {};

// Device address of the scratch array on the current device.  Host code sees
// only a host-side stand-in under the array's name, so the address is looked
// up once per device with cudaGetSymbolAddress and cached.
void* scratch_address(int dev) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (dev < 0 || dev >= 64) throw ifdda::EngineError{1, "ifdda_matvec_noalloc: device ordinal out of range"};
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, ifdda_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw ifdda::EngineError{1, std::string("ifdda_matvec_noalloc: cudaGetSymbolAddress failed: ") +
                                            cudaGetErrorString(e)};
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

template <class T>
bool run_noalloc(ifdda_green* g, int ndip, const int* tabdip_dev, const void* x, void* y, void* scratch) {
    using C = ifdda::cplx<T>;
    ifdda::Green& G = g->G;
    ifdda::MvArgs<T> a{};
    a.g = G.g;
    a.x = (const C*)x;
    a.b = (const C*)y;
    a.y = (C*)y;
    a.xstride = 3L * ndip;
    a.amode = ifdda::ALPHA_NONE;
    a.alpha = nullptr;
    a.nmax = 0;
    a.tabdip = tabdip_dev;
    a.B1 = (C*)scratch;
    a.B2 = a.B1 + G.g.b1_rhs;
    a.Gc = G.gc<T>();
    a.twx = G.tw<T>(0);
    a.twy = G.tw<T>(1);
    a.twz = G.tw<T>(2);
    a.status = nullptr;
    a.inv_m = (T)(1.0 / ((double)G.g.X * G.g.Y * G.g.Z));
    return ifdda::matvec_launch<T>(a, 1, tabdip_dev != nullptr, g->ctx->stream);
}

}  // namespace

extern "C" int ifdda_matvec_noalloc(ifdda_green* g, int precision, int ndip, const int* tabdip_dev,
                                    const void* FFX_dev, void* FFB_dev) {
    if (!g || !FFX_dev || !FFB_dev || ndip < 1) return 1;
    ifdda_ctx* ctx = g->ctx;
    try {
        if (precision != IFDDA_FP32 && precision != IFDDA_FP64)
            throw ifdda::EngineError{1, "ifdda_matvec_noalloc: precision must be IFDDA_FP32 or IFDDA_FP64"};
        int prev = -1;
        IFDDA_CUDA(cudaGetDevice(&prev));
        if (prev != ctx->device) IFDDA_CUDA(cudaSetDevice(ctx->device));
        struct Restore {
            int dev, prev;
            ~Restore() {
                if (prev >= 0 && prev != dev) cudaSetDevice(prev);
            }
        } restore{ctx->device, prev};
        const ifdda::MvGeom& geo = g->G.g;
        if (!tabdip_dev && ndip != g->G.uN)
            throw ifdda::EngineError{1, "ifdda_matvec_noalloc: ndip must be nx*ny*nz without tabdip"};
        // a padded lattice: its Tabdip goes to the buffer the handle holds
        tabdip_dev = lattice_tab(g, tabdip_dev, ctx->stream);
        const size_t elem = precision == IFDDA_FP32 ? sizeof(float2) : sizeof(double2);
        const size_t need = (size_t)(geo.b1_rhs + geo.b2_rhs) * elem;
        if (need > IFDDA_NOALLOC_SCRATCH_BYTES)
            throw ifdda::EngineError{1, "ifdda_matvec_noalloc: the grid needs " + std::to_string(need) +
                                            " bytes of scratch, above the fixed " +
                                            std::to_string((size_t)IFDDA_NOALLOC_SCRATCH_BYTES) + " bytes"};
        void* scratch = scratch_address(ctx->device);
        const bool ok = precision == IFDDA_FP32 ? run_noalloc<float>(g, ndip, tabdip_dev, FFX_dev, FFB_dev, scratch)
                                                : run_noalloc<double>(g, ndip, tabdip_dev, FFX_dev, FFB_dev, scratch);
        if (!ok) throw ifdda::EngineError{1, "FFT size not supported"};
        return 0;
    } catch (const ifdda::EngineError& e) {
        ctx->last_error = e.msg;
        return 1;
    } catch (const std::exception& e) {
        // e.g. std::bad_alloc from an error message, std::system_error from the mutex
        ctx->last_error = e.what();
        return 1;
    }
}
