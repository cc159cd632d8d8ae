// Launch wrappers for the mat-vec passes, dispatched on the FFT length of each
// axis.  Included by one translation unit per precision.
#pragma once
#include "engine.cuh"

namespace ifdda {

// brackets one pass launch with the optional timing events and counts it
struct PassScope {
    cudaEvent_t ev;
    cudaStream_t st;
    PassScope(int pass, int bytes, cudaStream_t s) : ev(timing_before(pass, bytes, s)), st(s) { count_launch(); }
    ~PassScope() { timing_after(ev, st); }
};

template <class T, int L, class Pre>
void launch_fwd_x(const MvArgs<T>& a, const Pre& pre, const MvRed& red, int nrhs, bool tab, cudaStream_t st) {
    using TT = MvTiles<T, L>;
    dim3 grid((a.g.ny + TT::TLX - 1) / TT::TLX, a.g.nz, nrhs);
    PassScope ps(PASS_FWD_X, TT::S, st);
    if (tab) {
        ensure_smem(k_fwd_x<T, L, true, TT, Pre>, TT::smem_x);
        launch_pdl(k_fwd_x<T, L, true, TT, Pre>, grid, TT::NTX, TT::smem_x, st, a, pre, red);
    } else {
        ensure_smem(k_fwd_x<T, L, false, TT, Pre>, TT::smem_x);
        launch_pdl(k_fwd_x<T, L, false, TT, Pre>, grid, TT::NTX, TT::smem_x, st, a, pre, red);
    }
}

template <class T, int L, int DIR, int V> void launch_pass_y_v(const MvArgs<T>& a, int nrhs, cudaStream_t st) {
    using TT = MvTiles<T, L, V>;
    dim3 grid((a.g.X + TT::TLY - 1) / TT::TLY, a.g.nz, 3 * nrhs);
    PassScope ps(DIR > 0 ? PASS_FWD_Y : PASS_INV_Y, TT::S, st);
    ensure_smem(k_pass_y<T, L, DIR, TT>, TT::smem_y);
    launch_pdl(k_pass_y<T, L, DIR, TT>, grid, TT::NTY, TT::smem_y, st, a);
}
template <class T, int L, int DIR> void launch_pass_y(const MvArgs<T>& a, int nrhs, cudaStream_t st) {
    if constexpr (tile_variants(L) > 1) {
        if (a.yvar == 1) return launch_pass_y_v<T, L, DIR, 1>(a, nrhs, st);
    }
    launch_pass_y_v<T, L, DIR, 0>(a, nrhs, st);
}

template <class T, int L, int V> void launch_zconv_v(const MvArgs<T>& a, int nrhs, cudaStream_t st) {
    using TT = MvTiles<T, L, V>;
    dim3 grid((3 - TT::MRZ) * nrhs, (a.g.X + TT::TLZ - 1) / TT::TLZ, a.g.ny + 1);
    PassScope ps(PASS_ZCONV, TT::S, st);
    ensure_smem(k_zconv<T, L, TT>, TT::smem_z);
    launch_pdl(k_zconv<T, L, TT>, grid, TT::NTZ, TT::smem_z, st, a);
}
template <class T, int L> void launch_zconv(const MvArgs<T>& a, int nrhs, cudaStream_t st) {
    if constexpr (tile_variants(L) > 1) {
        if (a.zvar == 1) return launch_zconv_v<T, L, 1>(a, nrhs, st);
    }
    launch_zconv_v<T, L, 0>(a, nrhs, st);
}

template <class T, int L, class Epi>
void launch_inv_x(const MvArgs<T>& a, const Epi& epi, const MvRed& red, int nrhs, bool tab, cudaStream_t st) {
    using TT = MvTiles<T, L>;
    dim3 grid((a.g.ny + TT::TLX - 1) / TT::TLX, a.g.nz, nrhs);
    PassScope ps(PASS_INV_X, TT::S, st);
    if (tab) {
        ensure_smem(k_inv_x<T, L, true, Epi, TT>, TT::smem_x);
        launch_pdl(k_inv_x<T, L, true, Epi, TT>, grid, TT::NTX, TT::smem_x, st, a, epi, red);
    } else {
        ensure_smem(k_inv_x<T, L, false, Epi, TT>, TT::smem_x);
        launch_pdl(k_inv_x<T, L, false, Epi, TT>, grid, TT::NTX, TT::smem_x, st, a, epi, red);
    }
}

#define IFDDA_CASE_FWDX(L) \
    case L: launch_fwd_x<T, L, Pre>(a, pre, red, nrhs, tab, st); break;
#define IFDDA_CASE_FWDY(L) \
    case L: launch_pass_y<T, L, +1>(a, nrhs, st); break;
#define IFDDA_CASE_INVY(L) \
    case L: launch_pass_y<T, L, -1>(a, nrhs, st); break;
#define IFDDA_CASE_ZC(L) \
    case L: launch_zconv<T, L>(a, nrhs, st); break;
#define IFDDA_CASE_INVX(L) \
    case L: launch_inv_x<T, L, Epi>(a, epi, red, nrhs, tab, st); break;

// The five passes with a solver's input functor (first x pass) and output
// functor (last x pass); red holds their reduction buffers.
template <class T, class Pre, class Epi>
bool matvec_launch_fused(const MvArgs<T>& a, const Pre& pre, const Epi& epi, const MvRed& red, int nrhs, bool tab,
                         cudaStream_t st) {
    if (!fft_length_supported(a.g.X) || !fft_length_supported(a.g.Y) || !fft_length_supported(a.g.Z)) return false;
    switch (a.g.X) { IFDDA_FFT_LENGTHS(IFDDA_CASE_FWDX) default: return false; }
    IFDDA_CUDA(cudaGetLastError());
    switch (a.g.Y) { IFDDA_FFT_LENGTHS(IFDDA_CASE_FWDY) default: return false; }
    IFDDA_CUDA(cudaGetLastError());
    switch (a.g.Z) { IFDDA_FFT_LENGTHS(IFDDA_CASE_ZC) default: return false; }
    IFDDA_CUDA(cudaGetLastError());
    switch (a.g.Y) { IFDDA_FFT_LENGTHS(IFDDA_CASE_INVY) default: return false; }
    IFDDA_CUDA(cudaGetLastError());
    switch (a.g.X) { IFDDA_FFT_LENGTHS(IFDDA_CASE_INVX) default: return false; }
    IFDDA_CUDA(cudaGetLastError());
    return true;
}

#define IFDDA_CASE_TY(L) \
    case L: launch_pass_y<T, L, +1>(a, nrhs, st); launch_pass_y<T, L, -1>(a, nrhs, st); break;
#define IFDDA_CASE_TZ(L) \
    case L: launch_zconv<T, L>(a, nrhs, st); break;

// Tile chooser: with G's mat-vec scratch for nrhs right-hand sides (whose
// contents are about to be overwritten by the next mat-vec anyway), time each
// tile variant of the y passes (forward then inverse) and of zconv, best of
// three launches with CUDA events on st, and record the choice for G's grid,
// device and precision (tile_put: every spectrum and batch size on that grid
// then uses it).  Variant 1 is taken only when it is at least 5% faster, so
// timing noise between near-equal shapes does not flip the choice.  Never
// runs while st is being captured.
template <class T> void tune_tiles_impl(Green& G, int nrhs, cudaStream_t st) {
    const int pk = sizeof(T) == 4 ? 1 : 0;
    TileChoice have;
    if (G.tile_choice<T>(have)) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    IFDDA_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return;
    MvArgs<T> a = mv_args<T>(G, nrhs, nullptr, nullptr, nullptr, 0, ALPHA_NONE, nullptr, 0, nullptr, nullptr);
    TileChoice tc{};
    const int nyv = tile_variants(G.g.Y), nzv = tile_variants(G.g.Z);
    if (nyv > 1 || nzv > 1) {
        cudaEvent_t e0, e1;
        IFDDA_CUDA(cudaEventCreate(&e0));
        IFDDA_CUDA(cudaEventCreate(&e1));
        auto time_it = [&](auto&& launch) {
            float best = 1e30f;
            for (int r = 0; r < 4; r++) {
                IFDDA_CUDA(cudaEventRecord(e0, st));
                launch();
                IFDDA_CUDA(cudaEventRecord(e1, st));
                IFDDA_CUDA(cudaEventSynchronize(e1));
                float ms = 0;
                IFDDA_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                if (r > 0) best = ms < best ? ms : best;  // the first launch sets up the kernel
            }
            return best;
        };
        for (int v = 0; v < nyv; v++) {
            a.yvar = v;
            tc.y_ms[v] = time_it([&] {
                switch (G.g.Y) { IFDDA_FFT_LENGTHS(IFDDA_CASE_TY) default: break; }
            });
            if (tc.y_ms[v] < 0.95f * tc.y_ms[tc.yvar]) tc.yvar = v;
        }
        for (int v = 0; v < nzv; v++) {
            a.zvar = v;
            tc.z_ms[v] = time_it([&] {
                switch (G.g.Z) { IFDDA_FFT_LENGTHS(IFDDA_CASE_TZ) default: break; }
            });
            if (tc.z_ms[v] < 0.95f * tc.z_ms[tc.zvar]) tc.zvar = v;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    tile_put(G.device, pk, G.g, tc);
}

}  // namespace ifdda
