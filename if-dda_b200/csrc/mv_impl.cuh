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

template <class T, int L, int DIR> void launch_pass_y(const MvArgs<T>& a, int nrhs, cudaStream_t st) {
    using TT = MvTiles<T, L>;
    dim3 grid((a.g.X + TT::TLY - 1) / TT::TLY, a.g.nz, 3 * nrhs);
    PassScope ps(DIR > 0 ? PASS_FWD_Y : PASS_INV_Y, TT::S, st);
    ensure_smem(k_pass_y<T, L, DIR>, TT::smem_y);
    launch_pdl(k_pass_y<T, L, DIR>, grid, TT::NTY, TT::smem_y, st, a);
}

template <class T, int L> void launch_zconv(const MvArgs<T>& a, int nrhs, cudaStream_t st) {
    using TT = MvTiles<T, L>;
    dim3 grid(nrhs, (a.g.X + TT::TLZ - 1) / TT::TLZ, a.g.ny + 1);
    PassScope ps(PASS_ZCONV, TT::S, st);
    ensure_smem(k_zconv<T, L>, TT::smem_z);
    launch_pdl(k_zconv<T, L>, grid, TT::NTZ, TT::smem_z, st, a);
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

}  // namespace ifdda
