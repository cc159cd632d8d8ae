// Definitions of the opaque C-ABI handles, shared by the translation units
// that implement entry points.
#pragma once
#include <string>
#include "../../include/ifdda_gpu.h"
#include "post.cuh"

struct ifdda_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // host-to-device uploads of ifdda_inverserig(_batch) that need no
    // allocation run here, so that they overlap the work already queued on
    // `stream`; `upload_done` orders the solve after them
    cudaStream_t upload_stream = nullptr;
    cudaEvent_t upload_done = nullptr;
    // a mixed solve's copies of the local field to the caller's page-locked
    // FFloc run on upload_stream too (SolveSpec::early_loc)
    cudaEvent_t loc_ready = nullptr, loc_copied = nullptr;
    std::string last_error;
    ifdda::DevBuf<int> flag;  // device error flag for post kernels
    ifdda::DevBuf<double2> partials;
    ifdda::DevBuf<unsigned> tickets;
    ifdda::DevBuf<ifdda::KState> st;
    ifdda::DevBuf<int> zstatus;
    // spectra created on this context and not yet destroyed; a destroy
    // request while some are alive is carried out by the last one's destroy
    int live_greens = 0;
    bool closing = false;
};

struct ifdda_green {
    ifdda_ctx* ctx = nullptr;
    ifdda::Green G;
    ifdda::SolverWork SW;
    // per-call device copies
    ifdda::DevBuf<int> tab;
    // Tabdip of the padded box (G.padded()): allocated with the handle
    ifdda::DevBuf<int> ptab;
    ifdda::DevBuf<double2> alpha, ff0, x, ffx, ffb;
    // incident fields and polarisabilities uploaded by ifdda_inverserig(_batch)
    // alone (no other entry point queues work on them, so an upload on the
    // context's upload stream cannot overwrite a buffer a queued kernel reads)
    ifdda::DevBuf<double2> up_ff0, up_alpha;
    ifdda::DevBuf<float2> ffx32, ffb32, alpha32;
    // a ragged batch solved with this handle's workspaces (the first object
    // of ifdda_inverserig_ragged): concatenated Tabdips and polarisabilities,
    // per right-hand side spectra and offsets
    ifdda::DevBuf<int> rtab, rtab_in;
    ifdda::DevBuf<double2> ralpha;
    ifdda::DevBuf<const double2*> rgc64;
    ifdda::DevBuf<const float2*> rgc32;
    ifdda::DevBuf<long> roff;
};

// The Tabdip the mat-vec kernels use for a lattice Tabdip src (device,
// caller's lattice; null for a full box): src itself, or, when the handle's
// lattice was padded to compiled FFT lengths, its padded form in g->ptab
const int* lattice_tab(ifdda_green* g, const int* src, cudaStream_t st);
