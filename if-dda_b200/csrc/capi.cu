// C-ABI of libifdda_gpu.so (declarations and reference seams: include/ifdda_gpu.h).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>
#include <string>
#include "../../include/ifdda_gpu.h"
#include "post.cuh"
#include "microscope.cuh"

using namespace ifdda;

#include "capi_types.cuh"

static void set_info(char* infostr, const char* msg) {
    if (!infostr) return;
    const size_t L = std::min<size_t>(strlen(msg), 64);
    memset(infostr, ' ', 64);
    memcpy(infostr, msg, L);
}

#define IFDDA_GUARD_BEGIN try {
#define IFDDA_GUARD_END(ctxp, info)                           \
    }                                                         \
    catch (const EngineError& e) {                            \
        if (ctxp) (ctxp)->last_error = e.msg;                 \
        set_info(info, e.msg.c_str());                        \
        return 1;                                             \
    }                                                         \
    catch (const std::exception& e) {                         \
        if (ctxp) (ctxp)->last_error = e.what();              \
        set_info(info, e.what());                             \
        return 1;                                             \
    }

namespace {
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) IFDDA_CUDA(cudaSetDevice(dev));
    }
    ~DeviceScope() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// A polarisability is stored compactly when every dipole's tensor is the
// same complex number times the identity (every object of the reference
// built with trope = 'iso').
bool pola_iso_range(const ifdda_dcmplx* pol, long i0, long i1, long nmax, const std::atomic<bool>& stop) {
    for (long i = i0; i < i1; i++) {
        if ((i & 4095) == 0 && stop.load(std::memory_order_relaxed)) return false;
        const ifdda_dcmplx d0 = pol[i];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                const ifdda_dcmplx v = pol[i + nmax * (a + 3 * b)];
                if (a == b) {
                    if (v.re != d0.re || v.im != d0.im) return false;
                } else if (v.re != 0.0 || v.im != 0.0) {
                    return false;
                }
            }
    }
    return true;
}

// Isotropy of dipoles [b0, b1): the scan reads 9 complex numbers of host
// memory per dipole; large ranges are split over up to 16 host threads (one
// chunk of at least 16K dipoles each).
int pola_mode_range(const ifdda_dcmplx* pol, long b0, long b1, long nmax) {
    constexpr long CHUNK = 16384;
    const long nb = b1 - b0;
    if (nb <= 0) return ALPHA_ISO;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::min<long>({(long)hw, 16L, std::max(1L, (nb + CHUNK - 1) / CHUNK)});
    std::atomic<bool> stop{false};
    if (nt == 1) return pola_iso_range(pol, b0, b1, nmax, stop) ? ALPHA_ISO : ALPHA_FULL;
    std::vector<std::thread> th;
    std::vector<char> iso(nt, 1);
    const long per = (nb + nt - 1) / nt;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t] {
            const long i0 = b0 + t * per, i1 = std::min<long>(b1, i0 + per);
            if (i0 < i1 && !pola_iso_range(pol, i0, i1, nmax, stop)) {
                iso[t] = 0;
                stop.store(true, std::memory_order_relaxed);
            }
        });
    for (auto& x : th) x.join();
    for (int t = 0; t < nt; t++)
        if (!iso[t]) return ALPHA_FULL;
    return ALPHA_ISO;
}

// every tabdip entry must name a dipole in [1, ndip] or be 0 (empty site)
void check_tabdip(const int* tab, long nsites, int ndip) {
    for (long s = 0; s < nsites; s++)
        if (tab[s] < 0 || tab[s] > ndip) throw EngineError{1, "tabdip entry out of range [0, nbsphere]"};
}

int method_code(const char* m) {
    char buf[13];
    memset(buf, ' ', 12);
    buf[12] = 0;
    if (m) memcpy(buf, m, std::min<size_t>(strnlen(m, 12), 12));
    // the reference's elseif chain (cdmlib/inverserigopt.f:42-1009) compares
    // prefixes of the blank-padded character(12) methodeit, in this order;
    // any other string answers "Iterative method not correct!"
    if (!strncmp(buf, "GPBICG1", 7)) return 1;
    if (!strncmp(buf, "GPBICG2", 7)) return 8;
    if (!strncmp(buf, "GPBICGsafe", 10)) return 7;
    if (!strncmp(buf, "GPBICGplus", 10)) return 9;
    if (!strncmp(buf, "GPBICGAR", 8)) return 10;  // 'GPBICGAR2' too: (1:8) is tested first
    if (!strncmp(buf, "BICGSTARPLUS", 12)) return 11;
    if (!strncmp(buf, "QMRCLA", 6)) return 14;
    if (!strncmp(buf, "TFQMR", 5)) return 6;
    if (!strncmp(buf, "CG   ", 5)) return 5;
    if (!strncmp(buf, "BICGSTAB", 8)) return 4;
    if (!strncmp(buf, "QMRBICGSTAB1", 12)) return 2;
    if (!strncmp(buf, "QMRBICGSTAB2", 12)) return 3;
    if (!strncmp(buf, "GPBICOR", 7)) return 13;
    if (!strncmp(buf, "CORS   ", 7)) return 12;
    return 0;
}

SolveSpec make_spec(int method, int nrhs, int nb, double tol, const ifdda_solve_options* opt) {
    SolveSpec sp;
    sp.method = method;
    sp.nrhs = nrhs;
    sp.n3 = 3L * nb;
    sp.tol = tol;
    if (opt) {
        if (opt->check_every > 0) sp.check_every = opt->check_every;
        if (opt->max_outer > 0) sp.max_outer = opt->max_outer;
        if (opt->inner_floor > 0) sp.inner_floor = opt->inner_floor;
        if (opt->maxit > 0) sp.maxit = opt->maxit;
    }
    return sp;
}

int report_results(const std::vector<SolveResult>& res, int method, double tol, bool check_tol, double* tol1,
                   int* nloop, int* ncompte, int* nstop, char* infostr);

// Runs a (batched) solve whose inputs are already on the device.
// check_tol: report tol1 >= tol as "Converge do not reach!" (cdmlib.f:1586-1591;
// the microscopes call the solver without that check).  sync_out: return with
// FF computed; a caller that next copies the outputs on the same stream and
// waits there passes false.  early_loc: a page-locked host array for the
// local field that a mixed solve fills on the context's upload stream after
// each refinement step (SolveSpec::early_loc); *loc_on_host tells whether it
// holds the result (the solve stream is ordered after that copy).
int solve_device(ifdda_green* g, int nrhs, int nb, int nmax, const int* tab_dev, const double2* alpha_dev, int amode,
                 const double2* ff0_dev, const char* methodeit, double tol, double2* ff_dev, double2* loc_dev,
                 double* tol1, int* nloop, int* ncompte, int* nstop, char* infostr, const ifdda_solve_options* opt,
                 bool check_tol = true, bool sync_out = true, double2* early_loc = nullptr,
                 bool* loc_on_host = nullptr) {
    if (loc_on_host) *loc_on_host = false;
    ifdda_ctx* ctx = g->ctx;
    const int method = method_code(methodeit);
    if (method == 0) {
        if (nstop) *nstop = 1;
        set_info(infostr, "Iterative method not correct!");
        return 1;
    }
    // cdmlib/cdmlib.f:462-471 rejects tolerances outside [1e-12, 0.5]
    if (tol < 1e-12) {
        if (nstop) *nstop = 1;
        set_info(infostr, "Tolerance for the iterative method too small!");
        return 1;
    }
    if (tol > 0.5) {
        if (nstop) *nstop = 1;
        set_info(infostr, "Tolerance  for the iterative method too large!");
        return 1;
    }
    SolveSpec sp = make_spec(method, nrhs, nb, tol, opt);
    sp.tabdip = tab_dev;
    sp.amode = amode;
    sp.alpha = alpha_dev;
    sp.nmax = amode == ALPHA_FULL ? nmax : nb;
    sp.cancel = (volatile int*)nstop;
    if (nstop && *nstop == -1) {
        set_info(infostr, "Calculation cancelled during iterative method");
        return -1;
    }
    const int prec = opt ? opt->precision : IFDDA_FP64;
    std::vector<SolveResult> res;
    if (prec == IFDDA_MIXED && early_loc) {
        sp.early_loc = early_loc;
        sp.early_stream = ctx->upload_stream;
        sp.loc_ready = ctx->loc_ready;
        sp.loc_copied = ctx->loc_copied;
    }
    if (prec == IFDDA_MIXED) solve_mixed(g->G, g->SW, sp, ff0_dev, loc_dev, res, ctx->stream);
    else solve_fp64(g->G, g->SW, sp, ff0_dev, loc_dev, res, ctx->stream);
    if (loc_on_host) *loc_on_host = !res.empty() && res[0].loc_on_host;
    // FF = polarisa . E (cdmlib/inverserigopt.f:92-97)
    apply_alpha_dev(loc_dev, ff_dev, nb, nrhs, 3L * nb, amode, alpha_dev, sp.nmax, ctx->stream);
    if (sync_out) IFDDA_CUDA(cudaStreamSynchronize(ctx->stream));
    return report_results(res, method, tol, check_tol, tol1, nloop, ncompte, nstop, infostr);
}

// Counters of every right-hand side and the nstop / infostr of the first one
// that failed, as the reference reports a solve (cdmlib/cdmlib.f:1586-1591,
// cdmlib/inverserigopt.f:47, :86, :609).
int report_results(const std::vector<SolveResult>& res, int method, double tol, bool check_tol, double* tol1,
                   int* nloop, int* ncompte, int* nstop, char* infostr) {
    const int nrhs = (int)res.size();
    int rc = 0;
    const char* msg = nullptr;
    for (int r = 0; r < nrhs; r++) {
        if (tol1) tol1[r] = res[r].tol1;
        if (nloop) nloop[r] = res[r].nloop;
        if (ncompte) ncompte[r] = res[r].ncompte;
        if (rc) continue;
        if (res[r].cancelled) {
            rc = -1;
            msg = "Calculation cancelled during iterative method";
        } else if (res[r].status < 0) {
            rc = 1;
            // the TFQMR branch of the reference words it without '!'
            // (cdmlib/inverserigopt.f:609)
            msg = method == 6 ? "Problem to solve Ax=b" : "Problem to solve Ax=b!";
        } else if (check_tol && !(res[r].tol1 < tol)) {
            rc = 1;
            msg = "Converge do not reach!";
        }
    }
    if (nstop) *nstop = rc;
    if (msg) set_info(infostr, msg);
    else if (infostr) memset(infostr, ' ', 64);
    return rc;
}
}  // namespace

// Tabdip of a padded lattice (Green::padded): site (i, j, k) of the caller's
// ux x uy x uz lattice maps to its dipole (src[site], or site + 1 for a full
// box without src), the padding sites to none
__global__ void k_pad_tab(const int* __restrict__ src, int* __restrict__ dst, int ux, int uy, int uz, int px, int py,
                          long np) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < np; q += (long)gridDim.x * blockDim.x) {
        const int i = (int)(q % px);
        const long r = q / px;
        const int j = (int)(r % py), k = (int)(r / py);
        int v = 0;
        if (i < ux && j < uy && k < uz) {
            const long s = i + (long)ux * (j + (long)uy * k);
            v = src ? src[s] : (int)(s + 1);
        }
        dst[q] = v;
    }
}

// The Tabdip the kernels use: src (device, caller's lattice, or null for a
// full box) itself, or its padded form in buf (G.g.N entries)
static const int* lattice_tab(const Green& G, int* buf, const int* src, cudaStream_t st) {
    if (!G.padded()) return src;
    const long np = G.g.N;
    count_launch();
    k_pad_tab<<<(int)std::min<long>((np + 255) / 256, 148L * 16), 256, 0, st>>>(src, buf, G.ux, G.uy, G.uz, G.g.nx,
                                                                               G.g.ny, np);
    IFDDA_CUDA(cudaGetLastError());
    return buf;
}
const int* lattice_tab(ifdda_green* g, const int* src, cudaStream_t st) {
    return lattice_tab(g->G, g->ptab.p, src, st);
}

// Ragged batch; the per-object arrays are host memory (dev = false) or
// device memory of the context's device (dev = true).
static int ragged_solve(int nobj, ifdda_green* const* greens, const int* nrhs, const int* nbsphere, const int* nmax,
                        const int* const* tabdip, const ifdda_dcmplx* const* polarisa, const ifdda_dcmplx* const* FF0,
                        const char* methodeit, double tol, ifdda_dcmplx* const* FF, ifdda_dcmplx* const* FFloc,
                        double* tol1, int* nloop, int* ncompte, int* nstop, char* infostr,
                        const ifdda_solve_options* opt, bool dev) {
    if (nobj < 1 || !greens || !greens[0] || !nrhs || !nbsphere || !nmax || !polarisa || !FF0 || !FF || !FFloc) {
        if (nstop) *nstop = 1;
        set_info(infostr, "invalid argument");
        return 1;
    }
    ifdda_green* g0 = greens[0];
    ifdda_ctx* ctx = g0->ctx;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    const int method = method_code(methodeit);
    if (method == 0) {
        if (nstop) *nstop = 1;
        set_info(infostr, "Iterative method not correct!");
        return 1;
    }
    if (method == 14) throw EngineError{1, "ragged batch: QMRCLA is not supported (its A^T products)"};
    if (tol < 1e-12 || tol > 0.5) throw EngineError{1, "ragged batch: tolerance outside [1e-12, 0.5]"};
    const MvGeom& box = g0->G.g;
    long R = 0, nbmax = 0, nalpha = 0;
    for (int i = 0; i < nobj; i++) {
        ifdda_green* g = greens[i];
        if (!g || g->ctx != ctx) throw EngineError{1, "ragged batch: every spectrum must belong to one context"};
        if (g->G.g.nx != box.nx || g->G.g.ny != box.ny || g->G.g.nz != box.nz || g->G.nquad != 0)
            throw EngineError{1, "ragged batch: every spectrum must be on one box (ifdda_green_create_box), nquad 0"};
        if (nrhs[i] < 1 || nbsphere[i] < 1 || nmax[i] < nbsphere[i] || !polarisa[i] || !FF0[i] || !FF[i] ||
            !FFloc[i])
            throw EngineError{1, "ragged batch: invalid object " + std::to_string(i)};
        if (!(tabdip && tabdip[i]) && nbsphere[i] != g->G.uN)
            throw EngineError{1, "ragged batch: a full-box object needs nbsphere = nx*ny*nz"};
        if (!dev && tabdip && tabdip[i]) check_tabdip(tabdip[i], g->G.uN, nbsphere[i]);
        if (!dev && pola_mode_range(polarisa[i], 0, nbsphere[i], nmax[i]) != ALPHA_ISO)
            throw EngineError{1, "ragged batch: only isotropic polarisabilities are supported"};
        R += nrhs[i];
        nbmax = std::max<long>(nbmax, nbsphere[i]);
        nalpha += nbsphere[i];
    }
    // every right-hand side is laid out on the box's sites (not on the batch's
    // largest object), so its vector length, reductions and kernels' work do
    // not depend on the other objects of the batch: a request gives the same
    // bits alone and inside any ragged batch on that box
    const long Nb = box.N, n3 = 3 * Nb, tot = R * n3;
    if (nbmax > Nb) throw EngineError{1, "ragged batch: an object has more dipoles than the box has sites"};
    g0->ff0.ensure(tot);
    g0->x.ensure(tot);
    g0->ffb.ensure(tot);
    g0->ralpha.ensure(nalpha);
    g0->rtab.ensure((size_t)nobj * Nb);
    g0->rgc64.ensure(R);
    g0->rgc32.ensure(R);
    g0->roff.ensure(2 * R);
    const cudaMemcpyKind in_kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out_kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (dev) IFDDA_CUDA(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), st));
    // right-hand sides of every object, each zero-padded to 3 Nbox
    IFDDA_CUDA(cudaMemsetAsync(g0->ff0.p, 0, tot * sizeof(double2), st));
    std::vector<const double2*> h64(R);
    std::vector<const float2*> h32(R);
    std::vector<long> hoff(2 * R);
    std::vector<long> aoff(nobj), roff(nobj);
    long r0 = 0, a0 = 0;
    for (int i = 0; i < nobj; i++) {
        ifdda_green* g = greens[i];
        const long n3i = 3L * nbsphere[i];
        for (int q = 0; q < nrhs[i]; q++) {
            IFDDA_CUDA(cudaMemcpyAsync(g0->ff0.p + (r0 + q) * n3, FF0[i] + q * n3i, n3i * sizeof(double2), in_kind,
                                       st));
            h64[r0 + q] = g->G.gc64.p;
            h32[r0 + q] = g->G.gc32.p;
            hoff[r0 + q] = a0;
            hoff[R + r0 + q] = (long)i * Nb;
        }
        // the isotropic value of dipole n is polarisa(n,1,1): the first
        // nbsphere entries of the (nmax,3,3) array (on the device, checked
        // for isotropy as it is compacted)
        if (dev)
            pola_compact_dev((const double2*)polarisa[i], nbsphere[i], nmax[i], g0->ralpha.p + a0, ctx->flag.p, st);
        else
            IFDDA_CUDA(cudaMemcpyAsync(g0->ralpha.p + a0, polarisa[i], nbsphere[i] * sizeof(double2),
                                       cudaMemcpyHostToDevice, st));
        // the object's Tabdip on the common box (identity for a full box)
        const int* src = nullptr;
        if (dev && tabdip && tabdip[i]) {
            src = tabdip[i];
        } else if (tabdip && tabdip[i]) {
            g0->rtab_in.ensure(g->G.uN);
            IFDDA_CUDA(cudaMemcpyAsync(g0->rtab_in.p, tabdip[i], g->G.uN * sizeof(int), cudaMemcpyHostToDevice, st));
            src = g0->rtab_in.p;
        }
        count_launch();
        k_pad_tab<<<(int)std::min<long>((Nb + 255) / 256, 148L * 16), 256, 0, st>>>(
            src, g0->rtab.p + (long)i * Nb, g->G.ux, g->G.uy, g->G.uz, box.nx, box.ny, Nb);
        IFDDA_CUDA(cudaGetLastError());
        // rtab_in is reused by the next object: its copy must be done
        if (src && !dev) IFDDA_CUDA(cudaStreamSynchronize(st));
        aoff[i] = a0;
        roff[i] = r0;
        r0 += nrhs[i];
        a0 += nbsphere[i];
    }
    IFDDA_CUDA(cudaMemcpyAsync(g0->rgc64.p, h64.data(), R * sizeof(const double2*), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(g0->rgc32.p, h32.data(), R * sizeof(const float2*), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(g0->roff.p, hoff.data(), 2 * R * sizeof(long), cudaMemcpyHostToDevice, st));
    SolveSpec sp = make_spec(method, (int)R, (int)Nb, tol, opt);
    sp.tabdip = g0->rtab.p;
    sp.amode = ALPHA_ISO;
    sp.alpha = g0->ralpha.p;
    sp.nmax = nalpha;
    sp.cancel = (volatile int*)nstop;
    sp.gc64_r = g0->rgc64.p;
    sp.gc32_r = g0->rgc32.p;
    sp.alpha_off = g0->roff.p;
    sp.tab_off = g0->roff.p + R;
    if (dev) {
        int aniso = 0;
        IFDDA_CUDA(cudaMemcpyAsync(&aniso, ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
        IFDDA_CUDA(cudaStreamSynchronize(st));
        if (aniso) throw EngineError{1, "ragged batch: only isotropic polarisabilities are supported"};
    }
    if (nstop && *nstop == -1) {
        set_info(infostr, "Calculation cancelled during iterative method");
        return -1;
    }
    std::vector<SolveResult> res;
    if (opt && opt->precision == IFDDA_MIXED) solve_mixed(g0->G, g0->SW, sp, g0->ff0.p, g0->x.p, res, st);
    else solve_fp64(g0->G, g0->SW, sp, g0->ff0.p, g0->x.p, res, st);
    for (int i = 0; i < nobj; i++) {
        const long n3i = 3L * nbsphere[i];
        // FF = polarisa . E (cdmlib/inverserigopt.f:92-97), per object
        apply_alpha_dev(g0->x.p + roff[i] * n3, g0->ffb.p + roff[i] * n3, nbsphere[i], nrhs[i], n3, ALPHA_ISO,
                        g0->ralpha.p + aoff[i], nbsphere[i], st);
        for (int q = 0; q < nrhs[i]; q++) {
            IFDDA_CUDA(cudaMemcpyAsync(FFloc[i] + q * n3i, g0->x.p + (roff[i] + q) * n3, n3i * sizeof(double2),
                                       out_kind, st));
            IFDDA_CUDA(cudaMemcpyAsync(FF[i] + q * n3i, g0->ffb.p + (roff[i] + q) * n3, n3i * sizeof(double2),
                                       out_kind, st));
        }
    }
    IFDDA_CUDA(cudaStreamSynchronize(st));
    return report_results(res, method, tol, true, tol1, nloop, ncompte, nstop, infostr);
    IFDDA_GUARD_END(ctx, infostr)
}

extern "C" {

int ifdda_abi_version(void) { return IFDDA_GPU_ABI_VERSION; }

int ifdda_ctx_create(int device, ifdda_ctx** out) {
    if (!out) return 1;
    *out = nullptr;
    auto* c = new ifdda_ctx();
    try {
        int n = 0;
        IFDDA_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw EngineError{1, "no such CUDA device"};
        c->device = device;
        DeviceScope ds(device);
        IFDDA_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        IFDDA_CUDA(cudaStreamCreateWithFlags(&c->upload_stream, cudaStreamNonBlocking));
        IFDDA_CUDA(cudaEventCreateWithFlags(&c->upload_done, cudaEventDisableTiming));
        IFDDA_CUDA(cudaEventCreateWithFlags(&c->loc_ready, cudaEventDisableTiming));
        IFDDA_CUDA(cudaEventCreateWithFlags(&c->loc_copied, cudaEventDisableTiming));
        AllocStreamScope as(c->stream);
        // keep freed blocks in the device's memory pool: re-allocating a
        // workspace then costs neither a cudaMalloc nor a device synchronisation
        cudaMemPool_t pool;
        IFDDA_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t keep = UINT64_MAX;
        IFDDA_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        c->flag.ensure(1);
        c->st.ensure(1);
        c->zstatus.ensure(1);
        c->tickets.ensure(1);
        IFDDA_CUDA(cudaMemset(c->zstatus.p, 0, sizeof(int)));
        IFDDA_CUDA(cudaMemset(c->tickets.p, 0, sizeof(unsigned)));
        c->partials.ensure(2048 * 8);  // reduction_blocks() partials of up to 8 sums
    } catch (const EngineError& e) {
        for (cudaEvent_t ev : {c->upload_done, c->loc_ready, c->loc_copied})
            if (ev) cudaEventDestroy(ev);
        if (c->upload_stream) cudaStreamDestroy(c->upload_stream);
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return 1;
    }
    *out = c;
    return 0;
}

namespace {
// Frees the context's buffers and stream.  Never throws: destroy calls come
// from finalisers and exit paths.
void ctx_free(ifdda_ctx* ctx) {
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(ctx->device) == cudaSuccess) {
        {
            AllocStreamScope as(ctx->stream);
            ctx->flag.release();
            ctx->partials.release();
            ctx->tickets.release();
            ctx->st.release();
            ctx->zstatus.release();
        }
        if (ctx->stream) {
            cudaStreamSynchronize(ctx->stream);
            cudaStreamDestroy(ctx->stream);
        }
        if (ctx->upload_stream) {
            cudaStreamSynchronize(ctx->upload_stream);
            cudaStreamDestroy(ctx->upload_stream);
        }
        if (ctx->upload_done) cudaEventDestroy(ctx->upload_done);
        if (ctx->loc_ready) cudaEventDestroy(ctx->loc_ready);
        if (ctx->loc_copied) cudaEventDestroy(ctx->loc_copied);
        destroy_retired_graph_execs();
        if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    }
    delete ctx;
}
}  // namespace

int ifdda_ctx_destroy(ifdda_ctx* ctx) {
    if (!ctx) return 0;
    if (ctx->live_greens > 0) {
        // spectra still use the stream: the last ifdda_green_destroy frees it
        ctx->closing = true;
        return 0;
    }
    ctx_free(ctx);
    return 0;
}

const char* ifdda_ctx_last_error(const ifdda_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int ifdda_ctx_synchronize(ifdda_ctx* ctx) {
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    IFDDA_CUDA(cudaStreamSynchronize(ctx->stream));
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

void* ifdda_ctx_stream(ifdda_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int ifdda_green_create(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, double k0, ifdda_green** out) {
    return ifdda_green_create_nquad(ctx, nx, ny, nz, aretecube, k0, 0, out);
}

int ifdda_green_create_nquad(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, double k0, int nquad,
                             ifdda_green** out) {
    if (!ctx || !out) return 1;
    *out = nullptr;
    std::unique_ptr<ifdda_green> g(new ifdda_green());
    g->ctx = ctx;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    if (ctx->closing) throw EngineError{1, "context already destroyed"};
    green_build(g->G, nx, ny, nz, aretecube, k0, ctx->stream, nquad, /*pad=*/true);
    if (g->G.padded()) g->ptab.ensure(g->G.g.N);
    *out = g.release();
    ctx->live_greens++;
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_green_create_box(ifdda_ctx* ctx, int nx, int ny, int nz, int bx, int by, int bz, double aretecube,
                           double k0, ifdda_green** out) {
    if (!ctx || !out) return 1;
    *out = nullptr;
    std::unique_ptr<ifdda_green> g(new ifdda_green());
    g->ctx = ctx;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    if (ctx->closing) throw EngineError{1, "context already destroyed"};
    const int box[3] = {bx, by, bz};
    green_build(g->G, nx, ny, nz, aretecube, k0, ctx->stream, 0, false, box);
    if (g->G.padded()) g->ptab.ensure(g->G.g.N);
    *out = g.release();
    ctx->live_greens++;
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_green_tiles(ifdda_green* g, int precision, int* zconv_variant, int* ypass_variant, float* times_ms) {
    if (!g || (precision != IFDDA_FP32 && precision != IFDDA_FP64)) return 1;
    TileChoice tc;
    const bool have = tile_get(g->G.device, precision == IFDDA_FP32 ? 1 : 0, g->G.g, tc);
    if (zconv_variant) *zconv_variant = have ? tc.zvar : -1;
    if (ypass_variant) *ypass_variant = have ? tc.yvar : -1;
    if (times_ms)
        for (int v = 0; v < 2; v++) {
            times_ms[v] = have ? tc.z_ms[v] : 0.f;
            times_ms[2 + v] = have ? tc.y_ms[v] : 0.f;
        }
    return 0;
}

int ifdda_green_set_tiles(ifdda_green* g, int precision, int zconv_variant, int ypass_variant) {
    if (!g || (precision != IFDDA_FP32 && precision != IFDDA_FP64)) return 1;
    const int pk = precision == IFDDA_FP32 ? 1 : 0;
    if (zconv_variant < 0 || ypass_variant < 0) {
        tile_erase(g->G.device, pk, g->G.g);
        return 0;
    }
    if (zconv_variant >= tile_variants(g->G.g.Z) || ypass_variant >= tile_variants(g->G.g.Y)) {
        g->ctx->last_error = "ifdda_green_set_tiles: no such tile variant for this grid";
        return 1;
    }
    TileChoice tc{};
    tc.zvar = zconv_variant;
    tc.yvar = ypass_variant;
    tile_put(g->G.device, pk, g->G.g, tc);
    return 0;
}

int ifdda_green_recompute(ifdda_green* g, double aretecube, double k0) {
    if (!g) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    if (!(aretecube > 0) || !(k0 > 0)) throw EngineError{1, "ifdda_green_recompute: aretecube and k0 must be > 0"};
    green_recompute(g->G, aretecube, k0, g->ctx->stream);
    return 0;
    IFDDA_GUARD_END(g->ctx, nullptr)
}

int ifdda_green_destroy(ifdda_green* g) {
    if (!g) return 0;
    ifdda_ctx* ctx = g->ctx;
    int prev = -1;
    cudaGetDevice(&prev);
    if (cudaSetDevice(ctx->device) == cudaSuccess) {
        AllocStreamScope as(ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        if (ctx->upload_stream) cudaStreamSynchronize(ctx->upload_stream);
        delete g;
        if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    } else {
        delete g;
    }
    if (--ctx->live_greens == 0 && ctx->closing) ctx_free(ctx);
    return 0;
}

int ifdda_green_release_workspace(ifdda_green* g) {
    if (!g) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    IFDDA_CUDA(cudaStreamSynchronize(g->ctx->stream));
    IFDDA_CUDA(cudaStreamSynchronize(g->ctx->upload_stream));
    g->SW.kw64.release();
    g->SW.kw32.release();
    g->SW.mixed.release();
    g->G.w32.B1.release();
    g->G.w32.B2.release();
    g->G.w64.B1.release();
    g->G.w64.B2.release();
    g->alpha.release();
    g->ff0.release();
    g->up_alpha.release();
    g->up_ff0.release();
    g->x.release();
    g->ffx.release();
    g->ffb.release();
    g->ffx32.release();
    g->ffb32.release();
    g->alpha32.release();
    g->tab.release();
    g->rtab.release();
    g->rtab_in.release();
    g->ralpha.release();
    g->rgc64.release();
    g->rgc32.release();
    g->roff.release();
    return 0;
    IFDDA_GUARD_END(g->ctx, nullptr)
}

int ifdda_green_export(ifdda_green* g, ifdda_dcmplx* xx, ifdda_dcmplx* xy, ifdda_dcmplx* xz, ifdda_dcmplx* yy,
                       ifdda_dcmplx* yz, ifdda_dcmplx* zz) {
    if (!g) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    if (g->G.padded()) throw EngineError{1, "export: the lattice was padded to compiled FFT lengths"};
    double2* out[6] = {(double2*)xx, (double2*)xy, (double2*)xz, (double2*)yy, (double2*)yz, (double2*)zz};
    green_export(g->G, out, g->ctx->stream);
    return 0;
    IFDDA_GUARD_END(g->ctx, nullptr)
}

int ifdda_matvec(ifdda_green* g, int precision, int ndip, const int* tabdip, const ifdda_dcmplx* FFX,
                 ifdda_dcmplx* FFB) {
    if (!g || !FFX || !FFB) return 1;
    IFDDA_GUARD_BEGIN
    if (precision != IFDDA_FP32 && precision != IFDDA_FP64)
        throw EngineError{1, "ifdda_matvec: precision must be IFDDA_FP32 or IFDDA_FP64"};
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    cudaStream_t st = g->ctx->stream;
    const long uN = g->G.uN;
    if (!tabdip && ndip != uN) throw EngineError{1, "ifdda_matvec: ndip must be nx*ny*nz without tabdip"};
    const long n3 = 3L * ndip;
    const int* tab = nullptr;
    if (tabdip) {
        check_tabdip(tabdip, uN, ndip);
        g->tab.ensure(uN);
        IFDDA_CUDA(cudaMemcpyAsync(g->tab.p, tabdip, uN * sizeof(int), cudaMemcpyHostToDevice, st));
        tab = g->tab.p;
    }
    tab = lattice_tab(g, tab, st);
    g->ffx.ensure(n3);
    g->ffb.ensure(n3);
    IFDDA_CUDA(cudaMemcpyAsync(g->ffx.p, FFX, n3 * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(g->ffb.p, FFB, n3 * sizeof(double2), cudaMemcpyHostToDevice, st));
    if (precision == IFDDA_FP32) {
        tune_tiles<float>(g->G, 1, st);
        g->ffx32.ensure(n3);
        g->ffb32.ensure(n3);
        cast_dev<float>(g->ffx.p, g->ffx32.p, n3, st);
        cast_dev<float>(g->ffb.p, g->ffb32.p, n3, st);
        MvArgs<float> a = mv_args<float>(g->G, 1, g->ffx32.p, g->ffb32.p, g->ffb32.p, n3, ALPHA_NONE, nullptr, 0, tab,
                                         nullptr);
        if (!matvec_launch<float>(a, 1, tab != nullptr, st)) throw EngineError{1, "FFT size not supported"};
        std::vector<float2> h(n3);
        IFDDA_CUDA(cudaMemcpyAsync(h.data(), g->ffb32.p, n3 * sizeof(float2), cudaMemcpyDeviceToHost, st));
        IFDDA_CUDA(cudaStreamSynchronize(st));
        for (long i = 0; i < n3; i++) FFB[i] = ifdda_dcmplx{h[i].x, h[i].y};
    } else {
        tune_tiles<double>(g->G, 1, st);
        MvArgs<double> a = mv_args<double>(g->G, 1, g->ffx.p, g->ffb.p, g->ffb.p, n3, ALPHA_NONE, nullptr, 0, tab,
                                           nullptr);
        if (!matvec_launch<double>(a, 1, tab != nullptr, st)) throw EngineError{1, "FFT size not supported"};
        IFDDA_CUDA(cudaMemcpyAsync(FFB, g->ffb.p, n3 * sizeof(double2), cudaMemcpyDeviceToHost, st));
        IFDDA_CUDA(cudaStreamSynchronize(st));
    }
    return 0;
    IFDDA_GUARD_END(g->ctx, nullptr)
}

int ifdda_matvec_device(ifdda_green* g, int precision, int nrhs, int ndip, const int* tabdip_dev,
                        const void* FFX_dev, void* FFB_dev) {
    if (!g || !FFX_dev || !FFB_dev || nrhs < 1 || ndip < 1) return 1;
    IFDDA_GUARD_BEGIN
    if (precision != IFDDA_FP32 && precision != IFDDA_FP64)
        throw EngineError{1, "ifdda_matvec_device: precision must be IFDDA_FP32 or IFDDA_FP64"};
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    cudaStream_t st = g->ctx->stream;
    if (!tabdip_dev && ndip != g->G.uN) throw EngineError{1, "ifdda_matvec_device: ndip must be nx*ny*nz"};
    const long n3 = 3L * ndip;
    tabdip_dev = lattice_tab(g, tabdip_dev, st);
    bool ok;
    if (precision == IFDDA_FP32) {
        tune_tiles<float>(g->G, nrhs, st);
        MvArgs<float> a = mv_args<float>(g->G, nrhs, (const float2*)FFX_dev, (const float2*)FFB_dev, (float2*)FFB_dev,
                                         n3, ALPHA_NONE, nullptr, 0, tabdip_dev, nullptr);
        ok = matvec_launch<float>(a, nrhs, tabdip_dev != nullptr, st);
    } else {
        tune_tiles<double>(g->G, nrhs, st);
        MvArgs<double> a = mv_args<double>(g->G, nrhs, (const double2*)FFX_dev, (const double2*)FFB_dev,
                                           (double2*)FFB_dev, n3, ALPHA_NONE, nullptr, 0, tabdip_dev, nullptr);
        ok = matvec_launch<double>(a, nrhs, tabdip_dev != nullptr, st);
    }
    if (!ok) throw EngineError{1, "FFT size not supported"};
    return 0;
    IFDDA_GUARD_END(g->ctx, nullptr)
}

int ifdda_inverserig_batch(ifdda_green* g, int nrhs, int nbsphere, int nmax, const int* tabdip,
                           const ifdda_dcmplx* polarisa, const ifdda_dcmplx* FF0, const char* methodeit, double tol,
                           ifdda_dcmplx* FF, ifdda_dcmplx* FFloc, double* tol1, int* nloop, int* ncompte,
                           int* nstop, char* infostr, const ifdda_solve_options* opt) {
    if (!g || !polarisa || !FF0 || !FF || !FFloc || nrhs < 1 || nbsphere < 1) {
        if (nstop) *nstop = 1;
        set_info(infostr, "invalid argument");
        return 1;
    }
    IFDDA_GUARD_BEGIN
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    cudaStream_t st = g->ctx->stream;
    const long uN = g->G.uN;
    if (!tabdip && nbsphere != uN)
        throw EngineError{1, "full-box solve: nbsphere must equal nx*ny*nz (or pass tabdip)"};
    if (nmax < nbsphere) throw EngineError{1, "nmax smaller than nbsphere"};
    const long n3 = 3L * nbsphere, tot = n3 * nrhs;
    const int* tab = nullptr;
    if (tabdip) check_tabdip(tabdip, uN, nbsphere);
    // The inputs are uploaded on the context's upload stream when their
    // buffers need no allocation, so that the copies overlap the work already
    // queued on the solve stream (in the reference's call sequence the
    // spectrum, cdmlib/cdmlib.f:1529, comes right before the solve, :1565);
    // the solve stream waits for them (upload_done) before the solve.  A
    // buffer that must grow is allocated and filled on the solve stream,
    // after the upload stream has drained (a pending upload may still target
    // the old buffer after an error).
    ifdda_ctx* ctx = g->ctx;
    // on every way out (errors included) the upload stream has finished with
    // the caller's arrays before the call returns
    struct UploadDrain {
        cudaStream_t s;
        ~UploadDrain() { cudaStreamSynchronize(s); }
    } drain{ctx->upload_stream};
    auto upload = [&](DevBuf<double2>& buf, const void* src, size_t n, bool side) {
        cudaStream_t s = st;
        if (side && n <= buf.n) {
            s = ctx->upload_stream;
        } else if (n > buf.n) {
            IFDDA_CUDA(cudaStreamSynchronize(ctx->upload_stream));
            buf.ensure(n);
        }
        IFDDA_CUDA(cudaMemcpyAsync(buf.p, src, n * sizeof(double2), cudaMemcpyHostToDevice, s));
    };
    // the incident field goes first, so that its copy overlaps the host scan
    // of the polarisability below (when FF0 is pinned)
    upload(g->up_ff0, FF0, (size_t)tot, true);
    g->x.ensure(tot);
    g->ffb.ensure(tot);
    if (tabdip) {
        g->tab.ensure(uN);
        IFDDA_CUDA(cudaMemcpyAsync(g->tab.p, tabdip, uN * sizeof(int), cudaMemcpyHostToDevice, st));
        tab = g->tab.p;
    }
    tab = lattice_tab(g, tab, st);
    // Isotropy: the first dipoles are checked here (an anisotropic object is
    // almost always anisotropic there); if they are isotropic the solve starts
    // with one alpha per dipole while host threads scan the rest, and it is
    // repeated with the full tensor in the rare case that the rest is not.
    const long head = std::min<long>(nbsphere, 4096);
    std::atomic<bool> nostop{false};
    const int amode = pola_iso_range(polarisa, 0, head, nmax, nostop) ? ALPHA_ISO : ALPHA_FULL;
    std::atomic<int> tail{ALPHA_ISO};
    std::thread scan;
    struct Joiner {
        std::thread& t;
        ~Joiner() {
            if (t.joinable()) t.join();
        }
    } joiner{scan};
    if (amode == ALPHA_ISO && nbsphere > head)
        scan = std::thread([&] { tail.store(pola_mode_range(polarisa, head, nbsphere, nmax)); });
    // the isotropic value of dipole i is polarisa(i,1,1): the first nb
    // entries of the (nmax,3,3) array, contiguous
    upload(g->up_alpha, polarisa, amode == ALPHA_ISO ? (size_t)nbsphere : (size_t)9 * nmax, true);
    IFDDA_CUDA(cudaEventRecord(ctx->upload_done, ctx->upload_stream));
    IFDDA_CUDA(cudaStreamWaitEvent(st, ctx->upload_done, 0));
    // A page-locked FFloc receives the local field from the mixed solve after
    // each refinement step, while the solve checks the new residual; the copy
    // after the last step is the result.  (A pageable copy would block this
    // thread, so a pageable FFloc gets the one copy at the end.)
    cudaPointerAttributes pa{};
    const bool loc_pinned = cudaPointerGetAttributes(&pa, FFloc) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();  // a host pointer the runtime does not know leaves no error behind
    bool loc_done = false;
    // the outputs are copied and waited for below, on the same stream
    int rc = solve_device(g, nrhs, nbsphere, nmax, tab, g->up_alpha.p, amode, g->up_ff0.p, methodeit, tol, g->ffb.p,
                          g->x.p, tol1, nloop, ncompte, nstop, infostr, opt, true, false,
                          loc_pinned ? (double2*)FFloc : nullptr, &loc_done);
    if (scan.joinable()) scan.join();
    if (amode == ALPHA_ISO && tail.load() == ALPHA_FULL && rc != -1) {
        // the first solve's kernels read up_alpha: the full tensor follows
        // them on the solve stream
        upload(g->up_alpha, polarisa, (size_t)9 * nmax, false);
        rc = solve_device(g, nrhs, nbsphere, nmax, tab, g->up_alpha.p, ALPHA_FULL, g->up_ff0.p, methodeit, tol,
                          g->ffb.p, g->x.p, tol1, nloop, ncompte, nstop, infostr, opt, true, false);
        loc_done = false;
    }
    if (!loc_done)
        IFDDA_CUDA(cudaMemcpyAsync(FFloc, g->x.p, tot * sizeof(double2), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaMemcpyAsync(FF, g->ffb.p, tot * sizeof(double2), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    return rc;
    IFDDA_GUARD_END(g->ctx, infostr)
}

int ifdda_inverserig_ragged(int nobj, ifdda_green* const* greens, const int* nrhs, const int* nbsphere,
                            const int* nmax, const int* const* tabdip, const ifdda_dcmplx* const* polarisa,
                            const ifdda_dcmplx* const* FF0, const char* methodeit, double tol, ifdda_dcmplx* const* FF,
                            ifdda_dcmplx* const* FFloc, double* tol1, int* nloop, int* ncompte, int* nstop,
                            char* infostr, const ifdda_solve_options* opt) {
    return ragged_solve(nobj, greens, nrhs, nbsphere, nmax, tabdip, polarisa, FF0, methodeit, tol, FF, FFloc, tol1,
                        nloop, ncompte, nstop, infostr, opt, false);
}

int ifdda_inverserig_ragged_device(int nobj, ifdda_green* const* greens, const int* nrhs, const int* nbsphere,
                                   const int* nmax, const int* const* tabdip_dev,
                                   const ifdda_dcmplx* const* polarisa_dev, const ifdda_dcmplx* const* FF0_dev,
                                   const char* methodeit, double tol, ifdda_dcmplx* const* FF_dev,
                                   ifdda_dcmplx* const* FFloc_dev, double* tol1, int* nloop, int* ncompte, int* nstop,
                                   char* infostr, const ifdda_solve_options* opt) {
    return ragged_solve(nobj, greens, nrhs, nbsphere, nmax, tabdip_dev, polarisa_dev, FF0_dev, methodeit, tol, FF_dev,
                        FFloc_dev, tol1, nloop, ncompte, nstop, infostr, opt, true);
}

int ifdda_incident_planewaves_device(ifdda_ctx* ctx, int nbsphere, const double* xs_dev, const double* ys_dev,
                                     const double* zs_dev, double k0, ifdda_dcmplx E0, int nrhs, const int* beam,
                                     const double* a1, const double* a2, const double* pp, ifdda_dcmplx* FF0_dev) {
    if (!ctx || !xs_dev || !ys_dev || !zs_dev || !beam || !a1 || !a2 || !pp || !FF0_dev || nbsphere < 1 || nrhs < 1)
        return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    DevBuf<double> d1, d2, dp;
    DevBuf<int> db;
    d1.ensure(nrhs);
    d2.ensure(nrhs);
    dp.ensure(nrhs);
    db.ensure(nrhs);
    IFDDA_CUDA(cudaMemcpyAsync(d1.p, a1, nrhs * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(d2.p, a2, nrhs * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dp.p, pp, nrhs * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(db.p, beam, nrhs * sizeof(int), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), st));
    planewaves_dev(nbsphere, xs_dev, ys_dev, zs_dev, k0, make_double2(E0.re, E0.im), nrhs, db.p, d1.p, d2.p, dp.p,
                   (double2*)FF0_dev, ctx->flag.p, st);
    int bad = 0;
    IFDDA_CUDA(cudaMemcpyAsync(&bad, ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    if (bad) throw EngineError{1, "problem in plance incident wave"};
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_inverserig(ifdda_green* g, int nbsphere, int nmax, const int* tabdip, const ifdda_dcmplx* polarisa,
                     const ifdda_dcmplx* FF0, const char* methodeit, double tol, ifdda_dcmplx* FF,
                     ifdda_dcmplx* FFloc, double* tol1, int* nloop, int* ncompte, int* nstop, char* infostr,
                     const ifdda_solve_options* opt) {
    return ifdda_inverserig_batch(g, 1, nbsphere, nmax, tabdip, polarisa, FF0, methodeit, tol, FF, FFloc, tol1, nloop,
                                  ncompte, nstop, infostr, opt);
}

int ifdda_inverserig_batch_device(ifdda_green* g, int nrhs, int nbsphere, int nmax, const int* tabdip_dev,
                                  const ifdda_dcmplx* polarisa_dev, const ifdda_dcmplx* FF0_dev,
                                  const char* methodeit, double tol, ifdda_dcmplx* FF_dev, ifdda_dcmplx* FFloc_dev,
                                  double* tol1, int* nloop, int* ncompte, int* nstop, char* infostr,
                                  const ifdda_solve_options* opt) {
    if (!g || !polarisa_dev || !FF0_dev || !FF_dev || !FFloc_dev || nrhs < 1 || nbsphere < 1) {
        if (nstop) *nstop = 1;
        set_info(infostr, "invalid argument");
        return 1;
    }
    IFDDA_GUARD_BEGIN
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    if (!tabdip_dev && nbsphere != g->G.uN)
        throw EngineError{1, "full-box solve: nbsphere must equal nx*ny*nz (or pass tabdip)"};
    // isotropic tensors are compacted on the device (one alpha per dipole)
    cudaStream_t st = g->ctx->stream;
    tabdip_dev = lattice_tab(g, tabdip_dev, st);
    g->alpha.ensure(nbsphere);
    IFDDA_CUDA(cudaMemsetAsync(g->ctx->flag.p, 0, sizeof(int), st));
    pola_compact_dev((const double2*)polarisa_dev, nbsphere, nmax, g->alpha.p, g->ctx->flag.p, st);
    int aniso = 0;
    IFDDA_CUDA(cudaMemcpyAsync(&aniso, g->ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    const double2* alpha = aniso ? (const double2*)polarisa_dev : g->alpha.p;
    return solve_device(g, nrhs, nbsphere, nmax, tabdip_dev, alpha, aniso ? ALPHA_FULL : ALPHA_ISO,
                        (const double2*)FF0_dev, methodeit, tol, (double2*)FF_dev, (double2*)FFloc_dev, tol1, nloop,
                        ncompte, nstop, infostr, opt);
    IFDDA_GUARD_END(g->ctx, infostr)
}

int ifdda_local_macro(ifdda_ctx* ctx, int nbsphere, int nmax, const ifdda_dcmplx* epsilon,
                      const ifdda_dcmplx* FFloc, double aretecube, double k0, ifdda_dcmplx* Em) {
    if (!ctx || !epsilon || !FFloc || !Em || nbsphere < 1 || nmax < nbsphere) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    DevBuf<double2> eps, loc, em;
    eps.ensure((size_t)9 * nmax);
    loc.ensure(3L * nbsphere);
    em.ensure(3L * nbsphere);
    IFDDA_CUDA(cudaMemcpyAsync(eps.p, epsilon, (size_t)9 * nmax * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(loc.p, FFloc, 3L * nbsphere * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), st));
    local_macro_dev(nbsphere, nmax, eps.p, loc.p, aretecube, k0, em.p, ctx->flag.p, st);
    int bad = 0;
    IFDDA_CUDA(cudaMemcpyAsync(Em, em.p, 3L * nbsphere * sizeof(double2), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaMemcpyAsync(&bad, ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    if (bad) throw EngineError{1, "problem in local-macro: singular 3x3 matrix"};
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_cross_sections(ifdda_ctx* ctx, int nbsphere, const ifdda_dcmplx* FF0, const ifdda_dcmplx* FF,
                         const ifdda_dcmplx* FFloc, double k0, double I0, double* Cext, double* Cabs) {
    if (!ctx || !FF0 || !FF || !FFloc || nbsphere < 1) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    const long n3 = 3L * nbsphere;
    DevBuf<double2> a, b, c;
    a.ensure(n3);
    b.ensure(n3);
    c.ensure(n3);
    IFDDA_CUDA(cudaMemcpyAsync(a.p, FF0, n3 * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(b.p, FF, n3 * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(c.p, FFloc, n3 * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemsetAsync(ctx->tickets.p, 0, sizeof(unsigned), st));
    cross_sections_dev(nbsphere, a.p, b.p, c.p, k0, ctx->partials.p, ctx->tickets.p, ctx->st.p, ctx->zstatus.p, st);
    KState h;
    IFDDA_CUDA(cudaMemcpyAsync(&h, ctx->st.p, sizeof(KState), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    const double pi = 3.14159265358979323846;
    if (Cext) *Cext = 4.0 * pi * k0 * h.alpha.x / I0;
    if (Cabs) *Cabs = 4.0 * pi * k0 * h.beta.x / I0;
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_incident_planewaves(ifdda_ctx* ctx, int nbsphere, const double* xs, const double* ys, const double* zs,
                              double k0, ifdda_dcmplx E0, int nrhs, const int* beam, const double* a1,
                              const double* a2, const double* pp, ifdda_dcmplx* FF0) {
    if (!ctx || !xs || !ys || !zs || !beam || !a1 || !a2 || !pp || !FF0 || nbsphere < 1 || nrhs < 1) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    DevBuf<double> dx, dy, dz, d1, d2, dp;
    DevBuf<int> db;
    DevBuf<double2> out;
    dx.ensure(nbsphere);
    dy.ensure(nbsphere);
    dz.ensure(nbsphere);
    d1.ensure(nrhs);
    d2.ensure(nrhs);
    dp.ensure(nrhs);
    db.ensure(nrhs);
    out.ensure(3L * nbsphere * nrhs);
    IFDDA_CUDA(cudaMemcpyAsync(dx.p, xs, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dy.p, ys, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dz.p, zs, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(d1.p, a1, nrhs * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(d2.p, a2, nrhs * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dp.p, pp, nrhs * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(db.p, beam, nrhs * sizeof(int), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), st));
    planewaves_dev(nbsphere, dx.p, dy.p, dz.p, k0, make_double2(E0.re, E0.im), nrhs, db.p, d1.p, d2.p, dp.p, out.p,
                   ctx->flag.p, st);
    int bad = 0;
    IFDDA_CUDA(cudaMemcpyAsync(FF0, out.p, 3L * nbsphere * nrhs * sizeof(double2), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaMemcpyAsync(&bad, ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    if (bad) throw EngineError{1, "problem in plance incident wave"};
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_farfield_csca(ifdda_ctx* ctx, int nbsphere, const double* xs, const double* ys, const double* zs,
                        const ifdda_dcmplx* FF, double k0, double I0, double theta, double phi, int ntheta, int nphi,
                        double* Cscai, double* gasym, double* poynting, double* thetafield, double* phifield) {
    if (!ctx || !xs || !ys || !zs || !FF || !Cscai || !gasym || nbsphere < 1) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    if (ntheta <= 10 || nphi <= 20) throw EngineError{1, "ntheta and nphi too small!"};
    const int ndir = (ntheta + 1) * nphi;
    DevBuf<double> dx, dy, dz, em;
    DevBuf<double2> ff, part;
    dx.ensure(nbsphere);
    dy.ensure(nbsphere);
    dz.ensure(nbsphere);
    ff.ensure(3L * nbsphere);
    part.ensure((size_t)ndir * farfield_chunks(nbsphere) * 3);
    em.ensure(ndir);
    IFDDA_CUDA(cudaMemcpyAsync(dx.p, xs, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dy.p, ys, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dz.p, zs, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(ff.p, FF, 3L * nbsphere * sizeof(double2), cudaMemcpyHostToDevice, st));
    farfield_dev(nbsphere, dx.p, dy.p, dz.p, ff.p, k0, ntheta, nphi, part.p, em.p, st);
    std::vector<double> emod(ndir);
    IFDDA_CUDA(cudaMemcpyAsync(emod.data(), em.p, ndir * sizeof(double), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    // the integration of cdmlib.f:2797-2872, in its order
    const double pi = 3.14159265358979323846, c = 299792458.0, quatpieps0 = 1.0 / (c * c * 1e-7);
    const double deltatheta = pi / (double)ntheta, deltaphi = 2.0 * pi / (double)nphi;
    const double k03 = k0 * k0 * k0;
    double cs = 0.0, g = 0.0;
    int cnt = 0;
    for (int itheta = 0; itheta <= ntheta; itheta++) {
        const double thetas = deltatheta * (double)itheta;
        for (int iphi = 0; iphi < nphi; iphi++, cnt++) {
            const double phis = deltaphi * (double)iphi;
            const double n0 = std::sin(thetas) * std::cos(phis), n1 = std::sin(thetas) * std::sin(phis),
                         n2 = std::cos(thetas);
            const double Emod = emod[cnt];
            if (poynting) poynting[cnt] = Emod * k0 * k0 * k0 * k0 * c / 8 / pi * quatpieps0;
            if (thetafield) thetafield[cnt] = thetas * 180.0 / pi;
            if (phifield) phifield[cnt] = phis * 180.0 / pi;
            cs = cs + deltaphi * deltatheta * std::sin(thetas) * Emod;
            g = g + deltaphi * deltatheta * std::sin(thetas) * Emod *
                        (n0 * std::sin(theta * pi / 180.0) * std::cos(phi * pi / 180.0) +
                         n1 * std::sin(theta * pi / 180.0) * std::sin(phi * pi / 180.0) +
                         n2 * std::cos(theta * pi / 180.0));
        }
    }
    *gasym = g / cs;
    *Cscai = cs * k03 * k0 / I0;
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_farfield_fft(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, const double* xs, const double* ys,
                       const double* zs, const ifdda_dcmplx* FF, double k0, double I0, double theta, double phi,
                       int nfft2d, int ntheta, int nphi, double* Cscai, double* gasym, double* poynting,
                       double* thetafield, double* phifield, int* imaxk0, double* kpos, double* kneg) {
    if (!ctx || !xs || !ys || !zs || !FF || !Cscai || !gasym || nx < 1 || ny < 1 || nz < 1 || nfft2d < 2) return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    const double pi = 3.14159265358979323846, c = 299792458.0, quatpieps0 = 1.0 / (c * c * 1e-7);
    const int n = nfft2d, n2 = n / 2;
    const long N = (long)nx * ny * nz;
    // diffractefft2d.f:29-74
    const double dkx = 2.0 * pi / ((double)n * aretecube), dky = dkx;
    if (n > 16384) throw EngineError{1, "nfft2d too large"};
    if (dkx >= k0) throw EngineError{1, "In FFT Poynting nfft2d too small"};
    const int imax = (int)std::lround(k0 / dkx) + 1, S = 2 * imax + 1;
    if (S > n || S < 7) throw EngineError{1, "In FFT diffract nfft2d too small"};
    if (nx > n || ny > n) throw EngineError{1, "nfft2d smaller than the object"};
    if (ntheta <= 10 || nphi <= 20) throw EngineError{1, "ntheta and nphi too small!"};
    MicGeom m{};
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.n = n;
    m.imax = imax;
    m.k0 = k0;
    m.dkx = dkx;
    m.dky = dky;
    m.numaper = k0;
    m.dside = 1.0;
    m.var1 = (xs[0] + (double)n2 * aretecube) * dkx;
    m.var2 = (ys[0] + (double)n2 * aretecube) * dky;
    m.gross = 1.0;
    std::vector<double> zp(nz);
    for (int k = 0; k < nz; k++) zp[k] = zs[(long)nx * ny * k];
    std::vector<double2> twh(n);
    for (int j = 0; j < n; j++) {
        const double a = 2.0 * pi * (double)j / (double)n;
        twh[j] = make_double2(std::cos(a), std::sin(a));
        if (4 * j == n) twh[j] = make_double2(0.0, 1.0);
        if (2 * j == n) twh[j] = make_double2(-1.0, 0.0);
        if (4 * j == 3 * n) twh[j] = make_double2(0.0, -1.0);
        if (j == 0) twh[j] = make_double2(1.0, 0.0);
    }
    DevBuf<double> zpl;
    DevBuf<double2> ff, tw, Q, Ed;
    zpl.ensure(nz);
    tw.ensure(n);
    ff.ensure(3 * N);
    Q.ensure((size_t)nz * ny * S * 3);
    Ed.ensure((size_t)2 * S * S * 3);
    IFDDA_CUDA(cudaMemcpyAsync(zpl.p, zp.data(), nz * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(tw.p, twh.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(ff.p, FF, 3 * N * sizeof(double2), cudaMemcpyHostToDevice, st));
    mic_farfield_dev(m, 1, ff.p, zpl.p, tw.p, Q.p, Ed.p, st, true);
    std::vector<double2> ed((size_t)2 * S * S * 3);
    IFDDA_CUDA(cudaMemcpyAsync(ed.data(), Ed.p, ed.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    // |E|^2 at pupil point (i, j) of side s (0: kz > 0, 1: kz < 0), as
    // cdabs(.)**2 sums
    auto emod = [&](int s, int i, int j) {
        const double2* e = ed.data() + (((size_t)s * S + (j + imax)) * S + (i + imax)) * 3;
        double v = 0.0;
        for (int q = 0; q < 3; q++) {
            const double a = std::hypot(e[q].x, e[q].y);
            v += a * a;
        }
        return v;
    };
    // Csca and g over the propagating waves (computegcfft2d.f:16-46)
    const double sth = std::sin(theta * pi / 180.0), cph = std::cos(phi * pi / 180.0),
                 sph = std::sin(phi * pi / 180.0), cth = std::cos(theta * pi / 180.0);
    double cs = 0.0, g = 0.0;
    int k = 0;
    for (int i = -imax; i <= imax; i++)
        for (int j = -imax; j <= imax; j++, k++) {
            const double kx = (double)i * dkx, ky = (double)j * dky;
            const bool prop = k0 * k0 - kx * kx - ky * ky > 0.0;
            if (kpos) kpos[k] = 0.0;
            if (kneg) kneg[k] = 0.0;
            if (!prop) continue;
            const double kz = std::sqrt(k0 * k0 - kx * kx - ky * ky);
            double e = emod(0, i, j);
            if (kpos) kpos[k] = e * k0 * k0 * k0 * k0 * c / 8 / pi * quatpieps0;
            cs = cs + dkx * dky * e / kz;
            g = g + dkx * dky * e / kz * (kx * sth * cph + ky * sth * sph + kz * cth) / k0;
            e = emod(1, i, j);
            if (kneg) kneg[k] = e * k0 * k0 * k0 * k0 * c / 8 / pi * quatpieps0;
            cs = cs + dkx * dky * e / kz;
            g = g + dkx * dky * e / kz * (kx * sth * cph + ky * sth * sph - kz * cth) / k0;
        }
    *gasym = g / cs;
    *Cscai = cs * (k0 * k0 * k0) / I0;
    if (imaxk0) *imaxk0 = imax;
    // Poynting vector on the (theta, phi) grid by bilinear interpolation of the
    // pupil grid (cdmlib.f:2990-3075), the reference's zero-count fallback
    // included
    const double deltatheta = pi / (double)ntheta, deltaphi = 2.0 * pi / (double)nphi;
    int cnt = 0;
    for (int itheta = 0; itheta <= ntheta; itheta++) {
        const double thetas = deltatheta * (double)itheta;
        for (int iphi = 0; iphi < nphi; iphi++, cnt++) {
            const double phis = deltaphi * (double)iphi;
            if (thetafield) thetafield[cnt] = thetas * 180.0 / pi;
            if (phifield) phifield[cnt] = phis * 180.0 / pi;
            const double kx = k0 * std::sin(thetas) * std::cos(phis), ky = k0 * std::sin(thetas) * std::sin(phis);
            int i2 = -imax, j2 = -imax;
            for (int i = -imax; i <= imax; i++)
                if (kx >= i * dkx) i2 = i;
            for (int j = -imax; j <= imax; j++)
                if (ky >= j * dkx) j2 = j;
            const int s = thetas <= pi / 2.0 ? 0 : 1;
            const double e11 = emod(s, i2, j2), e22 = emod(s, i2 + 1, j2 + 1), e21 = emod(s, i2 + 1, j2),
                         e12 = emod(s, i2, j2 + 1);
            const int test = (e11 == 0.0) + (e22 == 0.0) + (e21 == 0.0) + (e12 == 0.0);
            double e;
            if (test == 0)
                e = (e21 - e11) * (kx - dkx * i2) / dkx + (e12 - e11) * (ky - dkx * j2) / dkx +
                    (e11 + e22 - e12 - e21) * (kx - dkx * i2) / dkx * (ky - dkx * j2) / dkx + e11;
            else
                e = (e11 + e12 + e21 + e22) / (double)(4 - test);
            if (poynting) poynting[cnt] = e * k0 * k0 * k0 * k0 * c / 8.0 / pi * quatpieps0;
        }
    }
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_nearfield_wide(ifdda_ctx* ctx, int nx, int ny, int nz, int nxmp, int nymp, int nzmp, double aretecube,
                         double k0, int nquad, int nbsphere, int nmax, const double* xs, const double* ys,
                         const double* zs, const ifdda_dcmplx* FF, const ifdda_dcmplx* FF0,
                         const ifdda_dcmplx* epsilon, ifdda_dcmplx E0, double theta, double phi, double pp,
                         double* xswf, double* yswf, double* zswf, ifdda_dcmplx* incident, ifdda_dcmplx* local,
                         ifdda_dcmplx* macro) {
    if (!ctx || !xs || !ys || !zs || !FF || !FF0 || !epsilon || nbsphere < 1 || nmax < nbsphere || nx < 1 ||
        ny < 1 || nz < 1 || nxmp < 0 || nymp < 0 || nzmp < 0)
        return 1;
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    const int nxw = nx + 2 * nxmp, nyw = ny + 2 * nymp, nzw = nz + 2 * nzmp;
    const long nw = (long)nxw * nyw * nzw;
    // the enlarged box starts nxmp cells before the object's smallest x
    // (cdmlib.f:2034-2050, 2144-2150)
    double xmin = 1e300, ymin = 1e300, zmin = 1e300;
    for (int i = 0; i < nbsphere; i++) {
        xmin = std::min(xmin, xs[i]);
        ymin = std::min(ymin, ys[i]);
        zmin = std::min(zmin, zs[i]);
    }
    // object dipoles sit on box sites in the same z, y, x order; a site takes
    // the next dipole when their positions agree within lambda / 1000
    // (comparaison.f:41-50)
    const double err = 2.0 * 3.14159265358979323846 / k0 / 1000.0;
    std::vector<double> px(nw), py(nw), pz(nw);
    std::vector<int> map(nw, -1);
    long l = 0, s = 0;
    for (int i = 1; i <= nzw; i++)
        for (int j = 1; j <= nyw; j++)
            for (int k = 1; k <= nxw; k++, s++) {
                const double x = xmin + (double)(k - nxmp - 1) * aretecube;
                const double y = ymin + (double)(j - nymp - 1) * aretecube;
                const double z = zmin + (double)(i - nzmp - 1) * aretecube;
                px[s] = x;
                py[s] = y;
                pz[s] = z;
                if (l < nbsphere && x >= xs[l] - err && x <= xs[l] + err && y >= ys[l] - err && y <= ys[l] + err &&
                    z >= zs[l] - err && z <= zs[l] + err)
                    map[s] = (int)l++;
            }
    if (xswf) std::copy(px.begin(), px.end(), xswf);
    if (yswf) std::copy(py.begin(), py.end(), yswf);
    if (zswf) std::copy(pz.begin(), pz.end(), zswf);
    DevBuf<double> dx, dy, dz, a1, a2, dp;
    DevBuf<int> dmap, beam;
    DevBuf<double2> ff, ff0, eps, xr, xi, epsw, em;
    dx.ensure(nw);
    dy.ensure(nw);
    dz.ensure(nw);
    dmap.ensure(nw);
    ff.ensure(3L * nbsphere);
    ff0.ensure(3L * nbsphere);
    eps.ensure((size_t)9 * nmax);
    xr.ensure(3 * nw);
    xi.ensure(3 * nw);
    epsw.ensure((size_t)9 * nw);
    em.ensure(3 * nw);
    a1.ensure(1);
    a2.ensure(1);
    dp.ensure(1);
    beam.ensure(1);
    const int b0 = 0;
    IFDDA_CUDA(cudaMemcpyAsync(dx.p, px.data(), nw * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dy.p, py.data(), nw * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dz.p, pz.data(), nw * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dmap.p, map.data(), nw * sizeof(int), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(ff.p, FF, 3L * nbsphere * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(ff0.p, FF0, 3L * nbsphere * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(eps.p, epsilon, (size_t)9 * nmax * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(a1.p, &theta, sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(a2.p, &phi, sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dp.p, &pp, sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(beam.p, &b0, sizeof(int), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemsetAsync(ctx->flag.p, 0, sizeof(int), st));
    // incident field on every site (ondeplane), then the object's own
    planewaves_dev((int)nw, dx.p, dy.p, dz.p, k0, make_double2(E0.re, E0.im), 1, beam.p, a1.p, a2.p, dp.p, xr.p,
                   ctx->flag.p, st);
    wide_fill_dev(nw, dmap.p, ff.p, ff0.p, eps.p, nmax, xr.p, xi.p, epsw.p, st);
    if (incident) IFDDA_CUDA(cudaMemcpyAsync(incident, xr.p, 3 * nw * sizeof(double2), cudaMemcpyDeviceToHost, st));
    // E = E0 + G p on the enlarged box: one FP64 mat-vec (cdmlib.f:2274-2277)
    Green G;
    green_build(G, nxw, nyw, nzw, aretecube, k0, st, nquad, /*pad=*/true);
    DevBuf<int> wtab;
    if (G.padded()) wtab.ensure(G.g.N);
    const int* tab = lattice_tab(G, wtab.p, nullptr, st);
    MvArgs<double> a = mv_args<double>(G, 1, xi.p, xr.p, xr.p, 3 * nw, ALPHA_NONE, nullptr, 0, tab, nullptr);
    if (!matvec_launch<double>(a, 1, tab != nullptr, st)) throw EngineError{1, "FFT size not supported"};
    if (local) IFDDA_CUDA(cudaMemcpyAsync(local, xr.p, 3 * nw * sizeof(double2), cudaMemcpyDeviceToHost, st));
    // macroscopic field with the object's permittivity (identity elsewhere)
    local_macro_dev((int)nw, nw, epsw.p, xr.p, aretecube, k0, em.p, ctx->flag.p, st);
    if (macro) IFDDA_CUDA(cudaMemcpyAsync(macro, em.p, 3 * nw * sizeof(double2), cudaMemcpyDeviceToHost, st));
    int bad = 0;
    IFDDA_CUDA(cudaMemcpyAsync(&bad, ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    if (bad) throw EngineError{1, "problem in local-macro: singular 3x3 matrix"};
    return 0;
    IFDDA_GUARD_END(ctx, nullptr)
}

int ifdda_holography(ifdda_ctx* ctx, int nx, int ny, int nz, double aretecube, double k0, int nbsphere,
                     const double* xs, const double* ys, const double* zs, const ifdda_dcmplx* FF, ifdda_dcmplx E0,
                     double theta, double phi, double pp, int nfft2d, double numaper, double gross, double zlens,
                     int nside, int nquicklens, ifdda_dcmplx* image, ifdda_dcmplx* fourier, double* xy,
                     double* kxy, int* imaxk0, char* infostr) {
    if (!ctx || !xs || !ys || !zs || !FF || !image || nx < 1 || ny < 1 || nz < 1 || nbsphere < 1) {
        set_info(infostr, "invalid argument");
        return 1;
    }
    IFDDA_GUARD_BEGIN
    DeviceScope ds(ctx->device);
    AllocStreamScope as(ctx->stream);
    cudaStream_t st = ctx->stream;
    auto fail = [&](const char* msg) {
        set_info(infostr, msg);
        ctx->last_error = msg;
        return 1;
    };
    const int n = nfft2d;
    const long N = (long)nx * ny * nz;
    const bool quick = nquicklens == 1;
    if (nside != 0 && nside != 1) return fail("nside must be 0 (transmission) or 1 (reflection)");
    if (nquicklens != 0 && nquicklens != 1) return fail("nquicklens must be 0 or 1");
    if (quick && nbsphere != N) return fail("the FFT lens needs the full box (nbsphere = nx*ny*nz)");
    if (!image_length_supported(n)) return fail("nfft2d not supported: 32 to 4096, a power of two or 768, 1536, 3072");
    if (nx > n || ny > n) return fail("nfft2d smaller than the object");
    const double pi = 3.14159265358979323846, dside = nside == 1 ? -1.0 : 1.0;
    const double na = numaper * k0;
    double dkx = 2.0 * pi / ((double)n * aretecube);
    int imax;
    if (quick) {
        // diffractefft2dlens.f:29-73
        if (dkx >= na) return fail("In FFT lens nfft2d too small");
        imax = (int)std::lround(k0 / dkx) + 1;
        if (2 * imax + 1 > n) return fail("In FFT diffraction for lens nfft2d too small!");
        if (2 * imax + 1 < 7) return fail("In FFT diffract nfft2d too small");
    } else {
        // cdmlib.f:3818-3826: halve the pupil step until more than 20 points
        // cover k0; the pupil must fit the image grid (unchecked there)
        for (int k = 0;; k++) {
            dkx = 2.0 * pi / ((double)n * aretecube) / (double)(1 << k);
            imax = (int)std::lround(k0 / dkx) + 1;
            if (imax > 20) break;
        }
        if (2 * imax + 1 > n) return fail("In FFT lens nfft2d too small");
        // diffractefft2dinc.f:64-68 on the transmission side
        if (nside == 0 && dkx >= na) return fail("In FFT lens inc nfft2d too small");
    }
    const int S = 2 * imax + 1;
    MicGeom m{};
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.n = n;
    m.imax = imax;
    m.k0 = k0;
    m.dkx = dkx;
    m.dky = dkx;
    m.numaper = na;
    m.var1 = (xs[0] + (double)(n / 2) * aretecube) * dkx;
    m.var2 = (ys[0] + (double)(n / 2) * aretecube) * dkx;
    m.zlens = zlens * dside;
    m.gross = gross;
    m.dside = dside;
    // grid point of the incident wave (diffractefft2dinc.f:75-83, deltakroutine.f)
    const double kxinc = std::sin(theta * pi / 180.0) * std::cos(phi * pi / 180.0) * k0;
    const double kyinc = std::sin(theta * pi / 180.0) * std::sin(phi * pi / 180.0) * k0;
    int ik = (int)std::lround(kxinc / dkx), jk = (int)std::lround(kyinc / dkx);
    {
        const double kx = dkx * ik, ky = dkx * jk;
        if (!(kx * kx + ky * ky <= k0 * k0)) {
            ik = (int)(kxinc / dkx);
            jk = (int)(kyinc / dkx);
        }
    }
    std::vector<double> zp(nz);
    if (quick)
        for (int k = 0; k < nz; k++) zp[k] = zs[(long)nx * ny * k];
    std::vector<double2> twh(n);
    for (int j = 0; j < n; j++) {
        const double a = 2.0 * pi * (double)j / (double)n;
        twh[j] = make_double2(std::cos(a), std::sin(a));
        if (4 * j == n) twh[j] = make_double2(0.0, 1.0);
        if (2 * j == n) twh[j] = make_double2(-1.0, 0.0);
        if (4 * j == 3 * n) twh[j] = make_double2(0.0, -1.0);
        if (j == 0) twh[j] = make_double2(1.0, 0.0);
    }
    DevBuf<double> zpl, dx, dy, dz;
    DevBuf<double2> ff, tw, Q, Ed, F, four, T, cimg;
    zpl.ensure(nz);
    tw.ensure(n);
    ff.ensure(3L * nbsphere);
    if (quick) Q.ensure((size_t)nz * ny * S * 3);
    else Q.ensure((size_t)S * S * mic_direct_chunks(nbsphere) * 3);
    Ed.ensure((size_t)S * S * 3);
    F.ensure((size_t)6 * S * S);
    four.ensure((size_t)6 * S * S);
    T.ensure((size_t)6 * S * n);
    cimg.ensure((size_t)6 * n * n);
    IFDDA_CUDA(cudaMemcpyAsync(zpl.p, zp.data(), nz * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(tw.p, twh.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(ff.p, FF, 3L * nbsphere * sizeof(double2), cudaMemcpyHostToDevice, st));
    if (quick) {
        mic_farfield_dev(m, 1, ff.p, zpl.p, tw.p, Q.p, Ed.p, st);
    } else {
        dx.ensure(nbsphere);
        dy.ensure(nbsphere);
        dz.ensure(nbsphere);
        IFDDA_CUDA(cudaMemcpyAsync(dx.p, xs, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
        IFDDA_CUDA(cudaMemcpyAsync(dy.p, ys, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
        IFDDA_CUDA(cudaMemcpyAsync(dz.p, zs, nbsphere * sizeof(double), cudaMemcpyHostToDevice, st));
        mic_direct_dev(m, 1, nbsphere, dx.p, dy.p, dz.p, ff.p, Q.p, Ed.p, st);
    }
    if (!mic_holo_dev(m, Ed.p, ik, jk, pp, make_double2(E0.re, E0.im), !quick, F.p, four.p, tw.p, T.p, cimg.p, st))
        return fail("nfft2d not supported");
    IFDDA_CUDA(cudaMemcpyAsync(image, cimg.p, (size_t)6 * n * n * sizeof(double2), cudaMemcpyDeviceToHost, st));
    if (fourier)
        IFDDA_CUDA(cudaMemcpyAsync(fourier, four.p, (size_t)6 * S * S * sizeof(double2), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    const double deltax = 2.0 * pi / (double)n / dkx;
    for (int i = -n / 2; i <= n / 2 - 1; i++) {
        if (xy) xy[i + n / 2] = deltax * (double)i * gross;
        if (kxy) kxy[i + n / 2] = dkx * (double)i / k0;
    }
    if (imaxk0) *imaxk0 = imax;
    if (infostr) memset(infostr, ' ', 64);
    return 0;
    IFDDA_GUARD_END(ctx, infostr)
}

int ifdda_microscope(ifdda_green* g, int nbsphere, const int* tabdip, const double* xs, const double* ys,
                     const double* zs, const ifdda_dcmplx* polarisa, const char* methodeit, double tol,
                     const ifdda_microscope_options* mo, double* image, double* xy, double* kxy, int* ninc,
                     double* kxinc, double* kyinc, double* tol1, int* nloop, int* ncompte, int* nstop,
                     char* infostr, const ifdda_solve_options* opt) {
    if (!g || !xs || !ys || !zs || !polarisa || !mo || !image || !ninc || nbsphere < 1) {
        if (nstop) *nstop = 1;
        set_info(infostr, "invalid argument");
        return 1;
    }
    IFDDA_GUARD_BEGIN
    DeviceScope ds(g->ctx->device);
    AllocStreamScope as(g->ctx->stream);
    cudaStream_t st = g->ctx->stream;
    // the caller's lattice (the solve maps it onto a padded one, if any)
    const int nx = g->G.ux, ny = g->G.uy, nz = g->G.uz, nmax = (int)g->G.uN, N = nbsphere, n = mo->nfft2d;
    const bool quick = mo->nquicklens == 1;
    auto fail = [&](const char* msg) {
        if (nstop) *nstop = 1;
        set_info(infostr, msg);
        return 1;
    };
    if (mo->ntypemic != 1 && mo->ntypemic != 2) return fail("ntypemic must be 1 (bright field) or 2 (dark field)");
    if (mo->nquicklens != 0 && mo->nquicklens != 1) return fail("nquicklens must be 0 or 1");
    // the FFT lens reads the dipoles plane by plane: full box (cdmlib.f:631)
    if (quick && (tabdip || nbsphere != nmax)) return fail("the FFT lens needs the full box (nbsphere = nx*ny*nz)");
    if (!tabdip && nbsphere != nmax) return fail("full-box solve: nbsphere must equal nx*ny*nz (or pass tabdip)");
    if (tabdip) check_tabdip(tabdip, nmax, nbsphere);
    if (mo->nside != 0 && mo->nside != 1) return fail("nside must be 0 (transmission) or 1 (reflection)");
    // cdmlib.f:237-238, 389: the side's sign of kz, carried by zlens too
    const double dside = mo->nside == 1 ? -1.0 : 1.0;
    if (!image_length_supported(n)) return fail("nfft2d not supported: 32 to 4096, a power of two or 768, 1536, 3072");
    if (nx > n || ny > n) return fail("nfft2d smaller than the object");
    const double pi = 3.14159265358979323846;
    const double k0 = g->G.k0, d = g->G.d;
    const double numaper = mo->numaper * k0, numaperinc = mo->numaperinc, numaperk = k0 * numaperinc;
    // microsbf.f:83-88 (the reference tests numaper, not numaperinc, for <= 0)
    if (numaperinc >= 1.0 || numaper <= 0.0) return fail("NA inc strictly between 0 and 1");
    // step of the incidences (microsbf.f:91-135): the object's extent sets deltakm
    double xmax = -1e300, xmin = 1e300, ymax = -1e300, ymin = 1e300;
    for (int i = 0; i < N; i++) {
        xmax = std::max(xmax, xs[i]);
        xmin = std::min(xmin, xs[i]);
        ymax = std::max(ymax, ys[i]);
        ymin = std::min(ymin, ys[i]);
    }
    const double deltakm = pi / std::max(xmax - xmin, ymax - ymin);
    double dkx = 2.0 * pi / (d * (double)n);
    double deltak;
    int imaxinc, imaxk0 = 0;
    if (quick) {
        if (dkx >= numaperk) return fail("In FFT lens nfft2d too small:Increase size of FFT 1");
        int imul = (int)(deltakm / dkx);
        if (imul == 0) return fail("In FFT lens nfft2d too small:Increase size of FFT 2");
        for (;;) {
            deltak = dkx * (double)imul;
            imaxinc = (int)std::lround(k0 / deltak) + 1;
            if (imaxinc > 3) break;
            if (--imul == 0) return fail("In FFT lens nfft2d too small:Increase size of FFT 3");
        }
    } else {
        // microsbf.f:139-157: halve the pupil step until more than 5 points
        // cover k0, then the incidence step from the object's size
        for (int k = 0;; k++) {
            dkx = 2.0 * pi / ((double)n * d) / (double)(1 << k);
            imaxk0 = (int)std::lround(k0 / dkx) + 1;
            if (imaxk0 > 5) break;
        }
        for (int k = 0;; k++) {
            deltak = dkx * std::round(deltakm / dkx) / (double)(1 << k);
            imaxinc = (int)std::lround(k0 / deltak) + 1;
            if (imaxinc > 2) break;
        }
        // the pupil must fit the image grid (the reference does not check)
        if (2 * imaxk0 + 1 > n) return fail("In FFT lens nfft2d too small");
    }
    const double dky = dkx;
    // incidences of one polarisation: the grid inside the condenser's NA
    // (microsbf.f:161-171) or the ring at its NA (microsdf.f:160-162, 204-212)
    std::vector<double> kxi, kyi;
    if (mo->ntypemic == 1) {
        for (int id = -imaxinc; id <= imaxinc; id++)
            for (int jd = -imaxinc; jd <= imaxinc; jd++) {
                const double kx = id * deltak, ky = jd * deltak;
                if (kx * kx + ky * ky <= numaperk * numaperk) {
                    kxi.push_back(kx);
                    kyi.push_back(ky);
                }
            }
        if (deltak >= numaperk) return fail("In FFT lens nfft2d too small");
    } else {
        const double deltatheta = deltak / k0 * numaperinc;
        const int m = std::max((int)(2.0 * pi / deltatheta) + 1, 8);
        for (int id = 0; id < m; id++) {
            const double phi = (double)id * 2.0 * pi / (double)m;
            kxi.push_back(std::cos(phi) * k0 * numaperinc);
            kyi.push_back(std::sin(phi) * k0 * numaperinc);
        }
    }
    const int cnt = (int)kxi.size(), cap = *ninc;
    *ninc = cnt;
    for (int q = 0; q < cnt && q < cap; q++) {
        if (kxinc) kxinc[q] = kxi[q] / k0;
        if (kyinc) kyinc[q] = kyi[q] / k0;
    }
    // power shared by the 2 cnt illuminations (microsbf.f:206-207, irradiance.f)
    const double c = 299792458.0, eps0 = 1.0 / (c * c * 4.0 * pi * 1e-7);
    const double irra = mo->P0 / (double)(2 * cnt) / (mo->w0 * mo->w0 * pi);
    const double2 E0 = make_double2(std::sqrt(2.0 * irra / c / eps0), 0.0);
    // every incidence in the reference's order: s then p, then the list;
    // grid index of its specular wave (deltakroutine.f; microsbf.f passes the
    // incidence step, microsdf.f the pupil step)
    const int total = 2 * cnt;
    std::vector<double> a1(total), a2(total), ppv(total);
    std::vector<int> ikv(total), jkv(total);
    for (int t = 0; t < total; t++) {
        const int q = t % cnt;
        a1[t] = kxi[q];
        a2[t] = kyi[q];
        ppv[t] = t < cnt ? 0.0 : 1.0;
        const double sx = mo->ntypemic == 1 ? deltak : dkx, sy = mo->ntypemic == 1 ? deltak : dky;
        int i = (int)std::lround(a1[t] / sx), j = (int)std::lround(a2[t] / sy);
        const double kx = sx * i, ky = sy * j;
        if (!(kx * kx + ky * ky <= k0 * k0)) {
            i = (int)(a1[t] / sx);
            j = (int)(a2[t] / sy);
        }
        ikv[t] = i;
        jkv[t] = j;
    }
    // FFT lens (diffractefft2dlens.f:29-73)
    MicGeom m{};
    m.nx = nx;
    m.ny = ny;
    m.nz = nz;
    m.n = n;
    m.imax = quick ? (int)std::lround(k0 / dkx) + 1 : imaxk0;
    m.ntypemic = mo->ntypemic;
    m.k0 = k0;
    m.dkx = dkx;
    m.dky = dky;
    m.numaper = numaper;
    m.var1 = (xs[0] + (double)(n / 2) * d) * dkx;
    m.var2 = (ys[0] + (double)(n / 2) * d) * dky;
    m.zlens = mo->zlens * dside;
    m.gross = mo->gross;
    m.dside = dside;
    const int S = 2 * m.imax + 1;
    const char* lens_error = !quick         ? nullptr
                             : dkx >= numaper ? "In FFT lens nfft2d too small"
                             : S > n          ? "In FFT diffraction for lens nfft2d too small!"
                             : S < 7          ? "In FFT diffract nfft2d too small"
                                              : nullptr;
    const int B = std::max(1, std::min(total, mo->batch > 0 ? mo->batch : 64));
    const long n3 = 3L * N;
    DevBuf<double> dx, dy, dz, zpl, d1, d2, dpp, img;
    DevBuf<int> dbeam, dik, djk, dtab;
    DevBuf<double2> pol, alpha, ff0, ff, loc, tw, Q, Ed, F, T;
    dx.ensure(N);
    dy.ensure(N);
    dz.ensure(N);
    IFDDA_CUDA(cudaMemcpyAsync(dx.p, xs, N * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dy.p, ys, N * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(dz.p, zs, N * sizeof(double), cudaMemcpyHostToDevice, st));
    // the object ((nmax,3,3) tensor): one alpha per dipole when isotropic
    pol.ensure((size_t)9 * nmax);
    alpha.ensure(N);
    IFDDA_CUDA(cudaMemcpyAsync(pol.p, polarisa, (size_t)9 * nmax * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemsetAsync(g->ctx->flag.p, 0, sizeof(int), st));
    pola_compact_dev(pol.p, N, nmax, alpha.p, g->ctx->flag.p, st);
    if (tabdip) {
        dtab.ensure(nmax);
        IFDDA_CUDA(cudaMemcpyAsync(dtab.p, tabdip, nmax * sizeof(int), cudaMemcpyHostToDevice, st));
    }
    const int* stab = lattice_tab(g, tabdip ? dtab.p : nullptr, st);
    int aniso = 0;
    IFDDA_CUDA(cudaMemcpyAsync(&aniso, g->ctx->flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    // z of each lattice plane (FFT lens, full box), the roots of unity of the
    // pupil transforms
    std::vector<double> zp(nz);
    if (quick)
        for (int k = 0; k < nz; k++) zp[k] = zs[(long)nx * ny * k];
    std::vector<double2> twh(n);
    for (int j = 0; j < n; j++) {
        const double a = 2.0 * pi * (double)j / (double)n;
        twh[j] = make_double2(std::cos(a), std::sin(a));
        if (4 * j == n) twh[j] = make_double2(0.0, 1.0);
        if (2 * j == n) twh[j] = make_double2(-1.0, 0.0);
        if (4 * j == 3 * n) twh[j] = make_double2(0.0, -1.0);
        if (j == 0) twh[j] = make_double2(1.0, 0.0);
    }
    zpl.ensure(nz);
    tw.ensure(n);
    IFDDA_CUDA(cudaMemcpyAsync(zpl.p, zp.data(), nz * sizeof(double), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(tw.p, twh.data(), n * sizeof(double2), cudaMemcpyHostToDevice, st));
    std::vector<int> beam(B, 1);
    d1.ensure(B);
    d2.ensure(B);
    dpp.ensure(B);
    dbeam.ensure(B);
    dik.ensure(B);
    djk.ensure(B);
    IFDDA_CUDA(cudaMemcpyAsync(dbeam.p, beam.data(), B * sizeof(int), cudaMemcpyHostToDevice, st));
    ff0.ensure(n3 * B);
    ff.ensure(n3 * B);
    loc.ensure(n3 * B);
    if (quick) Q.ensure((size_t)B * nz * ny * S * 3);
    else Q.ensure((size_t)B * S * S * mic_direct_chunks(N) * 3);
    Ed.ensure((size_t)B * S * S * 3);
    F.ensure((size_t)B * 6 * S * S);
    T.ensure((size_t)B * 6 * S * n);
    img.ensure((size_t)6 * n * n);
    IFDDA_CUDA(cudaMemsetAsync(img.p, 0, (size_t)6 * n * n * sizeof(double), st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    const double2* al = aniso ? pol.p : alpha.p;
    const int amode = aniso ? ALPHA_FULL : ALPHA_ISO;
    std::vector<double> t1(B);
    std::vector<int> nl(B), nc(B);
    for (int t0 = 0; t0 < total; t0 += B) {
        const int nb = std::min(B, total - t0);
        IFDDA_CUDA(cudaMemcpyAsync(d1.p, a1.data() + t0, nb * sizeof(double), cudaMemcpyHostToDevice, st));
        IFDDA_CUDA(cudaMemcpyAsync(d2.p, a2.data() + t0, nb * sizeof(double), cudaMemcpyHostToDevice, st));
        IFDDA_CUDA(cudaMemcpyAsync(dpp.p, ppv.data() + t0, nb * sizeof(double), cudaMemcpyHostToDevice, st));
        IFDDA_CUDA(cudaMemcpyAsync(dik.p, ikv.data() + t0, nb * sizeof(int), cudaMemcpyHostToDevice, st));
        IFDDA_CUDA(cudaMemcpyAsync(djk.p, jkv.data() + t0, nb * sizeof(int), cudaMemcpyHostToDevice, st));
        planewaves_dev(N, dx.p, dy.p, dz.p, k0, E0, nb, dbeam.p, d1.p, d2.p, dpp.p, ff0.p, g->ctx->flag.p, st);
        const int rc = solve_device(g, nb, N, nmax, stab, al, amode, ff0.p, methodeit, tol, ff.p, loc.p, t1.data(),
                                    nl.data(), nc.data(), nstop, infostr, opt, false);
        if (tol1) *tol1 = t1[nb - 1];
        if (nloop) *nloop = nl[nb - 1];
        if (ncompte) *ncompte = nc[nb - 1];
        if (rc) return rc;
        // the lens checks of diffractefft2dlens.f run after the first solve
        if (lens_error) return fail(lens_error);
        if (quick) mic_farfield_dev(m, nb, ff.p, zpl.p, tw.p, Q.p, Ed.p, st);
        else mic_direct_dev(m, nb, N, dx.p, dy.p, dz.p, ff.p, Q.p, Ed.p, st);
        mic_lens_dev(m, nb, Ed.p, dik.p, djk.p, dpp.p, E0, F.p, st);
        if (!mic_image_dev(m, nb, F.p, tw.p, T.p, img.p, st)) return fail("nfft2d not supported");
    }
    mic_sqrt_dev((long)6 * n * n, img.p, st);
    IFDDA_CUDA(cudaMemcpyAsync(image, img.p, (size_t)6 * n * n * sizeof(double), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    // image and pupil axes (microsbf.f:846-857)
    const double deltax = 2.0 * pi / (double)n / dkx;
    for (int i = -n / 2; i <= n / 2 - 1; i++) {
        if (xy) xy[i + n / 2] = deltax * (double)i * mo->gross;
        if (kxy) kxy[i + n / 2] = dkx * (double)i / k0;
    }
    if (nstop) *nstop = 0;
    if (infostr) memset(infostr, ' ', 64);
    return 0;
    IFDDA_GUARD_END(g->ctx, infostr)
}

}  // extern "C"
