// Green spectrum build (replaces greencalculfft, cdmlib/calculgreenfft.f:1-104).
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include "engine.cuh"
#include "green_kernels.cuh"

namespace ifdda {

bool fft_length_supported(int L) {
    switch (L) {
#define IFDDA_CASE_OK(L) case L:
        IFDDA_FFT_LENGTHS(IFDDA_CASE_OK)
        return true;
#undef IFDDA_CASE_OK
        default:
            return false;
    }
}

namespace {
std::mutex g_tile_mu;
std::map<std::array<int, 5>, TileChoice>& tile_map() {
    static std::map<std::array<int, 5>, TileChoice> m;
    return m;
}
std::array<int, 5> tile_key(int dev, int prec, const MvGeom& g) { return {dev, prec, g.X, g.Y, g.Z}; }
}  // namespace

bool tile_get(int dev, int prec, const MvGeom& g, TileChoice& out) {
    std::lock_guard<std::mutex> lk(g_tile_mu);
    auto it = tile_map().find(tile_key(dev, prec, g));
    if (it == tile_map().end()) return false;
    out = it->second;
    return true;
}
void tile_put(int dev, int prec, const MvGeom& g, const TileChoice& tc) {
    std::lock_guard<std::mutex> lk(g_tile_mu);
    tile_map()[tile_key(dev, prec, g)] = tc;
}
void tile_erase(int dev, int prec, const MvGeom& g) {
    std::lock_guard<std::mutex> lk(g_tile_mu);
    tile_map().erase(tile_key(dev, prec, g));
}

MvGeom make_geom(int nx, int ny, int nz) {
    MvGeom g{};
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.X = 2 * nx;
    g.Y = 2 * ny;
    g.Z = 2 * nz;
    g.N = (long)nx * ny * nz;
    g.b1_rhs = 3L * nz * ny * g.X;
    g.b2_rhs = 3L * nz * g.Y * g.X;
    g.gc_comp = (long)(nx + 1) * (ny + 1) * (nz + 1);
    return g;
}

// twiddle table exp(+2 pi i j / L), j < L, computed in FP64 on the host
static void upload_twiddles(int L, DevBuf<double2>& t64, DevBuf<float2>& t32, cudaStream_t st) {
    std::vector<double2> h(L);
    std::vector<float2> hf(L);
    const double two_pi = 6.283185307179586476925286766559;
    for (int j = 0; j < L; j++) {
        // reduce the angle to the first octant-free form exactly where possible
        const double a = two_pi * (double)j / (double)L;
        h[j] = make_double2(std::cos(a), std::sin(a));
        if (4 * j == L) h[j] = make_double2(0.0, 1.0);
        if (2 * j == L) h[j] = make_double2(-1.0, 0.0);
        if (4 * j == 3 * L) h[j] = make_double2(0.0, -1.0);
        if (j == 0) h[j] = make_double2(1.0, 0.0);
        hf[j] = make_float2((float)h[j].x, (float)h[j].y);
    }
    t64.ensure(L);
    t32.ensure(L);
    IFDDA_CUDA(cudaMemcpyAsync(t64.p, h.data(), L * sizeof(double2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaMemcpyAsync(t32.p, hf.data(), L * sizeof(float2), cudaMemcpyHostToDevice, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
}

template <int L> static void launch_gx(const GreenGeom& gg, double2* GA, const double2* tw, cudaStream_t st) {
    using TT = GreenTiles<L>;
    dim3 grid((gg.ny + 1 + TT::TLX - 1) / TT::TLX, gg.nz + 1, 1);
    ensure_smem(k_green_x<L>, TT::smem_x);
    count_launch();
    k_green_x<L><<<grid, TT::NT, TT::smem_x, st>>>(gg, GA, tw);
}

template <int L, int AXIS>
static void launch_gyz(const GreenGeom& gg, const double2* src, double2* d64, float2* d32, const double2* tw,
                       cudaStream_t st) {
    using TT = GreenTiles<L>;
    const int W = gg.nx + 1;
    dim3 grid((W + TT::TLY - 1) / TT::TLY, AXIS == 1 ? gg.nz + 1 : gg.ny + 1, 6);
    ensure_smem(k_green_yz<L, AXIS>, TT::smem_y);
    count_launch();
    k_green_yz<L, AXIS><<<grid, TT::NT, TT::smem_y, st>>>(gg, src, d64, d32, tw);
}

// smallest n' >= n with 2 n' a compiled FFT length (n itself when none is)
static int padded_side(int n) {
    for (int m = n; m <= 4 * n && m <= 4096; m++)
        if (fft_length_supported(2 * m)) return m;
    return n;
}

// The spectrum of G's lattice for its current (d, k0, nquad) into G.gc64 /
// G.gc32, which are allocated; the twiddle tables are uploaded.
static void green_compute(Green& G, cudaStream_t st) {
    const int nx = G.g.nx, ny = G.g.ny, nz = G.g.nz, nquad = G.nquad;
    GreenGeom gg{nx, ny, nz, G.g.X, G.g.Y, G.g.Z, G.d, G.k0, nquad, nullptr};
    // cube-averaged tensor on the offsets i, j, k >= 0 within nquad
    DevBuf<double2> quad, qpart;
    DevBuf<int3> qoffs;
    if (nquad > 0) {
        std::vector<int3> offs;
        for (int k = 0; k <= nquad; k++)
            for (int j = 0; j <= nquad; j++)
                for (int i = 0; i <= nquad; i++)
                    if (i * i + j * j + k * k <= nquad * nquad) offs.push_back(make_int3(i, j, k));
        const int n1 = nquad + 1, nent = (int)offs.size();
        quad.ensure((size_t)n1 * n1 * n1 * 6);
        qpart.ensure((size_t)nent * QUAD_CHUNKS * 6);
        qoffs.ensure(nent);
        IFDDA_CUDA(cudaMemsetAsync(quad.p, 0, (size_t)n1 * n1 * n1 * 6 * sizeof(double2), st));
        IFDDA_CUDA(cudaMemcpyAsync(qoffs.p, offs.data(), nent * sizeof(int3), cudaMemcpyHostToDevice, st));
        count_launch();
        k_green_quad_part<<<dim3(nent, QUAD_CHUNKS), QUAD_NT, 0, st>>>(gg, qoffs.p, qpart.p);
        count_launch();
        k_green_quad_final<<<(nent + 63) / 64, 64, 0, st>>>(gg, qoffs.p, nent, qpart.p, quad.p);
        IFDDA_CUDA(cudaGetLastError());
        gg.quad = quad.p;
        IFDDA_CUDA(cudaStreamSynchronize(st));  // the offsets live on this stack frame
    }
    const long W = nx + 1;
    // the intermediate spectra are freed stream-ordered, after the kernels
    DevBuf<double2> GA, GB;
    GA.ensure((size_t)6 * (nz + 1) * (ny + 1) * W);
    GB.ensure((size_t)6 * (nz + 1) * (ny + 1) * W);
    switch (G.g.X) {
#define IFDDA_CASE_GX(L) \
    case L: launch_gx<L>(gg, GA.p, G.tw64[0].p, st); break;
        IFDDA_FFT_LENGTHS(IFDDA_CASE_GX)
#undef IFDDA_CASE_GX
    }
    switch (G.g.Y) {
#define IFDDA_CASE_GY(L) \
    case L: launch_gyz<L, 1>(gg, GA.p, GB.p, nullptr, G.tw64[1].p, st); break;
        IFDDA_FFT_LENGTHS(IFDDA_CASE_GY)
#undef IFDDA_CASE_GY
    }
    switch (G.g.Z) {
#define IFDDA_CASE_GZ(L) \
    case L: launch_gyz<L, 2>(gg, GB.p, G.gc64.p, G.gc32.p, G.tw64[2].p, st); break;
        IFDDA_FFT_LENGTHS(IFDDA_CASE_GZ)
#undef IFDDA_CASE_GZ
    }
    IFDDA_CUDA(cudaGetLastError());
    IFDDA_CUDA(cudaStreamSynchronize(st));
}

void green_build(Green& G, int nx, int ny, int nz, double d, double k0, cudaStream_t st, int nquad, bool pad,
                 const int* box) {
    if (nx < 1 || ny < 1 || nz < 1) throw EngineError{1, "Green: lattice dimensions must be positive"};
    if (nquad < 0 || nquad > 16) throw EngineError{1, "Green: nquad must be in [0, 16]"};
    G.ux = nx;
    G.uy = ny;
    G.uz = nz;
    G.uN = (long)nx * ny * nz;
    if (box) {
        if (box[0] < nx || box[1] < ny || box[2] < nz)
            throw EngineError{1, "Green: the box must hold the lattice (each side at least the lattice's)"};
        nx = box[0];
        ny = box[1];
        nz = box[2];
    } else if (pad) {
        nx = padded_side(nx);
        ny = padded_side(ny);
        nz = padded_side(nz);
    }
    G.g = make_geom(nx, ny, nz);
    if (!fft_length_supported(G.g.X) || !fft_length_supported(G.g.Y) || !fft_length_supported(G.g.Z))
        throw EngineError{1, "FFT size not supported: lattice sides above 320 (2*n above 640)"};
    G.d = d;
    G.k0 = k0;
    cudaGetDevice(&G.device);
    upload_twiddles(G.g.X, G.tw64[0], G.tw32[0], st);
    upload_twiddles(G.g.Y, G.tw64[1], G.tw32[1], st);
    upload_twiddles(G.g.Z, G.tw64[2], G.tw32[2], st);
    G.nquad = nquad;
    G.gc64.ensure((size_t)6 * G.g.gc_comp);
    G.gc32.ensure((size_t)6 * G.g.gc_comp);
    green_compute(G, st);
}

void green_recompute(Green& G, double d, double k0, cudaStream_t st) {
    if (!G.gc64.p || !G.gc32.p) throw EngineError{1, "Green: no spectrum to recompute"};
    G.d = d;
    G.k0 = k0;
    green_compute(G, st);
}

// parity of component c along axis a: +1 even, -1 odd (xx,xy,xz,yy,yz,zz)
static inline int parity(int c, int axis) {
    static const int P[6][3] = {{1, 1, 1}, {-1, -1, 1}, {-1, 1, -1}, {1, 1, 1}, {1, -1, -1}, {1, 1, 1}};
    return P[c][axis];
}

void green_export(const Green& G, double2* const out[6], cudaStream_t st) {
    const MvGeom& g = G.g;
    std::vector<double2> h((size_t)6 * g.gc_comp);
    IFDDA_CUDA(cudaMemcpyAsync(h.data(), G.gc64.p, h.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
    IFDDA_CUDA(cudaStreamSynchronize(st));
    const int W = g.nx + 1, H = g.ny + 1;
    for (int c = 0; c < 6; c++) {
        const double2* src = h.data() + (size_t)c * g.gc_comp;
        for (int kz = 0; kz < g.Z; kz++) {
            const int qz = kz <= g.nz ? kz : g.Z - kz;
            const int sz = kz <= g.nz ? 1 : parity(c, 2);
            for (int jy = 0; jy < g.Y; jy++) {
                const int qy = jy <= g.ny ? jy : g.Y - jy;
                const int sy = jy <= g.ny ? 1 : parity(c, 1);
                for (int ix = 0; ix < g.X; ix++) {
                    const int qx = ix <= g.nx ? ix : g.X - ix;
                    const int sx = ix <= g.nx ? 1 : parity(c, 0);
                    const double s = (double)(sx * sy * sz);
                    const double2 v = src[((size_t)qz * H + qy) * W + qx];
                    out[c][((size_t)kz * g.Y + jy) * g.X + ix] = make_double2(s * v.x, s * v.y);
                }
            }
        }
    }
}

}  // namespace ifdda
