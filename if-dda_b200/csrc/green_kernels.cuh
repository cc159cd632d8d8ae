// Green-tensor spectrum on sm_100a, FP64 (replaces cdmlib/calculgreenfft.f:1-104
// with cdmlib/espace_libre.f:2-43 evaluated on the fly).
//
//   gx : for every (j, k) line with j <= ny, k <= nz, evaluate the 6
//        independent components of T(r) at r = (i, j, k) d with wrapped
//        negative offsets along x and zero planes at i = nx, j = ny, k = nz
//        (calculgreenfft.f:25-69), FFT along x (sign +1), keep qx in [0, nx]
//                                                          -> GA[c][nz+1][ny+1][nx+1]
//   gy : FFT along y, keep qy in [0, ny]                   -> GB[c][nz+1][ny+1][nx+1]
//   gz : FFT along z, keep qz in [0, nz]                   -> Gc64, Gc32
// Only the parity octant is kept: every component is even or odd along each
// axis, so the rest of the spectrum is a mirror image (see matvec_kernels.cuh).
// The same parity holds in real space, T_c(x, -y, z) = Py(c) T_c(x, y, z) and
// T_c(x, y, -z) = Pz(c) T_c(x, y, z), so the x pass computes the lines with
// j, k >= 0 only and the y and z passes read the negative offsets as signed
// mirror images: a quarter of the x-pass lines and half of the y-pass lines,
// with the same values as lines computed at negative offsets (only signs
// change).
#pragma once
#include "fft_tile.cuh"
#include "reduce.cuh"

namespace ifdda {

struct GreenGeom {
    int nx, ny, nz, X, Y, Z;
    double d, k0;
    // integrated tensor (cdmlib/calculgreenquadfft.f): offsets with
    // i^2 + j^2 + k^2 <= nquad^2 take quad[((|k| (nquad+1) + |j|) (nquad+1)
    // + |i|) * 6 + c]; nquad = 0 is the plain tensor everywhere
    int nquad;
    const double2* quad;
};

template <int L> struct GreenTiles {
    static constexpr int S = 16;
    static constexpr int TLX = clamp_pow2(49152 / (L * 6 * S), 1, 8);
    static constexpr int TLY = clamp_pow2(49152 / (L * S), 2, 16);
    static constexpr int NT = 256;
    static constexpr int LSX = (6 * TLX) | 1;
    static constexpr size_t smem_x = (size_t)L * S + (size_t)L * LSX * S;
    static constexpr size_t smem_y = (size_t)L * S + (size_t)L * TLY * S;
};

// T_ab(r), the six independent components xx, xy, xz, yy, yz, zz
__device__ __forceinline__ void green_point(double rx, double ry, double rz, double k0, double2 (&t)[6]) {
    const double r2 = rx * rx + ry * ry + rz * rz;
    if (r2 == 0.0) {
#pragma unroll
        for (int q = 0; q < 6; q++) t[q] = make_double2(0, 0);
        return;
    }
    const double rab = sqrt(r2);
    // c1 = (1/R - i k0)/R^2, c2 = k0^2/R, e = exp(i k0 R)
    const double c1r = 1.0 / (rab * r2), c1i = -k0 / r2;
    const double c2 = k0 * k0 / rab;
    double sn, cs;
    sincos(k0 * rab, &sn, &cs);
    const double rv[3] = {rx, ry, rz};
    const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const double id = ia[q] == ib[q] ? 1.0 : 0.0;
        const double rr = rv[ia[q]] * rv[ib[q]] / r2;
        const double a = 3.0 * rr - id, b = id - rr;
        const double fr = a * c1r + b * c2, fi = a * c1i;
        t[q] = make_double2(fr * cs - fi * sn, fr * sn + fi * cs);
    }
}

// T at lattice offset (i, j, k): the plain tensor, or inside the nquad sphere
// the cube-averaged one, whose components keep T's parity (xy odd in x and y,
// xz in x and z, yz in y and z)
__device__ __forceinline__ void green_value(const GreenGeom& g, int i, int j, int k, double2 (&t)[6]) {
    if (g.nquad > 0 && i * i + j * j + k * k <= g.nquad * g.nquad) {
        const int n1 = g.nquad + 1;
        const double2* q = g.quad + (((long)abs(k) * n1 + abs(j)) * n1 + abs(i)) * 6;
        const double sx = i < 0 ? -1.0 : 1.0, sy = j < 0 ? -1.0 : 1.0, sz = k < 0 ? -1.0 : 1.0;
        const double s[6] = {1.0, sx * sy, sx * sz, 1.0, sy * sz, 1.0};
#pragma unroll
        for (int c = 0; c < 6; c++) t[c] = make_double2(s[c] * q[c].x, s[c] * q[c].y);
        return;
    }
    green_point(i * g.d, j * g.d, k * g.d, g.k0, t);
}

// Cube-averaged tensor, cdmlib/propaesplibreintsim.f: Simpson rule with 128
// steps per axis over the source cube [-d/2, d/2]^3, 129^3 nodes per offset.
// Stage 1: block (entry, chunk) sums the nodes of its chunk in a fixed order.
constexpr int QUAD_STEPS = 128, QUAD_NODES = 129 * 129 * 129, QUAD_CHUNKS = 64, QUAD_NT = 256;
__global__ void __launch_bounds__(QUAD_NT) k_green_quad_part(const GreenGeom g, const int3* __restrict__ offs,
                                                             double2* __restrict__ part) {
    const int3 o = offs[blockIdx.x];
    const double pas = g.d / QUAD_STEPS, h = g.d / 2;
    double2 acc[6];
#pragma unroll
    for (int c = 0; c < 6; c++) acc[c] = make_double2(0, 0);
    const int per = (QUAD_NODES + QUAD_CHUNKS - 1) / QUAD_CHUNKS;
    const int n0 = blockIdx.y * per, n1 = min(QUAD_NODES, n0 + per);
    for (int n = n0 + threadIdx.x; n < n1; n += QUAD_NT) {
        const int a = n / (129 * 129), b = (n / 129) % 129, c = n % 129;
        const auto wt = [](int m) { return m == 0 || m == QUAD_STEPS ? 1.0 : (m & 1 ? 4.0 : 2.0); };
        const double ww = wt(a) * wt(b) * wt(c);
        double2 t[6];
        green_point(-h + pas * a - o.x * g.d, -h + pas * b - o.y * g.d, -h + pas * c - o.z * g.d, g.k0, t);
#pragma unroll
        for (int q = 0; q < 6; q++) acc[q] = make_double2(acc[q].x + t[q].x * ww, acc[q].y + t[q].y * ww);
    }
    __shared__ double2 scratch[6 * 32];
    block_sum<QUAD_NT, 6>(acc, scratch);
    if (threadIdx.x == 0) {
        double2* p = part + ((long)blockIdx.x * QUAD_CHUNKS + blockIdx.y) * 6;
#pragma unroll
        for (int q = 0; q < 6; q++) p[q] = acc[q];
    }
}

// Stage 2: one thread per entry sums the chunks in order and scales; points
// closer than d/10 give 0, points beyond one wavelength the plain tensor.
__global__ void k_green_quad_final(const GreenGeom g, const int3* __restrict__ offs, int nent,
                                   const double2* __restrict__ part, double2* __restrict__ quad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nent) return;
    const int3 o = offs[e];
    const int n1 = g.nquad + 1;
    double2* out = quad + (((long)o.z * n1 + o.y) * n1 + o.x) * 6;
    const double rab = g.d * sqrt((double)(o.x * o.x + o.y * o.y + o.z * o.z));
    const double lambda = 2.0 * 3.14159265358979323846 / g.k0;
    if (rab <= 0.1 * g.d) {
#pragma unroll
        for (int q = 0; q < 6; q++) out[q] = make_double2(0, 0);
        return;
    }
    if (rab >= lambda) {
        double2 t[6];
        green_point(o.x * g.d, o.y * g.d, o.z * g.d, g.k0, t);
#pragma unroll
        for (int q = 0; q < 6; q++) out[q] = t[q];
        return;
    }
    double2 acc[6];
#pragma unroll
    for (int q = 0; q < 6; q++) acc[q] = make_double2(0, 0);
    for (int ch = 0; ch < QUAD_CHUNKS; ch++)
#pragma unroll
        for (int q = 0; q < 6; q++) {
            const double2 v = part[((long)e * QUAD_CHUNKS + ch) * 6 + q];
            acc[q] = make_double2(acc[q].x + v.x, acc[q].y + v.y);
        }
    const double pas = g.d / QUAD_STEPS;
    const double tmp = pas / 3.0 * pas / 3.0 * pas / 3.0 / g.d / g.d / g.d;
    const double fx = o.x == 0 ? 0.0 : 1.0, fy = o.y == 0 ? 0.0 : 1.0, fz = o.z == 0 ? 0.0 : 1.0;
    const double f[6] = {1.0, fx * fy, fx * fz, 1.0, fy * fz, 1.0};
#pragma unroll
    for (int q = 0; q < 6; q++) out[q] = make_double2(acc[q].x * tmp * f[q], acc[q].y * tmp * f[q]);
}

// parity of component c (xx, xy, xz, yy, yz, zz) under y -> -y and z -> -z
__device__ __forceinline__ double green_py(int c) { return (c == 1 || c == 4) ? -1.0 : 1.0; }
__device__ __forceinline__ double green_pz(int c) { return (c == 2 || c == 4) ? -1.0 : 1.0; }

template <int L>
__global__ void __launch_bounds__(GreenTiles<L>::NT) k_green_x(const GreenGeom g, double2* __restrict__ GA,
                                                               const double2* __restrict__ twx) {
    using C = double2;
    using TT = GreenTiles<L>;
    constexpr int TL = TT::TLX, NB = 6 * TL, LS = TT::LSX, NT = TT::NT;
    extern __shared__ __align__(16) unsigned char raw[];
    C* tw = reinterpret_cast<C*>(raw);
    C* sm = tw + L;
    const int j0 = blockIdx.x * TL, kk = blockIdx.y;  // j <= ny, k <= nz
    const int nl = min(TL, g.ny + 1 - j0);
    load_twiddles<C, L, NT>(tw, twx);
    const int k = kk;
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int jl = e / L, ii = e - jl * L;
        const int jj = j0 + jl;
        double2 t[6];
        if (jl < nl && ii != g.nx && jj != g.ny && kk != g.nz) {
            const int i = ii > g.nx ? ii - g.X : ii;
            const int j = jj;
            green_value(g, i, j, k, t);
        } else {
#pragma unroll
            for (int q = 0; q < 6; q++) t[q] = make_double2(0, 0);
        }
#pragma unroll
        for (int q = 0; q < 6; q++) sm[ii * LS + q * TL + jl] = t[q];
    }
    __syncthreads();
    tile_fft<C, L, NB, LS, NT, +1>(sm, tw);
    const int W = g.nx + 1;
    for (int e = threadIdx.x; e < NB * W; e += NT) {
        const int bl = e / W, q = e - bl * W;
        const int c = bl / TL, jl = bl - c * TL;
        if (jl < nl) GA[(((long)c * (g.nz + 1) + kk) * (g.ny + 1) + j0 + jl) * W + q] = sm[q * LS + bl];
    }
}

// AXIS 1: GA[c][nz+1][ny+1][W] -> GB[c][nz+1][ny+1][W], rows y > ny read as
// Py(c) times row Y - y;  AXIS 2: GB -> Gc[c][nz+1][ny+1][W], planes z > nz
// read as Pz(c) times plane Z - z
template <int L, int AXIS>
__global__ void __launch_bounds__(GreenTiles<L>::NT) k_green_yz(const GreenGeom g, const double2* __restrict__ src,
                                                                double2* __restrict__ dst64, float2* __restrict__ dst32,
                                                                const double2* __restrict__ tw_axis) {
    using C = double2;
    using TT = GreenTiles<L>;
    constexpr int TL = TT::TLY, NT = TT::NT;
    extern __shared__ __align__(16) unsigned char raw[];
    C* tw = reinterpret_cast<C*>(raw);
    C* sm = tw + L;
    const int W = g.nx + 1;
    const int q0 = blockIdx.x * TL, c = blockIdx.z;
    load_twiddles<C, L, NT>(tw, tw_axis);
    // AXIS 1: blockIdx.y = kk (0..nz), lines along y;  AXIS 2: blockIdx.y = qy (0..ny), lines along z
    const int o = blockIdx.y;
    const int keep = AXIS == 1 ? g.ny + 1 : g.nz + 1;
    const int half = AXIS == 1 ? g.ny : g.nz;
    const double sgn = AXIS == 1 ? green_py(c) : green_pz(c);
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int p = e / TL, il = e - p * TL;
        const int q = q0 + il;
        C v = make_double2(0, 0);
        if (q < W) {
            const int pm = p <= half ? p : L - p;  // the mirror of a negative offset
            long idx;
            if (AXIS == 1) idx = (((long)c * (g.nz + 1) + o) * (g.ny + 1) + pm) * W + q;
            else idx = (((long)c * (g.nz + 1) + pm) * (g.ny + 1) + o) * W + q;
            v = src[idx];
            if (p > half) v = make_double2(sgn * v.x, sgn * v.y);
        }
        sm[e] = v;
    }
    __syncthreads();
    tile_fft<C, L, TL, TL, NT, +1>(sm, tw);
    for (int e = threadIdx.x; e < TL * keep; e += NT) {
        const int p = e / TL, il = e - p * TL;
        const int q = q0 + il;
        if (q >= W) continue;
        long idx;
        if (AXIS == 1) idx = (((long)c * (g.nz + 1) + o) * (g.ny + 1) + p) * W + q;
        else idx = (((long)c * (g.nz + 1) + p) * (g.ny + 1) + o) * W + q;
        const C v = sm[e];
        dst64[idx] = v;
        if (AXIS == 2 && dst32) dst32[idx] = make_float2((float)v.x, (float)v.y);
    }
}

}  // namespace ifdda
