// Green-tensor spectrum on sm_100a, FP64 (replaces cdmlib/calculgreenfft.f:1-104
// with cdmlib/espace_libre.f:2-43 evaluated on the fly).
//
//   gx : for every (j, k) line of the padded grid, evaluate the 6 independent
//        components of T(r) at r = (i, j, k) d with wrapped negative offsets
//        and zero planes at i = nx, j = ny, k = nz (calculgreenfft.f:25-69),
//        FFT along x (sign +1), keep qx in [0, nx]        -> GA[c][Z][Y][nx+1]
//   gy : FFT along y, keep qy in [0, ny]                   -> GB[c][Z][ny+1][nx+1]
//   gz : FFT along z, keep qz in [0, nz]                   -> Gc64, Gc32
// Only the parity octant is kept: every component is even or odd along each
// axis, so the rest of the spectrum is a mirror image (see matvec_kernels.cuh).
#pragma once
#include "fft_tile.cuh"

namespace ifdda {

struct GreenGeom {
    int nx, ny, nz, X, Y, Z;
    double d, k0;
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

template <int L>
__global__ void __launch_bounds__(GreenTiles<L>::NT) k_green_x(const GreenGeom g, double2* __restrict__ GA,
                                                               const double2* __restrict__ twx) {
    using C = double2;
    using TT = GreenTiles<L>;
    constexpr int TL = TT::TLX, NB = 6 * TL, LS = TT::LSX, NT = TT::NT;
    extern __shared__ __align__(16) unsigned char raw[];
    C* tw = reinterpret_cast<C*>(raw);
    C* sm = tw + L;
    const int j0 = blockIdx.x * TL, kk = blockIdx.y;
    const int nl = min(TL, g.Y - j0);
    load_twiddles<C, L, NT>(tw, twx);
    const int k = kk > g.nz ? kk - g.Z : kk;
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int jl = e / L, ii = e - jl * L;
        const int jj = j0 + jl;
        double2 t[6];
        if (jl < nl && ii != g.nx && jj != g.ny && kk != g.nz) {
            const int i = ii > g.nx ? ii - g.X : ii;
            const int j = jj > g.ny ? jj - g.Y : jj;
            green_point(i * g.d, j * g.d, k * g.d, g.k0, t);
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
        if (jl < nl) GA[(((long)c * g.Z + kk) * g.Y + j0 + jl) * W + q] = sm[q * LS + bl];
    }
}

// AXIS 1: GA[c][Z][Y][W] -> GB[c][Z][ny+1][W];  AXIS 2: GB -> Gc[c][nz+1][ny+1][W]
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
    // AXIS 1: blockIdx.y = kk (0..Z-1), lines along y;  AXIS 2: blockIdx.y = qy (0..ny), lines along z
    const int o = blockIdx.y;
    const int keep = AXIS == 1 ? g.ny + 1 : g.nz + 1;
    for (int e = threadIdx.x; e < TL * L; e += NT) {
        const int p = e / TL, il = e - p * TL;
        const int q = q0 + il;
        C v = make_double2(0, 0);
        if (q < W) {
            long idx;
            if (AXIS == 1) idx = (((long)c * g.Z + o) * g.Y + p) * W + q;
            else idx = (((long)c * g.Z + p) * (g.ny + 1) + o) * W + q;
            v = src[idx];
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
        if (AXIS == 1) idx = (((long)c * g.Z + o) * (g.ny + 1) + p) * W + q;
        else idx = (((long)c * (g.nz + 1) + p) * (g.ny + 1) + o) * W + q;
        const C v = sm[e];
        dst64[idx] = v;
        if (AXIS == 2 && dst32) dst32[idx] = make_float2((float)v.x, (float)v.y);
    }
}

}  // namespace ifdda
