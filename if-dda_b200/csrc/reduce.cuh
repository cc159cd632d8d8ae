// Deterministic two-stage reductions of complex FP64 sums.
//
// Every block reduces its ND running sums in a fixed tree (warp shuffles, then
// one warp over the warp partials), writes them to partials[rhs][blk][ND],
// fences, and takes a ticket.  The block that takes the last ticket sums the
// partials of all blocks in a fixed order and calls the finisher (thread 0),
// which updates the solver scalars on the device.  The result does not depend
// on block scheduling, so repeated runs -- and a right-hand side solved alone
// or inside a batch -- give bit-identical scalars.
#pragma once
#include "cplx.cuh"

namespace ifdda {

__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ double2 shfl_down2(double2 v, int o) {
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, o), __shfl_down_sync(0xffffffffu, v.y, o));
}

// Sum acc over the block; the result is valid in thread 0.  scratch holds
// ND * 32 double2.
template <int NT, int ND>
__device__ __forceinline__ void block_sum(double2 (&acc)[ND], double2* scratch) {
    static_assert(NT % 32 == 0, "block size must be a multiple of 32");
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int m = 0; m < ND; m++) {
        double2 v = acc[m];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = dadd(v, shfl_down2(v, o));
        if (lane == 0) scratch[m * 32 + w] = v;
    }
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int m = 0; m < ND; m++) {
            double2 v = lane < NW ? scratch[m * 32 + lane] : make_double2(0, 0);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = dadd(v, shfl_down2(v, o));
            acc[m] = v;
        }
    }
    __syncthreads();
}

struct RedSlots {
    double2* partials;   // [nrhs][maxblk][ND]
    unsigned* tickets;   // [nrhs]
    int maxblk;          // stride between right-hand sides, in blocks
};

// Stage 2.  Returns true in the one block that finished the reduction; the
// final sums are then in `acc` of thread 0.
template <int NT, int ND>
__device__ __forceinline__ bool reduce_across_blocks(double2 (&acc)[ND], int rhs, int blk, int nblk,
                                                     const RedSlots& rs) {
    __shared__ double2 scratch[ND * 32];
    __shared__ bool am_last;
    block_sum<NT, ND>(acc, scratch);
    double2* part = rs.partials + ((long)rhs * rs.maxblk) * ND;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int m = 0; m < ND; m++) part[(long)blk * ND + m] = acc[m];
        __threadfence();
        const unsigned t = atomicAdd(&rs.tickets[rhs], 1u);
        am_last = (t == (unsigned)(nblk - 1));
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
#pragma unroll
    for (int m = 0; m < ND; m++) acc[m] = make_double2(0, 0);
    for (int q = threadIdx.x; q < nblk; q += NT) {
#pragma unroll
        for (int m = 0; m < ND; m++) acc[m] = dadd(acc[m], __ldcg(part + (long)q * ND + m));
    }
    block_sum<NT, ND>(acc, scratch);
    if (threadIdx.x == 0) rs.tickets[rhs] = 0u;
    return true;
}

// Reductions over the (gx, gy) grid of a mat-vec x pass, per right-hand
// side.  The x passes of one mat-vec have the same grid, so the first pass
// can leave NDP partial sums per block (ppart) that the last pass folds in.
struct MvRed {
    double2* ppart;   // [nrhs][gy][gxs][NDP]  partials of the first x pass
    double2* epart;   // [nrhs][gy][gxs][ND]   partials of the last x pass
    double2* rpart;   // [nrhs][gy][ND + NDP]  row sums
    unsigned* t1;     // [nrhs][gy]            row tickets
    unsigned* t2;     // [nrhs]                grid tickets
    int gxs;          // stride between rows, in blocks (>= gx)
};

// Block sum of acc written to out[0..ND) by thread 0.
template <int NT, int ND>
__device__ __forceinline__ void block_partial(double2 (&acc)[ND], double2* out) {
    __shared__ double2 scratch[ND * 32];
    block_sum<NT, ND>(acc, scratch);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int m = 0; m < ND; m++) out[m] = acc[m];
    }
}

// Two ticket levels: the last block of a row sums that row's ND partials and
// the row's NDP partials of the first pass; the last row sums the rows.  All
// sums run in index order, so the result does not depend on scheduling.
// Returns true in the one block that holds the totals (thread 0's tot).
template <int NT, int ND, int NDP>
__device__ __forceinline__ bool reduce_rows(double2 (&own)[ND], double2 (&tot)[ND + NDP], int rhs, int bx, int by,
                                            int gx, int gy, const MvRed& R) {
    constexpr int NA = ND + NDP;
    __shared__ double2 scratch[NA * 32];
    __shared__ bool last;
    block_sum<NT, ND>(own, scratch);
    const long row = (long)rhs * gy + by;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int m = 0; m < ND; m++) R.epart[(row * R.gxs + bx) * ND + m] = own[m];
        __threadfence();
        last = atomicAdd(&R.t1[row], 1u) == (unsigned)(gx - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int m = 0; m < NA; m++) tot[m] = make_double2(0, 0);
    for (int q = threadIdx.x; q < gx; q += NT) {
#pragma unroll
        for (int m = 0; m < ND; m++) tot[m] = dadd(tot[m], __ldcg(R.epart + (row * R.gxs + q) * ND + m));
#pragma unroll
        for (int m = 0; m < NDP; m++) tot[ND + m] = dadd(tot[ND + m], __ldcg(R.ppart + (row * R.gxs + q) * NDP + m));
    }
    block_sum<NT, NA>(tot, scratch);
    if (threadIdx.x == 0) {
        R.t1[row] = 0u;
#pragma unroll
        for (int m = 0; m < NA; m++) R.rpart[row * NA + m] = tot[m];
        __threadfence();
        last = atomicAdd(&R.t2[rhs], 1u) == (unsigned)(gy - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int m = 0; m < NA; m++) tot[m] = make_double2(0, 0);
    for (int q = threadIdx.x; q < gy; q += NT) {
#pragma unroll
        for (int m = 0; m < NA; m++) tot[m] = dadd(tot[m], __ldcg(R.rpart + ((long)rhs * gy + q) * NA + m));
    }
    block_sum<NT, NA>(tot, scratch);
    if (threadIdx.x == 0) R.t2[rhs] = 0u;
    return true;
}

}  // namespace ifdda
