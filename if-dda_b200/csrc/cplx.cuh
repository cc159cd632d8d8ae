// Complex arithmetic on float2 / double2 and small helpers shared by all kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ifdda {

// Programmatic dependent launch.  A kernel launched with it may start while
// the kernel before it on the stream is still finishing: its blocks run their
// prologue (constant tables, prefetches of constant data), then pdl_wait()
// blocks until the previous kernel has completed and its writes are visible.
// Every block calls pdl_wait() before it reads anything the previous kernel
// wrote and before it exits, so the chain of dependencies stays transitive.
// pdl_trigger() lets the next kernel's blocks be scheduled once every block
// of this one has started.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename T> struct cvec;
template <> struct cvec<float> { using type = float2; };
template <> struct cvec<double> { using type = double2; };
template <typename T> using cplx = typename cvec<T>::type;

__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

template <class C> __host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <class C> __host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <class C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
template <class C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
    return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <class C, class S> __host__ __device__ __forceinline__ C cscale(C a, S s) { return mk(a.x * s, a.y * s); }
template <class C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
// multiply by (sign * i)
template <int SIGN, class C> __host__ __device__ __forceinline__ C cmul_i(C a) {
    return SIGN > 0 ? mk(-a.y, a.x) : mk(a.y, -a.x);
}
template <class C> __host__ __device__ __forceinline__ C czero() { return mk(decltype(C().x)(0), decltype(C().x)(0)); }

// Global load that asks L2 to fetch the PF bytes (128 or 256; 0: a plain
// load) around the address from DRAM (PTX ld .L2::<PF>B): for narrow rows
// that neighbouring blocks read at the same time, the DRAM accesses become
// wider bursts.
template <int PF> __device__ __forceinline__ float2 ld_l2pf(const float2* p) {
    float2 v;
    if constexpr (PF == 256)
        asm volatile("ld.global.L2::256B.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    else if constexpr (PF == 128)
        asm volatile("ld.global.L2::128B.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    else
        v = *p;
    return v;
}
template <int PF> __device__ __forceinline__ double2 ld_l2pf(const double2* p) {
    double2 v;
    if constexpr (PF == 256)
        asm volatile("ld.global.L2::256B.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    else if constexpr (PF == 128)
        asm volatile("ld.global.L2::128B.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
    else
        v = *p;
    return v;
}

__host__ __device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }
__host__ __device__ __forceinline__ double2 to_d(double2 a) { return a; }
template <class C> __host__ __device__ __forceinline__ C from_d(double2 a);
template <> __host__ __device__ __forceinline__ float2 from_d<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __host__ __device__ __forceinline__ double2 from_d<double2>(double2 a) { return a; }

__host__ __device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
    // a / b with scaling against overflow (Smith's algorithm)
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    } else {
        double r = b.x / b.y, den = b.x * r + b.y;
        return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
    }
}
__host__ __device__ __forceinline__ bool zisnull(double2 a) { return a.x == 0.0 && a.y == 0.0; }
__host__ __device__ __forceinline__ double zabs(double2 a) { return hypot(a.x, a.y); }

}  // namespace ifdda
