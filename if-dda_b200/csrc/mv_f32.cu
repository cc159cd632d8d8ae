// FP32-complex mat-vec instantiations (inner Krylov iterations).
#include "mv_impl.cuh"

namespace ifdda {
template <> bool matvec_launch<float>(const MvArgs<float>& a, int nrhs, bool tab, cudaStream_t st) {
    return matvec_launch_epi<float, EpiNone>(a, EpiNone{}, nrhs, tab, st);
}
}  // namespace ifdda
