// FP64-complex mat-vec instantiations (plain drop-in and outer residuals).
#include "mv_impl.cuh"

namespace ifdda {
template <> bool matvec_launch<double>(const MvArgs<double>& a, int nrhs, bool tab, cudaStream_t st) {
    return matvec_launch_epi<double, EpiNone>(a, EpiNone{}, nrhs, tab, st);
}
}  // namespace ifdda
