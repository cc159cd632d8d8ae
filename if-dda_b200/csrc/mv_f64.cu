// FP64-complex mat-vec instantiations (plain drop-in and outer residuals).
#include "mv_impl.cuh"
#include "gpbicg_fused.cuh"

namespace ifdda {
template <> void tune_tiles<double>(Green& G, int nrhs, cudaStream_t st) { tune_tiles_impl<double>(G, nrhs, st); }
template <> bool matvec_launch<double>(const MvArgs<double>& a, int nrhs, bool tab, cudaStream_t st) {
    return matvec_launch_fused<double, PreNone<double>, EpiNone>(a, PreNone<double>{}, EpiNone{}, MvRed{}, nrhs, tab, st);
}
template bool matvec_launch_fused<double, PreGpP<double>, EpiGpAlpha<double>>(const MvArgs<double>&, const PreGpP<double>&,
                                                                   const EpiGpAlpha<double>&, const MvRed&, int,
                                                                   bool, cudaStream_t);
template bool matvec_launch_fused<double, PreGpYT<double>, EpiGpZeta<double>>(const MvArgs<double>&, const PreGpYT<double>&,
                                                                   const EpiGpZeta<double>&, const MvRed&, int,
                                                                   bool, cudaStream_t);
}  // namespace ifdda
