// FP32-complex mat-vec instantiations (inner Krylov iterations).
#include "mv_impl.cuh"
#include "gpbicg_fused.cuh"

namespace ifdda {
template <> void tune_tiles<float>(Green& G, int nrhs, cudaStream_t st) { tune_tiles_impl<float>(G, nrhs, st); }
template <> bool matvec_launch<float>(const MvArgs<float>& a, int nrhs, bool tab, cudaStream_t st) {
    return matvec_launch_fused<float, PreNone<float>, EpiNone>(a, PreNone<float>{}, EpiNone{}, MvRed{}, nrhs, tab, st);
}
template bool matvec_launch_fused<float, PreGpP<float>, EpiGpAlpha<float>>(const MvArgs<float>&, const PreGpP<float>&,
                                                                   const EpiGpAlpha<float>&, const MvRed&, int,
                                                                   bool, cudaStream_t);
template bool matvec_launch_fused<float, PreGpYT<float>, EpiGpZeta<float>>(const MvArgs<float>&, const PreGpYT<float>&,
                                                                   const EpiGpZeta<float>&, const MvRed&, int,
                                                                   bool, cudaStream_t);
}  // namespace ifdda
