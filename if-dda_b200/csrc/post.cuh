// Post-step and incident-field launchers (device pointers).
#pragma once
#include <algorithm>
#include "solver.cuh"

namespace ifdda {

void local_macro_dev(int nb, long nmax, const double2* eps, const double2* loc, double d, double k0, double2* em,
                     int* bad_dev, cudaStream_t st);
// sums land in stt->alpha.x (Cext sum) and stt->beta.x (Cabs sum)
void cross_sections_dev(int nb, const double2* ff0, const double2* ff, const double2* loc, double k0,
                        double2* partials, unsigned* tickets, KState* stt, int* zstatus, cudaStream_t st);
void planewaves_dev(int nb, const double* xs, const double* ys, const double* zs, double k0, double2 E0, int nrhs,
                    const int* beam, const double* a1, const double* a2, const double* pp, double2* out, int* bad,
                    cudaStream_t st);

// far field |E|^2 on the (ntheta+1) x nphi directions (direction itheta * nphi + iphi);
// part holds farfield_chunks(nb) * 3 values per direction
int farfield_chunks(long nb);
void farfield_dev(int nb, const double* xs, const double* ys, const double* zs, const double2* ff, double k0,
                  int ntheta, int nphi, double2* part, double* emod, cudaStream_t st);

// wide near field: fills the enlarged box from the object dipoles (map[s] = l or -1)
void wide_fill_dev(long nw, const int* map, const double2* ff, const double2* ff0, const double2* eps, long nmax,
                   double2* xr, double2* xi, double2* epsw, cudaStream_t st);

// one alpha per dipole from an isotropic (nmax,3,3) tensor; *aniso = 1 if not isotropic
void pola_compact_dev(const double2* pol, long nb, long nmax, double2* alpha, int* aniso, cudaStream_t st);

}  // namespace ifdda
