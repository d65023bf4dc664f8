// Launchers of the plain FP64 map kernels (map_plain.cu) for other translation units of the library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "acoular_b200.h"

namespace acb {

// Plain full-CSM map of nbins bins (csm (nbins, M, M) complex128, k (nbins,)); with rm != nullptr the
// distances r0 (G,), rm (G, M) are taken as given, else they are computed from mpos / gpos.
int map_plain_launch(const acb_map_params *p, int nbins, const void *csm, const double *k, const double *mpos,
                     const double *gpos, const double *r0, const double *rm, double *out_map, cudaStream_t s);

// Eigenvalue-form map (E components per bin, eigval (nbins, E), eigvec (nbins, M, E)); bins whose
// active[bin] is 0 are skipped (active may be nullptr).
int map_eig_launch(const acb_map_params *p, int nbins, int E, const double *eigval, const void *eigvec,
                   const double *k, const double *mpos, const double *gpos, const double *r0, const double *rm,
                   double *out_map, const int *active, cudaStream_t s);

// Eigenvalue-form map with given steering vectors steer (nbins, G, M) complex128 (custom steering: the
// result is the quadratic form times p->norm, no steering-type normalisation); bins with active[bin] == 0
// are skipped.
int map_eig_custom_launch(const acb_map_params *p, int nbins, int E, const double *eigval, const void *eigvec,
                          const void *steer, double *out_map, const int *active, cudaStream_t s);

}  // namespace acb
