// potential_launch.h — host entry of the slice-potential kernels (one instantiation per precision).
#pragma once

#include "common.cuh"

namespace ms {

struct PotParams;

// Launch the projected (full3d = false) or full 3-D potential kernel for `n_slices` consecutive slices
// starting at p.slice0; out holds n_slices res*res complex transmission values. tab3 / tabp: the FP32
// full-3D and projected term tables (pot3_table, potp_table), used by the FP32 build's kernels when set.
template <class T>
void launch_potential(cudaStream_t s, bool full3d, cplx<T> *out, int n_slices, const double *ax, const double *ay,
                      const double *az, const int *aZ, const int *block_start, const T *prm, const float4 *tab3,
                      const float2 *tabp, const PotParams &p);

}  // namespace ms
