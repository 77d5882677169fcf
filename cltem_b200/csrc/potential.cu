// potential.cu — launchers of the slice-potential kernels for one precision (compiled per MS_REAL;
// the FP64 build uses -fmad=false so the _d statements are not contracted).
#include "potential.cuh"
#include "potential_launch.h"

#include <type_traits>

#ifndef MS_REAL
#error "MS_REAL must be defined"
#endif

namespace ms {

// the FP32 full-3D kernel (a template, so that the FP64 build discards it)
template <class T>
bool potential_3d_f(cudaStream_t s, dim3 grd, dim3 blk, cplx<T> *out, const double *ax, const double *ay,
                    const double *az, const int *aZ, const int *block_start, const float4 *tab3, const PotParams &p) {
    if constexpr (std::is_same<T, float>::value) {
        constexpr int PX = kPot3Px;
        const dim3 b2(16 / PX, 16);   // PX pixels a thread
        if (p.form == 0) k_potential_3d_f<0, PX><<<grd, b2, 0, s>>>(out, ax, ay, az, aZ, block_start, tab3, p);
        else if (p.form == 1) k_potential_3d_f<1, PX><<<grd, b2, 0, s>>>(out, ax, ay, az, aZ, block_start, tab3, p);
        else k_potential_3d_f<2, PX><<<grd, b2, 0, s>>>(out, ax, ay, az, aZ, block_start, tab3, p);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}

// the FP32 projected kernel (a template, so that the FP64 build discards it)
template <class T>
bool potential_projected_f(cudaStream_t s, dim3 grd, cplx<T> *out, const double *ax, const double *ay, const int *aZ,
                           const int *block_start, const float2 *tabp, const PotParams &p) {
    if constexpr (std::is_same<T, float>::value) {
        constexpr int PX = kPotPPx;
        const dim3 b(16 / PX, 16);   // PX pixels a thread
        if (p.form == 0) k_potential_projected_f<0, PX><<<grd, b, 0, s>>>(out, ax, ay, aZ, block_start, tabp, p);
        else if (p.form == 1) k_potential_projected_f<1, PX><<<grd, b, 0, s>>>(out, ax, ay, aZ, block_start, tabp, p);
        else k_potential_projected_f<2, PX><<<grd, b, 0, s>>>(out, ax, ay, aZ, block_start, tabp, p);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}

// the FP64 kernels (a template, so that the FP32 build discards them)
template <class T>
void potential_d(cudaStream_t s, bool full3d, dim3 grd, dim3 blk, cplx<T> *out, const double *ax, const double *ay,
                 const double *az, const int *aZ, const int *block_start, const T *prm, const PotParams &p) {
    if constexpr (std::is_same<T, double>::value) {
        if (full3d) {
            if (p.form == 0) k_potential_3d<T, 0><<<grd, blk, 0, s>>>(out, ax, ay, az, aZ, block_start, prm, p);
            else if (p.form == 1) k_potential_3d<T, 1><<<grd, blk, 0, s>>>(out, ax, ay, az, aZ, block_start, prm, p);
            else k_potential_3d<T, 2><<<grd, blk, 0, s>>>(out, ax, ay, az, aZ, block_start, prm, p);
        } else {
            if (p.form == 0) k_potential_projected<T, 0><<<grd, blk, 0, s>>>(out, ax, ay, aZ, block_start, prm, p);
            else if (p.form == 1) k_potential_projected<T, 1><<<grd, blk, 0, s>>>(out, ax, ay, aZ, block_start, prm, p);
            else k_potential_projected<T, 2><<<grd, blk, 0, s>>>(out, ax, ay, aZ, block_start, prm, p);
        }
        MS_CUDA(cudaGetLastError());
    }
}

template <>
void launch_potential<MS_REAL>(cudaStream_t s, bool full3d, cplx<MS_REAL> *out, int n_slices, const double *ax,
                               const double *ay, const double *az, const int *aZ, const int *block_start,
                               const MS_REAL *prm, const float4 *tab3, const float2 *tabp, const PotParams &p) {
    using T = MS_REAL;
    if (p.width % 16 || p.height % 16) throw std::runtime_error("potential grid must be a multiple of 16");
    dim3 blk(16, 16), grd(p.width / 16, p.height / 16, n_slices);
    if (n_slices <= 0) return;
    if constexpr (std::is_same<T, float>::value) {   // the FP32 engine: the table kernels
        if (full3d ? tab3 == nullptr : tabp == nullptr)
            throw std::runtime_error("the FP32 potentials need the term tables of the loaded parameterisation");
        (void)prm;
        if (full3d) potential_3d_f<T>(s, grd, blk, out, ax, ay, az, aZ, block_start, tab3, p);
        else potential_projected_f<T>(s, grd, out, ax, ay, aZ, block_start, tabp, p);
    } else {   // the FP64 engine: the reference's _d statements
        potential_d<T>(s, full3d, grd, blk, out, ax, ay, az, aZ, block_start, prm, p);
    }
}


}  // namespace ms
