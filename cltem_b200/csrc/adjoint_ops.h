// adjoint_ops.h — host entry points of the differentiable-CTEM kernels (adjoint.cu).
#pragma once

#include "misc.cuh"

namespace ms {

// I = |W|^2, partial[b] = block sums of (I - target)^2, gW = 4 (I - target) W; reduction_blocks() partials
template <class R> void image_loss(cudaStream_t s, size_t n, const cplx<R> *W, const double *target, cplx<R> *gW,
                                   double *partial);
// gRecip = conj(H) gY and the partial sums of dL/dC10, dL/dC30 (H: ctem_image_d.cl transfer)
template <class R> void image_backward(cudaStream_t s, int n, const cplx<R> *recip, const cplx<R> *gY, cplx<R> *gRecip,
                                       const double *kx, const double *ky, double wavelength, const AberrD &A, double obj_ap,
                                       double ap_smooth, double beta, double delta, double *p10, double *p30);
// g <- conj(P) g scale inside the propagator cut
template <class R> void mul_conj_prop(cudaStream_t s, int n, cplx<R> *g, const cplx<R> *px, const cplx<R> *py,
                                      const double *kx2, const double *ky2, double kmax2, R scale);
// gV = sigma Im(conj(E) gE)
template <class R> void grad_v(cudaStream_t s, size_t count, const cplx<R> *E, const cplx<R> *gE, double sigma, double *gV);
// The atoms of up to kGradMaxSlices consecutive slices for one atom_grad launch: slice t holds the sorted
// atoms [start[t], start[t+1]) and reads gV + t * stride (the slices' gV stored one after the other).
constexpr int kGradMaxSlices = 32;
struct GradSlices {
    int start[kGradMaxSlices + 1];
    int n;
    size_t stride;
    // beam tilt of the projected potential: rho^2 = r^2 - tilt_s2 (r . (cphi, sphi))^2 (0: untilted)
    double tilt_s2 = 0, cphi = 1, sphi = 0;
};
// per-atom gradients (x, y) of the atoms of the slices in sl (sorted order) from gV of their slice (gather.cu);
// T is the precision of the per-pixel terms and of prm (the parameterisation table). tabp (FP32 only, may be
// null): the projected term table the FP32 forward kernel evaluates (potp_table); when set, the FP32
// gradient differentiates that same evaluation.
// work: atom_grad_work_doubles(atoms of sl) doubles of scratch (per-band partial sums)
template <class T>
void atom_grad(cudaStream_t s, const GradSlices &sl, const double *ax, const double *ay, const int *aZ, const double *gV,
               int n, double startx, double starty, double dx, int form, const T *prm, int i_lim, const float2 *tabp,
               double *gxy, double *work);
int atom_grad_work_doubles(int max_count);
// Full 3-D potential: dL/d(x, y, z) of every sorted atom, accumulated into grad (3 per atom) from gV of `count`
// slices starting at p.slice0 (gather3d.cu); wscale = the sub-slice thickness (dL/d(trapezoid sum) = wscale gV);
// prm the FP64 parameterisation table
struct PotParams;
void atom_grad_3d(cudaStream_t s, int form, const double *ax, const double *ay, const double *az, const int *aZ,
                  const int *block_start, const double *prm, const PotParams &p, int count, const double *gV,
                  double wscale, double *grad);
int reduction_blocks();

}  // namespace ms
