// misc.cuh — declarations of the non-FFT device operations (atoms, tables, reductions, imaging).
#pragma once

#include "common.cuh"

namespace ms {

struct SortGeom {
    double full_x0, full_x1, full_y0, full_y1;   // padded full limits (strict host filter + atom_sort range)
    double z0, z1;                               // padded z limits
    double dz;
    int blocks_x, blocks_y, n_slices;
};

// Atom binning: filter + atom_sort ids + stable sort by (slice, y bin, x bin) + block_start.
// Scratch (device): keys/idx in/out, cub temp. Returns nothing on the host; count_in_range lands in
// block_start[n_slices*bx*by].
struct AtomSortBuffers {
    int *keys_in, *keys_out, *idx_in, *idx_out;   // n each
    int *bid, *zid, *kept;                        // n each: atom_sort ids (input order), filter flag
    int *counts;                                  // n_bins + 1
    void *cub_temp;
    size_t cub_temp_bytes;
};
size_t atom_sort_temp_bytes(int n, int n_bins);
void atom_sort(cudaStream_t s, const SortGeom &g, int n, const int *Z, const double *x, const double *y, const double *z,
               AtomSortBuffers &buf, int *block_start, int *Zs, double *xs, double *ys, double *zs);

// init_probe_wave aperture + aberration phase table: chi[y*N+x] = (chi, inside ? 1 : 0)
struct AberrD {
    double C10, C30, C50;
    double2 C12, C21, C23, C32, C34, C41, C43, C45, C52, C54, C56;
};
void chi_table(cudaStream_t s, int n, const double *kx, const double *ky, double wavelength, const AberrD &A,
               double cond_ap, double ap_smooth, double2 *out);
// STEM detector bit masks in unshifted k-space pixel order (band_pass_d.cl:15-38 on fft-shifted pixels)
void detector_masks(cudaStream_t s, int n, int n_det, const double *innerPx, const double *outerPx, const double *xcPx,
                    const double *ycPx, uint16_t *out);
// Sum each wave's detector partials (fixed order), times sqrt(2) (sum_reduction_d.cl:30), into
// out[(o*n_det + d)*n_pix + pixel[b]]: Kahan-accumulated when comp != nullptr, stored otherwise.
void detector_reduce(cudaStream_t s, const double *partials, int n_blocks, int n_det, int batch, const int *pixel_of_wave,
                     int n_pix, int o, double *out, double *comp);
// Diffraction |fftshift(recip)|^2 (getDiffractionImage, simulationgeneral.cpp:772-806) into out (double);
// Kahan-accumulated when comp != nullptr.
template <class R> void diffraction(cudaStream_t s, int n, const cplx<R> *recip, double *out, double *comp);
// A translation of the diffraction pattern by (ix + sx, iy + sy) pixels, 0 <= sx, sy < 1
// (SimulationGeneral::translateDiffImage, simulationgeneral.cpp:832-853)
struct Shift2 {
    int ix, iy;
    double sx, sy;
};
// The diffraction pattern translated by sh (bilinear_translate_d.cl:18-77) into out, Kahan-accumulated when
// comp != nullptr (getDiffractionImage with d_kx, d_ky != 0, simulationgeneral.cpp:772-806)
template <class R> void diffraction_shifted(cudaStream_t s, int n, const cplx<R> *recip, Shift2 sh, double *out, double *comp);
// STEM detectors on each wave's translated pattern (getStemPixel with d_kx, d_ky != 0): FP64 block partials at
// partials[(wave * n_det + d) * blocks + block]; returns blocks (the n_blocks of detector_reduce)
template <class R> int detectors_shifted(cudaStream_t s, int n, int batch, const cplx<R> *recip, Shift2 sh, int n_det,
                                         const double *innerPx, const double *outerPx, const double *xcPx,
                                         const double *ycPx, double *partials);
// |psi|^2 into double
template <class R> void sqabs_to_double(cudaStream_t s, size_t count, const cplx<R> *in, double *out);
// ctem_image_d (kernels/ctem_image_d.cl:50-119) on the reciprocal exit wave
template <class R> void ctem_transfer(cudaStream_t s, int n, const cplx<R> *in, cplx<R> *out, const double *kx,
                                      const double *ky, double wavelength, const AberrD &A, double obj_ap, double ap_smooth,
                                      double beta, double delta);
// row-transformed plane wave: phi_0 = D_r(1) = res at kx = 0 in every row (init_plane_wave_d.cl value 1.0)
template <class R> void plane_wave_state(cudaStream_t s, int n, cplx<R> *wave);
// |z|^2 + 0i in place (sqabs_d.cl)
template <class R> void sqabs_complex(cudaStream_t s, size_t count, cplx<R> *io);
// CCD detective quantum efficiency (dqe = true: multiply by sqrt) or noise transfer function on an unshifted
// reciprocal image (ccd_dqe_d.cl, ccd_ntf_d.cl); table of 725 radial values per binned pixel
template <class R> void ccd_filter(cudaStream_t s, int n, cplx<R> *io, const double *table, int binning, bool dqe);
// the real part into double (SimulationCtem::getCtemImage)
template <class R> void real_part_to_double(cudaStream_t s, size_t count, const cplx<R> *in, double *out);
// complex copy with conversion
template <class R> void convert_to_double(cudaStream_t s, size_t count, const cplx<R> *in, double2 *out);
template <class R> void convert_from_double(cudaStream_t s, size_t count, const double2 *in, cplx<R> *out);

}  // namespace ms
