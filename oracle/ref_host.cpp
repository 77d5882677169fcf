// ref_host.cpp — runs the reference's own OpenCL kernels (kernels/*_d.cl, compiled for the CPU through
// ref_shim.h) over an NDRange. TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.py into
// oracle/_ref/libref.so from the sources under the reference tree; used to pin the oracle.
//
// Work items run one after another, except for the kernels with __local memory and barriers
// (transmission_potentials_*, sum_reduction), whose work groups run as teams of threads that share the
// group's __local arrays and meet at a real barrier.
#include "ref_shim.h"

#include <thread>
#include <vector>

thread_local RefWorkItem ref_wi;
thread_local std::barrier<> *ref_bar = nullptr;

namespace ref_atom_sort {
#include "atom_sort_d.inc"
}
namespace ref_band_limit {
#include "band_limit_d.inc"
}
namespace ref_band_pass {
#include "band_pass_d.inc"
}
namespace ref_bilinear_translate {
#include "bilinear_translate_d.inc"
}
namespace ref_complex_multiply {
#include "complex_multiply_d.inc"
}
namespace ref_complex_to_real {
#include "complex_to_real_d.inc"
}
namespace ref_fft_shift {
#include "fft_shift_d.inc"
}
namespace ref_init_plane_wave {
#include "init_plane_wave_d.inc"
}
namespace ref_init_probe_wave {
#include "init_probe_wave_d.inc"
}
namespace ref_propagator {
#include "propagator_d.inc"
}
namespace ref_sqabs {
#include "sqabs_d.inc"
}
namespace ref_sum_reduction {
#include "sum_reduction_d.inc"
}
namespace ref_projected {
#include "transmission_potentials_projected_d.inc"
}
namespace ref_full3d {
#include "transmission_potentials_full_3d_d.inc"
}
namespace ref_ctem_image {
#include "ctem_image_d.inc"
}

namespace {

void set_item(size_t gx, size_t gy, size_t lx, size_t ly, size_t LX, size_t LY, size_t GX, size_t GY) {
    ref_wi.lid[0] = lx; ref_wi.lid[1] = ly;
    ref_wi.grp[0] = gx; ref_wi.grp[1] = gy;
    ref_wi.lsz[0] = LX; ref_wi.lsz[1] = LY;
    ref_wi.gid[0] = gx * LX + lx; ref_wi.gid[1] = gy * LY + ly;
    ref_wi.gsz[0] = GX; ref_wi.gsz[1] = GY;
}

// NDRange without barriers: one work item at a time (local size 1)
template <class F> void ndrange(size_t GX, size_t GY, F &&f) {
    for (size_t y = 0; y < GY; y++)
        for (size_t x = 0; x < GX; x++) {
            set_item(x, y, 0, 0, 1, 1, GX, GY);
            f();
        }
}

// NDRange with work groups of LX*LY threads sharing __local memory and a barrier. A barrier also ends
// every group, so the next group's loads cannot overwrite __local data another thread still reads.
template <class F> void ndrange_groups(size_t GX, size_t GY, size_t LX, size_t LY, F &&f) {
    const size_t L = LX * LY, NGX = GX / LX, NGY = GY / LY;
    std::barrier<> bar((std::ptrdiff_t)L);
    std::vector<std::thread> team;
    for (size_t t = 0; t < L; t++)
        team.emplace_back([&, t] {
            ref_bar = &bar;
            for (size_t gy = 0; gy < NGY; gy++)
                for (size_t gx = 0; gx < NGX; gx++) {
                    set_item(gx, gy, t % LX, t / LX, LX, LY, GX, GY);
                    f();
                    bar.arrive_and_wait();
                }
        });
    for (auto &th : team) th.join();
}

double2 c2(const double *p) { return double2{p[0], p[1]}; }

}  // namespace

extern "C" {

void ref_atom_sort_d(const double *x, const double *y, const double *z, int n, double min_x, double max_x, double min_y,
                     double max_y, double min_z, double max_z, int blocks_x, int blocks_y, int *block_ids, int *z_ids,
                     double dz, int n_slices) {
    ndrange((size_t)n, 1, [&] {
        ref_atom_sort::atom_sort_d(x, y, z, n, min_x, max_x, min_y, max_y, min_z, max_z, blocks_x, blocks_y, block_ids,
                                   z_ids, dz, n_slices);
    });
}

void ref_band_limit_d(double *io, unsigned w, unsigned h, double k_max, double factor, double *kx, double *ky) {
    ndrange(w, h, [&] { ref_band_limit::band_limit_d((double2 *)io, w, h, k_max, factor, kx, ky); });
}

void ref_band_pass_d(const double *in, double *out, unsigned w, unsigned h, double inner, double outer, double xc, double yc) {
    ndrange(w, h, [&] { ref_band_pass::band_pass_d(in, out, w, h, inner, outer, xc, yc); });
}

void ref_bilinear_translate_d(const double *in, double *out, int ix, int iy, double sx, double sy, unsigned w, unsigned h) {
    ndrange(w, h, [&] { ref_bilinear_translate::bilinear_translate_d((double *)in, out, ix, iy, sx, sy, w, h); });
}

void ref_complex_multiply_d(double *a, double *b, double *out, unsigned w, unsigned h) {
    ndrange(w, h, [&] { ref_complex_multiply::complex_multiply_d((double2 *)a, (double2 *)b, (double2 *)out, w, h); });
}

void ref_complex_to_real_d(double *in, double *out, int method, unsigned w, unsigned h) {
    ndrange(w, h, [&] { ref_complex_to_real::complex_to_real_d((double2 *)in, out, method, w, h); });
}

void ref_fft_shift_d(const double *in, double *out, unsigned w, unsigned h) {
    ndrange(w, h, [&] { ref_fft_shift::fft_shift_d((const double2 *)in, (double2 *)out, w, h); });
}

void ref_init_plane_wave_d(double *out, unsigned w, unsigned h, double value) {
    ndrange(w, h, [&] { ref_init_plane_wave::init_plane_wave_d((double2 *)out, w, h, value); });
}

// ab: C12, C21, C23, C32, C34, C41, C43, C45, C52, C54, C56 as (re, im) pairs (22 doubles)
void ref_init_probe_wave_d(double *out, unsigned w, unsigned h, const double *kx, const double *ky, double pos_x, double pos_y,
                           double wavelength, double C10, double C30, double C50, const double *ab, double cond_ap,
                           double ap_smooth) {
    ndrange(w, h, [&] {
        ref_init_probe_wave::init_probe_wave_d((double2 *)out, w, h, kx, ky, pos_x, pos_y, wavelength, C10, c2(ab + 0),
                                               c2(ab + 2), c2(ab + 4), C30, c2(ab + 6), c2(ab + 8), c2(ab + 10), c2(ab + 12),
                                               c2(ab + 14), C50, c2(ab + 16), c2(ab + 18), c2(ab + 20), cond_ap, ap_smooth);
    });
}

void ref_ctem_image_d(const double *in, double *out, unsigned w, unsigned h, double *kx, double *ky, double wavelength,
                      double C10, double C30, double C50, const double *ab, double obj_ap, double ap_smooth, double beta,
                      double delta) {
    ndrange(w, h, [&] {
        ref_ctem_image::ctem_image_d((const double2 *)in, (double2 *)out, w, h, kx, ky, wavelength, C10, c2(ab + 0),
                                     c2(ab + 2), c2(ab + 4), C30, c2(ab + 6), c2(ab + 8), c2(ab + 10), c2(ab + 12),
                                     c2(ab + 14), C50, c2(ab + 16), c2(ab + 18), c2(ab + 20), obj_ap, ap_smooth, beta, delta);
    });
}

void ref_propagator_d(double *prop, double *kx, double *ky, unsigned w, unsigned h, double dz, double beam_k, double bkx,
                      double bky, double bkz, double k_max) {
    ndrange(w, h, [&] { ref_propagator::propagator_d((double2 *)prop, kx, ky, w, h, dz, beam_k, bkx, bky, bkz, k_max); });
}

void ref_sqabs_d(const double *in, double *out, unsigned w, unsigned h) {
    ndrange(w, h, [&] { ref_sqabs::sqabs_d((const double2 *)in, (double2 *)out, w, h); });
}

// global size = size, local size 256 (simulationstem.cpp:125-131); out holds size/256 group sums
void ref_sum_reduction_d(const double *in, double *out, unsigned size) {
    static double buffer[256];
    ndrange_groups(size, 1, 256, 1, [&] { ref_sum_reduction::sum_reduction_d(in, out, size, buffer); });
}

// pot: int args (param_selector, param_i_count, width, height, current_slice, total_slices, blocks_x,
//      blocks_y, block_load_x, block_load_y, slice_load_z, integrals)
//      double args (dz, pixelscale, max_x, min_x, max_y, min_y, sigma, startx, starty,
//                   beam_theta | current_z, beam_phi | shift_x, shift_y)
void ref_transmission_projected_d(double *out, const double *px, const double *py, const double *pz, const int *Z,
                                  const double *params, const int *ia, const double *da, const int *block_start) {
    ndrange_groups((size_t)ia[2], (size_t)ia[3], 16, 16, [&] {
        ref_projected::transmission_potentials_projected_d(
            (double2 *)out, px, py, pz, Z, params, (unsigned)ia[0], (unsigned)ia[1], block_start, (unsigned)ia[2],
            (unsigned)ia[3], ia[4], ia[5], da[0], da[1], ia[6], ia[7], da[2], da[3], da[4], da[5], ia[8], ia[9], ia[10],
            da[6], da[7], da[8], da[9], da[10]);
    });
}

void ref_transmission_full3d_d(double *out, const double *px, const double *py, const double *pz, const int *Z,
                               const double *params, const int *ia, const double *da, const int *block_start) {
    ndrange_groups((size_t)ia[2], (size_t)ia[3], 16, 16, [&] {
        ref_full3d::transmission_potentials_full_3d_d(
            (double2 *)out, px, py, pz, Z, params, (unsigned)ia[0], (unsigned)ia[1], block_start, (unsigned)ia[2],
            (unsigned)ia[3], ia[4], ia[5], da[0], da[1], ia[6], ia[7], da[2], da[3], da[4], da[5], ia[8], ia[9], ia[10],
            da[6], da[7], da[8], da[9], da[10], da[11], ia[11]);
    });
}

}  // extern "C"
