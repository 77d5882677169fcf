// plain.h — the plain per-probe FP64 comparison path (unfused, cuFFT Z2Z, sync per probe and slice).
#pragma once

#include "common.cuh"

namespace ms {

struct PlainArgs {
    int n, n_slices, n_det, n_outputs, slice_step, scan_nx;
    const double *kx, *ky;        // device k tables
    const double2 *chi;           // device probe chi table
    const double2 *trans;         // device band-limited transmission functions, FP64, n_slices*n*n
    double dz, beam_k, beam_kx, beam_ky, beam_kz, k_max_prop;
    double start_x, start_y, step_x, step_y, sim_x0, sim_y0;
    double fft_scale;             // clFFT scale 1/sqrtf(n*n)
    double innerPx[16], outerPx[16], xcPx[16], ycPx[16];
    unsigned long long *launches; // kernel launch counter (may be null)
};

// Buffers and cuFFT plan of the plain path, kept between calls as the reference keeps its buffers between
// jobs (SimulationGeneral::initialiseBuffers reallocates only when the resolution changes).
struct PlainWork {
    int n = 0;
    double2 *real = nullptr, *recip = nullptr, *tmp = nullptr, *prop = nullptr;
    double *t2 = nullptr, *t3 = nullptr, *red = nullptr;
    int plan = 0;            // cufftHandle
    bool has_plan = false;
    void release();
    ~PlainWork() { release(); }
};

void plain_stem(cudaStream_t s, const PlainArgs &a, PlainWork &w, const int *pixels, size_t n_pix, double *out);

}  // namespace ms
