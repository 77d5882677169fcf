// launch.cuh — host launchers of the pass kernels, one explicit instantiation per (precision, size).
#pragma once

#include "adjoint.cuh"
#include "passes.cuh"
#include "passes_tma.cuh"
#include "passes_tmx.cuh"

#include <string>

namespace ms {

template <class R>
struct PassOps {
    int n = 0;
    int col_blocks = 0;   // blocks per wave of a column pass (number of detector partials per wave)
    // row_step(..., xa, xb, load_all, tsel, tstride): active columns x < xa or x >= xb; tsel (or nullptr) the
    // transmission set of each wave, sets tstride elements apart (see k_row_step)
    // ..., variant): 0 plain; 1, 2 each block also prefetches into L2 the rows of the block one (two) residencies
    // of the grid later; 3 the grid in wave-fastest order (kWaveFastRows); 4-7 the same four with the two-row
    // step of the plain Stockham plan where the size's default row plan is a wide one; then (FP32 wide and
    // radix-24 plans) the same four with the transmission rows staged in shared memory by the copy engine
    // (row_variants of them); ..., err): the error word of the staged variants' bounded waits (tma.cuh StepError)
    void (*row_step)(cudaStream_t, cplx<R> *, int, const cplx<R> *, const cplx<R> *, R, int, int, int, const int *,
                     size_t, int, int *) = nullptr;
    int row_variants = 4;   // 8 or 12 where the alternative plan and the staged rows exist
    std::string (*row_variant_name)(int) = nullptr;   // a description of row variant v
    void (*row_fft)(cudaStream_t, const cplx<R> *, cplx<R> *, int, const cplx<R> *, R, int) = nullptr;
    // col_step(..., mode, tiles_lo, tiles_hi, variant): the leading tiles_lo and trailing tiles_hi column tiles;
    // variant picks the kernel of the plain step (COL_STEP without a reciprocal copy), 0 <= variant <
    // col_variants: 0 the one-block-per-tile kernel at its default tile, then (where valid for the size) the
    // persistent TMA-fed passes and the one-block-per-tile kernel at other tile widths (col_variant_name)
    void (*col_step)(cudaStream_t, cplx<R> *, int, const cplx<R> *, PropTables<R>, R, R, DetArgs, cplx<R> *, int, int,
                     int, int) = nullptr;
    int col_variants = 1;
    int default_col_variant = 0;   // the column kernel a batched STEM run uses until tuned (bit-identical to 0)
    std::string (*col_variant_name)(int) = nullptr;   // a description of column variant v
    int cols_per_tile = 0;
    void (*col_fft)(cudaStream_t, const cplx<R> *, cplx<R> *, int, const cplx<R> *, R, int) = nullptr;
    void (*col_bandlimit)(cudaStream_t, cplx<R> *, int, const cplx<R> *, const double *, const double *, double, R) = nullptr;
    // col_probe(..., pos, scale, dfac, wavelength): dfac (or nullptr) pi * defocus change / wavelength per wave
    void (*col_probe)(cudaStream_t, cplx<R> *, int, const cplx<R> *, const double2 *, const double *, const double *,
                      const double2 *, R, const double *, double) = nullptr;
    // differentiable CTEM (adjoint.cuh)
    void (*row_step_save)(cudaStream_t, cplx<R> *, int, const cplx<R> *, const cplx<R> *, R, cplx<R> *) = nullptr;
    void (*row_adjoint)(cudaStream_t, cplx<R> *, int, const cplx<R> *, const cplx<R> *, R, const cplx<R> *,
                        cplx<R> *) = nullptr;
};

// defined in inst.cu for every supported (R, N)
template <class R, int N> PassOps<R> make_pass_ops();
// switch over the supported sizes; throws for an unsupported one
template <class R> PassOps<R> pass_ops(int n);

#define MS_SIZES(X) X(64) X(96) X(128) X(256) X(384) X(512) X(768) X(1024) X(1536) X(2048) X(3072) X(4096) X(8192)

}  // namespace ms
