// passes.cuh — the fused row / column passes of the multislice step and their variants.
//
// Wave layout in HBM: a batch of res x res complex waves, wave b at wave + b*res*res, row-major with x
// fastest (element (x, y) at x + res*y, as the reference kernels index it). Between passes a wave is
// kept "row transformed": state phi = D_r psi, where D_r / D_c are the unnormalised 1-D DFTs along
// rows / columns. One multislice step of the reference (simulationgeneral.cpp:744-764:
// Recip = P * FFT(T psi); psi' = IFFT(Recip), clFFT unitary scale s2d = 1/sqrtf(res*res) per 2-D
// transform) then becomes two passes, each one read + one write of the wave:
//   row pass    : phi <- D_r( T_s * a * Dinv_r phi )                       (a = 1/res)
//   column pass : phi <- Dinv_c( b * P * D_c phi )                        (b = s2d^2 * res)
// and after the column pass's multiply by P the tile holds Recip / s2d, which is where the STEM
// detectors, the diffraction pattern and the CTEM image are read (times s2d).
#pragma once

#include "fft.cuh"
#include "fft_wide.cuh"
#include "fft_pair.cuh"
#include "tma.cuh"

#include <type_traits>

namespace ms {

constexpr int kMaxDetectors = 16;
constexpr size_t kMaxBlockSmem = 227 * 1024;   // dynamic shared memory one block may opt in to (sm_100)

template <class R>
struct PropTables {
    const cplx<R> *px;   // res: exp(-i pi dz (kx+bx)^2/kz) * f * exp(i pi dz (k^2-kz^2)/kz)
    const cplx<R> *py;   // res: exp(-i pi dz (ky+by)^2/kz)
    const double *kx2;   // res: kx*kx (FP64, the reference's k0x)
    const double *ky2;   // res: ky*ky
    double kmax2;        // (k_max * limit_factor)^2 of the propagator's strict cut (propagator_d.cl:34-36)
    const int2 *ycut;    // res: column x keeps rows y < ycut[x].x and y >= ycut[x].y, the same cut tabulated
    int *err = nullptr;  // error word of the persistent passes (passes_tma.cuh), or nullptr
    // FP32: the relative representation errors of px and py, (p64 - p32) / p32 formed in FP64 and rounded
    const cplx<R> *pxe = nullptr;
    const cplx<R> *pye = nullptr;
};

// v times the propagator factor px * py of its k (inside the strict cut; the caller zeroes the rest).
// FP64: v (px py), the reference's product. FP32: a factor rounded to FP32 carries a representation error
// that is the same at every slice, so it would add up linearly with thickness (tens of slices reach the
// 1e-5 tolerance). Here v is multiplied by px and then by py, whose roundings depend on v and do not repeat,
// and the product is then corrected by (1 + ex + ey), the relative errors of the FP32 factors against
// their FP64 values: the factor applied matches the FP64 propagator to second order in those errors.
template <class R>
__device__ __forceinline__ cplx<R> prop_mul(cplx<R> v, cplx<R> px, cplx<R> py, cplx<R> ex, cplx<R> ey) {
    if constexpr (sizeof(R) == 8) {
        (void)ex; (void)ey;
        return cmul(v, cmul(px, py));
    } else {
        const cplx<R> u = cmul(cmul(v, px), py);
        return cadd(u, cmul(u, cadd(ex, ey)));
    }
}

struct DetArgs {
    const uint16_t *mask;   // res*res bit masks of the detectors, unshifted k-space pixel order
    int n_det;
    double *partials;       // [batch][n_det][gridDim.x]
};

// Row tiles: ROWS rows per block, P::NT threads per row (P the FFT plan: the wide two-stage plan for FP32
// at 256 / 512 / 1024, the three-stage wide plan at 2048 to 8192 and the radix-24 plans at 384 to 3072,
// fft_wide.cuh; the radix-8/4/2/3 Stockham plan otherwise, fft.cuh).
template <int N, class R> struct RowCfg {
    static constexpr bool WIDE = wide_plan<R>(N);
    static constexpr bool WIDE3 = !WIDE && wide3_plan<R>(N);   // the three-stage wide plan (FP32 2048, 4096)
    static constexpr bool WIDE24 = wide24_plan<R>(N);            // the radix-24 plans (FP32 384 to 3072)
    using P = std::conditional_t<WIDE, WidePlan<N>,
                                 std::conditional_t<WIDE3, Wide3Plan<N>, std::conditional_t<WIDE24, Wide24Plan<N>, Plan<N>>>>;
    static constexpr int ROWS = WIDE ? 8 : (WIDE3 ? (N == 2048 ? 2 : 1) : (WIDE24 ? 128 / (N / 24)
                                                   : (N <= 128 ? 8 : (N <= 256 ? 8 : (N <= 512 ? 4 : (N <= 1024 ? 2 : 1))))));
    static_assert(N % ROWS == 0, "row tile must divide the grid");
    static_assert(P::NT * ROWS <= 1024, "row block too large");
    static constexpr int THREADS = P::NT * ROWS;
    static_assert(ROWS <= 15, "one named barrier per row");
    // radix-8 plan: a row's threads are whole warps, so each row synchronises on its own named barrier;
    // wide plan (and radix-24 plans of at most 32 threads a row): a row's threads lie inside one warp (two rows
    // per warp at 16 threads a row)
    static constexpr bool WARP = WIDE || (WIDE24 && P::NT <= 32);
    static constexpr bool NAMED = !WARP && (P::NT % 32) == 0 && ROWS > 1;
    static_assert(!WIDE || (P::NT == 32 || (P::NT == 16 && ROWS % 2 == 0)), "wide rows must tile whole warps");
    // twiddle entries staged in shared memory, and the offset of the row plan's table (Ctx::twiddles)
    static constexpr int TWN = WIDE ? WidePlan<N>::TW : (WIDE3 ? Wide3Plan<N>::TW : (WIDE24 ? Wide24Plan<N>::TW : N));
    static constexpr int TW_OFF = (WIDE || WIDE3 || WIDE24) ? N : 0;
    static constexpr int ROWSZ =
        WIDE ? WidePlan<N>::ROWSZ : (WIDE3 ? Wide3Plan<N>::ROWSZ : (WIDE24 ? Wide24Plan<N>::ROWSZ : RowAddr::size(N)));
    // the table is read from global memory (L1 / L2) when it and the rows do not both fit (FP64 8192)
    static constexpr bool TWG = sizeof(cplx<R>) * (size_t)(TWN + ROWS * ROWSZ) > kMaxBlockSmem;
    static constexpr int TWS = TWG ? 0 : TWN;   // twiddle entries staged in shared memory
    static constexpr size_t smem() { return sizeof(cplx<R>) * (size_t)(TWS + ROWS * ROWSZ); }
    static_assert(smem() <= kMaxBlockSmem, "row tile exceeds shared memory");
};
// Column tiles: COLS columns per block (a power of two dividing N), P::NT threads per column. FP64: wider
// tiles than one 16-byte column measured faster per probe·slice in a STEM run (768²: 4 against 2 columns
// −15%; 1536², 2048², 3072²: 2 against 1 −25%, −19%, −25%) and slower at 512² (8 against 4: +25%) and
// 1024² (4 against 2: +1%); at 4096² and 8192² two columns need more than 1,024 threads. Radix-8 plan:
// 512-thread blocks at the common sizes, a tile row of COLS complex values 64 B (FP32, N <= 512). Wide plan:
// 128-thread blocks. Columns use the radix-8 plan at every size: measured at 512^2 FP32, the wide plan's
// column pass (4 x 128-thread blocks per SM) took 609 us per 512-wave launch against 558 us for the radix-8
// tiles at 3 x 512 threads per SM, while the wide row pass took 470 us against 569 us.
constexpr bool kWideColumns = false;
template <int N, class R> struct ColCfg {
    static constexpr bool WIDE = kWideColumns && wide_plan<R>(N);
    using P = std::conditional_t<WIDE, WidePlan<N>, Plan<N>>;
    static constexpr int COLS = WIDE ? (N <= 512 ? 8 : 4)
                                     : (sizeof(R) == 4 ? (N <= 512 ? 8 : (N <= 1024 ? 4 : (N <= 4096 ? 2 : 1)))
                                                       : (N <= 768 ? 4 : (N <= 3072 ? 2 : 1)));
    static_assert(N % COLS == 0, "column tile must divide the grid");
    static constexpr int THREADS = P::NT * COLS;
    static_assert(THREADS <= 1024, "column block too large");
    static constexpr int TWN = WIDE ? WidePlan<N>::TW : N;
    static constexpr int COLSZ = WIDE ? WidePlan<N>::ROWSZ : N;   // shared elements of one column
    static constexpr bool TWG = sizeof(cplx<R>) * (size_t)(TWN + COLSZ * COLS) > kMaxBlockSmem;   // as RowCfg
    static constexpr int TWS = TWG ? 0 : TWN;
    static constexpr size_t smem() { return sizeof(cplx<R>) * (size_t)(TWS + COLSZ * COLS); }
    static_assert(smem() <= kMaxBlockSmem, "column tile exceeds shared memory");
    // Blocks per SM the step pass is compiled for: 3 x 512 threads for the FP32 radix-8 plans (a 42-register
    // budget; the 2 blocks of a 52-register build leave its global loads exposed), 4 x 128 threads for the
    // wide plan (128 registers), else what fits.
    static constexpr int STEP_MINB = WIDE ? 4 : ((sizeof(R) == 4 && Plan<N>::E == 8 && THREADS == 512) ? 3 : 1);
};

// the pass kernels' transforms over one row / one column tile (t: the thread's index within its transform)
template <class R, int N, int SIGN>
__device__ __forceinline__ void row_transform(cplx<R> (&v)[RowCfg<N, R>::P::E], cplx<R> *sm, int t, const cplx<R> *tw) {
    using RC = RowCfg<N, R>;
    if constexpr (RC::WIDE) fft_wide<R, N, SIGN>(v, sm, WideRowAddr<RC::P::E>(), t, tw, WarpSync());
    else if constexpr (RC::WIDE3 && RC::NAMED)
        fft_stages<R, N, SIGN, 0, WideRowAddr<32>, NamedSync, Wide3Plan<N>>(v, sm, WideRowAddr<32>(), t, tw,
                                                                            NamedSync{1 + (int)threadIdx.y, RC::P::NT});
    else if constexpr (RC::WIDE3)
        fft_stages<R, N, SIGN, 0, WideRowAddr<32>, BlockSync, Wide3Plan<N>>(v, sm, WideRowAddr<32>(), t, tw, BlockSync());
    else if constexpr (RC::WIDE24 && RC::WARP)
        fft_stages<R, N, SIGN, 0, Wide24Addr<N>, WarpSync, Wide24Plan<N>>(v, sm, Wide24Addr<N>(), t, tw, WarpSync());
    else if constexpr (RC::WIDE24 && RC::NAMED)
        fft_stages<R, N, SIGN, 0, Wide24Addr<N>, NamedSync, Wide24Plan<N>>(v, sm, Wide24Addr<N>(), t, tw,
                                                                          NamedSync{1 + (int)threadIdx.y, RC::P::NT});
    else if constexpr (RC::WIDE24)
        fft_stages<R, N, SIGN, 0, Wide24Addr<N>, BlockSync, Wide24Plan<N>>(v, sm, Wide24Addr<N>(), t, tw, BlockSync());
    else if constexpr (RC::NAMED) fft<R, N, SIGN>(v, sm, RowAddr(), t, tw, NamedSync{1 + (int)threadIdx.y, RC::P::NT});
    else fft<R, N, SIGN>(v, sm, RowAddr(), t, tw);
}
template <class R, int N, int SIGN>
__device__ __forceinline__ void col_transform(cplx<R> (&v)[ColCfg<N, R>::P::E], cplx<R> *sm, int t, const cplx<R> *tw) {
    using CC = ColCfg<N, R>;
    if constexpr (CC::WIDE) fft_wide<R, N, SIGN>(v, sm, WideColAddr<CC::P::E, CC::COLS>(), t, tw, BlockSync());
    else fft<R, N, SIGN>(v, sm, ColAddr<CC::COLS, (int)sizeof(cplx<R>), col_swz_shift<N>()>(), t, tw);
}

template <class R>
__device__ __forceinline__ void load_table(cplx<R> *tw, const cplx<R> *__restrict__ twg, int count, int tid, int nthreads) {
    for (int i = tid; i < count; i += nthreads) tw[i] = twg[i];
}
// the twiddle table a pass reads: count entries staged in shared memory at tws, or, when the Cfg's TWG is
// set, the global table itself (read through L1 / L2)
template <bool TWG, class R>
__device__ __forceinline__ const cplx<R> *twiddles_for(cplx<R> *tws, const cplx<R> *__restrict__ twg, int count,
                                                       int tid, int nthreads) {
    if constexpr (TWG) {
        (void)tws; (void)count; (void)tid; (void)nthreads;
        return twg;
    } else {
        load_table<R>(tws, twg, count, tid, nthreads);
        return tws;
    }
}

// L2 prefetch of [p, p + bytes) by the copy engine (cp.async.bulk.prefetch; a hint, no data returned):
// the part aligned to 16 bytes at both ends
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
    const uintptr_t a = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes) & ~uintptr_t(15);
    if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}
// Row passes with pf > 0: the block with linear index L asks the copy engine to bring the rows that block
// L + pf reads (its wave rows' active columns) into L2, so that a block launched a residency later finds
// them there rather than in HBM. rows: the rows this thread prefetches for (first row y0, count n).
template <class C>
__device__ __forceinline__ void prefetch_rows(const C *wave, int N, int rows_per_block, int pf, int xa, int xb,
                                             int load_all) {
    const long long L = (long long)blockIdx.x + (long long)blockIdx.y * gridDim.x + pf;
    if (L >= (long long)gridDim.x * gridDim.y) return;
    const int bx = (int)(L % gridDim.x), by = (int)(L / gridDim.x);
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    if (tid >= rows_per_block) return;
    const C *r = wave + (size_t)by * N * N + ((size_t)bx * rows_per_block + tid) * N;
    if (load_all) {
        prefetch_l2(r, (size_t)N * sizeof(C));
    } else {
        if (xa > 0) prefetch_l2(r, (size_t)xa * sizeof(C));
        if (xb < N) prefetch_l2(r + xb, (size_t)(N - xb) * sizeof(C));
    }
}

// ------------------------------------------------------------------------------------------------
// Row kernels: grid (res/ROWS, batch), block (NT, ROWS); with pf == kWaveFastRows the grid is (batch,
// res/ROWS) instead, so the blocks the scheduler issues together hold the same rows of consecutive waves and
// read the same transmission rows (from L2 after the first), where the usual order reads a whole wave's
// worth of wave rows between two reads of a transmission row (at 2048² a slice of T is 32 MB).
// ------------------------------------------------------------------------------------------------
constexpr int kWaveFastRows = -1;
// The multislice row pass: phi <- D_r(T * a * Dinv_r phi).
// Band limit: the column pass multiplies by P, which is zero in every column with kx^2 >= k_cut^2, so
// between passes only the columns x < xa or x >= xb (whole column tiles) carry data. The row pass reads
// those (or every column when load_all is set: the first slice after probe initialisation) and writes
// only those, since the column pass reads nothing else.
// FP64 step kernels: the radix-8 plans at 256 threads are compiled for 3 blocks per SM (80 registers), the
// 3·2^k plans for a 128-register budget (the compiler otherwise takes 186-234). Measured against the
// compiler's choice, in a 256-probe STEM run, with bit-identical results: row pass 256² −11%, 384² −4%,
// 512² −20%, 768² −4%, 1536² −12%, 2048² −4%, 3072² −19%; column pass 384² −7%, 768² −9%, 1024² −5%,
// 1536² −6%, 2048² −26%, 3072² −14%.
template <class R, int N, int THREADS, int OTHER> constexpr int fp64_step_minb() {
    return (sizeof(R) == 8 && THREADS == 256 && Plan<N>::E == 8) ? 3
         : (sizeof(R) == 8 && Plan<N>::E == 12 && THREADS * 128 < 65536) ? 65536 / (THREADS * 128) : OTHER;
}
// Row step with staged transmission rows (TST): the block's transmission rows are contiguous in HBM, and one
// thread asks the copy engine for the first row_ts_rows of them (cp.async.bulk into shared memory, completion
// on an mbarrier) as the block starts, so they arrive while the inverse row FFT runs. Without TST (and in a
// block's rows beyond those) every thread loads its T elements only after that FFT and waits for them there.
// The staged rows sit after the block's twiddles and exchange rows (16-byte aligned), the mbarrier after them.
template <int N, class R> constexpr size_t row_tstage_off() { return (RowCfg<N, R>::smem() + 15) / 16 * 16; }
// Rows of a block that are staged (the first TSR; the rest load T themselves): with 4 or more rows a block,
// as many as leave the plain kernel's blocks per SM (128 registers a thread, its shared memory); with fewer,
// all of them. Measured per probe·slice, row pass: 1024² with 4 of 8 rows staged (2 blocks an SM) 4.13 →
// 3.94 µs, where all 8 (1 block an SM) were slower than none; 384², 768² all rows fit at the plain kernel's
// 4 blocks; 1536², 3072², 8192² (1-2 rows a block) staging all rows wins although it costs blocks.
template <int N, class R> constexpr int row_ts_blocks(int r) {
    return (int)((228 * 1024) / (row_tstage_off<N, R>() + sizeof(cplx<R>) * (size_t)r * N + 8 + 1024));
}
template <int N, class R> constexpr int row_ts_rows() {
    constexpr int ROWS = RowCfg<N, R>::ROWS;
    constexpr int by_regs = 65536 / (RowCfg<N, R>::THREADS * 128);
    constexpr int by_smem = (int)((228 * 1024) / (RowCfg<N, R>::smem() + 1024));
    constexpr int plain = by_regs < by_smem ? by_regs : by_smem;
    if (ROWS < 4) return ROWS;
    for (int r = ROWS; r >= 1; r--)
        if (row_ts_blocks<N, R>(r) >= plain) return r;
    return ROWS;
}
template <int N, class R> constexpr size_t row_ts_smem() {
    return row_tstage_off<N, R>() + sizeof(cplx<R>) * (size_t)row_ts_rows<N, R>() * N + 8;
}
// the row step's body, shared by k_row_step and its FP64 3-blocks-per-SM build k_row_step_d; err (TST only):
// the error word a wait that is abandoned writes (tma.cuh StepError)
template <class R, int N, bool TST = false>
__device__ __forceinline__ void row_step_body(cplx<R> *__restrict__ wave, const cplx<R> *__restrict__ trans,
                                              const cplx<R> *__restrict__ twg, R a, int xa, int xb, int load_all,
                                              const int *__restrict__ tsel, size_t tstride, int pf, int *err = nullptr) {
    using RC = RowCfg<N, R>;
    using P = typename RC::P;
    constexpr int ROWS = RC::ROWS;
    if (pf > 0) prefetch_rows(wave, N, ROWS, pf, xa, xb, load_all);
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tws = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *sm = tws + RC::TWS + threadIdx.y * RC::ROWSZ;
    const int t = threadIdx.x;
    const cplx<R> *tw =
        twiddles_for<RC::TWG, R>(tws, twg + RC::TW_OFF, RC::TWN, t + threadIdx.y * P::NT, P::NT * ROWS);
    const int rblk = pf == kWaveFastRows ? blockIdx.y : blockIdx.x, w = pf == kWaveFastRows ? blockIdx.x : blockIdx.y;
    const int y = rblk * ROWS + threadIdx.y;
    cplx<R> *row = wave + (size_t)w * N * N + (size_t)y * N;
    // tsel (optional): transmission set of each wave; set k of this slice starts k * tstride after trans
    const cplx<R> *trow = trans + (tsel ? (size_t)tsel[w] * tstride : (size_t)0) + (size_t)y * N;
    cplx<R> *sT = reinterpret_cast<cplx<R> *>(smraw + row_tstage_off<N, R>());
    constexpr int TSR = row_ts_rows<N, R>();
    uint64_t *tbar = reinterpret_cast<uint64_t *>(smraw + row_tstage_off<N, R>() + sizeof(cplx<R>) * TSR * N);
    if constexpr (TST) {
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            mbar_init(tbar, 1);
            mbar_fence_init();
            constexpr unsigned bytes = (unsigned)(sizeof(cplx<R>) * TSR * N);
            mbar_arrive_expect_tx(tbar, bytes);
            bulk_load(sT, trow, bytes, tbar);   // thread (0, 0)'s row is the block's first
        }
    }
    cplx<R> v[P::E];
#pragma unroll
    for (int m = 0; m < P::E; m++) {
        const int x = t + m * P::NT;
        v[m] = (load_all || x < xa || x >= xb) ? row[x] : mk<R>(0, 0);
    }
    __syncthreads();
    row_transform<R, N, +1>(v, sm, t, tw);
    const bool staged = TST && (int)threadIdx.y < TSR;
    if constexpr (TST) {   // (an abandoned wait still lets the copy land before the block goes on)
        if (staged && !mbar_wait(tbar, 0, err, STEP_WAIT_FULL)) mbar_wait(tbar, 0, err, STEP_WAIT_DRAIN);
    }
    const cplx<R> *tr = staged ? sT + threadIdx.y * N : trow;
#pragma unroll
    for (int m = 0; m < P::E; m++) v[m] = cscale(cmul(v[m], tr[t + m * P::NT]), a);
    row_transform<R, N, -1>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) {
        const int x = t + m * P::NT;
        if (x < xa || x >= xb) row[x] = v[m];
    }
}

// No minimum-blocks hint: an explicit 1 lets the FP32 wide row pass take 170 registers instead of 128 (37%
// slower at 512²).
template <class R, int N>
__global__ void __launch_bounds__(RowCfg<N, R>::THREADS)
k_row_step(cplx<R> *__restrict__ wave, const cplx<R> *__restrict__ trans, const cplx<R> *__restrict__ twg, R a,
           int xa, int xb, int load_all, const int *__restrict__ tsel, size_t tstride, int pf) {
    row_step_body<R, N>(wave, trans, twg, a, xa, xb, load_all, tsel, tstride, pf);
}
template <int N> constexpr bool fp64_row_bounded() {
    return fp64_step_minb<double, N, RowCfg<N, double>::THREADS, 1>() > 1;
}
template <int N>
__global__ void __launch_bounds__(RowCfg<N, double>::THREADS, fp64_step_minb<double, N, RowCfg<N, double>::THREADS, 1>())
k_row_step_d(double2 *__restrict__ wave, const double2 *__restrict__ trans, const double2 *__restrict__ twg, double a,
             int xa, int xb, int load_all, const int *__restrict__ tsel, size_t tstride, int pf) {
    row_step_body<double, N>(wave, trans, twg, a, xa, xb, load_all, tsel, tstride, pf);
}
// The FP32 row step with the three-stage wide plan (2048, 4096, 8192), compiled for the blocks per SM its
// shared memory allows (4 x 128 threads at 2048, 3 x 128 at 4096, 1 x 256 at 8192): without the hint the
// compiler takes 175-185 registers a thread at 2048 and 4096, which leaves 2 blocks (8 warps) per SM.
// blocks per SM the FP32 row step of the three-stage wide plans and the radix-24 plans is compiled for (the
// radix-24 rows take 168 registers without a bound: 4 blocks of 128 threads give them 128)
template <int N> constexpr int wide3_minb() { return wide24_plan<float>(N) ? 4 : (N == 2048 ? 4 : (N == 4096 ? 3 : 1)); }
template <int N>
__global__ void __launch_bounds__(RowCfg<N, float>::THREADS, wide3_minb<N>())
k_row_step_w3(float2 *__restrict__ wave, const float2 *__restrict__ trans, const float2 *__restrict__ twg, float a,
              int xa, int xb, int load_all, const int *__restrict__ tsel, size_t tstride, int pf) {
    row_step_body<float, N>(wave, trans, twg, a, xa, xb, load_all, tsel, tstride, pf);
}

// The FP32 row step with staged transmission rows (TST above), for the wide, three-stage wide and radix-24 row
// plans where the extra shared memory fits. Blocks per SM: what the shared memory allows, at most the
// 128-register occupancy of the plain kernels.
template <int N> constexpr bool row_ts_ok() {
    return (RowCfg<N, float>::WIDE || RowCfg<N, float>::WIDE3 || RowCfg<N, float>::WIDE24) &&
           row_ts_smem<N, float>() <= kMaxBlockSmem;
}
template <int N> constexpr int row_ts_minb() {
    constexpr int by_smem = (int)((228 * 1024) / (row_ts_smem<N, float>() + 1024));
    constexpr int by_regs = 65536 / (RowCfg<N, float>::THREADS * 128);
    constexpr int m = by_smem < by_regs ? by_smem : by_regs;
    return m < 1 ? 1 : m;
}
template <int N>
__global__ void __launch_bounds__(RowCfg<N, float>::THREADS, row_ts_minb<N>())
k_row_step_ts(float2 *__restrict__ wave, const float2 *__restrict__ trans, const float2 *__restrict__ twg, float a,
              int xa, int xb, int load_all, const int *__restrict__ tsel, size_t tstride, int pf, int *err) {
    row_step_body<float, N, true>(wave, trans, twg, a, xa, xb, load_all, tsel, tstride, pf, err);
}

// The row step of the FP32 radix-8 / 3·2^k row plans (sizes without the wide plan) with each thread carrying
// the same element of two adjacent rows of a wave: the shared-memory exchanges move 16-byte pairs and each
// twiddle serves both rows (fft_pair.cuh; ColAddr<1, 16> keeps the stage writes conflict-free). Same
// arithmetic per element as k_row_step<float, N>. Measured against the one-row kernel in a 256-probe STEM
// run: 384² −10%, 768² −11%, 1536² −14%, 2048² −9%, 3072² −17%, 4096² −33%, with bit-identical results.
template <int N> constexpr int rowpair_base() { return RowCfg<N, float>::ROWS >= 2 ? RowCfg<N, float>::ROWS / 2 : 1; }
template <int N, int PAIRS_ = rowpair_base<N>()> struct RowPairCfg {
    using P = Plan<N>;
    static constexpr int PAIRS = PAIRS_;   // row pairs a block
    static constexpr int THREADS = P::NT * PAIRS;
    static constexpr size_t smem() { return sizeof(float2) * (size_t)N + sizeof(float4) * (size_t)N * PAIRS; }
    static constexpr bool ok = !RowCfg<N, float>::WIDE && !RowCfg<N, float>::WIDE3 && !RowCfg<N, float>::WIDE24 &&
                               THREADS <= 1024 &&
                               N % (2 * PAIRS) == 0 && smem() <= kMaxBlockSmem;
};
// Row pairs a block of the step: twice the base at 384² and 768² (measured in a STEM run per size, row-pass
// device time per probe·slice: −2.3% and −3.3%; 1536² to 4096² were 10-39% slower with 2 or 4 times the
// base, 8192² has no room)
template <int N> constexpr int rowpair_pairs() { return (N == 384 || N == 768 ? 2 : 1) * rowpair_base<N>(); }
template <int N> using RowPairStepCfg = RowPairCfg<N, rowpair_pairs<N>()>;
template <int N> constexpr bool pair_rows() { return RowPairStepCfg<N>::ok; }
// The two-row step on the sizes whose default row plan is a wide or radix-24 one: the plain Stockham plan of
// fft.cuh (radix-8 at 2^k, radix-4 then radix-12 at 3·2^k) as the autotuner's alternative FFT plan for the row
// pass (row variants 4 to 7). A different plan rounds differently: its results agree with the default plan's
// to FP32 rounding, not bit for bit. 128 threads a block (256 where a row takes more).
template <int N> constexpr int altrow_pairs() { return Plan<N>::NT >= 128 ? 1 : 128 / Plan<N>::NT; }
template <int N> constexpr bool alt_pair_rows() {
    return !RowPairStepCfg<N>::ok && (RowCfg<N, float>::WIDE || RowCfg<N, float>::WIDE3 || RowCfg<N, float>::WIDE24) &&
           RowPairCfg<N, altrow_pairs<N>()>::THREADS <= 1024 && N % (2 * altrow_pairs<N>()) == 0 &&
           RowPairCfg<N, altrow_pairs<N>()>::smem() <= kMaxBlockSmem;
}
// blocks per SM the two-row step is compiled for: a 128-register budget (measured against no cap: 2048² and
// 4096² the same, 384² to 3072² 6-21% faster at the cap)
template <int N, int PAIRS = rowpair_base<N>()> constexpr int rowpair_minb() {
    return RowPairCfg<N, PAIRS>::THREADS * 128 >= 65536 ? 1 : 65536 / (RowPairCfg<N, PAIRS>::THREADS * 128);
}

// grid (N / (2 PAIRS), batch), block (NT, PAIRS)
template <int N, int PAIRS_>
__global__ void __launch_bounds__(RowPairCfg<N, PAIRS_>::THREADS, rowpair_minb<N, PAIRS_>())
k_row_step_pair(float2 *__restrict__ wave, const float2 *__restrict__ trans, const float2 *__restrict__ twg, float a,
                int xa, int xb, int load_all, const int *__restrict__ tsel, size_t tstride, int pf) {
    using PC = RowPairCfg<N, PAIRS_>;
    using P = typename PC::P;
    constexpr int E = P::E, NT = P::NT;
    if (pf > 0) prefetch_rows(wave, N, 2 * PC::PAIRS, pf, xa, xb, load_all);
    extern __shared__ __align__(16) unsigned char smraw[];
    float2 *tw = reinterpret_cast<float2 *>(smraw);
    float4 *sm = reinterpret_cast<float4 *>(tw + N) + (size_t)threadIdx.y * N;
    const int t = threadIdx.x;
    load_table<float>(tw, twg, N, t + threadIdx.y * NT, NT * PC::PAIRS);
    const int rblk = pf == kWaveFastRows ? blockIdx.y : blockIdx.x, w = pf == kWaveFastRows ? blockIdx.x : blockIdx.y;
    const int y = (rblk * PC::PAIRS + threadIdx.y) * 2;
    float2 *ra = wave + (size_t)w * N * N + (size_t)y * N, *rb = ra + N;
    const float2 *ta = trans + (tsel ? (size_t)tsel[w] * tstride : (size_t)0) + (size_t)y * N, *tb = ta + N;
    float2 va[E], vb[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
        const int x = t + m * NT;
        const bool in = load_all || x < xa || x >= xb;
        va[m] = in ? ra[x] : mk<float>(0, 0);
        vb[m] = in ? rb[x] : mk<float>(0, 0);
    }
    __syncthreads();
    fft_pair<N, +1>(va, vb, sm, ColAddr<1, 16, col_swz_shift<N>()>(), t, tw);
#pragma unroll
    for (int m = 0; m < E; m++) {
        va[m] = cscale(cmul(va[m], ta[t + m * NT]), a);
        vb[m] = cscale(cmul(vb[m], tb[t + m * NT]), a);
    }
    fft_pair<N, -1>(va, vb, sm, ColAddr<1, 16, col_swz_shift<N>()>(), t, tw);
#pragma unroll
    for (int m = 0; m < E; m++) {
        const int x = t + m * NT;
        if (x < xa || x >= xb) { ra[x] = va[m]; rb[x] = vb[m]; }
    }
}

// A plain row transform (SIGN -1 forward, +1 inverse), scaled, in or out of place.
template <class R, int N, int SIGN>
__global__ void __launch_bounds__(RowCfg<N, R>::THREADS)
k_row_fft(const cplx<R> *in, cplx<R> *out, const cplx<R> *__restrict__ twg, R scale) {
    using RC = RowCfg<N, R>;
    using P = typename RC::P;
    constexpr int ROWS = RC::ROWS;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tws = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *sm = tws + RC::TWS + threadIdx.y * RC::ROWSZ;
    const int t = threadIdx.x;
    const cplx<R> *tw =
        twiddles_for<RC::TWG, R>(tws, twg + RC::TW_OFF, RC::TWN, t + threadIdx.y * P::NT, P::NT * ROWS);
    const int y = blockIdx.x * ROWS + threadIdx.y;
    const size_t off = (size_t)blockIdx.y * N * N + (size_t)y * N;
    cplx<R> v[P::E];
#pragma unroll
    for (int m = 0; m < P::E; m++) v[m] = in[off + t + m * P::NT];
    __syncthreads();
    row_transform<R, N, SIGN>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) out[off + t + m * P::NT] = cscale(v[m], scale);
}

// ------------------------------------------------------------------------------------------------
// Column kernels: grid (res/COLS, batch), block (COLS, NT)
// ------------------------------------------------------------------------------------------------
template <class R, int N>
__device__ __forceinline__ void col_load(cplx<R> (&v)[ColCfg<N, R>::P::E], const cplx<R> *base, int x, int t) {
    using P = typename ColCfg<N, R>::P;
#pragma unroll
    for (int m = 0; m < P::E; m++) v[m] = base[(size_t)(t + m * P::NT) * N + x];
}
template <class R, int N>
__device__ __forceinline__ void col_store(const cplx<R> (&v)[ColCfg<N, R>::P::E], cplx<R> *base, int x, int t) {
    using P = typename ColCfg<N, R>::P;
#pragma unroll
    for (int m = 0; m < P::E; m++) base[(size_t)(t + m * P::NT) * N + x] = v[m];
}

// Block-wide sum of one double per thread; the result is valid in thread 0. red: >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *red) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int nw = (blockDim.x * blockDim.y + 31) / 32;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    double s = 0;
    if (tid == 0)
        for (int w = 0; w < nw; w++) s += red[w];
    return s;
}

enum ColMode { COL_STEP = 0, COL_STEP_DET = 1, COL_DET_ONLY = 2 };

// The multislice column pass: D_c, * P (strict cut), [detectors / Recip copy], * b, Dinv_c.
// Block b works on column tile b for b < tiles_lo, else on tile N/COLS - (gridDim.x - b): the grid covers
// the leading and trailing tiles that hold columns inside the propagator's cut (all tiles when
// tiles_lo = N/COLS); the others would only be multiplied by zero.
template <class R, int N, int MODE>
__global__ void __launch_bounds__(ColCfg<N, R>::THREADS,
                                  fp64_step_minb<R, N, ColCfg<N, R>::THREADS, ColCfg<N, R>::STEP_MINB>())
k_col_step(cplx<R> *__restrict__ wave, const cplx<R> *__restrict__ twg, PropTables<R> pt, R bscale, R det_scale,
           DetArgs det, cplx<R> *__restrict__ recip_out, int tiles_lo) {
    using CC = ColCfg<N, R>;
    using P = typename CC::P;
    constexpr int COLS = CC::COLS;
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ double red[32];
    cplx<R> *tws = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *sm = tws + CC::TWS + threadIdx.x;
    const int c = threadIdx.x, t = threadIdx.y;
    const cplx<R> *tw = twiddles_for<CC::TWG, R>(tws, twg, CC::TWN, c + t * COLS, COLS * P::NT);
    const int tile = (int)blockIdx.x < tiles_lo ? (int)blockIdx.x : N / COLS - ((int)gridDim.x - (int)blockIdx.x);
    const int x = tile * COLS + c;
    cplx<R> *base = wave + (size_t)blockIdx.y * N * N;
    cplx<R> v[P::E];
    col_load<R, N>(v, base, x, t);
    __syncthreads();
    col_transform<R, N, -1>(v, sm, t, tw);
    const cplx<R> pxx = pt.px[x];
    const cplx<R> exx = sizeof(R) == 4 ? pt.pxe[x] : mk<R>(0, 0);
    const double kx2 = pt.kx2[x];
#pragma unroll
    for (int m = 0; m < P::E; m++) {
        const int y = t + m * P::NT;
        v[m] = (kx2 + pt.ky2[y] < pt.kmax2)
                   ? prop_mul<R>(v[m], pxx, pt.py[y], exx, sizeof(R) == 4 ? pt.pye[y] : mk<R>(0, 0))
                   : mk<R>(0, 0);
    }
    if constexpr (MODE == COL_STEP_DET || MODE == COL_DET_ONLY) {
        if (det.n_det > 0) {
            double e[P::E];
            uint16_t mk_[P::E];
#pragma unroll
            for (int m = 0; m < P::E; m++) {
                const int y = t + m * P::NT;
                double re = (double)v[m].x * (double)det_scale, im = (double)v[m].y * (double)det_scale;
                e[m] = re * re + im * im;
                mk_[m] = det.mask[(size_t)y * N + x];
            }
            for (int d = 0; d < det.n_det; d++) {
                double acc = 0;
#pragma unroll
                for (int m = 0; m < P::E; m++) acc += ((mk_[m] >> d) & 1) ? e[m] : 0.0;
                double s = block_sum(acc, red);
                if (c == 0 && t == 0) det.partials[((size_t)blockIdx.y * det.n_det + d) * gridDim.x + blockIdx.x] = s;
            }
        }
        if (recip_out) {
            cplx<R> *rb = recip_out + (size_t)blockIdx.y * N * N;
#pragma unroll
            for (int m = 0; m < P::E; m++) rb[(size_t)(t + m * P::NT) * N + x] = cscale(v[m], det_scale);
        }
    }
    if constexpr (MODE != COL_DET_ONLY) {
#pragma unroll
        for (int m = 0; m < P::E; m++) v[m] = cscale(v[m], bscale);
        col_transform<R, N, +1>(v, sm, t, tw);
        col_store<R, N>(v, base, x, t);
    }
}

// The plain step (COL_STEP) of the FP32 column plans (2^k and 3·2^k) with each thread carrying two adjacent
// columns of the tile: 16-byte loads, stores and shared-memory exchanges (fft_pair.cuh), and the
// propagator's cut read as a row band per column (PropTables::ycut) instead of an FP64 test per element.
// Same arithmetic per element as k_col_step<float, N, COL_STEP>. At the engine's column tile it measured,
// against the one-column kernel in a 256-probe STEM run: 256² −12%, 384² −11%, 512² −5%, 768² −32%,
// 1024² −5%, 1536² −25%, 2048² ±0, 3072² −13%, 4096² −18%, with bit-identical results. Its tile is now wider
// than the engine's (PairStepCfg below).
template <int N, int COLS_, bool LOOSE = false> struct PairCfg {
    using P = Plan<N>;
    static constexpr int COLS = COLS_;
    static constexpr int PAIRS = COLS / 2;
    static constexpr int THREADS = PAIRS * P::NT;
    // 64 registers a thread, or (LOOSE) 128
    static constexpr int MINB = LOOSE ? (THREADS * 128 >= 65536 ? 1 : 65536 / (THREADS * 128))
                                      : (THREADS <= 256 ? 4 : (THREADS <= 512 ? 2 : 1));
    static constexpr size_t smem() { return sizeof(float2) * (size_t)N + sizeof(float4) * (size_t)N * PAIRS; }
    static constexpr bool ok = !ColCfg<N, float>::WIDE && COLS >= 2 && N % COLS == 0 && THREADS <= 1024 &&
                               smem() <= kMaxBlockSmem;
};
// The step's tile: k times the engine's column tile (ColCfg::COLS), 64 or (LOOSE) 128 registers a thread.
// Measured in a STEM run at each size (batch of ~1 GiB of waves, column-pass device time per probe·slice),
// against the engine's tile at 64 registers:
//   256² 2x loose −7%, 384² 2x loose −9%, 512² 2x −2.5%, 768² 4x −19%, 1024² 2x −8%, 1536² 4x −25%,
//   2048² 4x −22%, 3072² 4x −22%, 4096² 2x −17%, 8192² 2x (two columns where the engine's tile has one) −33%.
// Wider tiles put whole 32-byte sectors (and more of each 128-byte line) behind every row a block loads.
template <int N> constexpr int pair_mult() {
    return (N == 768 || N == 1536 || N == 2048 || N == 3072) ? 4 : (N >= 256 ? 2 : 1);
}
template <int N> constexpr bool pair_loose() { return N == 256 || N == 384; }
template <int N> using PairStepCfg = PairCfg<N, pair_mult<N>() * ColCfg<N, float>::COLS, pair_loose<N>()>;
template <int N> constexpr bool pair_columns() { return PairStepCfg<N>::ok; }

// The propagator and scale b on the two columns x, x + 1 a thread holds (elements t + m NT), zero outside the
// cut (the row band of PropTables::ycut): shared by the two-column step kernels. b is folded into the column
// factors once (b px), which saves a scaling of every element; b = 1/N is a power of two on the 2^k grids,
// so there the products equal those of scaling afterwards bit for bit (the correction (1 + ex + ey) is relative).
__device__ __forceinline__ float2 prop_col(const PropTables<float> &pt, int x, float bscale) { return cscale(pt.px[x], bscale); }
template <int N>
__device__ __forceinline__ void prop_pair(float2 (&va)[Plan<N>::E], float2 (&vb)[Plan<N>::E], const PropTables<float> &pt,
                                          int x, int t, float bscale) {
    constexpr int E = Plan<N>::E, NT = Plan<N>::NT;
    const float2 pxa = prop_col(pt, x, bscale), pxb = prop_col(pt, x + 1, bscale), exa = pt.pxe[x], exb = pt.pxe[x + 1];
    const int2 ca = pt.ycut[x], cb = pt.ycut[x + 1];
#pragma unroll
    for (int m = 0; m < E; m++) {
        const int y = t + m * NT;
        const float2 py = pt.py[y], ey = pt.pye[y];
        va[m] = (y < ca.x || y >= ca.y) ? prop_mul<float>(va[m], pxa, py, exa, ey) : mk<float>(0, 0);
        vb[m] = (y < cb.x || y >= cb.y) ? prop_mul<float>(vb[m], pxb, py, exb, ey) : mk<float>(0, 0);
    }
}

template <int N, int COLS, bool LOOSE>
__global__ void __launch_bounds__(PairCfg<N, COLS, LOOSE>::THREADS, PairCfg<N, COLS, LOOSE>::MINB)
k_col_step_pair(float2 *__restrict__ wave, const float2 *__restrict__ twg, PropTables<float> pt, float bscale,
                int tiles_lo) {
    using PC = PairCfg<N, COLS, LOOSE>;
    using P = typename PC::P;
    constexpr int PAIRS = PC::PAIRS, E = P::E, NT = P::NT;
    extern __shared__ __align__(16) unsigned char smraw[];
    float2 *tw = reinterpret_cast<float2 *>(smraw);
    float4 *sm = reinterpret_cast<float4 *>(tw + N) + threadIdx.x;
    const int p = threadIdx.x, t = threadIdx.y;
    load_table<float>(tw, twg, N, p + t * PAIRS, PAIRS * NT);
    const int tile = (int)blockIdx.x < tiles_lo ? (int)blockIdx.x : N / PC::COLS - ((int)gridDim.x - (int)blockIdx.x);
    const int x = tile * PC::COLS + 2 * p;
    float4 *base = reinterpret_cast<float4 *>(wave + (size_t)blockIdx.y * N * N + x);
    float2 va[E], vb[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
        const float4 q = base[(size_t)(t + m * NT) * (N / 2)];
        va[m] = make_float2(q.x, q.y);
        vb[m] = make_float2(q.z, q.w);
    }
    __syncthreads();
    fft_pair<N, -1>(va, vb, sm, ColAddr<PAIRS, 16, col_swz_shift<N>()>(), t, tw);
    prop_pair<N>(va, vb, pt, x, t, bscale);
    fft_pair<N, +1>(va, vb, sm, ColAddr<PAIRS, 16, col_swz_shift<N>()>(), t, tw);
#pragma unroll
    for (int m = 0; m < E; m++)
        base[(size_t)(t + m * NT) * (N / 2)] = make_float4(va[m].x, va[m].y, vb[m].x, vb[m].y);
}

// A plain column transform, scaled, in or out of place.
template <class R, int N, int SIGN>
__global__ void __launch_bounds__(ColCfg<N, R>::THREADS)
k_col_fft(const cplx<R> *in, cplx<R> *out, const cplx<R> *__restrict__ twg, R scale) {
    using CC = ColCfg<N, R>;
    using P = typename CC::P;
    constexpr int COLS = CC::COLS;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tws = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *sm = tws + CC::TWS + threadIdx.x;
    const int c = threadIdx.x, t = threadIdx.y;
    const cplx<R> *tw = twiddles_for<CC::TWG, R>(tws, twg, CC::TWN, c + t * COLS, COLS * P::NT);
    const int x = blockIdx.x * COLS + c;
    const size_t off = (size_t)blockIdx.y * N * N;
    cplx<R> v[P::E];
    col_load<R, N>(v, in + off, x, t);
    __syncthreads();
    col_transform<R, N, SIGN>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) v[m] = cscale(v[m], scale);
    col_store<R, N>(v, out + off, x, t);
}

// Transmission band limit (simulationgeneral.cpp:596-602, band_limit_d.cl:13-32) on row-transformed
// slices: D_c, keep sqrt(kx^2+ky^2) <= lim (inclusive) times scale, Dinv_c.
template <class R, int N>
__global__ void __launch_bounds__(ColCfg<N, R>::THREADS)
k_col_bandlimit(cplx<R> *__restrict__ wave, const cplx<R> *__restrict__ twg, const double *__restrict__ kx2,
                const double *__restrict__ ky2, double lim, R scale) {
    using CC = ColCfg<N, R>;
    using P = typename CC::P;
    constexpr int COLS = CC::COLS;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tws = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *sm = tws + CC::TWS + threadIdx.x;
    const int c = threadIdx.x, t = threadIdx.y;
    const cplx<R> *tw = twiddles_for<CC::TWG, R>(tws, twg, CC::TWN, c + t * COLS, COLS * P::NT);
    const int x = blockIdx.x * COLS + c;
    cplx<R> *base = wave + (size_t)blockIdx.y * N * N;
    cplx<R> v[P::E];
    col_load<R, N>(v, base, x, t);
    __syncthreads();
    col_transform<R, N, -1>(v, sm, t, tw);
    const double k2x = kx2[x];
#pragma unroll
    for (int m = 0; m < P::E; m++) {
        double k = sqrt(k2x + ky2[t + m * P::NT]);
        v[m] = cscale(v[m], (k <= lim) ? scale : (R)0);
    }
    col_transform<R, N, +1>(v, sm, t, tw);
    col_store<R, N>(v, base, x, t);
}

// Probe initialisation (init_probe_wave_d.cl:49-118 then the column half of the IFFT,
// simulationcbed.cpp:91-99): generate the reciprocal-space probe of each wave of the batch, Dinv_c,
// scale. chi[y*N+x] = (chi(k), inside-aperture flag) in FP64; pos[b] = probe position relative to the
// simulation start (Å). The phase -2 pi (kx px + ky py) - chi is formed in FP64.
template <class R, int N>
__global__ void __launch_bounds__(ColCfg<N, R>::THREADS)
k_col_probe(cplx<R> *__restrict__ wave, const cplx<R> *__restrict__ twg, const double2 *__restrict__ chi,
            const double *__restrict__ kx, const double *__restrict__ ky, const double2 *__restrict__ pos, R scale,
            const double *__restrict__ dfac, double wl) {
    using CC = ColCfg<N, R>;
    using P = typename CC::P;
    constexpr int COLS = CC::COLS;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<R> *tws = reinterpret_cast<cplx<R> *>(smraw);
    cplx<R> *sm = tws + CC::TWS + threadIdx.x;
    const int c = threadIdx.x, t = threadIdx.y;
    const cplx<R> *tw = twiddles_for<CC::TWG, R>(tws, twg, CC::TWN, c + t * COLS, COLS * P::NT);
    const int x = blockIdx.x * COLS + c;
    const double2 pp = pos[blockIdx.y];
    // dfac (optional): pi * defocus change / wavelength of each wave; the aberration phase gains
    // 2 pi / lambda * dC10 |w|^2 / 2 = dfac * |w|^2 with w = lambda k (the C10 term of init_probe_wave_d.cl:83-101)
    const double df = dfac ? dfac[blockIdx.y] : 0.0;
    const double kxx = kx[x];
    cplx<R> v[P::E];
#pragma unroll
    for (int m = 0; m < P::E; m++) {
        const int y = t + m * P::NT;
        const double2 ch = chi[(size_t)y * N + x];
        if (ch.y != 0.0) {
            double posTerm = 2.0 * M_PI * (kxx * pp.x + ky[y] * pp.y);
            double arg = -posTerm - ch.x;
            if (dfac) {
                const double wx = wl * kxx, wy = wl * ky[y];
                arg -= df * (wx * wx + wy * wy);
            }
            if constexpr (sizeof(R) == 8) {
                v[m] = mk<R>((R)cos(arg), (R)sin(arg));
            } else {
                double red = arg - 6.283185307179586232 * rint(arg * 0.15915494309189534561);
                float s, co;
                sincosf((float)red, &s, &co);
                v[m] = mk<R>((R)co, (R)s);
            }
        } else {
            v[m] = mk<R>(0, 0);
        }
    }
    __syncthreads();
    col_transform<R, N, +1>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) v[m] = cscale(v[m], scale);
    col_store<R, N>(v, wave + (size_t)blockIdx.y * N * N, x, t);
}

}  // namespace ms
