// inst.cu — instantiates the pass kernels for one precision and one size.
// Compiled once per (MS_REAL, MS_N) pair by the build (e.g. -DMS_REAL=float -DMS_N=512).
#include "launch.cuh"

#include <type_traits>

#ifndef MS_REAL
#error "MS_REAL must be defined"
#endif
#ifndef MS_N
#error "MS_N must be defined"
#endif

namespace ms {

namespace {
using R = MS_REAL;
constexpr int N = MS_N;
using RC = RowCfg<N, R>;
using CC = ColCfg<N, R>;

template <class K> void set_smem(K kernel, size_t bytes) {
    MS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    // prefer the largest shared-memory carveout so several blocks fit per SM
    MS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
}

// the two-column step kernel of the FP32 plans (templates, so that the FP64 build discards them) with a tile of
// C columns: C = PairStepCfg::COLS (the measured default), half or twice that where the tile is valid; L the
// register budget (false: 64 registers a thread, true: 128; pair_loose is the measured default)
template <class RR, int C, bool L = pair_loose<N>()> constexpr bool pair_tile_ok() {
    if constexpr (std::is_same<RR, float>::value && pair_columns<N>() && C >= 2 && C <= N) {
        return PairCfg<N, C, L>::ok && C % CC::COLS == 0 && N % C == 0;
    } else {
        return false;
    }
}
template <class RR, int C, bool L = pair_loose<N>()> void pair_attrs() {
    if constexpr (pair_tile_ok<RR, C, L>()) {
        using PC = PairCfg<N, C, L>;
        set_smem(k_col_step_pair<N, C, L>, PC::smem());
    }
}
template <class RR, int C, bool L = pair_loose<N>()>
bool pair_step(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *tw, PropTables<RR> pt, RR b, int tiles_lo,
               int tiles_hi) {
    if constexpr (pair_tile_ok<RR, C, L>()) {
        using PC = PairCfg<N, C, L>;
        // the engine's tiles are CC::COLS wide and the step's tile covers k of them; the extra columns of a
        // partly active tile lie outside the propagator's cut and come out zero, and the row pass never
        // reads them
        constexpr int k = C / CC::COLS, total = N / C;
        static_assert(C % CC::COLS == 0, "the step's tile must cover whole engine tiles");
        int lo = (tiles_lo + k - 1) / k, hi = (tiles_hi + k - 1) / k;
        if (lo + hi > total) { lo = total; hi = 0; }
        k_col_step_pair<N, C, L><<<dim3(lo + hi, batch), dim3(PC::PAIRS, Plan<N>::NT), PC::smem(), s>>>(wave, tw, pt, b,
                                                                                                        lo);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}
// C of the default two-column step (a valid value for the FP64 build too, where nothing uses it)
constexpr int kPairC = pair_columns<N>() ? PairStepCfg<N>::COLS : 2;

// The persistent TMA-fed column passes of the FP32 plans (passes_tma.cuh), by variant, where
// their stages and tables fit in shared memory:
//   1: the step's tile (PairStepCfg::COLS columns), 3 stages, one block per SM
//   2: half that tile, 3 stages, two blocks per SM
//   3, 4: as 1, 2, with the results stored from the stage by TMA instead of from the consumers' registers
//   5, 6: half the step's tile, as many stages as fit (at most 6), one block per SM, stores from registers /
//         by TMA (the grids whose default tile is too tall for three stages, 1024^2 and up)
//   7: as 6 with the twiddles read from global memory, which frees room for one more stage (2048^2)
template <int V> struct TmaVariant;
template <> struct TmaVariant<1> { template <int NN> using Cfg = TmaColCfg<NN, PairStepCfg<NN>::COLS, 3, 1>; };
template <> struct TmaVariant<2> { template <int NN> using Cfg = TmaColCfg<NN, PairStepCfg<NN>::COLS / 2, 3, 2>; };
template <> struct TmaVariant<3> { template <int NN> using Cfg = TmaColCfg<NN, PairStepCfg<NN>::COLS, 3, 1, true>; };
template <> struct TmaVariant<4> { template <int NN> using Cfg = TmaColCfg<NN, PairStepCfg<NN>::COLS / 2, 3, 2, true>; };
template <> struct TmaVariant<5> {
    template <int NN> using Cfg = TmaColCfg<NN, PairStepCfg<NN>::COLS / 2, tma_fit_stages<NN, PairStepCfg<NN>::COLS / 2, false>(), 1>;
};
template <> struct TmaVariant<6> {
    template <int NN>
    using Cfg = TmaColCfg<NN, PairStepCfg<NN>::COLS / 2, tma_fit_stages<NN, PairStepCfg<NN>::COLS / 2, false>(), 1, true>;
};
template <> struct TmaVariant<7> {
    template <int NN>
    using Cfg = TmaColCfg<NN, PairStepCfg<NN>::COLS / 2, tma_fit_stages<NN, PairStepCfg<NN>::COLS / 2, true>(), 1, true, true>;
};
// The persistent passes with one barrier domain per column pair (passes_tmx.cuh), 3 stages, TMA loads and
// stores, no producer warp: 11 a tile of 8192 / N columns (512 threads, one block per SM), 12 half that tile
// (256 threads, two blocks per SM)
template <int V> struct TmxVariant;
// columns of a per-pair-barrier tile: the largest power of two at most budget / n (at least 2)
constexpr int tmx_cols(int n, int budget) {
    int c = 2;
    while (2 * c <= budget / n) c *= 2;
    return c;
}
template <> struct TmxVariant<11> { template <int NN> using Cfg = TmxColCfg<NN, tmx_cols(NN, 8192), 3, 1>; };
template <> struct TmxVariant<12> { template <int NN> using Cfg = TmxColCfg<NN, tmx_cols(NN, 4096), 3, 2>; };
// the 16-element plan (Plan16: one exchange fewer a transform, twice the elements a thread) at 1024 and 2048
template <> struct TmxVariant<13> {
    template <int NN> using Cfg = TmxColCfg<NN, tmx_cols(NN, 8192), 3, 1, std::conditional_t<plan16_ok(NN), Plan16<NN>, Plan<NN>>>;
};
template <class RR, int V> constexpr bool tmx_col_ok() {
    if constexpr (std::is_same<RR, float>::value && pair_columns<N>() && N >= 256 && (V != 13 || plan16_ok(N))) {
        using TC = typename TmxVariant<V>::template Cfg<N>;
        return TC::ok && TC::COLS % CC::COLS == 0 && N % TC::COLS == 0;
    } else {
        return false;
    }
}
template <class RR, int V> constexpr bool tma_col_ok() {
    if constexpr (std::is_same<RR, float>::value && pair_columns<N>()) {
        using TC = typename TmaVariant<V>::template Cfg<N>;
        return TC::ok && TC::COLS % CC::COLS == 0;   // the tile covers whole engine tiles
    } else {
        return false;
    }
}
// The column-step kernels of this size, by kind: 0 the two-column step at its default tile, 1 / 2 the
// persistent TMA-fed passes, 3 / 4 the two-column step at half / twice the default tile, 5 / 6 the persistent
// passes 1 / 2 storing through TMA, 7 / 8 / 10 the deep-ring persistent passes 5 / 6 / 7, 9 the two-column step
// at its default tile with the other register budget, 11 / 12 the per-pair-barrier passes. A variant index of PassOps::col_step is a position in the
// list of the kinds valid here (kind 0 always first).
struct KindList {
    int kind[14];
    int n;
};
template <class RR> constexpr KindList col_kinds() {
    KindList k{{0, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1}, 1};
    if (tma_col_ok<RR, 1>()) k.kind[k.n++] = 1;
    if (tma_col_ok<RR, 2>()) k.kind[k.n++] = 2;
    if (pair_tile_ok<RR, kPairC / 2>()) k.kind[k.n++] = 3;
    if (pair_tile_ok<RR, kPairC * 2>()) k.kind[k.n++] = 4;
    if (tma_col_ok<RR, 3>()) k.kind[k.n++] = 5;
    if (tma_col_ok<RR, 4>()) k.kind[k.n++] = 6;
    if (tma_col_ok<RR, 5>()) k.kind[k.n++] = 7;
    if (tma_col_ok<RR, 6>()) k.kind[k.n++] = 8;
    if (pair_tile_ok<RR, kPairC, !pair_loose<N>()>()) k.kind[k.n++] = 9;
    if (tma_col_ok<RR, 7>()) k.kind[k.n++] = 10;
    if (tmx_col_ok<RR, 11>()) k.kind[k.n++] = 11;
    if (tmx_col_ok<RR, 12>()) k.kind[k.n++] = 12;
    if (tmx_col_ok<RR, 13>()) k.kind[k.n++] = 13;
    return k;
}
template <class RR> constexpr int tma_col_variants() { return col_kinds<RR>().n; }
// the default column kernel before any tuning: the per-pair-barrier pass where it exists (the tuner's pick in
// every measured run at those grids: two blocks per SM at 256^2 to 768^2, one at 1024^2, 1536^2, 2048^2 and
// 3072^2), else 0
template <class RR> constexpr int default_col_variant() {
    constexpr KindList k = col_kinds<RR>();
    const int want = N <= 768 ? 12 : 11;
    for (int i = 0; i < k.n; i++)
        if (k.kind[i] == want) return i;
    for (int i = 0; i < k.n; i++)
        if (k.kind[i] == 11 || k.kind[i] == 12) return i;
    return 0;
}
// the name of column-step variant v of this size
std::string col_variant_name(int v) {
    constexpr KindList k = col_kinds<R>();
    if (v < 0 || v >= k.n) return "";
    const int kind = k.kind[v];
    auto cols = [](int c) { return std::to_string(c) + "-column tiles"; };
    if (kind == 0 && !std::is_same<R, float>::value) return "one block per column tile and wave";
    if (kind == 0) return "one block per (" + cols(kPairC) + ", wave), two columns a thread";
    if (kind == 3) return "one block per (" + cols(kPairC / 2) + ", wave), two columns a thread";
    if (kind == 4) return "one block per (" + cols(kPairC * 2) + ", wave), two columns a thread";
    if (kind == 1) return "persistent, TMA-fed, " + cols(kPairC) + ", 3 stages, 1 block per SM";
    if (kind == 2) return "persistent, TMA-fed, " + cols(kPairC / 2) + ", 3 stages, 2 blocks per SM";
    if (kind == 5) return "persistent, TMA loads and stores, " + cols(kPairC) + ", 3 stages, 1 block per SM";
    if (kind == 6) return "persistent, TMA loads and stores, " + cols(kPairC / 2) + ", 3 stages, 2 blocks per SM";
    auto stages = [](int n) { return std::to_string(n) + " stages"; };
    if (kind == 7)
        return "persistent, TMA-fed, " + cols(kPairC / 2) + ", " + stages(TmaVariant<5>::Cfg<N>::STAGES) +
               ", 1 block per SM";
    if (kind == 10)
        return "persistent, TMA loads and stores, " + cols(kPairC / 2) + ", " + stages(TmaVariant<7>::Cfg<N>::STAGES) +
               ", twiddles from L1, 1 block per SM";
    if (kind == 13)
        return "persistent, per-pair barriers, TMA loads and stores, 16-element FFT plan (radix 16 first; rounds "
               "differently), " + cols(TmxVariant<13>::Cfg<N>::COLS) + ", 3 stages, 1 block per SM";
    if (kind == 11 || kind == 12) {
        constexpr int c11 = TmxVariant<11>::Cfg<N>::COLS, c12 = TmxVariant<12>::Cfg<N>::COLS;
        return "persistent, per-pair barriers, TMA loads and stores, " + cols(kind == 11 ? c11 : c12) +
               ", 3 stages, " + (kind == 11 ? "1 block" : "2 blocks") + " per SM";
    }
    if (kind == 9) {   // the budget a thread gets: 64, or 128 where the block's threads leave room for it
        constexpr int threads = PairCfg<N, kPairC, !pair_loose<N>()>::THREADS;
        const int regs = pair_loose<N>() ? 64 : std::min(128, 65536 / threads);
        return "one block per (" + cols(kPairC) + ", wave), two columns a thread, " + std::to_string(regs) +
               "-register budget";
    }
    return "persistent, TMA loads and stores, " + cols(kPairC / 2) + ", " + stages(TmaVariant<6>::Cfg<N>::STAGES) +
           ", 1 block per SM";
}
int g_sms[64] = {};
int sm_count() {
    int dev = 0;
    MS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal out of range");
    if (!g_sms[dev]) MS_CUDA(cudaDeviceGetAttribute(&g_sms[dev], cudaDevAttrMultiProcessorCount, dev));
    return g_sms[dev];
}
template <class RR, int V> void tma_col_attrs() {
    if constexpr (tma_col_ok<RR, V>()) {
        using TC = typename TmaVariant<V>::template Cfg<N>;
        set_smem(k_col_step_tma<N, TC::COLS, TC::STAGES, TC::MINB, TC::TS, TC::TWG>, TC::smem());
    }
}
template <class RR, int V>
bool tma_col_step(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *tw, PropTables<RR> pt, RR b, int tiles_lo,
                  int tiles_hi) {
    if constexpr (tma_col_ok<RR, V>()) {
        using TC = typename TmaVariant<V>::template Cfg<N>;
        if (!pt.err) throw std::runtime_error("persistent column pass without an error word");
        constexpr int k = TC::COLS / CC::COLS, total = N / TC::COLS;
        static_assert(TC::COLS % CC::COLS == 0, "the step's tile must cover whole engine tiles");
        int lo = (tiles_lo + k - 1) / k, hi = (tiles_hi + k - 1) / k;
        if (lo + hi > total) { lo = total; hi = 0; }
        const long long items = (long long)(lo + hi) * batch;
        if (items > 0x7fffffffLL || (long long)batch * N > 0x7fffffffLL) throw std::runtime_error("batch too large");
        const CUtensorMap tm = wave_tensor_map(wave, 2ull * N, (unsigned long long)batch * N, TC::BOX_FLOATS, TC::BOX_ROWS);
        const int grid = (int)std::min<long long>(items, (long long)TC::MINB * sm_count());
        k_col_step_tma<N, TC::COLS, TC::STAGES, TC::MINB, TC::TS, TC::TWG><<<grid, TC::THREADS, TC::smem(), s>>>(
            tm, wave, tw, pt, b, lo, lo + hi, (int)items, pt.err);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}

template <class RR, int V> void tmx_col_attrs() {
    if constexpr (tmx_col_ok<RR, V>()) {
        using TC = typename TmxVariant<V>::template Cfg<N>;
        set_smem(k_col_step_tmx<N, TC::COLS, TC::STAGES, TC::MINB, typename TC::P>, TC::smem());
    }
}
template <class RR, int V>
bool tmx_col_step(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *tw, PropTables<RR> pt, RR b, int tiles_lo,
                  int tiles_hi) {
    if constexpr (tmx_col_ok<RR, V>()) {
        using TC = typename TmxVariant<V>::template Cfg<N>;
        if (!pt.err) throw std::runtime_error("persistent column pass without an error word");
        constexpr int k = TC::COLS / CC::COLS, total = N / TC::COLS;
        int lo = (tiles_lo + k - 1) / k, hi = (tiles_hi + k - 1) / k;
        if (lo + hi > total) { lo = total; hi = 0; }
        const long long items = (long long)(lo + hi) * batch;
        if (items > 0x7fffffffLL || (long long)batch * N > 0x7fffffffLL) throw std::runtime_error("batch too large");
        const CUtensorMap tm =
            wave_tensor_map(wave, 2ull * N, (unsigned long long)batch * N, TC::BOX_FLOATS, TC::BOX_ROWS, TC::SWIZZLE);
        const int grid = (int)std::min<long long>(items, (long long)TC::MINB * sm_count());
        // the 16-element plan's twiddles follow the other plans' tables (Ctx::twiddles, entries [2N, 3N))
        const cplx<RR> *twp = TC::P::E == 16 ? tw + 2 * N : tw;
        k_col_step_tmx<N, TC::COLS, TC::STAGES, TC::MINB, typename TC::P><<<grid, TC::THREADS, TC::smem(), s>>>(
            tm, twp, pt, b, lo, lo + hi, (int)items, pt.err);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}

// the two-row step kernel of the FP32 non-wide row plans
template <class RR> void rowpair_attrs() {
    if constexpr (std::is_same<RR, float>::value && pair_rows<N>())
        set_smem(k_row_step_pair<N, rowpair_pairs<N>()>, RowPairStepCfg<N>::smem());
    if constexpr (std::is_same<RR, float>::value && alt_pair_rows<N>())
        set_smem(k_row_step_pair<N, altrow_pairs<N>()>, RowPairCfg<N, altrow_pairs<N>()>::smem());
}

// blocks of kernel k (block size threads, dynamic smem bytes) resident on the whole device
template <class K> int resident_blocks(K k, int threads, size_t smem) {
    int per_sm = 0;
    MS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem));
    return std::max(1, per_sm) * sm_count();
}
template <class RR>
bool rowpair_step(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *trans, const cplx<RR> *tw, RR a, int xa,
                  int xb, int load_all, const int *tsel, size_t tstride, int variant) {
    if constexpr (std::is_same<RR, float>::value && pair_rows<N>()) {
        constexpr int PR = rowpair_pairs<N>();
        static int res[64] = {};
        int dev = 0;
        MS_CUDA(cudaGetDevice(&dev));
        if (variant > 0 && variant < 3 && !res[dev])
            res[dev] = resident_blocks(k_row_step_pair<N, PR>, Plan<N>::NT * PR, RowPairStepCfg<N>::smem());
        const int pf = variant == 3 ? kWaveFastRows : (variant > 0 ? variant * res[dev] : 0);
        const dim3 g = variant == 3 ? dim3(batch, N / (2 * PR)) : dim3(N / (2 * PR), batch);
        k_row_step_pair<N, PR><<<g, dim3(Plan<N>::NT, PR), RowPairStepCfg<N>::smem(), s>>>(wave, trans, tw, a, xa, xb,
                                                                                         load_all, tsel, tstride, pf);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}

// the two-row step of the plain plan as the alternative row plan (variants 4-7: prefetch / order mode v - 4)
template <class RR>
bool altrow_step(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *trans, const cplx<RR> *tw, RR a, int xa,
                 int xb, int load_all, const int *tsel, size_t tstride, int variant) {
    if constexpr (std::is_same<RR, float>::value && alt_pair_rows<N>()) {
        constexpr int PR = altrow_pairs<N>();
        using PC = RowPairCfg<N, PR>;
        static int res[64] = {};
        int dev = 0;
        MS_CUDA(cudaGetDevice(&dev));
        const int mode = variant - 4;
        if (mode > 0 && mode < 3 && !res[dev]) res[dev] = resident_blocks(k_row_step_pair<N, PR>, PC::THREADS, PC::smem());
        const int pf = mode == 3 ? kWaveFastRows : (mode > 0 ? mode * res[dev] : 0);
        if (mode != 3 && batch > 65535) throw std::runtime_error("batch too large for the row grid");
        const dim3 g = mode == 3 ? dim3(batch, N / (2 * PR)) : dim3(N / (2 * PR), batch);
        k_row_step_pair<N, PR><<<g, dim3(Plan<N>::NT, PR), PC::smem(), s>>>(wave, trans, tw, a, xa, xb, load_all, tsel,
                                                                          tstride, pf);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}
// row variants: 0-3 the default plan's kernel in the four prefetch / order modes; then, where they exist, the
// plain Stockham plan's two-row step in the same four modes (4-7), and the default plan's kernel with staged
// transmission rows (k_row_step_ts) in the same four modes (row_ts_first() on)
template <class RR> constexpr bool row_alt_ok() {
    if constexpr (std::is_same<RR, float>::value) return alt_pair_rows<N>();
    else return false;
}
template <class RR> constexpr bool row_ts_here() {
    if constexpr (std::is_same<RR, float>::value) return row_ts_ok<N>();
    else return false;
}
template <class RR> constexpr int row_ts_first() { return row_alt_ok<RR>() ? 8 : 4; }
template <class RR> constexpr int row_variant_count() { return row_ts_first<RR>() + (row_ts_here<RR>() ? 4 : 0); }
std::string row_variant_name(int v) {
    static const char *modes[4] = {"plain", "L2 prefetch of the rows one grid residency ahead",
                                   "L2 prefetch of the rows two grid residencies ahead",
                                   "wave-fastest grid order (the same rows of consecutive waves together)"};
    if (v < 0 || v >= row_variant_count<R>()) return "";
    if (v < 4) return modes[v];
    if (v >= row_ts_first<R>()) return std::string("transmission rows staged by the copy engine; ") + modes[v - row_ts_first<R>()];
    return std::string("plain Stockham plan (radix ") + (is_pow2(N) ? "8" : "4 then 12") + "), two rows a thread; " +
           modes[v - 4];
}
// the FP32 row step with staged transmission rows in prefetch / order mode `mode`
template <class RR>
bool row_step_ts(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *trans, const cplx<RR> *tw, RR a, int xa,
                 int xb, int load_all, const int *tsel, size_t tstride, int mode, int *err) {
    if constexpr (row_ts_here<RR>()) {
        // the copy engine's source: the block's rows start 16-byte aligned when trans and the set stride are
        if ((reinterpret_cast<uintptr_t>(trans) & 15) != 0 || (tstride * sizeof(cplx<RR>)) % 16 != 0 || err == nullptr)
            throw std::runtime_error("staged transmission rows need a 16-byte aligned transmission and an error word");
        static int res[64] = {};
        int dev = 0;
        MS_CUDA(cudaGetDevice(&dev));
        if (mode > 0 && mode < 3 && !res[dev]) res[dev] = resident_blocks(k_row_step_ts<N>, RC::THREADS, row_ts_smem<N, RR>());
        const int pf = mode == 3 ? kWaveFastRows : (mode > 0 ? mode * res[dev] : 0);
        k_row_step_ts<N><<<pf == kWaveFastRows ? dim3(batch, N / RC::ROWS) : dim3(N / RC::ROWS, batch),
                           dim3(RC::P::NT, RC::ROWS), row_ts_smem<N, RR>(), s>>>(wave, trans, tw, a, xa, xb, load_all,
                                                                                 tsel, tstride, pf, err);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}

template <class RR> void row_w3_attrs() {
    if constexpr (std::is_same<RR, float>::value && (RowCfg<N, RR>::WIDE3 || RowCfg<N, RR>::WIDE24)) set_smem(k_row_step_w3<N>, RC::smem());
}
// kernel attributes are per device: set once for each device this process launches on
bool g_attrs_done[64] = {};
void ensure_attrs() {
    int dev = 0;
    MS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || g_attrs_done[dev]) return;
    set_smem(k_row_step<R, N>, RC::smem());
    row_w3_attrs<R>();
    if constexpr (row_ts_here<R>()) set_smem(k_row_step_ts<N>, row_ts_smem<N, R>());
    if constexpr (std::is_same<R, double>::value && fp64_row_bounded<N>()) set_smem(k_row_step_d<N>, RC::smem());
    set_smem(k_row_fft<R, N, -1>, RC::smem());
    set_smem(k_row_fft<R, N, +1>, RC::smem());
    set_smem(k_col_step<R, N, COL_STEP>, CC::smem());
    pair_attrs<R, kPairC>();
    pair_attrs<R, kPairC / 2>();
    pair_attrs<R, kPairC * 2>();
    pair_attrs<R, kPairC, !pair_loose<N>()>();
    tma_col_attrs<R, 1>();
    tma_col_attrs<R, 2>();
    tma_col_attrs<R, 3>();
    tma_col_attrs<R, 4>();
    tma_col_attrs<R, 5>();
    tma_col_attrs<R, 6>();
    tma_col_attrs<R, 7>();
    tmx_col_attrs<R, 11>();
    tmx_col_attrs<R, 12>();
    tmx_col_attrs<R, 13>();
    rowpair_attrs<R>();
    set_smem(k_col_step<R, N, COL_STEP_DET>, CC::smem());
    set_smem(k_col_step<R, N, COL_DET_ONLY>, CC::smem());
    set_smem(k_col_fft<R, N, -1>, CC::smem());
    set_smem(k_col_fft<R, N, +1>, CC::smem());
    set_smem(k_col_bandlimit<R, N>, CC::smem());
    set_smem(k_col_probe<R, N>, CC::smem());
    set_smem(k_row_step_save<R, N>, RC::smem());
    set_smem(k_row_adjoint<R, N>, RC::smem());
    g_attrs_done[dev] = true;
}

inline dim3 row_grid(int batch) { return dim3(N / RC::ROWS, batch); }
inline dim3 row_grid_wave_fast(int batch) { return dim3(batch, N / RC::ROWS); }
inline dim3 row_block() { return dim3(RC::P::NT, RC::ROWS); }

// the FP64 row step built for 3 blocks per SM where that is set (fp64_step_minb)
template <class RR>
bool row_step_d(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *trans, const cplx<RR> *tw, RR a, int xa,
                int xb, int load_all, const int *tsel, size_t tstride, int pf) {
    if constexpr (std::is_same<RR, double>::value && fp64_row_bounded<N>()) {
        k_row_step_d<N><<<pf == kWaveFastRows ? row_grid_wave_fast(batch) : row_grid(batch), row_block(), RC::smem(),
                          s>>>(wave, trans, tw, a, xa, xb, load_all, tsel, tstride, pf);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}
// the FP32 row step with the three-stage wide plan or a radix-24 plan (RowCfg::WIDE3 / WIDE24), compiled for
// its blocks per SM
template <class RR>
bool row_step_w3(cudaStream_t s, int batch, cplx<RR> *wave, const cplx<RR> *trans, const cplx<RR> *tw, RR a, int xa,
                 int xb, int load_all, const int *tsel, size_t tstride, int pf) {
    if constexpr (std::is_same<RR, float>::value && (RowCfg<N, RR>::WIDE3 || RowCfg<N, RR>::WIDE24)) {
        k_row_step_w3<N><<<pf == kWaveFastRows ? row_grid_wave_fast(batch) : row_grid(batch), row_block(), RC::smem(),
                           s>>>(wave, trans, tw, a, xa, xb, load_all, tsel, tstride, pf);
        MS_CUDA(cudaGetLastError());
        return true;
    } else {
        return false;
    }
}
// blocks of the row step resident on the whole device
template <class RR> int row_resident() {
    if constexpr (std::is_same<RR, float>::value && (RowCfg<N, RR>::WIDE3 || RowCfg<N, RR>::WIDE24))
        return resident_blocks(k_row_step_w3<N>, RC::THREADS, RC::smem());
    else
        return resident_blocks(k_row_step<RR, N>, RC::THREADS, RC::smem());
}
inline dim3 col_grid(int batch) { return dim3(N / CC::COLS, batch); }
inline dim3 col_block() { return dim3(CC::COLS, CC::P::NT); }

void row_step(cudaStream_t s, cplx<R> *wave, int batch, const cplx<R> *trans, const cplx<R> *tw, R a, int xa, int xb,
              int load_all, const int *tsel, size_t tstride, int variant, int *err) {
    ensure_attrs();
    if (variant < 0 || variant >= row_variant_count<R>()) throw std::runtime_error("row pass variant out of range");
    if (variant >= row_ts_first<R>()) {
        if (variant - row_ts_first<R>() != 3 && batch > 65535) throw std::runtime_error("batch too large for the row grid");
        if (row_step_ts<R>(s, batch, wave, trans, tw, a, xa, xb, load_all, tsel, tstride, variant - row_ts_first<R>(), err))
            return;
        throw std::runtime_error("row pass variant out of range");
    }
    if (variant >= 4) {
        if (altrow_step<R>(s, batch, wave, trans, tw, a, xa, xb, load_all, tsel, tstride, variant)) return;
        throw std::runtime_error("row pass variant out of range");
    }
    if (batch > 65535 && variant != 3) throw std::runtime_error("batch too large for the row grid");
    if (rowpair_step<R>(s, batch, wave, trans, tw, a, xa, xb, load_all, tsel, tstride, variant)) return;
    static int res[64] = {};
    int dev = 0;
    MS_CUDA(cudaGetDevice(&dev));
    if (variant > 0 && variant < 3 && !res[dev]) res[dev] = row_resident<R>();
    const int pf = variant == 3 ? kWaveFastRows : (variant > 0 ? variant * res[dev] : 0);
    if (row_step_d<R>(s, batch, wave, trans, tw, a, xa, xb, load_all, tsel, tstride, pf)) return;
    if (row_step_w3<R>(s, batch, wave, trans, tw, a, xa, xb, load_all, tsel, tstride, pf)) return;
    k_row_step<R, N><<<pf == kWaveFastRows ? row_grid_wave_fast(batch) : row_grid(batch), row_block(), RC::smem(), s>>>(
        wave, trans, tw, a, xa, xb, load_all, tsel, tstride, pf);
    MS_CUDA(cudaGetLastError());
}
void row_fft(cudaStream_t s, const cplx<R> *in, cplx<R> *out, int batch, const cplx<R> *tw, R scale, int sign) {
    ensure_attrs();
    if (sign < 0) k_row_fft<R, N, -1><<<row_grid(batch), row_block(), RC::smem(), s>>>(in, out, tw, scale);
    else k_row_fft<R, N, +1><<<row_grid(batch), row_block(), RC::smem(), s>>>(in, out, tw, scale);
    MS_CUDA(cudaGetLastError());
}
void col_step(cudaStream_t s, cplx<R> *wave, int batch, const cplx<R> *tw, PropTables<R> pt, R b, R ds, DetArgs det,
              cplx<R> *recip, int mode, int tiles_lo, int tiles_hi, int variant) {
    ensure_attrs();
    if (tiles_lo < 0 || tiles_hi < 0 || tiles_lo + tiles_hi > N / CC::COLS || tiles_lo + tiles_hi == 0)
        throw std::runtime_error("column tile range out of bounds");
    if (variant < 0 || variant >= tma_col_variants<R>()) throw std::runtime_error("column pass variant out of range");
    dim3 g(tiles_lo + tiles_hi, batch);
    if (mode == COL_STEP && recip == nullptr && pt.ycut) {
        constexpr KindList kinds = col_kinds<R>();
        const int kind = kinds.kind[variant];
        if (kind == 1 && tma_col_step<R, 1>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 2 && tma_col_step<R, 2>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 5 && tma_col_step<R, 3>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 6 && tma_col_step<R, 4>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 7 && tma_col_step<R, 5>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 8 && tma_col_step<R, 6>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 9 && pair_step<R, kPairC, !pair_loose<N>()>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 10 && tma_col_step<R, 7>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 11 && tmx_col_step<R, 11>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 12 && tmx_col_step<R, 12>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 13 && tmx_col_step<R, 13>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 3 && pair_step<R, kPairC / 2>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (kind == 4 && pair_step<R, kPairC * 2>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
        if (pair_step<R, kPairC>(s, batch, wave, tw, pt, b, tiles_lo, tiles_hi)) return;
    }
    if (mode == COL_STEP && recip == nullptr)
        k_col_step<R, N, COL_STEP><<<g, col_block(), CC::smem(), s>>>(wave, tw, pt, b, ds, det, recip, tiles_lo);
    else if (mode == COL_DET_ONLY)
        k_col_step<R, N, COL_DET_ONLY><<<g, col_block(), CC::smem(), s>>>(wave, tw, pt, b, ds, det, recip, tiles_lo);
    else
        k_col_step<R, N, COL_STEP_DET><<<g, col_block(), CC::smem(), s>>>(wave, tw, pt, b, ds, det, recip, tiles_lo);
    MS_CUDA(cudaGetLastError());
}
void col_fft(cudaStream_t s, const cplx<R> *in, cplx<R> *out, int batch, const cplx<R> *tw, R scale, int sign) {
    ensure_attrs();
    if (sign < 0) k_col_fft<R, N, -1><<<col_grid(batch), col_block(), CC::smem(), s>>>(in, out, tw, scale);
    else k_col_fft<R, N, +1><<<col_grid(batch), col_block(), CC::smem(), s>>>(in, out, tw, scale);
    MS_CUDA(cudaGetLastError());
}
void col_bandlimit(cudaStream_t s, cplx<R> *wave, int batch, const cplx<R> *tw, const double *kx2, const double *ky2,
                   double lim, R scale) {
    ensure_attrs();
    k_col_bandlimit<R, N><<<col_grid(batch), col_block(), CC::smem(), s>>>(wave, tw, kx2, ky2, lim, scale);
    MS_CUDA(cudaGetLastError());
}
void col_probe(cudaStream_t s, cplx<R> *wave, int batch, const cplx<R> *tw, const double2 *chi, const double *kx,
               const double *ky, const double2 *pos, R scale, const double *dfac, double wavelength) {
    ensure_attrs();
    k_col_probe<R, N><<<col_grid(batch), col_block(), CC::smem(), s>>>(wave, tw, chi, kx, ky, pos, scale, dfac, wavelength);
    MS_CUDA(cudaGetLastError());
}
void row_step_save(cudaStream_t s, cplx<R> *wave, int batch, const cplx<R> *trans, const cplx<R> *tw, R a,
                   cplx<R> *save) {
    ensure_attrs();
    k_row_step_save<R, N><<<row_grid(batch), row_block(), RC::smem(), s>>>(wave, trans, tw, a, save);
    MS_CUDA(cudaGetLastError());
}
void row_adjoint(cudaStream_t s, cplx<R> *state, int batch, const cplx<R> *trans, const cplx<R> *tw, R a,
                 const cplx<R> *psi, cplx<R> *gT) {
    ensure_attrs();
    k_row_adjoint<R, N><<<row_grid(batch), row_block(), RC::smem(), s>>>(state, trans, tw, a, psi, gT);
    MS_CUDA(cudaGetLastError());
}
}  // namespace

template <>
PassOps<MS_REAL> make_pass_ops<MS_REAL, MS_N>() {
    PassOps<R> o;
    o.n = N;
    o.col_blocks = N / CC::COLS;
    o.cols_per_tile = CC::COLS;
    o.col_variants = tma_col_variants<R>();
    o.default_col_variant = default_col_variant<R>();
    o.col_variant_name = col_variant_name;
    o.row_variants = row_variant_count<R>();
    o.row_variant_name = row_variant_name;
    o.row_step = row_step;
    o.row_fft = row_fft;
    o.col_step = col_step;
    o.col_fft = col_fft;
    o.col_bandlimit = col_bandlimit;
    o.col_probe = col_probe;
    o.row_step_save = row_step_save;
    o.row_adjoint = row_adjoint;
    return o;
}

}  // namespace ms
