// passes_tma.cuh — persistent column pass of the FP32 multislice step fed by TMA tile loads.
//
// Same arithmetic per element as k_col_step_pair (passes.cuh): column FFT (two columns a thread, radix-8 /
// 3·2^k Stockham, fft_pair.cuh), times the propagator inside its cut and the scale b, inverse column FFT,
// so the results are bit-identical. What changes is how tiles reach the SM. One block runs per SM and
// loops over work items (wave, column tile):
//   - a producer warp streams the coming tiles of its items from HBM into a ring of STAGES shared-memory
//     stages with cp.async.bulk.tensor (a 2-D tensor map over the batch's rows), STAGES - 1 items ahead;
//   - the consumer threads read a stage into registers, run the transforms using the same stage as their
//     exchange space (the tile's row-major layout is the exchange layout of ColAddr<PAIRS, 16> when a tile
//     row is 128 bytes), hand the stage back (one mbarrier arrive per warp) and store the tile to HBM
//     straight from registers;
//   - or (TS) the consumers write the transformed tile back into its stage and the producer thread stores it
//     to HBM with cp.async.bulk.tensor before it refills the stage, so no consumer issues a global store.
// So a tile's global loads overlap the transforms of the tiles before it, and no consumer waits on a
// global load. Only this GPU's own wave buffer is read and written; no load uses cluster multicast.
#pragma once

#include "passes.cuh"
#include "tma.cuh"

namespace ms {

// the largest divisor of n that is at most 256 (a tensor-map box dimension is at most 256)
constexpr int tma_box_rows(int n, int d = 256) { return d <= 1 ? 1 : (n % d == 0 ? d : tma_box_rows(n, d - 1)); }

// Tile of COLS columns (two a consumer thread) of an N-row wave; the stage is the whole tile, loaded as
// N / BOX_ROWS boxes of BOX_ROWS rows. TWG: the FFT reads its twiddles from global memory (through L1)
// instead of a staged copy, which leaves room for one more stage where the tile column is tall (2048).
template <int N, int COLS_, int STAGES_ = 3, int MINB_ = 1, bool TS_ = false, bool TWG_ = false> struct TmaColCfg {
    using P = Plan<N>;
    static constexpr int COLS = COLS_;
    static constexpr bool TS = TS_;                    // results leave through the stage and a TMA store
    static constexpr bool TWG = TWG_;
    static constexpr int MINB = MINB_;                 // blocks per SM (the grid is MINB x the SM count)
    static constexpr int PAIRS = COLS / 2;
    static constexpr int NCONS = PAIRS * P::NT;        // consumer threads
    static constexpr int THREADS = NCONS + 32;         // + the producer warp
    static constexpr int STAGES = STAGES_;
    static constexpr int STAGE_BYTES = N * COLS * 8;
    static constexpr int BOX_ROWS = tma_box_rows(N);
    static constexpr int LOADS = N / BOX_ROWS;
    static constexpr int BOX_FLOATS = 2 * COLS;        // inner box extent in FP32 elements
    static constexpr int TABLES = (TWG ? 2 : 3) * N;   // staged float2 entries: twiddles (unless TWG), py, py errors
    // stages (128-byte aligned), twiddle table, the propagator's row tables (py and its errors, read at every
    // element; the column tables are read once per item from global memory), 2 mbarriers per stage
    static constexpr size_t smem() { return 128 + (size_t)STAGES * STAGE_BYTES + sizeof(float2) * TABLES + 16 * STAGES; }
    // one SM holds 228 KB of shared memory, 1 KB of it reserved per block
    static constexpr bool ok = STAGES >= 2 && N % BOX_ROWS == 0 && BOX_ROWS >= 16 && COLS >= 2 &&
                               (BOX_FLOATS * 4) % 16 == 0 && BOX_FLOATS <= 256 && NCONS % 32 == 0 &&
                               THREADS <= 1024 && smem() <= kMaxBlockSmem && MINB * (smem() + 1024) <= 228 * 1024 &&
                               (size_t)MINB * THREADS * 64 <= 65536;
};
// the most stages (at most 6) of a COLS-column tile that fit beside the tables in one block's shared memory
template <int N, int COLS, bool TWG> constexpr int tma_fit_stages() {
    constexpr size_t fixed = 128 + sizeof(float2) * (size_t)(TWG ? 2 : 3) * N;
    constexpr size_t per = (size_t)N * COLS * 8 + 16;
    constexpr int s = fixed < kMaxBlockSmem ? (int)((kMaxBlockSmem - fixed) / per) : 0;
    return s > 6 ? 6 : s;
}

// Work item i (0 <= i < n_items = batch * n_active): wave i / n_active, active tile j = i % n_active, which is
// column tile j for j < tiles_lo and tile N/COLS - (n_active - j) otherwise (the tiles holding columns inside
// the propagator's cut). err: the error word (tma.cuh StepError), written only when a wait is abandoned.
template <int N, int COLS, int STAGES, int MINB, bool TS, bool TWG>
__global__ void __launch_bounds__(TmaColCfg<N, COLS, STAGES, MINB, TS, TWG>::THREADS, MINB)
k_col_step_tma(const __grid_constant__ CUtensorMap tm, float2 *__restrict__ wave, const float2 *__restrict__ twg,
               PropTables<float> pt, float bscale, int tiles_lo, int n_active, int n_items, int *err) {
    using TC = TmaColCfg<N, COLS, STAGES, MINB, TS, TWG>;
    using P = Plan<N>;
    constexpr int PAIRS = TC::PAIRS, E = P::E, NT = P::NT, K = TC::STAGES, NCONS = TC::NCONS;
    extern __shared__ unsigned char smraw[];
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
    float4 *stages = reinterpret_cast<float4 *>(base);
    float2 *tabs = reinterpret_cast<float2 *>(base + (size_t)K * TC::STAGE_BYTES);
    // the propagator's row tables, read at every element: staged once per block, so no consumer waits on L1
    // for them (the column tables px, pxe and ycut are read once per item)
    float2 *s_tw = tabs, *s_py = TWG ? tabs : tabs + N, *s_pye = s_py + N;
    const float2 *tw = TWG ? twg : s_tw;
    uint64_t *full = reinterpret_cast<uint64_t *>(s_pye + N);
    uint64_t *empty = full + K;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < K; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCONS / 32);
        }
        mbar_fence_init();
    }
    for (int i = tid; i < N; i += TC::THREADS) {
        if constexpr (!TWG) s_tw[i] = twg[i];
        s_py[i] = pt.py[i];
        s_pye[i] = pt.pye[i];
    }
    __syncthreads();
    PropTables<float> spt = pt;
    spt.py = s_py;
    spt.pye = s_pye;

    if (tid >= NCONS) {   // producer warp: one elected thread issues the tile loads (and, with TS, stores)
        if (tid == NCONS) {
            tma_prefetch_desc(&tm);
            // wave and column tile of this block's k-th item
            auto item_of = [&](int kk, int &w, int &tile) {
                const int item = blockIdx.x + kk * gridDim.x;
                w = item / n_active;
                const int j = item - w * n_active;
                tile = j < tiles_lo ? j : N / COLS - (n_active - j);
            };
            // store the results of item kk, which the consumers left in its stage (TS)
            auto store = [&](int kk) {
                int w, tile;
                item_of(kk, w, tile);
                const unsigned char *src = base + (size_t)(kk % K) * TC::STAGE_BYTES;
#pragma unroll
                for (int l = 0; l < TC::LOADS; l++)
                    tma_store_2d(&tm, tile * TC::BOX_FLOATS, w * N + l * TC::BOX_ROWS,
                                 src + (size_t)l * TC::BOX_ROWS * COLS * 8);
                bulk_commit();
            };
            int k = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < n_items; item += gridDim.x, k++) {
                const int s = k % K;
                const unsigned use = (unsigned)(k / K);
                if (use > 0 && !mbar_wait(&empty[s], (use - 1) & 1, err, STEP_WAIT_EMPTY)) { ok = false; break; }
                if constexpr (TS) {
                    if (use > 0) {   // the stage holds item k - K's results: store them, then wait until read
                        store(k - K);
                        bulk_wait_read_all();
                    }
                }
                int w, tile;
                item_of(k, w, tile);
                unsigned char *dst = base + (size_t)s * TC::STAGE_BYTES;
                mbar_arrive_expect_tx(&full[s], TC::STAGE_BYTES);
#pragma unroll
                for (int l = 0; l < TC::LOADS; l++)
                    tma_load_2d(dst + (size_t)l * TC::BOX_ROWS * COLS * 8, &tm, tile * TC::BOX_FLOATS,
                                w * N + l * TC::BOX_ROWS, &full[s]);
            }
            if constexpr (TS) {   // the last (up to K) items: store each once its consumers are done
                for (int kk = k - K < 0 ? 0 : k - K; ok && kk < k; kk++) {
                    if (!mbar_wait(&empty[kk % K], (unsigned)(kk / K) & 1, err, STEP_WAIT_EMPTY)) { ok = false; break; }
                    store(kk);
                }
                bulk_wait_all();   // every store issued has written HBM and read its stage
            }
            if (!ok) {   // a wait was abandoned: let the loads already issued land before the block exits
                for (int d = 1; d <= K && k - d >= 0; d++) {
                    const int kk = k - d;
                    mbar_wait(&full[kk % K], (unsigned)(kk / K) & 1, err, STEP_WAIT_DRAIN);
                }
            }
        }
        return;
    }

    const int p = tid % PAIRS, t = tid / PAIRS;
    const NamedBar cbar{1, NCONS};
    int k = 0;
    for (int item = blockIdx.x; item < n_items; item += gridDim.x, k++) {
        const int s = k % K;
        if (!mbar_wait(&full[s], (unsigned)(k / K) & 1, err, STEP_WAIT_FULL)) break;
        const int w = item / n_active, j = item - w * n_active;
        const int tile = j < tiles_lo ? j : N / COLS - (n_active - j);
        const int x = tile * COLS + 2 * p;
        float4 *sm = stages + (size_t)s * (TC::STAGE_BYTES / 16);
        float2 va[E], vb[E];
#pragma unroll
        for (int m = 0; m < E; m++) {
            const float4 q = sm[(t + m * NT) * PAIRS + p];
            va[m] = make_float2(q.x, q.y);
            vb[m] = make_float2(q.z, q.w);
        }
        fft_pair<N, -1>(va, vb, sm + p, ColAddr<PAIRS, 16, col_swz_shift<N>()>(), t, tw, cbar);
        prop_pair<N>(va, vb, spt, x, t, bscale);
        fft_pair<N, +1>(va, vb, sm + p, ColAddr<PAIRS, 16, col_swz_shift<N>()>(), t, tw, cbar);
        if constexpr (TS) {
            // every consumer has read its last exchange values: the stage takes the results, which the
            // producer's TMA store then reads (the writes are ordered before it by the proxy fence and the
            // release of the arrive)
            cbar();
#pragma unroll
            for (int m = 0; m < E; m++) sm[(t + m * NT) * PAIRS + p] = make_float4(va[m].x, va[m].y, vb[m].x, vb[m].y);
            fence_proxy_async_smem();
            __syncwarp();
            if ((tid & 31) == 0) mbar_arrive(&empty[s]);
        } else {
            // the stage's last reads are done: hand it back to the producer (the copy engine writes it next)
            fence_proxy_async_smem();
            __syncwarp();
            if ((tid & 31) == 0) mbar_arrive(&empty[s]);
            float4 *gb = reinterpret_cast<float4 *>(wave + (size_t)w * N * N + x);
#pragma unroll
            for (int m = 0; m < E; m++)
                gb[(size_t)(t + m * NT) * (N / 2)] = make_float4(va[m].x, va[m].y, vb[m].x, vb[m].y);
        }
    }
}

}  // namespace ms
