// passes_tmx.cuh — persistent column pass with one barrier domain per column pair (FP32, 2^k and 3·2^k plans,
// and the 16-element plans at 1024 and 2048, whose results round differently from the 8-element plan's).
//
// With the size's own plan (Plan<N>): same arithmetic per element, in the same order, as k_col_step_pair /
// k_col_step_tma (column FFT of two adjacent columns a thread, times the propagator inside its cut with the
// scale b folded into its column factor, inverse column FFT), so the results are bit-identical. What changes
// is who waits for whom:
//   - the NT threads of one column pair are whole warps (thread t of pair p is thread p * NT + t), and each
//     pair synchronises its FFT exchanges on its own named barrier, so a pair that waits on shared memory
//     does not hold up the other pairs of the block (k_col_step_tma makes all 16 consumer warps meet at
//     every exchange);
//   - there is no producer warp: one thread of the first pair issues the tile loads and stores at item
//     boundaries, so the block is 16 warps of 128 registers instead of 17 of 96;
//   - each thread keeps the twiddles of its butterflies in registers (they depend only on its position in
//     the transform), so the exchanges are the only shared-memory traffic of the FFTs (at 1024 the second
//     and third stages' come from a shared copy of the table, see tmx_tw_reg_stages).
// Tile layout in a stage: element (row y, pair p), 16 bytes, at slot PAIRS * y + (p ^ h(y)), h(y) =
// (y * PAIRS >> 3) mod PAIRS: the copy engine's 128B / 64B / 32B swizzle for 8 / 4 / 2 pairs (16-byte chunks
// of a 1024-byte atom XORed with the row's position in it), none for one pair. The FFT exchanges store
// logical row i at physical row g(i) = i ^ H((i >> 3) & 7) with the same swizzle: H the identity for the 2^k
// plans; for the 3·2^k plans (radix-4 stages, a radix-2 stage, radix 12 last) H maps bits (1, 2, 4) to
// (1, 6, 4), since their radix-4 writes at span 4 gather rows that the identity folds onto 4 bank groups.
// The 16-element plans use g(i) = i ^ ((i >> 4) & 7) instead: their radix-16 first stage writes the rows of
// 8 consecutive threads 16 apart.
// Both layouts give every pair the same slots (each pair only ever touches its own), and every access pattern
// of the plans' stages meets 8 distinct 16-byte bank groups per quarter warp (checked exhaustively on the host
// for every grid and pair count). Both maps are linear over GF(2) in the bits of the row, and so are the
// stages' read and write positions (all spans Ns of stages that write are powers of two), so an address is a
// per-thread base combined with a constant: an add folded into the instruction where the constant's bits lie
// outside the base's, one XOR otherwise.
// Only this GPU's own wave buffer is read and written; no load uses cluster multicast.
#pragma once

#include "passes_tma.cuh"

namespace ms {

template <int PAIRS> __host__ __device__ constexpr int tmx_swz(int row) {
    return PAIRS == 1 ? 0 : ((row * PAIRS) >> 3) & (PAIRS - 1);
}
// 16-byte slot of logical row i of pair 0 in the copy engine's layout / in the exchange layout
template <int PAIRS> __host__ __device__ constexpr int tmx_tlay(int i) { return PAIRS * i ^ tmx_swz<PAIRS>(i); }
// the exchange's row permutation g of a plan: i ^ ((i >> 3) & 7) for the 8-element 2^k plans, i ^ ((i >> 4) & 7)
// for the 16-element plans (their radix-16 writes at span 1 put the rows of 8 consecutive threads 16 apart), and
// i ^ H((i >> 3) & 7) with H mapping bits (1, 2, 4) to (1, 6, 4) for the 3·2^k plans
template <class PL> __host__ __device__ constexpr int tmx_g(int i) {
    return PL::E == 16 ? i ^ ((i >> 4) & 7)
                       : (PL::pow2 ? i ^ ((i >> 3) & 7) : i ^ (((i >> 3) & 5) ^ (((i >> 3) & 2) * 3)));
}
template <class PL, int PAIRS> __host__ __device__ constexpr int tmx_lay(int i) { return tmx_tlay<PAIRS>(tmx_g<PL>(i)); }
// the exchange write position of butterfly j's output 0 at stage S (fft.cuh: (j / Ns) Ns RAD + j mod Ns)
template <class PL, int S> __host__ __device__ constexpr int tmx_wrow(int j) {
    return (j / PL::ns(S)) * PL::ns(S) * PL::radix(S) + j % PL::ns(S);
}
// every bit a per-thread base f(t) ^ p can have (t < NT, p < PAIRS)
template <int PAIRS, int NT> __host__ __device__ constexpr int tmx_mask_tlay() {
    int m = PAIRS - 1;
    for (int b = 1; b < NT; b <<= 1) m |= tmx_tlay<PAIRS>(b);
    return m;
}
template <class PL, int PAIRS> __host__ __device__ constexpr int tmx_mask_lay() {
    int m = PAIRS - 1;
    for (int b = 1; b < PL::NT; b <<= 1) m |= tmx_lay<PL, PAIRS>(b);
    return m;
}
template <class PL, int PAIRS, int S> __host__ __device__ constexpr int tmx_mask_w() {
    int m = PAIRS - 1;
    for (int b = 1; b < PL::NT; b <<= 1) m |= tmx_lay<PL, PAIRS>(tmx_wrow<PL, S>(b));
    return m;
}
// the plans whose stages that write to shared memory all have power-of-two spans: the 2^k plans (8 or 16
// elements) and the 3·2^k plans, whose radix-12 stage comes last
template <class PL> __host__ __device__ constexpr bool tmx_plan_ok() {
    return (PL::pow2 && (PL::E == 8 || PL::E == 16)) || (!PL::pow2 && PL::E == 12 && PL::radix(PL::nstages - 1) == 12);
}
// base combined with the constant c: the two share no bit when (c & mask) == 0, and then the sum is the XOR
__device__ __forceinline__ int tmx_at(int base, int c, int mask) { return (c & mask) == 0 ? base + c : base ^ c; }

// twiddles a thread holds: stage S >= 1 keeps NB (RAD - 1) of them, in stage order, up to stage
// tmx_tw_reg_stages; the later stages read theirs from a copy of the plan's table in shared memory. At 1024 with
// the 8-element plan (ptxas, 128 registers a thread) all three stages' twiddles in registers spill 120 bytes a
// thread, two stages' 88 bytes, one stage's none; at the other grids and plans every stage's are kept (2048
// spills either way, and its stages leave no room for the table).
template <int N, class PL> __host__ __device__ constexpr int tmx_tw_reg_stages() {
    return (N == 1024 && PL::E == 8) ? 1 : PL::nstages - 1;
}
template <int N, class PL> __host__ __device__ constexpr bool tmx_tw_staged() { return tmx_tw_reg_stages<N, PL>() < PL::nstages - 1; }
template <int N, class PL> __host__ __device__ constexpr int tmx_tw_off(int S) {
    int o = 0;
    for (int s = 1; s < S && s <= tmx_tw_reg_stages<N, PL>(); s++) o += (PL::E / PL::radix(s)) * (PL::radix(s) - 1);
    return o;
}
template <int N, class PL> constexpr int tmx_tw_count() { return tmx_tw_off<N, PL>(PL::nstages); }

// PL: the FFT plan (Plan<N>, or Plan16<N> at 1024 and 2048)
template <int N, int COLS_, int STAGES_, int MINB_ = 1, class PL = Plan<N>> struct TmxColCfg {
    using P = PL;
    static constexpr int COLS = COLS_;
    static constexpr int PAIRS = COLS / 2;
    static constexpr int NT = P::NT;
    static constexpr int THREADS = PAIRS * NT;
    static constexpr int STAGES = STAGES_;
    static constexpr int MINB = MINB_;
    static constexpr int STAGE_BYTES = N * COLS * 8;
    static constexpr int BOX_ROWS = tma_box_rows(N);
    static constexpr int LOADS = N / BOX_ROWS;
    static constexpr int BOX_FLOATS = 2 * COLS;
    static constexpr int TWR = tmx_tw_count<N, PL>();
    // 1024-byte alignment slack (the swizzle atom), stages, the propagator's row tables (py and its errors),
    // two mbarriers per stage
    // (and, where some stages read their twiddles from shared memory, the plan's table)
    static constexpr size_t smem() {
        return 1024 + (size_t)STAGES * STAGE_BYTES + sizeof(float2) * (tmx_tw_staged<N, PL>() ? 3 : 2) * N + 16 * STAGES;
    }
    static constexpr bool ok = tmx_plan_ok<PL>() && is_pow2(P::NT) && (PAIRS == 1 || PAIRS == 2 || PAIRS == 4 || PAIRS == 8) &&
                               NT % 32 == 0 && THREADS <= 1024 && PAIRS <= 15 && STAGES >= 3 && N % BOX_ROWS == 0 &&
                               BOX_ROWS >= 16 && smem() <= kMaxBlockSmem && MINB * (smem() + 1024) <= 228 * 1024 &&
                               (size_t)MINB * THREADS * 128 <= 65536;
    // the copy engine's swizzle span in bytes (a tile row), 0 for none
    static constexpr int SWIZZLE = PAIRS == 1 ? 0 : COLS * 8;
};

// Stage S of the pair FFT (fft_pair.cuh's fftp_stages with the layouts above and register twiddles).
// rbase: tmx_lay(t) ^ p; wb[S]: tmx_lay(tmx_wrow<N, S>(t)) ^ p.
template <int N, int PAIRS, int SIGN, int S, int TWR, class PL>
__device__ __forceinline__ void tmx_stages(float2 (&va)[PL::E], float2 (&vb)[PL::E], float4 *sm, int rbase,
                                           const int (&wb)[PL::nstages], const float2 (&twr)[TWR],
                                           const float2 *s_tw, int t, NamedBar bar) {
    using P = PL;
    constexpr int E = P::E, NT = P::NT;
    constexpr int RAD = P::radix(S);
    constexpr int Ns = P::ns(S);
    constexpr int NB = E / RAD;
    constexpr bool last = (S == P::nstages - 1);
    constexpr int TWO = tmx_tw_off<N, PL>(S > 0 ? S : 1);
    constexpr bool TWREG = S <= tmx_tw_reg_stages<N, PL>();
    constexpr int TWB = P::tw_base(S > 0 ? S : 1);
    if constexpr (S > 0) {
        constexpr int RM = tmx_mask_lay<PL, PAIRS>();
#pragma unroll
        for (int b = 0; b < NB; b++) {
#pragma unroll
            for (int r = 0; r < RAD; r++) {
                const float4 q = sm[tmx_at(rbase, tmx_lay<PL, PAIRS>(b * NT + r * (N / RAD)), RM)];
                va[b + r * NB] = make_float2(q.x, q.y);
                vb[b + r * NB] = make_float2(q.z, q.w);
            }
        }
    }
    float2 oa[E], ob[E];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        float2 a[RAD], c[RAD];
#pragma unroll
        for (int r = 0; r < RAD; r++) {
            float2 x = va[b + r * NB], y = vb[b + r * NB];
            if constexpr (S > 0) {
                if (r > 0) {
                    const float2 w = TWREG ? twr[TWREG ? TWO + b * (RAD - 1) + (r - 1) : 0]
                                           : s_tw[TWB + ((t + b * NT) % Ns) * (RAD - 1) + (r - 1)];
                    x = (SIGN < 0) ? cmul(x, w) : cmulc(x, w);
                    y = (SIGN < 0) ? cmul(y, w) : cmulc(y, w);
                }
            }
            a[r] = x;
            c[r] = y;
        }
        dft<float, RAD, SIGN>(a);
        dft<float, RAD, SIGN>(c);
#pragma unroll
        for (int m = 0; m < RAD; m++) {
            oa[b + m * NB] = a[m];
            ob[b + m * NB] = c[m];
        }
    }
    if constexpr (last) {
#pragma unroll
        for (int i = 0; i < E; i++) { va[i] = oa[i]; vb[i] = ob[i]; }
    } else {
        constexpr int WM = tmx_mask_w<PL, PAIRS, S>();
        bar();   // the pair's reads of the previous layout are done
#pragma unroll
        for (int b = 0; b < NB; b++) {
#pragma unroll
            for (int m = 0; m < RAD; m++)
                sm[tmx_at(wb[S], tmx_lay<PL, PAIRS>(tmx_wrow<PL, S>(b * NT) | (m * Ns)), WM)] =
                    make_float4(oa[b + m * NB].x, oa[b + m * NB].y, ob[b + m * NB].x, ob[b + m * NB].y);
        }
        bar();
        tmx_stages<N, PAIRS, SIGN, S + 1, TWR, PL>(va, vb, sm, rbase, wb, twr, s_tw, t, bar);
    }
}

// thread t's twiddles: stage S, butterfly j = t + b NT, k = j mod Ns, entries r = 1..RAD-1 of the packed table
template <int N, int S, int TWR, class PL>
__device__ __forceinline__ void tmx_load_twiddles(float2 (&twr)[TWR], const float2 *twg, int t) {
    if constexpr (S <= tmx_tw_reg_stages<N, PL>()) {
        using P = PL;
        constexpr int RAD = P::radix(S), Ns = P::ns(S), NB = P::E / RAD, NT = P::NT;
        constexpr int TWB = P::tw_base(S);
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int k = (t + b * NT) % Ns;
#pragma unroll
            for (int r = 1; r < RAD; r++) twr[tmx_tw_off<N, PL>(S) + b * (RAD - 1) + (r - 1)] = twg[TWB + k * (RAD - 1) + (r - 1)];
        }
        tmx_load_twiddles<N, S + 1, TWR, PL>(twr, twg, t);
    }
}
template <int PAIRS, int S, class PL> __device__ __forceinline__ void tmx_write_bases(int (&wb)[PL::nstages], int t, int p) {
    if constexpr (S < PL::nstages) {
        wb[S] = tmx_lay<PL, PAIRS>(tmx_wrow<PL, S>(t)) ^ p;
        tmx_write_bases<PAIRS, S + 1, PL>(wb, t, p);
    }
}

// Work item i (0 <= i < n_items = batch * n_active): wave i / n_active, active tile j = i % n_active (column
// tile j for j < tiles_lo, tile N/COLS - (n_active - j) otherwise), as k_col_step_tma. The block's items are
// blockIdx.x + k gridDim.x. Thread 0 keeps the ring: before item k it stores item k - 1 (once every warp has
// written its results into that stage) and loads item k + STAGES - 2 into the stage of item k - 2 (once
// that stage's store has read it). err: the error word (tma.cuh StepError), written only when a wait is
// abandoned; a producer that gives up stops loading, and the consumers then give up at the first item that
// was never loaded (no pair is left waiting at a barrier for a warp that left).
template <int N, int COLS, int STAGES, int MINB, class PL = Plan<N>>
__global__ void __launch_bounds__(TmxColCfg<N, COLS, STAGES, MINB, PL>::THREADS, MINB)
k_col_step_tmx(const __grid_constant__ CUtensorMap tm, const float2 *__restrict__ twg, PropTables<float> pt, float bscale,
               int tiles_lo, int n_active, int n_items, int *err) {
    using TC = TmxColCfg<N, COLS, STAGES, MINB, PL>;
    using P = PL;
    constexpr int PAIRS = TC::PAIRS, E = P::E, NT = P::NT, K = TC::STAGES, THREADS = TC::THREADS;
    extern __shared__ unsigned char smraw[];
    unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smraw) + 1023) & ~uintptr_t(1023));
    float4 *stages = reinterpret_cast<float4 *>(base);
    float2 *s_py = reinterpret_cast<float2 *>(base + (size_t)K * TC::STAGE_BYTES), *s_pye = s_py + N;
    float2 *s_tw = s_pye + N;   // the plan's table, where some stages read their twiddles from shared memory
    uint64_t *full = reinterpret_cast<uint64_t *>(s_tw + (tmx_tw_staged<N, PL>() ? N : 0));
    uint64_t *empty = full + K;
    const int tid = threadIdx.x;
    const int p = tid / NT, t = tid % NT;
    if (tid == 0) {
        for (int s = 0; s < K; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], THREADS / 32);
        }
        mbar_fence_init();
    }
    for (int i = tid; i < N; i += THREADS) {
        s_py[i] = pt.py[i];
        s_pye[i] = pt.pye[i];
        if constexpr (tmx_tw_staged<N, PL>()) s_tw[i] = twg[i];
    }
    float2 twr[TC::TWR];
    tmx_load_twiddles<N, 1, TC::TWR, PL>(twr, twg, t);
    int wb[P::nstages];
    tmx_write_bases<PAIRS, 0, PL>(wb, t, p);
    const int rbase = tmx_lay<PL, PAIRS>(t) ^ p, tbase = tmx_tlay<PAIRS>(t) ^ p;
    constexpr int TM = tmx_mask_tlay<PAIRS, NT>();
    const NamedBar bar{1 + p, NT};
    __syncthreads();

    const int n_mine = n_items > (int)blockIdx.x ? (n_items - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    // (producer, thread 0) wave and column tile of this block's k-th item
    auto item_of = [&](int kk, int &w, int &tile) {
        const int item = (int)blockIdx.x + kk * (int)gridDim.x;
        w = item / n_active;
        const int j = item - w * n_active;
        tile = j < tiles_lo ? j : N / COLS - (n_active - j);
    };
    auto load = [&](int kk) {
        int w, tile;
        item_of(kk, w, tile);
        unsigned char *dst = base + (size_t)(kk % K) * TC::STAGE_BYTES;
        mbar_arrive_expect_tx(&full[kk % K], TC::STAGE_BYTES);
#pragma unroll
        for (int l = 0; l < TC::LOADS; l++)
            tma_load_2d(dst + (size_t)l * TC::BOX_ROWS * COLS * 8, &tm, tile * TC::BOX_FLOATS, w * N + l * TC::BOX_ROWS,
                        &full[kk % K]);
    };
    auto store = [&](int kk) {
        int w, tile;
        item_of(kk, w, tile);
        const unsigned char *src = base + (size_t)(kk % K) * TC::STAGE_BYTES;
#pragma unroll
        for (int l = 0; l < TC::LOADS; l++)
            tma_store_2d(&tm, tile * TC::BOX_FLOATS, w * N + l * TC::BOX_ROWS, src + (size_t)l * TC::BOX_ROWS * COLS * 8);
        bulk_commit();
    };
    bool prod_ok = true;   // thread 0: false once a producer wait was abandoned (no more loads or stores)
    int issued = 0;        // thread 0: items whose loads were issued
    if (tid == 0) {
        tma_prefetch_desc(&tm);
        for (; issued < K - 2 && issued < n_mine; issued++) load(issued);
    }

    for (int k = 0; k < n_mine; k++) {
        if (tid == 0 && prod_ok) {
            if (k >= 1) {
                if (mbar_wait(&empty[(k - 1) % K], (unsigned)((k - 1) / K) & 1, err, STEP_WAIT_EMPTY)) store(k - 1);
                else prod_ok = false;
            }
            if (prod_ok && issued < n_mine) {   // issued == k + K - 2
                if (issued >= K) bulk_wait_read<1>();   // the store of item issued - K has read its stage
                load(issued++);
            }
        }
        __syncwarp();
        const int s = k % K;
        const int item = (int)blockIdx.x + k * (int)gridDim.x;
        const int w = item / n_active, j = item - w * n_active;
        const int tile = j < tiles_lo ? j : N / COLS - (n_active - j);
        const int x = tile * COLS + 2 * p;
        const float2 pxa = prop_col(pt, x, bscale), pxb = prop_col(pt, x + 1, bscale), exa = pt.pxe[x], exb = pt.pxe[x + 1];
        const int2 ca = pt.ycut[x], cb = pt.ycut[x + 1];
        if (!mbar_wait(&full[s], (unsigned)(k / K) & 1, err, STEP_WAIT_FULL)) break;
        float4 *sm = stages + (size_t)s * (TC::STAGE_BYTES / 16);
        float2 va[E], vb[E];
#pragma unroll
        for (int m = 0; m < E; m++) {
            const float4 q = sm[tmx_at(tbase, tmx_tlay<PAIRS>(m * NT), TM)];
            va[m] = make_float2(q.x, q.y);
            vb[m] = make_float2(q.z, q.w);
        }
        tmx_stages<N, PAIRS, -1, 0, TC::TWR, PL>(va, vb, sm, rbase, wb, twr, s_tw, t, bar);
#pragma unroll
        for (int m = 0; m < E; m++) {
            const int y = t + m * NT;
            const float2 py = s_py[y], ey = s_pye[y];
            va[m] = (y < ca.x || y >= ca.y) ? prop_mul<float>(va[m], pxa, py, exa, ey) : mk<float>(0, 0);
            vb[m] = (y < cb.x || y >= cb.y) ? prop_mul<float>(vb[m], pxb, py, exb, ey) : mk<float>(0, 0);
        }
        tmx_stages<N, PAIRS, +1, 0, TC::TWR, PL>(va, vb, sm, rbase, wb, twr, s_tw, t, bar);
        bar();   // the pair's last exchange reads are done: the stage takes its results
#pragma unroll
        for (int m = 0; m < E; m++)
            sm[tmx_at(tbase, tmx_tlay<PAIRS>(m * NT), TM)] = make_float4(va[m].x, va[m].y, vb[m].x, vb[m].y);
        fence_proxy_async_smem();
        __syncwarp();
        if ((tid & 31) == 0) mbar_arrive(&empty[s]);
    }

    if (tid == 0) {
        if (prod_ok && n_mine > 0) {   // the last item's results
            const int kk = n_mine - 1;
            if (mbar_wait(&empty[kk % K], (unsigned)(kk / K) & 1, err, STEP_WAIT_EMPTY)) store(kk);
            else prod_ok = false;
        }
        if (!prod_ok) {   // let the loads already issued land before the block exits
            for (int d = 1; d <= K && issued - d >= 0; d++) {
                const int kk = issued - d;
                mbar_wait(&full[kk % K], (unsigned)(kk / K) & 1, err, STEP_WAIT_DRAIN);
            }
        }
        bulk_wait_all();   // every store issued has read its stage and written HBM
    }
}

}  // namespace ms
