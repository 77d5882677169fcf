// fft_pair.cuh — the Stockham plans of fft.cuh (2^k and 3·2^k) applied to two adjacent columns at once (FP32).
//
// A thread holds element m of its two columns in va[m], vb[m] (v[m] = x[t + m*NT] as in fft.cuh). Both
// columns go through the same butterflies and twiddles in the same order as fft.cuh, so each column's
// result is the one fft<float, N, SIGN> gives. Every shared-memory exchange moves the pair as one 16-byte
// element, which halves the shared-memory instructions and twiddle loads per column; the column pass is
// bound by its shared-memory instruction queue, not by HBM.
#pragma once

#include "fft.cuh"

namespace ms {

template <int N, int SIGN, int S, class Addr, class Sync>
__device__ __forceinline__ void fftp_stages(float2 (&va)[Plan<N>::E], float2 (&vb)[Plan<N>::E], float4 *sm, Addr ad,
                                            int t, const float2 *tw, Sync sync) {
    using P = Plan<N>;
    constexpr int E = P::E, NT = P::NT;
    constexpr int RAD = P::radix(S);
    constexpr int Ns = P::ns(S);
    constexpr int NB = E / RAD;
    constexpr bool last = (S == P::nstages - 1);
    constexpr int TWB = plan_tw_index(N, S > 0 ? S : 1, 0, 1);
    if constexpr (S > 0) {
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int j = t + b * NT;
#pragma unroll
            for (int r = 0; r < RAD; r++) {
                const float4 q = sm[ad(j + r * (N / RAD))];
                va[b + r * NB] = make_float2(q.x, q.y);
                vb[b + r * NB] = make_float2(q.z, q.w);
            }
        }
    }
    float2 oa[E], ob[E];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * NT;
        const int k = j % Ns;
        float2 a[RAD], c[RAD];
#pragma unroll
        for (int r = 0; r < RAD; r++) {
            float2 x = va[b + r * NB], y = vb[b + r * NB];
            if constexpr (S > 0) {
                if (r > 0) {
                    const float2 w = tw[TWB + k * (RAD - 1) + (r - 1)];
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
        sync();
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int j = t + b * NT;
            const int k = j % Ns;
            const int idxD = (j / Ns) * Ns * RAD + k;
#pragma unroll
            for (int m = 0; m < RAD; m++)
                sm[ad(idxD + m * Ns)] = make_float4(oa[b + m * NB].x, oa[b + m * NB].y, ob[b + m * NB].x, ob[b + m * NB].y);
        }
        sync();
        fftp_stages<N, SIGN, S + 1, Addr, Sync>(va, vb, sm, ad, t, tw, sync);
    }
}

// sync: the barrier over the threads sharing sm (the whole block by default)
template <int N, int SIGN, class Addr, class Sync = BlockSync>
__device__ __forceinline__ void fft_pair(float2 (&va)[Plan<N>::E], float2 (&vb)[Plan<N>::E], float4 *sm, Addr ad, int t,
                                         const float2 *tw, Sync sync = Sync()) {
    fftp_stages<N, SIGN, 0, Addr, Sync>(va, vb, sm, ad, t, tw, sync);
}

}  // namespace ms
