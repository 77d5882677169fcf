// adjoint.cuh — row passes of the forward-with-save and adjoint multislice steps (differentiable CTEM).
//
// Forward step (passes.cuh): psi_{s+1} = s2d^2 Dinv(P D(T_s psi_s)). Its adjoint, as a real-linear map, is
//   G_{u_s}   = s2d^2 Dinv(conj(P) D(G_{psi_{s+1}})),   u_s = T_s psi_s
//   G_{psi_s} = conj(T_s) G_{u_s},      G_{T_s} = conj(psi_s) G_{u_s}
// (G = dL/dRe + i dL/dIm). With the wave held row-transformed between passes, the column pass with conj(P)
// maps D_r G_{psi_{s+1}} to D_r G_{u_s}, and the row-adjoint pass below maps D_r G_{u_s} to D_r G_{psi_s}
// while writing G_{T_s} in real space.
#pragma once

#include "passes.cuh"

namespace ms {

// Forward row pass that also stores psi_s = a * Dinv_r(phi) (real space, every column) in `save`.
template <class R, int N>
__global__ void __launch_bounds__(RowCfg<N, R>::THREADS)
k_row_step_save(cplx<R> *__restrict__ wave, const cplx<R> *__restrict__ trans, const cplx<R> *__restrict__ twg, R a,
                cplx<R> *__restrict__ save) {
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
    cplx<R> *row = wave + off;
    const cplx<R> *trow = trans + (size_t)y * N;
    cplx<R> v[P::E];
#pragma unroll
    for (int m = 0; m < P::E; m++) v[m] = row[t + m * P::NT];
    __syncthreads();
    row_transform<R, N, +1>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) {
        cplx<R> psi = cscale(v[m], a);
        save[off + t + m * P::NT] = psi;
        v[m] = cmul(psi, trow[t + m * P::NT]);
    }
    row_transform<R, N, -1>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) row[t + m * P::NT] = v[m];
}

// Adjoint row pass: g = a * Dinv_r(state) is G_{u_s} in real space; writes gT = conj(psi_s) g and
// state <- D_r(conj(T_s) g).
template <class R, int N>
__global__ void __launch_bounds__(RowCfg<N, R>::THREADS)
k_row_adjoint(cplx<R> *__restrict__ state, const cplx<R> *__restrict__ trans, const cplx<R> *__restrict__ twg, R a,
              const cplx<R> *__restrict__ psi, cplx<R> *__restrict__ gT) {
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
    cplx<R> *row = state + off;
    const cplx<R> *trow = trans + (size_t)y * N;
    cplx<R> v[P::E];
#pragma unroll
    for (int m = 0; m < P::E; m++) v[m] = row[t + m * P::NT];
    __syncthreads();
    row_transform<R, N, +1>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) {
        const int x = t + m * P::NT;
        cplx<R> g = cscale(v[m], a);
        gT[off + x] = cmulc(g, psi[off + x]);     // conj(psi) * g
        v[m] = cmulc(g, trow[x]);                 // conj(T) * g
    }
    row_transform<R, N, -1>(v, sm, t, tw);
#pragma unroll
    for (int m = 0; m < P::E; m++) row[t + m * P::NT] = v[m];
}

}  // namespace ms
