// fft.cuh — batched Stockham FFT building blocks staged in shared memory.
//
// One transform of length N is done by NT = N/E threads, each holding E elements in registers.
// Stage s (radix RAD, Ns = product of the radices before s) computes, for butterfly j in [0, N/RAD):
//     v[r] = x[j + r*N/RAD] * W_{Ns*RAD}^{r*(j mod Ns)},   y = DFT_RAD(v),
//     out[(j/Ns)*Ns*RAD + (j mod Ns) + m*Ns] = y[m]
// (the autosort Stockham formulation, Govindaraju et al., SC 2008). Thread t owns butterflies
// j = t + b*NT, b < E/RAD. With that assignment the first stage reads exactly the elements
// t + m*NT a thread loads from global memory, and the last stage writes exactly the elements
// t + m*NT it stores, so only the inner stage boundaries go through shared memory.
//
// Sizes: N = 2^k (E = 8, radix-8 stages plus one radix-2/4 stage) and N = 3*2^k (E = 12, radix-4 stages, an
// optional radix-2 stage and a radix-12 stage last). Unnormalised transforms; callers scale.
#pragma once

#include "common.cuh"

namespace ms {

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }
__host__ __device__ constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// The radix plan of a length, shared by the device stages and the host twiddle-table builder:
// 2^k: k/3 radix-8 stages, then one radix-2 or radix-4 stage if k%3 != 0;
// 3*2^k (k >= 2): (k-2)/2 radix-4 stages, a radix-2 stage if k is odd, then one radix-12 stage (a prime-factor
// 3 x 4 DFT: no twiddles inside, dft12). One exchange fewer than radix-3 and radix-4 stages apart (768: 4
// stages instead of 5). With the radix-12 stage last, every stage that writes to shared memory has a
// power-of-two span Ns, so its write positions (j / Ns) Ns R + j mod Ns + m Ns are bit fields of j and m.
__host__ __device__ constexpr int plan_k(int n) { return is_pow2(n) ? ilog2c(n) : ilog2c(n / 3); }
__host__ __device__ constexpr int plan_nstages(int n) {
    return is_pow2(n) ? (plan_k(n) / 3 + (plan_k(n) % 3 ? 1 : 0)) : (1 + (plan_k(n) - 2) / 2 + (plan_k(n) % 2));
}
__host__ __device__ constexpr int plan_radix(int n, int s) {
    return is_pow2(n) ? (s < plan_k(n) / 3 ? 8 : (plan_k(n) % 3 == 1 ? 2 : 4))
                      : (s == plan_nstages(n) - 1 ? 12 : (s < (plan_k(n) - 2) / 2 ? 4 : 2));
}
__host__ __device__ constexpr int plan_ns(int n, int s) { return s == 0 ? 1 : plan_ns(n, s - 1) * plan_radix(n, s - 1); }
// Twiddle table layout: stage s >= 1 stores W_n^(r*k*n/(Ns*R)) for k < Ns, 1 <= r < R at
// (Ns - Ns(1)) + k*(R-1) + (r-1): one entry per twiddle a stage uses, ordered so that the threads of a
// warp (consecutive k) read distinct banks. The table has n - R(0) entries.
__host__ __device__ constexpr int plan_tw_index(int n, int s, int k, int r) {
    return (plan_ns(n, s) - plan_ns(n, 1)) + k * (plan_radix(n, s) - 1) + (r - 1);
}

template <int N>
struct Plan {
    static constexpr bool pow2 = is_pow2(N);
    static_assert(pow2 || (N % 3 == 0 && is_pow2(N / 3) && N >= 12), "FFT length must be 2^k or 3*2^k, k >= 2");
    static constexpr int E = pow2 ? 8 : 12;
    static constexpr int NT = N / E;
    static constexpr int nstages = plan_nstages(N);
    __host__ __device__ static constexpr int radix(int s) { return plan_radix(N, s); }
    __host__ __device__ static constexpr int ns(int s) { return plan_ns(N, s); }
    // first entry of stage s's twiddles (s >= 1) in the packed table
    __host__ __device__ static constexpr int tw_base(int s) { return plan_tw_index(N, s, 0, 1); }
};

// A 16-element plan for the 2^k column passes at 1024 to 4096 (the per-pair-barrier kernels): a radix-16 stage,
// then radix-8 / radix-16 stages, 1024 = 16·8·8, 2048 = 16·16·8, 4096 = 16·16·16: one shared-memory exchange
// fewer than the 8-element plan (8·8·8·2, 8·8·8·4, 8·8·8·8) at twice the elements a thread. Its twiddle table
// has the packed layout of plan_tw_index (stage s at ns(s) - ns(1), N - 16 entries).
__host__ __device__ constexpr bool plan16_ok(int n) { return n == 1024 || n == 2048 || n == 4096; }
__host__ __device__ constexpr int plan16_radix(int n, int s) {
    return s == 0 ? 16 : (n == 1024 ? 8 : (n == 2048 ? (s == 1 ? 16 : 8) : 16));
}
template <int N>
struct Plan16 {
    static constexpr bool pow2 = true;
    static constexpr int E = 16;
    static constexpr int NT = N / E;
    static constexpr int nstages = 3;
    __host__ __device__ static constexpr int radix(int s) { return plan16_radix(N, s); }
    __host__ __device__ static constexpr int ns(int s) { return s == 0 ? 1 : ns(s - 1) * radix(s - 1); }
    __host__ __device__ static constexpr int tw_base(int s) { return ns(s) - ns(1); }
};

// ---- small DFTs in registers; SIGN = -1 forward, +1 inverse --------------------------------------
template <class C> __device__ __forceinline__ C mul_i(C a, int sign) {   // a * (sign * i)
    C r;
    if (sign > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
    return r;
}

template <class R, int SIGN> __device__ __forceinline__ void dft2(cplx<R> &a0, cplx<R> &a1) {
    cplx<R> t = a0;
    a0 = cadd(t, a1);
    a1 = csub(t, a1);
}
template <class R, int SIGN> __device__ __forceinline__ void dft4(cplx<R> &a0, cplx<R> &a1, cplx<R> &a2, cplx<R> &a3) {
    cplx<R> A0 = cadd(a0, a2), A1 = csub(a0, a2), A2 = cadd(a1, a3), A3 = mul_i(csub(a1, a3), SIGN);
    a0 = cadd(A0, A2);
    a2 = csub(A0, A2);
    a1 = cadd(A1, A3);
    a3 = csub(A1, A3);
}
// a sqrt(3)/2: FP32 as the FP32 value plus its remainder (as mul_rsqrt2 below), FP64 the FP64 value
template <class R> __device__ __forceinline__ R mul_sqrt3_2(R a) {
    if constexpr (sizeof(R) == 8) {
        return a * (R)0.86602540378443864676;
    } else {
        return fmaf(a, 0.8660253882408142f, a * 1.5543625053737742e-08f);
    }
}
template <class R, int SIGN> __device__ __forceinline__ void dft3(cplx<R> &a0, cplx<R> &a1, cplx<R> &a2) {
    cplx<R> t1 = cadd(a1, a2), t2 = csub(a1, a2);
    cplx<R> m = mk<R>(a0.x - (R)0.5 * t1.x, a0.y - (R)0.5 * t1.y);
    cplx<R> s = mul_i(mk<R>(mul_sqrt3_2<R>(t2.x), mul_sqrt3_2<R>(t2.y)), SIGN);
    a0 = cadd(a0, t1);
    a1 = cadd(m, s);
    a2 = csub(m, s);
}
// a / sqrt(2). FP32: times the FP32 value of 1/sqrt(2) plus its remainder, so the radix-8 twiddles keep
// modulus 1 to second order (an FFT round trip multiplies by |w|^2, and a modulus error would repeat at every
// slice and add up with thickness); FP64: times the FP64 value.
template <class R> __device__ __forceinline__ R mul_rsqrt2(R a) {
    if constexpr (sizeof(R) == 8) {
        return a * (R)0.70710678118654752440;
    } else {
        return fmaf(a, 0.7071067690849304f, a * 1.2101617485882343e-08f);
    }
}
template <class R, int SIGN> __device__ __forceinline__ void dft8(cplx<R> *a) {
    cplx<R> e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    cplx<R> o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<R, SIGN>(e0, e1, e2, e3);
    dft4<R, SIGN>(o0, o1, o2, o3);
    // W8^1 = (1 + SIGN i)/sqrt2, W8^2 = SIGN i, W8^3 = (-1 + SIGN i)/sqrt2
    cplx<R> w1o1, w2o2, w3o3;
    if (SIGN < 0) {
        w1o1 = mk<R>(mul_rsqrt2<R>(o1.x + o1.y), mul_rsqrt2<R>(o1.y - o1.x));
        w3o3 = mk<R>(mul_rsqrt2<R>(o3.y - o3.x), mul_rsqrt2<R>(-o3.x - o3.y));
    } else {
        w1o1 = mk<R>(mul_rsqrt2<R>(o1.x - o1.y), mul_rsqrt2<R>(o1.y + o1.x));
        w3o3 = mk<R>(mul_rsqrt2<R>(-o3.x - o3.y), mul_rsqrt2<R>(o3.x - o3.y));
    }
    w2o2 = mul_i(o2, SIGN);
    a[0] = cadd(e0, o0);
    a[4] = csub(e0, o0);
    a[1] = cadd(e1, w1o1);
    a[5] = csub(e1, w1o1);
    a[2] = cadd(e2, w2o2);
    a[6] = csub(e2, w2o2);
    a[3] = cadd(e3, w3o3);
    a[7] = csub(e3, w3o3);
}

// 12-point DFT as a prime-factor (Good-Thomas) 3 x 4 transform: with n = (4 n1 + 3 n2) mod 12 and
// k = (4 k1 + 9 k2) mod 12, W12^(nk) = W3^(n1 k1) W4^(n2 k2), so four 3-point DFTs over n1 and three 4-point
// DFTs over n2 give the transform with no twiddle products; the index maps cost nothing in registers.
template <class R, int SIGN> __device__ __forceinline__ void dft12(cplx<R> *a) {
    cplx<R> y[3][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
        cplx<R> x0 = a[(3 * n2) % 12], x1 = a[(4 + 3 * n2) % 12], x2 = a[(8 + 3 * n2) % 12];
        dft3<R, SIGN>(x0, x1, x2);
        y[0][n2] = x0;
        y[1][n2] = x1;
        y[2][n2] = x2;
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
        dft4<R, SIGN>(y[k1][0], y[k1][1], y[k1][2], y[k1][3]);
#pragma unroll
        for (int k2 = 0; k2 < 4; k2++) a[(4 * k1 + 9 * k2) % 12] = y[k1][k2];
    }
}

// 24-point DFT as a prime-factor (Good-Thomas) 3 x 8 transform: n = (8 n1 + 3 n2) mod 24 and
// k = (16 k1 + 9 k2) mod 24, so W24^(nk) = W3^(n1 k1) W8^(n2 k2): eight 3-point DFTs over n1, three 8-point
// DFTs over n2, no twiddle products
template <class R, int SIGN> __device__ __forceinline__ void dft24(cplx<R> *a) {
    cplx<R> y[3][8];
#pragma unroll
    for (int n2 = 0; n2 < 8; n2++) {
        cplx<R> x0 = a[(3 * n2) % 24], x1 = a[(8 + 3 * n2) % 24], x2 = a[(16 + 3 * n2) % 24];
        dft3<R, SIGN>(x0, x1, x2);
        y[0][n2] = x0;
        y[1][n2] = x1;
        y[2][n2] = x2;
    }
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
        dft8<R, SIGN>(y[k1]);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) a[(16 * k1 + 9 * k2) % 24] = y[k1][k2];
    }
}

// the wide radices (fft_wide.cuh), for plans that mix them with the radix-8 stages
template <class R, int SIGN> __device__ __forceinline__ void dft16(cplx<R> *a);
template <class R, int SIGN> __device__ __forceinline__ void dft32(cplx<R> *a);

template <class R, int RAD, int SIGN> __device__ __forceinline__ void dft(cplx<R> *a) {
    if constexpr (RAD == 2) dft2<R, SIGN>(a[0], a[1]);
    else if constexpr (RAD == 3) dft3<R, SIGN>(a[0], a[1], a[2]);
    else if constexpr (RAD == 4) dft4<R, SIGN>(a[0], a[1], a[2], a[3]);
    else if constexpr (RAD == 12) dft12<R, SIGN>(a);
    else if constexpr (RAD == 24) dft24<R, SIGN>(a);
    else if constexpr (RAD == 16) dft16<R, SIGN>(a);
    else if constexpr (RAD == 32) dft32<R, SIGN>(a);
    else dft8<R, SIGN>(a);
}

// ---- shared-memory addressing of one transform's elements ---------------------------------------
// Row transforms (8-byte elements, 16 threads per shared-memory wavefront): an XOR swizzle inside each
// aligned block of 16 elements, s(i) = i ^ g(i >> 4) with g(q) = (q & 7) | ((q & 4) << 1). It keeps the
// three access patterns of the radix-8 stages distinct modulo 16: stride-1 reads (t + c), the first
// stage's stride-8 writes (8t + m) and the second stage's grouped writes (64(t/8) + t%8 + 8m).
struct RowAddr {
    __device__ __forceinline__ int operator()(int i) const {
        const int q = i >> 4;
        return i ^ ((q & 7) | ((q & 4) << 1));
    }
    static constexpr int size(int n) { return n; }
};
// Column tiles: element i of column c at s(i)*COLS + c, threads of one row consecutive. The row swizzle
// s(i) = i ^ ((i >> SHIFT) & (RP - 1)), RP = rows per 128-byte wavefront, separates the rows a wavefront's
// threads touch in the first stage's writes (rows R t + m for radix R = 2^SHIFT: col_swz_shift).
template <int COLS, int ELEM_BYTES, int SHIFT = 3> struct ColAddr {
    static constexpr int RP = (128 / (COLS * ELEM_BYTES)) > 0 ? (128 / (COLS * ELEM_BYTES)) : 1;
    __device__ __forceinline__ int operator()(int i) const { return (i ^ ((i >> SHIFT) & (RP - 1))) * COLS; }
};
// the swizzle shift of a plan: log2 of its first radix (8 for the 2^k plans, 4 for the 3·2^k plans, whose
// radix-12 stage comes last); with it every stage's reads and writes of ColAddr tiles of 1 to 8 columns meet
// distinct banks (checked on the host for 384 to 3072)
template <int N> __host__ __device__ constexpr int col_swz_shift() { return Plan<N>::pow2 ? 3 : 2; }

// ---- synchronisation of the threads sharing a transform's shared memory ---------------------------
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
// A named barrier over the `count` threads (a multiple of 32) of one row transform.
struct NamedSync {
    int id, count;
    __device__ __forceinline__ void operator()() const { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory"); }
};

// ---- the stage recursion ----------------------------------------------------------------------
// v: E elements in "natural strided" order v[m] = x[t + m*NT] on entry and exit.
// sm: this transform's shared memory (element 0), ad: addressing, tw: the packed twiddle table.
// All threads of the block must call this together (it contains __syncthreads()).
// P: the radix plan (Plan<N>, or another with the same members: E, NT, nstages, radix, ns, tw_base).
template <class R, int N, int SIGN, int S, class Addr, class Sync, class P = Plan<N>>
__device__ __forceinline__ void fft_stages(cplx<R> (&v)[P::E], cplx<R> *sm, Addr ad, int t, const cplx<R> *tw,
                                           Sync sync) {
    constexpr int E = P::E, NT = P::NT;
    constexpr int RAD = P::radix(S);
    constexpr int Ns = P::ns(S);
    constexpr int NB = E / RAD;          // butterflies per thread
    constexpr bool last = (S == P::nstages - 1);
    constexpr int TWB = P::tw_base(S > 0 ? S : 1);   // this stage's block of the twiddle table
    if constexpr (S > 0) {
#pragma unroll
        for (int b = 0; b < NB; b++) {
            int j = t + b * NT;
#pragma unroll
            for (int r = 0; r < RAD; r++) v[b + r * NB] = sm[ad(j + r * (N / RAD))];
        }
    }
    cplx<R> out[E];
#pragma unroll
    for (int b = 0; b < NB; b++) {
        int j = t + b * NT;
        int k = j % Ns;
        cplx<R> a[RAD];
#pragma unroll
        for (int r = 0; r < RAD; r++) {
            cplx<R> x = v[b + r * NB];
            if constexpr (S > 0) {
                if (r > 0) {
                    cplx<R> w = tw[TWB + k * (RAD - 1) + (r - 1)];
                    x = (SIGN < 0) ? cmul(x, w) : cmulc(x, w);
                }
            }
            a[r] = x;
        }
        dft<R, RAD, SIGN>(a);
#pragma unroll
        for (int m = 0; m < RAD; m++) out[b + m * NB] = a[m];
    }
    if constexpr (last) {
#pragma unroll
        for (int i = 0; i < E; i++) v[i] = out[i];
    } else {
        sync();
#pragma unroll
        for (int b = 0; b < NB; b++) {
            int j = t + b * NT;
            int k = j % Ns;
            int idxD = (j / Ns) * Ns * RAD + k;
#pragma unroll
            for (int m = 0; m < RAD; m++) sm[ad(idxD + m * Ns)] = out[b + m * NB];
        }
        sync();
        fft_stages<R, N, SIGN, S + 1, Addr, Sync, P>(v, sm, ad, t, tw, sync);
    }
}

template <class R, int N, int SIGN, class Addr, class Sync = BlockSync>
__device__ __forceinline__ void fft(cplx<R> (&v)[Plan<N>::E], cplx<R> *sm, Addr ad, int t, const cplx<R> *tw,
                                    Sync sync = Sync()) {
    fft_stages<R, N, SIGN, 0, Addr, Sync>(v, sm, ad, t, tw, sync);
}

}  // namespace ms
