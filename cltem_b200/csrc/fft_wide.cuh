// fft_wide.cuh — two-stage Stockham FFT with wide radices for the FP32 passes at 256, 512 and 1024.
//
// N = E * R2 (E = 32 for N = 512 / 1024, 16 for N = 256; R2 = N / E <= E); NT = N / E threads per
// transform hold E elements each (v[m] = x[t + m*NT] on entry and exit, the layout of fft.cuh). Stage A is a
// radix-E DFT of each thread's elements in registers; stage B a radix-R2 DFT of E/R2 butterflies per thread
// with twiddles W_N^(r k) (butterfly k < E, 1 <= r < R2) read from a packed table at k (R2 - 1) + r - 1.
// One shared-memory exchange per transform instead of the radix-8 plan's two (the passes are bound by
// shared-memory traffic, not HBM). Shared layout: element i at (i / E)(E + 1) + i % E, rows of E padded by
// one, which keeps stage A's row writes and stage B's column reads free of bank conflicts (times COLS for
// a column tile, columns interleaved).
#pragma once

#include "fft.cuh"

namespace ms {

// the pass kernels at (precision, size) use the wide plan for FP32 at 256, 512 and 1024
template <class R> __host__ __device__ constexpr bool wide_plan(int n) {
    return sizeof(R) == 4 && (n == 256 || n == 512 || n == 1024);
}
__host__ __device__ constexpr int wide_E(int n) { return n >= 512 ? 32 : 16; }

template <int N> struct WidePlan {
    static constexpr int E = wide_E(N);
    static constexpr int R2 = N / E;
    static constexpr int NT = N / E;
    static constexpr int NB = R2 > 0 ? E / R2 : 1;   // stage B butterflies per thread
    static constexpr int TW = E * (R2 - 1);          // twiddle table entries
    static constexpr int ROWSZ = NT * (E + 1);       // padded shared elements of one transform
};

template <int E> struct WideRowAddr {
    __device__ __forceinline__ int operator()(int i) const { return (i / E) * (E + 1) + (i % E); }
};
template <int E, int COLS> struct WideColAddr {
    __device__ __forceinline__ int operator()(int i) const { return ((i / E) * (E + 1) + (i % E)) * COLS; }
};

// cos(phi pi / 16) for any integer phi
__device__ __forceinline__ double cos_pi16(int phi) {
    constexpr double c16[17] = {1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
                                0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173,
                                0.19509032201612826785, 0.0, -0.19509032201612826785, -0.38268343236508977173,
                                -0.55557023301960222474, -0.70710678118654752440, -0.83146961230254523708,
                                -0.92387953251128675613, -0.98078528040323044913, -1.0};
    phi &= 31;
    return phi <= 16 ? c16[phi] : c16[32 - phi];
}
// FP32 values of cos(m pi / 16), m = 0..8, each (cos, sin) pair (c[m], c[8 - m]) picked among the roundings of
// its two parts for the squared modulus closest to 1: an FFT round trip multiplies by |w|^2, and a modulus error
// repeats at every slice. cos(pi/4) = 0.70710677 leaves 2 c^2 - 1 = -3.4e-8, so cmul_wconst applies that one
// through mul_rsqrt2, which carries its remainder.
__device__ __forceinline__ float cos_pi16_f(int phi) {
    constexpr float c16[9] = {1.0f, 0.9807852506637573f, 0.9238795638084412f, 0.8314695954322815f, 0.7071067690849304f,
                              0.5555702447891235f, 0.3826833963394165f, 0.19509033858776093f, 0.0f};
    phi &= 31;
    const int m = phi <= 16 ? phi : 32 - phi;        // cos(phi pi/16) = cos((32 - phi) pi/16)
    return m <= 8 ? c16[m] : -c16[16 - m];             // cos((16 - m) pi/16) = -cos(m pi/16)
}

// x times exp(SIGN 2 pi i e / M) for M = 16 or 32: the angle is j pi / 16 with j = (32 / M) e; sin(x) = cos(x - pi/2).
// e is a compile-time constant at every call (unrolled loops), so the branches below fold away. FP32: the
// multiples of pi/2 are exact sign swaps (a product with 0 or 1 is not folded by the compiler under IEEE rules,
// so cmul would spend 2 instructions on them); the odd multiples of pi/4 scale the sum and difference of the
// parts by cos(pi/4) plus its remainder (mul_rsqrt2), 6 instructions where a compensated cmul takes 10 and
// exact to second order; the rest are one cmul with the constants above.
template <class R, int SIGN, int M> __device__ __forceinline__ cplx<R> cmul_wconst(cplx<R> x, int e) {
    const int j = ((32 / M) * e) & 31;
    if constexpr (sizeof(R) == 8) {
        return cmul(x, mk<R>((R)cos_pi16(j), (R)(SIGN * cos_pi16(j - 8))));
    } else {
        if (j == 0) return x;
        if (j == 16) return mk<R>(-x.x, -x.y);
        if (j == 8) return mul_i(x, SIGN);       // exp(SIGN i pi/2) = SIGN i
        if (j == 24) return mul_i(x, -SIGN);
        if ((j & 7) == 4) {                      // w = cos(pi/4) (sx, sy)
            const R sx = cos_pi16_f(j) > 0 ? (R)1 : (R)-1;
            const R sy = (R)SIGN * cos_pi16_f(j - 8) > 0 ? (R)1 : (R)-1;
            // x w = cos(pi/4) (sx x.x - sy x.y, sy x.x + sx x.y)
            return mk<R>(mul_rsqrt2<R>(sx * x.x - sy * x.y), mul_rsqrt2<R>(sy * x.x + sx * x.y));
        }
        return cmul(x, mk<R>(cos_pi16_f(j), (R)SIGN * cos_pi16_f(j - 8)));
    }
}

// 16-point DFT in registers as 4 x 4: n = 4 n1 + n2, k = k1 + 4 k2
template <class R, int SIGN> __device__ __forceinline__ void dft16(cplx<R> *a) {
    cplx<R> b[16];
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) {
        cplx<R> x0 = a[n2], x1 = a[n2 + 4], x2 = a[n2 + 8], x3 = a[n2 + 12];
        dft4<R, SIGN>(x0, x1, x2, x3);
        b[n2 * 4 + 0] = x0;
        b[n2 * 4 + 1] = cmul_wconst<R, SIGN, 16>(x1, n2 * 1);
        b[n2 * 4 + 2] = cmul_wconst<R, SIGN, 16>(x2, n2 * 2);
        b[n2 * 4 + 3] = cmul_wconst<R, SIGN, 16>(x3, n2 * 3);
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++) {
        cplx<R> y0 = b[k1], y1 = b[4 + k1], y2 = b[8 + k1], y3 = b[12 + k1];
        dft4<R, SIGN>(y0, y1, y2, y3);
        a[k1] = y0;
        a[k1 + 4] = y1;
        a[k1 + 8] = y2;
        a[k1 + 12] = y3;
    }
}

// 32-point DFT in registers: two 16-point DFTs of the even and odd elements and a radix-2 combination
template <class R, int SIGN> __device__ __forceinline__ void dft32(cplx<R> *a) {
    cplx<R> e[16], o[16];
#pragma unroll
    for (int k = 0; k < 16; k++) { e[k] = a[2 * k]; o[k] = a[2 * k + 1]; }
    dft16<R, SIGN>(e);
    dft16<R, SIGN>(o);
#pragma unroll
    for (int k = 0; k < 16; k++) {
        cplx<R> w = cmul_wconst<R, SIGN, 32>(o[k], k);
        a[k] = cadd(e[k], w);
        a[k + 16] = csub(e[k], w);
    }
}

template <class R, int RAD, int SIGN> __device__ __forceinline__ void dft_wide(cplx<R> *a) {
    static_assert(RAD == 16 || RAD == 32, "wide radices are 16 and 32");
    if constexpr (RAD == 32) dft32<R, SIGN>(a);
    else dft16<R, SIGN>(a);
}

// The three-stage wide plan of the FP32 rows at 2048, 4096 and 8192: stage A a radix-32 DFT of each thread's
// 32 elements in registers (no twiddles), then two Stockham stages of radix R1 x R2 (8 x 8 at 2048, 16 x 8 at
// 4096, 16 x 16 at 8192) through fft_stages, so a transform makes two shared-memory exchanges where the
// radix-8 plan makes three (four at 8192), with NT = N / 32 threads (2, 4 or 8 warps) a row. Rows of 32 elements are padded by one in shared
// memory (WideRowAddr<32>), which keeps stage A's row writes and the later strided reads conflict-free.
template <class R> __host__ __device__ constexpr bool wide3_plan(int n) {
    return sizeof(R) == 4 && (n == 2048 || n == 4096 || n == 8192);
}
template <int N> struct Wide3Plan {
    static constexpr int E = 32;
    static constexpr int NT = N / E;
    static constexpr int R1 = N == 2048 ? 8 : 16;
    static constexpr int R2 = N / (E * R1);
    static constexpr int nstages = 3;
    __host__ __device__ static constexpr int radix(int s) { return s == 0 ? E : (s == 1 ? R1 : R2); }
    __host__ __device__ static constexpr int ns(int s) { return s == 0 ? 1 : (s == 1 ? E : E * R1); }
    // the packed table (W_{Ns RAD}^(r k) of stage s >= 1 at tw_base(s) + k (RAD - 1) + r - 1, k < Ns)
    __host__ __device__ static constexpr int tw_base(int s) { return s <= 1 ? 0 : E * (R1 - 1); }
    static constexpr int TW = E * (R1 - 1) + E * R1 * (R2 - 1);   // = N - 32
    static constexpr int ROWSZ = NT * (E + 1);                     // padded shared elements of one transform
    static_assert((N != 2048 && N != 4096 && N != 8192) || (E * R1 * R2 == N && E % R1 == 0 && E % R2 == 0),
                  "three-stage wide plan");
};

// The radix-24 plans of the FP32 rows at 3·2^k: stage A a 24-point prime-factor DFT of each thread's 24
// elements in registers (no twiddles), then Stockham stages through fft_stages: 384 = 24·4·4, 768 = 24·8·4,
// 1536 = 24·8·8, 3072 = 24·8·8·2. Two shared-memory exchanges a transform (three at 3072) where the radix-12
// plan makes three (four at 1536, five stages at 3072), with NT = N / 24 threads a row (16, 32, 64, 128). The
// exchanges address element i at i ^ ((i / 24) & 15) (at 384, i ^ ((i >> 3) & 15)): a permutation of
// [0, N) that meets 2 wavefronts, the minimum, for every stage's reads and writes (checked exhaustively on
// the host for the four sizes), with no padding.
template <class R> __host__ __device__ constexpr bool wide24_plan(int n) {
    return sizeof(R) == 4 && (n == 384 || n == 768 || n == 1536 || n == 3072);
}
template <int N> struct Wide24Plan {
    static constexpr int E = 24;
    static constexpr int NT = N / E;
    static constexpr int nstages = N == 3072 ? 4 : 3;
    __host__ __device__ static constexpr int radix(int s) {
        return s == 0 ? 24 : (N == 384 ? 4 : (N == 768 ? (s == 1 ? 8 : 4) : (s <= 2 ? 8 : 2)));
    }
    __host__ __device__ static constexpr int ns(int s) { return s == 0 ? 1 : ns(s - 1) * radix(s - 1); }
    // the packed table (W_{Ns RAD}^(r k) of stage s >= 1 at tw_base(s) + k (RAD - 1) + r - 1, k < Ns)
    __host__ __device__ static constexpr int tw_base(int s) { return s <= 1 ? 0 : tw_base(s - 1) + ns(s - 1) * (radix(s - 1) - 1); }
    static constexpr int TW = tw_base(nstages);
    static constexpr int ROWSZ = N;   // shared elements of one transform (swizzled, unpadded)
};
template <int N> struct Wide24Addr {
    __device__ __forceinline__ int operator()(int i) const { return N == 384 ? i ^ ((i >> 3) & 15) : i ^ ((i / 24) & 15); }
};

// threads of one transform within one warp (row tiles of the wide plan)
struct WarpSync {
    __device__ __forceinline__ void operator()() const { __syncwarp(); }
};

// SIGN -1 forward, +1 inverse, unnormalised; sm: this transform's shared memory, ad its addressing
template <class R, int N, int SIGN, class Addr, class Sync>
__device__ __forceinline__ void fft_wide(cplx<R> (&v)[WidePlan<N>::E], cplx<R> *sm, Addr ad, int t, const cplx<R> *tw,
                                         Sync sync) {
    using P = WidePlan<N>;
    constexpr int E = P::E, NT = P::NT, R2 = P::R2, NB = P::NB;
    dft_wide<R, E, SIGN>(v);   // stage A (no twiddles)
    sync();                    // the previous transform's reads of sm are done
#pragma unroll
    for (int m = 0; m < E; m++) sm[ad(t * E + m)] = v[m];
    sync();
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * NT;   // butterfly index, < E
        cplx<R> a[R2];
#pragma unroll
        for (int r = 0; r < R2; r++) {
            cplx<R> x = sm[ad(j + r * E)];
            if (r > 0) {
                const cplx<R> w = tw[j * (R2 - 1) + (r - 1)];
                x = (SIGN < 0) ? cmul(x, w) : cmulc(x, w);
            }
            a[r] = x;
        }
        dft_wide<R, R2, SIGN>(a);
#pragma unroll
        for (int m = 0; m < R2; m++) v[b + m * NB] = a[m];
    }
}

}  // namespace ms
