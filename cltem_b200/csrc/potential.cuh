// potential.cuh — slice transmission functions from binned atoms.
//
// One 16x16 thread block per 16x16 pixel tile and one grid z-layer per slice. The bin ranges a tile
// reads are the reference's (transmission_potentials_projected_d.cl:227-246), so the set of atoms each
// pixel sums is identical; the atoms of a bin row are staged through shared memory in chunks of 256
// (the reference's single 256-atom __local load overflows for longer rows, :264-268; chunking keeps
// every atom). T = cos(sigma V) + i sin(sigma V).
//
// FP64 instantiation: the reference's _d statements in the same order (this translation unit is built
// with -fmad=false). FP32 instantiation: pixel-to-atom offsets in FP64, the potential sum in FP32.
#pragma once

#include "common.cuh"

namespace ms {

struct PotParams {
    int width, height, total_slices, slice0;
    double dz, pixelscale;
    int blocks_x, blocks_y;
    double max_x, min_x, max_y, min_y;
    int load_x, load_y, load_z;
    double sigma, startx, starty;
    double beam_theta_mrad, beam_phi;   // projected: tilt
    double z0;                          // full 3-D: padded z minimum; current_z = z0 + (S - k) dz
    double shift_x, shift_y;            // full 3-D: per-sub-slice tilt shift
    int integrals;
    int form, i_count;
};

__constant__ double c_k0pi[5] = {1.0, 2.346487949187396e-1, 1.187082088663404e-2, 2.150707366040937e-4, 1.425433617130587e-6};
__constant__ double c_k0qi[3] = {9.847324170755358e-1, 1.518396076767770e-2, 8.362215678646257e-5};
__constant__ double c_k0p[5] = {1.159315156584126e-1, 2.770731240515333e-1, 2.066458134619875e-2, 4.574734709978264e-4, 3.454715527986737e-6};
__constant__ double c_k0q[3] = {9.836249671709183e-1, 1.627693622304549e-2, 9.809660603621949e-5};
__constant__ double c_k0pp[8] = {1.253314137315499, 1.475731032429900e1, 6.123767403223466e1, 1.121012633939949e2,
                                 9.285288485892228e1, 3.198289277679660e1, 3.595376024148513, 6.160228690102976e-2};
__constant__ double c_k0qq[8] = {1.0, 1.189963006673403e1, 5.027773590829784e1, 9.496513373427093e1,
                                 8.318077493230258e1, 3.181399777449301e1, 4.443672926432041, 1.408295601966600e-1};
__constant__ double c_k1pi[5] = {0.5, 5.598072040178741e-2, 1.818666382168295e-3, 2.397509908859959e-5, 1.239567816344855e-7};
__constant__ double c_k1qi[3] = {9.870202601341150e-1, 1.292092053534579e-2, 5.881933053917096e-5};
__constant__ double c_k1p[5] = {-3.079657578292062e-1, -8.109417631822442e-2, -3.477550948593604e-3, -5.385594871975406e-5, -3.110372465429008e-7};
__constant__ double c_k1q[3] = {9.861813171751389e-1, 1.375094061153160e-2, 6.774221332947002e-5};
__constant__ double c_k1pp[8] = {1.253314137315502, 1.457171340220454e1, 6.063161173098803e1, 1.147386690867892e2,
                                 1.040442011439181e2, 4.356596656837691e1, 7.265230396353690, 3.144418558991021e-1};
__constant__ double c_k1qq[8] = {1.0, 1.125154514806458e1, 4.427488496597630e1, 7.616113213117645e1,
                                 5.863377227890893e1, 1.850303673841586e1, 1.857244676566022, 2.538540887654872e-2};

template <class T> __device__ __forceinline__ T dpoly(const double *cof, int n, T x) {
    T ans = (T)cof[n];
    for (int i = n - 1; i >= 0; --i) ans = ans * x + (T)cof[i];
    return ans;
}
__device__ __forceinline__ float flog(float x) { return logf(x); }
__device__ __forceinline__ double flog(double x) { return log(x); }
__device__ __forceinline__ float fexp(float x) { return expf(x); }
__device__ __forceinline__ double fexp(double x) { return exp(x); }
__device__ __forceinline__ float fsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double fsqrt(double x) { return sqrt(x); }

// Modified Bessel functions K0 / K1: Numerical Recipes in C 2nd ed. section 6.6 rational
// approximations with the coefficients the reference uses (projected_d.cl:57-102).
template <class T> __device__ __forceinline__ T bessk0(T x) {
    T ax = fabs(x);
    if (ax > (T)0 && ax <= (T)1) {
        T z = x * x;
        T term = dpoly<T>(c_k0pi, 4, z) * flog(x) * ((T)1 / dpoly<T>(c_k0qi, 2, (T)1 - z));
        return dpoly<T>(c_k0p, 4, z) * ((T)1 / dpoly<T>(c_k0q, 2, (T)1 - z)) - term;
    } else if (ax > (T)1) {
        T z = (T)1 / x;
        return fexp(-x) * dpoly<T>(c_k0pp, 7, z) * ((T)1 / dpoly<T>(c_k0qq, 7, z)) * ((T)1 / fsqrt(x));
    }
    return (T)1.79769313486231570815e+308;
}
template <class T> __device__ __forceinline__ T bessk1(T x) {
    T ax = fabs(x);
    if (ax > (T)0 && ax <= (T)1) {
        T z = x * x;
        T term = dpoly<T>(c_k1pi, 4, z) * flog(x) * ((T)1 / dpoly<T>(c_k1qi, 2, (T)1 - z));
        return x * (dpoly<T>(c_k1p, 4, z) * ((T)1 / dpoly<T>(c_k1q, 2, (T)1 - z)) + term) + (T)1 / x;
    } else if (ax > (T)1) {
        T z = (T)1 / x;
        return fexp(-x) * dpoly<T>(c_k1pp, 7, z) * ((T)1 / dpoly<T>(c_k1qq, 7, z)) * ((T)1 / fsqrt(x));
    }
    return (T)1.79769313486231570815e+308;
}

// Projected potentials (projected_d.cl:104-181): Kirkland eq. C.20, Peng (integrated), Lobato eq. 16.
template <class T> __device__ __forceinline__ T kirkland_p(const T *__restrict__ prm, int i_lim, int Z, T rad) {
    T suml = 0, sumg = 0;
    const T *p = prm + (Z - 1) * 12;
    T x = (T)(2.0 * M_PI) * rad;
    for (int i = 0; i < i_lim * 2; i += 2) suml += p[i] * bessk0<T>(x * fsqrt(p[i + 1]));
    x = (T)M_PI * rad;
    x = x * x;
    for (int i = i_lim * 2; i < i_lim * 4; i += 2) {
        T d_inv = (T)1 / p[i + 1];
        sumg += (p[i] * d_inv) * fexp(-x * d_inv);
    }
    return (T)300.8242834 * suml + (T)150.4121417 * sumg;
}
template <class T> __device__ __forceinline__ T lobato_p(const T *__restrict__ prm, int i_lim, int Z, T rad) {
    T sum = 0;
    const T *p = prm + (Z - 1) * 10;
    T x = (T)(2.0 * M_PI) * rad;
    for (int i = 0; i < i_lim; ++i) {
        T b_inv_root = (T)1 / fsqrt(p[i + 5]);
        sum += p[i] * (b_inv_root * b_inv_root * b_inv_root) * (bessk0<T>(x * b_inv_root) + rad * bessk1<T>(x * b_inv_root));
    }
    return (T)945.090144399935 * sum;
}
template <class T> __device__ __forceinline__ T peng_p(const T *__restrict__ prm, int i_lim, int Z, T rad) {
    T sum = 0;
    const T *p = prm + (Z - 1) * 10;
    T x = (T)M_PI * rad;
    x = x * x;
    for (int i = 0; i < i_lim; ++i) {
        T b_inv = (T)1 / p[i + 5];
        sum += p[i] * b_inv * fexp(-x * b_inv);
    }
    return (T)150.4121417 * sum;
}
// Full 3-D potentials (full_3d_d.cl:57-134): Kirkland eq. C.19, Peng, Lobato.
template <class T> __device__ __forceinline__ T kirkland_3(const T *__restrict__ prm, int i_lim, int Z, T rad) {
    T suml = 0, sumg = 0;
    const T *p = prm + (Z - 1) * 12;
    T x = (T)(2.0 * M_PI) * rad;
    for (int i = 0; i < i_lim * 2; i += 2) suml += p[i] * fexp(-x * fsqrt(p[i + 1]));
    x = (T)M_PI * rad;
    x = x * x;
    for (int i = i_lim * 2; i < i_lim * 4; i += 2) {
        T d_inv_root = (T)1 / fsqrt(p[i + 1]);
        sumg += p[i] * (d_inv_root * d_inv_root * d_inv_root) * fexp(-x * ((T)1 / p[i + 1]));
    }
    return (T)150.4121417 * ((T)1 / rad) * suml + (T)266.5157269 * sumg;
}
template <class T> __device__ __forceinline__ T lobato_3(const T *__restrict__ prm, int i_lim, int Z, T rad) {
    T sum = 0;
    const T *p = prm + (Z - 1) * 10;
    T x = (T)M_PI * rad;
    for (int i = 0; i < i_lim; ++i) {
        T b = p[i + 5];
        T b_inv_root = (T)1 / fsqrt(b);
        sum += p[i] * (b_inv_root * b_inv_root * b_inv_root) * fexp((T)-2.0 * x * b_inv_root) * (fsqrt(b) * ((T)1 / x) + (T)1);
    }
    return (T)472.545072199968 * sum;
}
template <class T> __device__ __forceinline__ T peng_3(const T *__restrict__ prm, int i_lim, int Z, T rad) {
    T sum = 0;
    const T *p = prm + (Z - 1) * 10;
    T x = (T)M_PI * rad;
    x = x * x;
    for (int i = 0; i < i_lim; ++i) {
        T b = p[i + 5];
        T b_inv_root = (T)1 / fsqrt(b);
        sum += p[i] * (b_inv_root * b_inv_root * b_inv_root) * fexp(-x * ((T)1 / b));
    }
    return (T)266.5157269 * sum;
}

// Bin range of a 16x16 tile, in FP64 exactly as the reference (projected_d.cl:227-246)
__device__ __forceinline__ void tile_bins(const PotParams &p, int gx, int gy, int &si, int &ei, int &sj, int &ej) {
    double group_size_x = 16 * p.pixelscale, group_size_y = 16 * p.pixelscale;
    double group_start_x = p.startx + gx * group_size_x;
    double group_end_x = group_start_x + group_size_x;
    double group_start_y = p.starty + gy * group_size_y;
    double group_end_y = group_start_y + group_size_y;
    double recip_range_x = 1.0 / (p.max_x - p.min_x);
    double recip_range_y = 1.0 / (p.max_y - p.min_y);
    si = (int)fmax(floor(p.blocks_x * (group_start_x - p.min_x) * recip_range_x) - p.load_x, 0.0);
    ei = (int)fmin(ceil(p.blocks_x * (group_end_x - p.min_x) * recip_range_x) + p.load_x, (double)(p.blocks_x - 1));
    sj = (int)fmax(floor(p.blocks_y * (group_start_y - p.min_y) * recip_range_y) - p.load_y, 0.0);
    ej = (int)fmin(ceil(p.blocks_y * (group_end_y - p.min_y) * recip_range_y) + p.load_y, (double)(p.blocks_y - 1));
}

template <class T> __device__ __forceinline__ void write_trans(cplx<T> *o, T phase);
template <> __device__ __forceinline__ void write_trans<float>(float2 *o, float phase) {
    float s, c;
    sincosf(phase, &s, &c);
    *o = make_float2(c, s);
}
template <> __device__ __forceinline__ void write_trans<double>(double2 *o, double phase) {
    *o = make_double2(cos(phase), sin(phase));
}

constexpr int kAtomChunk = 256;

// transmission_potentials_projected: grid (W/16, H/16, n_slices), block (16, 16)
template <class T, int FORM>
__global__ void __launch_bounds__(256)
k_potential_projected(cplx<T> *__restrict__ out, const double *__restrict__ ax, const double *__restrict__ ay,
                      const int *__restrict__ aZ, const int *__restrict__ block_start, const T *__restrict__ prm,
                      PotParams p) {
    __shared__ double sx[kAtomChunk], sy[kAtomChunk];
    __shared__ int sZ[kAtomChunk];
    const int lid = threadIdx.x + 16 * threadIdx.y;
    const int xid = blockIdx.x * 16 + threadIdx.x, yid = blockIdx.y * 16 + threadIdx.y;
    const int slice = blockIdx.z + p.slice0;
    int si, ei, sj, ej;
    tile_bins(p, blockIdx.x, blockIdx.y, si, ei, sj, ej);
    int k = slice;
    if (k < 0) k = 0;
    if (k >= p.total_slices) k = p.total_slices - 1;
    // tilt geometry, constant per launch (projected_d.cl:221, 283-289)
    const double beam_theta = M_PI_2 - p.beam_theta_mrad * 0.001;
    const double cos_beam_phi = cos(p.beam_phi), sin_beam_phi = sin(p.beam_phi);
    const double sin_beam_2theta = sin(2.0 * beam_theta);
    const double tan_beam_theta = tan(beam_theta);
    const double im_pos_x = p.startx + xid * p.pixelscale;
    const double im_pos_y = p.starty + yid * p.pixelscale;
    const double r_min = 0.25 * p.pixelscale;
    T sumz = 0;
    const size_t nb = (size_t)p.blocks_x * p.blocks_y;
    for (int j = sj; j <= ej; j++) {
        const int start = block_start[k * nb + p.blocks_x * j + si];
        const int end = block_start[k * nb + p.blocks_x * j + ei + 1];
        for (int c0 = start; c0 < end; c0 += kAtomChunk) {
            const int cn = min(kAtomChunk, end - c0);
            __syncthreads();
            if (lid < cn) { sx[lid] = ax[c0 + lid]; sy[lid] = ay[c0 + lid]; sZ[lid] = aZ[c0 + lid]; }
            __syncthreads();
            for (int l = 0; l < cn; l++) {
                double rad_x = im_pos_x - sx[l];
                double rad_y = im_pos_y - sy[l];
                double z_prime = -0.5 * (rad_x * cos_beam_phi + rad_y * sin_beam_phi) * sin_beam_2theta;
                double z_by_tan_beam_theta = z_prime / tan_beam_theta;
                double x_prime = rad_x + z_by_tan_beam_theta * cos_beam_phi;
                double y_prime = rad_y + z_by_tan_beam_theta * sin_beam_phi;
                const double rad2 = z_prime * z_prime + x_prime * x_prime + y_prime * y_prime;
                // sqrt(rad2) <= 8 needs rad2 <= 64 up to one rounding: candidates beyond 64 (1 + 1e-12) skip
                // the square root; the test itself is the reference's (projected_d.cl:290-296)
                if (rad2 > 64.000000000064) continue;
                double rad_d = sqrt(rad2);
                if (rad_d < r_min) rad_d = r_min;
                if (rad_d <= 8.0) {
                    const T rad = (T)rad_d;
                    if constexpr (FORM == 0) sumz += kirkland_p<T>(prm, p.i_count, sZ[l], rad);
                    else if constexpr (FORM == 1) sumz += peng_p<T>(prm, p.i_count, sZ[l], rad);
                    else sumz += lobato_p<T>(prm, p.i_count, sZ[l], rad);
                }
            }
        }
    }
    if (xid < p.width && yid < p.height)
        write_trans<T>(out + (size_t)blockIdx.z * p.width * p.height + (size_t)yid * p.width + xid, (T)p.sigma * sumz);
}

// transmission_potentials_full_3d: grid (W/16, H/16, n_slices), block (16, 16)
template <class T, int FORM>
__global__ void __launch_bounds__(256)
k_potential_3d(cplx<T> *__restrict__ out, const double *__restrict__ ax, const double *__restrict__ ay,
               const double *__restrict__ az, const int *__restrict__ aZ, const int *__restrict__ block_start,
               const T *__restrict__ prm, PotParams p) {
    __shared__ double sx[kAtomChunk], sy[kAtomChunk], sz[kAtomChunk];
    __shared__ int sZ[kAtomChunk];
    const int lid = threadIdx.x + 16 * threadIdx.y;
    const int xid = blockIdx.x * 16 + threadIdx.x, yid = blockIdx.y * 16 + threadIdx.y;
    const int slice = blockIdx.z + p.slice0;
    int si, ei, sj, ej;
    tile_bins(p, blockIdx.x, blockIdx.y, si, ei, sj, ej);
    int topz = slice - p.load_z, bottomz = slice + p.load_z;
    const double int_r = 1.0 / p.integrals;
    const double sub_slice_thickness = p.dz * int_r;
    if (topz < 0) topz = 0;
    if (bottomz >= p.total_slices) bottomz = p.total_slices - 1;
    const double current_z = p.z0 + (p.total_slices - slice) * p.dz;   // simulationgeneral.cpp:590
    const double im_pos_x = p.startx + xid * p.pixelscale;
    const double im_pos_y = p.starty + yid * p.pixelscale;
    const double r_min = 0.25 * p.pixelscale;
    const bool no_shift = p.shift_x == 0.0 && p.shift_y == 0.0;
    T sumz = 0;
    const size_t nb = (size_t)p.blocks_x * p.blocks_y;
    for (int k = topz; k <= bottomz; k++) {
        for (int j = sj; j <= ej; j++) {
            const int start = block_start[k * nb + p.blocks_x * j + si];
            const int end = block_start[k * nb + p.blocks_x * j + ei + 1];
            T p2 = 0;
            for (int c0 = start; c0 < end; c0 += kAtomChunk) {
                const int cn = min(kAtomChunk, end - c0);
                __syncthreads();
                if (lid < cn) { sx[lid] = ax[c0 + lid]; sy[lid] = ay[c0 + lid]; sz[lid] = az[c0 + lid]; sZ[lid] = aZ[c0 + lid]; }
                __syncthreads();
                for (int l = 0; l < cn; l++) {
                    double rad_x = im_pos_x - sx[l];
                    double rad_y = im_pos_y - sy[l];
                    // without tilt the shift is zero and the xy test is the same for every sample: an atom
                    // beyond 8 Å adds nothing and changes no trapezoid state, so it is skipped whole
                    const double xy0 = rad_x * rad_x + rad_y * rad_y;
                    if (no_shift && xy0 > 64.0) continue;
                    for (int h = 0; h <= p.integrals; h++) {
                        rad_x -= p.shift_x;   // cumulative (full_3d_d.cl:244-246)
                        rad_y -= p.shift_y;
                        double xyrad2 = no_shift ? xy0 : rad_x * rad_x + rad_y * rad_y;
                        double im_pos_z = current_z - h * p.dz * int_r;
                        double rad_z = im_pos_z - sz[l];
                        if (xyrad2 <= 64.0 && rad_z <= 3.0) {
                            // the distance is only used by samples that pass the test: taken here instead
                            // of for every candidate (same value as full_3d_d.cl:258-261)
                            double rad_d = sqrt(xyrad2 + rad_z * rad_z);
                            if (rad_d < r_min) rad_d = r_min;
                            const T rad = (T)rad_d;
                            T p1;
                            if constexpr (FORM == 0) p1 = kirkland_3<T>(prm, p.i_count, sZ[l], rad);
                            else if constexpr (FORM == 1) p1 = peng_3<T>(prm, p.i_count, sZ[l], rad);
                            else p1 = lobato_3<T>(prm, p.i_count, sZ[l], rad);
                            sumz += (h != 0) * (p1 + p2) * (T)0.5;
                            p2 = p1;
                        }
                    }
                }
            }
        }
    }
    if (xid < p.width && yid < p.height)
        write_trans<T>(out + (size_t)blockIdx.z * p.width * p.height + (size_t)yid * p.width + xid,
                       (T)(sub_slice_thickness * p.sigma) * sumz);
}

// ---- FP32 full 3-D potentials -------------------------------------------------------------------
// The FP32 engine's full-3D build is bound by instruction issue. This kernel makes the same geometric
// decisions as k_potential_3d:
// - the same FP64 offsets and FP64 tests (8 Å in xy, the one-sided 3 Å in z);
// - the same atom and sample order;
// - the same trapezoid pairing.
// It cuts the instructions per sample:
// - Each thread computes kPot3Px pixels of its tile row. The atom loads, the per-atom table reads and the
//   FP64 z tests are shared by its pixels.
// - The squared distance is rounded once to FP32; one rsqrtf gives both the distance and its reciprocal.
// - Each form is a sum of exponentials whose per-element constants come from a table built on the host
//   in FP64 and rounded once (pot3_table). A thread reads an atom's terms once into registers, and takes
//   exp as ex2.approx.ftz.f32 (relative error below 2^-22) of a pre-scaled exponent.
// - The atoms of all bin rows a tile reads are staged through shared memory as one list, instead of one
//   load (and two barriers) per bin row. A flag on the first atom of each bin row resets the trapezoid's
//   previous sample there, as the reference's per-row `p2 = 0` does (full_3d_d.cl:238).
// Table, per element Z and term i, float4 at (Z - 1) * kPot3Terms + i (terms beyond the parameterisation's
// count are zero):
// - Lobato (full_3d_d.cl:102-118), i < 5: (472.545·a·b^-3/2, -2π·log2(e)/√b, √b/π, 0);
//   term = x·exp2(y·r)·(z/r + 1).
// - Peng, i < 5: (266.516·a·b^-3/2, 0, 0, -π²·log2(e)/b); term = x·exp2(w·r²).
// - Kirkland, Lorentzian terms i < 3: (150.412·a, -2π·log2(e)·√b, 0, 0); the term x·exp2(y·r)/r.
//   Gaussian terms i = 3 + j: (266.516·c·d^-3/2, 0, 0, -π²·log2(e)/d); the term x·exp2(w·r²).
constexpr int kPot3Terms = 6;
constexpr int kPot3Rows = 64;            // bin rows staged per pass of the row list
constexpr int kPot3First = 1 << 30;     // flag on the first atom of a bin row in the staged Z

// 2^x by the special-function unit (hand-written PTX; flushes subnormal results to zero)
__device__ __forceinline__ float ex2a(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// terms of each kind per element: Kirkland 3 Lorentzian + 3 Gaussian, Peng / Lobato 5
template <int FORM> struct Pot3N {
    static constexpr int L = FORM == 0 ? 3 : 5;
    static constexpr int G = FORM == 0 ? 3 : 0;
};
template <int FORM>
__device__ __forceinline__ float pot3_eval_r(const float4 (&c)[Pot3N<FORM>::L + Pot3N<FORM>::G], float rad, float inv) {
    if constexpr (FORM == 2) {
        float sum = 0.0f;
#pragma unroll
        for (int i = 0; i < 5; i++) sum += c[i].x * ex2a(c[i].y * rad) * fmaf(c[i].z, inv, 1.0f);
        return sum;
    } else if constexpr (FORM == 1) {
        const float r2 = rad * rad;
        float sum = 0.0f;
#pragma unroll
        for (int i = 0; i < 5; i++) sum += c[i].x * ex2a(c[i].w * r2);
        return sum;
    } else {
        const float r2 = rad * rad;
        float suml = 0.0f, sumg = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; i++) suml += c[i].x * ex2a(c[i].y * rad);
#pragma unroll
        for (int i = 0; i < 3; i++) sumg += c[3 + i].x * ex2a(c[3 + i].w * r2);
        return suml * inv + sumg;
    }
}

// Pixels a thread computes in the FP32 full-3D kernel (x, x + 16/PX, ... of its tile row)
#ifndef MS_POT3_PX
#define MS_POT3_PX 4
#endif
constexpr int kPot3Px = MS_POT3_PX;

// grid (W/16, H/16, n_slices), block (16/PX, 16): each thread the pixels x + m·16/PX, m < PX, of its tile row
template <int FORM, int PX>
__global__ void __launch_bounds__(256 / PX)
k_potential_3d_f(float2 *__restrict__ out, const double *__restrict__ ax, const double *__restrict__ ay,
                 const double *__restrict__ az, const int *__restrict__ aZ, const int *__restrict__ block_start,
                 const float4 *__restrict__ tab, PotParams p) {
    constexpr int NTERM = Pot3N<FORM>::L + Pot3N<FORM>::G;
    constexpr int TX = 16 / PX, NTH = 256 / PX;
    __shared__ double sx[kAtomChunk], sy[kAtomChunk], sz[kAtomChunk];
    __shared__ int sZ[kAtomChunk];
    __shared__ int row_start[kPot3Rows], row_off[kPot3Rows + 1];
    const int lid = threadIdx.x + TX * threadIdx.y;
    const int xid0 = blockIdx.x * 16 + threadIdx.x, yid = blockIdx.y * 16 + threadIdx.y;
    const int slice = blockIdx.z + p.slice0;
    int si, ei, sj, ej;
    tile_bins(p, blockIdx.x, blockIdx.y, si, ei, sj, ej);
    int topz = slice - p.load_z, bottomz = slice + p.load_z;
    const double int_r = 1.0 / p.integrals;
    const double sub_slice_thickness = p.dz * int_r;
    if (topz < 0) topz = 0;
    if (bottomz >= p.total_slices) bottomz = p.total_slices - 1;
    const double current_z = p.z0 + (p.total_slices - slice) * p.dz;
    double pos_x[PX];
#pragma unroll
    for (int m = 0; m < PX; m++) pos_x[m] = p.startx + (xid0 + m * TX) * p.pixelscale;
    const double im_pos_y = p.starty + yid * p.pixelscale;
    const float r_min = (float)(0.25 * p.pixelscale);
    const float inv_r_min = 1.0f / r_min;
    const bool no_shift = p.shift_x == 0.0 && p.shift_y == 0.0;
    const size_t nb = (size_t)p.blocks_x * p.blocks_y;
    const int nj = ej - sj + 1;
    const int n_rows = (bottomz >= topz && nj > 0) ? (bottomz - topz + 1) * nj : 0;
    float sum[PX], q[PX];
#pragma unroll
    for (int m = 0; m < PX; m++) { sum[m] = 0.0f; q[m] = 0.0f; }
    for (int r0 = 0; r0 < n_rows; r0 += kPot3Rows) {
        const int nr = min(kPot3Rows, n_rows - r0);
        __syncthreads();   // the previous pass's readers of the row tables and the chunk are done
        if (lid < nr) {
            const int r = r0 + lid, k = topz + r / nj, j = sj + r % nj;
            const int start = block_start[k * nb + p.blocks_x * j + si];
            row_start[lid] = start;
            row_off[lid + 1] = block_start[k * nb + p.blocks_x * j + ei + 1] - start;   // count, summed below
        }
        __syncthreads();
        if (lid == 0) {
            row_off[0] = 0;
            for (int r = 0; r < nr; r++) row_off[r + 1] += row_off[r];
        }
        __syncthreads();
        const int total = row_off[nr];
        for (int c0 = 0; c0 < total; c0 += kAtomChunk) {
            const int cn = min(kAtomChunk, total - c0);
            __syncthreads();
            for (int w = lid; w < cn; w += NTH) {
                const int f = c0 + w;
                int lo = 0, hi = nr - 1;   // the last row whose offset is <= f (a non-empty row holds f)
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (row_off[mid] <= f) lo = mid;
                    else hi = mid - 1;
                }
                const int a = row_start[lo] + (f - row_off[lo]);
                sx[w] = ax[a]; sy[w] = ay[a]; sz[w] = az[a];
                sZ[w] = aZ[a] | (f == row_off[lo] ? kPot3First : 0);
            }
            __syncthreads();
            for (int l = 0; l < cn; l++) {
                const int zf = sZ[l];
                if (zf & kPot3First) {   // a new bin row
#pragma unroll
                    for (int m = 0; m < PX; m++) q[m] = 0.0f;
                }
                const double xl = sx[l];
                const double ry = im_pos_y - sy[l];
                const double yy = ry * ry;
                double rx[PX], xy0[PX];
                bool in[PX], any = false;
#pragma unroll
                for (int m = 0; m < PX; m++) {
                    rx[m] = pos_x[m] - xl;
                    xy0[m] = rx[m] * rx[m] + yy;
                    // without tilt the xy test is the same for every sample: beyond 8 Å the atom adds nothing
                    in[m] = !(no_shift && xy0[m] > 64.0);
                    any = any || in[m];
                }
                if (!any) continue;
                const int Z = zf & (kPot3First - 1);
                float4 c[NTERM];
                const float4 *t = tab + (Z - 1) * kPot3Terms;
#pragma unroll
                for (int i = 0; i < NTERM; i++) c[i] = __ldg(t + i);
                const double zl = sz[l];
                double ry_s = ry;
                for (int h = 0; h <= p.integrals; h++) {
#pragma unroll
                    for (int m = 0; m < PX; m++) rx[m] -= p.shift_x;   // cumulative (full_3d_d.cl:244-246)
                    ry_s -= p.shift_y;
                    const double rad_z = (current_z - h * p.dz * int_r) - zl;
                    if (rad_z <= 3.0) {
                        const double yys = no_shift ? yy : ry_s * ry_s;
                        const double zz = rad_z * rad_z;
#pragma unroll
                        for (int m = 0; m < PX; m++) {
                            const double xyr = no_shift ? xy0[m] : rx[m] * rx[m] + yys;
                            if (in[m] && xyr <= 64.0) {
                                const float r2f = (float)(xyr + zz);
                                float inv = rsqrtf(r2f), rad = r2f * inv;
                                if (!(rad >= r_min)) { rad = r_min; inv = inv_r_min; }   // also r2f = 0 (NaN)
                                const float p1 = pot3_eval_r<FORM>(c, rad, inv);
                                sum[m] += (h != 0) * (p1 + q[m]) * 0.5f;
                                q[m] = p1;
                            }
                        }
                    }
                }
            }
        }
    }
    const float sc = (float)(sub_slice_thickness * p.sigma);
    if (yid < p.height) {
        float2 *o = out + (size_t)blockIdx.z * p.width * p.height + (size_t)yid * p.width;
#pragma unroll
        for (int m = 0; m < PX; m++)
            if (xid0 + m * TX < p.width) write_trans<float>(o + xid0 + m * TX, sc * sum[m]);
    }
}

// ---- FP32 projected potentials ---------------------------------------------------------------------
// K0 / K1 by the same rational approximations as bessk0 / bessk1 (projected_d.cl:57-102), in FP32: the
// coefficients are the FP64 ones rounded to float at compile time (bessk0<float> rounds them at run
// time). exp is ex2.approx.ftz and log __logf (absolute error near 2^-21 on (0, 1], where the log term
// stays below the rational part); each branch's quotients share one __fdividef, and for x > 1 one rsqrtf
// gives both 1/sqrt(x) and 1/x. Errors of a few ulp of the result.
template <class... C> __device__ __forceinline__ float hornerf(float, float c0) { return c0; }
template <class... C> __device__ __forceinline__ float hornerf(float x, float c0, C... c) {
    return fmaf(hornerf(x, c...), x, c0);   // c0 + x (c1 + x (c2 + ...))
}
#define F(v) ((float)(v))
__device__ __forceinline__ float k0f(float x) {
    if (x <= 1.0f) {   // (P2 Q1 - P1 log(x) Q2) / (Q1 Q2): one reciprocal for the two quotients
        const float z = x * x, w = 1.0f - z;
        const float p1 = hornerf(z, F(1.0), F(2.346487949187396e-1), F(1.187082088663404e-2),
                                 F(2.150707366040937e-4), F(1.425433617130587e-6));
        const float q1 = hornerf(w, F(9.847324170755358e-1), F(1.518396076767770e-2), F(8.362215678646257e-5));
        const float p2 = hornerf(z, F(1.159315156584126e-1), F(2.770731240515333e-1), F(2.066458134619875e-2),
                                 F(4.574734709978264e-4), F(3.454715527986737e-6));
        const float q2 = hornerf(w, F(9.836249671709183e-1), F(1.627693622304549e-2), F(9.809660603621949e-5));
        return __fdividef(p2 * q1 - p1 * __logf(x) * q2, q1 * q2);
    }
    const float rs = rsqrtf(x), z = rs * rs;   // 1/sqrt(x) and 1/x from one reciprocal square root
    const float p = hornerf(z, F(1.253314137315499), F(1.475731032429900e1), F(6.123767403223466e1),
                            F(1.121012633939949e2), F(9.285288485892228e1), F(3.198289277679660e1),
                            F(3.595376024148513), F(6.160228690102976e-2));
    const float q = hornerf(z, F(1.0), F(1.189963006673403e1), F(5.027773590829784e1), F(9.496513373427093e1),
                            F(8.318077493230258e1), F(3.181399777449301e1), F(4.443672926432041),
                            F(1.408295601966600e-1));
    return ex2a(-1.44269504088896341f * x) * __fdividef(p * rs, q);
}
__device__ __forceinline__ float k1f(float x) {
    if (x <= 1.0f) {   // (x^2 (P2 Q1 + P1 log(x) Q2) + Q1 Q2) / (x Q1 Q2): one reciprocal
        const float z = x * x, w = 1.0f - z;
        const float p1 = hornerf(z, F(0.5), F(5.598072040178741e-2), F(1.818666382168295e-3),
                                 F(2.397509908859959e-5), F(1.239567816344855e-7));
        const float q1 = hornerf(w, F(9.870202601341150e-1), F(1.292092053534579e-2), F(5.881933053917096e-5));
        const float p2 = hornerf(z, F(-3.079657578292062e-1), F(-8.109417631822442e-2), F(-3.477550948593604e-3),
                                 F(-5.385594871975406e-5), F(-3.110372465429008e-7));
        const float q2 = hornerf(w, F(9.861813171751389e-1), F(1.375094061153160e-2), F(6.774221332947002e-5));
        const float qq = q1 * q2;
        return __fdividef(z * (p2 * q1 + p1 * __logf(x) * q2) + qq, x * qq);
    }
    const float rs = rsqrtf(x), z = rs * rs;
    const float p = hornerf(z, F(1.253314137315502), F(1.457171340220454e1), F(6.063161173098803e1),
                            F(1.147386690867892e2), F(1.040442011439181e2), F(4.356596656837691e1),
                            F(7.265230396353690), F(3.144418558991021e-1));
    const float q = hornerf(z, F(1.0), F(1.125154514806458e1), F(4.427488496597630e1), F(7.616113213117645e1),
                            F(5.863377227890893e1), F(1.850303673841586e1), F(1.857244676566022),
                            F(2.538540887654872e-2));
    return ex2a(-1.44269504088896341f * x) * __fdividef(p * rs, q);
}
#undef F

// Table of the FP32 projected kernel, per element Z and term i, float2 at (Z - 1) * kPotPTerms + i (terms
// beyond the parameterisation's count are zero; projected_d.cl:104-181):
// - Kirkland, i < 3: (300.824·a, 2π√b), the term x·K0(y·r); i = 3 + j: (150.412·c/d, -π²·log2(e)/d), the
//   term x·exp2(y·r²).
// - Lobato, i < 5: (945.090·a·b^-3/2, 2π/√b), the term x·(K0(y·r) + r·K1(y·r)).
// - Peng, i < 5: (150.412·a/b, -π²·log2(e)/b), the term x·exp2(y·r²).
constexpr int kPotPTerms = 6;
#ifndef MS_POTP_PX
#define MS_POTP_PX 4
#endif
constexpr int kPotPPx = MS_POTP_PX;   // pixels a thread in the FP32 projected kernel

template <int FORM>
__device__ __forceinline__ float potp_eval(const float2 (&c)[FORM == 0 ? 6 : 5], float rad) {
    if constexpr (FORM == 0) {
        const float r2 = rad * rad;
        float suml = 0.0f, sumg = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; i++) suml += c[i].x * k0f(c[i].y * rad);
#pragma unroll
        for (int i = 0; i < 3; i++) sumg += c[3 + i].x * ex2a(c[3 + i].y * r2);
        return suml + sumg;
    } else if constexpr (FORM == 1) {
        const float r2 = rad * rad;
        float sum = 0.0f;
#pragma unroll
        for (int i = 0; i < 5; i++) sum += c[i].x * ex2a(c[i].y * r2);
        return sum;
    } else {
        float sum = 0.0f;
#pragma unroll
        for (int i = 0; i < 5; i++) {
            const float x = c[i].y * rad;
            sum += c[i].x * (k0f(x) + rad * k1f(x));
        }
        return sum;
    }
}

// The FP32 projected potential: the bins, atoms and 8 Å test of k_potential_projected, with
// - PX pixels a thread (x + m·16/PX of its tile row), sharing the atom loads and the per-atom table reads;
// - the tilt geometry in FP64 with z' / tan θ taken as z' · (1 / tan θ), and without tilt (θ = 0) the plain
//   distance, which the tilt terms change by under 1e-32 Å² there;
// - the form from the per-element table and the FP32 Bessel functions above.
// grid (W/16, H/16, n_slices), block (16/PX, 16)
template <int FORM, int PX>
__global__ void __launch_bounds__(256 / PX)
k_potential_projected_f(float2 *__restrict__ out, const double *__restrict__ ax, const double *__restrict__ ay,
                        const int *__restrict__ aZ, const int *__restrict__ block_start, const float2 *__restrict__ tab,
                        PotParams p) {
    constexpr int NTERM = FORM == 0 ? 6 : 5;
    constexpr int TX = 16 / PX, NTH = 256 / PX;
    __shared__ double sx[kAtomChunk], sy[kAtomChunk];
    __shared__ int sZ[kAtomChunk];
    __shared__ int row_start[kPot3Rows], row_off[kPot3Rows + 1];
    const int lid = threadIdx.x + TX * threadIdx.y;
    const int xid0 = blockIdx.x * 16 + threadIdx.x, yid = blockIdx.y * 16 + threadIdx.y;
    const int slice = blockIdx.z + p.slice0;
    int si, ei, sj, ej;
    tile_bins(p, blockIdx.x, blockIdx.y, si, ei, sj, ej);
    int k = slice;
    if (k < 0) k = 0;
    if (k >= p.total_slices) k = p.total_slices - 1;
    const bool tilt = p.beam_theta_mrad != 0.0;
    const double beam_theta = M_PI_2 - p.beam_theta_mrad * 0.001;
    const double cos_beam_phi = cos(p.beam_phi), sin_beam_phi = sin(p.beam_phi);
    const double sin_beam_2theta = sin(2.0 * beam_theta);
    const double inv_tan_beam_theta = 1.0 / tan(beam_theta);
    double pos_x[PX];
#pragma unroll
    for (int m = 0; m < PX; m++) pos_x[m] = p.startx + (xid0 + m * TX) * p.pixelscale;
    const double im_pos_y = p.starty + yid * p.pixelscale;
    const float r_min = (float)(0.25 * p.pixelscale);
    float sum[PX];
#pragma unroll
    for (int m = 0; m < PX; m++) sum[m] = 0.0f;
    const size_t nb = (size_t)p.blocks_x * p.blocks_y;
    const int n_rows = ej - sj + 1;
    for (int r0 = 0; r0 < n_rows; r0 += kPot3Rows) {
        const int nr = min(kPot3Rows, n_rows - r0);
        __syncthreads();   // the previous pass's readers of the row tables and the chunk are done
        if (lid < nr) {
            const int j = sj + r0 + lid;
            const int start = block_start[k * nb + p.blocks_x * j + si];
            row_start[lid] = start;
            row_off[lid + 1] = block_start[k * nb + p.blocks_x * j + ei + 1] - start;   // count, summed below
        }
        __syncthreads();
        if (lid == 0) {
            row_off[0] = 0;
            for (int r = 0; r < nr; r++) row_off[r + 1] += row_off[r];
        }
        __syncthreads();
        const int total = row_off[nr];
        for (int c0 = 0; c0 < total; c0 += kAtomChunk) {
            const int cn = min(kAtomChunk, total - c0);
            __syncthreads();
            for (int w = lid; w < cn; w += NTH) {
                const int f = c0 + w;
                int lo = 0, hi = nr - 1;   // the last row whose offset is <= f (a non-empty row holds f)
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (row_off[mid] <= f) lo = mid;
                    else hi = mid - 1;
                }
                const int a = row_start[lo] + (f - row_off[lo]);
                sx[w] = ax[a]; sy[w] = ay[a]; sZ[w] = aZ[a];
            }
            __syncthreads();
            for (int l = 0; l < cn; l++) {
                const double xl = sx[l];
                const double rad_y = im_pos_y - sy[l];
                double rad2[PX];
                bool any = false;
#pragma unroll
                for (int m = 0; m < PX; m++) {
                    const double rad_x = pos_x[m] - xl;
                    if (tilt) {
                        const double zp = -0.5 * (rad_x * cos_beam_phi + rad_y * sin_beam_phi) * sin_beam_2theta;
                        const double zt = zp * inv_tan_beam_theta;
                        const double xp = rad_x + zt * cos_beam_phi, yp = rad_y + zt * sin_beam_phi;
                        rad2[m] = zp * zp + xp * xp + yp * yp;
                    } else {
                        rad2[m] = rad_x * rad_x + rad_y * rad_y;
                    }
                    any = any || rad2[m] <= 64.0;
                }
                if (!any) continue;
                float2 c[NTERM];
                const float2 *t = tab + (sZ[l] - 1) * kPotPTerms;
#pragma unroll
                for (int i = 0; i < NTERM; i++) c[i] = __ldg(t + i);
#pragma unroll
                for (int m = 0; m < PX; m++) {
                    if (rad2[m] <= 64.0) {
                        const float rad = fmaxf(sqrtf((float)rad2[m]), r_min);
                        sum[m] += potp_eval<FORM>(c, rad);
                    }
                }
            }
        }
    }
    if (yid < p.height) {
        float2 *o = out + (size_t)blockIdx.z * p.width * p.height + (size_t)yid * p.width;
#pragma unroll
        for (int m = 0; m < PX; m++)
            if (xid0 + m * TX < p.width) write_trans<float>(o + xid0 + m * TX, (float)p.sigma * sum[m]);
    }
}

}  // namespace ms
