// gather.cu — atom-position gradients of the differentiable CTEM loss.
//
// dL/dx_a, dL/dy_a of the atoms of one or more consecutive slices (sorted order; one launch per checkpoint
// segment of the adjoint, so the grid holds several slices' atoms): the sum over the pixels within
// 8 Å of atom a of gV(r) V'(rho) d rho / d(x_a, y_a), rho = |r - r_a| (tilt-corrected under a beam tilt, TiltT),
// with V' the derivative of the
// projected form the forward potential kernel sums (potential.cuh; transmission_potentials_projected_d.cl)
// and zero where the forward clamps rho to r_min = dx/4.
//
// Threads of a block are tiled 32 x 8 over a band of the atom's pixel box. Pixel-to-atom offsets
// are formed in FP64 (as in the forward kernel); rho, V'(rho) and the per-thread sums are in the engine's
// precision; the block sums are FP64. The FP64 engine differentiates the restated forms (k_atom_grad); the
// FP32 engine differentiates the table form its forward kernel evaluates (k_atom_grad_f). Built without
// -fmad=false: nothing here restates a reference statement bit for bit.
#include "adjoint_ops.h"
#include "potential.cuh"

#include <type_traits>

namespace ms {

// d/drho of kirkland_p / peng_p / lobato_p (potential.cuh), using K0' = -K1 and K1' = -K0 - K1/x
template <class T>
__device__ __forceinline__ T dpot_drho(int form, const T *__restrict__ prm, int i_lim, int Z, T rho) {
    const T two_pi = (T)(2.0 * M_PI), pi2 = (T)(M_PI * M_PI);
    T s = 0;
    if (form == 0) {   // Kirkland eq. C.20: 300.82 a K0(2 pi rho sqrt b) + 150.41 (c/d) exp(-pi^2 rho^2 / d)
        const T *p = prm + (Z - 1) * 12;
        for (int i = 0; i < i_lim; i++) {
            const T sb = fsqrt(p[2 * i + 1]);
            s -= (T)300.8242834 * p[2 * i] * bessk1<T>(two_pi * rho * sb) * two_pi * sb;
        }
        for (int i = 0; i < i_lim; i++) {
            const T c = p[2 * i_lim + 2 * i], d_inv = (T)1 / p[2 * i_lim + 2 * i + 1];
            s -= (T)150.4121417 * (c * d_inv) * fexp(-pi2 * rho * rho * d_inv) * ((T)2 * pi2 * rho * d_inv);
        }
    } else if (form == 1) {   // Peng: 150.41 (a/b) exp(-pi^2 rho^2 / b)
        const T *p = prm + (Z - 1) * 10;
        for (int i = 0; i < i_lim; i++) {
            const T a = p[i], b_inv = (T)1 / p[i + 5];
            s -= (T)150.4121417 * (a * b_inv) * fexp(-pi2 * rho * rho * b_inv) * ((T)2 * pi2 * rho * b_inv);
        }
    } else {   // Lobato eq. 16: 945.09 a b^-3/2 (K0(c rho) + rho K1(c rho)), c = 2 pi / sqrt b
        const T *p = prm + (Z - 1) * 10;
        for (int i = 0; i < i_lim; i++) {
            const T a = p[i], bir = (T)1 / fsqrt(p[i + 5]);
            const T c = two_pi * bir, x = c * rho;
            s -= (T)945.090144399935 * a * (bir * bir * bir) * c * (bessk1<T>(x) + rho * bessk0<T>(x));
        }
    }
    return s;
}

// The beam tilt of the projected kernel (transmission_potentials_projected_d.cl:283-297, theta = pi/2 - tilt):
// z' = -u sin t cos t, x' = rx - u sin^2 t cos phi, y' = ry - u sin^2 t sin phi with u = rx cos phi + ry sin phi,
// so its radius is rho^2 = rx^2 + ry^2 - sin^2(t) u^2, and d rho / d rx = (rx - sin^2(t) u cos phi) / rho.
template <class T> struct TiltT {
    T s2, c, s;   // sin^2(tilt), cos(phi), sin(phi)
};

// One 256-thread block per (atom, band of pixel rows): kGatherBands blocks share an atom's pixel box so a
// slice's ~100-200 atoms still fill the GPU; each block writes its two sums to work[], and k_atom_grad_sum
// adds the bands of every atom in a fixed order (deterministic results).
constexpr int kGatherBands = 8;

// the slice t of sl holding sorted atom a: start[t] <= a < start[t+1] (empty slices are passed over)
__device__ __forceinline__ int slice_of(const GradSlices &sl, int a) {
    int t = 0;
    while (t + 1 < sl.n && a >= sl.start[t + 1]) t++;
    return t;
}

template <class T>
__global__ void __launch_bounds__(256)
k_atom_grad(const GradSlices sl, const double *__restrict__ ax, const double *__restrict__ ay,
            const int *__restrict__ aZ, const double *__restrict__ gV, int n, double startx, double starty, double dx, int form,
            const T *__restrict__ prm, int i_lim, double *__restrict__ work) {
    __shared__ double red[2][8];
    const int a = sl.start[0] + blockIdx.x;
    const double *gVs = gV + (size_t)slice_of(sl, a) * sl.stride;
    const double xa = ax[a], ya = ay[a];
    const int Z = aZ[a];
    const T r_min2 = (T)(0.0625 * dx * dx);   // (dx / 4)^2
    int ix0 = (int)floor((xa - 8.0 - startx) / dx), ix1 = (int)ceil((xa + 8.0 - startx) / dx);
    int iy0 = (int)floor((ya - 8.0 - starty) / dx), iy1 = (int)ceil((ya + 8.0 - starty) / dx);
    ix0 = max(ix0, 0); iy0 = max(iy0, 0); ix1 = min(ix1, n - 1); iy1 = min(iy1, n - 1);
    // this block's rows: band blockIdx.y of kGatherBands equal bands of [iy0, iy1]
    const int rows = iy1 - iy0 + 1;
    const int r0 = iy0 + (int)(((long long)rows * blockIdx.y) / kGatherBands);
    const int r1 = iy0 + (int)(((long long)rows * (blockIdx.y + 1)) / kGatherBands) - 1;
    const double ox = startx - xa, oy = starty - ya;   // pixel px sits at ox + px dx from the atom
    const TiltT<T> ts{(T)sl.tilt_s2, (T)sl.cphi, (T)sl.sphi};
    T gx = 0, gy = 0;
    for (int py = r0 + (int)threadIdx.y; py <= r1; py += 8) {
        const T ry = (T)(oy + py * dx);
        const double *grow = gVs + (size_t)py * n;
        for (int px = ix0 + (int)threadIdx.x; px <= ix1; px += 32) {
            const T rx = (T)(ox + px * dx);
            const T u = rx * ts.c + ry * ts.s;
            const T rho2 = rx * rx + ry * ry - ts.s2 * u * u;
            if (rho2 > r_min2 && rho2 <= (T)64) {
                const T rho = fsqrt(rho2);
                const T f = (T)grow[px] * dpot_drho<T>(form, prm, i_lim, Z, rho) / rho;
                gx -= f * (rx - ts.s2 * u * ts.c);   // d rho / d x_a = -(rx - s2 u cos phi) / rho
                gy -= f * (ry - ts.s2 * u * ts.s);
            }
        }
    }
    double sx = (double)gx, sy = (double)gy;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_down_sync(0xffffffffu, sx, o);
        sy += __shfl_down_sync(0xffffffffu, sy, o);
    }
    if (threadIdx.x == 0) { red[0][threadIdx.y] = sx; red[1][threadIdx.y] = sy; }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double tx = 0, ty = 0;
        for (int i = 0; i < 8; i++) { tx += red[0][i]; ty += red[1][i]; }
        const size_t w = ((size_t)blockIdx.x * kGatherBands + blockIdx.y) * 2;
        work[w] = tx;
        work[w + 1] = ty;
    }
}

// The FP32 gradient of the FP32 projected kernel's evaluation (k_potential_projected_f): the terms of the
// table (potential.cuh, potp_table) differentiated with K0' = -K1 and K1' = -K0 - K1/x, evaluated by the same
// FP32 K0 / K1. Same blocks, bands, pixel offsets, r_min and 8 Å limits as k_atom_grad.
template <int FORM>
__device__ __forceinline__ float dpotp_drho(const float2 (&c)[FORM == 0 ? 6 : 5], float rho) {
    constexpr float kLn2x2 = 1.38629436111989061883f;   // 2 ln 2
    if constexpr (FORM == 0) {
        const float r2 = rho * rho;
        float s = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; i++) s -= c[i].x * c[i].y * k1f(c[i].y * rho);
#pragma unroll
        for (int i = 0; i < 3; i++) s += c[3 + i].x * ex2a(c[3 + i].y * r2) * (kLn2x2 * c[3 + i].y * rho);
        return s;
    } else if constexpr (FORM == 1) {
        const float r2 = rho * rho;
        float s = 0.0f;
#pragma unroll
        for (int i = 0; i < 5; i++) s += c[i].x * ex2a(c[i].y * r2) * (kLn2x2 * c[i].y * rho);
        return s;
    } else {
        float s = 0.0f;
#pragma unroll
        for (int i = 0; i < 5; i++) {
            const float x = c[i].y * rho;
            s -= c[i].x * c[i].y * (k1f(x) + rho * k0f(x));
        }
        return s;
    }
}

template <int FORM>
__global__ void __launch_bounds__(256)
k_atom_grad_f(const GradSlices sl, const double *__restrict__ ax, const double *__restrict__ ay,
              const int *__restrict__ aZ, const double *__restrict__ gV, int n, double startx, double starty, double dx,
              const float2 *__restrict__ tab, double *__restrict__ work) {
    constexpr int NTERM = FORM == 0 ? 6 : 5;
    __shared__ double red[2][8];
    const int a = sl.start[0] + blockIdx.x;
    const double *gVs = gV + (size_t)slice_of(sl, a) * sl.stride;
    const double xa = ax[a], ya = ay[a];
    float2 c[NTERM];
    const float2 *t = tab + (aZ[a] - 1) * kPotPTerms;
#pragma unroll
    for (int i = 0; i < NTERM; i++) c[i] = __ldg(t + i);
    const float r_min2 = (float)(0.0625 * dx * dx);   // (dx / 4)^2
    int ix0 = (int)floor((xa - 8.0 - startx) / dx), ix1 = (int)ceil((xa + 8.0 - startx) / dx);
    int iy0 = (int)floor((ya - 8.0 - starty) / dx), iy1 = (int)ceil((ya + 8.0 - starty) / dx);
    ix0 = max(ix0, 0); iy0 = max(iy0, 0); ix1 = min(ix1, n - 1); iy1 = min(iy1, n - 1);
    const int rows = iy1 - iy0 + 1;
    const int r0 = iy0 + (int)(((long long)rows * blockIdx.y) / kGatherBands);
    const int r1 = iy0 + (int)(((long long)rows * (blockIdx.y + 1)) / kGatherBands) - 1;
    const double ox = startx - xa, oy = starty - ya;
    const TiltT<float> ts{(float)sl.tilt_s2, (float)sl.cphi, (float)sl.sphi};
    float gx = 0, gy = 0;
    for (int py = r0 + (int)threadIdx.y; py <= r1; py += 8) {
        const float ry = (float)(oy + py * dx);
        const double *grow = gVs + (size_t)py * n;
        for (int px = ix0 + (int)threadIdx.x; px <= ix1; px += 32) {
            const float rx = (float)(ox + px * dx);
            const float u = rx * ts.c + ry * ts.s;
            const float rho2 = rx * rx + ry * ry - ts.s2 * u * u;
            if (rho2 > r_min2 && rho2 <= 64.0f) {
                const float rho = sqrtf(rho2);
                const float f = (float)grow[px] * __fdividef(dpotp_drho<FORM>(c, rho), rho);
                gx -= f * (rx - ts.s2 * u * ts.c);   // d rho / d x_a = -(rx - s2 u cos phi) / rho
                gy -= f * (ry - ts.s2 * u * ts.s);
            }
        }
    }
    double sx = (double)gx, sy = (double)gy;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_down_sync(0xffffffffu, sx, o);
        sy += __shfl_down_sync(0xffffffffu, sy, o);
    }
    if (threadIdx.x == 0) { red[0][threadIdx.y] = sx; red[1][threadIdx.y] = sy; }
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double tx = 0, ty = 0;
        for (int i = 0; i < 8; i++) { tx += red[0][i]; ty += red[1][i]; }
        const size_t w = ((size_t)blockIdx.x * kGatherBands + blockIdx.y) * 2;
        work[w] = tx;
        work[w + 1] = ty;
    }
}

__global__ void k_atom_grad_sum(int a0, int count, const double *__restrict__ work, double *__restrict__ gxy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double tx = 0, ty = 0;
    for (int b = 0; b < kGatherBands; b++) {
        tx += work[((size_t)i * kGatherBands + b) * 2];
        ty += work[((size_t)i * kGatherBands + b) * 2 + 1];
    }
    gxy[2 * (size_t)(a0 + i)] = tx;
    gxy[2 * (size_t)(a0 + i) + 1] = ty;
}

template <class T>
void atom_grad(cudaStream_t s, const GradSlices &sl, const double *ax, const double *ay, const int *aZ, const double *gV,
               int n, double startx, double starty, double dx, int form, const T *prm, int i_lim, const float2 *tabp,
               double *gxy, double *work) {
    if (sl.n < 1 || sl.n > kGradMaxSlices) throw std::runtime_error("atom_grad: 1 to kGradMaxSlices slices a launch");
    const int a0 = sl.start[0], count = sl.start[sl.n] - a0;
    if (count <= 0) return;
    const dim3 grd(count, kGatherBands), blk(32, 8);
    if constexpr (std::is_same<T, float>::value) {   // the FP32 engine differentiates its table kernel
        if (tabp == nullptr) throw std::runtime_error("the FP32 gradient needs the term table of the parameterisation");
        (void)prm; (void)i_lim;
        if (form == 0) k_atom_grad_f<0><<<grd, blk, 0, s>>>(sl, ax, ay, aZ, gV, n, startx, starty, dx, tabp, work);
        else if (form == 1) k_atom_grad_f<1><<<grd, blk, 0, s>>>(sl, ax, ay, aZ, gV, n, startx, starty, dx, tabp, work);
        else k_atom_grad_f<2><<<grd, blk, 0, s>>>(sl, ax, ay, aZ, gV, n, startx, starty, dx, tabp, work);
    } else {   // the FP64 engine: the FP64 derivative of the restated forms
        (void)tabp;
        k_atom_grad<T><<<grd, blk, 0, s>>>(sl, ax, ay, aZ, gV, n, startx, starty, dx, form, prm, i_lim, work);
    }
    MS_CUDA(cudaGetLastError());
    k_atom_grad_sum<<<(count + 127) / 128, 128, 0, s>>>(a0, count, work, gxy);
    MS_CUDA(cudaGetLastError());
}
int atom_grad_work_doubles(int max_count) { return 2 * kGatherBands * max_count; }

template void atom_grad<float>(cudaStream_t, const GradSlices &, const double *, const double *, const int *,
                               const double *, int, double, double, double, int, const float *, int, const float2 *,
                               double *, double *);
template void atom_grad<double>(cudaStream_t, const GradSlices &, const double *, const double *, const int *,
                                const double *, int, double, double, double, int, const double *, int, const float2 *,
                                double *, double *);

}  // namespace ms
