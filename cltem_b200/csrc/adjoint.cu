// adjoint.cu — pointwise and gather kernels of the differentiable CTEM image (built with -fmad=false).
//
// Loss L = sum over pixels of (I - I_target)^2, I = |W|^2, W = s2d Dinv(H Recip), H the objective-lens
// transfer of ctem_image_d.cl:50-119. Gradients use G = dL/dRe + i dL/dIm.
#include "adjoint_ops.h"
#include "optics.cuh"

namespace ms {

// per-block partial sums (fixed order) of one double per thread
__device__ __forceinline__ void block_partial(double v, double *out, double *red) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) s += red[w];
        out[blockIdx.x] = s;
    }
}

// I = |W|^2; partial sums of (I - target)^2; G_W = 4 (I - target) W
template <class R>
__global__ void k_image_loss(size_t n, const cplx<R> *__restrict__ W, const double *__restrict__ target,
                             cplx<R> *__restrict__ gW, double *__restrict__ partial) {
    __shared__ double red[32];
    double acc = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double re = (double)W[i].x, im = (double)W[i].y;
        double d = re * re + im * im - target[i];
        acc += d * d;
        gW[i] = mk<R>((R)(4.0 * d * re), (R)(4.0 * d * im));
    }
    block_partial(acc, partial, red);
}

// The objective-lens transfer H at one pixel (ctem_image_d.cl:73-111) and dlnH/dC10, dlnH/dC30
struct HGrad {
    double2 H;
    double chi10, chi30;   // dchi/dC10, dchi/dC30
    double e10, e30;       // dlnE_s/dC10, dlnE_s/dC30
};
__device__ __forceinline__ HGrad transfer_at(double kxv, double kyv, double wavelength, const AberrD &A, double obj_ap,
                                             double ap_smooth, double beta, double delta) {
    HGrad h;
    h.H = make_double2(0, 0);
    h.chi10 = h.chi30 = h.e10 = h.e30 = 0;
    double obj_ap2 = (obj_ap * 0.001) / wavelength;
    double beta2 = (beta * 0.001) / wavelength;
    double k = sqrt((kxv * kxv) + (kyv * kyv));
    double ap_smooth_radius = (ap_smooth * 0.001) / wavelength;
    if (k < obj_ap2 + ap_smooth_radius) {
        double2 w = make_double2(wavelength * kxv, wavelength * kyv);
        double w2 = cModSq(w);
        double temporalCoh = exp(-0.25 * M_PI * M_PI * delta * delta * w2 * w2 / (wavelength * wavelength));
        double sp = (A.C10 + A.C30 * w2 + A.C50 * w2 * w2);
        double spatialCoh = exp(-1.0 * M_PI * M_PI * beta2 * beta2 * w2 * (sp * sp));
        double chi = 2.0 * M_PI * cchi_of(A, w) / wavelength;
        double edge_factor = 1.0;
        if (fabs(k - obj_ap2) < ap_smooth_radius) {
            double e0 = obj_ap2 - ap_smooth_radius, e1 = obj_ap2 + ap_smooth_radius;
            double t = fmin(fmax((k - e0) / (e1 - e0), 0.0), 1.0);
            edge_factor = 1.0 - t * t * (3.0 - 2.0 * t);
        }
        double amp = edge_factor * temporalCoh * spatialCoh;
        h.H = make_double2(amp * cos(chi), -amp * sin(chi));   // out = in * exp(-i chi) * amp
        h.chi10 = 2.0 * M_PI / wavelength * 0.5 * w2;
        h.chi30 = 2.0 * M_PI / wavelength * 0.25 * w2 * w2;
        double de = -1.0 * M_PI * M_PI * beta2 * beta2 * w2 * 2.0 * sp;
        h.e10 = de;
        h.e30 = de * w2;
    }
    return h;
}

// G_Recip = conj(H) G_Y; partial sums of dL/dC10 = sum Re(Z) e10 + Im(Z) chi10 with Z = H Recip conj(G_Y)
// (dH/dtheta = H (-i dchi/dtheta + dlnE/dtheta)); likewise C30
template <class R>
__global__ void k_image_backward(int n, const cplx<R> *__restrict__ recip, const cplx<R> *__restrict__ gY,
                                 cplx<R> *__restrict__ gRecip, const double *__restrict__ kx, const double *__restrict__ ky,
                                 double wavelength, AberrD A, double obj_ap, double ap_smooth, double beta, double delta,
                                 double *__restrict__ partial10, double *__restrict__ partial30) {
    __shared__ double red[32];
    double a10 = 0, a30 = 0;
    const size_t total = (size_t)n * n;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int xid = (int)(i % n), yid = (int)(i / n);
        HGrad h = transfer_at(kx[xid], ky[yid], wavelength, A, obj_ap, ap_smooth, beta, delta);
        double2 g = make_double2((double)gY[i].x, (double)gY[i].y);
        double2 r = make_double2((double)recip[i].x, (double)recip[i].y);
        double2 gr = make_double2(h.H.x * g.x + h.H.y * g.y, h.H.x * g.y - h.H.y * g.x);   // conj(H) g
        gRecip[i] = mk<R>((R)gr.x, (R)gr.y);
        double2 y = make_double2(h.H.x * r.x - h.H.y * r.y, h.H.x * r.y + h.H.y * r.x);    // H recip
        double zr = y.x * g.x + y.y * g.y, zi = y.y * g.x - y.x * g.y;                     // y conj(g)
        a10 += zr * h.e10 + zi * h.chi10;
        a30 += zr * h.e30 + zi * h.chi30;
    }
    block_partial(a10, partial10, red);
    __syncthreads();
    block_partial(a30, partial30, red);
}

// conj(P) g * scale inside the propagator's strict cut, zero outside
template <class R>
__global__ void k_mul_conj_prop(int n, cplx<R> *__restrict__ g, const cplx<R> *__restrict__ px, const cplx<R> *__restrict__ py,
                                const double *__restrict__ kx2, const double *__restrict__ ky2, double kmax2, R scale) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t i = (size_t)yid * n + xid;
    cplx<R> p = (kx2[xid] + ky2[yid] < kmax2) ? cmul(px[xid], py[yid]) : mk<R>(0, 0);
    g[i] = cscale(cmulc(g[i], p), scale);
}

// gV = sigma Im(conj(E) G_E)
template <class R>
__global__ void k_grad_v(size_t count, const cplx<R> *__restrict__ E, const cplx<R> *__restrict__ gE, double sigma,
                         double *__restrict__ gV) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double ex = (double)E[i].x, ey = (double)E[i].y, gx = (double)gE[i].x, gy = (double)gE[i].y;
    gV[i] = sigma * (ex * gy - ey * gx);
}

// ---------------------------------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------------------------------
constexpr int kRedBlocks = 256, kRedThreads = 256;

template <class R> void image_loss(cudaStream_t s, size_t n, const cplx<R> *W, const double *target, cplx<R> *gW,
                                   double *partial) {
    k_image_loss<R><<<kRedBlocks, kRedThreads, 0, s>>>(n, W, target, gW, partial);
    MS_CUDA(cudaGetLastError());
}
template <class R> void image_backward(cudaStream_t s, int n, const cplx<R> *recip, const cplx<R> *gY, cplx<R> *gRecip,
                                       const double *kx, const double *ky, double wavelength, const AberrD &A, double obj_ap,
                                       double ap_smooth, double beta, double delta, double *p10, double *p30) {
    k_image_backward<R><<<kRedBlocks, kRedThreads, 0, s>>>(n, recip, gY, gRecip, kx, ky, wavelength, A, obj_ap, ap_smooth,
                                                           beta, delta, p10, p30);
    MS_CUDA(cudaGetLastError());
}
template <class R> void mul_conj_prop(cudaStream_t s, int n, cplx<R> *g, const cplx<R> *px, const cplx<R> *py,
                                      const double *kx2, const double *ky2, double kmax2, R scale) {
    dim3 b(128), gr((n + 127) / 128, n);
    k_mul_conj_prop<R><<<gr, b, 0, s>>>(n, g, px, py, kx2, ky2, kmax2, scale);
    MS_CUDA(cudaGetLastError());
}
template <class R> void grad_v(cudaStream_t s, size_t count, const cplx<R> *E, const cplx<R> *gE, double sigma, double *gV) {
    k_grad_v<R><<<(unsigned)((count + 255) / 256), 256, 0, s>>>(count, E, gE, sigma, gV);
    MS_CUDA(cudaGetLastError());
}
int reduction_blocks() { return kRedBlocks; }

#define MS_INST_ADJ(R)                                                                                                  \
    template void image_loss<R>(cudaStream_t, size_t, const cplx<R> *, const double *, cplx<R> *, double *);           \
    template void image_backward<R>(cudaStream_t, int, const cplx<R> *, const cplx<R> *, cplx<R> *, const double *,     \
                                    const double *, double, const AberrD &, double, double, double, double, double *,  \
                                    double *);                                                                         \
    template void mul_conj_prop<R>(cudaStream_t, int, cplx<R> *, const cplx<R> *, const cplx<R> *, const double *,      \
                                   const double *, double, R);                                                         \
    template void grad_v<R>(cudaStream_t, size_t, const cplx<R> *, const cplx<R> *, double, double *);
MS_INST_ADJ(float)
MS_INST_ADJ(double)

}  // namespace ms
