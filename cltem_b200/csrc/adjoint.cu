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

// d/drho of the projected potentials (projected_d.cl:104-181): K0' = -K1, K1' = -K0 - K1/x
__device__ double k0d(double x) {   // NR 6.6 rational forms, same coefficients as the forward kernels
    const double p0[5] = {1.0, 2.346487949187396e-1, 1.187082088663404e-2, 2.150707366040937e-4, 1.425433617130587e-6};
    const double q0[3] = {9.847324170755358e-1, 1.518396076767770e-2, 8.362215678646257e-5};
    const double pp0[5] = {1.159315156584126e-1, 2.770731240515333e-1, 2.066458134619875e-2, 4.574734709978264e-4, 3.454715527986737e-6};
    const double qq0[3] = {9.836249671709183e-1, 1.627693622304549e-2, 9.809660603621949e-5};
    const double a0[8] = {1.253314137315499, 1.475731032429900e1, 6.123767403223466e1, 1.121012633939949e2,
                          9.285288485892228e1, 3.198289277679660e1, 3.595376024148513, 6.160228690102976e-2};
    const double b0[8] = {1.0, 1.189963006673403e1, 5.027773590829784e1, 9.496513373427093e1,
                          8.318077493230258e1, 3.181399777449301e1, 4.443672926432041, 1.408295601966600e-1};
    auto poly = [](const double *c, int m, double z) { double s = c[m]; for (int i = m - 1; i >= 0; --i) s = s * z + c[i]; return s; };
    if (x <= 1.0) {
        double z = x * x;
        return poly(pp0, 4, z) / poly(qq0, 2, 1.0 - z) - poly(p0, 4, z) * log(x) / poly(q0, 2, 1.0 - z);
    }
    double z = 1.0 / x;
    return exp(-x) * poly(a0, 7, z) / poly(b0, 7, z) / sqrt(x);
}
__device__ double k1d(double x) {
    const double p1[5] = {0.5, 5.598072040178741e-2, 1.818666382168295e-3, 2.397509908859959e-5, 1.239567816344855e-7};
    const double q1[3] = {9.870202601341150e-1, 1.292092053534579e-2, 5.881933053917096e-5};
    const double pp1[5] = {-3.079657578292062e-1, -8.109417631822442e-2, -3.477550948593604e-3, -5.385594871975406e-5, -3.110372465429008e-7};
    const double qq1[3] = {9.861813171751389e-1, 1.375094061153160e-2, 6.774221332947002e-5};
    const double a1[8] = {1.253314137315502, 1.457171340220454e1, 6.063161173098803e1, 1.147386690867892e2,
                          1.040442011439181e2, 4.356596656837691e1, 7.265230396353690, 3.144418558991021e-1};
    const double b1[8] = {1.0, 1.125154514806458e1, 4.427488496597630e1, 7.616113213117645e1,
                          5.863377227890893e1, 1.850303673841586e1, 1.857244676566022, 2.538540887654872e-2};
    auto poly = [](const double *c, int m, double z) { double s = c[m]; for (int i = m - 1; i >= 0; --i) s = s * z + c[i]; return s; };
    if (x <= 1.0) {
        double z = x * x;
        return x * (poly(pp1, 4, z) / poly(qq1, 2, 1.0 - z) + poly(p1, 4, z) * log(x) / poly(q1, 2, 1.0 - z)) + 1.0 / x;
    }
    double z = 1.0 / x;
    return exp(-x) * poly(a1, 7, z) / poly(b1, 7, z) / sqrt(x);
}

__device__ double dpot_drho(int form, const double *__restrict__ prm, int i_lim, int Z, double rho) {
    if (form == 0) {   // Kirkland C.20
        const double *p = prm + (Z - 1) * 12;
        double s = 0;
        for (int i = 0; i < i_lim; i++) {
            double sb = sqrt(p[2 * i + 1]);
            s += 300.8242834 * p[2 * i] * (-k1d(2.0 * M_PI * rho * sb)) * 2.0 * M_PI * sb;
        }
        for (int i = 0; i < i_lim; i++) {
            double c = p[2 * i_lim + 2 * i], d = p[2 * i_lim + 2 * i + 1];
            s += 150.4121417 * (c / d) * exp(-M_PI * M_PI * rho * rho / d) * (-2.0 * M_PI * M_PI * rho / d);
        }
        return s;
    } else if (form == 1) {   // Peng
        const double *p = prm + (Z - 1) * 10;
        double s = 0;
        for (int i = 0; i < i_lim; i++) {
            double a = p[i], b = p[i + 5];
            s += 150.4121417 * (a / b) * exp(-M_PI * M_PI * rho * rho / b) * (-2.0 * M_PI * M_PI * rho / b);
        }
        return s;
    }
    const double *p = prm + (Z - 1) * 10;   // Lobato eq. 16
    double s = 0;
    for (int i = 0; i < i_lim; i++) {
        double a = p[i], b = p[i + 5];
        double c = 2.0 * M_PI / sqrt(b), x = c * rho;
        s += 945.090144399935 * a / (b * sqrt(b)) * (-c) * (k1d(x) + rho * k0d(x));
    }
    return s;
}

// dL/dx_a, dL/dy_a of the atoms [a0, a1) of slice k (sorted order): sum over pixels within 8 Å of
// gV_k(r) V'(rho) d rho / d(x_a, y_a), rho = |r - r_a| clamped below at r_min (zero derivative there)
__global__ void k_atom_grad(int a0, const double *__restrict__ ax, const double *__restrict__ ay, const int *__restrict__ aZ,
                            const double *__restrict__ gV, int n, double startx, double starty, double dx, int form,
                            const double *__restrict__ prm, int i_lim, double *__restrict__ gxy) {
    __shared__ double red[32];
    const int a = a0 + blockIdx.x;
    const double xa = ax[a], ya = ay[a];
    const int Z = aZ[a];
    const double r_min = 0.25 * dx;
    int ix0 = (int)floor((xa - 8.0 - startx) / dx), ix1 = (int)ceil((xa + 8.0 - startx) / dx);
    int iy0 = (int)floor((ya - 8.0 - starty) / dx), iy1 = (int)ceil((ya + 8.0 - starty) / dx);
    ix0 = max(ix0, 0); iy0 = max(iy0, 0); ix1 = min(ix1, n - 1); iy1 = min(iy1, n - 1);
    const int w = ix1 - ix0 + 1, h = iy1 - iy0 + 1;
    double gx = 0, gy = 0;
    for (int i = threadIdx.x; i < w * h; i += blockDim.x) {
        int px = ix0 + i % w, py = iy0 + i / w;
        double rx = (startx + px * dx) - xa, ry = (starty + py * dx) - ya;
        double rho = sqrt(rx * rx + ry * ry);
        if (rho > r_min && rho <= 8.0) {
            double f = gV[(size_t)py * n + px] * dpot_drho(form, prm, i_lim, Z, rho) / rho;
            gx -= f * rx;   // d rho / d x_a = -rx / rho
            gy -= f * ry;
        }
    }
    // block sums of (gx, gy); thread 0 stores them for atom a
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gx += __shfl_down_sync(0xffffffffu, gx, o);
        gy += __shfl_down_sync(0xffffffffu, gy, o);
    }
    __shared__ double redy[32];
    if ((threadIdx.x & 31) == 0) { red[threadIdx.x >> 5] = gx; redy[threadIdx.x >> 5] = gy; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sx = 0, sy = 0;
        for (int i = 0; i < (int)(blockDim.x + 31) / 32; i++) { sx += red[i]; sy += redy[i]; }
        gxy[2 * (size_t)a] = sx;
        gxy[2 * (size_t)a + 1] = sy;
    }
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
void atom_grad(cudaStream_t s, int a0, int count, const double *ax, const double *ay, const int *aZ, const double *gV,
               int n, double startx, double starty, double dx, int form, const double *prm, int i_lim, double *gxy) {
    if (count <= 0) return;
    k_atom_grad<<<count, 256, 0, s>>>(a0, ax, ay, aZ, gV, n, startx, starty, dx, form, prm, i_lim, gxy);
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
