// plain.cu — the plain per-probe FP64 path: the reference's unfused kernel order on one probe at a
// time (SimulationGeneral::doMultiSliceStep, simulationgeneral.cpp:736-768; getStemPixel,
// simulationstem.cpp:74-132), with cuFFT Z2Z standing in for clFFT and a device sync after every
// probe and slice (:767). It is the comparison path the fused engine is measured against, not a
// fallback: it runs on the same device with the same transmission functions.
#include "plain.h"

#include <cufft.h>

#include <vector>

namespace ms {

// complex_multiply_d.cl:12-25 (times a real scale that carries clFFT's 1/sqrt(N) of the preceding transform)
__global__ void k_plain_cmul(const double2 *__restrict__ a, const double2 *__restrict__ b, double2 *__restrict__ out, int n,
                             double scale) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)xid + (size_t)n * yid;
    double2 x = a[id], y = b[id];
    out[id] = make_double2((x.x * y.x - x.y * y.y) * scale, (x.x * y.y + x.y * y.x) * scale);
}
// init_probe_wave_d.cl:49-118 from the precomputed chi table
__global__ void k_plain_probe(double2 *__restrict__ out, int n, const double *__restrict__ kx, const double *__restrict__ ky,
                              const double2 *__restrict__ chi, double px, double py) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)xid + (size_t)n * yid;
    double2 ch = chi[id];
    if (ch.y != 0.0) {
        double posTerm = 2.0 * M_PI * (kx[xid] * px + ky[yid] * py);
        out[id] = make_double2(cos(-posTerm - ch.x), sin(-posTerm - ch.x));
    } else {
        out[id] = make_double2(0.0, 0.0);
    }
}
// propagator_d.cl:18-52
__global__ void k_plain_propagator(double2 *__restrict__ prop, const double *__restrict__ kx, const double *__restrict__ ky,
                                   int n, double dz, double beam_k, double beam_k_x, double beam_k_y, double beam_k_z,
                                   double k_max) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)xid + (size_t)n * yid;
    double k0x = kx[xid] * kx[xid], k0y = ky[yid] * ky[yid];
    double k_max_2 = k_max * k_max;
    if (k0x + k0y < k_max_2) {
        double f = beam_k_z / beam_k;
        double s_u = beam_k * beam_k - beam_k_z * beam_k_z - (beam_k_x + kx[xid]) * (beam_k_x + kx[xid]) -
                     (beam_k_y + ky[yid]) * (beam_k_y + ky[yid]);
        s_u = s_u / (beam_k_z);
        prop[id] = make_double2(f * cos(M_PI * s_u * dz), f * sin(M_PI * s_u * dz));
    } else {
        prop[id] = make_double2(0.0, 0.0);
    }
}
// fft_shift_d.cl + complex_to_real_d.cl method 4 + band_pass_d.cl fused into their three launches
__global__ void k_plain_shift(const double2 *__restrict__ in, double2 *__restrict__ out, int n) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)xid + (size_t)yid * n;
    size_t Yshift = (size_t)n * n / 2;
    int Xshift = n / 2, Xmid = n / 2, Ymid = n / 2;
    if (xid < Xmid && yid < Ymid) out[id + Yshift + Xshift] = in[id];
    else if (xid >= Xmid && yid < Ymid) out[id + Yshift - Xshift] = in[id];
    else if (xid < Xmid && yid >= Ymid) out[id - Yshift + Xshift] = in[id];
    else out[id - Yshift - Xshift] = in[id];
}
__global__ void k_plain_c2r(const double2 *__restrict__ in, double *__restrict__ out, int n) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)xid + (size_t)n * yid;
    out[id] = in[id].x * in[id].x + in[id].y * in[id].y;
}
__global__ void k_plain_bandpass(const double *__restrict__ in, double *__restrict__ out, int n, double inner, double outer,
                                 double xc, double yc) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)xid + (size_t)yid * n;
    double centX = n / 2.0 + xc, centY = n / 2.0 + yc;
    double radius = sqrt((xid - centX) * (xid - centX) + (yid - centY) * (yid - centY));
    out[id] = (radius <= outer && radius >= inner) ? in[id] : 0.0;
}
// sum_reduction_d.cl:13-35: one item per work item, local size 256
__global__ void k_plain_sum(const double *__restrict__ in, double *__restrict__ out, unsigned size) {
    __shared__ double buffer[256];
    size_t idx = threadIdx.x;
    size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    buffer[idx] = 0.0;
    if (gid < size) buffer[idx] += in[gid];
    __syncthreads();
    if (!idx) {
        double sum = 0.0;
        for (int i = 0; i < 256; ++i) sum += fabs(buffer[i]);
        out[blockIdx.x] = sum * 1.41421356237309504880;
    }
}

static void cufft_check(cufftResult r, const char *what) {
    if (r != CUFFT_SUCCESS) throw CudaError(std::string(what) + " failed (cufft status " + std::to_string((int)r) + ")");
}

void PlainWork::release() {
    if (has_plan) cufftDestroy((cufftHandle)plan);
    has_plan = false;
    cudaFree(real); cudaFree(recip); cudaFree(tmp); cudaFree(prop); cudaFree(t2); cudaFree(t3); cudaFree(red);
    real = recip = tmp = prop = nullptr;
    t2 = t3 = red = nullptr;
    n = 0;
}

void plain_stem(cudaStream_t s, const PlainArgs &a, PlainWork &w, const int *pixels, size_t n_pix, double *out) {
    const int n = a.n;
    const size_t NN = (size_t)n * n;
    const unsigned nGroups = (unsigned)(NN / 256);
    try {
        if (w.n != n) {
            w.release();
            MS_CUDA(cudaMalloc(&w.real, NN * sizeof(double2)));
            MS_CUDA(cudaMalloc(&w.recip, NN * sizeof(double2)));
            MS_CUDA(cudaMalloc(&w.tmp, NN * sizeof(double2)));
            MS_CUDA(cudaMalloc(&w.prop, NN * sizeof(double2)));
            MS_CUDA(cudaMalloc(&w.t2, NN * sizeof(double)));
            MS_CUDA(cudaMalloc(&w.t3, NN * sizeof(double)));
            MS_CUDA(cudaMalloc(&w.red, nGroups * sizeof(double)));
            cufftHandle plan = 0;
            cufft_check(cufftPlan2d(&plan, n, n, CUFFT_Z2Z), "cufftPlan2d");
            w.plan = (int)plan;
            w.has_plan = true;
            w.n = n;
        }
        double2 *real = w.real, *recip = w.recip, *tmp = w.tmp, *prop = w.prop;
        double *t2 = w.t2, *t3 = w.t3, *red = w.red;
        const cufftHandle plan = (cufftHandle)w.plan;
        cufft_check(cufftSetStream(plan, s), "cufftSetStream");
        dim3 b(128), g((n + 127) / 128, n);
        k_plain_propagator<<<g, b, 0, s>>>(prop, a.kx, a.ky, n, a.dz, a.beam_k, a.beam_kx, a.beam_ky, a.beam_kz, a.k_max_prop);
        MS_CUDA(cudaGetLastError());
        if (a.launches) *a.launches += 1;
        std::vector<double> sums(nGroups);
        const double sc = a.fft_scale;
        for (size_t i = 0; i < n_pix; i++) {
            const int p = pixels[i];
            const int x_i = p % a.scan_nx;
            const int y_i = p / a.scan_nx;
            double px = a.start_x + x_i * a.step_x - a.sim_x0;
            double py = a.start_y + y_i * a.step_y - a.sim_y0;
            k_plain_probe<<<g, b, 0, s>>>(recip, n, a.kx, a.ky, a.chi, px, py);
            MS_CUDA(cudaGetLastError());
            cufft_check(cufftExecZ2Z(plan, (cufftDoubleComplex *)recip, (cufftDoubleComplex *)real, CUFFT_INVERSE), "cufftExecZ2Z");
            double pending = sc;   // clFFT's scale of the last transform, applied by the next multiply
            if (a.launches) *a.launches += 1;
            int oc = 0;
            for (int sl = 0; sl < a.n_slices; sl++) {
                k_plain_cmul<<<g, b, 0, s>>>(a.trans + (size_t)sl * NN, real, recip, n, pending);
                cufft_check(cufftExecZ2Z(plan, (cufftDoubleComplex *)recip, (cufftDoubleComplex *)tmp, CUFFT_FORWARD), "cufftExecZ2Z");
                k_plain_cmul<<<g, b, 0, s>>>(tmp, prop, recip, n, sc);
                cufft_check(cufftExecZ2Z(plan, (cufftDoubleComplex *)recip, (cufftDoubleComplex *)real, CUFFT_INVERSE), "cufftExecZ2Z");
                pending = sc;
                MS_CUDA(cudaGetLastError());
                MS_CUDA(cudaStreamSynchronize(s));
                if (a.launches) *a.launches += 2;
                bool is_out = (a.slice_step > 0 && (sl + 1) % a.slice_step == 0) || (sl == a.n_slices - 1 && oc < a.n_outputs);
                if (is_out) {
                    for (int d = 0; d < a.n_det; d++) {
                        k_plain_shift<<<g, b, 0, s>>>(recip, tmp, n);
                        k_plain_c2r<<<g, b, 0, s>>>(tmp, t3, n);
                        k_plain_bandpass<<<g, b, 0, s>>>(t3, t2, n, a.innerPx[d], a.outerPx[d], a.xcPx[d], a.ycPx[d]);
                        k_plain_sum<<<nGroups, 256, 0, s>>>(t2, red, (unsigned)NN);
                        MS_CUDA(cudaGetLastError());
                        MS_CUDA(cudaMemcpyAsync(sums.data(), red, nGroups * sizeof(double), cudaMemcpyDeviceToHost, s));
                        MS_CUDA(cudaStreamSynchronize(s));
                        if (a.launches) *a.launches += 4;
                        double sum = 0;
                        for (unsigned gi = 0; gi < nGroups; gi++) sum += sums[gi];
                        out[((size_t)oc * a.n_det + d) * n_pix + i] = sum;
                    }
                    oc++;
                }
            }
        }
    } catch (...) {
        w.release();
        throw;
    }
}

}  // namespace ms
