// misc.cu — atom binning, tables, reductions and imaging kernels. Built with -fmad=false: the FP64
// expressions below follow the reference's _d kernels statement by statement and must not be contracted.
#include "misc.cuh"
#include "optics.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace ms {

// ------------------------------------------------------------------------------------------------
// Atom binning (SimulationGeneral::sortAtoms, simulationgeneral.cpp:147-342)
// ------------------------------------------------------------------------------------------------
// Per atom: the strict host range filter on the padded full limits (:206-210), then atom_sort
// (kernels/atom_sort_d.cl:28-69) on the atoms that pass. Sort key = z id * bx*by + block id, or
// n_bins for atoms that are filtered out or outside the xy range (they sort last and are never read).
__global__ void k_atom_keys(int n, const double *__restrict__ x, const double *__restrict__ y, const double *__restrict__ z,
                            SortGeom g, int *__restrict__ keys, int *__restrict__ idx, int *__restrict__ bid_out,
                            int *__restrict__ zid_out, int *__restrict__ kept) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int n_bins = g.n_slices * g.blocks_x * g.blocks_y;
    double xi = x[i], yi = y[i], zi = z[i];
    bool in = xi > g.full_x0 && xi < g.full_x1 && yi > g.full_y0 && yi < g.full_y1 && zi > g.z0 && zi < g.z1;
    int key = n_bins, bid = -1, zid = -1;
    if (in) {
        if (xi >= g.full_x0 && xi <= g.full_x1 && yi >= g.full_y0 && yi <= g.full_y1) {
            int bidx = (int)floor((xi - g.full_x0) * (1.0 / (g.full_x1 - g.full_x0)) * g.blocks_x);
            int bidy = (int)floor((yi - g.full_y0) * (1.0 / (g.full_y1 - g.full_y0)) * g.blocks_y);
            zid = (int)floor((g.z1 - zi) * (1.0 / (g.dz)));
            zid -= (zid == g.n_slices);
            bidx -= (bidx == g.blocks_x);
            bidy -= (bidy == g.blocks_y);
            bid = bidx + g.blocks_x * bidy;
        }
        // zid < n_slices holds for a geometry whose slice count covers z_lims (mslice_geometry_compute); the test
        // keeps a caller-filled geometry that does not from forming keys beyond the bins
        if (bid >= 0 && zid >= 0 && zid < g.n_slices) key = zid * g.blocks_x * g.blocks_y + bid;
    }
    keys[i] = key;
    idx[i] = i;
    bid_out[i] = bid;
    zid_out[i] = zid;
    kept[i] = in ? 1 : 0;
}

__global__ void k_atom_gather(int n, const int *__restrict__ idx, const int *__restrict__ Z, const double *__restrict__ x,
                              const double *__restrict__ y, const double *__restrict__ z, int *__restrict__ Zs,
                              double *__restrict__ xs, double *__restrict__ ys, double *__restrict__ zs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int j = idx[i];
    Zs[i] = Z[j];
    xs[i] = x[j];
    ys[i] = y[j];
    zs[i] = z[j];
}

__global__ void k_atom_hist(int n, const int *__restrict__ keys, int n_bins, int *__restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = keys[i];
    if ((unsigned)k < (unsigned)n_bins) atomicAdd(&counts[k], 1);
}

static int key_bits(int n_bins) {
    int b = 1;
    while ((1ll << b) <= (long long)n_bins) b++;
    return b;
}

size_t atom_sort_temp_bytes(int n, int n_bins) {
    size_t a = 0, b = 0;
    MS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, a, (const int *)nullptr, (int *)nullptr, (const int *)nullptr,
                                            (int *)nullptr, n, 0, key_bits(n_bins)));
    MS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, b, (const int *)nullptr, (int *)nullptr, n_bins + 1));
    return a > b ? a : b;
}

void atom_sort(cudaStream_t s, const SortGeom &g, int n, const int *Z, const double *x, const double *y, const double *z,
               AtomSortBuffers &buf, int *block_start, int *Zs, double *xs, double *ys, double *zs) {
    const int n_bins = g.n_slices * g.blocks_x * g.blocks_y;
    MS_CUDA(cudaMemsetAsync(buf.counts, 0, sizeof(int) * (n_bins + 1), s));
    if (n > 0) {
        const int T = 256, B = (n + T - 1) / T;
        k_atom_keys<<<B, T, 0, s>>>(n, x, y, z, g, buf.keys_in, buf.idx_in, buf.bid, buf.zid, buf.kept);
        MS_CUDA(cudaGetLastError());
        size_t bytes = buf.cub_temp_bytes;
        // LSD radix sort: stable, so atoms of one bin keep their input order (the reference's push_back order)
        MS_CUDA(cub::DeviceRadixSort::SortPairs(buf.cub_temp, bytes, buf.keys_in, buf.keys_out, buf.idx_in, buf.idx_out, n,
                                                0, key_bits(n_bins), s));
        k_atom_gather<<<B, T, 0, s>>>(n, buf.idx_out, Z, x, y, z, Zs, xs, ys, zs);
        MS_CUDA(cudaGetLastError());
        k_atom_hist<<<B, T, 0, s>>>(n, buf.keys_in, n_bins, buf.counts);
        MS_CUDA(cudaGetLastError());
    }
    size_t bytes = buf.cub_temp_bytes;
    MS_CUDA(cub::DeviceScan::ExclusiveSum(buf.cub_temp, bytes, buf.counts, block_start, n_bins + 1, s));
}

// ------------------------------------------------------------------------------------------------
// Probe aberration table (init_probe_wave_d.cl:49-118 without the position term)
// ------------------------------------------------------------------------------------------------
__global__ void k_chi_table(int n, const double *__restrict__ kx, const double *__restrict__ ky, double wavelength, AberrD A,
                            double cond_ap, double ap_smooth, double2 *__restrict__ out) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    double cond_ap2 = (cond_ap * 0.001) / wavelength;
    double k = sqrt((kx[xid] * kx[xid]) + (ky[yid] * ky[yid]));
    double ap_smooth_radius = (ap_smooth * 0.001) / wavelength;
    double2 r = make_double2(0.0, 0.0);
    if (k < cond_ap2 + ap_smooth_radius) {
        double2 w = make_double2(wavelength * kx[xid], wavelength * ky[yid]);
        double cchi = cchi_of(A, w);
        r = make_double2(2.0 * M_PI * cchi / wavelength, 1.0);
    }
    out[(size_t)yid * n + xid] = r;
}

void chi_table(cudaStream_t s, int n, const double *kx, const double *ky, double wavelength, const AberrD &A, double cond_ap,
               double ap_smooth, double2 *out) {
    dim3 b(128), gr((n + 127) / 128, n);
    k_chi_table<<<gr, b, 0, s>>>(n, kx, ky, wavelength, A, cond_ap, ap_smooth, out);
    MS_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------------------------------------
// Detectors
// ------------------------------------------------------------------------------------------------
struct DetDesc {
    double in[16], out[16], xc[16], yc[16];
};

__global__ void k_detmask(int n, int n_det, DetDesc D, uint16_t *__restrict__ out) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    // pixel (xid, yid) of the unshifted pattern sits at (xs, ys) after fft_shift (fft_shift_d.cl:12-48)
    int xs = (xid + n / 2) % n, ys = (yid + n / 2) % n;
    uint16_t m = 0;
    for (int d = 0; d < n_det; d++) {
        double centX = n / 2.0 + D.xc[d];
        double centY = n / 2.0 + D.yc[d];
        double radius = sqrt((xs - centX) * (xs - centX) + (ys - centY) * (ys - centY));
        if (radius <= D.out[d] && radius >= D.in[d]) m |= (uint16_t)(1u << d);
    }
    out[(size_t)yid * n + xid] = m;
}

void detector_masks(cudaStream_t s, int n, int n_det, const double *innerPx, const double *outerPx, const double *xcPx,
                    const double *ycPx, uint16_t *out) {
    DetDesc D;
    for (int d = 0; d < 16; d++) {
        D.in[d] = d < n_det ? innerPx[d] : 0;
        D.out[d] = d < n_det ? outerPx[d] : 0;
        D.xc[d] = d < n_det ? xcPx[d] : 0;
        D.yc[d] = d < n_det ? ycPx[d] : 0;
    }
    dim3 b(128), gr((n + 127) / 128, n);
    k_detmask<<<gr, b, 0, s>>>(n, n_det, D, out);
    MS_CUDA(cudaGetLastError());
}

__device__ __forceinline__ void kahan_add(double &sum, double &c, double v) {
    double yv = v - c;
    double t = sum + yv;
    c = (t - sum) - yv;
    sum = t;
}

__global__ void k_det_reduce(const double *__restrict__ partials, int n_blocks, int n_det, int batch,
                             const int *__restrict__ pixel_of_wave, int n_pix, int o, double *__restrict__ out,
                             double *__restrict__ comp) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch * n_det) return;
    int b = i / n_det, d = i % n_det;
    const double *p = partials + ((size_t)b * n_det + d) * n_blocks;
    double s = 0;
    for (int k = 0; k < n_blocks; k++) s += p[k];
    double v = s * 1.41421356237309504880;   // M_SQRT2 of sum_reduction_d.cl:30
    size_t oi = ((size_t)o * n_det + d) * n_pix + pixel_of_wave[b];
    if (comp) {
        double sum = out[oi], c = comp[oi];
        kahan_add(sum, c, v);
        out[oi] = sum;
        comp[oi] = c;
    } else {
        out[oi] = v;
    }
}

void detector_reduce(cudaStream_t s, const double *partials, int n_blocks, int n_det, int batch, const int *pixel_of_wave,
                     int n_pix, int o, double *out, double *comp) {
    int n = batch * n_det;
    if (n == 0) return;
    k_det_reduce<<<(n + 127) / 128, 128, 0, s>>>(partials, n_blocks, n_det, batch, pixel_of_wave, n_pix, o, out, comp);
    MS_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------------------------------------
// Diffraction, |psi|^2, CTEM image transfer, plane wave, conversions
// ------------------------------------------------------------------------------------------------
template <class R>
__global__ void k_diffraction(int n, const cplx<R> *__restrict__ recip, double *__restrict__ out, double *__restrict__ comp) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    cplx<R> v = recip[(size_t)yid * n + xid];
    double re = (double)v.x, im = (double)v.y;
    double e = re * re + im * im;
    size_t oi = (size_t)((yid + n / 2) % n) * n + (xid + n / 2) % n;
    if (comp) {
        double sum = out[oi], c = comp[oi];
        kahan_add(sum, c, e);
        out[oi] = sum;
        comp[oi] = c;
    } else {
        out[oi] = e;
    }
}
template <class R> void diffraction(cudaStream_t s, int n, const cplx<R> *recip, double *out, double *comp) {
    dim3 b(128), gr((n + 127) / 128, n);
    k_diffraction<R><<<gr, b, 0, s>>>(n, recip, out, comp);
    MS_CUDA(cudaGetLastError());
}

// ---- the diffraction pattern translated after a plasmon tilt ---------------------------------------------
// Pixel (X, Y) of |fftshift(recip)|^2 translated by bilinear_translate_d (kernels/bilinear_translate_d.cl:18-77):
// the source pixel (X - ix, Y - iy), wrapped once, and its left, upper and upper-left neighbours (wrapped),
// weighted by the sub-pixel shift (sx, sy); 0 where one wrap does not bring the source into the grid. The
// shifted image at (X', Y') is |recip| ^2 at ((X' + n/2) % n, (Y' + n/2) % n) (fft_shift_d.cl:12-48, even n).
template <class R>
__device__ __forceinline__ double translated_intensity(const cplx<R> *__restrict__ recip, int n, int X, int Y, Shift2 sh) {
    int nx = X - sh.ix, ny = Y - sh.iy;
    if (nx < 0) nx += n; else if (nx >= n) nx -= n;
    if (ny < 0) ny += n; else if (ny >= n) ny -= n;
    if (nx < 0 || nx >= n || ny < 0 || ny >= n) return 0.0;
    const int xl = nx == 0 ? n - 1 : nx - 1, yu = ny == 0 ? n - 1 : ny - 1;   // left and upper neighbours
    auto I = [&](int xs, int ys) {
        const cplx<R> v = recip[(size_t)((ys + n / 2) % n) * n + (xs + n / 2) % n];
        const double re = (double)v.x, im = (double)v.y;
        return re * re + im * im;
    };
    const double f_br = sh.sx * sh.sy, f_bl = (1.0 - sh.sx) * sh.sy;
    const double f_tr = sh.sx * (1.0 - sh.sy), f_tl = (1.0 - sh.sx) * (1.0 - sh.sy);
    return f_tl * I(nx, ny) + f_tr * I(xl, ny) + f_bl * I(nx, yu) + f_br * I(xl, yu);
}

template <class R>
__global__ void k_diffraction_shifted(int n, const cplx<R> *__restrict__ recip, Shift2 sh, double *__restrict__ out,
                                      double *__restrict__ comp) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y;
    if (X >= n) return;
    const double e = translated_intensity<R>(recip, n, X, Y, sh);
    const size_t oi = (size_t)Y * n + X;
    if (comp) {
        double sum = out[oi], c = comp[oi];
        kahan_add(sum, c, e);
        out[oi] = sum;
        comp[oi] = c;
    } else {
        out[oi] = e;
    }
}
template <class R> void diffraction_shifted(cudaStream_t s, int n, const cplx<R> *recip, Shift2 sh, double *out, double *comp) {
    dim3 b(128), gr((n + 127) / 128, n);
    k_diffraction_shifted<R><<<gr, b, 0, s>>>(n, recip, sh, out, comp);
    MS_CUDA(cudaGetLastError());
}

// STEM detectors on the translated pattern (getStemPixel with d_kx, d_ky != 0, simulationstem.cpp:74-132):
// band_pass_d's annulus on the translated |fftshift(recip)|^2 of every wave of a batch (waves n*n apart);
// per block and detector an FP64 partial sum at partials[(wave * n_det + d) * gridDim.x + block]
template <class R>
__global__ void __launch_bounds__(256) k_det_shifted(int n, const cplx<R> *__restrict__ recip, Shift2 sh, int n_det, DetDesc D,
                                                     double *__restrict__ partials) {
    __shared__ double red[8];
    const size_t id = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int X = (int)(id % n), Y = (int)(id / n);
    const bool in = id < (size_t)n * n;
    const double e = in ? translated_intensity<R>(recip + (size_t)blockIdx.y * n * n, n, X, Y, sh) : 0.0;
    for (int d = 0; d < n_det; d++) {
        const double centX = n / 2.0 + D.xc[d], centY = n / 2.0 + D.yc[d];
        const double radius = sqrt((X - centX) * (X - centX) + (Y - centY) * (Y - centY));
        double v = (in && radius <= D.out[d] && radius >= D.in[d]) ? e : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0;
            for (int w = 0; w < (int)(blockDim.x / 32); w++) t += red[w];
            partials[((size_t)blockIdx.y * n_det + d) * gridDim.x + blockIdx.x] = t;
        }
    }
}
template <class R>
int detectors_shifted(cudaStream_t s, int n, int batch, const cplx<R> *recip, Shift2 sh, int n_det, const double *innerPx,
                      const double *outerPx, const double *xcPx, const double *ycPx, double *partials) {
    DetDesc D;
    for (int d = 0; d < 16; d++) {
        D.in[d] = d < n_det ? innerPx[d] : 0;
        D.out[d] = d < n_det ? outerPx[d] : 0;
        D.xc[d] = d < n_det ? xcPx[d] : 0;
        D.yc[d] = d < n_det ? ycPx[d] : 0;
    }
    const int blocks = (int)(((size_t)n * n + 255) / 256);
    k_det_shifted<R><<<dim3(blocks, batch), 256, 0, s>>>(n, recip, sh, n_det, D, partials);
    MS_CUDA(cudaGetLastError());
    return blocks;
}

template <class R>
__global__ void k_sqabs(size_t count, const cplx<R> *__restrict__ in, double *__restrict__ out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    double re = (double)in[i].x, im = (double)in[i].y;
    out[i] = re * re + im * im;
}
template <class R> void sqabs_to_double(cudaStream_t s, size_t count, const cplx<R> *in, double *out) {
    if (!count) return;
    k_sqabs<R><<<(unsigned)((count + 255) / 256), 256, 0, s>>>(count, in, out);
    MS_CUDA(cudaGetLastError());
}

template <class R>
__global__ void k_ctem_transfer(int n, const cplx<R> *__restrict__ input, cplx<R> *__restrict__ output,
                                const double *__restrict__ kx, const double *__restrict__ ky, double wavelength, AberrD A,
                                double obj_ap, double ap_smooth, double beta, double delta) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)yid * n + xid;
    double obj_ap2 = (obj_ap * 0.001) / wavelength;
    double beta2 = (beta * 0.001) / wavelength;
    double k = sqrt((kx[xid] * kx[xid]) + (ky[yid] * ky[yid]));
    double ap_smooth_radius = (ap_smooth * 0.001) / wavelength;
    cplx<R> o = mk<R>(0, 0);
    if (k < obj_ap2 + ap_smooth_radius) {
        double2 w = make_double2(wavelength * kx[xid], wavelength * ky[yid]);
        double temporalCoh = exp(-0.25 * M_PI * M_PI * delta * delta * cModSq(w) * cModSq(w) / (wavelength * wavelength));
        double sp = (A.C10 + A.C30 * cModSq(w) + A.C50 * cModSq(w) * cModSq(w));
        double spatialCoh = exp(-1.0 * M_PI * M_PI * beta2 * beta2 * cModSq(w) * (sp * sp));   // pow(sp, 2), correctly rounded
        double cchi = cchi_of(A, w);
        double chi = 2.0 * M_PI * cchi / wavelength;
        double edge_factor = 1.0;
        if (fabs(k - obj_ap2) < ap_smooth_radius) {
            // smoothstep (OpenCL C 1.2 section 6.12.4): t*t*(3-2t), t = clamp((x-e0)/(e1-e0), 0, 1)
            double e0 = obj_ap2 - ap_smooth_radius, e1 = obj_ap2 + ap_smooth_radius;
            double t = fmin(fmax((k - e0) / (e1 - e0), 0.0), 1.0);
            edge_factor = 1.0 - t * t * (3.0 - 2.0 * t);
        }
        double ix = (double)input[id].x, iy = (double)input[id].y;
        double cc = cos(chi), ss = sin(chi);
        o = mk<R>((R)(edge_factor * temporalCoh * spatialCoh * (ix * cc + iy * ss)),
                  (R)(edge_factor * temporalCoh * spatialCoh * (iy * cc - ix * ss)));
    }
    output[id] = o;
}
template <class R>
void ctem_transfer(cudaStream_t s, int n, const cplx<R> *in, cplx<R> *out, const double *kx, const double *ky,
                   double wavelength, const AberrD &A, double obj_ap, double ap_smooth, double beta, double delta) {
    dim3 b(128), gr((n + 127) / 128, n);
    k_ctem_transfer<R><<<gr, b, 0, s>>>(n, in, out, kx, ky, wavelength, A, obj_ap, ap_smooth, beta, delta);
    MS_CUDA(cudaGetLastError());
}

template <class R>
__global__ void k_plane_state(int n, cplx<R> *__restrict__ wave) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    wave[(size_t)yid * n + xid] = mk<R>(xid == 0 ? (R)n : (R)0, (R)0);
}
template <class R> void plane_wave_state(cudaStream_t s, int n, cplx<R> *wave) {
    dim3 b(128), gr((n + 127) / 128, n);
    k_plane_state<R><<<gr, b, 0, s>>>(n, wave);
    MS_CUDA(cudaGetLastError());
}

template <class R>
__global__ void k_to_double(size_t count, const cplx<R> *__restrict__ in, double2 *__restrict__ out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = make_double2((double)in[i].x, (double)in[i].y);
}
template <class R>
__global__ void k_from_double(size_t count, const double2 *__restrict__ in, cplx<R> *__restrict__ out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = mk<R>((R)in[i].x, (R)in[i].y);
}
template <class R> void convert_to_double(cudaStream_t s, size_t count, const cplx<R> *in, double2 *out) {
    if (!count) return;
    k_to_double<R><<<(unsigned)((count + 255) / 256), 256, 0, s>>>(count, in, out);
    MS_CUDA(cudaGetLastError());
}
template <class R> void convert_from_double(cudaStream_t s, size_t count, const double2 *in, cplx<R> *out) {
    if (!count) return;
    k_from_double<R><<<(unsigned)((count + 255) / 256), 256, 0, s>>>(count, in, out);
    MS_CUDA(cudaGetLastError());
}

// |z|^2 kept as a complex value with zero imaginary part (sqabs_d.cl:11-27 writes double2)
template <class R>
__global__ void k_sqabs_complex(size_t count, cplx<R> *__restrict__ io) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const R re = io[i].x, im = io[i].y;
    io[i] = mk<R>(re * re + im * im, (R)0);
}
template <class R> void sqabs_complex(cudaStream_t s, size_t count, cplx<R> *io) {
    if (!count) return;
    k_sqabs_complex<R><<<(unsigned)((count + 255) / 256), 256, 0, s>>>(count, io);
    MS_CUDA(cudaGetLastError());
}

// ccd_dqe_d / ccd_ntf_d (kernels/ccd_dqe_d.cl:13-50, ccd_ntf_d.cl:13-49): radial table lookup in unshifted
// reciprocal pixels, linear interpolation between entries floor(r/binning) and +1 (clamped at 724), and a
// multiply by sqrt(value) (DQE) or value (NTF)
template <class R>
__global__ void k_ccd_filter(cplx<R> *__restrict__ io, const double *__restrict__ table, int n, int binning, int use_sqrt) {
    int xid = blockIdx.x * blockDim.x + threadIdx.x, yid = blockIdx.y;
    if (xid >= n) return;
    size_t id = (size_t)xid + (size_t)yid * n;
    int midx = xid < n / 2 ? 0 : n;
    int midy = yid < n / 2 ? 0 : n;
    double xp = xid - midx, yp = yid - midy;
    double rad = sqrt(xp * xp + yp * yp);
    int i1 = (int)floor(rad / binning);
    int i2 = i1 + 1;
    double v1 = table[min(i1, 724)], v2 = table[min(i2, 724)];
    double interp = rad / binning - floor(rad / binning);
    double f = interp * v2 + (1 - interp) * v1;
    double m = use_sqrt ? sqrt(f) : f;
    double re = (double)io[id].x, im = (double)io[id].y;
    io[id] = mk<R>((R)(re * m), (R)(im * m));
}
template <class R> void ccd_filter(cudaStream_t s, int n, cplx<R> *io, const double *table, int binning, bool dqe) {
    dim3 b(128), gr((n + 127) / 128, n);
    k_ccd_filter<R><<<gr, b, 0, s>>>(io, table, n, binning, dqe ? 1 : 0);
    MS_CUDA(cudaGetLastError());
}

template <class R>
__global__ void k_real_part(size_t count, const cplx<R> *__restrict__ in, double *__restrict__ out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) out[i] = (double)in[i].x;
}
template <class R> void real_part_to_double(cudaStream_t s, size_t count, const cplx<R> *in, double *out) {
    if (!count) return;
    k_real_part<R><<<(unsigned)((count + 255) / 256), 256, 0, s>>>(count, in, out);
    MS_CUDA(cudaGetLastError());
}

#define MS_INST(R)                                                                                                       \
    template void real_part_to_double<R>(cudaStream_t, size_t, const cplx<R> *, double *);                            \
    template void sqabs_complex<R>(cudaStream_t, size_t, cplx<R> *);                                                    \
    template void ccd_filter<R>(cudaStream_t, int, cplx<R> *, const double *, int, bool);                              \
    template void diffraction<R>(cudaStream_t, int, const cplx<R> *, double *, double *);                               \
    template void diffraction_shifted<R>(cudaStream_t, int, const cplx<R> *, Shift2, double *, double *);               \
    template int detectors_shifted<R>(cudaStream_t, int, int, const cplx<R> *, Shift2, int, const double *,             \
                                      const double *, const double *, const double *, double *);                        \
    template void sqabs_to_double<R>(cudaStream_t, size_t, const cplx<R> *, double *);                                  \
    template void ctem_transfer<R>(cudaStream_t, int, const cplx<R> *, cplx<R> *, const double *, const double *, double, \
                                   const AberrD &, double, double, double, double);                                    \
    template void plane_wave_state<R>(cudaStream_t, int, cplx<R> *);                                                    \
    template void convert_to_double<R>(cudaStream_t, size_t, const cplx<R> *, double2 *);                               \
    template void convert_from_double<R>(cudaStream_t, size_t, const double2 *, cplx<R> *);
MS_INST(float)
MS_INST(double)

}  // namespace ms
