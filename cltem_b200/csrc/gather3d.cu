// gather3d.cu — atom-position gradients of the differentiable CTEM loss under the full 3-D potential.
//
// The full 3-D slice potential (k_potential_3d, potential.cuh; transmission_potentials_full_3d_d.cl) is a
// trapezoid over the sub-slice samples of each bin row: every sample that passes the 8 Å xy and the one-sided
// 3 Å z tests adds (p1 + p2) / 2 for h > 0, where p1 is its own value V(r) and p2 the value of the previous
// passing sample of the same bin row, which belongs to another atom whenever this atom's earlier samples failed
// the z test. So one atom's potential at a pixel depends on its neighbours' samples, and the gradient cannot be
// gathered atom by atom as in gather.cu. Here each thread replays the forward kernel's loops for its pixel in the
// same order (bin rows, atoms, samples, the cumulative tilt shift) and attributes the derivative of every term
// to the atoms whose samples it pairs: dL/d(x, y, z)_a += g/2 dV/dr dr/d(x, y, z)_a for each sample of atom a in
// a term, with g = dL/dV of the pixel times the sub-slice thickness, dr/dx_a = -rx / r (rx the shifted
// offset), dr/dz_a = -rz / r, and zero where the forward clamps r to r_min = dx/4. The tests are discrete
// decisions and contribute nothing. Derivatives are FP64 of the restated forms (potential.cuh kirkland_3,
// peng_3, lobato_3) for both engines. A block's contributions to the atoms of its staged chunk are summed per
// warp, then in shared memory, then added to the FP64 gradient with one atomic per atom and coordinate; the
// pairs that cross atoms add theirs directly. Atomic order varies, so the gradient is reproducible to FP64
// rounding, not bit for bit.
#include "adjoint_ops.h"
#include "potential.cuh"

namespace ms {

// d/dr of kirkland_3 / peng_3 / lobato_3 (potential.cuh)
template <int FORM>
__device__ __forceinline__ double dpot3_dr(const double *__restrict__ prm, int i_lim, int Z, double r) {
    const double pi = M_PI;
    if constexpr (FORM == 0) {   // 150.41 (1/r) sum a e^(-2 pi r sqrt b) + 266.52 sum c d^-3/2 e^(-pi^2 r^2 / d)
        const double *p = prm + (Z - 1) * 12;
        double sl = 0, dsl = 0, dsg = 0;
        for (int i = 0; i < i_lim * 2; i += 2) {
            const double sb = sqrt(p[i + 1]), e = p[i] * exp(-2.0 * pi * r * sb);
            sl += e;
            dsl -= e * 2.0 * pi * sb;
        }
        for (int i = i_lim * 2; i < i_lim * 4; i += 2) {
            const double d = p[i + 1], dir = 1.0 / sqrt(d);
            dsg += p[i] * dir * dir * dir * exp(-pi * pi * r * r / d) * (-2.0 * pi * pi * r / d);
        }
        return 150.4121417 * (dsl / r - sl / (r * r)) + 266.5157269 * dsg;
    } else if constexpr (FORM == 1) {   // 266.52 sum a b^-3/2 e^(-pi^2 r^2 / b)
        const double *p = prm + (Z - 1) * 10;
        double s = 0;
        for (int i = 0; i < i_lim; i++) {
            const double b = p[i + 5], bir = 1.0 / sqrt(b);
            s += p[i] * bir * bir * bir * exp(-pi * pi * r * r / b) * (-2.0 * pi * pi * r / b);
        }
        return 266.5157269 * s;
    } else {   // 472.55 sum a b^-3/2 e^(-2 pi r / sqrt b) (sqrt b / (pi r) + 1)
        const double *p = prm + (Z - 1) * 10;
        double s = 0;
        for (int i = 0; i < i_lim; i++) {
            const double sb = sqrt(p[i + 5]), a = p[i] / (sb * sb * sb);
            const double e = exp(-2.0 * pi * r / sb);
            s += a * e * (-(2.0 * pi / sb) * (sb / (pi * r) + 1.0) - sb / (pi * r * r));
        }
        return 472.545072199968 * s;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// grid (W/16, H/16, count) over slices slice0.. of p, block (16, 16); gV: dL/dV of those slices, wscale: the
// sub-slice thickness; grad: 3 per sorted atom (x, y, z), accumulated
template <int FORM>
__global__ void __launch_bounds__(256)
k_atom_grad_3d(const double *__restrict__ ax, const double *__restrict__ ay, const double *__restrict__ az,
               const int *__restrict__ aZ, const int *__restrict__ block_start, const double *__restrict__ prm, PotParams p,
               const double *__restrict__ gV, double wscale, double *__restrict__ grad) {
    __shared__ double sx[kAtomChunk], sy[kAtomChunk], sz[kAtomChunk];
    __shared__ int sZ[kAtomChunk];
    __shared__ double sg[kAtomChunk][3];
    const int lid = threadIdx.x + 16 * threadIdx.y, lane = lid & 31;
    const int xid = blockIdx.x * 16 + threadIdx.x, yid = blockIdx.y * 16 + threadIdx.y;
    const int slice = blockIdx.z + p.slice0;
    int si, ei, sj, ej;
    tile_bins(p, blockIdx.x, blockIdx.y, si, ei, sj, ej);
    int topz = slice - p.load_z, bottomz = slice + p.load_z;
    const double int_r = 1.0 / p.integrals;
    if (topz < 0) topz = 0;
    if (bottomz >= p.total_slices) bottomz = p.total_slices - 1;
    const double current_z = p.z0 + (p.total_slices - slice) * p.dz;
    const double im_pos_x = p.startx + xid * p.pixelscale;
    const double im_pos_y = p.starty + yid * p.pixelscale;
    const double r_min = 0.25 * p.pixelscale;
    const bool no_shift = p.shift_x == 0.0 && p.shift_y == 0.0;
    const bool inside = xid < p.width && yid < p.height;
    // half the weight of a sample in a term: 1/2 dL/dsum, dsum = the pixel's trapezoid sum
    const double g = inside ? 0.5 * wscale * gV[(size_t)blockIdx.z * p.width * p.height + (size_t)yid * p.width + xid] : 0.0;
    const size_t nb = (size_t)p.blocks_x * p.blocks_y;
    for (int k = topz; k <= bottomz; k++) {
        for (int j = sj; j <= ej; j++) {
            const int start = block_start[k * nb + p.blocks_x * j + si];
            const int end = block_start[k * nb + p.blocks_x * j + ei + 1];
            int prev = -1;                 // sorted index of the atom of the previous passing sample (p2), or none
            double pdx = 0, pdy = 0, pdz = 0;   // that sample's dV/d(x, y, z) of its atom
            for (int c0 = start; c0 < end; c0 += kAtomChunk) {
                const int cn = min(kAtomChunk, end - c0);
                __syncthreads();
                if (lid < cn) {
                    sx[lid] = ax[c0 + lid]; sy[lid] = ay[c0 + lid]; sz[lid] = az[c0 + lid]; sZ[lid] = aZ[c0 + lid];
                    sg[lid][0] = sg[lid][1] = sg[lid][2] = 0.0;
                }
                __syncthreads();
                for (int l = 0; l < cn; l++) {
                    double rad_x = im_pos_x - sx[l];
                    double rad_y = im_pos_y - sy[l];
                    const double xy0 = rad_x * rad_x + rad_y * rad_y;
                    double ox = 0, oy = 0, oz = 0;   // this thread's contributions to atom c0 + l
                    if (!(no_shift && xy0 > 64.0)) {
                        for (int h = 0; h <= p.integrals; h++) {
                            rad_x -= p.shift_x;
                            rad_y -= p.shift_y;
                            const double xyrad2 = no_shift ? xy0 : rad_x * rad_x + rad_y * rad_y;
                            const double rad_z = (current_z - h * p.dz * int_r) - sz[l];
                            if (xyrad2 <= 64.0 && rad_z <= 3.0) {
                                double rad_d = sqrt(xyrad2 + rad_z * rad_z);
                                const bool clamped = rad_d < r_min;
                                if (clamped) rad_d = r_min;
                                const double f = clamped ? 0.0 : dpot3_dr<FORM>(prm, p.i_count, sZ[l], rad_d) / rad_d;
                                const double dxa = -f * rad_x, dya = -f * rad_y, dza = -f * rad_z;
                                if (h != 0) {   // the term (p1 + p2) / 2
                                    ox += g * dxa; oy += g * dya; oz += g * dza;
                                    if (prev == c0 + l) {
                                        ox += g * pdx; oy += g * pdy; oz += g * pdz;
                                    } else if (prev >= 0 && g != 0.0) {   // p2 from another atom's sample
                                        atomicAdd(&grad[3 * (size_t)prev], g * pdx);
                                        atomicAdd(&grad[3 * (size_t)prev + 1], g * pdy);
                                        atomicAdd(&grad[3 * (size_t)prev + 2], g * pdz);
                                    }
                                }
                                prev = c0 + l;
                                pdx = dxa; pdy = dya; pdz = dza;
                            }
                        }
                    }
                    // the block's sum for atom c0 + l: per warp, then in shared memory
                    ox = warp_sum(ox); oy = warp_sum(oy); oz = warp_sum(oz);
                    if (lane == 0 && (ox != 0.0 || oy != 0.0 || oz != 0.0)) {
                        atomicAdd(&sg[l][0], ox);
                        atomicAdd(&sg[l][1], oy);
                        atomicAdd(&sg[l][2], oz);
                    }
                }
                __syncthreads();
                if (lid < cn && (sg[lid][0] != 0.0 || sg[lid][1] != 0.0 || sg[lid][2] != 0.0)) {
                    atomicAdd(&grad[3 * (size_t)(c0 + lid)], sg[lid][0]);
                    atomicAdd(&grad[3 * (size_t)(c0 + lid) + 1], sg[lid][1]);
                    atomicAdd(&grad[3 * (size_t)(c0 + lid) + 2], sg[lid][2]);
                }
            }
        }
    }
}

void atom_grad_3d(cudaStream_t s, int form, const double *ax, const double *ay, const double *az, const int *aZ,
                  const int *block_start, const double *prm, const PotParams &p, int count, const double *gV,
                  double wscale, double *grad) {
    if (count <= 0) return;
    const dim3 grd((p.width + 15) / 16, (p.height + 15) / 16, count), blk(16, 16);
    if (form == 0) k_atom_grad_3d<0><<<grd, blk, 0, s>>>(ax, ay, az, aZ, block_start, prm, p, gV, wscale, grad);
    else if (form == 1) k_atom_grad_3d<1><<<grd, blk, 0, s>>>(ax, ay, az, aZ, block_start, prm, p, gV, wscale, grad);
    else k_atom_grad_3d<2><<<grd, blk, 0, s>>>(ax, ay, az, aZ, block_start, prm, p, gV, wscale, grad);
    MS_CUDA(cudaGetLastError());
}

}  // namespace ms
