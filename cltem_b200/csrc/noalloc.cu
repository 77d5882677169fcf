// noalloc.cu — atom binning that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application that owns the whole device-memory budget
// through its own pool (and rejects allocations it did not make), or a pipeline stage that must not pay
// cudaMalloc/cudaFree's latency and implicit device synchronisation between two of its launches. For
// them, mslice_bin_atoms_noalloc runs the same binning as mslice_set_atoms on device buffers the caller
// already owns, and keeps its working memory (sort keys, indices, per-bin counts and the radix-sort
// temporary storage) in one fixed array of device memory that is part of the loaded library.
#include "../../include/mslice.h"
#include "misc.cuh"

#include <cmath>
#include <string>

namespace ms {
void set_last_error(const std::string &msg);   // engine.cu
}

namespace {

// The library's scratch for mslice_bin_atoms_noalloc: 8 MiB of device memory, present on every device
// that loads the library until the process exits. Host code must not use the symbol's address directly
// (on the host it names a stand-in, not device memory); the device address comes from
// cudaGetSymbolAddress below.
constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr size_t kMaxAtoms = 131072;
constexpr size_t kMaxBins = 65535;
__device__ __align__(256) unsigned char g_bin_scratch[kScratchBytes];

// Device address of g_bin_scratch on the current device. It is looked up on every call (the lookup is
// cheap), so an address cached before a device reset or a primary-context teardown is never reused.
void *scratch_address() {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_bin_scratch);
    if (e != cudaSuccess || p == nullptr)
        throw ms::CudaError(std::string("cudaGetSymbolAddress of the binning scratch failed: ") + cudaGetErrorString(e));
    return p;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace

extern "C" int mslice_bin_atoms_noalloc(const mslice_geometry *geo, const int *Z, const double *x, const double *y,
                                        const double *z, size_t n, int *block_start, int *Z_sorted, double *x_sorted,
                                        double *y_sorted, double *z_sorted, void *stream) {
    try {
        if (!geo || !block_start || (n && (!Z || !x || !y || !z || !Z_sorted || !x_sorted || !y_sorted || !z_sorted)))
            throw std::invalid_argument("null argument");
        if (geo->n_slices < 1 || geo->blocks_x < 1 || geo->blocks_y < 1 || !(geo->dz > 0))
            throw std::invalid_argument("geometry is not initialised (use mslice_geometry_compute)");
        // the limits must be ordered and the slice count must cover z_lims as mslice_geometry_compute makes it
        // (sliceCount, simulationcell.cpp:75-83), so every kept atom's slice index lies below n_slices
        if (!(geo->full_x[1] > geo->full_x[0]) || !(geo->full_y[1] > geo->full_y[0]) || !(geo->z_lims[1] > geo->z_lims[0]))
            throw std::invalid_argument("geometry limits are empty or reversed");
        if ((double)geo->n_slices < std::ceil((geo->z_lims[1] - geo->z_lims[0]) / geo->dz - 0.000001))
            throw std::invalid_argument("geometry: n_slices does not cover z_lims at slice thickness dz");
        const size_t n_bins = (size_t)geo->n_slices * geo->blocks_x * geo->blocks_y;
        if (n > kMaxAtoms)
            throw std::invalid_argument("mslice_bin_atoms_noalloc: " + std::to_string(n) + " atoms exceed its limit of " +
                                        std::to_string(kMaxAtoms));
        if (n_bins > kMaxBins)
            throw std::invalid_argument("mslice_bin_atoms_noalloc: " + std::to_string(n_bins) +
                                        " bins (slices x blocks) exceed its limit of " + std::to_string(kMaxBins));
        // carve the fixed scratch: seven per-atom int arrays, the bin counts, the radix-sort storage
        const size_t per_atom = align256(sizeof(int) * (n ? n : 1));
        const size_t counts_bytes = align256(sizeof(int) * (n_bins + 1));
        const size_t cub_bytes = ms::atom_sort_temp_bytes((int)(n ? n : 1), (int)n_bins);
        if (7 * per_atom + counts_bytes + cub_bytes > kScratchBytes)
            throw std::invalid_argument("mslice_bin_atoms_noalloc: this size needs more than the 8 MiB of scratch");
        unsigned char *base = (unsigned char *)scratch_address();
        ms::AtomSortBuffers b;
        b.keys_in = (int *)(base + 0 * per_atom);
        b.keys_out = (int *)(base + 1 * per_atom);
        b.idx_in = (int *)(base + 2 * per_atom);
        b.idx_out = (int *)(base + 3 * per_atom);
        b.bid = (int *)(base + 4 * per_atom);
        b.zid = (int *)(base + 5 * per_atom);
        b.kept = (int *)(base + 6 * per_atom);
        b.counts = (int *)(base + 7 * per_atom);                 // zeroed on the stream by atom_sort
        b.cub_temp = base + 7 * per_atom + counts_bytes;
        b.cub_temp_bytes = cub_bytes;
        ms::SortGeom g;
        g.full_x0 = geo->full_x[0]; g.full_x1 = geo->full_x[1];
        g.full_y0 = geo->full_y[0]; g.full_y1 = geo->full_y[1];
        g.z0 = geo->z_lims[0]; g.z1 = geo->z_lims[1]; g.dz = geo->dz;
        g.blocks_x = geo->blocks_x; g.blocks_y = geo->blocks_y; g.n_slices = geo->n_slices;
        ms::atom_sort((cudaStream_t)stream, g, (int)n, Z, x, y, z, b, block_start, Z_sorted, x_sorted, y_sorted, z_sorted);
        return MSLICE_OK;
    } catch (const ms::CudaError &e) {
        ms::set_last_error(e.what());
        return MSLICE_ERR_CUDA;
    } catch (const std::exception &e) {
        ms::set_last_error(e.what());
        return MSLICE_ERR_ARG;
    }
}
