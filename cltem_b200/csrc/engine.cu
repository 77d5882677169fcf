// engine.cu — host side of the multislice engine and the C ABI of include/mslice.h.
//
// The simulation object mirrors clTEM's SimulationGeneral / SimulationStem / SimulationCbed /
// SimulationCtem state (src/simulation/microscope/*.cpp): geometry derived from the config as
// SimulationManager / SimulationCell do, binned atoms, the band-limited transmission function of every
// slice, and a batch of waves that the fused row / column passes (passes.cuh) step through the slices.
#include "../../include/mslice.h"
#include "adjoint_ops.h"
#include "draws.h"
#include "fft.cuh"
#include "fft_wide.cuh"
#include "launch.cuh"
#include "misc.cuh"
#include "plain.h"
#include "potential.cuh"
#include "potential_launch.h"

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

namespace ms {

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }

struct ArgError : std::runtime_error { using std::runtime_error::runtime_error; };
struct StateError : std::runtime_error { using std::runtime_error::runtime_error; };
struct OomError : std::runtime_error { using std::runtime_error::runtime_error; };
struct Cancelled : std::runtime_error { using std::runtime_error::runtime_error; };
struct Unsupported : std::runtime_error { using std::runtime_error::runtime_error; };

// ------------------------------------------------------------------------------------------------
// Geometry (host): SimulationArea / SimulationCell / SimulationManager / MicroscopeParameters
// ------------------------------------------------------------------------------------------------
static const double kPi = M_PI;

static double wavelength_of(double V) {   // commonstructs.h:269-271
    const double h = 6.6262e-034, c = 299792458.0, e = 1.6021773e-019, m = 9.10938291e-031;
    return h * c / std::sqrt(e * (V * 1000) * (2 * m * c * c + e * (V * 1000))) * 1e+10;
}
static double sigma_of(double V) {   // commonstructs.h:278-280
    const double c = 299792458.0, e = 1.6021773e-019, m = 9.10938291e-031;
    return (2 * kPi / (wavelength_of(V) * (V * 1000))) * (m * c * c + e * (V * 1000)) / (2 * m * c * c + e * (V * 1000));
}

static bool valid_resolution(const mslice_config &c) {
    int r = c.resolution;
    if (c.allow_any_resolution) {
        int m = r % 3 == 0 ? r / 3 : r;
        return r >= 64 && (m & (m - 1)) == 0;
    }
    return r == 256 || r == 512 || r == 768 || r == 1024 || r == 1536 || r == 2048 || r == 3072 || r == 4096 || r == 8192;
}

static void corrected_limits(double xs, double xf, double ys, double yf, double pad, double *x, double *y) {
    // SimulationArea::getCorrectedLimitsX/Y (commonstructs.cpp:33-59)
    double range_x = xf - xs, range_y = yf - ys;
    double range_total = std::max(range_x, range_y) + pad;
    double x_diff = (range_total - range_x) / 2, y_diff = (range_total - range_y) / 2;
    x[0] = xs - x_diff; x[1] = xf + x_diff;
    y[0] = ys - y_diff; y[1] = yf + y_diff;
}

struct HostGeom {
    mslice_geometry g;
    std::vector<double> kx, ky;
};

// Moving STEM frame: paddedSimLimitsX/Y(pixel) when the static area is off
// (SimulationManager::currentAreaBase, simulationmanager.cpp:485-505; StemArea::getPixelSimArea,
// commonstructs.h:379-396). The window of stem_padding sits at the scan origin plus the pixel's offset
// rounded down to the pixel size of the static frame; the SimulationCell padding is added around it.
static void stem_frame(const mslice_config &c, int pixel, double x[2], double y[2]) {
    double fx[2], fy[2];
    corrected_limits(c.stem_area[0], c.stem_area[1], c.stem_area[2], c.stem_area[3], c.stem_padding, fx, fy);
    const double pad_range = c.padding_xy - (-c.padding_xy);
    const double rs = (pad_range + (fx[1] - fx[0])) / static_cast<double>(c.resolution);
    const unsigned int x_px = (unsigned int)pixel % (unsigned int)c.stem_pixels_x;
    const unsigned int y_px = (unsigned int)std::floor(pixel / c.stem_pixels_x);
    const double pos_x = (c.stem_area[1] - c.stem_area[0]) / c.stem_pixels_x * x_px;
    const double pos_y = (c.stem_area[3] - c.stem_area[2]) / c.stem_pixels_y * y_px;
    const double xp = c.stem_area[0] + rs * std::floor(pos_x / rs), yp = c.stem_area[2] + rs * std::floor(pos_y / rs);
    corrected_limits(xp, xp, yp, yp, c.stem_padding, x, y);
    x[0] += -c.padding_xy; x[1] += c.padding_xy;
    y[0] += -c.padding_xy; y[1] += c.padding_xy;
}

static void compute_geometry(const mslice_config &c, HostGeom &H) {
    if (c.mode != MSLICE_MODE_CTEM && c.mode != MSLICE_MODE_STEM && c.mode != MSLICE_MODE_CBED)
        throw ArgError("unknown simulation mode " + std::to_string(c.mode));
    if (!valid_resolution(c)) throw ArgError("invalid resolution " + std::to_string(c.resolution));
    if (!(c.slice_thickness > 0)) throw ArgError("slice thickness must be positive");
    if (!(c.voltage > 0)) throw ArgError("voltage must be positive");
    if (c.full3d && c.full3d_integrals < 1) throw ArgError("full 3d integrals must be >= 1");
    if (c.n_detectors < 0 || c.n_detectors > MSLICE_MAX_DETECTORS) throw ArgError("too many detectors");
    if (c.mode == MSLICE_MODE_STEM && (c.stem_pixels_x < 1 || c.stem_pixels_y < 1)) throw ArgError("STEM scan needs pixels");
    if (c.iterations < 0 || c.mixed_static < 0 || c.stem_job_pixels < 0) throw ArgError("negative incoherence count");
    if (c.stem_moving_frame && c.mode != MSLICE_MODE_STEM) throw ArgError("the moving frame is a STEM option");
    if (c.mixed_static > 1 && c.stem_moving_frame)
        throw Unsupported("mixed static potentials with the moving STEM frame are not supported");
    if (c.chromatic && !(c.chromatic_cc >= 0)) throw ArgError("chromatic Cc must be >= 0");
    if (c.plasmon) {
        if (!(c.plasmon_mfp > 0) || !(c.plasmon_char_angle > 0) || !(c.plasmon_crit_angle >= 0) || c.plasmon_individual < 0)
            throw ArgError("plasmon settings need a positive mean free path and characteristic angle");
        // plasmons turn precalculated transmissions off, and with them mixed static potentials
        // (SimulationManager::parallelPotentialsCount, simulationmanager.h:185-232)
        if (c.mixed_static > 1) throw Unsupported("mixed static potentials are off when plasmons are on");
    }
    if (c.source_size && !(c.source_fwhm >= 0)) throw ArgError("source size FWHM must be >= 0");
    mslice_geometry &g = H.g;
    std::memset(&g, 0, sizeof(g));
    double fx[2], fy[2];
    if (c.mode == MSLICE_MODE_STEM)
        corrected_limits(c.stem_area[0], c.stem_area[1], c.stem_area[2], c.stem_area[3], c.stem_padding, fx, fy);
    else if (c.mode == MSLICE_MODE_CBED)
        corrected_limits(c.cbed_x, c.cbed_x, c.cbed_y, c.cbed_y, c.cbed_padding, fx, fy);
    else
        corrected_limits(c.ctem_area[0], c.ctem_area[1], c.ctem_area[2], c.ctem_area[3], 0.0, fx, fy);
    // + SimulationCell padding (paddedFullLimitsX/Y, simulationmanager.cpp:446-452)
    fx[0] += -c.padding_xy; fx[1] += c.padding_xy;
    fy[0] += -c.padding_xy; fy[1] += c.padding_xy;
    g.full_x[0] = g.sim_x[0] = fx[0]; g.full_x[1] = g.sim_x[1] = fx[1];
    g.full_y[0] = g.sim_y[0] = fy[0]; g.full_y[1] = g.sim_y[1] = fy[1];
    if (c.mode == MSLICE_MODE_STEM && c.stem_moving_frame) stem_frame(c, 0, g.sim_x, g.sim_y);   // paddedSimLimitsX/Y(0)

    // SimulationCell::roundPaddingZ (simulationcell.cpp:43-61) and sliceCount (:75-83)
    const double dz = c.slice_thickness, off = c.slice_offset;
    int pad_slices_pre = (int)std::ceil((std::abs(c.padding_z) - off) / dz);
    double pre_pad = off + pad_slices_pre * dz;
    double zw = c.struct_limits[5] - c.struct_limits[4];
    int struct_slices = (int)std::ceil((zw + off) / dz);
    double left_over = struct_slices * dz - off - zw;
    int pad_slices_post = (int)std::ceil((std::abs(-c.padding_z) - left_over) / dz);
    double post_pad = pad_slices_post * dz + left_over;
    g.padding_z[0] = -post_pad; g.padding_z[1] = pre_pad;
    g.z_lims[0] = c.struct_limits[4] + g.padding_z[0];
    g.z_lims[1] = c.struct_limits[5] + g.padding_z[1];
    unsigned int ns = (unsigned int)std::ceil(((g.z_lims[1] - g.z_lims[0]) / dz) - 0.000001);
    ns += (ns == 0);
    g.n_slices = (int)ns;
    g.pre_slices = (int)(unsigned int)(g.padding_z[1] / dz);
    g.dz = dz;

    const int res = c.resolution;
    double x_r = g.sim_x[1] - g.sim_x[0], y_r = g.sim_y[1] - g.sim_y[0];
    g.real_scale = std::max(x_r, y_r) / res;                 // simulationmanager.cpp:211-222
    g.inverse_scale = 1.0 / (g.real_scale * res);            // :224-230
    g.wavelength = wavelength_of(c.voltage);
    g.wavenumber = 1.0 / g.wavelength;
    g.angle_scale = 1000.0 * g.inverse_scale * g.wavelength;  // :241-247
    const double k = g.wavenumber;
    g.wavevector[0] = k * std::sin(c.beam_tilt / 1000.0) * std::cos(c.beam_azimuth);
    g.wavevector[1] = k * std::sin(c.beam_tilt / 1000.0) * std::sin(c.beam_azimuth);
    g.wavevector[2] = k * std::cos(c.beam_tilt / 1000.0);
    g.sigma = sigma_of(c.voltage) * g.wavenumber / g.wavevector[2];   // simulationgeneral.cpp:418

    double xr = g.full_x[1] - g.full_x[0], yr = g.full_y[1] - g.full_y[0];
    int nb = (int)std::ceil(std::max(xr, yr) / 8.0);            // calculateBlocks :393-408
    if (nb < 1) throw ArgError("empty simulation area");
    g.blocks_x = g.blocks_y = nb;
    g.block_scale_x = xr / nb; g.block_scale_y = yr / nb;
    g.load_blocks_x = (int)std::ceil(8.0 / g.block_scale_x);    // simulationgeneral.cpp:517-521
    g.load_blocks_y = (int)std::ceil(8.0 / g.block_scale_y);
    g.load_blocks_z = (int)std::ceil(3.0 / dz);

    // k tables + bandwidth k_max (simulationgeneral.cpp:427-455)
    const double L = g.real_scale * res;
    H.kx.resize(res); H.ky.resize(res);
    unsigned int imid = (unsigned int)std::floor(static_cast<double>(res) / 2.0 + 0.5);
    for (int i = 0; i < res; i++) H.kx[i] = H.ky[i] = (i >= (int)imid) ? double(i - res) / L : i / L;
    g.k_max = std::min(std::abs(H.ky[imid]), std::abs(H.kx[imid]));

    double rx0, rx1, ry0, ry1;   // raw limits of the mode's area (imageCrop, :410-428)
    if (c.mode == MSLICE_MODE_STEM) { rx0 = c.stem_area[0]; rx1 = c.stem_area[1]; ry0 = c.stem_area[2]; ry1 = c.stem_area[3]; }
    else if (c.mode == MSLICE_MODE_CBED) { rx0 = rx1 = c.cbed_x; ry0 = ry1 = c.cbed_y; }
    else { rx0 = c.ctem_area[0]; rx1 = c.ctem_area[1]; ry0 = c.ctem_area[2]; ry1 = c.ctem_area[3]; }
    double crop_lr = (std::floor(x_r - (rx1 - rx0)) / g.real_scale);
    double crop_tb = (std::floor(y_r - (ry1 - ry0)) / g.real_scale);
    unsigned int cl = (unsigned int)std::floor(crop_lr / 2.0), cb = (unsigned int)std::floor(crop_tb / 2.0);
    g.crop[0] = (unsigned int)(crop_tb - cb); g.crop[1] = cl; g.crop[2] = cb; g.crop[3] = (unsigned int)(crop_lr - cl);
    g.n_outputs = c.intermediate_slices > 0 ? (int)std::ceil((float)g.n_slices / c.intermediate_slices) : 1;
}

// output slices: (s+1) % step == 0, then the exit if the count is not reached (simulationstem.cpp:237-275)
static std::vector<int> output_slices(const mslice_config &c, const mslice_geometry &g) {
    std::vector<int> o;
    if (c.intermediate_slices > 0)
        for (int s = 0; s < g.n_slices; s++)
            if ((s + 1) % c.intermediate_slices == 0) o.push_back(s);
    if ((int)o.size() < g.n_outputs) o.push_back(g.n_slices - 1);
    return o;
}

// ------------------------------------------------------------------------------------------------
// Context
// ------------------------------------------------------------------------------------------------
struct Params {
    int form = -1, i_count = 0;
    std::vector<double> values;
    int max_z = 0;
};

// The per-element term table of the FP32 full-3D kernel (potential.cuh, k_potential_3d_f): for each element
// Z = 1..max_z and term, float4 at (Z - 1) * kPot3Terms + term, formed in FP64 from the parameterisation
// table `v` (12 values per element for Kirkland, 10 for Peng / Lobato) and rounded once.
std::vector<float4> pot3_table(int form, int i_count, const std::vector<double> &v, int max_z) {
    constexpr double kLog2e = 1.44269504088896340736;
    std::vector<float4> t((size_t)std::max(max_z, 0) * kPot3Terms, make_float4(0, 0, 0, 0));
    const int stride = form == 0 ? 12 : 10;
    for (int Z = 1; Z <= max_z; Z++) {
        const double *q = v.data() + (size_t)(Z - 1) * stride;
        float4 *o = t.data() + (size_t)(Z - 1) * kPot3Terms;
        for (int i = 0; i < i_count; i++) {
            if (form == 2) {   // Lobato
                const double b = q[i + 5];
                if (!(b > 0)) continue;
                const double bir = 1.0 / std::sqrt(b);
                o[i] = make_float4((float)(472.545072199968 * q[i] * (bir * bir * bir)), (float)(-2.0 * M_PI * bir * kLog2e),
                                   (float)(std::sqrt(b) / M_PI), 0.0f);
            } else if (form == 1) {   // Peng
                const double b = q[i + 5];
                if (!(b > 0)) continue;
                const double bir = 1.0 / std::sqrt(b);
                o[i] = make_float4((float)(266.5157269 * q[i] * (bir * bir * bir)), 0.0f, 0.0f,
                                   (float)(-M_PI * M_PI / b * kLog2e));
            } else {   // Kirkland: Lorentzian terms at 0..2, Gaussian terms at 3..5
                const double a = q[2 * i], b = q[2 * i + 1];
                if (b >= 0) o[i] = make_float4((float)(150.4121417 * a), (float)(-2.0 * M_PI * std::sqrt(b) * kLog2e), 0.0f, 0.0f);
                const double c = q[2 * i_count + 2 * i], d = q[2 * i_count + 2 * i + 1];
                if (d > 0) {
                    const double dir = 1.0 / std::sqrt(d);
                    o[3 + i] = make_float4((float)(266.5157269 * c * (dir * dir * dir)), 0.0f, 0.0f,
                                           (float)(-M_PI * M_PI / d * kLog2e));
                }
            }
        }
    }
    return t;
}

// The per-element term table of the FP32 projected kernel (potential.cuh, k_potential_projected_f): for each
// element Z = 1..max_z and term, float2 at (Z - 1) * kPotPTerms + term, formed in FP64 and rounded once.
// Terms the parameterisation does not use are (0, 1): a zero weight on a finite K0(r), K1(r) or exp2(r²)
// (a zero argument would make K0 infinite and the zero term NaN).
std::vector<float2> potp_table(int form, int i_count, const std::vector<double> &v, int max_z) {
    constexpr double kLog2e = 1.44269504088896340736;
    std::vector<float2> t((size_t)std::max(max_z, 0) * kPotPTerms, make_float2(0, 1));
    const int stride = form == 0 ? 12 : 10;
    for (int Z = 1; Z <= max_z; Z++) {
        const double *q = v.data() + (size_t)(Z - 1) * stride;
        float2 *o = t.data() + (size_t)(Z - 1) * kPotPTerms;
        for (int i = 0; i < i_count; i++) {
            if (form == 2) {   // Lobato
                const double b = q[i + 5];
                if (!(b > 0)) continue;
                const double bir = 1.0 / std::sqrt(b);
                o[i] = make_float2((float)(945.090144399935 * q[i] * (bir * bir * bir)), (float)(2.0 * M_PI * bir));
            } else if (form == 1) {   // Peng
                const double b = q[i + 5];
                if (!(b > 0)) continue;
                o[i] = make_float2((float)(150.4121417 * q[i] / b), (float)(-M_PI * M_PI / b * kLog2e));
            } else {   // Kirkland: K0 terms at 0..2, Gaussian terms at 3..5
                const double a = q[2 * i], b = q[2 * i + 1];
                if (b > 0) o[i] = make_float2((float)(300.8242834 * a), (float)(2.0 * M_PI * std::sqrt(b)));
                const double c = q[2 * i_count + 2 * i], d = q[2 * i_count + 2 * i + 1];
                if (d > 0) o[3 + i] = make_float2((float)(150.4121417 * c / d), (float)(-M_PI * M_PI / d * kLog2e));
            }
        }
    }
    return t;
}

// A twiddle (cos a, sin a) rounded to R. FP32: of the roundings down and up of its two parts, the pair whose
// squared modulus is closest to 1 (then the nearest): an FFT round trip multiplies by |w|^2, and a modulus
// error would repeat at every slice and add up with thickness, while a phase error of up to an ulp does not
// (the inverse transform's conjugate twiddle undoes it). FP64: the nearest doubles.
template <class R> cplx<R> round_unit(long double c, long double s) {
    if constexpr (sizeof(R) == 8) {
        return mk<R>((R)c, (R)s);
    } else {
        auto down = [](long double v) { float f = (float)v; return (long double)f > v ? std::nextafter(f, -2.0f) : f; };
        auto up = [](long double v) { float f = (float)v; return (long double)f < v ? std::nextafter(f, 2.0f) : f; };
        const float cs[2] = {down(c), up(c)}, ss[2] = {down(s), up(s)};
        float bc = (float)c, bs = (float)s;
        long double best_m = std::fabs((long double)bc * bc + (long double)bs * bs - 1.0L);
        long double best_d = std::fabs((long double)bc - c) + std::fabs((long double)bs - s);
        for (float cc : cs)
            for (float sc : ss) {
                const long double m = std::fabs((long double)cc * cc + (long double)sc * sc - 1.0L);
                const long double d = std::fabs((long double)cc - c) + std::fabs((long double)sc - s);
                if (m < best_m || (m == best_m && d < best_d)) { best_m = m; best_d = d; bc = cc; bs = sc; }
            }
        return mk<R>(bc, bs);
    }
}

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t mem_limit = 0, mem_used = 0;
    unsigned long long launches = 0;
    Params params;
    double *prm_d = nullptr;
    float *prm_f = nullptr;
    size_t prm_n = 0;
    float4 *pot3_tab = nullptr;   // pot3_table of the loaded parameterisation (FP32 full-3D kernel)
    size_t pot3_n = 0;
    float2 *potp_tab = nullptr;   // potp_table of the loaded parameterisation (FP32 projected kernel)
    size_t potp_n = 0;
    std::map<int, void *> tw_f, tw_d;   // twiddle tables per size
    std::mutex mtx;
    int *step_err = nullptr;   // error word of the persistent step passes (tma.cuh StepError; 0 = none)

    void *alloc(size_t bytes) {
        if (bytes == 0) return nullptr;
        if (mem_limit && mem_used + bytes > mem_limit) throw OomError("device memory limit of the context exceeded");
        void *p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); throw OomError("cudaMalloc of " + std::to_string(bytes) + " bytes failed"); }
        MS_CUDA(e);
        mem_used += bytes;
        return p;
    }
    void release(void *p, size_t bytes) {
        if (!p) return;
        cudaFree(p);
        mem_used -= std::min(mem_used, bytes);
    }
    template <class R> const cplx<R> *twiddles(int n) {
        auto &m = sizeof(R) == 4 ? tw_f : tw_d;
        auto it = m.find(n);
        if (it != m.end()) return (const cplx<R> *)it->second;
        // entries [0, n): the radix-8 plan's packed per-stage table (fft.cuh, plan_tw_index),
        // W_n^(r*k*n/(Ns*R)) = exp(-2 pi i r k / (Ns*R)); for sizes whose row passes use the wide two-stage
        // plan (fft_wide.cuh) entries [n, 2n) hold its table, W_n^(r k) at k (R2 - 1) + r - 1; for the
        // three-stage wide plan and the radix-24 plans they hold their stages' tables in the packed layout
        // (Wide3Plan::tw_base, Wide24Plan::tw_base)
        // (FP32 at 1024, 2048 and 4096: entries [2n, 3n) hold the 16-element column plan's table, Plan16::tw_base)
        const bool wide = wide_plan<R>(n), wide3 = !wide && wide3_plan<R>(n), wide24 = wide24_plan<R>(n);
        const bool p16 = sizeof(R) == 4 && plan16_ok(n);
        const size_t count = (size_t)n * (p16 ? 3 : ((wide || wide3 || wide24) ? 2 : 1));
        std::vector<cplx<R>> h(count, mk<R>(0, 0));
        const long double two_pi = 2.0L * 3.14159265358979323846264338327950288L;
        for (int s = 1; s < plan_nstages(n); s++) {
            const int Ns = plan_ns(n, s), RAD = plan_radix(n, s);
            for (int k = 0; k < Ns; k++)
                for (int r = 1; r < RAD; r++) {
                    long double a = -two_pi * (long double)(r * k) / (long double)(Ns * RAD);
                    h[plan_tw_index(n, s, k, r)] = round_unit<R>(std::cos(a), std::sin(a));
                }
        }
        if (wide3 || wide24) {
            auto fill = [&](auto plan) {
                using P = decltype(plan);
                for (int st = 1; st < P::nstages; st++) {
                    const int Ns = P::ns(st), RAD = P::radix(st);
                    for (int k = 0; k < Ns; k++)
                        for (int r = 1; r < RAD; r++) {
                            long double a = -two_pi * (long double)(r * k) / (long double)(Ns * RAD);
                            h[n + P::tw_base(st) + k * (RAD - 1) + (r - 1)] = round_unit<R>(std::cos(a), std::sin(a));
                        }
                }
            };
            if (n == 2048) fill(Wide3Plan<2048>());
            else if (n == 4096) fill(Wide3Plan<4096>());
            else if (n == 8192) fill(Wide3Plan<8192>());
            else if (n == 384) fill(Wide24Plan<384>());
            else if (n == 768) fill(Wide24Plan<768>());
            else if (n == 1536) fill(Wide24Plan<1536>());
            else fill(Wide24Plan<3072>());
        }
        if (p16) {
            auto fill16 = [&](auto plan) {
                using P = decltype(plan);
                for (int st = 1; st < P::nstages; st++) {
                    const int Ns = P::ns(st), RAD = P::radix(st);
                    for (int k = 0; k < Ns; k++)
                        for (int r = 1; r < RAD; r++) {
                            long double a = -two_pi * (long double)(r * k) / (long double)(Ns * RAD);
                            h[2 * (size_t)n + P::tw_base(st) + k * (RAD - 1) + (r - 1)] = round_unit<R>(std::cos(a), std::sin(a));
                        }
                }
            };
            if (n == 1024) fill16(Plan16<1024>());
            else if (n == 2048) fill16(Plan16<2048>());
            else fill16(Plan16<4096>());
        }
        if (wide) {
            const int E = wide_E(n), R2 = n / E;
            for (int k = 0; k < E; k++)
                for (int r = 1; r < R2; r++) {
                    long double a = -two_pi * (long double)(r * k) / (long double)n;
                    h[n + k * (R2 - 1) + (r - 1)] = round_unit<R>(std::cos(a), std::sin(a));
                }
        }
        void *d = alloc(sizeof(cplx<R>) * count);
        MS_CUDA(cudaMemcpy(d, h.data(), sizeof(cplx<R>) * count, cudaMemcpyHostToDevice));
        m[n] = d;
        return (const cplx<R> *)d;
    }
    ~Ctx() {
        cudaSetDevice(device);
        cudaFree(step_err);
        for (auto &kv : tw_f) cudaFree(kv.second);
        for (auto &kv : tw_d) cudaFree(kv.second);
        cudaFree(prm_d);
        cudaFree(prm_f);
        cudaFree(pot3_tab);
        cudaFree(potp_tab);
        if (stream) cudaStreamDestroy(stream);
    }
};

template <class T> struct DevBuf {
    Ctx *ctx = nullptr;
    T *p = nullptr;
    size_t n = 0;
    void ensure(Ctx *c, size_t count) {
        if (count <= n && p) return;
        free();
        ctx = c;
        p = (T *)c->alloc(sizeof(T) * std::max<size_t>(count, 1));
        n = std::max<size_t>(count, 1);
    }
    void free() {
        if (p && ctx) ctx->release(p, sizeof(T) * n);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { free(); }
};

// ------------------------------------------------------------------------------------------------
// Simulation
// ------------------------------------------------------------------------------------------------
struct SimBase {
    Ctx *ctx;
    mslice_config cfg;
    bool adj_valid = false;   // the state of the last adjoint forward is intact (Sim::ctem_forward)
    HostGeom H;
    std::atomic<bool> cancel{false};
    mslice_progress_cb progress = nullptr;
    void *progress_user = nullptr;
    double timing[3] = {0, 0, 0};
    // per-kernel event timing (mslice_profile_enable)
    bool prof = false;
    double prof_ms[MSLICE_K_COUNT] = {};
    double prof_bytes[MSLICE_K_COUNT] = {};
    unsigned long long prof_n[MSLICE_K_COUNT] = {};
    struct Pending { int kind; cudaEvent_t a, b; double bytes; bool graph_owned = false; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> ev_pool;
    cudaEvent_t take_event() {
        if (!ev_pool.empty()) { cudaEvent_t e = ev_pool.back(); ev_pool.pop_back(); return e; }
        cudaEvent_t e;
        MS_CUDA(cudaEventCreate(&e));
        return e;
    }
    template <class F> void timed(cudaStream_t s, int kind, double bytes, F &&launch) {
        if (!prof) { launch(); return; }
        // inside a stream capture a plain record only orders the capture; the external flag makes it a
        // record node of the graph, so every replay records the event
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        MS_CUDA(cudaStreamIsCapturing(s, &cs));
        const unsigned flags = cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
        cudaEvent_t a = take_event(), b = take_event();
        MS_CUDA(cudaEventRecordWithFlags(a, s, flags));
        launch();
        MS_CUDA(cudaEventRecordWithFlags(b, s, flags));
        pending.push_back({kind, a, b, bytes});
    }
    // after a stream sync: fold the recorded launch durations into the totals. The pending list is taken
    // over first, so an error part-way leaves no event listed twice (the remaining ones are destroyed).
    void flush_profile() {
        std::vector<Pending> todo;
        todo.swap(pending);
        size_t i = 0;
        try {
            for (; i < todo.size(); i++) {
                const Pending &p = todo[i];
                float ms = 0;
                MS_CUDA(cudaEventSynchronize(p.b));
                MS_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
                prof_ms[p.kind] += ms;
                prof_bytes[p.kind] += p.bytes;
                prof_n[p.kind]++;
                if (p.graph_owned) continue;
                ev_pool.push_back(p.a);
                ev_pool.push_back(p.b);
            }
        } catch (...) {
            for (; i < todo.size(); i++)
                if (!todo[i].graph_owned) { cudaEventDestroy(todo[i].a); cudaEventDestroy(todo[i].b); }
            throw;
        }
    }
    virtual ~SimBase() {
        for (auto &p : pending)
            if (!p.graph_owned) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
        for (auto e : ev_pool) cudaEventDestroy(e);
    }
    virtual void set_atoms(const int *Z, const double *x, const double *y, const double *z, size_t n, bool host) = 0;
    virtual void get_sorted(int *Z, double *x, double *y, double *z, size_t cap, int *bs, size_t cap_bs, int *bid, int *zid,
                            size_t *n_out) = 0;
    virtual void build_transmission() = 0;
    virtual void get_transmission(int slice, int band_limited, double *out) = 0;
    virtual void get_propagator(double *out) = 0;
    virtual void get_probe(double x, double y, double *out) = 0;
    virtual void stem_run(const int *pixels, size_t n, double *out) = 0;
    virtual void cbed_run(double *diff) = 0;
    virtual void ctem_run(double *ew, double *diff, double *image) = 0;
    virtual void stage(int n_configs, const size_t *counts, const int *Z, const double *x, const double *y, const double *z) = 0;
    virtual void run_staged(int mode) = 0;
    virtual void run_staged_async() = 0;
    virtual void wait_run() = 0;
    virtual void staged_result(double *out, size_t cap) = 0;
    virtual void stem_plain(const int *pixels, size_t n, double *out) = 0;
    virtual void ctem_loss_grad(const double *target, double *loss, double *gxyz, double *g10, double *g30, int ck,
                                bool want_grad) = 0;
    virtual void ctem_loss_forward(const double *target, double *loss, int ck, unsigned long long *token) = 0;
    virtual void ctem_loss_backward(unsigned long long token, double *gxyz, double *g10, double *g30) = 0;
    virtual void set_c10_c30(double c10, double c30) = 0;
    virtual void tune_batch(const int *cands, int n, int reps, int *best, double *rate) = 0;
    virtual void set_step_variant(int col, int row) = 0;
    virtual std::string step_variant_name(int which, int index) = 0;
    virtual void get_tuning(int *batch, int *col, int *n_col, int *row, int *n_row) = 0;
    virtual void set_ccd(const double *dqe, const double *ntf, size_t n, int binning, double dose) = 0;
};

template <class R>
struct Sim : SimBase {
    using C = cplx<R>;
    int N = 0;
    size_t NN = 0;
    PassOps<R> ops;
    double s2d = 0;   // clFFT scale 1/sqrtf(N*N)

    // tables
    DevBuf<double> kx, ky, kx2, ky2;
    DevBuf<int2> ycut;   // per column, the band of rows the propagator's cut keeps
    PlainWork plain_work;   // buffers and plan of the plain FP64 path (stem_plain)
    DevBuf<C> px, py, pxc, pyc;   // propagator factors and their conjugates (adjoint)
    DevBuf<C> pxe, pye, pxec, pyec;   // FP32: relative representation errors of px, py and of their conjugates
    DevBuf<double2> chi;
    DevBuf<uint16_t> detmask;
    double k_prop = 0;   // k_max * limit factor of the propagator cut
    // column tiles holding columns inside the propagator cut (kx^2 < k_prop^2): the leading tiles_lo and
    // trailing tiles_hi; xa = tiles_lo*COLS, xb = N - tiles_hi*COLS bound the active columns
    int tiles_lo = 0, tiles_hi = 0, xa = 0, xb = 0;
    double fa = 1.0;   // fraction of columns the step passes read and write
    // atoms
    size_t n_atoms = 0, atom_cap = 0;
    bool atoms_set = false, trans_built = false;
    // incoherence: transmission sets (set k of slice s at trans + (k * n_slices + s) * NN), the set of each
    // wave at each slice (tsel, [slice][wave]) and the defocus phase factor of each probe (dfac)
    int n_sets = 1;
    double build_x0 = 0, build_y0 = 0;   // frame start (Å) of the transmission being built
    DevBuf<int> tsel;
    DevBuf<double> dfac;
    // CTEM dose simulation (SimulationCtem::simulateImageDose): CCD tables, binning, dose (e-/Å^2) and the
    // number of dosed images made so far (the pass of their noise draws)
    DevBuf<double> ccd_dqe, ccd_ntf;
    int ccd_binning = 0;
    double ccd_dose = 0;
    int dose_pass = 0;
    // differentiable CTEM work buffers (ctem_loss_grad)
    DevBuf<C> E, ck_buf, save, fw, gT, w1, w2;
    DevBuf<double> tgt, part, gV, gxy, gwork;
    std::vector<int> h_sel;
    std::vector<double> h_dfac;
    DevBuf<int> aZ, aZs, keys_in, keys_out, idx_in, idx_out, bid, zid, kept, counts, block_start;
    DevBuf<double> ax, ay, az, axs, ays, azs;
    DevBuf<unsigned char> cub_temp;
    size_t cub_bytes = 0;
    // transmission
    DevBuf<C> trans;
    // waves
    int batch_cap = 0;
    DevBuf<C> wave, recip, tmp;
    DevBuf<double> partials;
    DevBuf<int> pix;
    DevBuf<double2> pos;
    std::vector<int> h_pix;
    std::vector<double2> h_pos;
    // staged configurations and accumulators
    int n_configs = 0;
    std::vector<size_t> cfg_counts, cfg_offsets;
    DevBuf<int> sZ;
    DevBuf<double> sx, sy, sz;
    DevBuf<double> acc, comp;
    size_t acc_n = 0;
    int acc_configs = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};

    cudaStream_t st() const { return ctx->stream; }

    Sim(Ctx *c, const mslice_config &cf) {
        ctx = c;
        cfg = cf;
        compute_geometry(cfg, H);
        N = cfg.resolution;
        NN = (size_t)N * N;
        ops = pass_ops<R>(N);
        col_variant = ops.default_col_variant;
        s2d = (double)(1.0f / sqrtf((float)((size_t)N * N)));
        if (ctx->params.form < 0) throw StateError("no parameterisation loaded (mslice_params_load)");
        if (cfg.full3d && ctx->params.form < 0) throw StateError("no parameterisation loaded");
        const mslice_geometry &g = H.g;
        // k tables
        std::vector<double> hx2(N), hy2(N);
        for (int i = 0; i < N; i++) { hx2[i] = H.kx[i] * H.kx[i]; hy2[i] = H.ky[i] * H.ky[i]; }
        kx.ensure(ctx, N); ky.ensure(ctx, N); kx2.ensure(ctx, N); ky2.ensure(ctx, N);
        MS_CUDA(cudaMemcpyAsync(kx.p, H.kx.data(), N * sizeof(double), cudaMemcpyHostToDevice, st()));
        MS_CUDA(cudaMemcpyAsync(ky.p, H.ky.data(), N * sizeof(double), cudaMemcpyHostToDevice, st()));
        MS_CUDA(cudaMemcpyAsync(kx2.p, hx2.data(), N * sizeof(double), cudaMemcpyHostToDevice, st()));
        MS_CUDA(cudaMemcpyAsync(ky2.p, hy2.data(), N * sizeof(double), cudaMemcpyHostToDevice, st()));
        // separable propagator (propagator_d.cl:18-52): phase pi dz s, s = (k^2 - kz^2 - (kx+bx)^2 - (ky+by)^2)/kz
        k_prop = g.k_max * cfg.inverse_limit_factor;
        {   // the strict cut kx^2 + ky^2 < kp^2 per column as rows [0, a) and [b, N): ky^2 rises from row 0 to the
            // middle row and falls after it, so the kept rows are such a band; the test is the kernels' FP64 one
            const double kp2 = k_prop * k_prop;
            std::vector<int2> hc(N);
            for (int x = 0; x < N; x++) {
                int a = 0;
                while (a < N && hx2[x] + hy2[a] < kp2) a++;
                int b = N;
                while (b > a && hx2[x] + hy2[b - 1] < kp2) b--;
                for (int y = a; y < b; y++)
                    if (hx2[x] + hy2[y] < kp2) throw StateError("propagator cut is not a band of rows");
                hc[x] = make_int2(a, b);
            }
            ycut.ensure(ctx, N);
            MS_CUDA(cudaMemcpyAsync(ycut.p, hc.data(), N * sizeof(int2), cudaMemcpyHostToDevice, st()));
        }
        set_propagator(g.wavevector[0], g.wavevector[1], g.wavevector[2]);
        {
            const int C = ops.cols_per_tile, nt = N / C;
            const double km2 = k_prop * k_prop;
            std::vector<char> act(nt, 0);
            for (int x = 0; x < N; x++)
                if (H.kx[x] * H.kx[x] < km2) act[x / C] = 1;
            tiles_lo = 0;
            while (tiles_lo < nt && act[tiles_lo]) tiles_lo++;
            tiles_hi = 0;
            while (tiles_hi < nt - tiles_lo && act[nt - 1 - tiles_hi]) tiles_hi++;
            // the active columns must be one run at each end (k_x increases away from both ends)
            for (int i = tiles_lo; i < nt - tiles_hi; i++)
                if (act[i]) { tiles_lo = nt; tiles_hi = 0; break; }
            if (tiles_lo == 0 && tiles_hi == 0) tiles_lo = nt;   // degenerate cut: keep every tile
            xa = tiles_lo * C;
            xb = N - tiles_hi * C;
            fa = (double)(xa + (N - xb)) / N;
        }
        // probe aberration table
        chi.ensure(ctx, NN);
        chi_table(st(), N, kx.p, ky.p, g.wavelength, aberr(cfg.C10), cfg.cond_ap, cfg.cond_ap_smooth, chi.p);
        ctx->launches++;
        // detectors (getStemPixel, simulationstem.cpp:105-109)
        detmask.ensure(ctx, NN);
        double in[16] = {}, out[16] = {}, xc[16] = {}, yc[16] = {};
        for (int d = 0; d < cfg.n_detectors; d++) {
            in[d] = cfg.detectors[d].inner / g.angle_scale;
            out[d] = cfg.detectors[d].outer / g.angle_scale;
            xc[d] = cfg.detectors[d].xcentre / g.angle_scale;
            yc[d] = cfg.detectors[d].ycentre / g.angle_scale;
        }
        detector_masks(st(), N, cfg.n_detectors, in, out, xc, yc, detmask.p);
        ctx->launches++;
        trans.ensure(ctx, (size_t)g.n_slices * NN);
        for (int i = 0; i < 4; i++) MS_CUDA(cudaEventCreate(&ev[i]));
        MS_CUDA(cudaStreamSynchronize(st()));
    }
    ~Sim() override {
        if (run_in_flight) cudaStreamSynchronize(st());
        release_run_graph();
        drop_graphs();
        for (auto e : ev) if (e) cudaEventDestroy(e);
    }

    // The separable propagator (propagator_d.cl:18-52) for the beam wavevector (bx, by, bz): phase pi dz s,
    // s = (k^2 - kz^2 - (kx+bx)^2 - (ky+by)^2)/kz with k the wavenumber, as px[x] * py[y]; the FP32 tables'
    // relative representation errors; the conjugates for the adjoint. Copied in stream order and waited for.
    void set_propagator(double bx, double by, double bz) {
        const mslice_geometry &g = H.g;
        const double bk = g.wavenumber;
        const double f = bz / bk;
        const double c0 = kPi * g.dz * (bk * bk - bz * bz) / bz;
        std::vector<C> hpx(N), hpy(N), hex(N), hey(N);
        // relative error (p64 - p) / p of a factor rounded to R, in FP64 (zero in the FP64 engine)
        auto rel_err = [](double re, double im, C r) {
            const double dr = re - (double)r.x, di = im - (double)r.y, n2 = (double)r.x * r.x + (double)r.y * r.y;
            return mk<R>((R)((dr * r.x + di * r.y) / n2), (R)((di * r.x - dr * r.y) / n2));
        };
        for (int i = 0; i < N; i++) {
            double ax_ = -kPi * g.dz * (bx + H.kx[i]) * (bx + H.kx[i]) / bz + c0;
            double ay_ = -kPi * g.dz * (by + H.ky[i]) * (by + H.ky[i]) / bz;
            hpx[i] = mk<R>((R)(f * std::cos(ax_)), (R)(f * std::sin(ax_)));
            hpy[i] = mk<R>((R)std::cos(ay_), (R)std::sin(ay_));
            hex[i] = rel_err(f * std::cos(ax_), f * std::sin(ax_), hpx[i]);
            hey[i] = rel_err(std::cos(ay_), std::sin(ay_), hpy[i]);
        }
        px.ensure(ctx, N); py.ensure(ctx, N); pxc.ensure(ctx, N); pyc.ensure(ctx, N);
        pxe.ensure(ctx, N); pye.ensure(ctx, N); pxec.ensure(ctx, N); pyec.ensure(ctx, N);
        std::vector<C> cpx(hpx), cpy(hpy), cex(hex), cey(hey);
        for (int i = 0; i < N; i++) {
            cpx[i].y = -cpx[i].y; cpy[i].y = -cpy[i].y;
            cex[i].y = -cex[i].y; cey[i].y = -cey[i].y;   // conj(p (1 + e)) = conj(p) (1 + conj(e))
        }
        const std::pair<C *, const std::vector<C> *> up[8] = {{px.p, &hpx},  {py.p, &hpy},  {pxe.p, &hex},  {pye.p, &hey},
                                                              {pxc.p, &cpx}, {pyc.p, &cpy}, {pxec.p, &cex}, {pyec.p, &cey}};
        for (const auto &u : up)
            MS_CUDA(cudaMemcpyAsync(u.first, u.second->data(), N * sizeof(C), cudaMemcpyHostToDevice, st()));
        MS_CUDA(cudaStreamSynchronize(st()));   // the host vectors go out of scope on return
    }

    // ---- plasmon scattering: the slice loops of SimulationStem/Cbed/Ctem::simulate with plasmons on -------------
    // (simulationstem.cpp:190-232, simulationcbed.cpp:145-187, simulationctem.cpp:316-357). A job's beam starts
    // as (0, 0, k) turned by the beam tilt and azimuth; after each slice whose exit depth (below the padding
    // slices) reaches the job's next scattering depth, it turns by a drawn polar angle about the current azimuth
    // axis and a drawn azimuth about the old beam, and modifyBeamTilt rebuilds the propagator (and, in the full
    // 3-D model, the sub-slice shifts of the transmissions that follow).
    struct Beam {
        double k[3], y[3];            // wavevector and the axis the polar rotation turns about
        std::vector<double> depths;   // scattering depths (Å), the last +inf
        int count = 0;                // events so far
        uint64_t job = 0;
        bool tilted = false;          // an event has changed the propagator
    };
    bool shift_override = false;      // the full 3-D sub-slice shifts of the current beam (pot_params)
    double ov_shift_x = 0, ov_shift_y = 0;
    Beam beam_of_job(uint64_t job) const {
        Beam b;
        b.job = job;
        b.k[0] = 0; b.k[1] = 0; b.k[2] = H.g.wavenumber;
        b.y[0] = 0; b.y[1] = 1; b.y[2] = 0;
        draws::rotate_spherical(b.k, b.y, cfg.beam_tilt / 1000.0, cfg.beam_azimuth);
        // the crystal's thickness (CrystalStructure::limitsZ, clTEM_cmd main.cpp:712-714)
        const double thk = cfg.struct_limits[5] - cfg.struct_limits[4];
        if (!draws::plasmon_depths(cfg.seed, job, cfg.plasmon_mfp, thk, cfg.plasmon_individual, b.depths))
            throw ArgError("Could not generate valid plasmon configuration (job " + std::to_string(job) + ")");
        return b;
    }
    // after slice s of job b: a scattering event when the exit depth reaches the next depth
    // (PlasmonScattering::getGeneratedDepth, plasmon.cpp:122-141); true when one happened
    bool plasmon_step(Beam &b, int s) {
        const mslice_geometry &g = H.g;
        const double depth = (s + 1 - g.pre_slices) * g.dz;
        const double next = b.count < (int)b.depths.size() ? b.depths[b.count] : std::numeric_limits<double>::infinity();
        if (!(depth >= next)) return false;
        double polar, az;
        draws::plasmon_angles(cfg.seed, b.job, (uint64_t)b.count, cfg.plasmon_char_angle, cfg.plasmon_crit_angle, polar, az);
        draws::rotate_spherical(b.k, b.y, polar / 1000.0, az);
        b.count++;
        modify_beam(b.k, s);
        b.tilted = true;
        return true;
    }
    // SimulationGeneral::modifyBeamTilt (simulationgeneral.cpp:649-679) after slice s
    void modify_beam(const double k[3], int s) {
        if (!cfg.full3d)   // the reference stops here: see below
            throw Unsupported("plasmon scattering event with the projected potential: the reference's modifyBeamTilt "
                              "sets argument 29 of transmission_potentials_projected, which has 29 arguments (0-28), so "
                              "clSetKernelArg fails and the simulation stops (simulationgeneral.cpp:662-668)");
        const mslice_geometry &g = H.g;
        const int ints = cfg.full3d_integrals > 0 ? cfg.full3d_integrals : 1;
        // both sub-slice shifts from kx, as the reference writes them (:657-661)
        ov_shift_x = (k[0] / k[2]) * g.dz / ints;
        ov_shift_y = (k[0] / k[2]) * g.dz / ints;
        shift_override = true;
        set_propagator(k[0], k[1], k[2]);
        // the transmissions of the slices still to come, with the new shifts (the reference builds every slice's
        // transmission as it reaches it when plasmons are on, simulationgeneral.cpp:697-729)
        const int S = g.n_slices;
        if (s + 1 < S) {
            potentials(trans.p + (size_t)(s + 1) * NN, s + 1, S - s - 1);
            band_limit(trans.p + (size_t)(s + 1) * NN, S - s - 1);
        }
    }
    // back to the configuration's beam after a tilted job: propagator and transmissions of the frame in use
    void restore_beam() {
        const mslice_geometry &g = H.g;
        shift_override = false;
        set_propagator(g.wavevector[0], g.wavevector[1], g.wavevector[2]);
        potentials(trans.p, 0, g.n_slices);
        band_limit(trans.p, g.n_slices);
    }
    // the translation of diffraction outputs after tilts (getDiffractionImage / getStemPixel with d_k =
    // k_vec - orig_k, translateDiffImage simulationgeneral.cpp:832-853)
    Shift2 out_shift(const Beam &b) const {
        const mslice_geometry &g = H.g;
        const double shx = (b.k[0] - g.wavevector[0]) / g.inverse_scale, shy = (b.k[1] - g.wavevector[1]) / g.inverse_scale;
        Shift2 sh;
        sh.ix = (int)std::floor(shx);
        sh.iy = (int)std::floor(shy);
        sh.sx = shx - sh.ix;
        sh.sy = shy - sh.iy;
        return sh;
    }

    AberrD aberr(double c10) const {
        auto cx = [](mslice_aberration a) { return make_double2(a.mag * std::cos(a.ang), a.mag * std::sin(a.ang)); };
        AberrD A;
        A.C10 = c10; A.C30 = cfg.C30; A.C50 = cfg.C50;
        A.C12 = cx(cfg.C12); A.C21 = cx(cfg.C21); A.C23 = cx(cfg.C23); A.C32 = cx(cfg.C32); A.C34 = cx(cfg.C34);
        A.C41 = cx(cfg.C41); A.C43 = cx(cfg.C43); A.C45 = cx(cfg.C45); A.C52 = cx(cfg.C52); A.C54 = cx(cfg.C54);
        A.C56 = cx(cfg.C56);
        return A;
    }

    const R *params_dev() {
        if constexpr (sizeof(R) == 8) return ctx->prm_d;
        else return ctx->prm_f;
    }

    SortGeom sort_geom() const {
        const mslice_geometry &g = H.g;
        SortGeom s;
        s.full_x0 = g.full_x[0]; s.full_x1 = g.full_x[1]; s.full_y0 = g.full_y[0]; s.full_y1 = g.full_y[1];
        s.z0 = g.z_lims[0]; s.z1 = g.z_lims[1]; s.dz = g.dz;
        s.blocks_x = g.blocks_x; s.blocks_y = g.blocks_y; s.n_slices = g.n_slices;
        return s;
    }

    void ensure_atom_capacity(size_t n) {
        const mslice_geometry &g = H.g;
        const int n_bins = g.n_slices * g.blocks_x * g.blocks_y;
        if (n > (size_t)0x7fffffff) throw ArgError("too many atoms");
        if (n > atom_cap || atom_cap == 0) {
            size_t cap = std::max<size_t>(n, 1);
            aZ.ensure(ctx, cap); ax.ensure(ctx, cap); ay.ensure(ctx, cap); az.ensure(ctx, cap);
            aZs.ensure(ctx, cap); axs.ensure(ctx, cap); ays.ensure(ctx, cap); azs.ensure(ctx, cap);
            keys_in.ensure(ctx, cap); keys_out.ensure(ctx, cap); idx_in.ensure(ctx, cap); idx_out.ensure(ctx, cap);
            bid.ensure(ctx, cap); zid.ensure(ctx, cap); kept.ensure(ctx, cap);
            cub_bytes = atom_sort_temp_bytes((int)cap, n_bins);
            cub_temp.ensure(ctx, cub_bytes);
            atom_cap = cap;
        }
        counts.ensure(ctx, (size_t)n_bins + 1);
        block_start.ensure(ctx, (size_t)n_bins + 1);
    }

    void check_Z(const int *Z, size_t n) const {
        int maxz = ctx->params.max_z;
        for (size_t i = 0; i < n; i++)
            if (Z[i] < 1 || Z[i] > maxz)
                throw ArgError("atomic number " + std::to_string(Z[i]) + " not covered by the loaded parameterisation");
    }

    // device-resident atom arrays (already in ax/ay/az/aZ or given device pointers) -> sorted + bins
    void sort_device(const int *Z, const double *x, const double *y, const double *z, size_t n) {
        AtomSortBuffers b{keys_in.p, keys_out.p, idx_in.p, idx_out.p, bid.p, zid.p, kept.p, counts.p, cub_temp.p, cub_bytes};
        atom_sort(st(), sort_geom(), (int)n, Z, x, y, z, b, block_start.p, aZs.p, axs.p, ays.p, azs.p);
        ctx->launches += 5;
        n_atoms = n;
        atoms_set = true;
        trans_built = false;
    }

    void set_atoms(const int *Z, const double *x, const double *y, const double *z, size_t n, bool host) override {
        if (host) check_Z(Z, n);
        ensure_atom_capacity(n);
        if (host) {
            if (n) {
                MS_CUDA(cudaMemcpyAsync(aZ.p, Z, n * sizeof(int), cudaMemcpyHostToDevice, st()));
                MS_CUDA(cudaMemcpyAsync(ax.p, x, n * sizeof(double), cudaMemcpyHostToDevice, st()));
                MS_CUDA(cudaMemcpyAsync(ay.p, y, n * sizeof(double), cudaMemcpyHostToDevice, st()));
                MS_CUDA(cudaMemcpyAsync(az.p, z, n * sizeof(double), cudaMemcpyHostToDevice, st()));
            }
            sort_device(aZ.p, ax.p, ay.p, az.p, n);
        } else {
            sort_device(Z, x, y, z, n);
        }
    }

    void get_sorted(int *Z, double *x, double *y, double *z, size_t cap, int *bs, size_t cap_bs, int *bido, int *zido,
                    size_t *n_out) override {
        if (!atoms_set) throw StateError("atoms not set");
        const mslice_geometry &g = H.g;
        const size_t nbins = (size_t)g.n_slices * g.blocks_x * g.blocks_y + 1;
        if (cap_bs < nbins) throw ArgError("block_start capacity too small");
        std::vector<int> hkept(n_atoms), hbid(n_atoms), hzid(n_atoms), hbs(nbins);
        MS_CUDA(cudaStreamSynchronize(st()));
        if (n_atoms) {
            MS_CUDA(cudaMemcpy(hkept.data(), kept.p, n_atoms * sizeof(int), cudaMemcpyDeviceToHost));
            MS_CUDA(cudaMemcpy(hbid.data(), bid.p, n_atoms * sizeof(int), cudaMemcpyDeviceToHost));
            MS_CUDA(cudaMemcpy(hzid.data(), zid.p, n_atoms * sizeof(int), cudaMemcpyDeviceToHost));
        }
        MS_CUDA(cudaMemcpy(hbs.data(), block_start.p, nbins * sizeof(int), cudaMemcpyDeviceToHost));
        size_t nf = 0;
        for (size_t i = 0; i < n_atoms; i++) nf += hkept[i] ? 1 : 0;
        if (nf > cap) throw ArgError("atom capacity too small");
        size_t nin = (size_t)hbs[nbins - 1];
        if (nin) {
            MS_CUDA(cudaMemcpy(Z, aZs.p, nin * sizeof(int), cudaMemcpyDeviceToHost));
            MS_CUDA(cudaMemcpy(x, axs.p, nin * sizeof(double), cudaMemcpyDeviceToHost));
            MS_CUDA(cudaMemcpy(y, ays.p, nin * sizeof(double), cudaMemcpyDeviceToHost));
            MS_CUDA(cudaMemcpy(z, azs.p, nin * sizeof(double), cudaMemcpyDeviceToHost));
        }
        std::copy(hbs.begin(), hbs.end(), bs);
        size_t k = 0;
        for (size_t i = 0; i < n_atoms; i++)
            if (hkept[i]) {
                if (bido) bido[k] = hbid[i];
                if (zido) zido[k] = hzid[i];
                k++;
            }
        *n_out = nf;
    }

    PotParams pot_params(int slice0) const {
        const mslice_geometry &g = H.g;
        PotParams p;
        p.width = N; p.height = N; p.total_slices = g.n_slices; p.slice0 = slice0;
        p.dz = g.dz; p.pixelscale = g.real_scale;
        p.blocks_x = g.blocks_x; p.blocks_y = g.blocks_y;
        p.max_x = g.full_x[1]; p.min_x = g.full_x[0]; p.max_y = g.full_y[1]; p.min_y = g.full_y[0];
        p.load_x = g.load_blocks_x; p.load_y = g.load_blocks_y; p.load_z = g.load_blocks_z;
        p.sigma = g.sigma; p.startx = build_x0; p.starty = build_y0;
        p.beam_theta_mrad = cfg.beam_tilt; p.beam_phi = cfg.beam_azimuth;
        p.z0 = g.z_lims[0];
        p.integrals = cfg.full3d_integrals > 0 ? cfg.full3d_integrals : 1;
        p.shift_x = (g.wavevector[0] / g.wavevector[2]) * g.dz / p.integrals;   // simulationgeneral.cpp:562-563
        p.shift_y = (g.wavevector[1] / g.wavevector[2]) * g.dz / p.integrals;
        if (shift_override) {   // after a plasmon event (modify_beam)
            p.shift_x = ov_shift_x;
            p.shift_y = ov_shift_y;
        }
        p.form = ctx->params.form; p.i_count = ctx->params.i_count;
        return p;
    }

    void potentials(C *out, int slice0, int count) {
        timed(st(), MSLICE_K_POTENTIAL, (double)count * NN * sizeof(C), [&] {
            launch_potential<R>(st(), cfg.full3d != 0, out, count, axs.p, ays.p, azs.p, aZs.p, block_start.p, params_dev(),
                                ctx->pot3_tab, ctx->potp_tab, pot_params(slice0));
        });
        ctx->launches++;
    }

    void band_limit(C *t, int count) {
        // FFT -> band_limit (k <= k_max * factor, inclusive) -> IFFT, clFFT scale s2d per transform
        const cplx<R> *tw = ctx->twiddles<R>(N);
        timed(st(), MSLICE_K_BANDLIMIT, 3.0 * count * NN * 2 * sizeof(C), [&] {
            ops.row_fft(st(), t, t, count, tw, (R)1, -1);
            ops.col_bandlimit(st(), t, count, tw, kx2.p, ky2.p, H.g.k_max * cfg.inverse_limit_factor, (R)(s2d * s2d));
            ops.row_fft(st(), t, t, count, tw, (R)1, +1);
        });
        ctx->launches += 3;
    }

    // room for k transmission sets (contents are rebuilt by the caller)
    void ensure_sets(int k) {
        if (k <= n_sets && trans.p) return;
        trans.ensure(ctx, (size_t)k * H.g.n_slices * NN);
        n_sets = k;
        trans_built = false;
    }

    // source-size shift of transmission build b (SimulationCbed::initialiseSimulation, simulationcbed.cpp:103-113)
    void source_shift(int b, double &dx, double &dy) const {
        dx = dy = 0;
        if (cfg.source_size && cfg.mode != MSLICE_MODE_CTEM) draws::source_shift(cfg.seed, b, cfg.source_fwhm, dx, dy);
    }

    // the band-limited transmission of every slice into set k, frame starting at (x0, y0) Å
    void build_set(int k, double x0, double y0) {
        if (!atoms_set) throw StateError("atoms not set (mslice_set_atoms)");
        const int S = H.g.n_slices;
        build_x0 = x0;
        build_y0 = y0;
        C *base = trans.p + (size_t)k * S * NN;
        const int chunk = 1024;   // slices in chunks so one launch's grid stays within limits
        for (int s0 = 0; s0 < S; s0 += chunk) {
            int cnt = std::min(chunk, S - s0);
            potentials(base + (size_t)s0 * NN, s0, cnt);
            band_limit(base + (size_t)s0 * NN, cnt);
        }
    }

    // transmission of the current configuration in the frame of pixel 0 (build 0 of a run)
    void build_transmission() override {
        double dx, dy;
        source_shift(0, dx, dy);
        build_set(0, H.g.sim_x[0] + dx, H.g.sim_y[0] + dy);
        trans_built = true;
    }

    void copy_out_complex(const C *d, size_t count, double *out) {
        std::vector<C> h(count);
        MS_CUDA(cudaMemcpyAsync(h.data(), d, count * sizeof(C), cudaMemcpyDeviceToHost, st()));
        MS_CUDA(cudaStreamSynchronize(st()));
        for (size_t i = 0; i < count; i++) { out[2 * i] = (double)h[i].x; out[2 * i + 1] = (double)h[i].y; }
    }

    void get_transmission(int slice, int band_limited, double *out) override {
        if (slice < 0 || slice >= H.g.n_slices) throw ArgError("slice out of range");
        if (band_limited) {
            if (!trans_built) throw StateError("transmission not built (mslice_build_transmission)");
            copy_out_complex(trans.p + (size_t)slice * NN, NN, out);
        } else {
            if (!atoms_set) throw StateError("atoms not set");
            ensure_waves(1);
            double dx, dy;
            source_shift(0, dx, dy);
            build_x0 = H.g.sim_x[0] + dx;
            build_y0 = H.g.sim_y[0] + dy;
            potentials(tmp.p, slice, 1);
            copy_out_complex(tmp.p, NN, out);
        }
    }

    void get_propagator(double *out) override {
        std::vector<C> hpx(N), hpy(N);
        MS_CUDA(cudaMemcpy(hpx.data(), px.p, N * sizeof(C), cudaMemcpyDeviceToHost));
        MS_CUDA(cudaMemcpy(hpy.data(), py.p, N * sizeof(C), cudaMemcpyDeviceToHost));
        const double km2 = k_prop * k_prop;
        for (int y = 0; y < N; y++)
            for (int x = 0; x < N; x++) {
                size_t i = (size_t)y * N + x;
                bool in = H.kx[x] * H.kx[x] + H.ky[y] * H.ky[y] < km2;
                C v = in ? cmul(hpx[x], hpy[y]) : mk<R>(0, 0);
                out[2 * i] = (double)v.x;
                out[2 * i + 1] = (double)v.y;
            }
    }

    void ensure_waves(int b) {
        if (b <= batch_cap && wave.p) return;
        drop_graphs();
        wave.ensure(ctx, (size_t)b * NN);
        recip.ensure(ctx, (size_t)b * NN);
        tmp.ensure(ctx, (size_t)b * NN);
        partials.ensure(ctx, (size_t)b * std::max(1, cfg.n_detectors) * ops.col_blocks);
        pix.ensure(ctx, b);
        pos.ensure(ctx, b);
        tsel.ensure(ctx, (size_t)b * H.g.n_slices);
        dfac.ensure(ctx, b);
        batch_cap = b;
    }

    void get_probe(double x, double y, double *out) override {
        // reciprocal-space probe: generate + column IFFT into wave, then undo the column IFFT with a
        // forward column FFT (scale compensates), read back
        ensure_waves(1);
        const mslice_geometry &g = H.g;
        double2 p = make_double2(x - g.sim_x[0], y - g.sim_y[0]);
        MS_CUDA(cudaMemcpyAsync(pos.p, &p, sizeof(double2), cudaMemcpyHostToDevice, st()));
        const cplx<R> *tw = ctx->twiddles<R>(N);
        ops.col_probe(st(), wave.p, 1, tw, chi.p, kx.p, ky.p, pos.p, (R)1, nullptr, g.wavelength);
        ops.col_fft(st(), wave.p, wave.p, 1, tw, (R)(1.0 / N), -1);
        ctx->launches += 2;
        copy_out_complex(wave.p, NN, out);
    }

    int tuned_batch = 0;   // set by tune_batch (or the per-process cache of earlier tunings)
    int col_variant = 0;   // kernel of the batched column step (PassOps::col_step): the size's default, then tune_batch's
    int row_variant = 0;   // L2 prefetch distance of the batched row step (PassOps::row_step), set by tune_batch

    // the error word of the persistent passes: read after the stream's work is done, reset, reported
    void check_step_err() {
        int e = 0;
        MS_CUDA(cudaMemcpyAsync(&e, ctx->step_err, sizeof(int), cudaMemcpyDeviceToHost, st()));
        MS_CUDA(cudaStreamSynchronize(st()));
        if (e != 0) {
            MS_CUDA(cudaMemsetAsync(ctx->step_err, 0, sizeof(int), st()));
            throw CudaError("a persistent step pass abandoned a wait (code " + std::to_string(e) + "); results are invalid");
        }
    }
    int default_batch() const {
        if (cfg.probe_batch > 0) return cfg.probe_batch;
        if (tuned_batch > 0) return tuned_batch;
        size_t bytes = NN * sizeof(C);
        int b = (int)std::max<size_t>(1, ((size_t)1 << 30) / bytes);   // ~1 GiB of waves per pass (512 at 512^2 FP32)
        return std::min(b, 4096);
    }

    // STEM probe positions of scan pixels (simulationstem.cpp:152-188)
    double2 probe_pos(int p) const { return probe_pos(p, H.g.sim_x[0], H.g.sim_y[0]); }
    // relative to the frame starting at (x0, y0) Å (initialiseProbeWave subtracts paddedSimLimits(pixel)[0])
    double2 probe_pos(int p, double x0, double y0) const {
        int num_x = cfg.stem_pixels_x;
        double step_x = (cfg.stem_area[1] - cfg.stem_area[0]) / cfg.stem_pixels_x;
        double step_y = (cfg.stem_area[3] - cfg.stem_area[2]) / cfg.stem_pixels_y;
        int x_i = p % num_x;
        int y_i = (int)std::floor(p / num_x);
        double x_pos = cfg.stem_area[0] + x_i * step_x, y_pos = cfg.stem_area[2] + y_i * step_y;
        return make_double2(x_pos - x0, y_pos - y0);
    }

    void check_cancel() {
        if (cancel.load()) {
            cancel.store(false);
            cudaStreamSynchronize(st());
            throw Cancelled("simulation cancelled");
        }
    }

    // The launch sequence of one STEM batch depends only on the batch size, the output buffers and the
    // engine's own device buffers; the probe positions and output pixel indices are device arrays that the
    // kernels read. So the first batch of a shape runs eagerly, the second is captured into a CUDA graph and
    // later batches replay it (a few microseconds of host time instead of 2 launches per slice). With
    // profiling on, the graph holds its own timing events, read back after every replay.
    struct BatchGraph {
        cudaGraphExec_t exec = nullptr;
        int nb = 0, n_pix = 0;
        bool prof = false;
        const void *key[7] = {};
        unsigned long long nodes = 0, last_use = 0;
        std::vector<Pending> events;   // owned by the graph
    };
    std::vector<BatchGraph> graphs;
    unsigned long long graph_clock = 0;
    // MSLICE_NO_GRAPHS=1 launches every batch eagerly (for kernel profilers that filter launches by name)
    const bool use_graphs = [] {
        const char *e = std::getenv("MSLICE_NO_GRAPHS");
        return !(e && e[0] == '1');
    }();
    static constexpr size_t kMaxGraphs = 4;
    void release(BatchGraph &gr) {
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
        pending.erase(std::remove_if(pending.begin(), pending.end(),
                                     [&](const Pending &p) {
                                         return p.graph_owned && std::any_of(gr.events.begin(), gr.events.end(),
                                                                             [&](const Pending &q) { return q.a == p.a; });
                                     }),
                      pending.end());
        for (auto &p : gr.events) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
        gr.exec = nullptr;
        gr.events.clear();
    }
    void drop_graphs() {
        for (auto &gr : graphs) release(gr);
        graphs.clear();
        if (run_in_flight) cudaStreamSynchronize(st());
        release_run_graph();
    }

    // Propagate `nb` STEM probes through all slices: probe i at hpos[i] (Å, in the frame of its transmission
    // set); detector values of output slice o go to out[(o*n_det + d)*n_pix + out_index[i]] (Kahan-accumulated
    // if comp). with_sel: h_sel holds the set of every wave at every slice ([slice][wave]); with_df: h_dfac
    // holds each probe's defocus phase factor.
    void stem_batch(const double2 *hpos, const int *out_index, int nb, int n_pix, double *out, double *comp,
                    bool with_sel, bool with_df) {
        h_pix.assign(out_index, out_index + nb);
        MS_CUDA(cudaMemcpyAsync(pos.p, hpos, nb * sizeof(double2), cudaMemcpyHostToDevice, st()));
        MS_CUDA(cudaMemcpyAsync(pix.p, h_pix.data(), nb * sizeof(int), cudaMemcpyHostToDevice, st()));
        if (with_sel)
            MS_CUDA(cudaMemcpyAsync(tsel.p, h_sel.data(), (size_t)nb * H.g.n_slices * sizeof(int), cudaMemcpyHostToDevice, st()));
        if (with_df) MS_CUDA(cudaMemcpyAsync(dfac.p, h_dfac.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st()));
        const int *sel = with_sel ? tsel.p : nullptr;
        const double *df = with_df ? dfac.p : nullptr;
        const void *key[7] = {out, comp, wave.p, trans.p, partials.p, sel, df};
        BatchGraph *gr = nullptr;
        for (auto &c : graphs)
            if (c.nb == nb && c.n_pix == n_pix && c.prof == prof && std::equal(key, key + 7, c.key)) gr = &c;
        if (!use_graphs) {
            enqueue_batch(nb, n_pix, out, comp, sel, df);
            return;
        }
        if (!gr) {   // first batch of this shape: run eagerly, remember its launch count
            unsigned long long l0 = ctx->launches;
            enqueue_batch(nb, n_pix, out, comp, sel, df);
            if (graphs.size() == kMaxGraphs) {
                auto lru = std::min_element(graphs.begin(), graphs.end(),
                                            [](const BatchGraph &x, const BatchGraph &y) { return x.last_use < y.last_use; });
                release(*lru);
                graphs.erase(lru);
            }
            graphs.emplace_back();
            BatchGraph &ng = graphs.back();
            ng.nb = nb; ng.n_pix = n_pix; ng.prof = prof;
            std::copy(key, key + 7, ng.key);
            ng.nodes = ctx->launches - l0;
            ng.last_use = ++graph_clock;
            return;
        }
        gr->last_use = ++graph_clock;
        if (!gr->exec) {   // second batch of this shape: capture
            const size_t p0 = pending.size();
            cudaGraph_t graph = nullptr;
            MS_CUDA(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_batch(nb, n_pix, out, comp, sel, df);
            } catch (...) {
                cudaStreamEndCapture(st(), &graph);
                if (graph) cudaGraphDestroy(graph);
                throw;
            }
            MS_CUDA(cudaStreamEndCapture(st(), &graph));
            cudaError_t e = cudaGraphInstantiate(&gr->exec, graph, 0);
            cudaGraphDestroy(graph);
            // the events recorded during the capture belong to the graph from now on
            gr->events.assign(pending.begin() + p0, pending.end());
            pending.resize(p0);
            MS_CUDA(e);
            ctx->launches -= gr->nodes;   // the capture only recorded the launches
        }
        if (!gr->events.empty()) {
            // a replay re-records the graph's events: read the previous replay's durations first
            const cudaEvent_t first = gr->events[0].a;
            if (std::any_of(pending.begin(), pending.end(), [&](const Pending &p) { return p.a == first; })) flush_profile();
        }
        MS_CUDA(cudaGraphLaunch(gr->exec, st()));
        ctx->launches += gr->nodes;
        for (auto &p : gr->events) pending.push_back({p.kind, p.a, p.b, p.bytes, true});
    }

    // positions (pos_d) and output pixel indices (pix_d) of the batch's waves: the batch arrays unless given
    void enqueue_batch(int nb, int n_pix, double *out, double *comp, const int *sel, const double *df,
                       const double2 *pos_d = nullptr, const int *pix_d = nullptr) {
        const mslice_geometry &g = H.g;
        const cplx<R> *tw = ctx->twiddles<R>(N);
        const size_t set_stride = (size_t)g.n_slices * NN;
        if (!pos_d) pos_d = pos.p;
        if (!pix_d) pix_d = pix.p;
        timed(st(), MSLICE_K_PROBE, (double)nb * NN * (sizeof(C) + sizeof(double2)), [&] {
            ops.col_probe(st(), wave.p, nb, tw, chi.p, kx.p, ky.p, pos_d, (R)(s2d * N), df, g.wavelength);
        });
        ctx->launches++;
        PropTables<R> pt{px.p, py.p, kx2.p, ky2.p, k_prop * k_prop, ycut.p, ctx->step_err, pxe.p, pye.p};
        DetArgs det{detmask.p, cfg.n_detectors, partials.p};
        std::vector<int> outs = output_slices(cfg, g);
        size_t oi = 0;
        const R a = (R)(1.0 / N), b = (R)(s2d * s2d * N), ds = (R)s2d;
        for (int s = 0; s < g.n_slices; s++) {
            timed(st(), MSLICE_K_ROW_STEP, (double)nb * NN * sizeof(C) * ((s == 0 ? 1.0 : fa) + 1.0 + fa), [&] {
                ops.row_step(st(), wave.p, nb, trans.p + (size_t)s * NN, tw, a, xa, xb, s == 0 ? 1 : 0,
                             sel ? sel + (size_t)s * nb : nullptr, set_stride, row_variant, ctx->step_err);
            });
            bool is_out = oi < outs.size() && outs[oi] == s;
            int mode = !is_out ? COL_STEP : (s == g.n_slices - 1 ? COL_DET_ONLY : COL_STEP_DET);
            timed(st(), MSLICE_K_COL_STEP, (double)nb * NN * sizeof(C) * fa * (mode == COL_DET_ONLY ? 1.0 : 2.0), [&] {
                ops.col_step(st(), wave.p, nb, tw, pt, b, ds, det, nullptr, mode, tiles_lo, tiles_hi, col_variant);
            });
            ctx->launches += 2;
            if (is_out) {
                detector_reduce(st(), partials.p, tiles_lo + tiles_hi, cfg.n_detectors, nb, pix_d, n_pix, (int)oi, out, comp);
                ctx->launches++;
                oi++;
            }
        }
    }

    // pi * (chromatic defocus change) / wavelength of each probe of pass `pass` (0 when chromatic is off)
    void fill_defocus(int pass, const int *pid, int nb) {
        h_dfac.resize(nb);
        for (int i = 0; i < nb; i++)
            h_dfac[i] = kPi *
                        draws::defocus_change(cfg.seed, pass, pid[i], cfg.chromatic_cc, cfg.chromatic_hwhm_neg,
                                              cfg.chromatic_hwhm_pos, cfg.voltage) /
                        H.g.wavelength;
    }

    // One pass of STEM probes over scan pixels ids[0..n): `pass` numbers the random draws. Detector values
    // go to out at out_index (stem_batch). The static frame uses the built transmission (set 0, or the
    // mixed static sets); the moving frame splits the pixels into jobs of stem_job_pixels consecutive
    // entries (SimulationRunner::SplitJobs, simulationrunner.cpp:52-134) and builds each job's window here,
    // several jobs per batch, one transmission set per job.
    void stem_pass(int pass, const int *ids, const int *out_index, size_t n, int n_pix, double *out, double *comp,
                   bool sync_each) {
        const mslice_geometry &g = H.g;
        const int S = g.n_slices;
        if (cfg.plasmon) {
            stem_pass_plasmon(pass, ids, out_index, n, n_pix, out, comp);
            return;
        }
        const int K = cfg.mixed_static > 1 ? cfg.mixed_static : 1;
        const bool chrom = cfg.chromatic != 0;
        auto after_batch = [&](size_t done) {
            if (!sync_each) return;
            MS_CUDA(cudaStreamSynchronize(st()));
            check_step_err();
            flush_profile();
            if (progress) progress((double)done / n, progress_user);
        };
        if (!cfg.stem_moving_frame) {
            for (size_t b0 = 0; b0 < n; b0 += batch_cap) {
                check_cancel();
                const int nb = (int)std::min<size_t>(batch_cap, n - b0);
                h_pos.resize(nb);
                for (int i = 0; i < nb; i++) h_pos[i] = probe_pos(ids[b0 + i]);
                if (K > 1) {
                    h_sel.resize((size_t)nb * S);
                    for (int sl = 0; sl < S; sl++)
                        for (int i = 0; i < nb; i++) h_sel[(size_t)sl * nb + i] = draws::set_of(cfg.seed, pass, ids[b0 + i], sl, K);
                }
                if (chrom) fill_defocus(pass, ids + b0, nb);
                stem_batch(h_pos.data(), out_index + b0, nb, n_pix, out, comp, K > 1, chrom);
                after_batch(b0 + nb);
            }
            return;
        }
        const int P = std::max(1, cfg.stem_job_pixels);
        const size_t n_jobs = (n + P - 1) / P;
        const size_t set_bytes = (size_t)S * NN * sizeof(C);
        size_t J = std::max(1, batch_cap / P);
        J = std::min(J, std::max<size_t>(1, ((size_t)1 << 30) / set_bytes));   // at most ~1 GiB of job windows
        J = std::min(J, std::max<size_t>(n_jobs, 1));
        ensure_sets((int)J);
        std::vector<double2> origin(J);
        for (size_t j0 = 0; j0 < n_jobs; j0 += J) {
            check_cancel();
            const int nj = (int)std::min(J, n_jobs - j0);
            for (int j = 0; j < nj; j++) {   // each job's frame: paddedSimLimitsX/Y of its first pixel
                double fx[2], fy[2], dx, dy;
                stem_frame(cfg, ids[(j0 + j) * P], fx, fy);
                source_shift((int)((size_t)pass * n_jobs + j0 + j), dx, dy);
                build_set(j, fx[0] + dx, fy[0] + dy);
                origin[j] = make_double2(fx[0], fy[0]);
            }
            const size_t w0 = j0 * P, w1 = std::min(n, (j0 + nj) * P);
            for (size_t b0 = w0; b0 < w1; b0 += batch_cap) {
                check_cancel();
                const int nb = (int)std::min<size_t>(batch_cap, w1 - b0);
                h_pos.resize(nb);
                h_sel.resize((size_t)nb * S);
                for (int i = 0; i < nb; i++) {
                    const int j = (int)((b0 + i) / P - j0);
                    h_pos[i] = probe_pos(ids[b0 + i], origin[j].x, origin[j].y);
                    for (int sl = 0; sl < S; sl++) h_sel[(size_t)sl * nb + i] = j;
                }
                if (chrom) fill_defocus(pass, ids + b0, nb);
                stem_batch(h_pos.data(), out_index + b0, nb, n_pix, out, comp, true, chrom);
                after_batch(b0 + nb);
            }
        }
        trans_built = false;   // the sets now hold job windows
    }

    // STEM with plasmons (SimulationStem::simulate, simulationstem.cpp:143-278): jobs of stem_job_pixels consecutive
    // pixels, job `pass * n_jobs + j` (SimulationRunner::SplitJobs numbers the jobs of pass after pass; the
    // reference's pixel shuffle is clock-seeded and not reproduced), each one batch with its own tilt history,
    // launched slice by slice. At an output slice the column pass keeps the reciprocal wave and, after the
    // event check, the detectors read its translated pattern (the identity while the beam is untilted).
    DevBuf<double> tpart;   // detector partials of the translated readout
    void stem_pass_plasmon(int pass, const int *ids, const int *out_index, size_t n, int n_pix, double *out, double *comp) {
        const mslice_geometry &g = H.g;
        if (cfg.stem_moving_frame) throw Unsupported("plasmon scattering with the moving STEM frame is not supported");
        const int P = std::max(1, cfg.stem_job_pixels);
        const size_t n_jobs = (n + P - 1) / P;
        ensure_waves((int)std::min<size_t>((size_t)P, std::max<size_t>(n, 1)));
        const int nd = cfg.n_detectors;
        double in[16] = {}, outr[16] = {}, xc[16] = {}, yc[16] = {};
        for (int d = 0; d < nd; d++) {
            in[d] = cfg.detectors[d].inner / g.angle_scale;
            outr[d] = cfg.detectors[d].outer / g.angle_scale;
            xc[d] = cfg.detectors[d].xcentre / g.angle_scale;
            yc[d] = cfg.detectors[d].ycentre / g.angle_scale;
        }
        const int det_blocks = (int)((NN + 255) / 256);
        tpart.ensure(ctx, (size_t)batch_cap * std::max(1, nd) * det_blocks);
        const cplx<R> *tw = ctx->twiddles<R>(N);
        PropTables<R> pt{px.p, py.p, kx2.p, ky2.p, k_prop * k_prop, ycut.p, ctx->step_err, pxe.p, pye.p};
        DetArgs nodet{detmask.p, 0, partials.p};
        const std::vector<int> outs = output_slices(cfg, g);
        const R a = (R)(1.0 / N), b = (R)(s2d * s2d * N), ds = (R)s2d;
        const bool chrom = cfg.chromatic != 0;
        for (size_t j = 0; j < n_jobs; j++) {
            check_cancel();
            const size_t i0 = j * P, i1 = std::min(n, i0 + P);
            const int nb = (int)(i1 - i0);
            Beam beam = beam_of_job((uint64_t)pass * n_jobs + j);
            BeamScope scope{this};
            plasmon_beam = &beam;
            h_pos.resize(nb);
            for (int i = 0; i < nb; i++) h_pos[i] = probe_pos(ids[i0 + i]);
            h_pix.assign(out_index + i0, out_index + i1);
            MS_CUDA(cudaMemcpyAsync(pos.p, h_pos.data(), nb * sizeof(double2), cudaMemcpyHostToDevice, st()));
            MS_CUDA(cudaMemcpyAsync(pix.p, h_pix.data(), nb * sizeof(int), cudaMemcpyHostToDevice, st()));
            if (chrom) {
                fill_defocus(pass, ids + i0, nb);
                MS_CUDA(cudaMemcpyAsync(dfac.p, h_dfac.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st()));
            }
            // columns outside the propagator's cut are never written by the column pass: zero there
            MS_CUDA(cudaMemsetAsync(recip.p, 0, (size_t)nb * NN * sizeof(C), st()));
            ops.col_probe(st(), wave.p, nb, tw, chi.p, kx.p, ky.p, pos.p, (R)(s2d * N), chrom ? dfac.p : nullptr,
                          g.wavelength);
            ctx->launches++;
            size_t oi = 0;
            for (int s = 0; s < g.n_slices; s++) {
                ops.row_step(st(), wave.p, nb, trans.p + (size_t)s * NN, tw, a, xa, xb, s == 0 ? 1 : 0, nullptr, 0, 0,
                             ctx->step_err);
                const bool is_out = oi < outs.size() && outs[oi] == s;
                const int mode = !is_out ? COL_STEP : (s == g.n_slices - 1 ? COL_DET_ONLY : COL_STEP_DET);
                pt.px = px.p; pt.py = py.p; pt.pxe = pxe.p; pt.pye = pye.p;   // set_propagator keeps the buffers
                ops.col_step(st(), wave.p, nb, tw, pt, b, ds, nodet, is_out ? recip.p : nullptr, mode, tiles_lo, tiles_hi, 0);
                ctx->launches += 2;
                plasmon_step(beam, s);
                if (is_out) {
                    const int blocks = detectors_shifted<R>(st(), N, nb, recip.p, out_shift(beam), nd, in, outr, xc, yc, tpart.p);
                    detector_reduce(st(), tpart.p, blocks, nd, nb, pix.p, n_pix, (int)oi, out, comp);
                    ctx->launches += 2;
                    oi++;
                }
            }
            MS_CUDA(cudaStreamSynchronize(st()));
        }
    }

    void stem_run(const int *pixels, size_t n, double *out) override {
        if (cfg.mode != MSLICE_MODE_STEM) throw StateError("simulation is not in STEM mode");
        if (cfg.mixed_static > 1)
            throw StateError("mixed static potentials draw from staged configurations (mslice_stem_run_staged)");
        const int np = cfg.stem_pixels_x * cfg.stem_pixels_y;
        for (size_t i = 0; i < n; i++)
            if (pixels[i] < 0 || pixels[i] >= np) throw ArgError("scan pixel index out of range");
        if (!cfg.stem_moving_frame && !trans_built) build_transmission();
        const int B = default_batch();
        ensure_waves(std::min<int>(B, (int)std::max<size_t>(n, 1)));
        const mslice_geometry &g = H.g;
        DevBuf<double> dout;
        size_t tot = (size_t)g.n_outputs * cfg.n_detectors * n;
        dout.ensure(ctx, tot);
        MS_CUDA(cudaMemsetAsync(dout.p, 0, std::max<size_t>(tot, 1) * sizeof(double), st()));
        std::vector<int> idx(n);
        for (size_t i = 0; i < n; i++) idx[i] = (int)i;
        stem_pass(0, pixels, idx.data(), n, (int)n, dout.p, nullptr, true);
        if (tot) MS_CUDA(cudaMemcpy(out, dout.p, tot * sizeof(double), cudaMemcpyDeviceToHost));
    }

    // one probe (CBED) or plane wave (CTEM) through all slices with outputs at the output slices
    // (pass numbers the random draws: the mixed static set of each slice, the chromatic defocus change)
    template <class F>
    void single_wave(bool plane, int pass, F &&on_output) {
        const mslice_geometry &g = H.g;
        const cplx<R> *tw = ctx->twiddles<R>(N);
        ensure_waves(1);
        const int K = cfg.mixed_static > 1 ? cfg.mixed_static : 1;
        const size_t set_stride = (size_t)g.n_slices * NN;
        // plasmons: the job of a CTEM / CBED pass is the pass (SimulationRunner::SplitJobs, simulationrunner.cpp:62-67)
        Beam beam;
        BeamScope scope{this};
        if (cfg.plasmon) {
            beam = beam_of_job((uint64_t)pass);
            plasmon_beam = &beam;
        }
        if (K > 1) {
            h_sel.resize(g.n_slices);
            for (int sl = 0; sl < g.n_slices; sl++) h_sel[sl] = draws::set_of(cfg.seed, pass, 0, sl, K);
            MS_CUDA(cudaMemcpyAsync(tsel.p, h_sel.data(), g.n_slices * sizeof(int), cudaMemcpyHostToDevice, st()));
        }
        if (plane) {
            plane_wave_state<R>(st(), N, wave.p);
        } else {
            double2 p = make_double2(cfg.cbed_x - g.sim_x[0], cfg.cbed_y - g.sim_y[0]);
            MS_CUDA(cudaMemcpyAsync(pos.p, &p, sizeof(double2), cudaMemcpyHostToDevice, st()));
            const int pid = 0;
            if (cfg.chromatic) {
                fill_defocus(pass, &pid, 1);
                MS_CUDA(cudaMemcpyAsync(dfac.p, h_dfac.data(), sizeof(double), cudaMemcpyHostToDevice, st()));
            }
            ops.col_probe(st(), wave.p, 1, tw, chi.p, kx.p, ky.p, pos.p, (R)(s2d * N), cfg.chromatic ? dfac.p : nullptr,
                          g.wavelength);
        }
        ctx->launches++;
        PropTables<R> pt{px.p, py.p, kx2.p, ky2.p, k_prop * k_prop, ycut.p, ctx->step_err, pxe.p, pye.p};
        DetArgs det{detmask.p, 0, partials.p};
        std::vector<int> outs = output_slices(cfg, g);
        size_t oi = 0;
        const R a = (R)(1.0 / N), b = (R)(s2d * s2d * N), ds = (R)s2d;
        for (int s = 0; s < g.n_slices; s++) {
            check_cancel();
            // single waves keep every column so the exit wave and the reciprocal copy are complete
            timed(st(), MSLICE_K_ROW_STEP, 3.0 * NN * sizeof(C), [&] {
                ops.row_step(st(), wave.p, 1, trans.p + (size_t)s * NN, tw, a, N, N, 1, K > 1 ? tsel.p + s : nullptr,
                             set_stride, 0, ctx->step_err);
            });
            bool is_out = oi < outs.size() && outs[oi] == s;
            timed(st(), MSLICE_K_COL_STEP, (is_out ? 3.0 : 2.0) * NN * sizeof(C), [&] {
                ops.col_step(st(), wave.p, 1, tw, pt, b, ds, det, is_out ? recip.p : nullptr, is_out ? COL_STEP_DET : COL_STEP,
                             N / ops.cols_per_tile, 0, 0);
            });
            ctx->launches += 2;
            if (plasmon_beam) plasmon_step(*plasmon_beam, s);   // the event check comes before the slice's outputs
            if (is_out) { on_output((int)oi); oi++; }
            if (progress) progress((double)(s + 1) / g.n_slices, progress_user);
        }
    }

    // ends a plasmon job on every exit path: the configuration's beam back if an event tilted it
    struct BeamScope {
        Sim *sim;
        ~BeamScope() {
            if (!sim->plasmon_beam) return;
            if (sim->plasmon_beam->tilted) {
                try {
                    sim->restore_beam();
                } catch (...) {   // a failing restore leaves the tables of the tilted beam: rebuilt by the next run
                    sim->trans_built = false;
                }
            }
            sim->plasmon_beam = nullptr;
        }
    };

    // the diffraction output of the single wave in recip: translated while a plasmon event has tilted the beam
    Beam *plasmon_beam = nullptr;   // the beam of the job single_wave is running (plasmons on), else nullptr
    void diff_out(double *out, double *comp) {
        if (plasmon_beam && plasmon_beam->tilted) diffraction_shifted<R>(st(), N, recip.p, out_shift(*plasmon_beam), out, comp);
        else diffraction<R>(st(), N, recip.p, out, comp);
        ctx->launches++;
    }

    void cbed_run(double *diff) override {
        if (cfg.mode != MSLICE_MODE_CBED) throw StateError("simulation is not in CBED mode");
        if (cfg.mixed_static > 1)
            throw StateError("mixed static potentials draw from staged configurations (mslice_cbed_run_staged)");
        if (!trans_built) build_transmission();
        DevBuf<double> d;
        d.ensure(ctx, (size_t)H.g.n_outputs * NN);
        single_wave(false, 0, [&](int o) {
            diff_out(d.p + (size_t)o * NN, nullptr);
        });
        MS_CUDA(cudaStreamSynchronize(st()));
        MS_CUDA(cudaMemcpy(diff, d.p, (size_t)H.g.n_outputs * NN * sizeof(double), cudaMemcpyDeviceToHost));
    }

    // SimulationCtem::simulateImageDose (simulationctem.cpp:171-264) on the image wave `w` (real space, after
    // the objective lens): |w|^2 -> FFT -> DQE -> IFFT -> Poisson counts of mean N_tot * value (N_tot = dose
    // per binned pixel, conversion factor 1) -> FFT -> NTF -> IFFT; the image is the real part. Transforms use
    // clFFT's unitary scale both ways. The counts are drawn on the host, as the reference does, from the seeded
    // stream of pass dose_pass (one pass per dosed image).
    void dose_image(C *w, double *out) {
        const cplx<R> *tw = ctx->twiddles<R>(N);
        auto fft = [&](int sign) {
            ops.row_fft(st(), w, w, 1, tw, (R)1, sign);
            ops.col_fft(st(), w, w, 1, tw, (R)s2d, sign);
            ctx->launches += 2;
        };
        sqabs_complex<R>(st(), NN, w);
        fft(-1);
        ccd_filter<R>(st(), N, w, ccd_dqe.p, ccd_binning, true);
        fft(+1);
        ctx->launches += 2;
        std::vector<C> h(NN);
        MS_CUDA(cudaMemcpyAsync(h.data(), w, NN * sizeof(C), cudaMemcpyDeviceToHost, st()));
        MS_CUDA(cudaStreamSynchronize(st()));
        const double dose_per_pix = ccd_dose * H.g.real_scale * H.g.real_scale;
        const double n_tot = dose_per_pix * ccd_binning * ccd_binning;
        for (size_t i = 0; i < NN; i++)
            h[i] = mk<R>((R)draws::poisson(cfg.seed, dose_pass, i, n_tot * (double)h[i].x), (R)0);
        dose_pass++;
        MS_CUDA(cudaMemcpyAsync(w, h.data(), NN * sizeof(C), cudaMemcpyHostToDevice, st()));
        fft(-1);
        ccd_filter<R>(st(), N, w, ccd_ntf.p, ccd_binning, false);
        fft(+1);
        ctx->launches++;
        real_part_to_double<R>(st(), NN, w, out);
        ctx->launches++;
        MS_CUDA(cudaStreamSynchronize(st()));   // h is released on return
    }

    void set_ccd(const double *dqe, const double *ntf, size_t n, int binning, double dose) override {
        if (n == 0) {   // back to the perfect image
            ccd_binning = 0;
            return;
        }
        if (n != 725) throw ArgError("CCD tables hold 725 values (Utils::ccdToDqeNtf)");
        if (binning < 1) throw ArgError("CCD binning must be >= 1");
        if (!(dose > 0)) throw ArgError("CCD dose must be positive");
        ccd_dqe.ensure(ctx, n);
        ccd_ntf.ensure(ctx, n);
        MS_CUDA(cudaMemcpy(ccd_dqe.p, dqe, n * sizeof(double), cudaMemcpyHostToDevice));
        MS_CUDA(cudaMemcpy(ccd_ntf.p, ntf, n * sizeof(double), cudaMemcpyHostToDevice));
        ccd_binning = binning;
        ccd_dose = dose;
        dose_pass = 0;
    }

    void ctem_run(double *ew, double *diff, double *image) override {
        if (cfg.mode != MSLICE_MODE_CTEM) throw StateError("simulation is not in CTEM mode");
        if (cfg.mixed_static > 1) throw Unsupported("mixed static potentials are implemented for STEM and CBED runs");
        if (!trans_built) build_transmission();
        const int no = H.g.n_outputs;
        DevBuf<double> dd, di;
        DevBuf<double2> de;
        if (ew) de.ensure(ctx, (size_t)no * NN);
        if (diff) dd.ensure(ctx, (size_t)no * NN);
        if (image && cfg.ctem_image) di.ensure(ctx, (size_t)no * NN);
        const cplx<R> *tw = ctx->twiddles<R>(N);
        const mslice_geometry &g = H.g;
        single_wave(true, 0, [&](int o) {
            if (ew) {   // psi = (1/N) Dinv_r phi  (getExitWaveImage, simulationgeneral.cpp:808-830)
                ops.row_fft(st(), wave.p, tmp.p, 1, tw, (R)(1.0 / N), +1);
                convert_to_double<R>(st(), NN, tmp.p, de.p + (size_t)o * NN);
                ctx->launches += 2;
            }
            if (diff) diff_out(dd.p + (size_t)o * NN, nullptr);
            if (image && cfg.ctem_image) {   // simulateImagePerfect (simulationctem.cpp:114-166)
                ctem_transfer<R>(st(), N, recip.p, tmp.p, kx.p, ky.p, g.wavelength, aberr(cfg.C10), cfg.obj_ap,
                                 cfg.obj_ap_smooth, cfg.alpha, cfg.delta);
                ops.row_fft(st(), tmp.p, tmp.p, 1, tw, (R)1, +1);
                ops.col_fft(st(), tmp.p, tmp.p, 1, tw, (R)s2d, +1);
                ctx->launches += 3;
                if (ccd_binning > 0) {
                    dose_image(tmp.p, di.p + (size_t)o * NN);
                } else {
                    sqabs_to_double<R>(st(), NN, tmp.p, di.p + (size_t)o * NN);
                    ctx->launches++;
                }
            }
        });
        MS_CUDA(cudaStreamSynchronize(st()));
        if (ew) MS_CUDA(cudaMemcpy(ew, de.p, (size_t)no * NN * sizeof(double2), cudaMemcpyDeviceToHost));
        if (diff) MS_CUDA(cudaMemcpy(diff, dd.p, (size_t)no * NN * sizeof(double), cudaMemcpyDeviceToHost));
        if (image && cfg.ctem_image) MS_CUDA(cudaMemcpy(image, di.p, (size_t)no * NN * sizeof(double), cudaMemcpyDeviceToHost));
    }

    // ---- staged frozen-phonon configurations ------------------------------------------------
    void stage(int nc, const size_t *cnt, const int *Z, const double *x, const double *y, const double *z) override {
        if (nc < 1) throw ArgError("need at least one configuration");
        size_t tot = 0, mx = 0;
        cfg_counts.assign(cnt, cnt + nc);
        cfg_offsets.resize(nc);
        for (int c = 0; c < nc; c++) { cfg_offsets[c] = tot; tot += cnt[c]; mx = std::max(mx, cnt[c]); }
        check_Z(Z, tot);
        sZ.ensure(ctx, tot); sx.ensure(ctx, tot); sy.ensure(ctx, tot); sz.ensure(ctx, tot);
        if (tot) {
            MS_CUDA(cudaMemcpyAsync(sZ.p, Z, tot * sizeof(int), cudaMemcpyHostToDevice, st()));
            MS_CUDA(cudaMemcpyAsync(sx.p, x, tot * sizeof(double), cudaMemcpyHostToDevice, st()));
            MS_CUDA(cudaMemcpyAsync(sy.p, y, tot * sizeof(double), cudaMemcpyHostToDevice, st()));
            MS_CUDA(cudaMemcpyAsync(sz.p, z, tot * sizeof(double), cudaMemcpyHostToDevice, st()));
        }
        ensure_atom_capacity(mx);
        n_configs = nc;
    }

    // ---- a whole staged STEM run as one CUDA graph -------------------------------------------------------
    // With the static frame, one transmission set, no plasmons and no progress callback, the launch sequence of
    // a staged run (per pass: binning of the pass's configuration, its transmission build, then every probe
    // batch) depends only on the staged layout and the buffers: the positions of all scan pixels (and the
    // chromatic defocus of every pass) are uploaded first, the run is captured once into a graph, and every run
    // of the same layout is one cudaGraphLaunch. The graph keeps its own timing events when profiling is on.
    struct RunGraph {
        cudaGraphExec_t exec = nullptr;
        std::vector<uintptr_t> key;
        std::vector<Pending> events;   // owned by the graph
        unsigned long long nodes = 0;
    } run_graph;
    DevBuf<double2> run_pos;   // probe position of every scan pixel (static frame)
    DevBuf<int> run_pix;       // 0..n_pix-1
    DevBuf<double> run_dfac;   // chromatic defocus factor of every (pass, pixel)
    bool async_run = false;    // mslice_stem_run_staged_async: launch and return
    bool run_in_flight = false;
    int run_passes = 0;
    bool run_graph_ok() const {
        return use_graphs && cfg.mode == MSLICE_MODE_STEM && cfg.mixed_static <= 1 && !cfg.stem_moving_frame &&
               !cfg.plasmon && progress == nullptr;
    }
    void release_run_graph() {
        if (run_graph.exec) cudaGraphExecDestroy(run_graph.exec);
        pending.erase(std::remove_if(pending.begin(), pending.end(),
                                     [&](const Pending &p) {
                                         return p.graph_owned &&
                                                std::any_of(run_graph.events.begin(), run_graph.events.end(),
                                                            [&](const Pending &q) { return q.a == p.a; });
                                     }),
                      pending.end());
        for (auto &p : run_graph.events) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
        run_graph = RunGraph();
    }
    // the whole run's launches (pass = binning + build + every batch), for capture
    void enqueue_run(int passes, int np) {
        const mslice_geometry &g = H.g;
        const bool chrom = cfg.chromatic != 0;
        for (int it = 0; it < passes; it++) {
            const int c = it % n_configs;
            sort_device(sZ.p + cfg_offsets[c], sx.p + cfg_offsets[c], sy.p + cfg_offsets[c], sz.p + cfg_offsets[c],
                        cfg_counts[c]);
            double dx, dy;
            source_shift(it, dx, dy);
            build_set(0, g.sim_x[0] + dx, g.sim_y[0] + dy);
            for (int b0 = 0; b0 < np; b0 += batch_cap) {
                const int nb = std::min(batch_cap, np - b0);
                enqueue_batch(nb, np, acc.p, comp.p, nullptr, chrom ? run_dfac.p + (size_t)it * np + b0 : nullptr,
                              run_pos.p + b0, run_pix.p + b0);
            }
        }
    }
    void launch_run_graph(int passes, int np) {
        const bool chrom = cfg.chromatic != 0;
        // per-pixel (and per-pass) inputs of every batch, uploaded before the capture
        run_pos.ensure(ctx, np);
        run_pix.ensure(ctx, np);
        std::vector<double2> hp(np);
        std::vector<int> hi(np);
        for (int i = 0; i < np; i++) { hp[i] = probe_pos(i); hi[i] = i; }
        MS_CUDA(cudaMemcpyAsync(run_pos.p, hp.data(), np * sizeof(double2), cudaMemcpyHostToDevice, st()));
        MS_CUDA(cudaMemcpyAsync(run_pix.p, hi.data(), np * sizeof(int), cudaMemcpyHostToDevice, st()));
        std::vector<double> hd;
        if (chrom) {
            run_dfac.ensure(ctx, (size_t)passes * np);
            hd.resize((size_t)passes * np);
            for (int it = 0; it < passes; it++) {
                fill_defocus(it, hi.data(), np);
                std::copy(h_dfac.begin(), h_dfac.end(), hd.begin() + (size_t)it * np);
            }
            MS_CUDA(cudaMemcpyAsync(run_dfac.p, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice, st()));
        }
        MS_CUDA(cudaStreamSynchronize(st()));   // the host staging vectors go out of scope
        std::vector<uintptr_t> key = {(uintptr_t)acc.p, (uintptr_t)comp.p, (uintptr_t)wave.p, (uintptr_t)trans.p,
                                      (uintptr_t)partials.p, (uintptr_t)sZ.p, (uintptr_t)sx.p, (uintptr_t)sy.p,
                                      (uintptr_t)sz.p, (uintptr_t)run_pos.p, (uintptr_t)run_pix.p,
                                      (uintptr_t)(chrom ? run_dfac.p : nullptr), (uintptr_t)passes, (uintptr_t)np,
                                      (uintptr_t)n_configs, (uintptr_t)batch_cap, (uintptr_t)prof,
                                      (uintptr_t)col_variant, (uintptr_t)row_variant};
        for (int c = 0; c < n_configs; c++) { key.push_back(cfg_offsets[c]); key.push_back(cfg_counts[c]); }
        if (!run_graph.exec || key != run_graph.key) {
            release_run_graph();
            (void)ctx->twiddles<R>(N);   // allocated on first use: never inside the capture
            const size_t p0 = pending.size();
            const unsigned long long l0 = ctx->launches;
            cudaGraph_t graph = nullptr;
            MS_CUDA(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_run(passes, np);
            } catch (...) {
                cudaStreamEndCapture(st(), &graph);
                if (graph) cudaGraphDestroy(graph);
                for (size_t i = p0; i < pending.size(); i++) { cudaEventDestroy(pending[i].a); cudaEventDestroy(pending[i].b); }
                pending.resize(p0);
                ctx->launches = l0;
                throw;
            }
            MS_CUDA(cudaStreamEndCapture(st(), &graph));
            cudaError_t e = cudaGraphInstantiate(&run_graph.exec, graph, 0);
            cudaGraphDestroy(graph);
            run_graph.events.assign(pending.begin() + p0, pending.end());
            pending.resize(p0);
            if (e != cudaSuccess) {
                for (auto &p : run_graph.events) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
                run_graph = RunGraph();
                MS_CUDA(e);
            }
            run_graph.nodes = ctx->launches - l0;
            ctx->launches = l0;
            run_graph.key = key;
        }
        if (!run_graph.events.empty()) {   // a replay re-records the graph's events: read the previous replay first
            const cudaEvent_t first = run_graph.events[0].a;
            if (std::any_of(pending.begin(), pending.end(), [&](const Pending &p) { return p.a == first; })) {
                MS_CUDA(cudaStreamSynchronize(st()));
                flush_profile();
            }
        }
        MS_CUDA(cudaEventRecord(ev[2], st()));
        MS_CUDA(cudaGraphLaunch(run_graph.exec, st()));
        MS_CUDA(cudaEventRecord(ev[3], st()));
        ctx->launches += run_graph.nodes;
        for (auto &p : run_graph.events) pending.push_back({p.kind, p.a, p.b, p.bytes, true});
        trans_built = true;
        run_in_flight = true;
    }
    // wait for a graph run, then its timing, error word, profile and pass count
    void finish_run() {
        if (!run_in_flight) return;
        run_in_flight = false;
        MS_CUDA(cudaEventSynchronize(ev[3]));
        check_step_err();
        flush_profile();
        float tot = 0;
        MS_CUDA(cudaEventElapsedTime(&tot, ev[2], ev[3]));
        timing[0] = -1.0;   // one graph: the build / propagation split is not timed
        timing[1] = -1.0;
        timing[2] = tot;
        acc_configs = run_passes;
    }

    // launch a staged STEM run and return: one graph launch when run_graph_ok(), else the synchronous run
    void run_staged_async() override {
        async_run = true;
        try {
            run_staged(MSLICE_MODE_STEM);
        } catch (...) {
            async_run = false;
            throw;
        }
        async_run = false;
    }
    void wait_run() override { finish_run(); }

    void run_staged(int mode) override {
        if (n_configs < 1) throw StateError("no configurations staged (mslice_stage_configs)");
        finish_run();   // a run still in flight owns the accumulators
        if (mode != cfg.mode) throw StateError("staged run of the wrong mode");
        const mslice_geometry &g = H.g;
        const int np = cfg.stem_pixels_x * cfg.stem_pixels_y;
        if (mode == MSLICE_MODE_STEM) acc_n = (size_t)g.n_outputs * cfg.n_detectors * np;
        else acc_n = (size_t)g.n_outputs * NN;
        acc.ensure(ctx, acc_n); comp.ensure(ctx, acc_n);
        MS_CUDA(cudaMemsetAsync(acc.p, 0, std::max<size_t>(acc_n, 1) * sizeof(double), st()));
        MS_CUDA(cudaMemsetAsync(comp.p, 0, std::max<size_t>(acc_n, 1) * sizeof(double), st()));
        std::vector<int> ids(np);
        for (int i = 0; i < np; i++) ids[i] = i;
        if (mode == MSLICE_MODE_STEM) ensure_waves(std::min(default_batch(), np));
        // passes: one per staged configuration, or cfg.iterations passes cycling through them; with mixed
        // static potentials the first mixed_static configurations are built once as the sets (the reference
        // keeps them across jobs, simulationgeneral.cpp:358) and every pass draws new sets
        const int K = cfg.mixed_static > 1 ? cfg.mixed_static : 1;
        if (K > 1 && n_configs < K) throw StateError("mixed static potentials need mixed_static staged configurations");
        const int passes = K > 1 ? std::max(1, cfg.iterations) : (cfg.iterations > 0 ? cfg.iterations : n_configs);
        if (mode == MSLICE_MODE_STEM && run_graph_ok()) {   // every pass and batch in one graph launch
            check_cancel();
            launch_run_graph(passes, np);
            run_passes = passes;
            if (!async_run) finish_run();
            return;
        }
        float t_build = 0, t_prop = 0;
        MS_CUDA(cudaEventRecord(ev[2], st()));
        if (K > 1) {
            MS_CUDA(cudaEventRecord(ev[0], st()));
            ensure_sets(K);
            double dx, dy;
            source_shift(0, dx, dy);
            for (int k = 0; k < K; k++) {
                sort_device(sZ.p + cfg_offsets[k], sx.p + cfg_offsets[k], sy.p + cfg_offsets[k], sz.p + cfg_offsets[k],
                            cfg_counts[k]);
                build_set(k, g.sim_x[0] + dx, g.sim_y[0] + dy);
            }
            trans_built = true;
            MS_CUDA(cudaEventRecord(ev[1], st()));
            MS_CUDA(cudaEventSynchronize(ev[1]));
            MS_CUDA(cudaEventElapsedTime(&t_build, ev[0], ev[1]));
        }
        for (int it = 0; it < passes; it++) {
            check_cancel();
            MS_CUDA(cudaEventRecord(ev[0], st()));
            if (K == 1) {
                const int c = it % n_configs;
                sort_device(sZ.p + cfg_offsets[c], sx.p + cfg_offsets[c], sy.p + cfg_offsets[c], sz.p + cfg_offsets[c],
                            cfg_counts[c]);
                if (!(mode == MSLICE_MODE_STEM && cfg.stem_moving_frame)) {   // the moving frame builds per job
                    double dx, dy;
                    source_shift(it, dx, dy);
                    build_set(0, g.sim_x[0] + dx, g.sim_y[0] + dy);
                    trans_built = true;
                }
            }
            MS_CUDA(cudaEventRecord(ev[1], st()));
            if (mode == MSLICE_MODE_STEM) {
                stem_pass(it, ids.data(), ids.data(), (size_t)np, np, acc.p, comp.p, false);
            } else {
                single_wave(false, it, [&](int o) {
                    diff_out(acc.p + (size_t)o * NN, comp.p + (size_t)o * NN);
                });
            }
            MS_CUDA(cudaEventRecord(ev[3], st()));
            MS_CUDA(cudaEventSynchronize(ev[3]));
            check_step_err();
            flush_profile();
            float a = 0, b = 0;
            MS_CUDA(cudaEventElapsedTime(&a, ev[0], ev[1]));
            MS_CUDA(cudaEventElapsedTime(&b, ev[1], ev[3]));
            t_build += a;
            t_prop += b;
            if (progress) progress((double)(it + 1) / passes, progress_user);
        }
        float tot = 0;
        MS_CUDA(cudaEventElapsedTime(&tot, ev[2], ev[3]));
        timing[0] = t_build; timing[1] = t_prop; timing[2] = tot;
        acc_configs = passes;
    }

    void staged_result(double *out, size_t cap) override {
        finish_run();
        if (acc_configs < 1) throw StateError("no staged run");
        if (cap < acc_n) throw ArgError("output capacity too small");
        MS_CUDA(cudaStreamSynchronize(st()));
        MS_CUDA(cudaMemcpy(out, acc.p, acc_n * sizeof(double), cudaMemcpyDeviceToHost));
        // Image::getWeightedSlice: sum / weight, weight = number of configurations per pixel
        for (size_t i = 0; i < acc_n; i++) out[i] /= (double)acc_configs;
    }

    // Autotuner of the probe batch and of the column step's kernel: time `reps` STEM slice steps (one row and
    // one column pass) for each candidate batch and each column-pass variant (PassOps::col_variants: the
    // one-launch-per-tile kernel and the persistent TMA-fed passes) on zeroed scratch waves with the current
    // transmission tables, and keep the pair with the most waves per second. Results are cached per
    // (device, grid, precision) for the process.
    struct Tuning { int batch; double rate; int col_variant; int row_variant; };
    static std::map<std::tuple<int, int, int>, Tuning> &tune_cache() {
        static std::map<std::tuple<int, int, int>, Tuning> m;
        return m;
    }
    void tune_batch(const int *cands, int n, int reps, int *best, double *rate) override {
        if (n < 1 || reps < 1) throw ArgError("need candidate batches and repetitions");
        const auto key = std::make_tuple(ctx->device, N, (int)sizeof(R));
        {
            std::lock_guard<std::mutex> lk(ctx->mtx);
            auto it = tune_cache().find(key);
            if (it != tune_cache().end() && cands == nullptr) {
                tuned_batch = it->second.batch;
                col_variant = it->second.col_variant;
                row_variant = it->second.row_variant;
                if (best) *best = it->second.batch;
                if (rate) *rate = it->second.rate;
                return;
            }
        }
        std::vector<int> cs;
        if (cands) cs.assign(cands, cands + n);
        else cs = {64, 128, 256, 512, 1024, 2048};
        const size_t wave_bytes = NN * sizeof(C);
        int bmax = 0;
        for (int b : cs) {
            if (b < 1 || b > 65535) throw ArgError("candidate batch out of range");
            // three wave-sized buffers per probe; stay within a quarter of the device's free memory
            size_t fr = 0, tot = 0;
            MS_CUDA(cudaMemGetInfo(&fr, &tot));
            if ((size_t)b <= (size_t)batch_cap || 3 * (size_t)b * wave_bytes < fr / 4) bmax = std::max(bmax, b);
        }
        if (bmax == 0) throw OomError("no candidate batch fits in device memory");
        ensure_waves(bmax);
        MS_CUDA(cudaMemsetAsync(wave.p, 0, (size_t)bmax * wave_bytes, st()));
        if (!trans_built) MS_CUDA(cudaMemsetAsync(trans.p, 0, NN * sizeof(C), st()));
        const cplx<R> *tw = ctx->twiddles<R>(N);
        PropTables<R> pt{px.p, py.p, kx2.p, ky2.p, k_prop * k_prop, ycut.p, ctx->step_err, pxe.p, pye.p};
        DetArgs det{detmask.p, cfg.n_detectors, partials.p};
        const R a = (R)(1.0 / N), b2 = (R)(s2d * s2d * N), ds = (R)s2d;
        // time one slice step of each (batch, row variant, column variant)
        auto rate_of = [&](int b, int row_v, int col_v) {
            auto step = [&] {
                ops.row_step(st(), wave.p, b, trans.p, tw, a, xa, xb, 0, nullptr, 0, row_v, ctx->step_err);
                ops.col_step(st(), wave.p, b, tw, pt, b2, ds, det, nullptr, COL_STEP, tiles_lo, tiles_hi, col_v);
                ctx->launches += 2;
            };
            step();   // warm-up
            MS_CUDA(cudaEventRecord(ev[0], st()));
            for (int r = 0; r < reps; r++) step();
            MS_CUDA(cudaEventRecord(ev[1], st()));
            MS_CUDA(cudaEventSynchronize(ev[1]));
            float ms = 0;
            MS_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            return (double)b * reps / (ms * 1e-3);
        };
        double best_rate = -1;
        int best_b = cs[0], best_v = 0, best_rv = 0;
        for (int variant = 0; variant < ops.col_variants; variant++)   // batch and column kernel
            for (int b : cs) {
                if (b > bmax) continue;
                const double r_ = rate_of(b, 0, variant);
                if (r_ > best_rate) { best_rate = r_; best_b = b; best_v = variant; }
            }
        for (int rv = 1; rv < ops.row_variants; rv++) {   // then the row pass's prefetch / order at that pair
            const double r_ = rate_of(best_b, rv, best_v);
            if (r_ > best_rate) { best_rate = r_; best_rv = rv; }
        }
        check_step_err();
        tuned_batch = best_b;
        col_variant = best_v;
        row_variant = best_rv;
        if (cands == nullptr) {   // only the default candidate set is shared through the cache
            std::lock_guard<std::mutex> lk(ctx->mtx);
            tune_cache()[key] = {best_b, best_rate, best_v, best_rv};
        }
        // release the scratch waves: runs allocate batches of the tuned size (batch_cap sets their size)
        MS_CUDA(cudaStreamSynchronize(st()));
        drop_graphs();
        wave.free(); recip.free(); tmp.free(); partials.free(); pix.free(); pos.free(); tsel.free(); dfac.free();
        batch_cap = 0;
        if (best) *best = best_b;
        if (rate) *rate = best_rate;
    }

    void set_step_variant(int col, int row) override {
        if (col < 0 || col >= ops.col_variants)
            throw ArgError("column step variant " + std::to_string(col) + " out of range [0, " +
                           std::to_string(ops.col_variants) + ")");
        if (row < 0 || row >= ops.row_variants)
            throw ArgError("row step variant " + std::to_string(row) + " out of range [0, " +
                           std::to_string(ops.row_variants) + ")");
        if (col != col_variant || row != row_variant) drop_graphs();   // captured batches hold the previous kernels
        col_variant = col;
        row_variant = row;
    }
    std::string step_variant_name(int which, int index) override {
        if (which == 0) {
            if (index < 0 || index >= ops.col_variants) throw ArgError("column step variant out of range");
            return ops.col_variant_name ? ops.col_variant_name(index) : std::string();
        }
        if (which != 1 || index < 0 || index >= ops.row_variants) throw ArgError("row step variant out of range");
        return ops.row_variant_name ? ops.row_variant_name(index) : std::string();
    }
    void get_tuning(int *batch, int *col, int *n_col, int *row, int *n_row) override {
        if (batch) *batch = default_batch();
        if (col) *col = col_variant;
        if (n_col) *n_col = ops.col_variants;
        if (row) *row = row_variant;
        if (n_row) *n_row = ops.row_variants;
    }

    void set_c10_c30(double c10, double c30) override {
        cfg.C10 = c10;
        cfg.C30 = c30;
        chi_table(st(), N, kx.p, ky.p, H.g.wavelength, aberr(cfg.C10), cfg.cond_ap, cfg.cond_ap_smooth, chi.p);
        ctx->launches++;
    }

    // ---- differentiable CTEM -------------------------------------------------------------
    // The adjoint's forward half: the loss and, with want_grad, the checkpoints and state its backward half
    // reads. Any other call on the simulation in between invalidates that state (adj_valid).
    unsigned long long adj_token = 0;
    int adj_c = 1, adj_nck = 1, adj_nred = 0;
    void ctem_forward(const double *target, double *loss, int ck, bool want_grad) {
        adj_valid = false;
        const mslice_geometry &g = H.g;
        if (cfg.mode != MSLICE_MODE_CTEM) throw StateError("the image loss needs a CTEM simulation");
        if (cfg.mixed_static > 1) throw Unsupported("gradients are implemented without mixed static potentials");
        if (cfg.plasmon) throw Unsupported("gradients are implemented without plasmon scattering");
        if (!atoms_set) throw StateError("atoms not set");
        const int S = g.n_slices;
        const int c = ck <= 0 ? (int)std::ceil(std::sqrt((double)S)) : std::min(ck, S);
        const int n_ck = (S + c - 1) / c;
        const cplx<R> *tw = ctx->twiddles<R>(N);
        const R a = (R)(1.0 / N), b = (R)(s2d * s2d * N), ds = (R)s2d;
        const int all_tiles = N / ops.cols_per_tile;
        // work buffers persist across calls (grow only): no allocation or implicit device sync per call
        E.ensure(ctx, (size_t)S * NN);
        ensure_waves(1);
        w1.ensure(ctx, NN); w2.ensure(ctx, NN);
        tgt.ensure(ctx, NN);
        const int nred = reduction_blocks();
        part.ensure(ctx, 3 * (size_t)nred);
        MS_CUDA(cudaMemcpyAsync(tgt.p, target, NN * sizeof(double), cudaMemcpyHostToDevice, st()));
        // raw E_s = exp(i sigma V_s) for every slice, then T_s = bandlimit(E_s)
        potentials(E.p, 0, S);
        MS_CUDA(cudaMemcpyAsync(trans.p, E.p, (size_t)S * NN * sizeof(C), cudaMemcpyDeviceToDevice, st()));
        band_limit(trans.p, S);
        trans_built = true;
        if (want_grad) {
            ck_buf.ensure(ctx, (size_t)n_ck * NN);
            save.ensure(ctx, (size_t)(c == 1 ? S : c) * NN);
        }
        PropTables<R> pt{px.p, py.p, kx2.p, ky2.p, k_prop * k_prop, ycut.p, ctx->step_err, pxe.p, pye.p};
        DetArgs nodet{detmask.p, 0, partials.p};
        // forward: plane wave through every slice, checkpoints of the row-transformed state
        plane_wave_state<R>(st(), N, wave.p);
        for (int s = 0; s < S; s++) {
            if (want_grad && s % c == 0)
                MS_CUDA(cudaMemcpyAsync(ck_buf.p + (size_t)(s / c) * NN, wave.p, NN * sizeof(C), cudaMemcpyDeviceToDevice, st()));
            if (want_grad && c == 1) ops.row_step_save(st(), wave.p, 1, trans.p + (size_t)s * NN, tw, a, save.p + (size_t)s * NN);
            else ops.row_step(st(), wave.p, 1, trans.p + (size_t)s * NN, tw, a, N, N, 1, nullptr, 0, 0, ctx->step_err);
            bool last = s == S - 1;
            ops.col_step(st(), wave.p, 1, tw, pt, b, ds, nodet, last ? recip.p : nullptr, last ? COL_STEP_DET : COL_STEP,
                         all_tiles, 0, 0);
            ctx->launches += 2;
        }
        // image W = s2d Dinv(H Recip), loss, G_W = 4 (I - target) W
        ctem_transfer<R>(st(), N, recip.p, w1.p, kx.p, ky.p, g.wavelength, aberr(cfg.C10), cfg.obj_ap, cfg.obj_ap_smooth,
                         cfg.alpha, cfg.delta);
        ops.row_fft(st(), w1.p, w1.p, 1, tw, (R)1, +1);
        ops.col_fft(st(), w1.p, w1.p, 1, tw, (R)s2d, +1);
        image_loss<R>(st(), NN, w1.p, tgt.p, w2.p, part.p);
        ctx->launches += 4;
        std::vector<double> hp((size_t)nred);
        MS_CUDA(cudaMemcpyAsync(hp.data(), part.p, nred * sizeof(double), cudaMemcpyDeviceToHost, st()));
        MS_CUDA(cudaStreamSynchronize(st()));
        double L = 0;
        for (int i = 0; i < nred; i++) L += hp[i];
        if (loss) *loss = L;
        if (want_grad) {
            adj_c = c;
            adj_nck = n_ck;
            adj_nred = nred;
            adj_token++;
            adj_valid = true;
        }
    }

    // The backward half: dL/dxyz, dL/dC10, dL/dC30 from the state of the last ctem_forward with want_grad.
    void ctem_backward(double *gxyz, double *g10, double *g30) {
        if (!adj_valid) throw StateError("no forward state for the adjoint (run mslice_ctem_loss_forward; any other call on "
                                         "the simulation in between invalidates it)");
        adj_valid = false;
        const mslice_geometry &g = H.g;
        const int S = g.n_slices;
        const int c = adj_c, n_ck = adj_nck, nred = adj_nred;
        const cplx<R> *tw = ctx->twiddles<R>(N);
        const R a = (R)(1.0 / N), b = (R)(s2d * s2d * N), ds = (R)s2d;
        const int all_tiles = N / ops.cols_per_tile;
        PropTables<R> pt{px.p, py.p, kx2.p, ky2.p, k_prop * k_prop, ycut.p, ctx->step_err, pxe.p, pye.p};
        DetArgs nodet{detmask.p, 0, partials.p};
        std::vector<double> hp(3 * (size_t)nred);
        // G_Y = s2d D(G_W); G_Recip = conj(H) G_Y and dL/dC10, dL/dC30
        ops.row_fft(st(), w2.p, w2.p, 1, tw, (R)1, -1);
        ops.col_fft(st(), w2.p, w2.p, 1, tw, (R)s2d, -1);
        image_backward<R>(st(), N, recip.p, w2.p, w1.p, kx.p, ky.p, g.wavelength, aberr(cfg.C10), cfg.obj_ap,
                          cfg.obj_ap_smooth, cfg.alpha, cfg.delta, part.p + nred, part.p + 2 * (size_t)nred);
        // backward state D_r G_{u_{S-1}} = s2d N Dinv_c(conj(P) G_Recip)
        mul_conj_prop<R>(st(), N, w1.p, px.p, py.p, kx2.p, ky2.p, k_prop * k_prop, (R)1);
        ops.col_fft(st(), w1.p, wave.p, 1, tw, (R)(s2d * N), +1);
        ctx->launches += 5;
        // sorted atoms of each slice
        const size_t nb = (size_t)g.blocks_x * g.blocks_y;
        std::vector<int> hbs((size_t)S * nb + 1);
        MS_CUDA(cudaMemcpyAsync(hbs.data(), block_start.p, hbs.size() * sizeof(int), cudaMemcpyDeviceToHost, st()));
        MS_CUDA(cudaStreamSynchronize(st()));
        const int n_in = hbs.back();
        const int ncomp = cfg.full3d ? 3 : 2;   // gradient components gathered per atom (z only under the full 3-D model)
        gxy.ensure(ctx, ncomp * (size_t)std::max(n_in, 1));
        {   // scratch of the atom gather: the atoms of the largest checkpoint segment
            int mx = 1;
            for (int s0 = 0; s0 < S; s0 += c) {
                const int s1 = std::min(s0 + c, S);
                mx = std::max(mx, hbs[(size_t)s1 * nb] - hbs[(size_t)s0 * nb]);
            }
            gwork.ensure(ctx, (size_t)atom_grad_work_doubles(mx));
        }
        MS_CUDA(cudaMemsetAsync(gxy.p, 0, ncomp * (size_t)std::max(n_in, 1) * sizeof(double), st()));
        // gT and gV of every slice of a segment, so that the band limit, gV and the atom gather run once per
        // segment over all its slices (batch-1 launches of those kernels leave most of the GPU idle)
        fw.ensure(ctx, NN); gT.ensure(ctx, (size_t)c * NN); gV.ensure(ctx, (size_t)c * NN);
        PropTables<R> ptc{pxc.p, pyc.p, kx2.p, ky2.p, k_prop * k_prop, ycut.p, ctx->step_err, pxec.p, pyec.p};
        for (int k = n_ck - 1; k >= 0; k--) {
            const int s0 = k * c, s1 = std::min(s0 + c, S), m = s1 - s0;
            if (c > 1) {   // recompute psi_s of the segment from its checkpoint
                MS_CUDA(cudaMemcpyAsync(fw.p, ck_buf.p + (size_t)k * NN, NN * sizeof(C), cudaMemcpyDeviceToDevice, st()));
                for (int s = s0; s < s1; s++) {
                    ops.row_step_save(st(), fw.p, 1, trans.p + (size_t)s * NN, tw, a, save.p + (size_t)(s - s0) * NN);
                    if (s < s1 - 1) ops.col_step(st(), fw.p, 1, tw, pt, b, ds, nodet, nullptr, COL_STEP, all_tiles, 0, 0);
                    ctx->launches += s < s1 - 1 ? 2 : 1;
                }
            }
            for (int s = s1 - 1; s >= s0; s--) {
                check_cancel();
                if (s < S - 1) ops.col_step(st(), wave.p, 1, tw, ptc, b, ds, nodet, nullptr, COL_STEP, all_tiles, 0, 0);
                const C *psi = save.p + (size_t)(c == 1 ? s : s - s0) * NN;
                ops.row_adjoint(st(), wave.p, 1, trans.p + (size_t)s * NN, tw, a, psi, gT.p + (size_t)(s - s0) * NN);
                ctx->launches += s < S - 1 ? 2 : 1;
            }
            band_limit(gT.p, m);   // G_E = bandlimit(G_T): the band limit is self-adjoint
            grad_v<R>(st(), (size_t)m * NN, E.p + (size_t)s0 * NN, gT.p, g.sigma, gV.p);
            ctx->launches++;
            if (cfg.full3d) {   // the full 3-D trapezoid pairs samples across atoms: replayed per pixel
                const PotParams pp = pot_params(s0);
                atom_grad_3d(st(), ctx->params.form, axs.p, ays.p, azs.p, aZs.p, block_start.p, ctx->prm_d, pp, m, gV.p,
                             g.dz / pp.integrals, gxy.p);
                ctx->launches++;
            }
            for (int t0 = 0; t0 < m && !cfg.full3d; t0 += kGradMaxSlices) {
                GradSlices gs{};
                gs.n = std::min(kGradMaxSlices, m - t0);
                gs.stride = NN;
                // the projected kernel's tilt-corrected radius: rho^2 = r^2 - sin^2(tilt) (r . e_phi)^2
                gs.tilt_s2 = std::sin(cfg.beam_tilt / 1000.0) * std::sin(cfg.beam_tilt / 1000.0);
                gs.cphi = std::cos(cfg.beam_azimuth);
                gs.sphi = std::sin(cfg.beam_azimuth);
                for (int i = 0; i <= gs.n; i++) gs.start[i] = hbs[(size_t)(s0 + t0 + i) * nb];
                atom_grad<R>(st(), gs, axs.p, ays.p, aZs.p, gV.p + (size_t)t0 * NN, N, g.sim_x[0], g.sim_y[0],
                             g.real_scale, ctx->params.form, params_dev(), ctx->params.i_count, ctx->potp_tab, gxy.p,
                             gwork.p);
                ctx->launches += 2;
            }
        }
        MS_CUDA(cudaMemcpyAsync(hp.data(), part.p, 3 * (size_t)nred * sizeof(double), cudaMemcpyDeviceToHost, st()));
        std::vector<double> hg(ncomp * (size_t)std::max(n_in, 1));
        std::vector<int> hidx(std::max<size_t>(n_atoms, 1));
        MS_CUDA(cudaMemcpyAsync(hg.data(), gxy.p, hg.size() * sizeof(double), cudaMemcpyDeviceToHost, st()));
        if (n_atoms) MS_CUDA(cudaMemcpyAsync(hidx.data(), idx_out.p, n_atoms * sizeof(int), cudaMemcpyDeviceToHost, st()));
        MS_CUDA(cudaStreamSynchronize(st()));
        double d10 = 0, d30 = 0;
        for (int i = 0; i < nred; i++) { d10 += hp[nred + i]; d30 += hp[2 * nred + i]; }
        if (g10) *g10 = d10;
        if (g30) *g30 = d30;
        if (gxyz) {
            std::fill(gxyz, gxyz + 3 * n_atoms, 0.0);
            for (int i = 0; i < n_in; i++) {   // sorted position i holds input atom idx_out[i]
                const int o = hidx[i];
                for (int q = 0; q < ncomp; q++) gxyz[3 * (size_t)o + q] = hg[ncomp * (size_t)i + q];
            }
        }
    }

    void ctem_loss_grad(const double *target, double *loss, double *gxyz, double *g10, double *g30, int ck,
                        bool want_grad) override {
        ctem_forward(target, loss, ck, want_grad);
        if (want_grad) ctem_backward(gxyz, g10, g30);
    }
    void ctem_loss_forward(const double *target, double *loss, int ck, unsigned long long *token) override {
        ctem_forward(target, loss, ck, true);
        if (token) *token = adj_token;
    }
    void ctem_loss_backward(unsigned long long token, double *gxyz, double *g10, double *g30) override {
        if (!adj_valid || token != adj_token)
            throw StateError("the forward state of this adjoint is gone: another forward or run used the simulation since");
        ctem_backward(gxyz, g10, g30);
    }

    void stem_plain(const int *pixels, size_t n, double *out) override {
        if constexpr (sizeof(R) != 8) {
            (void)pixels; (void)n; (void)out;
            throw StateError("the plain path is the FP64 path: create the simulation with double_precision = 1");
        } else {
            if (cfg.mode != MSLICE_MODE_STEM) throw StateError("simulation is not in STEM mode");
            if (!trans_built) build_transmission();
            const mslice_geometry &g = H.g;
            PlainArgs a;
            std::memset(&a, 0, sizeof(a));
            a.n = N; a.n_slices = g.n_slices; a.n_det = cfg.n_detectors; a.n_outputs = g.n_outputs;
            a.slice_step = cfg.intermediate_slices; a.scan_nx = cfg.stem_pixels_x;
            a.kx = kx.p; a.ky = ky.p; a.chi = chi.p; a.trans = (const double2 *)trans.p;
            a.dz = g.dz; a.beam_k = g.wavenumber; a.beam_kx = g.wavevector[0]; a.beam_ky = g.wavevector[1];
            a.beam_kz = g.wavevector[2]; a.k_max_prop = k_prop;
            a.start_x = cfg.stem_area[0]; a.start_y = cfg.stem_area[2];
            a.step_x = (cfg.stem_area[1] - cfg.stem_area[0]) / cfg.stem_pixels_x;
            a.step_y = (cfg.stem_area[3] - cfg.stem_area[2]) / cfg.stem_pixels_y;
            a.sim_x0 = g.sim_x[0]; a.sim_y0 = g.sim_y[0];
            a.fft_scale = s2d;
            for (int d = 0; d < cfg.n_detectors; d++) {
                a.innerPx[d] = cfg.detectors[d].inner / g.angle_scale;
                a.outerPx[d] = cfg.detectors[d].outer / g.angle_scale;
                a.xcPx[d] = cfg.detectors[d].xcentre / g.angle_scale;
                a.ycPx[d] = cfg.detectors[d].ycentre / g.angle_scale;
            }
            a.launches = &ctx->launches;
            plain_stem(st(), a, plain_work, pixels, n, out);
        }
    }
};

template <class R> PassOps<R> pass_ops(int n) {
    switch (n) {
#define MS_CASE(N) case N: return make_pass_ops<R, N>();
        MS_SIZES(MS_CASE)
#undef MS_CASE
    }
    throw Unsupported("grid size " + std::to_string(n) + " is not built into this library");
}
template PassOps<float> pass_ops<float>(int);
template PassOps<double> pass_ops<double>(int);

}  // namespace ms

// =================================================================================================
// C ABI
// =================================================================================================
struct mslice_sim;
struct mslice_ctx {
    ms::Ctx impl;
    std::vector<mslice_sim *> sims;   // simulations created on this context; destroyed with it
};
struct mslice_sim {
    mslice_ctx *ctx;
    std::unique_ptr<ms::SimBase> impl;
};

namespace {
template <class F> int guarded(F &&f) {
    // clear a non-sticky error a previous call may have left in this thread's runtime state
    cudaGetLastError();
    try {
        f();
        return MSLICE_OK;
    } catch (const ms::ArgError &e) { ms::g_last_error = e.what(); return MSLICE_ERR_ARG; }
    catch (const ms::StateError &e) { ms::g_last_error = e.what(); return MSLICE_ERR_STATE; }
    catch (const ms::OomError &e) { ms::g_last_error = e.what(); return MSLICE_ERR_OOM; }
    catch (const ms::Cancelled &e) { ms::g_last_error = e.what(); return MSLICE_ERR_CANCELLED; }
    catch (const ms::Unsupported &e) { ms::g_last_error = e.what(); return MSLICE_ERR_UNSUPPORTED; }
    catch (const ms::CudaError &e) { ms::g_last_error = e.what(); return MSLICE_ERR_CUDA; }
    catch (const std::bad_alloc &) { ms::g_last_error = "host allocation failed"; return MSLICE_ERR_OOM; }
    catch (const std::exception &e) { ms::g_last_error = e.what(); return MSLICE_ERR_ARG; }
    catch (...) { ms::g_last_error = "unknown error"; return MSLICE_ERR_ARG; }
}
void need(bool c, const char *what) {
    if (!c) throw ms::ArgError(what);
}
void use_device(mslice_ctx *c) { MS_CUDA(cudaSetDevice(c->impl.device)); }
}  // namespace

extern "C" {

const char *mslice_version(void) { return "mslice-b200 1 (sm_100a)"; }
const char *mslice_last_error(void) { return ms::g_last_error.c_str(); }

int mslice_ctx_create(int device, mslice_ctx **out) {
    return guarded([&] {
        need(out != nullptr, "out is null");
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) {
            cudaGetLastError();
            throw ms::CudaError(std::string("no CUDA device available: ") + cudaGetErrorString(e));
        }
        need(device >= 0 && device < n, "device index out of range");
        MS_CUDA(cudaSetDevice(device));
        auto c = std::make_unique<mslice_ctx>();
        c->impl.device = device;
        MS_CUDA(cudaStreamCreateWithFlags(&c->impl.stream, cudaStreamNonBlocking));
        MS_CUDA(cudaMalloc(&c->impl.step_err, sizeof(int)));
        MS_CUDA(cudaMemset(c->impl.step_err, 0, sizeof(int)));
        *out = c.release();
    });
}

int mslice_ctx_destroy(mslice_ctx *ctx) {
    return guarded([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->impl.device);
        cudaStreamSynchronize(ctx->impl.stream);
        for (mslice_sim *s : ctx->sims) delete s;   // simulations still alive go with their context
        ctx->sims.clear();
        delete ctx;
        cudaGetLastError();
    });
}

int mslice_ctx_set_memory_limit(mslice_ctx *ctx, size_t bytes) {
    return guarded([&] {
        need(ctx != nullptr, "ctx is null");
        ctx->impl.mem_limit = bytes;
    });
}

int mslice_params_load(mslice_ctx *ctx, int form, int i_per_atom, const double *p, size_t n) {
    return guarded([&] {
        need(ctx != nullptr && (p != nullptr || n == 0), "null argument");
        need(form >= 0 && form <= 2, "unknown parameterisation form");
        need(i_per_atom > 0, "terms per atom must be positive");
        size_t per = (size_t)i_per_atom * (form == MSLICE_KIRKLAND ? 4 : 2);
        if (form == MSLICE_KIRKLAND) need(i_per_atom <= 3, "Kirkland tables hold at most 3 terms of each kind");
        else need(i_per_atom <= 5, "Peng/Lobato tables hold at most 5 terms");
        // Parameterisation (structureparameters.h:30-33)
        if (n % per != 0 || n == 0) throw ms::ArgError("Parameterisation does not contain correct parameters per atom");
        // the kernels index (Z-1)*12 or (Z-1)*10 (projected_d.cl:110,148,167)
        size_t stride = form == MSLICE_KIRKLAND ? 12 : 10;
        need(n % stride == 0, "parameter table must hold 12 (Kirkland) or 10 (Peng/Lobato) values per element");
        use_device(ctx);
        ms::Ctx &c = ctx->impl;
        c.params.form = form;
        c.params.i_count = i_per_atom;
        c.params.values.assign(p, p + n);
        c.params.max_z = (int)(n / stride);
        if (c.prm_d) { c.release(c.prm_d, c.prm_n * sizeof(double)); c.prm_d = nullptr; }
        if (c.prm_f) { c.release(c.prm_f, c.prm_n * sizeof(float)); c.prm_f = nullptr; }
        c.prm_n = n;
        c.prm_d = (double *)c.alloc(n * sizeof(double));
        c.prm_f = (float *)c.alloc(n * sizeof(float));
        std::vector<float> pf(p, p + n);
        MS_CUDA(cudaMemcpy(c.prm_d, p, n * sizeof(double), cudaMemcpyHostToDevice));
        MS_CUDA(cudaMemcpy(c.prm_f, pf.data(), n * sizeof(float), cudaMemcpyHostToDevice));
        if (c.pot3_tab) { c.release(c.pot3_tab, c.pot3_n * sizeof(float4)); c.pot3_tab = nullptr; }
        const std::vector<float4> t3 = ms::pot3_table(form, i_per_atom, c.params.values, c.params.max_z);
        c.pot3_n = t3.size();
        c.pot3_tab = (float4 *)c.alloc(t3.size() * sizeof(float4));
        MS_CUDA(cudaMemcpy(c.pot3_tab, t3.data(), t3.size() * sizeof(float4), cudaMemcpyHostToDevice));
        if (c.potp_tab) { c.release(c.potp_tab, c.potp_n * sizeof(float2)); c.potp_tab = nullptr; }
        const std::vector<float2> tp = ms::potp_table(form, i_per_atom, c.params.values, c.params.max_z);
        c.potp_n = tp.size();
        c.potp_tab = (float2 *)c.alloc(tp.size() * sizeof(float2));
        MS_CUDA(cudaMemcpy(c.potp_tab, tp.data(), tp.size() * sizeof(float2), cudaMemcpyHostToDevice));
    });
}

int mslice_geometry_compute(const mslice_config *cfg, mslice_geometry *out) {
    return guarded([&] {
        need(cfg && out, "null argument");
        ms::HostGeom H;
        ms::compute_geometry(*cfg, H);
        *out = H.g;
    });
}

int mslice_sim_create(mslice_ctx *ctx, const mslice_config *cfg, mslice_sim **out) {
    return guarded([&] {
        need(ctx && cfg && out, "null argument");
        use_device(ctx);
        auto s = std::make_unique<mslice_sim>();
        s->ctx = ctx;
        if (cfg->double_precision) s->impl = std::make_unique<ms::Sim<double>>(&ctx->impl, *cfg);
        else s->impl = std::make_unique<ms::Sim<float>>(&ctx->impl, *cfg);
        ctx->sims.push_back(s.get());
        *out = s.release();
    });
}

int mslice_sim_destroy(mslice_sim *sim) {
    return guarded([&] {
        if (!sim) return;
        use_device(sim->ctx);
        cudaStreamSynchronize(sim->ctx->impl.stream);
        auto &v = sim->ctx->sims;
        v.erase(std::remove(v.begin(), v.end(), sim), v.end());
        delete sim;
    });
}

int mslice_sim_geometry(mslice_sim *sim, mslice_geometry *out) {
    return guarded([&] {
        need(sim && out, "null argument");
        *out = sim->impl->H.g;
    });
}

int mslice_set_progress(mslice_sim *sim, mslice_progress_cb cb, void *user) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        sim->impl->progress = cb;
        sim->impl->progress_user = user;
    });
}

int mslice_cancel(mslice_sim *sim) {
    if (!sim) return MSLICE_ERR_ARG;
    sim->impl->cancel.store(true);
    return MSLICE_OK;
}

int mslice_set_atoms(mslice_sim *sim, const int *Z, const double *x, const double *y, const double *z, size_t n) {
    return guarded([&] {
        need(sim && (n == 0 || (Z && x && y && z)), "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->set_atoms(Z, x, y, z, n, true);
    });
}

int mslice_get_sorted_atoms(mslice_sim *sim, int *Z, double *x, double *y, double *z, size_t cap, int *block_start,
                            size_t cap_block_start, int *block_ids, int *z_ids, size_t *n_out) {
    return guarded([&] {
        need(sim && Z && x && y && z && block_start && n_out, "null argument");
        use_device(sim->ctx);
        sim->impl->get_sorted(Z, x, y, z, cap, block_start, cap_block_start, block_ids, z_ids, n_out);
    });
}

int mslice_build_transmission(mslice_sim *sim) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->build_transmission();
        MS_CUDA(cudaStreamSynchronize(sim->ctx->impl.stream));
    });
}

int mslice_get_transmission(mslice_sim *sim, int slice, int band_limited, double *out) {
    return guarded([&] {
        need(sim && out, "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->get_transmission(slice, band_limited, out);
    });
}

int mslice_get_propagator(mslice_sim *sim, double *out) {
    return guarded([&] {
        need(sim && out, "null argument");
        use_device(sim->ctx);
        sim->impl->get_propagator(out);
    });
}

int mslice_get_probe(mslice_sim *sim, double x, double y, double *out) {
    return guarded([&] {
        need(sim && out, "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->get_probe(x, y, out);
    });
}

int mslice_stem_run(mslice_sim *sim, const int *pixels, size_t n_pixels, double *out) {
    return guarded([&] {
        need(sim && (n_pixels == 0 || (pixels && out)), "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->stem_run(pixels, n_pixels, out);
    });
}

int mslice_cbed_run(mslice_sim *sim, double *diff) {
    return guarded([&] {
        need(sim && diff, "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->cbed_run(diff);
    });
}

int mslice_ctem_run(mslice_sim *sim, double *ew, double *diff, double *image) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->ctem_run(ew, diff, image);
    });
}

int mslice_ctem_loss_grad(mslice_sim *sim, const double *target, double *loss, double *grad_xyz, double *grad_c10,
                          double *grad_c30, int checkpoint_every) {
    return guarded([&] {
        need(sim && target, "null argument");
        use_device(sim->ctx);
        sim->impl->ctem_loss_grad(target, loss, grad_xyz, grad_c10, grad_c30, checkpoint_every, true);
    });
}

int mslice_tune_batch(mslice_sim *sim, const int *candidates, int n_candidates, int reps, int *best_batch,
                      double *waves_per_second) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->tune_batch(candidates, candidates ? n_candidates : 1, reps, best_batch, waves_per_second);
    });
}

int mslice_set_step_variant(mslice_sim *sim, int col_variant, int row_variant) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->set_step_variant(col_variant, row_variant);
    });
}

int mslice_step_variant_name(mslice_sim *sim, int which, int index, char *buf, size_t cap) {
    return guarded([&] {
        need(sim && buf && cap > 0, "null argument");
        const std::string nm = sim->impl->step_variant_name(which, index);
        const size_t n = std::min(nm.size(), cap - 1);
        std::memcpy(buf, nm.data(), n);
        buf[n] = 0;
    });
}

int mslice_get_tuning(mslice_sim *sim, int *batch, int *col_variant, int *n_col_variants, int *row_variant,
                      int *n_row_variants) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        sim->impl->get_tuning(batch, col_variant, n_col_variants, row_variant, n_row_variants);
    });
}

int mslice_set_ccd(mslice_sim *sim, const double *dqe, const double *ntf, size_t n, int binning, double dose) {
    return guarded([&] {
        need(sim != nullptr && (n == 0 || (dqe != nullptr && ntf != nullptr)), "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->set_ccd(dqe, ntf, n, binning, dose);
    });
}

int mslice_set_c10_c30(mslice_sim *sim, double c10, double c30) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->set_c10_c30(c10, c30);
    });
}

int mslice_ctem_loss_forward(mslice_sim *sim, const double *target, double *loss, int checkpoint_every,
                             unsigned long long *token) {
    return guarded([&] {
        need(sim && target, "null argument");
        use_device(sim->ctx);
        sim->impl->ctem_loss_forward(target, loss, checkpoint_every, token);
    });
}

int mslice_ctem_loss_backward(mslice_sim *sim, unsigned long long token, double *grad_xyz, double *grad_c10,
                              double *grad_c30) {
    return guarded([&] {
        need(sim != nullptr, "null argument");
        use_device(sim->ctx);
        sim->impl->ctem_loss_backward(token, grad_xyz, grad_c10, grad_c30);
    });
}

int mslice_ctem_loss(mslice_sim *sim, const double *target, double *loss) {
    return guarded([&] {
        need(sim && target, "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->ctem_loss_grad(target, loss, nullptr, nullptr, nullptr, 0, false);
    });
}

int mslice_stage_configs(mslice_sim *sim, int n_configs, const size_t *counts, const int *Z, const double *x,
                         const double *y, const double *z) {
    return guarded([&] {
        need(sim && counts && n_configs > 0, "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->stage(n_configs, counts, Z, x, y, z);
    });
}

int mslice_stem_run_staged(mslice_sim *sim) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->run_staged(MSLICE_MODE_STEM);
    });
}

int mslice_cbed_run_staged(mslice_sim *sim) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->run_staged(MSLICE_MODE_CBED);
    });
}

int mslice_stem_run_staged_async(mslice_sim *sim) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        if (sim->impl->cfg.mode != MSLICE_MODE_STEM) throw ms::StateError("simulation is not in STEM mode");
        sim->impl->run_staged_async();
    });
}

int mslice_sim_wait(mslice_sim *sim) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        sim->impl->wait_run();
    });
}

int mslice_staged_result(mslice_sim *sim, double *out, size_t cap) {
    return guarded([&] {
        need(sim && out, "null argument");
        use_device(sim->ctx);
        sim->impl->staged_result(out, cap);
    });
}

int mslice_stem_simulate(mslice_sim *sim, int n_configs, const size_t *counts, const int *Z, const double *x,
                         const double *y, const double *z, double *out, size_t cap) {
    return guarded([&] {
        need(sim && counts && out && n_configs > 0, "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->stage(n_configs, counts, Z, x, y, z);
        sim->impl->run_staged(MSLICE_MODE_STEM);
        sim->impl->staged_result(out, cap);
    });
}

int mslice_stem_run_plain(mslice_sim *sim, const int *pixels, size_t n_pixels, double *out) {
    return guarded([&] {
        need(sim && (n_pixels == 0 || (pixels && out)), "null argument");
        use_device(sim->ctx);
        sim->impl->adj_valid = false;   // the adjoint's forward state is gone
        sim->impl->stem_plain(pixels, n_pixels, out);
    });
}

int mslice_fft2(mslice_ctx *ctx, int n, int inverse, int double_precision, int batch, const double *in, double *out) {
    return guarded([&] {
        need(ctx && in && out && batch > 0, "null argument");
        use_device(ctx);
        ms::Ctx &c = ctx->impl;
        const size_t NN = (size_t)n * n, tot = NN * batch;
        const double s2d = (double)(1.0f / sqrtf((float)NN));
        auto run = [&](auto tag) {
            using R = decltype(tag);
            ms::PassOps<R> ops = ms::pass_ops<R>(n);
            ms::DevBuf<ms::cplx<R>> d;
            ms::DevBuf<double2> dd;
            d.ensure(&c, tot);
            dd.ensure(&c, tot);
            MS_CUDA(cudaMemcpyAsync(dd.p, in, tot * sizeof(double2), cudaMemcpyHostToDevice, c.stream));
            ms::convert_from_double<R>(c.stream, tot, dd.p, d.p);
            const ms::cplx<R> *tw = c.twiddles<R>(n);
            int sign = inverse ? +1 : -1;
            ops.row_fft(c.stream, d.p, d.p, batch, tw, (R)1, sign);
            ops.col_fft(c.stream, d.p, d.p, batch, tw, (R)s2d, sign);
            ms::convert_to_double<R>(c.stream, tot, d.p, dd.p);
            c.launches += 4;
            MS_CUDA(cudaMemcpyAsync(out, dd.p, tot * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
            MS_CUDA(cudaStreamSynchronize(c.stream));
        };
        if (double_precision) run(double(0));
        else run(float(0));
    });
}

int mslice_ctx_stream(mslice_ctx *ctx, void **stream) {
    return guarded([&] {
        need(ctx && stream, "null argument");
        *stream = (void *)ctx->impl.stream;
    });
}

int mslice_ctx_launch_count(mslice_ctx *ctx, unsigned long long *count) {
    return guarded([&] {
        need(ctx && count, "null argument");
        *count = ctx->impl.launches;
    });
}

int mslice_profile_enable(mslice_sim *sim, int on) {
    return guarded([&] {
        need(sim != nullptr, "sim is null");
        use_device(sim->ctx);
        MS_CUDA(cudaStreamSynchronize(sim->ctx->impl.stream));
        sim->impl->flush_profile();
        sim->impl->prof = on != 0;
    });
}

int mslice_profile_read(mslice_sim *sim, int kernel, double *total_ms, unsigned long long *launches, double *bytes,
                        int reset) {
    return guarded([&] {
        need(sim && total_ms && launches, "null argument");
        need(kernel >= 0 && kernel < MSLICE_K_COUNT, "unknown kernel kind");
        use_device(sim->ctx);
        MS_CUDA(cudaStreamSynchronize(sim->ctx->impl.stream));
        sim->impl->flush_profile();
        *total_ms = sim->impl->prof_ms[kernel];
        *launches = sim->impl->prof_n[kernel];
        if (bytes) *bytes = sim->impl->prof_bytes[kernel];
        if (reset)
            for (int k = 0; k < MSLICE_K_COUNT; k++) {
                sim->impl->prof_ms[k] = 0;
                sim->impl->prof_n[k] = 0;
                sim->impl->prof_bytes[k] = 0;
            }
    });
}

int mslice_incoherence_draws(const mslice_config *cfg, int pass, const int *pixels, size_t n_pixels, double *defocus,
                             int *sets, int n_slices, int n_builds, double *shift) {
    return guarded([&] {
        need(cfg != nullptr && (pixels != nullptr || n_pixels == 0), "null argument");
        need(n_slices >= 0 && n_builds >= 0, "negative count");
        for (size_t i = 0; i < n_pixels; i++) {
            if (defocus)
                defocus[i] = cfg->chromatic ? ms::draws::defocus_change(cfg->seed, pass, pixels[i], cfg->chromatic_cc,
                                                                          cfg->chromatic_hwhm_neg, cfg->chromatic_hwhm_pos,
                                                                          cfg->voltage)
                                            : 0.0;
            if (sets)
                for (int s = 0; s < n_slices; s++)
                    sets[i * n_slices + s] =
                        cfg->mixed_static > 1 ? ms::draws::set_of(cfg->seed, pass, pixels[i], s, cfg->mixed_static) : 0;
        }
        if (shift)
            for (int b = 0; b < n_builds; b++) {
                double dx = 0, dy = 0;
                if (cfg->source_size && cfg->mode != MSLICE_MODE_CTEM) ms::draws::source_shift(cfg->seed, b, cfg->source_fwhm, dx, dy);
                shift[2 * b] = dx;
                shift[2 * b + 1] = dy;
            }
    });
}

int mslice_plasmon_draws(const mslice_config *cfg, unsigned long long job, double thickness, double *depths, size_t cap,
                         size_t *n_depths, int n_events, double *angles) {
    return guarded([&] {
        need(cfg != nullptr, "null argument");
        if (depths || n_depths) {
            need(depths != nullptr && n_depths != nullptr, "depths and n_depths go together");
            std::vector<double> d;
            if (!ms::draws::plasmon_depths(cfg->seed, job, cfg->plasmon_mfp, thickness, cfg->plasmon_individual, d))
                throw ms::ArgError("Could not generate valid plasmon configuration");
            need(d.size() <= cap, "depth capacity too small");
            std::copy(d.begin(), d.end(), depths);
            *n_depths = d.size();
        }
        if (angles)
            for (int e = 0; e < n_events; e++)
                ms::draws::plasmon_angles(cfg->seed, job, (uint64_t)e, cfg->plasmon_char_angle, cfg->plasmon_crit_angle,
                                          angles[2 * e], angles[2 * e + 1]);
    });
}

int mslice_last_timing(mslice_sim *sim, double *ms3) {
    return guarded([&] {
        need(sim && ms3, "null argument");
        for (int i = 0; i < 3; i++) ms3[i] = sim->impl->timing[i];
    });
}

}  // extern "C"
