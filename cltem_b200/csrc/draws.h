// Seeded random draws of the incoherence effects (host code).
//
// The reference draws from clock-seeded std::mt19937_64 engines in call order
// (src/simulation/incoherence/chromaticaberration.cpp:8-16, probesourcesize.cpp:8-12,
// src/simulation/microscope/simulationgeneral.cpp:44-46), so its runs cannot be repeated. Here every draw
// is a pure function of (seed, kind, pass, index...): a run is reproducible, independent of batching and
// of the order in which probes are processed, and a CPU restatement can make exactly the same draws.
// Each draw hashes its coordinates with the SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014); normals come from the Box-Muller transform.
#pragma once
#include <cmath>
#include <cstdint>
#include <limits>
#include <vector>

namespace ms {
namespace draws {

enum Kind : uint64_t { SET = 1, DEFOCUS = 2, SOURCE = 3, DOSE = 4, PLASMON_DEPTH = 5, PLASMON_ANGLE = 6 };

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t key(uint64_t seed, uint64_t kind, uint64_t a, uint64_t b, uint64_t c) {
    return mix64(mix64(mix64(mix64(seed ^ (kind << 56)) ^ a) ^ b) ^ c);
}
// uniform on [0, 1) from the top 53 bits
inline double uniform(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
// standard normal (Box-Muller, cosine branch); 1 - u keeps the logarithm finite
inline double normal(uint64_t h1, uint64_t h2) {
    const double u1 = 1.0 - uniform(h1), u2 = uniform(h2);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
}

// Transmission set of scan pixel `pixel` at `slice` in pass `pass`: uniform over 0..n_sets-1, the role of
// dist(rng) in SimulationGeneral::doMultiSliceStep (simulationgeneral.cpp:740-742).
inline int set_of(uint64_t seed, int pass, int pixel, int slice, int n_sets) {
    return (int)(key(seed, SET, (uint64_t)pass, (uint64_t)pixel, (uint64_t)slice) % (uint64_t)n_sets);
}

// HWHM -> sigma (ChromaticAberration::setHalfWidthHalfMax*, chromaticaberration.cpp:104-112)
inline double sigma_of_hwhm(double hwhm) { return 2.0 * std::fabs(hwhm) / (2.0 * std::sqrt(2.0 * std::log(2.0))); }
// FWHM -> sigma (ProbeSourceSize::setFullWidthHalfMax, probesourcesize.cpp:18-20)
inline double sigma_of_fwhm(double fwhm) { return fwhm / (2.0 * std::sqrt(2.0 * std::log(2.0))); }

// Defocus change (Å) of the probe of `pixel` in pass `pass`: ChromaticAberration::getFocusChange with the
// two-sided half-normal of generateDist (chromaticaberration.cpp:39-56, 88-95). cc in mm, energies in eV.
inline double defocus_change(uint64_t seed, int pass, int pixel, double cc_mm, double hwhm_neg, double hwhm_pos,
                             double kilo_volts) {
    const double sig_neg = sigma_of_hwhm(hwhm_neg), sig_pos = sigma_of_hwhm(hwhm_pos);
    double ratio = sig_neg / sig_pos;
    ratio = ratio / (ratio + 1.0);
    const double selector = uniform(key(seed, DEFOCUS, (uint64_t)pass, (uint64_t)pixel, 0));
    const double d1 = std::fabs(normal(key(seed, DEFOCUS, (uint64_t)pass, (uint64_t)pixel, 1),
                                       key(seed, DEFOCUS, (uint64_t)pass, (uint64_t)pixel, 2)));
    const double dist = selector >= ratio ? d1 * sig_pos : -1.0 * (d1 * sig_neg);
    return 10000 * cc_mm * dist / kilo_volts;
}

// Shift (Å) of the transmission's reference frame for transmission build `build`: two draws of
// ProbeSourceSize::getOffset (probesourcesize.cpp:29-31) as taken in SimulationCbed::initialiseSimulation
// (simulationcbed.cpp:103-113).
inline void source_shift(uint64_t seed, int build, double fwhm, double &dx, double &dy) {
    const double sd = sigma_of_fwhm(fwhm);
    dx = normal(key(seed, SOURCE, (uint64_t)build, 0, 0), key(seed, SOURCE, (uint64_t)build, 0, 1)) * sd;
    dy = normal(key(seed, SOURCE, (uint64_t)build, 1, 0), key(seed, SOURCE, (uint64_t)build, 1, 1)) * sd;
}

// Poisson deviate of mean lam for image pixel `pixel` in dose pass `pass` (the role of
// std::poisson_distribution in SimulationCtem::simulateImageDose, simulationctem.cpp:224-236): inversion by
// sequential search for lam < 10, else the transformed rejection method PTRS of W. Hormann ("The
// transformed rejection method for generating Poisson random variables", Insurance: Mathematics and
// Economics 12 (1993) 39-45). The i-th uniform of a pixel is uniform(key(seed, DOSE, pass, pixel, i)).
inline double poisson(uint64_t seed, int pass, uint64_t pixel, double lam) {
    if (!(lam > 0)) return 0.0;
    uint64_t i = 0;
    auto U = [&]() { return uniform(key(seed, DOSE, (uint64_t)pass, pixel, i++)); };
    if (lam < 10.0) {
        double p = std::exp(-lam), F = p;
        const double u = U();
        int k = 0;
        while (u > F && k < 1000) {
            k++;
            p *= lam / k;
            F += p;
        }
        return (double)k;
    }
    const double slam = std::sqrt(lam), loglam = std::log(lam);
    const double b = 0.931 + 2.53 * slam, a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4), vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int it = 0; it < 1000; it++) {
        const double u = U() - 0.5, v = U();
        const double us = 0.5 - std::fabs(u);
        if (!(us > 0)) continue;
        const double k = std::floor((2.0 * a / us + b) * u + lam + 0.43);
        if (us >= 0.07 && v <= vr) return k;
        if (k < 0 || (us < 0.013 && v > us)) continue;
        if (std::log(v) + std::log(invalpha) - std::log(a / (us * us) + b) <= -lam + k * loglam - std::lgamma(k + 1.0))
            return k;
    }
    return std::floor(lam);
}

// ---- plasmon scattering (PlasmonScattering, src/simulation/incoherence/inelastic/plasmon.cpp) ----------------
// The reference draws every plasmon number from one clock-seeded std::uniform_real_distribution<>(0, 1) stream in
// call order: the depth tables of all jobs at set-up (clTEM_cmd main.cpp:710-727), the angles of each event
// while the jobs run. Here each draw is a function of (seed, job, attempt or event, index).

// Scattering depths (Å) of job `job` for a crystal `thickness` Å thick: getDistancesforCombined
// (plasmon.cpp:93-120), cumulative distances -mfp ln(u) while they stay <= thickness, then +inf. With
// `individual` > 0 it is getDistancesForIndividual (:69-91): whole tables are drawn again (attempt 0, 1, ...)
// until one has exactly `individual` entries counting the closing +inf, i.e. individual - 1 scattering
// events, as the reference compares the table's size with the requested number. Returns false where the
// reference gives up (more than 1e10 events in a table; or, for `individual`, no table of the asked size
// within max_attempts attempts).
inline bool plasmon_depths(uint64_t seed, uint64_t job, double mfp, double thickness, int individual,
                           std::vector<double> &out, uint64_t max_attempts = 10000000ull) {
    auto table = [&](uint64_t attempt, std::vector<double> &d) {
        d.clear();
        uint64_t i = 0;
        auto distance = [&]() { return -1.0 * mfp * std::log(uniform(key(seed, PLASMON_DEPTH, job, attempt, i++))); };
        double t = distance();
        double c = 0;
        while (t <= thickness && c < 1e10) {
            d.push_back(t);
            t += distance();
            c++;
        }
        if (c >= 1e10) { d.clear(); return false; }
        d.push_back(std::numeric_limits<double>::infinity());
        return true;
    };
    if (individual <= 0) return table(0, out) && !out.empty();
    for (uint64_t a = 0; a < max_attempts; a++) {
        if (table(a, out) && out.size() == (size_t)individual) return true;
    }
    out.clear();
    return false;
}

// Polar angle (mrad) and azimuth (rad) of scattering event `event` of job `job` (getScatteringPolar,
// plasmon.cpp:22-31, then getScatteringAzimuth, :17-20, in the order simulate() asks for them).
inline void plasmon_angles(uint64_t seed, uint64_t job, uint64_t event, double char_angle, double crit_angle,
                           double &polar_mrad, double &azimuth) {
    const double crit_2 = crit_angle * crit_angle, char_2 = char_angle * char_angle;
    const double u1 = uniform(key(seed, PLASMON_ANGLE, job, event, 0));
    const double ang_2 = char_2 * (std::pow((crit_2 + char_2) / char_2, u1) - 1);
    polar_mrad = std::sqrt(ang_2);
    azimuth = 2.0 * 3.14159265358979323846 * uniform(key(seed, PLASMON_ANGLE, job, event, 1));
}

// Utils::generateRotationAroundVector (vectorutils.cpp:8-19): Rodrigues' rotation by `angle` about `ax`
// (normalised first), applied to v.
inline void rotate_about(const double ax_in[3], double angle, double v[3]) {
    const double n = std::sqrt(ax_in[0] * ax_in[0] + ax_in[1] * ax_in[1] + ax_in[2] * ax_in[2]);
    const double a[3] = {ax_in[0] / n, ax_in[1] / n, ax_in[2] / n};
    const double s = std::sin(angle), c1 = 1 - std::cos(angle);
    // R = I + s [a]x + (1 - cos) [a]x^2, [a]x = ((0, -a2, a1), (a2, 0, -a0), (-a1, a0, 0))
    const double K[3][3] = {{0.0, -a[2], a[1]}, {a[2], 0.0, -a[0]}, {-a[1], a[0], 0.0}};
    double K2[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) K2[i][j] = K[i][0] * K[0][j] + K[i][1] * K[1][j] + K[i][2] * K[2][j];
    double r[3];
    for (int i = 0; i < 3; i++) {
        double acc = 0;
        for (int j = 0; j < 3; j++) acc += ((i == j ? 1.0 : 0.0) + K[i][j] * s + K2[i][j] * c1) * v[j];
        r[i] = acc;
    }
    v[0] = r[0]; v[1] = r[1]; v[2] = r[2];
}
// Utils::rotateVectorSpherical (vectorutils.cpp:21-31): both rotations are formed from the incoming axes,
// z is turned by theta about y and then by phi about the old z, y by phi about the old z.
inline void rotate_spherical(double z[3], double y[3], double theta, double phi) {
    const double z0[3] = {z[0], z[1], z[2]}, y0[3] = {y[0], y[1], y[2]};
    rotate_about(y0, theta, z);
    rotate_about(z0, phi, z);
    rotate_about(z0, phi, y);
}

}  // namespace draws
}  // namespace ms
