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

namespace ms {
namespace draws {

enum Kind : uint64_t { SET = 1, DEFOCUS = 2, SOURCE = 3, DOSE = 4 };

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

}  // namespace draws
}  // namespace ms
