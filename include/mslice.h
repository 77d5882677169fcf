/*
 * mslice.h — C ABI of the B200 multislice engine (libmslice.so).
 *
 * This ABI replaces the two internal interfaces that clTEM's simulation path sits behind:
 *   - the kernel ABI: KernelSource/clKernel SetArg+run (src/simulation/kernels.h:22-101,
 *     src/simulation/clwrapper/clkernel.h:51-95) and clFourier::run (clwrapper/clfourier.h:70-98);
 *   - the job ABI: SimulationWorker<T>::Run(job) (src/simulation/microscope/simulationworker.cpp:8-61)
 *     returning images through SimulationManager::updateImages (src/simulation/simulationmanager.cpp:274-350).
 *
 * Conventions
 *   - Every entry point returns an int status (MSLICE_OK = 0). Nothing throws across the ABI;
 *     mslice_last_error() returns the message of the last failure on the calling thread.
 *   - Plain pointers and sizes only. Host arrays are caller-owned and copied.
 *   - One mslice_ctx per CUDA device; calls on one ctx (and its sims) are serialised by the caller,
 *     distinct ctxs may be driven from distinct host threads (clTEM's one-thread-per-device model,
 *     src/simulation/threading/threadpool.cpp:9-19).
 *   - Units are the reference's internal units after its JSON conversion
 *     (src/simulation/utilities/jsonutils.cpp:15-366): lengths in Å, aberration magnitudes in Å,
 *     aberration angles and azimuths in rad, apertures / tilt / detector radii in mrad, voltage in kV.
 *   - Complex arrays are interleaved (re, im) doubles, row-major with x fastest: element (x, y) of a
 *     res×res image is at index x + res*y, as in the reference kernels (e.g. kernels/complex_multiply_d.cl:21).
 *   - There is no CPU fallback: every compute entry point runs CUDA kernels on the ctx's device and
 *     fails with MSLICE_ERR_CUDA when no device is usable.
 */
#ifndef MSLICE_H
#define MSLICE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MSLICE_ABI_VERSION 1

/* status codes */
#define MSLICE_OK 0
#define MSLICE_ERR_ARG 1         /* invalid argument / config (clTEM: std::runtime_error from checks) */
#define MSLICE_ERR_CUDA 2        /* CUDA runtime / driver failure, or no device                        */
#define MSLICE_ERR_STATE 3       /* call out of order (e.g. run before atoms were set)                  */
#define MSLICE_ERR_CANCELLED 4   /* mslice_cancel() was honoured (clTEM: pool.isStopped())             */
#define MSLICE_ERR_OOM 5         /* device allocation failed or exceeded the ctx memory cap             */
#define MSLICE_ERR_UNSUPPORTED 6 /* valid request this build does not implement                         */

/* simulation modes, ids as src/simulation/utilities/enums.h:8-14 */
#define MSLICE_MODE_CTEM 1
#define MSLICE_MODE_STEM 2
#define MSLICE_MODE_CBED 3

/* parameterisation forms, as src/simulation/structure/structureparameters.h:16-20 */
#define MSLICE_KIRKLAND 0
#define MSLICE_PENG 1
#define MSLICE_LOBATO 2

#define MSLICE_MAX_DETECTORS 16

typedef struct mslice_ctx mslice_ctx;
typedef struct mslice_sim mslice_sim;

/* ComplexAberration (src/simulation/utilities/commonstructs.h:201-208): value = mag * exp(i ang). */
typedef struct mslice_aberration {
    double mag; /* Å */
    double ang; /* rad */
} mslice_aberration;

/* StemDetector (commonstructs.h:292-300). Radii and centre in mrad. */
typedef struct mslice_detector {
    char name[48];
    double inner, outer, xcentre, ycentre;
} mslice_detector;

/*
 * POD mirror of the SimulationManager fields the multislice path reads
 * (src/simulation/simulationmanager.h, defaults simulationmanager.cpp:8-50), after the reference's
 * JSON unit conversion. struct_limits are the limits of the UNDISPLACED structure as
 * CrystalStructure::updateLimits leaves them (structure/crystalstructure.cpp:238-267).
 */
typedef struct mslice_config {
    int mode;                    /* MSLICE_MODE_* */
    int double_precision;        /* 0: FP32 complex64 engine, 1: FP64 complex128 engine */
    int resolution;              /* grid side; clTEM allows {256,512,768,1024,1536,2048,3072,4096,8192},
                                    all built; with allow_any_resolution also 64, 96, 128 and 384 */
    int allow_any_resolution;    /* extension: accept other sizes of the form 2^a or 3*2^a (e.g. 384) */
    double slice_thickness;      /* Å */
    double slice_offset;         /* Å */
    double padding_xy;           /* default xy padding value p: padding = {-p, +p} (simulationcell.cpp:8) */
    double padding_z;            /* default z padding value p: {-p, +p} before rounding (simulationcell.cpp:43-61) */
    int full3d;                  /* full 3-D potential (transmission_potentials_full_3d) instead of projected */
    int full3d_integrals;        /* sub-slice integrals for full 3-D */
    double inverse_limit_factor; /* band limit as a fraction of k_max (reference default 2/3) */
    double struct_limits[6];     /* min_x, max_x, min_y, max_y, min_z, max_z (Å) */

    double voltage;              /* kV */
    double C10;                  /* Å */
    mslice_aberration C12, C21, C23;
    double C30;                  /* Å */
    mslice_aberration C32, C34, C41, C43, C45;
    double C50;                  /* Å */
    mslice_aberration C52, C54, C56;
    double cond_ap, cond_ap_smooth; /* mrad */
    double obj_ap, obj_ap_smooth;   /* mrad */
    double beam_tilt;            /* mrad */
    double beam_azimuth;         /* rad */
    double alpha;                /* mrad (CTEM spatial coherence, passed as beta to ctem_image) */
    double delta;                /* Å (CTEM defocus spread) */

    double ctem_area[4];         /* raw CTEM area: x start, x finish, y start, y finish (Å) */
    double stem_area[4];         /* raw STEM scan area (Å) */
    int stem_pixels_x, stem_pixels_y;
    double stem_padding;         /* StemArea padding (Å) */
    double cbed_x, cbed_y, cbed_padding;

    int n_detectors;
    mslice_detector detectors[MSLICE_MAX_DETECTORS];

    int intermediate_slices;     /* output every n slices (0 = only the exit) */
    int ctem_image;              /* CTEM: also form the objective-lens image */
    int probe_batch;             /* STEM probes propagated together (0 = engine default) */

    /* ---- incoherence (IncoherentEffects, src/simulation/incoherence/; all off when zero) ---- */
    int iterations;              /* passes of a staged run ("incoherence/iterations"); 0: one pass per staged
                                    configuration, pass i using configuration i */
    int mixed_static;            /* mixed static potentials: n > 1 transmission sets built from the first n staged
                                    configurations; every probe takes a random set at every slice
                                    (simulationgeneral.cpp:42-54,576-613,731-742) */
    int stem_moving_frame;       /* STEM without the static area ("stem/static area/enabled" false): each job
                                    simulates a window of +-stem_padding around its first pixel
                                    (SimulationManager::currentAreaBase, simulationmanager.cpp:485-505) */
    int stem_job_pixels;         /* pixels per job in the moving frame ("concurrent pixels"), >= 1 */
    int chromatic;               /* random defocus change per probe per pass (ChromaticAberration) */
    double chromatic_cc;         /* Cc (mm) */
    double chromatic_hwhm_neg, chromatic_hwhm_pos;   /* energy spread half widths (eV) */
    int source_size;             /* random shift of the transmission frame per build (ProbeSourceSize) */
    double source_fwhm;          /* Å */
    unsigned long long seed;     /* seed of every random draw (sets, defocus changes, frame shifts, plasmons) */

    /* ---- plasmon scattering (PlasmonScattering, src/simulation/incoherence/inelastic/plasmon.h) ---------- */
    int plasmon;                 /* 1: scattering events tilt the beam of each job ("inelastic scattering/plasmon") */
    int plasmon_individual;      /* 0: type "full"; n >= 1: type "individual" with "individual" n, which the reference
                                    meets with tables of n entries counting the closing +inf: n - 1 events */
    double plasmon_mfp;          /* mean free path (Å; the JSON's nm x 10) */
    double plasmon_char_angle;   /* characteristic angle (mrad) */
    double plasmon_crit_angle;   /* critical angle (mrad) */
} mslice_config;

/* Derived geometry (what SimulationManager / SimulationCell compute from a config). */
typedef struct mslice_geometry {
    double sim_x[2], sim_y[2];   /* paddedSimLimitsX/Y(0)   simulationmanager.cpp:434-440 */
    double full_x[2], full_y[2]; /* paddedFullLimitsX/Y     simulationmanager.cpp:446-452 */
    double z_lims[2];            /* paddedSimLimitsZ        simulationmanager.cpp:442-444 */
    double padding_z[2];         /* SimulationCell::roundPaddingZ  simulationcell.cpp:43-61 */
    double real_scale;           /* realScale               simulationmanager.cpp:211-222 */
    double inverse_scale;        /* inverseScale            simulationmanager.cpp:224-230 */
    double angle_scale;          /* inverseScaleAngle (mrad/px) simulationmanager.cpp:241-247 */
    double wavelength, wavenumber; /* commonstructs.h:269-275 */
    double sigma;                /* Sigma()*k/kz as passed to the potential kernels (simulationgeneral.cpp:418) */
    double wavevector[3];        /* commonstructs.h:282-289 */
    double k_max;                /* bandwidth k_max (simulationgeneral.cpp:451-455) */
    double dz;                   /* slice thickness */
    int n_slices;                /* SimulationCell::sliceCount  simulationcell.cpp:75-83 */
    int pre_slices;              /* SimulationCell::preSliceCount simulationcell.cpp:85-87 */
    int blocks_x, blocks_y;      /* calculateBlocks         simulationmanager.cpp:393-408 */
    int load_blocks_x, load_blocks_y, load_blocks_z; /* simulationgeneral.cpp:517-521 */
    double block_scale_x, block_scale_y;              /* simulationmanager.cpp:371-381 */
    unsigned int crop[4];        /* imageCrop t, l, b, r    simulationmanager.cpp:410-428 */
    int n_outputs;               /* output slices per run (intermediate output + exit) */
} mslice_geometry;

typedef void (*mslice_progress_cb)(double slice_fraction, void *user);

/* ---- library / context ---------------------------------------------------------------------- */
const char *mslice_version(void);
const char *mslice_last_error(void);

/* Create / destroy a device context. Replaces clContext + queue creation
 * (src/simulation/clwrapper/clcontext.h:28-114). */
int mslice_ctx_create(int device, mslice_ctx **out);
int mslice_ctx_destroy(mslice_ctx *ctx);
/* Optional cap on device bytes the ctx may allocate (0 = none); exceeding it gives MSLICE_ERR_OOM. */
int mslice_ctx_set_memory_limit(mslice_ctx *ctx, size_t bytes);

/* Load a parameterisation table (Utils::readParams, src/simulation/utilities/stringutils.cpp:149-184;
 * Parameterisation, structure/structureparameters.h:22-37). n must be a multiple of
 * i_per_atom * (4 for Kirkland, 2 for Peng/Lobato). Uploaded as ClParameterisation
 * (src/simulation/microscope/simulationgeneral.cpp:375-378). */
int mslice_params_load(mslice_ctx *ctx, int form, int i_per_atom, const double *p, size_t n);

/* Host-only geometry of a config (no device needed). Validates like
 * checkSimulationPrerequisites (src/simulation/utilities/simutils.cpp:8-89) for the fields it reads. */
int mslice_geometry_compute(const mslice_config *cfg, mslice_geometry *out);

/* ---- simulation object (SimulationWorker / SimulationGeneral state) ------------------------- */
int mslice_sim_create(mslice_ctx *ctx, const mslice_config *cfg, mslice_sim **out);
int mslice_sim_destroy(mslice_sim *sim);
int mslice_sim_geometry(mslice_sim *sim, mslice_geometry *out);
int mslice_set_progress(mslice_sim *sim, mslice_progress_cb cb, void *user);
/* Thread-safe; the running call returns MSLICE_ERR_CANCELLED at its next slice boundary
 * (the reference polls pool.isStopped() once per slice, simulationstem.cpp:234,253). */
int mslice_cancel(mslice_sim *sim);

/* Set ONE atom configuration (already displaced by the caller for frozen phonons). Replaces
 * SimulationGeneral::sortAtoms (simulationgeneral.cpp:147-342): the strict host range filter on the
 * padded full limits (:206-210), the atom_sort kernel (kernels/atom_sort_d.cl:28-69) and the
 * z-major / y / x stable binning into block_start_pos (:270-338), all on the device. */
int mslice_set_atoms(mslice_sim *sim, const int *Z, const double *x, const double *y, const double *z, size_t n);
/* Read back the binned atoms and block_start_pos of the current configuration.
 * n_out receives the number of atoms kept by the range filter; block_start must hold
 * n_slices*blocks_x*blocks_y + 1 ints. block_ids/z_ids (optional, may be NULL) receive the
 * atom_sort ids of the FILTERED list in filter order (-1,-1 for atoms outside the xy range). */
int mslice_get_sorted_atoms(mslice_sim *sim, int *Z, double *x, double *y, double *z, size_t cap,
                            int *block_start, size_t cap_block_start, int *block_ids, int *z_ids, size_t *n_out);

/* Build the band-limited transmission function of every slice for the current configuration
 * (precalc loop, simulationgeneral.cpp:576-613: potential kernel -> FFT -> band_limit -> IFFT). */
int mslice_build_transmission(mslice_sim *sim);
/* Read back slice `slice` of the transmission function (2*res*res doubles). band_limited = 0 returns
 * the potential kernel's raw output before the FFT band limit. */
int mslice_get_transmission(mslice_sim *sim, int slice, int band_limited, double *out);
/* The propagator P(k) (kernels/propagator_d.cl:18-52) as the engine applies it (2*res*res doubles). */
int mslice_get_propagator(mslice_sim *sim, double *out);
/* The reciprocal-space probe of init_probe_wave (kernels/init_probe_wave_d.cl:49-118) at position
 * (x, y) in Å in the same frame as the STEM/CBED areas (2*res*res doubles). */
int mslice_get_probe(mslice_sim *sim, double x, double y, double *out);

/* ---- mode drivers for the current configuration (one job) ----------------------------------- */
/* STEM (SimulationStem::simulate, simulationstem.cpp:143-278): propagate the given scan pixels
 * (index p -> x_i = p % px, y_i = p / px) through all slices and write the detector values
 * out[(o * n_detectors + d) * n_pixels + i] for output slice o, detector d, pixel i. */
int mslice_stem_run(mslice_sim *sim, const int *pixels, size_t n_pixels, double *out);
/* CBED (simulationcbed.cpp:122-210): out[o * res*res + k] = |fftshift(psi(k))|^2. */
int mslice_cbed_run(mslice_sim *sim, double *diff);
/* CTEM (simulationctem.cpp:285-400): exit wave (interleaved, cropped by imageCrop: n_outputs *
 * 2*cw*ch), diffraction (n_outputs*res*res) and, if cfg.ctem_image, image (n_outputs*cw*ch).
 * Any output pointer may be NULL. */
int mslice_ctem_run(mslice_sim *sim, double *ew, double *diff, double *image);

/* ---- differentiable CTEM (image loss and its gradients) ------------------------------------------- */
/* Loss L = sum over pixels of (I - target)^2 for the CTEM objective-lens image I of the current atom
 * configuration (simulateImagePerfect, microscope/simulationctem.cpp:114-166), and its gradients by the
 * hand-written adjoint of the multislice: dL/d(x, y, z) of every atom passed to mslice_set_atoms (input
 * order, 3 per atom; z is 0 in the projected model, where z only selects the slice, and a true derivative
 * under the full 3-D model), dL/dC10 and dL/dC30 (per Å). target holds res*res doubles (x fastest). Slice
 * waves are checkpointed every `checkpoint_every` slices (0: ceil(sqrt(n_slices)); 1: every slice, no
 * recomputation) and recomputed segment by segment in the backward pass. Projected (with or without beam
 * tilt) and full 3-D potentials; mixed static potentials and plasmons fail with MSLICE_ERR_UNSUPPORTED. The
 * full 3-D gradients gather with FP64 atomics, so they are reproducible to FP64 rounding rather than bit for
 * bit; they are the derivative within the current binning (the full 3-D loss jumps where an atom crosses a bin
 * edge, which reorders the trapezoid's samples). Any output pointer may be NULL. The same as mslice_ctem_loss_forward followed by
 * mslice_ctem_loss_backward. */
int mslice_ctem_loss_grad(mslice_sim *sim, const double *target, double *loss, double *grad_xyz, double *grad_c10,
                          double *grad_c30, int checkpoint_every);
/* The two halves of mslice_ctem_loss_grad, for autograd frameworks that run the backward pass later: the
 * forward computes the loss and keeps the checkpoints and state the adjoint needs, returning a token; the
 * backward turns that state into the gradients. Any other call on the simulation in between (a run, new
 * atoms or lens, another forward) invalidates the state and the backward fails with MSLICE_ERR_STATE. */
int mslice_ctem_loss_forward(mslice_sim *sim, const double *target, double *loss, int checkpoint_every,
                             unsigned long long *token);
int mslice_ctem_loss_backward(mslice_sim *sim, unsigned long long token, double *grad_xyz, double *grad_c10,
                              double *grad_c30);
/* The same loss without gradients (forward only); used to time the forward model. */
int mslice_ctem_loss(mslice_sim *sim, const double *target, double *loss);
/* CTEM dose simulation (SimulationCtem::simulateImageDose, microscope/simulationctem.cpp:88-108,171-264):
 * with a CCD set, the CTEM image of mslice_ctem_run is filtered by the detective quantum efficiency, given
 * Poisson noise for `dose` electrons per Å^2 (times realScale^2 per pixel and binning^2 per binned pixel) and
 * filtered by the noise transfer function. dqe / ntf: the 725-value radial tables of a clTEM ccds .dat file.
 * n = 0 clears the CCD (the perfect image). The noise is drawn from cfg.seed; the k-th dosed image after
 * this call uses pass k (the reference draws from a clock-seeded std::mt19937_64). */
int mslice_set_ccd(mslice_sim *sim, const double *dqe, const double *ntf, size_t n, int binning, double dose);
/* Change the defocus C10 and spherical aberration C30 (Å) of an existing simulation (the objective lens
 * of the CTEM image and the probe of STEM/CBED both follow). */
int mslice_set_c10_c30(mslice_sim *sim, double c10, double c30);

/* ---- frozen-phonon jobs over many configurations, one persistent call ---------------------- */
/* Stage n_configs atom configurations on the device (concatenated host arrays, counts[c] atoms each).
 * A staged set stays resident until the next stage call or mslice_sim_destroy. */
int mslice_stage_configs(mslice_sim *sim, int n_configs, const size_t *counts, const int *Z,
                         const double *x, const double *y, const double *z);
/* Run every staged configuration and every STEM scan pixel (all px*py in scan order), accumulating
 * the detector values over configurations in FP64 with Kahan compensation on the device. With the static
 * frame, one transmission set, no plasmons and no progress callback, the whole run (every pass's binning,
 * transmission build and probe batches) is captured once into a CUDA graph and each run of the same staged
 * layout is a single graph launch (MSLICE_NO_GRAPHS=1 launches eagerly); mslice_last_timing then reports
 * the whole run only (build and propagation -1). */
int mslice_stem_run_staged(mslice_sim *sim);
/* The same run, returning once it is queued (no counterpart in the reference): with the single-launch path
 * above the call enqueues the graph on the context's stream and returns, so runs on different contexts
 * (streams) overlap; otherwise it runs synchronously. mslice_sim_wait waits for it (and reports a failed
 * wait of the step kernels); mslice_staged_result and the next run wait as well. */
int mslice_stem_run_staged_async(mslice_sim *sim);
int mslice_sim_wait(mslice_sim *sim);
/* Same for CBED: accumulates |psi(k)|^2 over configurations. */
int mslice_cbed_run_staged(mslice_sim *sim);
/* Averaged result of the last *_run_staged call: STEM out[(o*n_det + d)*px*py + p], CBED
 * out[o*res*res + k], each divided by the number of configurations (Image::getWeightedSlice,
 * src/simulation/utilities/commonstructs.h:149-158). */
int mslice_staged_result(mslice_sim *sim, double *out, size_t cap);
/* One call from host buffers to host result: stage + run + result (the end-to-end API). */
int mslice_stem_simulate(mslice_sim *sim, int n_configs, const size_t *counts, const int *Z,
                         const double *x, const double *y, const double *z, double *out, size_t cap);

/* The random draws a run makes, host only (no device needed). The reference draws from clock-seeded
 * std::mt19937_64 engines; these are pure functions of (cfg.seed, pass, pixel, slice), so runs repeat
 * exactly. For pass `pass` and scan pixels[i]: defocus[i] = the chromatic defocus change in Å (0 when
 * chromatic is off), sets[i * n_slices + s] = the transmission set taken at slice s (0 unless
 * mixed_static > 1); shift[2*b], shift[2*b+1] = the source-size frame shift in Å of transmission build
 * b (builds are numbered per run: pass p in the static frame, p * n_jobs + j for job j in the moving
 * frame; 0 for the mixed static sets). Any output pointer may be NULL; shift receives n_builds pairs. */
int mslice_incoherence_draws(const mslice_config *cfg, int pass, const int *pixels, size_t n_pixels, double *defocus,
                             int *sets, int n_slices, int n_builds, double *shift);
/* The seeded plasmon draws of job `job` (host only; replaces the clock-seeded stream of PlasmonScattering,
 * src/simulation/incoherence/inelastic/plasmon.cpp): the scattering depths (Å) of generateScatteringDepths for a
 * crystal `thickness` Å thick, closed by +inf (n_depths entries into depths[cap]; MSLICE_ERR_ARG where the
 * reference could not make a valid table), and the (polar mrad, azimuth rad) pairs of events 0..n_events-1 into
 * angles[2 * n_events]. Jobs are numbered as the runs number them: the pass for CTEM / CBED, pass * n_jobs + j
 * for STEM job j of stem_job_pixels consecutive pixels. Any output may be NULL. */
int mslice_plasmon_draws(const mslice_config *cfg, unsigned long long job, double thickness, double *depths, size_t cap,
                         size_t *n_depths, int n_events, double *angles);

/* Autotuner of the probe batch and of the step kernels (no counterpart in the reference, which propagates
 * `parallel pixels` probes one at a time): times `reps` slice steps (one fused row and one fused column pass)
 * for each candidate batch size and each column-pass variant, then each row-pass variant at the best pair (see
 * mslice_set_step_variant), on zeroed scratch waves, and makes the fastest the simulation's default (the batch
 * is used when cfg.probe_batch is 0). candidates = NULL tries 64..2048 and reuses a result
 * cached for this device, grid and precision in the process. Candidates whose waves would take more than
 * a quarter of the free device memory are skipped. best_batch / waves_per_second may be NULL. */
int mslice_tune_batch(mslice_sim *sim, const int *candidates, int n_candidates, int reps, int *best_batch,
                      double *waves_per_second);
/* The kernels of the batched STEM step (no counterpart in the reference). Column step: 0 = one block per
 * column tile and wave at the default tile width; the further variants of the grid and precision (FP32) are
 * the persistent passes, one or two blocks per SM, that stream tiles into a ring of shared-memory stages with
 * TMA (where their shared memory fits; among them the passes with one barrier domain per
 * column pair at 256^2 to 3072^2), and the one-block-per-tile kernel at other tile widths and register budgets
 * (mslice_step_variant_name describes each). Row step: 0 = plain; 1, 2 = each block also asks the copy engine
 * to prefetch into L2 the rows that the blocks one or two residencies of the grid later will read; 3 = the
 * grid in wave-fastest order, so blocks issued together read the same transmission rows; where the grid's
 * default row plan is a wide one (FP32 256^2 to 8192^2 and the 3*2^k grids), 4-7 = the same four with the plain
 * Stockham plan in the two-row step, and 8-11 = the same four as 0-3 with each block's transmission rows staged
 * into shared memory by the copy engine as the block starts. All variants give bit-identical results except
 * row variants 4-7, a different FFT plan, which agree with the others to FP32 rounding. Until it is tuned or set, a batched STEM
 * run uses the grid's default column kernel (FP32 256^2 to 3072^2: the per-pair-barrier pass; otherwise 0) and
 * row variant 0; mslice_get_tuning reports them. Out-of-range values fail with MSLICE_ERR_ARG. */
int mslice_set_step_variant(mslice_sim *sim, int col_variant, int row_variant);
/* A description of step-kernel variant `index` (which: 0 column, 1 row) of this simulation's grid and
 * precision into buf (NUL-terminated, at most cap bytes). */
int mslice_step_variant_name(mslice_sim *sim, int which, int index, char *buf, size_t cap);
/* The batch the next STEM run uses, the column- and row-step variants and their counts for this grid and
 * precision (any pointer may be NULL). */
int mslice_get_tuning(mslice_sim *sim, int *batch, int *col_variant, int *n_col_variants, int *row_variant,
                      int *n_row_variants);

/* ---- comparison paths and building blocks ---------------------------------------------------- */
/* Plain per-probe STEM in the reference's unfused kernel order (simulationgeneral.cpp:736-768):
 * complex multiply, cuFFT Z2Z/C2C forward, complex multiply with P, inverse, one probe at a time,
 * device sync per probe and slice. Same output layout as mslice_stem_run. */
int mslice_stem_run_plain(mslice_sim *sim, const int *pixels, size_t n_pixels, double *out);
/* Unitary 2-D DFT of `batch` n×n complex arrays with the engine's own shared-memory FFT kernels
 * (clFourier semantics: out-of-place, scale 1/sqrt(n*n) both directions, clfourier.cpp:70-73). */
int mslice_fft2(mslice_ctx *ctx, int n, int inverse, int double_precision, int batch,
                const double *in, double *out);

/* Device-stream timing hooks for benchmarks: the CUDA stream every kernel of this ctx runs on
 * (returned as an opaque cudaStream_t value) and the number of kernels the ctx has launched. */
int mslice_ctx_stream(mslice_ctx *ctx, void **stream);
int mslice_ctx_launch_count(mslice_ctx *ctx, unsigned long long *count);
/* Device time (ms, CUDA events on the ctx stream) of the last mslice_stem_run_staged call split into
 * [transmission build, propagation passes, total]. */
int mslice_last_timing(mslice_sim *sim, double *ms3);

/* Per-kernel device timing: when enabled, every launch of the kinds below is bracketed by CUDA events
 * on the ctx stream and its duration accumulated (adds two event records per launch). */
#define MSLICE_K_ROW_STEP 0   /* fused row pass of the multislice step        */
#define MSLICE_K_COL_STEP 1   /* fused column pass of the multislice step     */
#define MSLICE_K_POTENTIAL 2  /* slice potential / transmission kernel        */
#define MSLICE_K_BANDLIMIT 3  /* the three passes of the transmission band limit */
#define MSLICE_K_PROBE 4      /* probe generation + column inverse FFT        */
#define MSLICE_K_COUNT 5
int mslice_profile_enable(mslice_sim *sim, int on);
/* Accumulated device ms, launch count and algorithmic bytes (the bytes the launches must read and write
 * in HBM by design: waves, transmission slices, tables; columns outside the propagator cut are neither
 * read nor written) of one kernel kind since the last reset; reset != 0 clears every kind. */
int mslice_profile_read(mslice_sim *sim, int kernel, double *total_ms, unsigned long long *launches, double *bytes,
                        int reset);

/* Atom binning without any device allocation (no counterpart in the reference).
 * For callers that cannot call cudaMalloc: a host application that manages all device memory through its
 * own pool, or a pipeline stage that must not take cudaMalloc/cudaFree's latency and implicit device
 * synchronisation. Bins n atoms exactly like mslice_set_atoms (same order, same block_start) for the
 * geometry `geo` (from mslice_geometry_compute), reading Z/x/y/z and writing block_start
 * (n_slices*blocks_x*blocks_y + 1 ints) and the four sorted arrays (n each) — all DEVICE pointers owned by
 * the caller — on `stream` (a cudaStream_t, NULL for the default stream); it returns once the work is
 * queued. Its working memory is one fixed 8 MiB device array inside the library, held on every device that
 * loads the library until the process exits; the limits are 131072 atoms and 65535 bins, and larger
 * requests fail with MSLICE_ERR_ARG, as does a geometry whose limits are empty or whose n_slices does not
 * cover z_lims at thickness dz. Every call looks the array's device address up (cudaGetSymbolAddress, so no
 * address outlives a device reset); the first call on a device also loads the library's device code there,
 * so make that first call before any stream capture. Every call reuses the same array: calls whose work
 * overlaps on the GPU (two streams, two host threads) race on it, so serialise them. */
int mslice_bin_atoms_noalloc(const mslice_geometry *geo, const int *Z, const double *x, const double *y, const double *z,
                             size_t n, int *block_start, int *Z_sorted, double *x_sorted, double *y_sorted,
                             double *z_sorted, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MSLICE_H */
