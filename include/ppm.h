/*
 * ppm.h — C ABI of the B200 pulse-profile engine (libppm_b200.so).
 *
 * The engine computes phase-resolved X-ray pulse profiles of hot spots on a
 * rotating oblate neutron star: HEALPix surface tiling, Schwarzschild lensing
 * lookups, Doppler/aberration, time-of-flight phase shifts, NSX-atmosphere or
 * blackbody intensity, Gauss-Legendre phase-bin integration, and the
 * energy-to-channel response fold.
 *
 * Every entry point below replaces one interface of fizban007/gpu_ppm; the
 * reference file:line is cited beside each declaration.  All pointers are
 * plain host pointers unless the name ends in `_device`.  Every call returns a
 * status code (PPM_OK on success); the reference's `exit(EXIT_FAILURE)` error
 * paths (gpu/error.cuh:5-26, gpu/read_file.cuh:11-15, cpu/nsx.hpp:91-93) become
 * non-zero codes with a message retrievable by ppm_last_error_string().
 * Out-of-range table lookups are clamped exactly like the reference CPU path
 * (cpu/hunt.hpp:99-116) and counted in ppm_result_info instead of printed.
 */
#ifndef PPM_H
#define PPM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PPM_OK 0
#define PPM_E_INVALID 1 /* bad argument / inconsistent parameters */
#define PPM_E_IO 2      /* file missing or malformed */
#define PPM_E_RANGE 3   /* size or value beyond what a table / the engine supports */
#define PPM_E_OOM 4     /* device or host allocation failed, or memory budget exceeded */
#define PPM_E_TIMEOUT 5 /* a bounded wait ran out */
#define PPM_E_CUDA 6    /* CUDA runtime error */
#define PPM_E_STATE 7   /* call out of order (e.g. tables not loaded) */

/* ---- enums ------------------------------------------------------------- */
/* spot kinds */
#define PPM_SPOT_HEALPIX 0 /* disk1 \ disk2 on a HEALPix grid: disk, ring, crescent, difference of disks
                              (cpu/grid.hpp:175-190 DiskDifference, gpu/devarshi24st_gpu.cu:117-134) */
#define PPM_SPOT_POINT 1   /* single element of a cap's solid angle (cpu/grid.hpp:18-27 PointSource) */

/* atmospheres */
#define PPM_ATM_NSX 0       /* NSX table, interpolated (cpu/nsx.hpp:173-321) */
#define PPM_ATM_BLACKBODY 1 /* Planck intensity Ibb (cpu/unit.hpp:28-31) */

/* NSX interpolators (cpu/nsx.hpp; cpu/t_interp.cpp:420-428 interp_type) */
#define PPM_INTERP_4C 0      /* cubic in all 4 axes, Interp_IT3_4c(use_sg=false) */
#define PPM_INTERP_4C_SG 1   /* as 4C, negative results set to 0, Interp_IT3_4c(use_sg=true) */
#define PPM_INTERP_4C_LE 2   /* cubic, linear in mu near the mu edge, Interp_IT3_4c_le */
#define PPM_INTERP_2L2C_LE 3 /* linear logT/logg, cubic E/mu, linear mu edge, Interp_IT3_2l2c_le */
#define PPM_INTERP_4L 4      /* linear in all 4 axes, Interp_IT3_4l */

/* blackbody beaming (cpu/os1_cpu.cpp:128-136) */
#define PPM_BEAM_ISO 0  /* 'i' */
#define PPM_BEAM_SIN2 1 /* 's': 1 - mu'^2 */
#define PPM_BEAM_COS2 2 /* 'c': mu'^2 */

/* integrand arithmetic */
#define PPM_PREC_FP32 0 /* FP32 integrand, FP64 phase/ToF and accumulation */
#define PPM_PREC_FP64 1 /* FP64 everywhere (blackbody only) */

/* response fold arithmetic */
#define PPM_FOLD_BF16X3 0 /* tcgen05 tensor cores, BF16 hi/lo split, 3 products, FP32 accumulate */
#define PPM_FOLD_FP32 1   /* FP32 SIMT */
#define PPM_FOLD_FP64 2   /* FP64 SIMT */

/* ---- tables -------------------------------------------------------------- */

/* Lensing tables on uniform grids, as written by c_lensing.py:35-44,109-110,155
 * and read by cpu/lensing.hpp:33-41 / gpu/lensing.cuh:27-54. */
typedef struct ppm_lensing_desc {
  double u_min, u_max;
  int32_t n_u;
  double cos_psi_min, cos_psi_max;
  int32_t n_cos_psi;
  double cos_alpha_min, cos_alpha_max;
  int32_t n_cos_alpha;
  const double* cos_alpha_of_u_cos_psi;    /* [n_u][n_cos_psi] */
  const double* lf_of_u_cos_psi;           /* [n_u][n_cos_psi] */
  const double* cdt_over_R_of_u_cos_alpha; /* [n_u][n_cos_alpha] */
} ppm_lensing_desc;

/* Grid for generating lensing tables (c_lensing.py:8-32). */
typedef struct ppm_lensing_spec {
  double u_min, u_max;
  int32_t n_u;
  double cos_psi_min, cos_psi_max;
  int32_t n_cos_psi;
  double cos_alpha_min, cos_alpha_max;
  int32_t n_cos_alpha;
  int32_t n_threads; /* host threads; <=0 means all cores */
} ppm_lensing_spec;

/* NSX atmosphere grid (cpu/nsx.hpp:11-51 NsxConfig; file layout cpu/nsx.hpp:98-134).
 * log_I_T3 holds column 3 of the NSX file (log10 of I/T^3), loop order
 * logT -> logg -> logEkT -> mu.  logT/logg/logEkT are uniform axes; mu is the
 * file's (strictly descending) mu column. */
typedef struct ppm_nsx_desc {
  int32_t n_logT, n_logg, n_logEkT, n_mu;
  double logT_min, logT_max;
  double logg_min, logg_max;
  double logEkT_min, logEkT_max;
  const double* mu;       /* [n_mu] */
  const double* log_I_T3; /* [n_logT][n_logg][n_logEkT][n_mu] */
} ppm_nsx_desc;

/* ---- per-profile parameters ---------------------------------------------- */

/* One emitting region: disk1 minus disk2 (angles in radians).  A plain disk has
 * angrad2 = 0; a ring has equal centres; a crescent has offset centres.
 * Replaces StarData (cpu/devarshi24st_cpu.cpp:12-15, gpu/devarshi24st_gpu.cu:79-87). */
typedef struct ppm_spot {
  double theta1, phi1, angrad1;
  double theta2, phi2, angrad2;
  double logT;   /* NSX: log10(T / K) (cpu/devarshi24st_cpu.cpp:57) */
  double kT_keV; /* blackbody: kT in keV (cpu/os1_cpu.cpp:32) */
  int32_t kind;  /* PPM_SPOT_* */
  int32_t reserved;
} ppm_spot;

/* Everything one profile depends on.  The reference hard-codes these as
 * constexpr (gpu/devarshi24st_gpu.cu:20-44, cpu/devarshi24st_cpu.cpp:48-59). */
typedef struct ppm_params {
  double mass_msun;       /* M */
  double r_eq_km;         /* equatorial radius Re */
  double spin_hz;         /* nu */
  double inclination_rad; /* observer colatitude (obs_theta / inc) */
  double distance_kpc;    /* D = distance_kpc * kpc_in_km */
  double exposure_s;      /* exposure_time (fold scale only) */
  ppm_spot spots[2];
  int32_t n_spots;      /* 1 or 2; contributions add */
  int32_t atmosphere;   /* PPM_ATM_* */
  int32_t interp;       /* PPM_INTERP_* (NSX) */
  int32_t beaming;      /* PPM_BEAM_* (blackbody) */
  int32_t n_side;       /* HEALPix N_side (any positive integer) */
  int32_t n_bins;       /* output phase bins */
  int32_t n_gl;         /* Gauss-Legendre points per bin, 1..6; 0 = sample at phases k/n_bins */
  int32_t n_fine;       /* fine phase samples per rotation (reference: 6*n_bins) */
  int32_t energy_grid;  /* id from ppm_engine_add_energy_grid */
  int32_t response;     /* id from ppm_engine_add_response, or -1 for flux only */
  int32_t precision;    /* PPM_PREC_* */
  int32_t fold;         /* PPM_FOLD_* */
} ppm_params;

/* Diagnostics per profile (the reference prints these, cpu/hunt.hpp:16-18,104,111). */
typedef struct ppm_result_info {
  int64_t n_active;        /* active surface elements (all spots) */
  int64_t n_rings;         /* rings with at least one active element */
  int64_t n_dropped_rings; /* rings skipped because the first/last fine sample is invisible */
  int64_t n_points;        /* visible (element, phase node) pairs that were integrated */
  int64_t n_clamped;       /* lookups clamped to a table edge (u per ring, logEkT per point) */
  int64_t n_active_integrated; /* active elements on rings that were integrated (not dropped) */
  int32_t status;
  int32_t reserved;
} ppm_result_info;

typedef struct ppm_engine ppm_engine;

typedef struct ppm_engine_config {
  int32_t device;             /* CUDA device ordinal */
  int32_t max_batch;          /* largest batch ppm_profile_batch accepts (profiles) */
  int64_t memory_budget;      /* bytes of device memory for in-flight request state (0 = 64 GiB); also
                                 the most device memory the engine keeps cached between synchronous calls */
  int32_t autotune;           /* 1: time candidate launch shapes at first use */
  int32_t n_streams;          /* serving: concurrent batches in flight (0 = 3: batches overlap on the GPU
                                 while the next is staged); the server also pins n_streams + 4 staging
                                 buffers of 32 MiB and, per stream, a small upload area for the batch
                                 build's host-to-device copies when it starts (first ppm_submit) */
} ppm_engine_config;

/* ---- engine ---------------------------------------------------------------- */

/* Creates an engine on one device.  Replaces the table constructors plus the
 * per-call cudaMalloc of gpu/devarshi24st_gpu.cu:442-450; all device memory is
 * owned by the engine (gpu/lensing.cuh:56-61, gpu/nsx.cuh:130-134 free_gpu_memory). */
int ppm_engine_create(const ppm_engine_config* cfg, ppm_engine** out);
void ppm_engine_destroy(ppm_engine* e);

/* Lensing tables (replaces Lens(setting) gpu/lensing.cuh:27-54, Lensing(setting) cpu/lensing.hpp:33). */
int ppm_engine_load_lensing(ppm_engine* e, const ppm_lensing_desc* lens);
/* Reads tables/lensing/<setting>/{u,cos_psi,cos_alpha,...}.txt from `dir` (the <setting> folder). */
int ppm_engine_load_lensing_dir(ppm_engine* e, const char* dir);

/* NSX table (replaces NSX() gpu/nsx.cuh:83-128, cpu/nsx.hpp:83-148). */
int ppm_engine_load_nsx(ppm_engine* e, const ppm_nsx_desc* nsx);
/* Reads a 5-column NSX text file with the given axis description (desc->mu and
 * desc->log_I_T3 are ignored).  Axis values are checked as in cpu/nsx.hpp:110-147. */
int ppm_engine_load_nsx_file(ppm_engine* e, const char* path, const ppm_nsx_desc* axes);

/* Observed-energy grid in keV (replaces IsmInst::E_obs, gpu/ism_inst.cuh:18-32). */
int ppm_engine_add_energy_grid(ppm_engine* e, int32_t n_e, const double* e_keV, int32_t* grid_id);
/* Response matrix rsp[n_ch][n_e] on an energy grid (replaces IsmInst::rsp). */
int ppm_engine_add_response(ppm_engine* e, int32_t grid_id, int32_t n_ch, const double* rsp, int32_t* rsp_id);
/* Reads tables/ism_inst/<setting>/{num,E_obs,rsp}.txt (cpu/ism_inst.hpp:65-69) and registers both. */
int ppm_engine_load_ism_inst_dir(ppm_engine* e, const char* dir, int32_t* grid_id, int32_t* rsp_id);

/* ---- profiles ---------------------------------------------------------------- */

/* Plain form: one profile, one pass of the kernels, synchronous.
 * Replaces calc_one_star (gpu/devarshi24st_gpu.cu:432-511, gpu/os1_gpu.cu:304-349):
 * KernelFunc + cublasSgemm fold + D2H.
 * flux:   [n_bins][n_e]   photon flux per (phase bin, energy), the reference
 *         CPU's total_flux(i_phase_bin, i_E) (cpu/devarshi24st_cpu.cpp:238); may be NULL.
 * counts: [n_ch][n_bins]  exposure * (1/n_bins) * sum_E rsp[ch][E] flux[bin][E]
 *         (cpu/devarshi24st_cpu.cpp:249-258); may be NULL; needs a response. */
int ppm_profile(ppm_engine* e, const ppm_params* p, double* flux, double* counts, ppm_result_info* info);

/* Batched form: n independent profiles in one graph-captured persistent launch
 * that pulls (profile, spot, ring-chunk) tiles from a device work queue.
 * flux / counts are concatenations of each profile's arrays in order; either may be NULL. */
int ppm_profile_batch(ppm_engine* e, int32_t n, const ppm_params* p, double* flux, double* counts,
                      ppm_result_info* info);

/* Device-resident batches.  ppm_batch_create converts and uploads n profiles,
 * allocates their device output pools and captures one pass of the kernels
 * (plan -> integrand -> fold) in a CUDA graph; ppm_batch_launch replays it on
 * `stream` (a cudaStream_t, NULL = the engine stream) without host
 * synchronisation; outputs stay in device memory until collected. */
typedef struct ppm_batch ppm_batch;
int ppm_batch_create(ppm_engine* e, int32_t n, const ppm_params* p, ppm_batch** out);
int ppm_batch_launch(ppm_engine* e, ppm_batch* b, void* stream);
/* Device pointers and sizes (doubles) of the batch's flux and counts pools. */
int ppm_batch_device_outputs(ppm_batch* b, double** flux, int64_t* n_flux, double** counts, int64_t* n_counts);
/* Ring-window forms, for splitting one large profile over several GPUs: only
 * HEALPix rings i with ring_begin <= i < ring_end contribute (rings are
 * 1 .. 4 N_side - 1; a point-source spot counts as ring 0).  The flux and the
 * counts are linear in the rings, so the sum of the outputs over a partition of
 * [0, 4 N_side) is the full profile (one reduce of the counts finishes it).
 * The reference integrates all rings of a star in one call
 * (gpu/devarshi24st_gpu.cu:181-427, cpu/devarshi24st_cpu.cpp:86-241). */
int ppm_batch_create_rings(ppm_engine* e, int32_t n, const ppm_params* p, int32_t ring_begin, int32_t ring_end,
                           ppm_batch** out);
int ppm_profile_rings(ppm_engine* e, const ppm_params* p, int32_t ring_begin, int32_t ring_end, double* flux,
                      double* counts, ppm_result_info* info);
/* Waits for the last launch and copies the outputs to host memory (either may be NULL). */
int ppm_batch_collect(ppm_engine* e, ppm_batch* b, double* flux, double* counts, ppm_result_info* info);
void ppm_batch_destroy(ppm_engine* e, ppm_batch* b);
/* Profiling form of ppm_batch_launch: the same pass launched kernel by kernel
 * with CUDA events between the phases; waits and returns the device time in
 * milliseconds of ms[0] = clear + plan, ms[1] = integrand, ms[2] = fold. */
int ppm_batch_launch_timed(ppm_engine* e, ppm_batch* b, void* stream, float* ms);
/* Number of engine kernels one pass of the batch launches. */
int ppm_batch_kernel_count(ppm_engine* e, ppm_batch* b, int32_t* n);

/* Allocation-free plain form, for callers that may not allocate device memory
 * while they run (a sampler that reserved the whole GPU for its own pool at
 * start-up, a framework whose caching allocator owns the device, or a loop
 * where cudaMalloc's implicit device synchronisation would stall other
 * streams).  No counterpart in the reference: it has no allocation-free path.
 * Enqueues one profile on `stream` (a cudaStream_t, NULL = engine stream)
 * without waiting for it to finish (its few small uploads come from pageable
 * host memory, so CUDA may first wait for earlier work on that stream);
 * flux_device [n_bins][n_e] (required) and counts_device [n_ch][n_bins]
 * (optional) are caller-owned device buffers.  A stream that is being
 * captured is refused with PPM_E_STATE: the uploads' host memory is released
 * when the call returns.
 * All other working state lives in one 1 MiB device array that the library
 * declares statically (held on every device that loads the library until
 * process exit); profiles whose tables and work queue do not fit — about
 * N_side > 512 with two spots — are rejected with PPM_E_RANGE.  The first call
 * on a device looks up the array's address; make it before any stream capture.
 * Calls share the array, so calls that overlap on the GPU race. */
int ppm_profile_noalloc(ppm_engine* e, const ppm_params* p, double* flux_device, double* counts_device, void* stream);
/* Outcome of the last ppm_profile_noalloc call: waits for `stream` (NULL =
 * engine stream), fills info (active elements, rings, phase points, clamped
 * lookups) from the counters in the static array, and returns PPM_E_TIMEOUT if
 * a bounded wait of its tensor-core fold ran out, PPM_E_RANGE if its work
 * queue overflowed, else PPM_OK.  Allocates nothing.  The status belongs to
 * that call alone: other calls of the engine neither see nor clear it. */
int ppm_profile_noalloc_result(ppm_engine* e, void* stream, ppm_result_info* info);

/* Autotuner: times candidate launch shapes of the integrand — candidate
 * elements per work tile (ring granularity), CTAs per SM the register budget
 * targets, the NSX kernel (home-cell or pooled-polynomial) with its energy
 * cells per lane and warp sets per CTA, or phase points per polynomial
 * sub-batch and energies per thread — on the given sample profiles by
 * coordinate descent with CUDA events, keeps the fastest for every later
 * launch, and writes a one-line-per-candidate report (truncated to
 * report_len; report may be NULL).  No counterpart in the reference, whose
 * launch shape is fixed (one CTA per ring, gpu/devarshi24st_gpu.cu:460-463). */
int ppm_engine_autotune(ppm_engine* e, int32_t n, const ppm_params* sample, char* report, int32_t report_len);

/* ---- fit statistics (sampler likelihood) ------------------------------------ */

/* Goodness of fit of one profile's counts m[ch][bin] against observed counts
 * d[ch][bin] of the same response and bin count, computed on the device right
 * after the fold so that a sampler receives scalars instead of count arrays.
 *   chi2    = cal_chi2 of p_devarshi24st.py:43-49: both arrays scaled by
 *             fac = 1e6 / sum(m), chi2 = sum (fac d - fac m)^2 / (fac m);
 *             entries with m <= 0 are left out (numpy gives inf/nan there)
 *   loglike = Poisson log-likelihood sum (d ln m - m - lgamma(d + 1)); an
 *             entry with m <= 0 adds -m when d == 0 and makes it -inf otherwise
 * FP64 throughout, summed in a fixed order (equal counts give bitwise equal
 * statistics). */
typedef struct ppm_fit {
  double chi2;
  double loglike;
  double model_total;   /* sum(m) */
  int64_t n_zero_model; /* entries with m <= 0 */
} ppm_fit;

/* Registers observed counts [n_ch][n_bins] (the counts layout, n_ch of the
 * response) and keeps them on the device; returns its id. */
int ppm_engine_add_observed(ppm_engine* e, int32_t response, int32_t n_bins, const double* counts, int32_t* observed_id);
/* Fit statistics of every profile of a batch after its last launch: enqueued
 * on `stream` (NULL = the stream of the last launch), waits, writes n entries.
 * Every profile must use the observed data's response and bin count. */
int ppm_batch_fit(ppm_engine* e, ppm_batch* b, int32_t observed_id, ppm_fit* out, void* stream);
/* Plain form: computes one profile and returns only its fit statistics. */
int ppm_profile_fit(ppm_engine* e, const ppm_params* p, int32_t observed_id, ppm_fit* out, ppm_result_info* info);

/* The response fold on its own, for flux computed elsewhere (replaces matmul,
 * gpu/matmul.cuh:12-36, which the reference calls after its kernel,
 * gpu/devarshi24st_gpu.cu:469-477):
 *   counts[j][ch][b] = alpha[j] * sum_E rsp[ch][E] flux[j][b][E]
 * for n_profiles arrays flux[j] of [n_bins][n_e] (n_e of the response's grid),
 * with the arithmetic `fold` (PPM_FOLD_*).  alpha is per profile (the plain
 * form uses exposure / n_bins).  ppm_fold takes host arrays and waits;
 * ppm_fold_device takes device arrays and enqueues on `stream` (NULL = engine
 * stream) without waiting. */
int ppm_fold(ppm_engine* e, int32_t response, int32_t fold, int32_t n_profiles, int32_t n_bins, const double* alpha,
             const double* flux, double* counts);
int ppm_fold_device(ppm_engine* e, int32_t response, int32_t fold, int32_t n_profiles, int32_t n_bins,
                    const double* alpha, const double* flux_device, double* counts_device, void* stream);

/* Sizes of the output arrays for a parameter set (doubles). */
int ppm_output_sizes(ppm_engine* e, const ppm_params* p, int64_t* n_flux, int64_t* n_counts);

/* ---- serving (continuous batching) ------------------------------------------- */

/* Queues a request; returns immediately with a ticket.  Requests that arrive
 * while others are on the device are admitted into the next batch as stream
 * slots and the memory budget free up; a batch takes at most one 32 MiB
 * staging buffer's worth of results.  flux / counts must stay valid until
 * the ticket completes.  Returns PPM_E_OOM if the request alone exceeds the budget. */
int ppm_submit(ppm_engine* e, const ppm_params* p, double* flux, double* counts, uint64_t* ticket);
/* done = 1 once the ticket finished (its status is then in info via ppm_wait). */
int ppm_poll(ppm_engine* e, uint64_t ticket, int32_t* done);
/* Waits at most timeout_ms (negative: no limit) for a ticket. */
int ppm_wait(ppm_engine* e, uint64_t ticket, int32_t timeout_ms, ppm_result_info* info);
/* Latency of a finished ticket, in microseconds: from the entry of ppm_submit
 * to the moment its results are in the caller's buffers (ppm_wait can return). */
int ppm_ticket_latency_us(ppm_engine* e, uint64_t ticket, double* latency_us);
/* Forgets a finished ticket (its status, info and latency); afterwards the
 * ticket is unknown.  A long-running client releases each ticket once it has
 * read it, so the engine's record of tickets stays bounded.  PPM_E_STATE if the
 * ticket has not finished. */
int ppm_ticket_release(ppm_engine* e, uint64_t ticket);

/* One served batch, times in microseconds since the server started (its first
 * ppm_submit). */
typedef struct ppm_serve_batch_trace {
  double t_admit;     /* requests taken from the queue */
  double t_launched;  /* built, uploaded and enqueued on its stream */
  double t_finished;  /* its results reached the pinned staging buffer */
  double t_published; /* results copied to the callers, tickets completed */
  int32_t n_requests;
  int32_t stream_slot;
  int64_t staging_bytes; /* pinned staging capacity the batch used */
} ppm_serve_batch_trace;

/* The most recent served batches (at most the last 4096), oldest first:
 * copies min(cap, available) records to out and their number to n_out. */
int ppm_serve_trace(ppm_engine* e, ppm_serve_batch_trace* out, int32_t cap, int32_t* n_out);

/* ---- tables & files ----------------------------------------------------------- */

/* Generates lensing tables with the Schwarzschild ray integrals of
 * c_lensing.py:47-155 (arrays sized as in ppm_lensing_desc). */
int ppm_lensing_generate(const ppm_lensing_spec* spec, double* cos_alpha_of_u_cos_psi, double* lf_of_u_cos_psi,
                         double* cdt_over_R_of_u_cos_alpha);

/* Instrument response on the integrand's energy grid, the computation of
 * c_ism_inst.py:59-96: rsp[ch][i] = sum_j rmf[ch][j] area[j] ism[j] C[j][i],
 * where C[j][i] integrates, over fine bin j = [e_lo[j], e_hi[j]], the
 * not-a-knot cubic spline (scipy.interpolate.CubicSpline, the script's
 * dependency) through the unit vector e_i on the knots e_obs[0..n_obs).
 * rmf [n_ch][n_fine], area/e_lo/e_hi/ism [n_fine] (ism may be NULL: no
 * interstellar factor), e_obs [n_obs] strictly increasing, rsp [n_ch][n_obs]. */
int ppm_response_prepare(int32_t n_ch, int32_t n_fine, const double* rmf, const double* area, const double* e_lo,
                         const double* e_hi, const double* ism, int32_t n_obs, const double* e_obs, double* rsp);
/* c_ism_inst.py:30-101 as a library call: reads the RMF (last column of each
 * line after 3 header lines, energy-major), the ARF (E_lo E_hi area after 3
 * header lines) and, unless ism_path is NULL, the ISM table (columns 0 and 2:
 * energy, transmission, splined at the bin middles and raised to the 5th
 * power); keeps energies [i_e_min, i_e_max) and channels [i_ch_min, i_ch_max);
 * builds E_obs = geomspace(E_lo[first], E_hi[last], n_e_obs); writes num.txt,
 * E_obs.txt and rsp.txt (zeroing |v| < 1e-300) into out_dir, the folder that
 * ppm_engine_load_ism_inst_dir reads. */
int ppm_ism_inst_prepare(const char* rmf_path, const char* arf_path, const char* ism_path, int32_t i_e_min,
                         int32_t i_e_max, int32_t i_ch_min, int32_t i_ch_max, int32_t n_e_obs, const char* out_dir);

/* Writes counts[n_ch][n_bins] as n_ch lines of n_bins space-separated values,
 * the format of gpu/devarshi24st_gpu.cu:491-505 (precision 16) and
 * cpu/devarshi24st_cpu.cpp:246-260 (precision 10). */
int ppm_write_counts(const char* path, int32_t n_ch, int32_t n_bins, const double* counts, int32_t precision);
/* Writes one line of n values (the os1 light-curve format, cpu/os1_cpu.cpp:185-193). */
int ppm_write_row(const char* path, int32_t n, const double* values, int32_t precision);

/* Message of the last failing call on this thread. */
const char* ppm_last_error_string(void);
/* Library version string. */
const char* ppm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PPM_H */
