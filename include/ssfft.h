/*
 * ssfft.h -- C ABI of libssfft, the sm_100a SmallStrainFFT solver.
 *
 * This is the boundary a host (the Python drop-in classes through ctypes, or any C/C++
 * caller) binds.  It replaces the body of materialite's SmallStrainFFT solve
 * (materialite/models/small_strain_fft/small_strain_fft.py:60-382, materialite 0.1.3)
 * and the per-voxel constitutive protocol of Elastic, ElasticViscoplastic and
 * Multiphase (elastic.py:23-31, elastic_viscoplastic.py:52-271, multiphase.py:31-61).
 *
 * Conventions
 *   - Symmetric second-order tensors are Mandel 6-vectors [11,22,33,23,13,12] with
 *     sqrt(2) on shears (materialite/basis_operations.py:37-48); stiffnesses are 6x6
 *     Mandel matrices, row major.
 *   - Points are in C order of (x, y, z), z fastest (materialite/util/util.py:40-42).
 *   - Rotation matrices take specimen components to crystal components, row major
 *     (materialite/tensor.py:1855-1896).
 *   - Every function returns 0 on success or a negative SSFFT_E* code; the message of
 *     the last failure on the calling thread is available from ssfft_last_error().
 *   - A handle owns all of its device memory and one CUDA stream.  Host pointers passed
 *     in are only read during the call.  One handle must not be used from two host
 *     threads at the same time; distinct handles are independent.
 */
#ifndef SSFFT_H
#define SSFFT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSFFT_OK 0
#define SSFFT_E_INVALID (-1)      /* bad argument or call order */
#define SSFFT_E_CUDA (-2)         /* CUDA runtime error (message has the CUDA text) */
#define SSFFT_E_NOMEM (-3)        /* device allocation failed */
#define SSFFT_E_UNSUPPORTED (-4)  /* grid size or model outside what the kernels handle */
#define SSFFT_E_NAN (-5)          /* non-finite value in a reduction */

/* Arithmetic of the solve.
 * FP64  : every field, FFT and Krylov vector in double.
 * MIXED : fields, FFTs, Green operator and Krylov vectors in float; Krylov dot products,
 *         equilibrium/stress norms and the per-voxel crystal-plasticity Newton in double. */
#define SSFFT_FP64 0
#define SSFFT_MIXED 1

/* Hardening laws (materialite/models/small_strain_fft/hardening_laws.py:18-90). */
#define SSFFT_HARDENING_PERFECT 0 /* props unused */
#define SSFFT_HARDENING_LINEAR 1  /* props[0] = hardening_rate */
#define SSFFT_HARDENING_VOCE 2    /* props = {tau_1, theta_0, theta_1} */
#define SSFFT_HARDENING_AF 3      /* props = {direct_hardening, dynamic_recovery} */

#define SSFFT_MAX_PHASES 8
#define SSFFT_MAX_SLIP 12

/* Output fields for ssfft_get_field.  All are returned as float64, point-major. */
#define SSFFT_FIELD_STRESS 0            /* (V,6) */
#define SSFFT_FIELD_STRAIN 1            /* (V,6) */
#define SSFFT_FIELD_SLIP_RESISTANCES 2  /* (V,S) trial values of the last constitutive call */
#define SSFFT_FIELD_PLASTIC_STRAINS 3   /* (V,6) committed, specimen frame */
#define SSFFT_FIELD_SLIP_SHEAR_STRAINS 4 /* (V,S) trial values of the last constitutive call */
#define SSFFT_FIELD_RESIDUAL 5          /* (V,6) last equilibrium residual b */
#define SSFFT_FIELD_YIELD_STRESSES 6    /* (V,1) J2 yield stresses, trial values of the last call */
#define SSFFT_FIELD_EQ_PLASTIC_STRAINS 7 /* (V,1) J2 equivalent plastic strains, trial values */

typedef struct ssfft_handle ssfft_handle;

/* Grid and solver options; the run() keyword arguments of SmallStrainFFT
 * (small_strain_fft.py:60-71) plus the stress mask of the LoadSchedule
 * (load_schedule.py:17-24), which fixes Gamma-hat(0) (small_strain_fft.py:363-367). */
typedef struct {
  int32_t n[3];                   /* grid points in x, y, z */
  int32_t precision;              /* SSFFT_FP64 or SSFFT_MIXED */
  int32_t device;                 /* CUDA device ordinal */
  int32_t max_newton_iterations;  /* 100 in the reference (small_strain_fft.py:125) */
  int64_t max_krylov_iterations;  /* <= 0: 5 * ndof, scipy's minres default */
  double global_tolerance;        /* default 1e-3 */
  double strain_correction_tolerance; /* default 1e-2 */
  double linear_solver_tolerance; /* default 1e-5 */
  double stress_mask[6];          /* 0/1 per Mandel component */
  /* Absolute floor of the MINRES stopping test, as a fraction of global_tolerance: a
   * solve also stops once its residual |b - A x|_2 is at most
   * krylov_floor * global_tolerance * (mean von Mises stress).  For a linear material the
   * next equilibrium residual is that MINRES residual, and max|r| <= |r|_2, so the floor
   * keeps the next equilibrium error at or below krylov_floor * global_tolerance.  0 (the
   * reference's test alone, small_strain_fft.py:289-293) unless set. */
  double krylov_floor;
  /* Relative forcing of the MINRES stopping test (inexact Newton): a solve also stops once
   * |b - A x|_2 <= krylov_forcing * |b|_2.  0 (the reference's test alone) unless set; in
   * [0, 1). */
  double krylov_forcing;
} ssfft_config;

/* Per load step inputs: the LoadSchedule closures evaluated at (t, dt)
 * (small_strain_fft.py:108-110) and the solver's step bookkeeping. */
typedef struct {
  double strain_increment[6];
  double stress_increment[6];
  double mean_applied_stress[6];
  double dt;
  double summed_von_mises_stress; /* sum of mean von Mises stress of converged steps */
  int32_t time_step_id;           /* number of converged steps so far */
  int32_t reset_fluctuation;      /* 1 when the load reverses (small_strain_fft.py:113-116) */
} ssfft_step_in;

typedef struct {
  int32_t converged;              /* 1: Newton converged, state may be committed */
  int32_t constitutive_failed;    /* 1: a constitutive update did not converge */
  int32_t newton_iterations;
  int32_t max_constitutive_iterations;
  int64_t krylov_iterations;      /* summed over the step's linear solves */
  int32_t linear_solves;
  int32_t status;                 /* 0 or a negative SSFFT_E* code */
  double equilibrium_error;
  double scaled_strain_error;
  double mean_von_mises_stress;
  double mean_stress[6];
  double mean_strain[6];
} ssfft_step_out;

/* Thread-local message of the last failure ("" if none). */
const char *ssfft_last_error(void);

/* Create a solver for one RVE grid (the state SmallStrainFFT.run builds at
 * small_strain_fft.py:73-105).  Allocates all grid-sized device buffers. */
int ssfft_create(const ssfft_config *cfg, ssfft_handle **out);
int ssfft_destroy(ssfft_handle *h);

/* Bytes of device memory a handle with this config and these phase kinds will hold
 * (used by the serving admission control before ssfft_create). */
int ssfft_estimate_bytes(const ssfft_config *cfg, int any_evp, int n_slip, size_t *bytes);

/* Phase definitions.  Elastic: elastic.py:16-31.  EVP: elastic_viscoplastic.py:20-50
 * (stiffness, Schmid tensors sym(d (x) n) as Mandel 6-vectors, reference_slip_rate,
 * rate_exponent, initial slip_resistance, hardening law).  latent_ratio = 1 is the
 * reference; other values enable this library's latent-hardening extension. */
int ssfft_set_phase_elastic(ssfft_handle *h, int phase, const double stiffness[36]);
int ssfft_set_phase_evp(ssfft_handle *h, int phase, const double stiffness[36], int n_slip,
                        const double *schmid, double reference_slip_rate,
                        double rate_exponent, double slip_resistance, int hardening,
                        const double *hardening_props, int n_props, double latent_ratio);
/* J2 small-strain plasticity, IsotropicElasticPlastic(modulus, shear_modulus,
 * yield_stress, hardening_function, hardening_properties)
 * (isotropic_elastic_plastic.py:17-53): isotropic elasticity, radial return with the
 * reference's fixed-point iteration (tolerance 1e-7 on the equivalent plastic strain
 * increment, at most 100 iterations, all points iterated until all have converged).  The
 * hardening laws take the equivalent plastic strain rate as their single slip rate. */
int ssfft_set_phase_j2(ssfft_handle *h, int phase, double modulus, double shear_modulus,
                       double yield_stress, int hardening, const double *hardening_props,
                       int n_props);

/* Microstructure: n_orient unique rotations (n_orient x 9) and per-point indices into
 * them and into the phase table (phase_of_point may be NULL for a single phase 0).
 * Replaces constitutive_model.initialize(orientations) (small_strain_fft.py:94). */
int ssfft_set_microstructure(ssfft_handle *h, int n_orient, const double *rotations,
                             const int32_t *orient_of_point, const int32_t *phase_of_point);

/* Change tolerances, iteration limits and the stress mask of an existing handle (same
 * grid and precision).  Phases may be redefined and ssfft_set_microstructure called again
 * on a handle: buffers are reused when large enough, so one handle can serve a sequence
 * of solves of the same grid. */
int ssfft_set_options(ssfft_handle *h, const ssfft_config *cfg);

/* Reset the solve state to t = start (zero strain/stress, initial slip resistances). */
int ssfft_reset(ssfft_handle *h);

/* One load increment: strain guess, Newton loop with device MINRES and the convergence
 * tests of small_strain_fft.py:106-211. */
int ssfft_step(ssfft_handle *h, const ssfft_step_in *in, ssfft_step_out *out);

/* After a converged step: update_state_variables and old_* <- current
 * (small_strain_fft.py:213-218).  Then the fluctuation carried to the next step is
 * scaled by fluctuation_scale (new_dt / dt, small_strain_fft.py:236-238). */
int ssfft_commit(ssfft_handle *h, double fluctuation_scale);

/* After a failed step: scale the carried fluctuation (1/2 on cutback,
 * small_strain_fft.py:242-244). */
int ssfft_scale_fluctuation(ssfft_handle *h, double factor);

/* Constant-rate load schedule: LoadSchedule.from_constant_rates
 * (load_schedule.py:32-40) with the stress mask of the handle's config, and the time
 * controls of SmallStrainFFT (small_strain_fft.py:30-51). */
typedef struct {
  double strain_rate[6];
  double stress_rate[6];
  double start_time;
  double end_time;
  double initial_time_increment;
  double max_time_increment;   /* <= 0: initial_time_increment */
  double min_time_increment;   /* <= 0: 1e-9 */
} ssfft_rate_schedule;

typedef struct {
  int32_t status;              /* 0, or a negative SSFFT_E* code */
  int32_t steps;               /* converged load increments */
  int32_t cutbacks;
  int32_t reserved;
  int64_t newton_iterations;
  int64_t krylov_iterations;
  double device_seconds;       /* summed device time of the steps */
  double mean_stress[6];
  double mean_strain[6];
  int64_t kernel_launches;     /* kernels this solve launched (graph replays included) */
} ssfft_solve_out;

/* The whole time loop of SmallStrainFFT.run (small_strain_fft.py:106-246) for a
 * constant-rate schedule, natively: reset, steps with cutback and dt adaptation, commits.
 * Used by the serving loop; the Python drop-in drives ssfft_step itself. */
int ssfft_solve_constant_rates(ssfft_handle *h, const ssfft_rate_schedule *sched,
                               ssfft_solve_out *out);

/* ---- serving ---------------------------------------------------------------------
 * A server solves many RVE requests at once on one GPU.  Requests of one class (grid,
 * precision, elastic or crystal-plasticity tangents, slip-system count, stress rates or
 * not) share a group of up to max_slots slots; every kernel launch of a group covers all
 * of its resident requests, whose Newton iterations advance together in rounds run by a
 * CUDA graph, with the Newton decisions, commits, dt adaptation and cutbacks made on the
 * device.  A queued request joins its group at the next round boundary when a slot is
 * free; a slot's device memory (ssfft_estimate_bytes) is allocated on its first use, when
 * it fits both the server's budget and cudaMemGetInfo's free memory.  Classes run
 * concurrently.  Results do not depend on what else runs: every reduction of a request is
 * private to its slot and summed in a fixed order. */

/* One phase of a request (the arguments of ssfft_set_phase_elastic / _evp). */
typedef struct {
  int32_t kind;                /* 0: elastic, 1: crystal elasto-viscoplastic */
  int32_t n_slip;
  int32_t hardening;           /* SSFFT_HARDENING_* */
  int32_t n_props;
  double stiffness[36];
  double schmid[SSFFT_MAX_SLIP * 6];
  double reference_slip_rate, rate_exponent, slip_resistance, latent_ratio;
  double hardening_props[4];
} ssfft_phase;

typedef struct {
  ssfft_config config;         /* grid, precision, tolerances, stress mask, device ignored */
  int32_t n_phases;
  int32_t n_orient;
  ssfft_phase phases[SSFFT_MAX_PHASES];
  const double *rotations;     /* n_orient x 9, copied at submit */
  const int32_t *orient_of_point; /* V, copied at submit */
  const int32_t *phase_of_point;  /* V or NULL, copied at submit */
  ssfft_rate_schedule schedule;
  int64_t tag;                 /* caller's request id, returned in the completion */
  double *stress_out;          /* optional host V x 6: final stress, written before the
                                  completion is posted (caller keeps it alive) */
} ssfft_request;

typedef struct {
  int64_t tag;
  int32_t status;              /* 0 or a negative SSFFT_E* code */
  int32_t slot;
  double submit_time;          /* seconds on the server clock */
  double start_time;           /* admitted: resources allocated, solve starts */
  double end_time;             /* solve finished and results copied out */
  size_t device_bytes;
  ssfft_solve_out result;
  char message[160];           /* ssfft_last_error() of the failing call, or "" */
} ssfft_completion;

typedef struct ssfft_server ssfft_server;

int ssfft_server_create(int device, int max_slots, size_t hbm_budget_bytes,
                        ssfft_server **out);
int ssfft_server_submit(ssfft_server *s, const ssfft_request *req);
/* Move up to max finished requests into out; *n_out = how many.  Non-blocking. */
int ssfft_server_poll(ssfft_server *s, ssfft_completion *out, int max, int *n_out);
/* Requests submitted but not yet polled (queued + running + finished-unpolled). */
int ssfft_server_pending(ssfft_server *s);
double ssfft_server_clock(ssfft_server *s);
/* Kernels the server's groups have launched so far (graph replays counted per kernel). */
int ssfft_server_launches(ssfft_server *s, int64_t *kernel_launches);
/* Stops accepting work, finishes running and queued requests, joins the threads. */
int ssfft_server_destroy(ssfft_server *s);

/* Voronoi region of every point of a dims[0] x dims[1] x dims[2] grid (points at
 * origin + index * spacing, C order with the last axis fastest): the index of the nearest
 * of num_regions seeds (num_regions x 3 host array), over the 27 periodic images shifted by
 * period (the material's sizes, spacing * (dims - 1)) when periodic != 0.  Replaces the
 * cKDTree query of Material.create_voronoi (material.py:337-383, images as
 * util.py:57-88) and matches it except for exact distance ties.  region_of_point: host
 * array of V int32.  Allocates and frees its own device buffers on `device`. */
int ssfft_voronoi(const int32_t dims[3], const double origin[3], const double spacing[3],
                  const double period[3], const double *seeds, int num_regions, int periodic,
                  int device, int32_t *region_of_point);

/* Copy a field out as float64 (V x width).  to_host = 1: dst is host memory;
 * 0: dst is device memory of the handle's device. */
int ssfft_get_field(ssfft_handle *h, int field, double *dst, int to_host);

/* Number of slip systems of the widest EVP phase (0 if none). */
int ssfft_num_slip(ssfft_handle *h);

/* Operator-level entry points used by tests and by the projection apply of
 * small_strain_fft.py:376-382: out = ifftn(Gamma-hat : fftn(in)).real on the handle's
 * grid, in (V,6) float64 host arrays. */
int ssfft_apply_projection(ssfft_handle *h, const double *in_host, double *out_host);

/* Device-pointer variant in the handle's precision: component-planar arrays
 * (6 planes of V values, float or double by precision), on the handle's stream. */
int ssfft_apply_projection_device(ssfft_handle *h, const void *in_dev, void *out_dev);

/* Allocation-free projection, for callers that cannot allocate device memory (code
 * that runs where cudaMalloc is unavailable or forbidden: host callbacks, hooks inside
 * a framework whose allocator owns the device, loops that may not block on an
 * allocation).  No counterpart in the reference: it is the double-precision
 * ssfft_apply_projection_device without a handle.
 *   n, stress_mask : grid and Gamma-hat(0) mask, as in ssfft_config
 *   in_dev, out_dev: caller-owned device arrays, 6 planes of V doubles each
 *   stream         : cudaStream_t to launch on (NULL: the legacy default stream);
 *                    the call waits for it before returning
 * Its scratch (spectrum and FFT tables) is one file-scope device array of about 13 MB
 * that every GPU loading the library holds until exit; grids are limited to
 * nx*ny*(nz/2+1) <= 135168 (64^3) and 1024 points per axis, larger ones are rejected.
 * The first call on a device (current device) looks up the array's address once and
 * keeps it for the life of the process; make it before any stream capture, and do not
 * call again on a device after cudaDeviceReset() there.  All calls share the array:
 * calls that overlap on the GPU race.  Calls no cudaMalloc, cudaFree or allocating library routine. */
int ssfft_apply_projection_noalloc(const int32_t n[3], const double stress_mask[6],
                                   const double *in_dev, double *out_dev, void *stream);

/* Seconds of device time of the last ssfft_step, and kernel launch counters. */
int ssfft_stats(ssfft_handle *h, double *step_seconds, int64_t *kernel_launches);

/* Event timer on the handle's stream: start = 1 records the start event; start = 0
 * records the stop event, waits for it and returns the elapsed seconds. */
int ssfft_timer(ssfft_handle *h, int start, double *seconds);

/* Kernel timing for roofline reports: runs `reps` Krylov iterations' kernels in
 * isolation on the handle's current tangent (the MINRES buffers are overwritten) and
 * returns the mean seconds per launch of each kernel, measured with CUDA events:
 * seconds[0..4] = zfwd (forward transform of tau), yfwd, xpass, yinv, zinv (inverse
 * transform, P tau stored); the y slots are ~0 when the plane-fused passes run the y
 * transforms inside the z kernels; [5] = the update kernel (the previous iteration's vector
 * update and tau = K v); [6] = the epilogue kernel (y' and the MINRES dot products);
 * [7] = one whole Krylov iteration timed back to back.
 * The microstructure must be set and a solve must have run (non-uniform stress). */
int ssfft_profile_krylov(ssfft_handle *h, int reps, double seconds[8]);

#ifdef __cplusplus
}
#endif

#endif /* SSFFT_H */
