/*
 * qnd.h — C ABI of the B200-native split-operator TDSE engine (libqnd_b200.so).
 *
 * This is the drop-in boundary for QuantumND's hot path (jonathan-dubois/
 * TDSE_ND_MPI). It replaces, inside the reference's C drivers, the FFTW-MPI plans
 * and every loop of integrators.c / calculate_observables.c / the Gram-Schmidt of
 * QuantumND_imag.c. The whole N-D grid lives in one GPU's HBM.
 *
 * Conventions
 *  - Every function returns QND_OK (0) or a non-zero QND_E* code; the message is
 *    in qnd_last_error() (per host thread). The reference aborts instead
 *    (MPI_Abort everywhere); drivers map non-zero codes to stderr + exit(1).
 *  - Arrays are row-major with axis 0 slowest (meshgrid.c:205-211).
 *  - Wavefunctions on the device ("psi_dev") are complex128 (interleaved re, im)
 *    for QND_FP64 contexts and complex64 for QND_MIXED contexts; qnd_state_bytes()
 *    gives the size. Host-side wavefunctions passed to qnd_state_upload/download are
 *    always complex128 (C99 double complex), like the reference's arrays.
 *  - Field samples E/A are host arrays laid out [nsteps][s][dim] exactly like
 *    F.E / F.A (integrators.c:81-101).
 *  - A context is bound to one CUDA device and one stream; it is not re-entrant.
 *  - Observable names are the reference's (calculate_observables.c:48-56): "dipole_r",
 *    "dipole_v", "energy", "Lz", and the zero-width "PMD", "PED", "wavefunction",
 *    "none"; plus two extensions: "norm" (1 value) and "accel" (dim values,
 *    -<dV/dx_j>, needs qnd_set_gradv).
 */
#ifndef QND_H
#define QND_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QND_OK 0
#define QND_EINVAL 1       /* bad argument */
#define QND_ECUDA 2        /* CUDA runtime error */
#define QND_ENOMEM 3       /* device allocation failed */
#define QND_ENORM 4        /* Gram-Schmidt norm below 1e-12 (QuantumND_imag.c:297-304) */
#define QND_EUNSUPPORTED 5 /* configuration outside what this build implements */
#define QND_ENONFINITE 6   /* QND_CHECK_FINITE=1: the state holds NaN or Inf after a run */

#define QND_FP64 0  /* complex128 state, FP64 everywhere */
#define QND_MIXED 1 /* complex64 state, FFT and phases in FP32, all reductions in FP64 */

typedef struct qnd_ctx qnd_ctx;

const char *qnd_version(void);
const char *qnd_last_error(void);

/* ---- context: replaces Initialize_meshgrid (meshgrid.c:17-179) and
 *      Initialize_integrator (integrators.c:13-71). dim is 1 to 6 (the reference takes any
 *      DIMENSION, parameters.c:46-48). nr[j] must be a power of two
 *      (parameters.c:72-76) between 2 and 2^24 (QND_EUNSUPPORTED beyond); axes longer than
 *      4096 points take a four-step transform. integrator: Verlet, BM4, BM6, RKN4. */
int qnd_ctx_create(int dim, const int64_t *nr, const double *dr, const char *integrator, double dt, int precision,
                   qnd_ctx **out);
int qnd_ctx_destroy(qnd_ctx *ctx);
/* Use an existing cudaStream_t (passed as void*); NULL selects the context's own stream. */
int qnd_ctx_set_stream(qnd_ctx *ctx, void *stream);
/* Grid facts: total points, stages s, as_scaled[0..2s) (integrators.c:64), dNr, dNp (meshgrid.c:23-28). */
int qnd_ctx_info(qnd_ctx *ctx, int64_t *n_total, int *s_integrator, double *as_scaled, double *dNr, double *dNp);
int qnd_state_bytes(qnd_ctx *ctx, int64_t *bytes_per_state);

/* ---- potentials (meshgrid.c:133-153) */
int qnd_set_potential_named(qnd_ctx *ctx, const char *name); /* H_1D H_2D H_3D Ne_2D Ne_short_2D Ar_2D Kr_2D Xe_2D */
int qnd_set_potential(qnd_ctx *ctx, const double *vpot_host); /* custom V on the grid [N] */
int qnd_set_cap(qnd_ctx *ctx, double strength, double length); /* quadratic CAP, meshgrid.c:133-135 */
int qnd_set_vcap(qnd_ctx *ctx, const double *vcap_host);       /* custom CAP on the grid [N] */
/* Extensions (no reference counterpart): dV/dx_axis on the grid for "accel"; a per-axis
 * multiplicative mask m_axis[N_axis] applied to psi after every real-time step (NULL clears). */
int qnd_set_gradv(qnd_ctx *ctx, int axis, const double *gradv_host);
int qnd_set_mask_axis(qnd_ctx *ctx, int axis, const double *mask_host);

/* ---- device state helpers (the reference allocates with fftw_alloc_complex,
 *      QuantumND_imag.c:130, QuantumND_real.c:135) */
int qnd_state_alloc(qnd_ctx *ctx, int64_t nstates, void **psi_dev);
int qnd_state_free(qnd_ctx *ctx, void *psi_dev);
int qnd_state_upload(qnd_ctx *ctx, void *psi_dev, const double *psi_host_c128);
int qnd_state_download(qnd_ctx *ctx, double *psi_host_c128, const void *psi_dev);
int qnd_synchronize(qnd_ctx *ctx);

/* ---- split-operator steps (integrators.c:135-232), nsteps consecutive steps on the device */
/* Integration_step_imag (integrators.c:135-163): psi in r-space. */
int qnd_step_imag(qnd_ctx *ctx, void *psi_dev, int64_t nsteps);
/* Integration_step_length (integrators.c:170-194): psi in the unitary p-representation
 * (QuantumND_real.c:190-192); E host [nsteps][s][dim]. */
int qnd_step_length(qnd_ctx *ctx, void *psi_p_dev, const double *E_host, int64_t nsteps);
/* Integration_step_velocity (integrators.c:201-232): psi in r-space; A host [nsteps][s][dim]. */
int qnd_step_velocity(qnd_ctx *ctx, void *psi_dev, const double *A_host, int64_t nsteps);
/* Unitary representation changes used by the length-gauge driver (QuantumND_real.c:190-192, 200-202). */
int qnd_to_p(qnd_ctx *ctx, void *psi_dev);
int qnd_to_r(qnd_ctx *ctx, void *psi_dev);

/* ---- driver loops */
/* Real-time length gauge as QuantumND_real.c:188-229: psi_r_dev in r-space in and out;
 * obs_host [nsteps][nvalues] receives the observables of psi(t_it) before step it, exactly the
 * rows the reference writes (QuantumND_real.c:197-207). obs_host may be NULL when nobs == 0. */
int qnd_run_length(qnd_ctx *ctx, void *psi_r_dev, const double *E_host, int64_t nsteps, int nobs,
                   const char *const *names, double *obs_host);
/* Real-time velocity gauge as QuantumND_real.c:168-187; alpha_host [nsteps][dim] = A(t_it) for
 * the observables (the Field_vectors call at QuantumND_real.c:173). */
int qnd_run_velocity(qnd_ctx *ctx, void *psi_r_dev, const double *A_host, const double *alpha_host, int64_t nsteps,
                     int nobs, const char *const *names, double *obs_host);
/* Gram_Schmidt_orthonormalization (QuantumND_imag.c:265-311) of states_dev[j] against
 * states_dev[0..j); norm2_out (may be NULL) receives ||v||^2 dNr. QND_ENORM below 1e-12. */
int qnd_gram_schmidt(qnd_ctx *ctx, void *const *states_dev, int j, double *norm2_out);
/* The imaginary-time loop body of QuantumND_imag.c:182-185: nsteps x {step, Gram-Schmidt}. */
int qnd_imag_propagate(qnd_ctx *ctx, void *const *states_dev, int j, int64_t nsteps);

/* Device-resident variant of qnd_run_length for pipelines that keep the field and the
 * observable rows on the GPU (no host synchronisation, no host copies): E_dev
 * [nsteps][s][dim] and obs_dev [nsteps][nvalues] are device pointers, and row i holds the
 * observables of psi after step i (the reference's row i+1). Same per-step work as the
 * loop of QuantumND_real.c:195-223. */
int qnd_run_length_dev(qnd_ctx *ctx, void *psi_r_dev, const double *E_dev, int64_t nsteps, int nobs,
                       const char *const *names, double *obs_dev);

/* ---- launch accounting (no reference counterpart; the reference only prints wall
 *      times, QuantumND_real.c:231-235). When enabled, every fused-pass launch is
 *      bracketed by CUDA events on the context's stream. */
int qnd_ctx_set_profiling(qnd_ctx *ctx, int enable);
/* Kernels launched since the last reset, pass launches timed, and their summed device time.
 * Synchronises the stream. reset != 0 clears the counters afterwards. */
int qnd_ctx_get_profile(qnd_ctx *ctx, int64_t *kernels_launched, int64_t *passes_timed, double *pass_ms_total,
                        int reset);

/* ---- observables (calculate_observables.c:89-266) */
int qnd_observable_count(qnd_ctx *ctx, int nobs, const char *const *names, int *nvalues);
/* Calculation_global_observables (calculate_observables.c:119-140) on an r-space psi; alpha [dim]. */
int qnd_observables(qnd_ctx *ctx, const void *psi_r_dev, int nobs, const char *const *names, const double *alpha,
                    double *out_host);
/* Calculation_global_energies (calculate_observables.c:89-116): out[m] = Re <psi|H^(m+1)|psi> dNr. */
int qnd_energies(qnd_ctx *ctx, const void *psi_r_dev, int n, double *out_host);

/* ---- final photoelectron spectra: Write_final_observables (io_functions.c:136-287) on the device.
 * psi_r_dev (not modified) is multiplied by the radial mask of R_MASK (sin^2 between r_mask_min and
 * r_mask_max, 1 beyond; io_functions.c:159-167) and taken to the unitary p-representation.
 *  - npr_host[dim] (may be NULL) receives the kept momenta per axis, |p_j| <= pr_max[j] (the NPR
 *    header of PMD.real).
 *  - ped_host[ne] (may be NULL): the energy distribution S(j de), Gaussian width de, over the kept
 *    momenta (io_functions.c:192-199; the rows of PED.real are j*de, ped_host[j]).
 *  - pmd_host[2 * prod(npr)] (may be NULL): (|psi~|^2, arg psi~) of the kept momenta in flat FFT
 *    order, the binary block of PMD.real (io_functions.c:266-274).
 * Call with both NULL to get the counts first. Synchronises. */
int qnd_final_spectra(qnd_ctx *ctx, const void *psi_r_dev, double r_mask_min, double r_mask_max, const double *pr_max,
                      double de, int ne, double *ped_host, int64_t *npr_host, double *pmd_host);

/* ---- r-space observables without allocation (no reference counterpart).
 * Computes the "norm", "dipole_r" and "accel" values of qnd_observables, in the same row layout,
 * with the same reduction, into the caller's device buffer out_dev[nvalues]. It is asynchronous
 * on the context's stream.
 * It allocates no memory, for callers that must not call cudaMalloc/cudaFree: a monitor sampling
 * a state between the steps of a device-resident loop (cudaFree synchronises the whole device),
 * or a process whose device memory is already reserved by another allocator's pool.
 * Scratch: a fixed 38,144-byte device array per device (partial sums of up to 592 CTAs + a ticket
 * counter that must be zero at launch; the kernel leaves it zero).
 * The first call on a device does a one-time set-up that synchronises the stream; make it before
 * any stream capture. Concurrent calls on one device share the scratch and race: serialise them.
 * Limits: at most 64 values per call (QND_EINVAL beyond). "dipole_v", "energy" and "Lz" give
 * QND_EUNSUPPORTED. "accel" needs qnd_set_gradv for every axis. */
int qnd_observables_rspace_noalloc(qnd_ctx *ctx, const void *psi_r_dev, int nobs, const char *const *names,
                                   double *out_dev);

/* ---- a sweep of independent members in one graph (no reference counterpart: the reference runs
 *      one propagation per job). Member i is qnd_run_length_dev(ctxs[i], psi_r_dev[i], E_dev[i],
 *      nsteps, nobs, names, obs_dev[i]) (same nsteps and observables; grids, integrators, precisions
 *      and potentials may differ; every context on the same device, each once). Per chunk of steps
 *      the members' chains are the parallel branches of one CUDA graph, captured once and replayed,
 *      so the small grids' passes overlap on the GPU with one graph launch per chunk. Members whose
 *      observables need more than the fused reductions run one after another instead. Returns
 *      after the last chunk has run (synchronises). */
int qnd_run_length_batch(int count, qnd_ctx *const *ctxs, void *const *psi_r_dev, const double *const *E_dev,
                         int64_t nsteps, int nobs, const char *const *names, double *const *obs_dev);

/* ---- the same sweep in one persistent kernel (no reference counterpart). Every member's passes are
 *      recorded with the arguments qnd_run_length_dev would launch them with (chunk by chunk, as with
 *      QND_NO_GRAPH set), then one cooperative launch per segment of 512 steps runs all of them: the
 *      CTAs claim line groups in round order (pass r of every member, then pass r + 1) and wait, with
 *      a bounded wait, only for the member's own previous pass, so members advance independently and
 *      small grids fill the GPU together. Members must share one precision; every axis length is 128
 *      to 1024 (QND_EUNSUPPORTED otherwise, or for observables beyond one fused reduction: use
 *      qnd_run_length_batch). A wait that runs out makes the call return QND_ECUDA. Synchronises. */
int qnd_run_length_sweep(int count, qnd_ctx *const *ctxs, void *const *psi_r_dev, const double *const *E_dev,
                         int64_t nsteps, int nobs, const char *const *names, double *const *obs_dev);

/* ---- adjoint gradient of a length-gauge run (no reference counterpart: the differentiation
 *      extension). From psi0_dev (r-space, not modified) it runs nsteps length-gauge steps with the
 *      field samples E_host [nsteps][s][dim] (the step mask applies as in qnd_run_length), evaluates
 *      J = dNr sum_x w(x) |psi_T(x)|^2 for the real weight w_host[n] (natural order; e.g. 1 beyond
 *      |r| > R: the norm absorbed there), and writes dJ/dE[k][ia][j] for every sample into
 *      grad_host [nsteps][s][dim], by running the adjoint state backward through the steps.
 *      The forward states are kept every `checkpoint` steps and recomputed in between: the device
 *      holds ceil(nsteps/checkpoint) + checkpoint + s + 2 states. J_out and psiT_dev (psi(T)) may be
 *      NULL. Synchronises. */
int qnd_adjoint_length(qnd_ctx *ctx, const void *psi0_dev, const double *E_host, int64_t nsteps, const double *w_host,
                       int64_t checkpoint, double *J_out, double *grad_host, void *psiT_dev);
/* The same for a velocity-gauge run (qnd_step_velocity's steps, the step mask after each): dJ/dA for
 * every vector-potential sample A_host [nsteps][s][dim]. */
int qnd_adjoint_velocity(qnd_ctx *ctx, const void *psi0_dev, const double *A_host, int64_t nsteps,
                         const double *w_host, int64_t checkpoint, double *J_out, double *grad_host, void *psiT_dev);

/* ---- laser field on the device: replaces Initialize_field_vectors (integrators.c:74-101) and
 *      Field_vectors (parameters.c:899-949).
 * One mode of the field, as the reference holds it after parameters.c:805-810: frequency
 * omega = 45.5637639947958 / LAMBDA, amplitude F0 = 5.33803e-9 sqrt(INTENSITY), ELLIPTICITY, CEP,
 * DELAY, DURATION, and the envelope (QND_ENV_*: "constant", "trapz", "cos2", "cos4"). */
#define QND_ENV_CONSTANT 0
#define QND_ENV_TRAPZ 1
#define QND_ENV_COS2 2
#define QND_ENV_COS4 3
typedef struct {
    double frequency, amplitude, ellipticity, cep, delay, duration;
    int envelope;
} qnd_laser_mode;

/* E and A summed over the modes (components 0 and, for dim >= 2, 1; the rest 0) at the
 * integrator's sub-step times of steps 0 .. nsteps-1: t = i dt + as[0], then
 * t += as[2j+1] + as[2j+2] between sub-steps j and j+1 (integrators.c:90-99). E_out and A_out are
 * [nsteps][s][dim] (the F.E / F.A layout, ready for qnd_run_length / qnd_run_velocity);
 * alpha_out is [nsteps][dim] = A(i dt), the velocity-gauge observables' shift (QuantumND_real.c:173).
 * Any output may be NULL. on_device = 0: host arrays (the samples are computed on the device and
 * copied back; synchronises); 1: device arrays, filled asynchronously on the context's stream
 * (for qnd_run_length_dev). */
int qnd_field_samples(qnd_ctx *ctx, int nmodes, const qnd_laser_mode *modes, int64_t nsteps, double *E_out,
                      double *A_out, double *alpha_out, int on_device);

/* ---- initial state on the device: the centring and superposition of Read_wavefunction_MPI
 *      (io_functions.c:292-459).
 * psi_dev <- (accumulate ? psi_dev : 0) + coeff * src, where src (host, complex128) is a state on a
 * grid of nr_src[dim] points with this grid's spacing, placed so that point i_j of axis j lands on
 * i_j + (nr[j] - nr_src[j]) / 2; points that fall outside this grid are dropped. Call once per
 * OUTPUT_IMAG state with accumulate = 0 for the first. */
int qnd_state_embed(qnd_ctx *ctx, void *psi_dev, const double *src_host, const int64_t *nr_src, double coeff_re,
                    double coeff_im, int accumulate);

#ifdef __cplusplus
}
#endif
#endif /* QND_H */
