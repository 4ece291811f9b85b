/*
 * gpe_ssf.h -- C ABI of the B200 split-step Fourier propagator.
 *
 * Plain C types only: device buffers are passed as `void*` device pointers,
 * host buffers as typed host pointers, CUDA streams as `void*`
 * (a cudaStream_t; NULL = legacy default stream).  Every entry point returns a
 * status code (GPE_OK = 0); gpe_last_error() gives the message of the last
 * failure on the calling host thread.  A plan is not thread-safe: use one plan
 * per host thread.  All launch functions are asynchronous on `stream` unless
 * stated otherwise.
 *
 * Arrays are cubes `[x][y][z]` in C order (z fastest), complex64
 * (interleaved float re,im) or complex128 (interleaved double re,im), as in the
 * reference (`gpe/make_propagator.py:23-36`).
 *
 * Reference interfaces replaced (paths within PoyntingZhang/GPE_simulator):
 *   gpe_plan_create      make_real_propagator / make_imag_propagator
 *                        (gpe/make_propagator.py:5-8,106-108) + kernel factories
 *                        (gpe/make_kernel.py:4-136); potentials from
 *                        gpe/expressions.py:9-30 (as bytecode, not CUDA text)
 *   gpe_set_static_potential   stage.staticV (gpe/stage.py:56-62)
 *   gpe_step             the returned closures time_independent_propagator
 *                        (gpe/make_propagator.py:12-54), time_dependent_propagator
 *                        (:57-103), standard_imaginary_step (:109-151), called
 *                        nsteps times as gpe/launch.py:8-13 does
 *   gpe_step_at          one call of time_dependent_propagator(stage, t)
 *                        (gpe/make_propagator.py:57-103)
 *   gpe_halfstep         static_real_halfstep / dynamic_real_halfstep /
 *                        imag_static_real_halfstep (gpe/make_kernel.py:14-119)
 *   gpe_fft3d            cp.fft.fftn / cp.fft.ifftn (gpe/make_propagator.py:50,52)
 *   gpe_norm             get_N (gpe/helper.py:81-88)
 *   gpe_normalise        normalise (gpe/helper.py:91-93)
 *   gpe_kinetic_energy   get_E (gpe/helper.py:135-140)
 *   gpe_nk_extraction    nk_extraction (gpe/nk_extraction.py:16-45)
 *   gpe_diagnostics      save_outputs' scalar + n(k) path (gpe/save.py:31-57),
 *                        fused, plus total energy and chemical potential
 */
#ifndef GPE_SSF_H
#define GPE_SSF_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define GPE_OK              0
#define GPE_ERR_ARG         1   /* bad argument (reference: AssertionError / TypeError) */
#define GPE_ERR_UNSUPPORTED 2   /* grid size with a prime factor > 13, or too large */
#define GPE_ERR_CUDA        3   /* CUDA runtime error */
#define GPE_ERR_OOM         4   /* device allocation failed */
#define GPE_ERR_NONFINITE   5   /* a reduction saw NaN/Inf or a zero norm */
#define GPE_ERR_TIMEOUT     6   /* a bounded device wait ran out */

#define GPE_C64   0
#define GPE_C128  1
#define GPE_IMAGINARY 0
#define GPE_REAL      1

/* static potential array kinds for gpe_set_static_potential */
#define GPE_V_NONE     0
#define GPE_V_REAL64   1   /* float64 real cube (imaginary-time staticV) */
#define GPE_V_CPLX128  2   /* complex128 cube U - i Gamma (real-time staticV) */

/* Potential-expression bytecode: a flat double array, opcodes as doubles.
 * Stack machine evaluated in FP64 per grid point. */
#define GPE_OP_CONST 1  /* followed by one double operand */
#define GPE_OP_X     2
#define GPE_OP_Y     3
#define GPE_OP_Z     4
#define GPE_OP_T     5
#define GPE_OP_ADD   6
#define GPE_OP_SUB   7
#define GPE_OP_MUL   8
#define GPE_OP_DIV   9
#define GPE_OP_POW   10
#define GPE_OP_NEG   11
#define GPE_OP_SIN   13
#define GPE_OP_COS   14
#define GPE_OP_TAN   15
#define GPE_OP_EXP   16
#define GPE_OP_SQRT  17
#define GPE_OP_TANH  18
#define GPE_OP_ABS   19
#define GPE_OP_LOG   20
#define GPE_PROGRAM_MAX   2048  /* doubles */
#define GPE_STACK_MAX     32

typedef struct gpe_plan gpe_plan;

typedef struct gpe_desc {
    int n;                    /* grid points per axis (prime factors <= 13, 2 <= n <= 1024) */
    int dtype;                /* GPE_C64 or GPE_C128 */
    int kind;                 /* GPE_IMAGINARY or GPE_REAL */
    double beta;              /* nonlinear coefficient (stage.beta) */
    double dt;                /* time step (stage.dt) */
    double kinetic_coeff;     /* 1.0 = reference convention exp(-i k^2 dt) */
    const double* x_array;    /* host, n values (stage.x_array) */
    const double* k_array;    /* host, n values (stage.k_array) */
    /* static potential = vx(x) + vy(y) + vz(z) + vg(x,y,z); each program optional */
    const double* static_x;  int static_x_len;
    const double* static_y;  int static_y_len;
    const double* static_z;  int static_z_len;
    const double* static_g;  int static_g_len;
    /* time-dependent potential V(x,y,z,t) (real time only), optional */
    const double* dynamic_g; int dynamic_g_len;
    /* momentum cutoff (real time only) */
    int k_cut_enabled;        double k_cut;
    /* built-in rotating Gaussian stirring beam (real time only):
     * amp*exp(-((x-r cos th)^2+(y-r sin th)^2)/w^2),
     * th(t) = omega*(m^2/(2 t_ramp) + t - m), m = min(t, t_ramp); FP64 angle */
    int beam_enabled;
    double beam_amp, beam_width, beam_radius, beam_omega, beam_t_ramp;
    /* n(k) shells: 0 = reference binning (width 2pi/L), else number of uniform bins */
    int nk_bins;
    /* complex64 plans: 1 = evaluate and apply the local half-step factor in FP64
     * (0 = FP32 phase evaluation); ignored for complex128 */
    int local_fp64;
    /* sweep path: 0 = fastest available (register-resident sweeps for n = 32, 48,
     * 64, 96, 128, 160, 256, else generic); 1 = generic mixed-radix sweeps only;
     * 2 = same as 0; 3 = complex64 n = 128, 256: the y and z sweeps of each
     * x-plane fused into one persistent launch (psi crosses HBM once per launch
     * instead of once per sweep; identical results, measured slower on B200
     * because the sweeps are issue-bound, not HBM-bound); 4 = as 0, and
     * complex64 n = 128, 256 stage the pencils of their plain y/x sweeps by TMA
     * in persistent double-buffered launches (identical results; the y sweep
     * times the same alone, and the step is 4-5% slower because a persistent
     * grid ends the overlap of neighbouring launches). */
    int generic_only;
    /* 1 = exact local sub-flows (an accuracy mode that departs from the reference
     * on purpose; evaluated in FP64 on the generic sweeps): imaginary time
     * psi e^{-Vh} / sqrt(1 + 2 beta |psi|^2 s), s = -expm1(-2Vh)/(2V) (h at V = 0);
     * real time with an absorber U - i Gamma, nonlinear phase beta |psi|^2 tau,
     * tau = -expm1(-2 Gamma h)/(2 Gamma) (h at Gamma = 0).  0 = the reference's
     * frozen-density half-step. */
    int exact_local;
} gpe_desc;

/* library */
int  gpe_version(void);
int  gpe_last_error(char* buf, size_t len);

/* plans */
int  gpe_plan_create(const gpe_desc* desc, gpe_plan** plan);
int  gpe_plan_destroy(gpe_plan* plan);
int  gpe_plan_info(const gpe_plan* plan, int* n, int* dtype, int* kind, int* nk_bins);
int  gpe_set_static_potential(gpe_plan* plan, const void* v, int v_kind, void* stream);

/* propagation (in place on psi; device pointer) */
/* nsteps Strang steps; step i (i = step0 .. step0+nsteps-1) evaluates time-dependent
 * potentials at t_mid = i*dt + dt/2 (gpe/launch.py:10 + gpe/make_propagator.py:94) */
int  gpe_step(gpe_plan* plan, void* psi, int nsteps, long long step0, void* stream);
/* one Strang step at an arbitrary time t (the closure call propagator(stage, t)) */
int  gpe_step_at(gpe_plan* plan, void* psi, double t, void* stream);
int  gpe_halfstep(gpe_plan* plan, void* psi, double t, void* stream);
int  gpe_fft3d(gpe_plan* plan, const void* in, void* out, int inverse, void* stream);
int  gpe_normalise(gpe_plan* plan, void* psi, void* stream);

/* reductions (synchronise `stream`, results on the host) */
int  gpe_norm(gpe_plan* plan, const void* psi, double* norm, void* stream);
int  gpe_kinetic_energy(gpe_plan* plan, const void* psi_k, double* e_kin, void* stream);
int  gpe_nk_extraction(gpe_plan* plan, const void* psi_k, double* occupation,
                       long long* counts, void* stream);
/* scalars[6] = {N, E_kin, E_pot, E_int, E, mu}; nk (nullable) = Nk per shell
 * (length nk_bins from gpe_plan_info), counts (nullable) = modes per shell */
int  gpe_diagnostics(gpe_plan* plan, const void* psi, double t, double* scalars,
                     double* nk, long long* counts, void* stream);

/* Lz = Re integral psi* (x p_y - y p_x) psi dV with spectral momenta (reference
 * gpe/helper.py:143-156 get_L); three sweeps through the plan's work buffer,
 * synchronises `stream` */
int  gpe_angular_momentum(gpe_plan* plan, const void* psi, double* lz, void* stream);

/* Image outputs of the reference's save_outputs (gpe/save.py:59-90): bits select
 * the images; `out` (host) receives n*n doubles (row-major) per selected image,
 * in bit order.  Momentum images are of |fftn(psi)|^2, fftshifted, scaled by
 * dx^3/(M dk^3) (the column sums also by dk); the phase is NaN where the z = n/2
 * slice density is below 1e-12 of its maximum.  Synchronises `stream`. */
#define GPE_PROJ_TOF_XY           1u   /* sum over kz */
#define GPE_PROJ_TOF_YZ           2u   /* sum over kx */
#define GPE_PROJ_TOF_SLICE_XY     4u   /* kz = 0 */
#define GPE_PROJ_TOF_SLICE_YZ     8u   /* kx = 0 */
#define GPE_PROJ_DENSITY_XY      16u   /* dx * sum over z of |psi|^2 */
#define GPE_PROJ_DENSITY_SLICE_XY 32u  /* |psi|^2 at z = n/2 */
#define GPE_PROJ_PHASE_XY        64u   /* arg psi at z = n/2 */
int  gpe_projections(gpe_plan* plan, const void* psi, unsigned which, double* out, void* stream);

/* accounting: kernel launches issued by this plan since creation */
int  gpe_launch_count(const gpe_plan* plan, long long* count);
/* per-launch timing: enable = 1 brackets every sweep launch with CUDA events on its
 * stream (enable = 0 stops; both discard earlier records); read synchronises and
 * returns total milliseconds and launches per sweep axis (ms[3], count[3]: z, y, x) */
int  gpe_profile(gpe_plan* plan, int enable);
int  gpe_profile_read(gpe_plan* plan, double* ms, long long* count);

/* device status word: bit 0 non-finite norm, bit 1 timeout, bit 2 a sweep refused its
 * shared-memory layout (its tiles were not transformed); read and clear (synchronises) */
int  gpe_status(gpe_plan* plan, int* flags, void* stream);

/* Batches: many independent solves (mixed grid sizes, one dtype) advanced together:
 * imaginary-time ground states, and real-time stirred evolutions with the built-in
 * beam (a stirring-rate sweep).  Instances are grouped by grid size and kind; each
 * sweep is one launch per group over (tiles x instances), and one step of all
 * groups is replayed from a CUDA graph with a parallel branch per group.  Replaces
 * calling standard_imaginary_step (gpe/make_propagator.py:109-151) or
 * time_dependent_propagator (:57-103) for each solve in turn.  Every instance
 * computes the arithmetic of its own plan's one-step call (gpe_step with
 * nsteps = 1), so results are identical alone and batched.
 *   gpe_batch_create: count >= 0 instances (an empty batch takes its dtype from
 *     the first gpe_batch_add when count = 0 -- complex64 otherwise).  Real-time
 *     instances take no dynamic expression (the built-in beam only).
 *   gpe_batch_add / gpe_batch_remove: grow or shrink a running batch (continuous
 *     batching); add returns the new instance's index (a freed index is reused).
 *   gpe_batch_bind: psi pointers of every instance (device, C-contiguous) and an
 *     optional active mask (NULL = all); rebinding discards the captured graph.
 *   gpe_batch_step: nsteps steps of every bound instance (imaginary time
 *     renormalised every step; real time at t = step * dt of each instance's clock).
 *   gpe_batch_set_step / gpe_batch_get_step: a real-time instance's clock (steps
 *     taken; its next step evaluates the beam at t_mid = step * dt + dt/2).
 *   gpe_batch_diagnostics: scalars[6*i .. 6*i+5] = {N, E_kin, E_pot, E_int, E, mu}
 *     of every bound instance i (synchronises); real-time instances at their clock's t.
 *   gpe_batch_run: up to nchunks chunks of `chunk` imaginary-time steps with the
 *     convergence test on the device, one synchronisation per call (the loop of
 *     gpe/launch.py:8-13 over standard_imaginary_step with an energy check every
 *     `chunk` steps, for many solves at once).  Per slot i, in and out: live[i]
 *     (nonzero: still advancing), steps[i] (steps taken), e_last[i] (energy at the
 *     previous check; NaN: the first check cannot converge).  After each chunk a
 *     live instance adds `chunk` to steps[i], takes its energy E and stops advancing
 *     when |E - e_last[i]| / (chunk |E|) < tol or steps[i] >= max_steps; e_last[i]
 *     becomes E.  scalars as gpe_batch_diagnostics, at each instance's last check.
 *     Every bound instance must be imaginary-time; frozen instances stay bound
 *     (their launches return at once) until the caller rebinds without them.
 *     Results equal gpe_batch_step(chunk) + gpe_batch_diagnostics per check. */
typedef struct gpe_batch gpe_batch;
int  gpe_batch_create(const gpe_desc* descs, int count, gpe_batch** batch);
int  gpe_batch_destroy(gpe_batch* batch);
int  gpe_batch_add(gpe_batch* batch, const gpe_desc* desc, int* index);
int  gpe_batch_remove(gpe_batch* batch, int index);
int  gpe_batch_bind(gpe_batch* batch, void* const* psis, const int* active, void* stream);
int  gpe_batch_step(gpe_batch* batch, int nsteps, void* stream);
int  gpe_batch_diagnostics(gpe_batch* batch, double* scalars, void* stream);
int  gpe_batch_run(gpe_batch* batch, int chunk, int nchunks, double tol, long long max_steps, int* live,
                   long long* steps, double* e_last, double* scalars, void* stream);
int  gpe_batch_set_step(gpe_batch* batch, int index, long long step);
int  gpe_batch_get_step(const gpe_batch* batch, int index, long long* step);
int  gpe_batch_launch_count(const gpe_batch* batch, long long* count);

/* Renormalise psi in place (psi /= sqrt(N), N = dx^3 sum |psi|^2) without allocating
 * any device memory and without a plan.  No counterpart in the reference: it is for
 * callers that cannot call cudaMalloc -- host frameworks whose memory pool already
 * owns the free HBM, plugin hosts that forbid allocation inside their step callbacks.
 * The reduction scratch is a fixed 16 KiB file-scope device array per GPU (held
 * until the process exits).  Limit: n <= 1024 (2^30 points); larger grids are
 * rejected with GPE_ERR_UNSUPPORTED.  All calls on a device share that array, so
 * calls that overlap on the GPU race.  The first call in each CUDA context looks up
 * the array's address and loads the kernels of both precisions; make it before any
 * stream capture.  Every call synchronises `stream`: norm (nullable, host) receives
 * N, and a zero, NaN or infinite N returns GPE_ERR_NONFINITE with psi unchanged. */
int  gpe_normalise_noalloc(void* psi, int n, int dtype, double dx, double* norm, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GPE_SSF_H */
