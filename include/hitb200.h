/*
 * hitb200.h — C ABI of the B200 (sm_100a) backend for the HIT_Solver hot path:
 * the hybrid compact/WENO7 right-hand side, its shock sensor, the viscous and
 * source terms, the biharmonic hyperviscosity, the SSP-RK3 step and the
 * reductions that drive time step, forcing and Mach control.
 *
 * Conventions
 *   - State arrays are device pointers to C-contiguous double[4][ny][nx]
 *     ordered [rho, rho*u, rho*v, E] (OOP/equations.py:126-130).  Scalar
 *     fields are double[ny][nx]; masks are uint8_t[ny][nx] (0/1).
 *   - Every call is stream-ordered on the given cudaStream_t (passed as
 *     void*; NULL = legacy default stream) and returns an int status
 *     (HITB200_OK = 0).  Only calls documented as "synchronises" wait for the
 *     device.
 *   - The caller owns every array it passes.  A plan owns its scratch, which
 *     it allocates in hitb200_plan_create and releases in
 *     hitb200_plan_destroy (to the library's block cache; see
 *     hitb200_release_cached_blocks).
 *   - Plans are not thread-safe; distinct plans may be used concurrently.
 *
 * Each entry point names the reference interface it replaces (file:line
 * within the HIT_Solver project).
 */
#ifndef HITB200_H
#define HITB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define HITB200_OK 0
#define HITB200_ERR_INVALID 1     /* bad argument or descriptor  -> ValueError        */
#define HITB200_ERR_CUDA 2        /* CUDA runtime failure        -> RuntimeError      */
#define HITB200_ERR_NONFINITE 3   /* NaN/Inf in the state        -> FloatingPointError */
#define HITB200_ERR_NONPOSITIVE 4 /* rho <= 0 or p <= 0          -> FloatingPointError */
#define HITB200_ERR_OOM 5         /* device allocation failed    -> MemoryError       */
#define HITB200_ERR_UNSUPPORTED 6 /* grid or option outside the supported range        */

/* ---- rhs term selection (bit mask) --------------------------------------- */
#define HITB200_TERM_INVISCID 1 /* -dF/dx - dG/dy, hybrid scheme  */
#define HITB200_TERM_VISCOUS 2  /* viscous stress + heat flux     */
#define HITB200_TERM_FORCING 4  /* rho f source (fx, fy given)    */
#define HITB200_TERM_DRAG 8     /* low-k momentum drag            */
#define HITB200_TERM_COOLING 16 /* uniform mean-pressure sink     */
#define HITB200_TERM_ALL 31

/* ---- solve descriptor ----------------------------------------------------- */
/* One grid and its physics.  NaN in an optional double means "None" in the
 * reference's Python API.  hitb200_desc_init fills the reference defaults of
 * HIT2DConfig (OOP/hit2d.py:36-80). */
typedef struct hitb200_desc {
  int32_t nx, ny;
  double x_min, x_max, y_min, y_max;
  int32_t periodic;  /* 1: periodic (HIT); 0: outflow with guard cells (Riemann) */
  int32_t precision; /* 0: FP64 throughout; 1: FP32 stencil/WENO/flux arithmetic, FP64 state */
  int32_t scheme;    /* 0: hybrid compact/WENO; 1: WENO on every face (Riemann "weno") */
  double gamma;
  /* shock sensor (OOP/spatial_operator.py:252-304, riemann_config3.py:278-326) */
  int32_t sensor_width;
  int32_t boundary_guard; /* outflow only: band forced to WENO before dilation */
  double compression_threshold;
  double jump_threshold;
  double shear_threshold; /* NaN: shear part off */
  /* viscous / thermal (OOP/equations.py:211-267); viscosity 0 turns it off */
  double viscosity, prandtl, gas_constant;
  /* hyperviscosity (OOP/spatial_operator.py:380-435, riemann_config3.py:381-416) */
  double hv_mn;
  double hv_weight[4];
  int32_t hv_interval; /* steps between applications inside hitb200_step; 0: never */
  int32_t guard_cells; /* outflow guard (riemann_config3.py:419-429) */
  /* HIT sources (OOP/hit2d.py:264-426) */
  double drag_coefficient, drag_kmax; /* coefficient <= 0: off */
  double cooling_time;                /* <= 0 or NaN: off */
  double cooling_target_pressure;     /* NaN: 1/gamma */
  /* OU forcing (OOP/forcing.py:11-130) */
  int32_t forcing_on;
  double forcing_kmin, forcing_kmax, forcing_correlation_time, forcing_rms;
  double target_power; /* NaN: None */
  double min_power;
  double max_rescale;  /* NaN: None */
  double alpha_memory;
  /* Mach control (OOP/hit2d.py:293-349) */
  int32_t mach_control;
  double mach_target, mach_memory, mach_exponent;
  double mach_min_power, mach_max_power; /* NaN: None */
  /* time stepping */
  double cfl, tfinal;
  int32_t fixed_dt;   /* 1: dt fixed by hitb200_set_time (Riemann); 0: CFL dt each step (HIT) */
  int32_t noise_mode; /* 0: forcing noise fields uploaded by the caller; 1: device RNG;
                         2: the reference's NumPy stream (PCG64 + ziggurat normals) generated
                         on the device from a state set by hitb200_set_noise_stream */
  uint64_t seed;      /* device RNG seed (noise_mode 1) */
} hitb200_desc;

typedef struct hitb200_plan hitb200_plan;

/* Scalar slots readable with hitb200_read_scalars (doubles). */
enum hitb200_scalar {
  HITB200_S_ALPHA_X = 0,  /* Lax-Friedrichs speed of the last RHS, x */
  HITB200_S_ALPHA_Y = 1,
  HITB200_S_DIV_RMS = 2,  /* sensor divergence rms of the last RHS */
  HITB200_S_VORT_RMS = 3,
  HITB200_S_DT = 4,       /* time step of the current / last step */
  HITB200_S_TIME = 5,
  HITB200_S_STEP = 6,
  HITB200_S_ACTIVE = 7,   /* 1 while time < tfinal (and step < max_steps) */
  HITB200_S_MACH = 8,     /* Mt of the step's start state */
  HITB200_S_POWER = 9,    /* adaptive forcing power target */
  HITB200_S_POWER_DESIRED = 10,
  HITB200_S_F_ALPHA = 11, /* forcing info (OOP/forcing.py:119-130) */
  HITB200_S_F_ALPHA_TARGET = 12,
  HITB200_S_F_POWER_BEFORE = 13,
  HITB200_S_F_INJECTED = 14,
  HITB200_S_F_FXX = 15,
  HITB200_S_F_FYY = 16,
  HITB200_S_F_FXY = 17,
  HITB200_S_F_AF = 18,
  HITB200_S_F_DECAY = 19,
  HITB200_S_F_SCALE = 20, /* factor applied to the unit-rms forcing shape */
  HITB200_S_MAX_STEPS = 21,
  HITB200_S_STATUS = 22,  /* OR of status bits found by the step's reductions */
  HITB200_S_NEAR_THRESHOLD = 23, /* sensor nodes within roundoff of a threshold */
  HITB200_S_HV_APPLIED = 24,     /* hyperviscosity applications so far */
  HITB200_S_COUNT = 32
};
/* Bits of HITB200_S_STATUS. */
#define HITB200_ST_NONFINITE 1    /* NaN/Inf in a state the step read            */
#define HITB200_ST_NONPOS_RHO 2   /* raw density <= 0 (validation)               */
#define HITB200_ST_NONPOS_P 4     /* raw pressure <= 0 (validation)              */
#define HITB200_ST_BARRIER 8      /* a fused prepass/sensor grid barrier timed out
                                     (about 2 s); that step's results are invalid */
#define HITB200_ST_NOISE 16       /* the device noise stream ran short of draws
                                     (noise_mode 2; never expected) */

/* ---- plan ---------------------------------------------------------------- */
/* Defaults of HIT2DConfig (OOP/hit2d.py:36-80) on a 2*pi periodic square. */
int hitb200_desc_init(hitb200_desc* desc);
/* Replaces constructing the sensor/operator/hyperviscosity/forcing objects
 * (OOP/hit2d.py:773-803, OOP/problems/riemann_config3.py:689-707). */
int hitb200_plan_create(const hitb200_desc* desc, hitb200_plan** plan);
/* Synchronises the plan's device, then returns its arena to the block cache. */
int hitb200_plan_destroy(hitb200_plan* plan);
/* Device bytes a plan of this descriptor allocates (admission control). */
size_t hitb200_plan_device_bytes(const hitb200_desc* desc);
/* Block cache: destroyed plans' arenas and batches' tables stay allocated
 * (at most 8 GiB, 2 MiB granules) and serve later plans and batches of the
 * same device, since a cudaFree / cudaMalloc pair per retired and admitted
 * solve stalls a serving loop.  An allocation that fails first frees its
 * device's cached blocks.  hitb200_release_cached_blocks frees them all
 * (every device); hitb200_cached_block_bytes is the total held. */
int hitb200_release_cached_blocks(void);
size_t hitb200_cached_block_bytes(void);
const char* hitb200_status_string(int status);
/* Library build identifier, for logs. */
const char* hitb200_version(void);
/* sizeof(hitb200_desc), so that bindings can check their struct layout. */
size_t hitb200_desc_size(void);

/* ---- operators on caller arrays (stream ordered) --------------------------- */
/* EulerEquation2D.enforce_physical_state (OOP/equations.py:165-181). */
int hitb200_enforce(hitb200_plan* plan, const double* q, double* out, void* stream);
/* The same without a plan: ncells = nx * ny nodes of a [4][ny][nx] state. */
int hitb200_enforce_state(const double* q, double* out, int64_t ncells, double gamma,
                          void* stream);
/* PeriodicEulerShockSensor2D.detect (OOP/spatial_operator.py:263-304) and
 * NonPeriodicEulerShockSensor2D.detect (riemann_config3.py:288-326).
 * enforce_first=1 evaluates it on enforce_physical_state(q), as rhs() does. */
int hitb200_sensor(hitb200_plan* plan, const double* q, uint8_t* mask, int enforce_first,
                   void* stream);
/* _axis_derivative (OOP/spatial_operator.py:321-342, riemann_config3.py:344-357)
 * on enforce_physical_state(q) with a caller mask; axis 0 = x, 1 = y. */
int hitb200_axis_derivative(hitb200_plan* plan, const double* q, const uint8_t* mask, int axis,
                            double* out, void* stream);
/* PeriodicHybridEuler2DOperator.rhs (OOP/spatial_operator.py:344-367) when
 * terms = HITB200_TERM_INVISCID; rhs_with_forcing (OOP/hit2d.py:847-867) with
 * all terms; any subset gives the sum of those terms (e.g. HITB200_TERM_DRAG
 * alone is large_scale_drag_source, OOP/hit2d.py:370-399).  fx, fy (may be
 * NULL without HITB200_TERM_FORCING) are the step's forcing accelerations. */
int hitb200_rhs(hitb200_plan* plan, const double* q, int terms, const double* fx,
                const double* fy, double* out, void* stream);
/* CompressibleNavierStokes2D.viscous_rhs (OOP/equations.py:232-267). */
int hitb200_viscous_rhs(hitb200_plan* plan, const double* q, double* out, void* stream);
/* PeriodicHyperviscosity2D.apply (OOP/spatial_operator.py:407-435) and
 * LocalHyperviscosity2D.apply (riemann_config3.py:398-416); active == NULL
 * returns HITB200_ERR_INVALID as the reference raises ValueError. */
int hitb200_hyperviscosity(hitb200_plan* plan, const double* q, const uint8_t* active,
                           double* out, void* stream);
/* apply_outflow_guard, in place (riemann_config3.py:419-429). */
int hitb200_outflow_guard(hitb200_plan* plan, double* q, void* stream);
/* stable_time_step (OOP/spatial_operator.py:369-377); synchronises. */
int hitb200_stable_time_step(hitb200_plan* plan, const double* q, double cfl,
                             double remaining_time, double* dt_out);
/* validate_raw_physical_state (riemann_config3.py:442-452); synchronises and
 * returns HITB200_ERR_NONFINITE / HITB200_ERR_NONPOSITIVE. */
int hitb200_validate(hitb200_plan* plan, const double* q);
/* Stable time step without a plan, allocating nothing.  No counterpart in the
 * reference (its NumPy stable_time_step allocates freely).  For callers that
 * must not allocate device memory where they need the CFL step: creating a
 * plan calls cudaMalloc and destroying it cudaFree, which synchronises the
 * device; a serving loop sharing the GPU, or a process whose device memory is
 * reserved by its own pool, can take neither.
 * Writes min(cfl / max_cells((|u|+c)/dx + (|v|+c)/dy), remaining_time) (NaN
 * remaining_time: no limit), the value hitb200_stable_time_step returns, to
 * the device double *dt_out, asynchronously on `stream`.  q: device double
 * [4][ny][nx].  The reduction scratch is a static device array of 8448 bytes
 * (held by every GPU that loads the library until exit): grids of more than
 * 1024 tiles of 32 x 32 cells are rejected with HITB200_ERR_UNSUPPORTED.  Its
 * ticket counter must be zero when a call starts; it is zero at module load
 * and each call leaves it zero.  Each call looks up the scratch address of
 * the current device's context (the first call on a device may load the
 * module: make it before any stream capture), so the entry point stays valid
 * after a cudaDeviceReset.  All calls on a device share the scratch, so calls that may overlap on the
 * GPU (other streams or threads) race.  A NaN in any cell makes dt NaN, as
 * the reference's np.max does. */
int hitb200_stable_time_step_noalloc(const double* q, int32_t nx, int32_t ny, double dx,
                                     double dy, double gamma, double cfl,
                                     double remaining_time, double* dt_out, void* stream);

/* ---- forcing ---------------------------------------------------------------- */
/* IsotropicShellOUForcing2D.update (OOP/forcing.py:70-130) for the state q
 * (its primitives give rho, u, v).  noise: device double[ny][nx] white noise
 * (NULL with noise_mode 1 draws it on the device).  Writes fx, fy (the final,
 * scaled accelerations) and updates the plan's OU potential and alpha; the
 * info values are then in the scalar slots HITB200_S_F_*. */
int hitb200_forcing_update(hitb200_plan* plan, const double* q, const double* noise, double dt,
                           double target_power, double* fx, double* fy, void* stream);

/* ---- time stepping ---------------------------------------------------------- */
/* One step of the reference's loop body (OOP/hit2d.py:829-879,
 * riemann_config3.py:729-740): time step from CFL (or the fixed dt), Mach
 * control, forcing update, SSPRK3.step (OOP/time_operator.py:21-26) with
 * rhs_with_forcing and the clean filter, then hyperviscosity every
 * hv_interval steps.  q is advanced in place.  noise: this step's white-noise
 * field (noise_mode 0 with forcing on) or NULL.  Time, step count and every
 * control scalar stay on the device. */
int hitb200_step(hitb200_plan* plan, double* q, const double* noise, void* stream);
/* nsteps calls of hitb200_step replayed from one captured CUDA graph
 * (noise_mode 1 or forcing off).  Steps after time reaches tfinal (or
 * max_steps) are no-ops on the device. */
int hitb200_run(hitb200_plan* plan, double* q, int32_t nsteps, void* stream);
/* One hitb200_step run uncaptured with a CUDA event before every kernel
 * launch; synchronises.  For launch i < cap: ms[i] = its device time and
 * bytes[i] = its algorithmic DRAM bytes (unique inputs read once plus outputs
 * written once, at stored precision).  *count = launches in the step; names
 * receives their labels, one per line.  No reference counterpart: it
 * instruments the step for roofline measurement. */
int hitb200_step_profile(hitb200_plan* plan, double* q, const double* noise, float* ms,
                         double* bytes, int32_t cap, int32_t* count, char* names,
                         size_t names_size, void* stream);
/* Set time, step count, dt (used when fixed_dt = 1) and max_steps (< 0: no limit). */
int hitb200_set_time(hitb200_plan* plan, double time, int64_t step, double dt, int64_t max_steps);
/* Copy scalar slots [0, n) to host memory; synchronises. */
int hitb200_read_scalars(hitb200_plan* plan, double* out, int32_t n);
/* Copy the device scalar slots asynchronously into caller memory
 * (host-pinned or device), n doubles. */
int hitb200_copy_scalars_async(hitb200_plan* plan, double* dst, int32_t n, void* stream);
/* The plan's whole device scalar block: the slots above plus the sensor
 * limits, the drag and forcing coefficients and the OU potential of every
 * forced mode.  A solve's state q and this block are all it carries from one
 * step to the next (the device forcing noise is keyed by seed and step), so
 * saving both and loading them into a plan of the same descriptor resumes the
 * solve bit for bit: the serving loop's checkpoint and restore.  No
 * reference counterpart (its loops keep these values in Python objects).
 * n must equal hitb200_state_block_size(); both calls synchronise. */
size_t hitb200_state_block_size(void);
int hitb200_save_state_block(hitb200_plan* plan, double* out, size_t n);
int hitb200_load_state_block(hitb200_plan* plan, const double* in, size_t n);
/* The PCG64 state of a noise_mode 2 plan's forcing-noise stream: {state low
 * 64 bits, state high, increment low, increment high}, as NumPy's
 * PCG64.state holds them.  Each step then draws standard_normal((ny, nx))
 * from it draw for draw as numpy.random.Generator.standard_normal does
 * (OOP/forcing.py:66,77) and advances it past the draws used.  Both
 * synchronise. */
int hitb200_set_noise_stream(hitb200_plan* plan, const uint64_t* stream_state);
int hitb200_get_noise_stream(hitb200_plan* plan, uint64_t* stream_state);
/* One standard_normal((ny, nx)) field of that stream into out (device
 * double [ny][nx]), advancing it: the field the next step would draw.
 * Stream ordered.  A no-op while the plan's solve is inactive (past its end). */
int hitb200_noise_field(hitb200_plan* plan, double* out, void* stream);
/* Failure injection for the fused prepass/sensor's grid barrier, a test hook
 * with no reference counterpart: the barrier waits for extra_arrivals (0 or
 * 1) CTAs beyond its launch and gives up after limit_seconds of the global
 * timer (default 2 s), each CTA withdrawing its arrival; the step then sets
 * HITB200_ST_BARRIER (its results are invalid) and the GPU stays usable.
 * extra_arrivals = 1 makes every fused step's wait run out; 0 restores
 * normal use.  Applies to the current device; synchronises. */
int hitb200_set_barrier_test(int32_t extra_arrivals, double limit_seconds);
/* Scalar diagnostics of compute_diagnostics (OOP/hit2d.py:471-548), without
 * the spectral divergence/vorticity, plus conservation sums and extrema:
 * out[0..16] = kinetic_energy, Kx, Ky, A_K, C_uv, rms_velocity,
 * turbulent_mach, mean_density, mean_pressure, mass (mean rho * area),
 * x-momentum, y-momentum, total energy (integrals over the domain),
 * raw rho min, rho max, p min, p max.  Synchronises. */
int hitb200_diagnostics(hitb200_plan* plan, const double* q, double* out, int32_t n);

/* ---- initial states on the device ---------------------------------------------- */
/* The streamfunction of initialize_hit_2d (OOP/hit2d.py:158-189):
 * psi[j][i] = sum_m amplitude_m cos(kx_m x_i + ky_m y_j + phase_m) with
 * x_i = x_min + dx (i + 1/2), y_j likewise, accumulated in mode order as the
 * reference does.  modes: device double [n_modes][4] = (kx, ky, amplitude,
 * phase), the phases drawn by the caller in the reference's order;
 * psi: device double [ny][nx]. */
int hitb200_hit_streamfunction(const double* modes, int32_t n_modes, int32_t nx, int32_t ny,
                               double x_min, double dx, double y_min, double dy, double* psi,
                               void* stream);
/* The rest of initialize_hit_2d (OOP/hit2d.py:191-204) from the spectral
 * velocity u = dpsi/dy, v = -dpsi/dx (device double [ny][nx]): removes the
 * means, scales the velocity to target_mach * c_mean / rms (c_mean: the
 * mean sound speed of rho = 1, p = 1/gamma, as the caller's NumPy forms it)
 * and writes the conservative state q (device double [4][ny][nx]) and the rms
 * before scaling to the device double *vrms_out (the reference raises when
 * it is not above machine epsilon).  workspace: device memory of
 * hitb200_hit_compose_workspace_bytes() bytes. */
size_t hitb200_hit_compose_workspace_bytes(void);
int hitb200_hit_compose(const double* u, const double* v, int32_t nx, int32_t ny, double gamma,
                        double target_mach, double c_mean, double* q, double* vrms_out,
                        void* workspace, size_t workspace_bytes, void* stream);
/* Four-quadrant Riemann state (OOP/problems/riemann_config3.py:59-99;
 * riemann_config6.py, riemann_config3_08.py): states = host double [4][4],
 * the primitive (rho, u, v, p) of the lower-left, lower-right, upper-left and
 * upper-right quadrants; a cell is upper when y_j >= y_split and right when
 * x_i >= x_split (cell centres as above); q (device double [4][ny][nx]) =
 * conservative_from_primitive with the density and pressure floors. */
int hitb200_riemann_initial_state(const double* states, int32_t nx, int32_t ny, double x_min,
                                  double dx, double y_min, double dy, double x_split,
                                  double y_split, double gamma, double* q, void* stream);

/* ---- shell spectra ------------------------------------------------------------ */
/* The per-snapshot part of HIT2DSpectra.compute (OOP/postprocess/spectra.py:
 * 48-149) for n_snap snapshots of one grid at once, in three steps on
 * `stream`:
 *   1. hitb200_spectra_fields (snapshot arrays) or hitb200_spectra_state_fields
 *      (conservative states, primitives as primitive_from_conservative,
 *      OOP/equations.py:136-145) writes out[s] = [sqrt(rho) u', sqrt(rho) v',
 *      u', v'], device double [n_snap][4][ny][nx]; u' = u - mean(u) (favre 0,
 *      spectra.py:206-209) or u - mean(rho u) / mean(rho) (favre 1, :202-205);
 *   2. the caller's unnormalised forward real-to-complex 2-D FFT of `out` over
 *      its last two axes: complex double [n_snap][4][ny][nx/2+1] (cuFFT /
 *      numpy.fft.rfft2 layout and sign);
 *   3. hitb200_spectra_shells bins 1/2 (|U|^2 + |V|^2) / (nx ny)^2 (energy) and
 *      1/2 |kx V' - ky U'|^2 / (nx ny)^2 (enstrophy) of every mode into shell
 *      rint(|k| / dk), dk = min(2 pi / (nx dx), 2 pi / (ny dy)), k from
 *      2 pi fftfreq (spectra.py:84-121): energy, enstrophy: device double
 *      [n_snap][min(nx, ny)/2 + 1]; modes beyond the last shell are dropped.
 * The workspace is device memory of hitb200_spectra_workspace_bytes bytes
 * (same n_snap, nx, ny and device) shared by steps 1 and 3.  Sums run in a
 * fixed order.  Grids with min(nx, ny) above 2049 -> HITB200_ERR_UNSUPPORTED. */
size_t hitb200_spectra_workspace_bytes(int32_t n_snap, int32_t nx, int32_t ny);
int hitb200_spectra_fields(const double* rho, const double* u, const double* v, int32_t n_snap,
                           int32_t nx, int32_t ny, int32_t favre, double* out, void* workspace,
                           size_t workspace_bytes, void* stream);
int hitb200_spectra_state_fields(const double* q, int32_t n_snap, int32_t nx, int32_t ny,
                                 int32_t favre, double* out, void* workspace,
                                 size_t workspace_bytes, void* stream);
int hitb200_spectra_shells(const void* spec, int32_t n_snap, int32_t nx, int32_t ny, double dx,
                           double dy, double* energy, double* enstrophy, void* workspace,
                           size_t workspace_bytes, void* stream);

/* ---- line transforms ------------------------------------------------------------ */
/* Hand-written mixed-radix transforms of grid lines (any length up to 1024)
 * with NumPy's fft conventions; the workspaces are caller device memory of
 * the stated size.
 *
 * The spectral diagnostics of a periodic plan's state q: out[0] =
 * divergence_rms and out[1] = vorticity_rms of the spectral derivatives
 * (divergence_and_vorticity, OOP/hit2d.py:146-155, 459-468, in
 * compute_diagnostics :471-548), out[2] = large_scale_kinetic_fraction
 * (:429-449) for the band 0 < |k| <= kmax (0 when kmax <= 0); div and vort
 * (device double [ny][nx], may be NULL) receive the fields themselves (the
 * snapshot's, :571-597).  Synchronises. */
size_t hitb200_spectral_workspace_bytes(int32_t nx, int32_t ny);
int hitb200_spectral_diagnostics(hitb200_plan* plan, const double* q, double kmax, double* out,
                                 double* div, double* vort, void* workspace, size_t workspace_bytes,
                                 void* stream);
/* u = d psi / dy, v = -d psi / dx by spectral derivatives (the initial
 * condition's, OOP/hit2d.py:186-188): psi, u, v device double [ny][nx].
 * Synchronises (its root tables are copied from host memory). */
size_t hitb200_hit_velocity_workspace_bytes(int32_t nx, int32_t ny);
int hitb200_hit_velocity(const double* psi, int32_t nx, int32_t ny, double dx, double dy, double* u,
                         double* v, void* workspace, size_t workspace_bytes, void* stream);
/* numpy.fft.rfft2 of n_fields real arrays [ny][nx] (device doubles) into
 * out, complex double [n_fields][ny][nx/2+1] (the shell spectra's transform,
 * OOP/postprocess/spectra.py:84-121).  Synchronises. */
size_t hitb200_rfft2_workspace_bytes(int32_t nx, int32_t ny);
int hitb200_rfft2(const double* in, int32_t n_fields, int32_t nx, int32_t ny, void* out, void* workspace,
                  size_t workspace_bytes, void* stream);

/* ---- batched form ------------------------------------------------------------- */
/* Many independent solves (any mix of grid sizes) advanced by one launch per
 * kernel of the step: the "ensemble" / serving form.  All descriptors must
 * share precision. */
typedef struct hitb200_batch hitb200_batch;
int hitb200_batch_create(const hitb200_desc* descs, int32_t n, hitb200_batch** batch);
/* A batch over existing plans (no counterpart in the reference: the serving
 * loop regroups resident solves as they arrive and finish).  The batch does
 * not own the plans: hitb200_batch_destroy hands them back, with their
 * scalars and bound states, usable alone or in a later batch.  A plan belongs
 * to at most one batch at a time and is advanced only through it meanwhile.
 * Bind the members' states with hitb200_batch_bind before stepping. */
int hitb200_batch_from_plans(hitb200_plan* const* plans, int32_t n, hitb200_batch** batch);
/* Destroys the batch (waits for the device first) and the plans it owns. */
int hitb200_batch_destroy(hitb200_batch* batch);
/* The member plan of solve i (for per-solve set_time / read_scalars). */
hitb200_plan* hitb200_batch_plan(hitb200_batch* batch, int32_t i);
/* Bind the state array of every solve (device pointers, kept until rebound). */
int hitb200_batch_bind(hitb200_batch* batch, double* const* q);
/* One step of every member.  Each member's sweeps run in a launch of its own
 * nodes-per-thread class (the class its lines give it alone), so a member's
 * results are bit for bit those of its solo run, in any mix. */
int hitb200_batch_step(hitb200_batch* batch, void* stream);
/* nsteps steps replayed from a graph captured at the first call on a stream:
 * the members in two halves (balanced by cells) on two branches of the graph,
 * so that one half's kernels fill the other's tails.  Results are the same
 * as hitb200_batch_step's. */
int hitb200_batch_run(hitb200_batch* batch, int32_t nsteps, void* stream);
/* ---- kernel variants (autotuner knobs; no counterpart in the reference) -------- */
/* Each knob picks the variant of one kernel family: 0 = latency variant
 * (more registers per thread, for launches that cannot fill the GPU), 1 =
 * throughput variant (more resident CTAs per SM, for many solves per
 * launch).  Plans and batches start from a default chosen by launch size;
 * -1 restores that default.  Results do not depend on the knobs, only
 * speed.  Setting a knob drops the captured graph (recaptured on the next
 * run). */
#define HITB200_TUNE_SWEEP_X 0
#define HITB200_TUNE_SWEEP_Y 1
#define HITB200_TUNE_PREPASS 2
/* 1: a single plan whose sensor tiles all fit on the GPU at once fuses each
 * prepass into the following sensor launch (one cooperative launch with a
 * grid barrier instead of two launches); ignored where it cannot apply
 * (batches, larger grids).  Off by default.  Results are bit-identical
 * either way. */
#define HITB200_TUNE_FUSED_SENSOR 3
/* Tile shape of the y sweep: 0 = the default panel width (columns per CTA:
 * 2 for single plans, 4 for batches with many columns), 1 = the other width
 * (4 or 2) where every member's panel fits in shared memory; ignored
 * otherwise.  Results are bit-identical either way. */
#define HITB200_TUNE_Y_PANEL 4
/* 1: a batch advances each SSP-RK3 stage in one persistent launch: the
 * stage's prepass, sensor, y-sweep and x-sweep work of every member taken
 * from one queue, each item waiting (bounded) only for its own solve's
 * previous phase.  Applies to FP32-bulk batches whose members all have
 * sensor width 4 and whose x and y lines all fall in one class (up to 128,
 * 256 or 512 nodes); elsewhere (and for single plans) it reads back 0.  Off by default; the
 * autotuner keeps it where it measures faster.  Results are bit-identical
 * either way. */
#define HITB200_TUNE_PERSISTENT 5
#define HITB200_TUNE_COUNT 6
int hitb200_plan_set_tuning(hitb200_plan* plan, const int32_t* knobs, int32_t n);
int hitb200_plan_get_tuning(const hitb200_plan* plan, int32_t* knobs, int32_t n);
int hitb200_batch_set_tuning(hitb200_batch* batch, const int32_t* knobs, int32_t n);
int hitb200_batch_get_tuning(const hitb200_batch* batch, int32_t* knobs, int32_t n);
/* hitb200_step_profile for a batch (launches cover all member solves). */
int hitb200_batch_step_profile(hitb200_batch* batch, float* ms, double* bytes, int32_t cap,
                               int32_t* count, char* names, size_t names_size, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HITB200_H */
