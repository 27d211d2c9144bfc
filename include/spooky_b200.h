/*
 * spooky_b200.h -- C ABI of the B200-native SPOOKY hot path.
 *
 * The library advances incompressible HD / MHD / Boussinesq fields (with
 * field-aligned anisotropic conduction) in a triply periodic box with the
 * low-storage RK3 integrator and RKL2 super-time-stepping, on one B200.
 *
 * State layout (the reference's): U[f][i][j][k], k < NZ/2+1, complex FP64
 * interleaved (re, im), fields in the order vx vy vz [bx by bz] [th]
 * (heat-equation mode: th only).  i runs over x (slowest), k over z.
 *
 * Every entry point returns an int status (SPK_OK == 0).  A context is not
 * thread safe; all of its GPU work is issued on the one CUDA stream given at
 * creation (NULL: the context creates its own non-blocking stream, since a
 * CUDA graph cannot be captured on the legacy default stream).  No entry point allocates
 * device memory after spk_ctx_create, and spk_advance issues no host
 * synchronisation.
 *
 * Reference interfaces replaced (paths inside LorenzoLMP/spooky-git):
 *   spk_ctx_create       Supervisor::Supervisor + Fields::allocate_and_move_to_gpu
 *                        + Wavevector::Wavevector + init_plan
 *                        (src/supervisor/supervisor.cu:19-66, src/fields/fields.cu:297-363,
 *                         src/fields/wavevector.cu:22-112, src/cuda/cufft_routines.cu:84-96)
 *   spk_set_state /      the device mega-array d_all_fields (src/fields/fields.hpp:64-68)
 *   spk_get_state
 *   spk_clean_divergence Fields::CleanFieldDivergence (src/fields/symmetries.cu:114-130)
 *   spk_compute_dt       TimeStepping::compute_dt (src/timestepping/compute_dt.cu:15-309)
 *   spk_compute_dfield   TimeStepping::compute_dfield (src/timestepping/compute_dfield.cu:11-90)
 *   spk_advance          Supervisor::executeMainLoop body: CleanFieldDivergence +
 *                        TimeStepping::HydroMHDAdvance (src/supervisor/supervisor.cu:179-192,
 *                        src/timestepping/hydro_mhd_advance.cu:18-189)
 *   spk_rkl_cycle        RKLegendre::compute_cycle (src/rkl/rkl.cu:185-199; STS :207-283,
 *                        RKL1 :286-434, RKL2 :437-591)
 *   spk_to_real          Supervisor::Complex2RealFields (src/supervisor/supervisor.cu:261-272)
 *   spk_budgets          computeEnergy (src/io/spooky_output_functions.cu:23-55)
 */
#ifndef SPOOKY_B200_H
#define SPOOKY_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SPK_OK                 0
#define SPK_ERR_ARG            1   /* bad argument (null pointer, bad size)          */
#define SPK_ERR_UNSUPPORTED    2   /* configuration outside what the kernels cover    */
#define SPK_ERR_CUDA           3   /* a CUDA runtime call failed                      */
#define SPK_ERR_ALLOC          4   /* device allocation failed at context creation    */
#define SPK_ERR_NONFINITE      5   /* dt reduction saw NaN/Inf in the real fields     */
#define SPK_ERR_CONFIG         6   /* inconsistent modules (Parameters::checkParameters) */

/* ---- arithmetic forms --------------------------------------------------- */
#define SPK_FORM_PLAIN  0   /* FFT passes and products in FP64 (reference precision)   */
#define SPK_FORM_FP32   1   /* FFT passes and products in FP32, FP64 state and RK/RKL  */

/* ---- super-time-stepping algorithms (Parameters::sts_algorithm) ---------- */
#define SPK_STS_STS     1   /* "sts": damped Chebyshev sub-steps (Alexiades, Amiez & Gremaud 1996) */
#define SPK_STS_RKL1    2   /* "rkl1": first-order Runge-Kutta-Legendre */
#define SPK_STS_RKL2    3   /* "rkl2": second-order Runge-Kutta-Legendre (the default) */

/* ---- integrators --------------------------------------------------------- */
#define SPK_INT_RK3     0   /* TimeStepping::RungeKutta3 (default)                       */
#define SPK_INT_EULER   1   /* TimeStepping::ForwardEuler (the reference's STS test build) */

/* Parameters: the subset of spooky.cfg that the hot path reads
 * (src/parameters/parameters.cu:77-505).  Diffusivities are the inverses of
 * the cfg's reynolds* keys, as the reference computes them (:205-219). */
typedef struct spk_params {
    /* physics.gridsize, physics.boxsize */
    int    nx, ny, nz;
    double lx, ly, lz;
    /* modules */
    int    incompressible, heat_equation, mhd, boussinesq;
    int    stratification, strat_direction;      /* 0=x 1=y 2=z            */
    int    anisotropic_diffusion;
    int    supertimestepping, sts_algorithm;     /* SPK_STS_*              */
    unsigned sts_vars_mask;                      /* bit f: field f is STS  */
    int    with2d, antialiasing;
    /* physics */
    double nu, nu_m, nu_th;                      /* 1/reynolds, 1/reynolds_magnetic, 1/reynolds_thermic */
    double reynolds_ani;                         /* chi_parallel = 1/reynolds_ani */
    double N2, OmegaT2;                          /* brunt_vaissala_squared, mti_frequency_squared */
    /* code */
    double cfl, cfl_par, cfl_sts, safety_source;
    int    safety_sts;
    double t_initial, t_final, toutput_flow;
    /* extensions (not in the reference cfg) */
    double fixed_dt;        /* > 0: use this dt instead of the CFL dt (then clamped like the CFL dt) */
    int    integrator;      /* SPK_INT_RK3 or SPK_INT_EULER                                        */
    int    sts_every_step;  /* 1: RKL cycle after the integrator on every step (the STS test build) */
    int    form;            /* SPK_FORM_PLAIN or SPK_FORM_FP32                                     */
    int    closure;         /* 1, 2 or 3: reserve the learned closure's gradient channels for that
                               variant (HD/MHD; weights from spk_closure_set)                      */
    double closure_kc_frac; /* variant 2: the small scales are |k| > closure_kc_frac * k_c
                               (0: 1/2)                                                            */
    /* shearing box with rotation (modules.shearing, modules.rotating,
     * physics.shear, physics.omega; TimeStepping::ShiftTime / RemapField,
     * Physics::BackgroundShear / BackgroundRotation).  The Coriolis force
     * acts only when shearing is on too (shear_rotation.cu:47), while the dt
     * rule counts omega whenever rotating is on (compute_dt.cu:112-118),
     * both as in the reference. */
    int    shearing, rotating;
    double shear, omega;
} spk_params_t;

/* Fill *p with the reference's defaults (parameters.cu:77-505). */
void spk_params_default(spk_params_t* p);

/* Parameters::Parameters(Supervisor&, char* configfile)
 * (src/parameters/parameters.cu:59-505) for the keys this path reads, then
 * Parameters::checkParameters (:511-566).  The text is libconfig format (the
 * reference's spooky.cfg); *p starts from spk_params_default and each key
 * keeps its default when absent or of another type (an integer written for a
 * float key is ignored, as libconfig's typed lookups do).  form, fixed_dt,
 * integrator and sts_every_step are not configuration keys and keep their
 * defaults.  Returns SPK_OK, SPK_ERR_ARG (unreadable or malformed: the
 * message from spk_last_error(NULL) names the line) or SPK_ERR_CONFIG
 * (inconsistent modules: *p is filled, the message says why). */
int spk_params_from_file(const char* path, spk_params_t* p);
int spk_params_from_string(const char* text, spk_params_t* p);

/* Any key of a spooky.cfg text (the keys of Parameters::Parameters that
 * spk_params_t does not carry: output directory and lists, snapshot and
 * time-series steps, wall-clock limit, initial conditions, ...), with
 * libconfig's typed lookups and the same path syntax ("output.output_dir",
 * "physics.boxsize.[0]").  Return 1 when the key exists with that type (the
 * value is written), 0 when it is absent or of another type (nothing is
 * written), -1 when the text does not parse or an argument is bad
 * (spk_last_error(NULL)).  spk_cfg_setting_length: the element count of a
 * group, array or list, 0 for a scalar, -1 when absent. */
int spk_cfg_lookup_int(const char* text, const char* path, int* out);
int spk_cfg_lookup_bool(const char* text, const char* path, int* out);
int spk_cfg_lookup_float(const char* text, const char* path, double* out);
int spk_cfg_lookup_string(const char* text, const char* path, char* buf, size_t len);
int spk_cfg_setting_length(const char* text, const char* path);

typedef struct spk_ctx spk_ctx;

/* Create a context: validates the modules (checkParameters), builds the
 * wavevector tables and the FFT twiddles, allocates every device buffer.
 * cuda_stream: a cudaStream_t (NULL: a stream owned by the context). */
int spk_ctx_create(const spk_params_t* p, void* cuda_stream, spk_ctx** out);
int spk_ctx_destroy(spk_ctx* ctx);

/* Number of fields F and complex modes Nc = NX*NY*(NZ/2+1) per field. */
int spk_sizes(const spk_ctx* ctx, int* num_fields, size_t* n_complex);

/* where: 0 = device pointer, 1 = host pointer (one cudaMemcpyAsync; pinned
 * host memory gives full PCIe/C2C bandwidth).  Work queued earlier on other
 * streams that produced a device U must be complete before the call. */
int spk_set_state(spk_ctx* ctx, const double* U, int where);
int spk_get_state(spk_ctx* ctx, double* U, int where);

int spk_set_time(spk_ctx* ctx, double t, int step, double t_lastsnap);
int spk_get_time(spk_ctx* ctx, double* t, double* dt, int* step);

/* Fields::CleanFieldDivergence on the context state. */
int spk_clean_divergence(spk_ctx* ctx);

/* TimeStepping::compute_dt on the context state (no divergence cleaning).
 * Outputs may be NULL.  dt_current is the clamped step the integrator uses. */
int spk_compute_dt(spk_ctx* ctx, double* dt_hyp, double* dt_par, double* dt_sts, double* dt_current);

/* TimeStepping::compute_dfield: dU = RHS(U), real buffer = C2R(U).
 * U, dU: device pointers in the state layout ([F][Nc] complex FP64). */
int spk_compute_dfield(spk_ctx* ctx, const double* U, double* dU);

/* nsteps x { CleanFieldDivergence; HydroMHDAdvance } on the context state.
 * Asynchronous on the context stream; captured once into a CUDA graph. */
int spk_advance(spk_ctx* ctx, int nsteps);

/* One RKLegendre::compute_cycle of params.sts_algorithm on the context state
 * with the last dt (uses the real-space B of the last compute_dt / to_real).
 * *s_out (may be NULL) receives the stage or sub-step count. */
int spk_rkl_cycle(spk_ctx* ctx, int* s_out);

/* Supervisor::Complex2RealFields: real fields R[f][i][j][z] (unpadded, FP64)
 * of the context state into a device buffer of F*NX*NY*NZ doubles. */
int spk_to_real(spk_ctx* ctx, double* R);

/* Wait for the context stream; returns the first asynchronous error seen. */
int spk_synchronize(spk_ctx* ctx);

/* ---- the same operations on the caller's state array ---------------------
 * The reference's TimeStepping and RKLegendre members take the device
 * mega-array d_all_fields as an argument (src/timestepping/timestepping.hpp:39-43,
 * src/rkl/rkl.hpp:42).  These forms work in place on such an array, U
 * ([F][Nc] complex FP64, device), with the context's scratch, time, step and
 * dt, so that a caller keeping its own state makes no copies.  Single-box
 * contexts only.  After any of them the context's own state is treated as
 * set from outside (cleaned again before its next step).
 *
 * spk_advance_fields    nsteps x { CleanFieldDivergence; HydroMHDAdvance } on U
 *                       (supervisor.cu:179-192; hydro_mhd_advance.cu:18-75); the
 *                       step graph is recorded once per array and replayed.
 * spk_compute_dt_fields TimeStepping::compute_dt(complexFields, realBuffer)
 *                       (compute_dt.cu:15-309) on U.
 * spk_rk3_fields        TimeStepping::RungeKutta3(complex_Fields, real_Buffer)
 *                       (hydro_mhd_advance.cu:79-189; ForwardEuler with
 *                       SPK_INT_EULER) on U with the dt of the last
 *                       compute_dt: no dt reduction, no cleaning, no
 *                       super-time-stepping.
 * spk_rkl_cycle_fields  RKLegendre::compute_cycle(complex_Fields, real_Buffer)
 *                       (rkl.cu:185-199) on U with the last dt and dt_sts.
 *
 * TimeStepping::compute_dfield's only other input in the reference, the RK
 * stage counter stage_step (compute_dfield.cu:36-46), says whether the real
 * buffer left by compute_dt is still current; spk_compute_dfield always
 * transforms U itself, so it takes no stage argument. */
int spk_advance_fields(spk_ctx* ctx, double* U, int nsteps);
int spk_compute_dt_fields(spk_ctx* ctx, const double* U, double* dt_hyp, double* dt_par, double* dt_sts,
                          double* dt_current);
int spk_rk3_fields(spk_ctx* ctx, double* U);
int spk_rkl_cycle_fields(spk_ctx* ctx, double* U, int* s_out);

/* ---- real-space state and snapshot files ---------------------------------
 * spk_get_state_real   Supervisor::Complex2RealFields + Fields::copy_back_to_host
 *                      (supervisor.cu:261-272, check_output.cu:74-85): the real
 *                      fields R[f][i][j][k] (unpadded, k fastest, FP64) of the
 *                      context state, to host (where = 1) or device (0) memory.
 * spk_set_state_real   the restart's R2C (the unnormalised transform of cuFFT's
 *                      D2Z) of real fields in that layout into the context state,
 *                      which is cleaned before the next step.
 * Both transform on the device in FP64 (a direct sum per line) through the
 * context's RK scratch; they are meant for snapshots, not for every step.
 *
 * spk_write_snapshot   InputOutput::WriteDataFile (src/io/hdf5_io.cu:19-111): an
 *                      HDF5 file with f8 datasets t_start, t_save, t_lastsnap,
 *                      t_lastvar and i4 step (1 element each) and one f8 dataset of
 *                      NX*NY*NZ values per field, named vx vy vz bx by bz th, the
 *                      real field in C order.  t_save and step are the context's.
 *                      With the shearing box the fields are first translated
 *                      along y as InputOutput::UnshearOutput does
 *                      (src/io/unshear_output.cu: exp(-i ky tvel Lx S / 2),
 *                      tvel = fmod(t_save, 2 Ly / (S Lx))); reading applies no
 *                      inverse, as the reference's restart does not.
 * spk_read_snapshot    InputOutput::ReadDataFile's reading part (hdf5_io.cu:159-231):
 *                      sets the state from the file's fields and the time, step
 *                      and t_lastsnap from its scalars; returns t_lastsnap and
 *                      t_lastvar (either may be NULL).  Choosing the file
 *                      (restart -1 = the most recent snapNNNN.h5) is the
 *                      caller's, as in Supervisor::Restart.
 * The files use the format libhdf5 writes with default settings (superblock
 * version 0, a symbol-table root group, version-1 object headers, contiguous
 * data), written and read by the library itself: no HDF5 library is needed.
 *
 * spk_h5_write / spk_h5_read: the same file format for any list of 1-D
 * datasets (host memory; no context, no GPU).  Reading converts the stored
 * integer or floating-point type to the requested one; n must equal the
 * stored element count.  Errors: spk_last_error(NULL). */
int spk_get_state_real(spk_ctx* ctx, double* R, int where);
int spk_set_state_real(spk_ctx* ctx, const double* R, int where);
int spk_write_snapshot(spk_ctx* ctx, const char* path, double t_start, double t_lastsnap, double t_lastvar);
int spk_read_snapshot(spk_ctx* ctx, const char* path, double* t_lastsnap, double* t_lastvar);

#define SPK_H5_F64 0   /* IEEE double, little-endian on write */
#define SPK_H5_I32 1   /* 32-bit signed integer, little-endian on write */
typedef struct spk_h5_dataset {
    const char* name;
    int type;        /* SPK_H5_F64 or SPK_H5_I32 */
    size_t n;        /* elements */
    void* data;      /* write: the n values; read: room for n values */
} spk_h5_dataset_t;
int spk_h5_write(const char* path, const spk_h5_dataset_t* ds, int nds);
int spk_h5_read(const char* path, spk_h5_dataset_t* ds, int nds);

/* Energy budgets in FP64 with the reference's half-spectrum weighting
 * (computeEnergy: (2*sum|q|^2 - sum_{kz=0}|q|^2) / (2 N^6)) per field. */
typedef struct spk_budgets {
    double energy[8];        /* per field: 0.5 <q^2>                       */
    double dissipation[8];   /* per field: <|grad q|^2> (k^2-weighted)     */
} spk_budgets_t;
int spk_budgets(spk_ctx* ctx, spk_budgets_t* out);

/* Time-series quantities of InputOutput::WriteTimevarOutput
 * (src/io/spooky_output_timevar.cu:18-213) beyond the energies of spk_budgets,
 * as FP64 reductions of the context state (Parseval sums over the half
 * spectrum, or grid means of the real magnetic field).  A quantity the
 * modules do not define is -1, the reference's value for it.  Synchronises
 * the context stream.
 *   w2        computeEnstrophy(u): 1/2 <|curl u|^2>, computeEnergy's weighting
 *             (every kz index > 0 counted twice, the Nyquist plane included)
 *   hv        computeHelicity(u): <A . u> with A = i k x u / k^2 (the
 *             reference's Helicity kernel, curl A = u)
 *   j2, hm    the same of B (current, magnetic helicity <A . B>)
 *   hc        <u . B> (twoFieldCorrelation)
 *   thetaB    <|B_z| / |B|>;  bz2 <(B_z / |B|)^2>;  phiB <acos(|B_x| / |B_h|)>
 *             (averagebz, averagebz2, averagephiB, with the 1e-16 guards and
 *             the single-precision acos of user_defined_cuda_kernels.cu:17-46)
 *   dissgradT computeDissipation(th): 1/2 <|grad th|^2> (-1 with anisotropic
 *             conduction and MHD, where the reference reports the field-aligned
 *             form, not computed here)
 *   pv        <curl u . grad th> (potentialVorticity) */
typedef struct spk_diagnostics {
    double w2, hv, j2, hm, hc, thetaB, bz2, phiB, dissgradT, pv;
} spk_diagnostics_t;
int spk_diagnostics(spk_ctx* ctx, spk_diagnostics_t* out);

/* Transfer spectra of InputOutput::WriteSpectrumOutput
 * (src/io/spooky_output_spectrum.cu:186-460): the shell spectrum, as
 * spk_spectrum computes it, of a state field against a nonlinear term built
 * as the reference builds it (real-space products, their transform, the
 * masked wavenumber contraction):
 *   "advec"          u_i  vs  -i mask k_j (u_i u_j)^      (NonLinearAdvection of u), i = x y z
 *   "lorentz"        u_i  vs  -i mask k_j (B_i B_j)^      (NonLinearAdvection of B)
 *   "emfpower"       B_i  vs  i mask (k x (u x B)^)_i    (CurlEMF)
 *   "helicity"       B_i  vs  (i k x B / k^2)_i          (MagneticHelicity)
 *   "th_advec"       th   vs  -i mask k.(u th)^          (AdvectTemperature)
 *   "th_aniso_diss"  th   vs  i mask k.(b (b.grad th) / |b|^2)^   (AnisotropicDissipation, chi = 1)
 *   "th_aniso_inj"   th   vs  i mask k.(b b_s / |b|^2)^           (AnisotropicInjection)
 * out: [ncomp][max_bins] (ncomp 3, or 1 for the th terms); totals[ncomp]
 * (may be NULL): the Parseval sums, i.e. the grid means of field x term --
 * the time series' dissgradT (with anisotropic conduction and MHD: minus
 * the th_aniso_diss total) and fluxbbgradT (the th_aniso_inj total).  The
 * reference accumulates the dissipation term into a scratch array it does
 * not clear (anisotropic_conduction.cu:157); here the term is the divergence
 * alone.  SPK_ERR_UNSUPPORTED when the modules do not define the term.  Uses
 * the pass buffers and the RK scratch; the state is unchanged.
 * Synchronises the context stream. */
int spk_transfer_spectra(spk_ctx* ctx, const char* kind, double* out, int max_bins, int* ncomp, int* nbins,
                         double* deltak, double* totals);

/* Shell spectrum of fields f1, f2 of the context state:
 * InputOutput::computeSpectrum1d / Spectrum1d (src/io/spooky_output_spectrum.cu:424-442,
 * src/cuda/cuda_kernels_generic.cu:441-472).  out[m] (m < min(max_bins, nbins)) is
 * the sum over modes with m = (int)(|k|/deltak + 0.5) of w Re(U_f1/N conj(U_f2/N)),
 * N = NX*NY*NZ, w = 2 for kz index > 0; deltak = 2 pi/min(lx, ly, lz) and
 * nbins = (int)(kmax/deltak + 0.5) with the dealiased kmax (wavevector.cu:100-111).
 * Shells m >= nbins are left out (the reference's kernel adds them past the end
 * of its array).  *total (may be NULL): the Parseval sum with weight 1 at kz = 0
 * and at the Nyquist plane, i.e. the grid mean of f1 f2 (twoFieldCorrelation,
 * src/io/spooky_output_functions.cu).  Synchronises the context stream. */
int spk_spectrum(spk_ctx* ctx, int f1, int f2, double* out, int max_bins, int* nbins, double* deltak,
                 double* total);

/* Launch accounting of one recorded main-loop step: kernels launched per
 * step (RKL stages counted at their recorded bound) and the algorithmic HBM
 * bytes of one RK3 step of this pass design (every array a pass must touch,
 * read once and written once; dealiased regions excluded).  No reference
 * counterpart: it reports on the B200 pipeline. */
int spk_step_info(spk_ctx* ctx, int* kernels_per_step, double* bytes_per_step);

/* Per-pass timing of one RK3 stage: each pass of stage 2 (no cleaning, no
 * dt reduction) is launched `reps` times between CUDA events on the context
 * stream.  out[i]: pass name, average ms per launch, algorithmic bytes per
 * launch, launches per step.  With deferred masked modes (HD/MHD RK3: the
 * RHS of stages 0-1 updates the kept modes only and stage 2 also moves the
 * modes outside the 2/3 mask once) the stage-2 RHS ("rhs_rk", once per step)
 * and the stage-1 RHS ("rhs_rk_01", twice) are reported apart.  The passes
 * update the context state (stage updates), so call it on a context whose
 * state may change.  No reference counterpart. */
typedef struct spk_pass_stat {
    char   name[24];
    double ms;
    double bytes;
    int    launches_per_step;
} spk_pass_stat_t;
int spk_profile_passes(spk_ctx* ctx, int reps, spk_pass_stat_t* out, int max_out, int* n_out);

/* TimeStepping::compute_dfield for callers that cannot allocate device
 * memory.  No counterpart in the reference.
 *
 * Some callers cannot call cudaMalloc: their device memory belongs to another
 * allocator (a fixed pool, an embedding framework), they run in a real-time
 * loop that must not take cudaMalloc's implicit device synchronisation, or
 * they must not fail for lack of memory once started.  This entry point
 * computes dU = RHS(U) like spk_compute_dfield, with no context and no
 * allocation: every scratch array it needs (pass buffers, wavevector tables,
 * FFT twiddles, device scalars) lives in one file-scope device array of
 * SPK_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * the process exits.  The caller passes the input U and the output dU
 * (device pointers, [F][Nc] complex FP64) and a stream (NULL: the legacy
 * default stream); the work is queued on that stream.
 *
 * - The scratch needed is about 2 * C * nx * ny * nzs * (8 bytes in the FP32
 *   form, 16 in the plain form), nzs = nz/2+1 rounded up to even (to a
 *   multiple of 16 / 8 from 64 up), C = 5 (HD),
 *   8 (MHD or Boussinesq), 14 (MHD + Boussinesq + anisotropic conduction);
 *   the heat equation needs only tables.  So every configuration fits at
 *   32^3, and at 64^3 the FP32 form of HD, MHD and Boussinesq does.  Larger
 *   grids are rejected with SPK_ERR_UNSUPPORTED and a message
 *   (spk_last_error(NULL)) giving the size needed.
 * - The first call on a device looks up the array's device address; make
 *   that first call before any stream capture.
 * - Every call shares the one array and clears what must start at zero;
 *   calls whose GPU work overlaps (other streams, other threads) race on it.
 * - Each call copies the wavevector tables, twiddles and starting scalars
 *   from host memory that lives only while the call runs; a call made on a
 *   stream that is being captured returns SPK_ERR_UNSUPPORTED.
 * - The learned closure is not available here: p->closure != 0 returns
 *   SPK_ERR_UNSUPPORTED.
 * - Calls no cudaMalloc/cudaFree and no allocating library routine; errors
 *   are reported through spk_last_error(NULL).  The first-call set-up is
 *   guarded by a lock, so host threads may make their first calls at once. */
#define SPK_NOALLOC_SCRATCH_BYTES (24u << 20)
int spk_compute_dfield_noalloc(const spk_params_t* p, const double* U, double* dU, void* cuda_stream);

/* Ensembles of independent boxes.  No counterpart in the reference, which
 * advances one box per process.  Boxes that share everything but their
 * viscosity, resistivity and thermal diffusivity form a group: one set of
 * arrays holds the group's boxes side by side and every pass kernel covers
 * all of them in one launch, each box with its own dt.  Groups run as
 * parallel branches of one CUDA graph: spk_ensemble_advance launches it once
 * per step.  Super-time-stepping that alternates between steps is not
 * supported (SPK_ERR_UNSUPPORTED), nor super-time-stepping boxes sharing a
 * group.  Boxes are numbered in the order given; state arrays are a box's
 * [F][Nc] complex FP64 (where: 0 device, 1 host).  Per-box calls made while
 * a step is in flight are ordered after it; spk_ensemble_synchronize waits
 * for the whole ensemble and reports the first error of any box. */
typedef struct spk_ensemble spk_ensemble;
int spk_ensemble_create(const spk_params_t* boxes, int nbox, void* cuda_stream, spk_ensemble** out);
int spk_ensemble_destroy(spk_ensemble* ens);
int spk_ensemble_size(const spk_ensemble* ens, int* nbox, int* ngroups);
int spk_ensemble_set_state(spk_ensemble* ens, int box, const double* U, int where);
int spk_ensemble_get_state(spk_ensemble* ens, int box, double* U, int where);
int spk_ensemble_get_time(spk_ensemble* ens, int box, double* t, double* dt, int* step);
int spk_ensemble_budgets(spk_ensemble* ens, int box, spk_budgets_t* out);
int spk_ensemble_advance(spk_ensemble* ens, int nsteps);
int spk_ensemble_synchronize(spk_ensemble* ens);
int spk_ensemble_kernels_per_step(const spk_ensemble* ens, int* kernels);

/* ---- learned subgrid closure ---------------------------------------------
 * No counterpart in the reference.  A pointwise MLP maps eight
 * rotation-invariant, dimensionless features of the resolved velocity
 * gradient A = grad u (A[i][j] = du_i/dx_j) and field gradient G = grad B to
 * an eddy viscosity and an eddy resistivity:
 *   S = (A + A^T)/2, w = curl u, S_B = (G + G^T)/2, J = curl B,
 *   n^2 = S:S + |w|^2/2 + S_B:S_B + |J|^2/2 (+1e-30),
 *   features  S:S/n^2, |w|^2/(2n^2), S_B:S_B/n^2, |J|^2/(2n^2),
 *             tr(S^3)/n^3, w.S.w/n^3, J.S.J/n^3, (w.J)^2/(4n^4);
 *   o = W3 tanh(W2 tanh(W1 f + b1) + b2) + b3           (8 -> 32 -> 32 -> 2)
 *   nu_t = Delta^2 n softplus(o0),  eta_t = Delta^2 n softplus(o1),
 *   Delta^2 = (pi/kxmax * pi/kymax * pi/kzmax)^(2/3)    (dealiased cut-offs).
 * The RHS adds -2 nu_t S to the Basdevant stress and -eta_t J to the EMF
 * before their forward transforms, so both terms only remove energy; the dt
 * rule adds max(nu_t) and max(eta_t) to the parabolic rates.  Parameters
 * are floats in the order W1[32][8] b1[32] W2[32][32] b2[32] W3[2][32] b3[2].
 *
 * Training samples are SoA float rows (row r of every sample contiguous,
 * rows `stride` floats apart): features[8], S[5] (xx xy xz yy yz), J[3],
 * Delta^2 n, target stress[5] (the Basdevant channels: xx xy xz yy yz),
 * target EMF[3], and the strain Sf[5] and current Jf[3] of the whole
 * resolved field (equal to S, J in variant 1).  The loss is the mean over
 * samples of
 *   w0 |dT - T_target|_F^2 + w1 |dE - E_target|^2 + w2 (P - P_target)^2
 * (the full traceless symmetric stress in the Frobenius norm), where
 * P = -dT:Sf - dE.Jf = 2 nu_t S:Sf + eta_t J.Jf is the model's transfer of
 * resolved energy to the subgrid scales and P_target = -T_target:Sf -
 * E_target.Jf the true one (dissipation matching). */
#define SPK_CLOSURE_NFEAT   8
#define SPK_CLOSURE_HIDDEN  32
#define SPK_CLOSURE_NPARAM  (32 * 8 + 32 + 32 * 32 + 32 + 2 * 32 + 2)
#define SPK_CLOSURE_ROWS    33
/* sample rows */
#define SPK_CLOSURE_ROW_FEAT   0
#define SPK_CLOSURE_ROW_S      8
#define SPK_CLOSURE_ROW_J      13
#define SPK_CLOSURE_ROW_SCALE  16
#define SPK_CLOSURE_ROW_TT     17
#define SPK_CLOSURE_ROW_TE     22
#define SPK_CLOSURE_ROW_SF     25
#define SPK_CLOSURE_ROW_JF     30

/* Variant 3 (spk_params_t.closure = 3), the tensor network: the 18 raw
 * gradients of the whole resolved field, made dimensionless,
 *   x = (A[0..8], G[0..8]) / n                       (n as above; HD: G = 0),
 *   h1 = tanh(W1 x + b1), h2 = tanh(W2 h1 + b2), h3 = tanh(W3 h2 + b3),
 *   o = W4 h3 + b4                                   (18 -> 64 -> 64 -> 64 -> 12),
 * in BF16 on the tensor cores: the weights and every layer input (x, h1,
 * h2, h3) are rounded to BF16 (nearest even), the products summed in FP32
 * onto the FP32 bias; tanh in FP32.  With s = Delta^2 n^2 o, s[0..5] is a
 * symmetric stress (xx xy xz yy yz zz) whose traceless part
 *   dT = (s0 - tr/3, s1, s2, s3 - tr/3, s4),   tr = s0 + s3 + s5,
 * is added to the Basdevant stress, and s[6..11] are the off-diagonal
 * entries M_xy M_xz M_yx M_yz M_zx M_zy of an induction tensor whose
 * antisymmetric part is added to the EMF (MHD):
 *   dE = ((M_yz - M_zy)/2, (M_zx - M_xz)/2, (M_xy - M_yx)/2).
 * In the RHS both are multiplied by the backscatter ramp
 *   r = clamp(P / (0.1 Pm + 1e-30), 0, 1),  P = -dT:S - dE.J,
 *   Pm = |dT|_F |S|_F + |dE| |J|
 * (S, J the point's own strain and current; |.|_F over the full 3x3
 * tensors, zz = -(xx + yy) for dT), so that the terms only take energy from
 * the resolved scales; the dt rule adds the largest |r dT|_F / (2 n) and
 * (MHD) |r dE| / n to the parabolic rates.  Parameters are floats in the
 * order W1[64][18] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[12][64]
 * b4[12]; the context and the trainer round the weights to BF16 on upload
 * (the trainer keeps FP32 masters for Adam).  Its samples carry 18 more
 * rows, the raw gradients A (SPK_CLOSURE_ROW_A) and G (SPK_CLOSURE_ROW_G);
 * the loss is the one above with dT, dE of this model (no ramp) and its
 * gradient is taken through the BF16 roundings as if they were absent
 * (straight-through). */
#define SPK_CLOSURE3_NIN     18
#define SPK_CLOSURE3_HIDDEN  64
#define SPK_CLOSURE3_NOUT    12
#define SPK_CLOSURE3_NPARAM  (64 * 18 + 64 + 2 * (64 * 64 + 64) + 12 * 64 + 12)
#define SPK_CLOSURE3_ROWS    51
#define SPK_CLOSURE_ROW_A      33
#define SPK_CLOSURE_ROW_G      42

/* Variants (spk_params_t.closure): 1 -- the gradients of the whole
 * resolved field; 2 -- the gradients of its small scales only, the modes with
 * |k| > f k_c (k_c the smallest dealiased cut-off, f =
 * spk_params_t.closure_kc_frac, 1/2 when 0): features, strain and
 * current all come from that high-passed field, so that the eddy terms act
 * mainly near the cut-off (a variational-multiscale form).  The samples of a
 * coarse context follow its variant. */

/* Switch the closure on (params: spk_closure_nparam(variant) host floats,
 * the context's variant) or off (params NULL) for the context's RHS, steps
 * and dt rule.  HD and MHD contexts; the next step re-records the step
 * graph. */
int spk_closure_set(spk_ctx* ctx, const float* params);

/* The spectral products of U before their divergence / curl: the Basdevant
 * stress (xx xy xz yy yz, traceless symmetric u u - B B) and, with MHD, the
 * EMF u x B, forward-transformed, dealiased modes kept and the others zero
 * (hydro.cu:19-75, mhd.cu:20-62 up to the R2C).  P: device [nprod][Nc]
 * complex FP64, nprod = 5 (HD) or 8 (MHD).  With the closure on, the
 * closure terms are included. */
int spk_products(spk_ctx* ctx, const double* U, double* P, int* nprod);

/* Training samples from one fine-grid state: the fine state Uf and its
 * products are truncated to the coarse grid's dealiased modes (a sharp
 * spectral filter at the coarse cut-off); the targets are the subgrid
 * stress and EMF, products(filtered fine) - products(coarse of the filtered
 * state), and the features come from the filtered state -- one sample per
 * coarse grid point, nx*ny*nz of them, written as SoA rows (stride >=
 * nx*ny*nz floats) into the device array samples.  Both contexts are HD or
 * both MHD, with the same box, and the coarse grid is not finer than the
 * fine one along any axis.  `scratch` is a device buffer of at least
 * *scratch_bytes (from spk_closure_samples_size); the coarse context's
 * state is overwritten with the filtered state. */
int spk_closure_samples_size(const spk_ctx* fine, const spk_ctx* coarse, size_t* scratch_bytes, size_t* nsamples);
int spk_closure_samples(spk_ctx* fine, const double* Uf, spk_ctx* coarse, float* samples, size_t stride,
                        void* scratch, size_t scratch_bytes);

/* Trainer: the MLP's parameters, Adam moments and gradient scratch on the
 * device, trained on device samples by the library's own forward/backward
 * kernels (deterministic: fixed-order reductions).  Minibatch i of a run
 * takes samples (a * (i*batch + r) + c) mod n, r < batch, for an a coprime
 * with n: each pass over n samples visits every sample once. */
typedef struct spk_trainer spk_trainer;
int spk_trainer_create(void* cuda_stream, spk_trainer** out);                 /* variants 1, 2 */
/* A trainer for the network of a variant (1 and 2: the eddy-coefficient
 * network; 3: the tensor network, whose samples have SPK_CLOSURE3_ROWS rows). */
int spk_trainer_create_variant(void* cuda_stream, int variant, spk_trainer** out);
/* Parameters and sample rows of a variant's network (0 for another value). */
int spk_closure_nparam(int variant);
int spk_closure_rows(int variant);
int spk_trainer_destroy(spk_trainer* tr);
int spk_trainer_set_params(spk_trainer* tr, const float* params);        /* host floats; resets Adam */
int spk_trainer_get_params(spk_trainer* tr, float* params);              /* host floats (FP32 masters) */
int spk_trainer_set_samples(spk_trainer* tr, const float* samples, size_t n, size_t stride, const float w[3]);
/* Full-batch mean loss and gradient at the current parameters (host outputs). */
int spk_trainer_loss_grad(spk_trainer* tr, float* loss, float* grad);
/* nsteps Adam steps (lr) on minibatches of `batch` samples; loss_hist
 * (host, may be NULL) receives each step's minibatch loss. */
int spk_trainer_train(spk_trainer* tr, int nsteps, int batch, float lr, float* loss_hist);

/* Schedule autotuner (no reference counterpart).  Picks, by timing whole
 * recorded steps with CUDA events, the launch choices that leave the
 * arithmetic unchanged: the axis tile width of short axes, the z pass's
 * lines per CTA, the axis passes' pipeline stages and the RHS grid (CTAs
 * per SM), by coordinate descent
 * over candidate values; the tuned context computes the same bits as an
 * untuned one.  `steps` timed steps per candidate.  The state and the step
 * scalars are saved (one temporary device copy of the state, freed on
 * return) and restored, so the call leaves the simulation where it was.
 * Outputs (may be NULL): the chosen values (0: the launcher's own model)
 * and the ms per step before and after. */
int spk_autotune(spk_ctx* ctx, int steps, int* z_lines, int* axis_stages, int* rhs_ctas_per_sm, double* ms_before,
                 double* ms_after);
/* The same for every group of an ensemble (each group tuned on its own). */
int spk_ensemble_autotune(spk_ensemble* ens, int steps);
/* The context's launch schedule: the three knobs above (0: the launcher's
 * own model) and the axis tile divisor -- 2 gives the axis passes of axes up
 * to 64 long half-width tiles (a 64^3 box has 33 kz columns, 21 below the
 * 2/3 cut-off, in a 64-column tile), 1 the full tiles; the autotuner tries
 * both where an axis is that short.  Setting it (e.g. a schedule tuned on
 * another context of the same grid) re-records the step graph; the values
 * computed do not change. */
int spk_get_schedule(const spk_ctx* ctx, int* z_lines, int* axis_stages, int* rhs_ctas_per_sm, int* axis_tile_div);
int spk_set_schedule(spk_ctx* ctx, int z_lines, int axis_stages, int rhs_ctas_per_sm, int axis_tile_div);

/* Human-readable text of the last error on this context (or of the last
 * failed spk_ctx_create when ctx is NULL). */
const char* spk_last_error(const spk_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* SPOOKY_B200_H */
