/*
 * coral_b200.h -- C-ABI of the B200 plane-layer IMEX timestep.
 *
 * This is the drop-in boundary for Coral's plane-layer hot path: the Fortran
 * driver (src/plane_layer/plane_layer_main.f90) binds these functions with
 * ISO_C_BINDING exactly like it already binds the C text readers of
 * src/text_parsing/cwraps.f90:1-23.  All arguments are plain pointers, sizes
 * and doubles; no C++ or torch types cross the boundary.
 *
 * Conventions
 *  - Complex arrays are interleaved (re, im) doubles: the memory layout of
 *    Fortran complex(kind=8).
 *  - Multi-dimensional arrays use the reference's Fortran (column-major)
 *    shapes, named here with the first index fastest:
 *      coupled-system state  field(T, NYAA, NX/2)       complex
 *      spectral scalar       spec (NZ, NYAA, NX/2)      complex
 *      physical scalar       phys (NZAA, NXAA, NYAA)    real
 *      mean-system state     field(T)                   real
 *    (src/plane_layer/PL_IMEX_timestepping.f90:90-112,
 *     src/slabs.fftw3mpi/transforms.f90:107-131).
 *  - Every function returns 0 on success or a negative CORAL_E* code; the
 *    text of the last error is returned by coral_last_error().  The reference
 *    prints and stops instead (e.g. src/plane_layer/PL_algebra_z_3D.f90:238-240);
 *    a Fortran shim maps a non-zero code to `error stop`.
 *  - One host thread per handle; a handle owns one CUDA stream and all of its
 *    device memory.  Host buffers are only read or written during the call.
 */
#ifndef CORAL_B200_H
#define CORAL_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define CORAL_OK 0
#define CORAL_EBADARG -1      /* invalid argument or size                       */
#define CORAL_ENOMEM -2       /* device allocation failed                       */
#define CORAL_ECUDA -3        /* a CUDA call or kernel launch failed            */
#define CORAL_ESINGULAR -4    /* zero pivot in a band LU factorisation          */
#define CORAL_ENONFINITE -5   /* NaN/Inf detected in the state                  */
#define CORAL_EPARSE -6       /* equation or parameter file could not be read   */
#define CORAL_EIO -7          /* file input/output failed                       */
#define CORAL_EUNSUPPORTED -8 /* recipe feature outside this build              */
#define CORAL_ENODEV -9       /* no usable CUDA device                          */

typedef struct coral_handle coral_handle;

/* Quantities for coral_query(). */
#define CORAL_Q_NX 0
#define CORAL_Q_NY 1
#define CORAL_Q_NZ 2
#define CORAL_Q_NXAA 3
#define CORAL_Q_NYAA 4
#define CORAL_Q_NZAA 5
#define CORAL_Q_N_KXKY_SYSTEMS 6
#define CORAL_Q_N_ZERO_SYSTEMS 7
#define CORAL_Q_N_FULL_VARS 8
#define CORAL_Q_N_QUAD_VARS 9
#define CORAL_Q_STAGES 10
#define CORAL_Q_DEVICE_BYTES 11
#define CORAL_Q_KERNEL_LAUNCHES 12   /* kernels launched by this handle so far */
#define CORAL_Q_SYS_T 100            /* + isys: size T of kxky system isys      */
#define CORAL_Q_ZSYS_T 200           /* + isys: size of mean system isys        */
#define CORAL_Q_SYS_NVARS 300        /* + isys: coupled vars of kxky system     */
#define CORAL_Q_ZSYS_NVARS 400       /* + isys: coupled vars of mean system     */
#define CORAL_Q_SYS_KL 500           /* + isys: sub-diagonals of the evolution band   */
#define CORAL_Q_SYS_KU 600           /* + isys: super-diagonals of the evolution band */
#define CORAL_Q_SYS_REAL 700         /* + isys: 1 if its LU factors are stored real-scaled (8-byte entries),
                                        0 if complex (16-byte entries) */
#define CORAL_Q_SYS_CLASSES 800      /* + isys: independent blocks its solve is split into (1 or 2) */
#define CORAL_Q_SYS_CLASS_T 900      /* + isys: positions per block (= SYS_T when not split)        */
#define CORAL_Q_SYS_CLASS_KL 1000    /* + isys: sub-diagonals of one block's band                   */
#define CORAL_Q_SYS_CLASS_KU 1100    /* + isys: super-diagonals of one block's band                 */
#define CORAL_Q_SYS_FACTOR_ENTRIES 1200 /* + isys: LU band entries per block that the substitution reads
                                        (L and U entries nonzero in some block, and the diagonal),
                                        summed over the block's columns; 0 before coral_factorize or
                                        when the solve reads the whole band */

/*
 * Create a solver from the text of coral.equations and coral.parameters.in.
 * Replaces, for one rank: main%recipe%build (src/plane_layer/PL_equations.f90:435),
 * main%geometry%init (src/plane_layer/PL_geometry.f90:80), main%init
 * (src/plane_layer/PL_IMEX_timestepping.f90:510) and dct_planner
 * (src/slabs.fftw3mpi/transforms.f90:304).  scheme may be NULL (use the one in
 * the parameter text, e.g. 'ARS_222').  The state starts at zero.
 */
int coral_create(const char* equations_text, const char* parameters_text, const char* scheme,
                 int device, coral_handle** out);
/* Same, reading the two files. */
int coral_create_from_files(const char* equations_path, const char* parameters_path,
                            const char* scheme, int device, coral_handle** out);
/*
 * coral_create with the reference's command-line switches that change the
 * solver, space-separated in args (NULL or "" for none):
 *   --withHorizontalSmagorinsky      the full variable nuSmago, the horizontal
 *                                    Smagorinsky viscosity (plane_layer_main.f90:82,
 *                                    PL_equations.f90:519-526, marching.f90:516-541)
 *   --smagorinsky-prefactor X        its prefactor (default 1)
 *   --cflFactor-along-z X            the factor of the vertical CFL term (default 1;
 *                                    at or below 1e-10 the term is left out)
 * (PL_IMEX_timestepping.f90:526-552).  Any other word is CORAL_EBADARG.
 */
int coral_create_with_args(const char* equations_text, const char* parameters_text, const char* scheme,
                           int device, const char* args, coral_handle** out);
void coral_destroy(coral_handle* h);
/* Text of the last error of h (or of the last failed create when h is NULL). */
const char* coral_last_error(const coral_handle* h);
int coral_query(const coral_handle* h, int what, long long* value);

/*
 * Build E = M - dt*a11*L for every (kx,ky) system and LU-factorise it with
 * partial pivoting on the GPU.  Replaces main%factorize_operators
 * (src/plane_layer/PL_IMEX_timestepping.f90:351-422 with
 * src/plane_layer/PL_algebra_z_3D.f90:245-276).
 */
int coral_factorize(coral_handle* h, double dt);

/*
 * Advance nsteps timesteps of size dt (refactorising first if dt differs from
 * the factorised one).  Replaces main%march_forward = one_step_beyond
 * (src/plane_layer/PL_IMEX_timestepping_marching.f90:3-48).  The work is
 * queued on the handle's stream; the call returns after the launches.
 */
int coral_march(coral_handle* h, double dt, int nsteps);

/* Wait for the handle's stream; reports device-side errors. */
int coral_synchronize(coral_handle* h);

/* State of kxky system isys in the layout field(T, NYAA, NX/2) (complex). */
int coral_get_field(coral_handle* h, int isys, double* field);
int coral_set_field(coral_handle* h, int isys, const double* field);
/* State of mean system isys, field(T) (real). */
int coral_get_mean_field(coral_handle* h, int isys, double* field);
int coral_set_mean_field(coral_handle* h, int isys, const double* field);

/*
 * Transforms of one scalar.  Replace PS_fields_T%spec_to_phys = c2r_transform
 * and PS_fields_T%phys_to_spec = r2c_transform
 * (src/slabs.fftw3mpi/transforms.f90:155-301) with the slab transposes done
 * on the device.
 */
int coral_spec_to_phys(coral_handle* h, const double* spec, double* phys);
int coral_phys_to_spec(coral_handle* h, const double* phys, double* spec);

/*
 * Full variable ivar (uFull, vFull, ...) in physical space, phys(NZAA, NXAA, NYAA),
 * as computed from the current state (compute_full_variables_in_physical_space,
 * src/plane_layer/PL_IMEX_timestepping_marching.f90:420-588).
 */
int coral_get_full_phys(coral_handle* h, int ivar, double* phys);

/*
 * Read / write the QuickSave files of a directory (…/QuickSave.kxky.sysSSS.varVVV.rollingR,
 * …/QuickSave.zero.sysSSS.varVVV.rollingR; physical fields in z-fastest, y, x order).
 * Replace main%import_quickSave and main%export_checkpoints
 * (src/plane_layer/PL_IMEX_timestepping_output.f90:309-456).  As the reference's
 * export does, coral_export_checkpoint then replaces each coupled variable's
 * state by the projection of the field it wrote (the state becomes what
 * importing the files gives; a round-off change on the represented modes).
 */
int coral_import_quicksave(coral_handle* h, const char* directory, int rolling);
int coral_export_checkpoint(coral_handle* h, const char* directory, int rolling);

/*
 * Set one coupled variable (ivar of kxky system isys) from a physical field
 * phys(NZAA, NXAA, NYAA), or one mean variable from a profile prof(NZAA): the
 * per-variable step of import_quickSave (transform, square-stencil projection
 * onto the Galerkin basis, insertion; PL_IMEX_timestepping_output.f90:338-381).
 * The projection replaces that variable's coefficients.
 */
int coral_set_var_phys(coral_handle* h, int isys, int ivar, const double* phys);
int coral_set_mean_var_profile(coral_handle* h, int isys, int ivar, const double* prof);

/*
 * The CUDA stream (a cudaStream_t, returned as void*) on which the handle
 * queues all its work, so that callers can order their own work or record
 * CUDA events around coral_march.
 */
int coral_stream(coral_handle* h, void** stream);

/*
 * Run one timestep of size dt with eager launches and CUDA events around each
 * kernel class; ms[k] receives the device time of class k summed over the
 * stages (k = 0 inverse y pass, 1 inverse x pass, 2 inverse z pass (0: fused
 * into class 3), 3 z passes with the products (inverse z, CFL maxima, products,
 * forward z), 4 forward x pass, 5 forward y pass, 6 NL assembly (complex
 * factors only), 7 right-hand side with the NL assembly (real-scaled factors)
 * or stage update + banded solve (complex factors), 8 mean systems,
 * 9 banded substitutions, 10 K_std and stage output).  n >= 11.
 * The step advances the state exactly like coral_march(h, dt, 1).
 * (The reference has wall-clock prints only, plane_layer_main.f90:166-171.)
 */
int coral_profile_step(coral_handle* h, double dt, double* ms, int n);

/*
 * coral_spec_to_phys_noalloc -- no counterpart in the reference.
 *
 * The inverse transform of coral_spec_to_phys for one scalar, for callers that
 * cannot allocate device memory (their memory belongs to another allocator or
 * runtime, or allocation is forbidden after start-up).  No handle is needed and
 * nothing is allocated: spec (NZ, NYAA, NX/2 complex) and phys (NZAA, NXAA, NYAA
 * real) are the caller's device buffers, and the transform's intermediate
 * arrays live in a 64 MiB __device__ array that every GPU loading this library
 * holds until exit.  Grids whose intermediates need more than 64 MiB (about
 * 128 x 128 x 96 modes) are rejected with CORAL_EBADARG.  The work is queued on
 * stream (a cudaStream_t; NULL = the legacy default stream) and the call returns
 * after the launches.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and sets kernel attributes: make it before any
 * stream capture.  All calls on a device share the array, so calls that can
 * overlap on the GPU (different streams, no ordering) race.
 */
int coral_spec_to_phys_noalloc(int NX, int NY, int NZ, const double* spec, double* phys, void* stream);

/*
 * Diagnostics of the first stage of the last step: out[0] = cargo%cfl_based_DT
 * (marching.f90:200-254), out[1] = cargo%KE_display = sum of the volume
 * averages of uu, vv and ww (PL_IMEX_timestepping_output.f90:84-102; 0 when
 * those quadratic variables are absent), out[2] = 1 if any state entry is
 * non-finite.
 */
int coral_diagnostics(coral_handle* h, double* out3);

/*
 * Timeseries objects: the text of coral.timeseries (lines
 * '>>Volume_average :: NAME <<' and '>>Horizontal_avg :: NAME ;; Position= K <<'
 * up to '>>EOF<<', NAME a full or quadratic variable, K a 1-based z grid index;
 * at most 16 objects).  Replaces master_recipe%add_timeseries
 * (src/plane_layer/PL_equations.f90:233-320).  Every later step evaluates the
 * objects on its first stage's physical fields, as output_global_quantities
 * does (src/plane_layer/PL_IMEX_timestepping_output.f90:5-127).
 */
int coral_set_timeseries(coral_handle* h, const char* timeseries_text);
int coral_set_timeseries_from_file(coral_handle* h, const char* path);
/* Values of the objects at the last step, in the reference's buffer order
 * (full variables in recipe order, then quadratic variables); n >= count. */
int coral_timeseries(coral_handle* h, double* values, int n);

/*
 * Time keeping of the driver loop (src/misc/timeKeeping.f90): set the time,
 * the current dt and the step index, e.g. from CheckPoints/dt.sav after the
 * reference's dt / 50 restart rule (read_timings_from_file, :92-134; dt is
 * capped at dt_max).  A new handle starts at t = 0, dt = dt_max, step 1.
 * coral_get_time: out4 = (time, dt_current, i_timestep, refactorisations so far).
 */
int coral_set_time(coral_handle* h, double time, double dt, long long i_timestep);
int coral_get_time(coral_handle* h, double* out4);

/*
 * The time loop of src/plane_layer/plane_layer_main.f90:138-205 for nsteps
 * steps: before each step dt_current takes the CFL target when they differ by
 * more than tolerance * dt_current, with refactorisation (update_dt_if_needed,
 * timeKeeping.f90:171-183; factorize_operators); after it the target becomes
 * CFL_C * cfl_based_DT capped at dt_max, and the run stops with
 * CORAL_ENONFINITE below dt_min = 1e-9 (compare_dt_against_CFL, :78-89).  The
 * timeseries objects are written every 20 steps and at the end to
 * output_directory/Timeseries/ in the reference's files (time.dat,
 * NAME_volAvg.dat, NAME_XYavg_zKKKKK.dat: raw float64, step k at offset 8(k-1);
 * PL_IMEX_timestepping_output.f90:136-231); output_directory may be NULL or empty (no files).
 * Synchronous: returns when the steps are done.
 */
int coral_run(coral_handle* h, int nsteps, const char* output_directory);

/*
 * User outputs: the text of coral.usrOutput (lines '>>Volume :: NAME ;; Period= P <<',
 * '>>XSlice :: NAME ;; Period= P ;; Position= I <<' and likewise '>>YSlice ::',
 * '>>ZSlice ::', '>>Zsummed:: NAME ;; Period= P <<', '>>Profile:: NAME ;; Period= P <<'
 * up to '>>EOF<<'; NAME a full or quadratic variable, I a 1-based grid index,
 * entries beyond the grid ignored).  Replaces master_recipe%add_outputs
 * (src/plane_layer/PL_equations.f90:322-427).  coral_run then writes, at the
 * first stage of each step (from the state at its start), the objects whose
 * counter reaches their period (output_slices_volumes_and_profiles,
 * PL_IMEX_timestepping_marching.f90:639-697; counters and the time index start
 * from the step index, as initialise_bookkeeping_counters, :620-637, and
 * restart with coral_set_time) into output_directory/Volumes, /Slices and
 * /Profiles under the reference's names (linear_varVV_timeTTTTTTTT_full.dat,
 * linear_varVV_zKKKKK_..., _yKKKKK_, _xKKKKK_, _zAvged_, quadra_varVV_...), raw
 * float64 in its order: a volume x-major then y then z; a z slice and the
 * weighted z sum x-major then y; a y slice x-major then z; an x slice y-major
 * then z; a profile z (PL_IMEX_timestepping_output.f90:250-307,489-581,685-715;
 * src/slabs.fftw3mpi/transforms.f90:53-105,772-866).  Quadratic variables are
 * the products of their full variables, with the vertical mean removed where
 * the recipe asks; a Zsummed object of a quadratic variable is refused
 * (CORAL_EUNSUPPORTED: the reference stops there).
 */
int coral_set_usr_output(coral_handle* h, const char* usr_output_text);
int coral_set_usr_output_from_file(coral_handle* h, const char* path);
/* Write every user-output object now, from the current state, with time index
 * time_integer (export_allPhys / export_allProfiles for a driver that steps
 * with coral_march); the periods and counters are not used. */
int coral_export_usr_output(coral_handle* h, const char* output_directory, long long time_integer);

/*
 * on != 0: after every step, replace the kx = 0 line of every coupled state by
 * its Hermitian part (f(0,ky) + conj f(0,-ky)) / 2.  Off by default, which
 * reproduces the reference's arithmetic.  Every physical value is unchanged:
 * the inverse transform keeps only the real part of the kx = 0 coefficient
 * (src/slabs.fftw3mpi/transforms.f90:197-210), so the anti-Hermitian part of
 * that line is invisible, receives no nonlinear feedback and, where the
 * (kx = 0, ky) operators are unstable, grows exponentially from round-off
 * until it contaminates the fields (seen in the rotating convection benchmark
 * after ~0.2 diffusive times).  Has no counterpart in the reference.
 */
int coral_set_hermitian_kx0(coral_handle* h, int on);

/*
 * Positions (0-based, within T) of the Galerkin coefficients of coupled variable
 * ivar of kxky system isys in the interleaved state layout
 * (src/plane_layer/PL_IMEX_timestepping.f90:1344-1414).  *size receives the
 * variable's coefficient count; positions (may be NULL) needs n >= that count.
 */
int coral_var_positions(coral_handle* h, int isys, int ivar, int* positions, int n, int* size);

/*
 * The form of the z (Chebyshev) transforms inside the time step:
 *   0  FP64 FFT-based transforms fused with the products (default);
 *   1  split precision: the transforms as dense contractions on the tensor
 *      cores (tcgen05.mma kind::i8) with both operands in five int8 digits
 *      (a shared exponent per data column), exact INT32 accumulation and one
 *      rounding to FP64 -- about 39 significant bits relative to a column's
 *      largest value; the x / y FFTs, the band solves and the stage sums stay
 *      FP64.  Needs NZ and 3 NZ / 2 to be multiples of 96 (CORAL_EUNSUPPORTED
 *      otherwise).
 * The reference does these transforms with FFTW r2r in FP64
 * (src/slabs.fftw3mpi/transforms.f90:216-249); form 1 has no counterpart there.
 */
int coral_set_z_transform(coral_handle* h, int form);

/*
 * Source NN of the mean equations' 'add_rhs_source :: ... sourceNN' terms
 * (marching.f90:398-415): its physical values on the Gauss-Chebyshev grid,
 * NZAA doubles, z(i) = center + cos(pi (2i - 1) / (2 NZAA)) gap / 2.  Replaces
 * the reference's compiled-in PL_user_sources_definitions.f90; without a call,
 * source01 and source02 are that file's defaults (source01 from sourceParam
 * HovEll, source02 = -1) and a step with any other source referenced fails
 * with CORAL_EBADARG.
 */
int coral_set_source(coral_handle* h, int index, const double* profile);
/*
 * The penalisation mask (the maximum over the user's masks) on the physical
 * grid, NYAA x NXAA x NZAA doubles, z fastest (phys(NZAA, NXAA, NYAA) of the
 * reference).  Every 'enable_penalisation' variable's field becomes
 * strength (1 + tanh(width mask)) / 2 (init_penalisation, marching.f90:778-822).
 * Replaces the compiled-in PL_user_penalisation_mask.f90, whose two example
 * masks are the default.
 */
int coral_set_penalisation_mask(coral_handle* h, const double* mask);

/*
 * Ensembles: n independent runs (each its own coral.equations /
 * coral.parameters.in text: grid, parameters and recipe may differ; the IMEX
 * scheme's stage count may not) advanced together on one CUDA stream with one
 * CUDA graph per step.  Per stage the band substitutions of every member's
 * (kx, ky) systems run as one persistent launch when every member's systems
 * use the split thread-per-block layout with the plane-layer band (9, 23)
 * (coral_ensemble_query(e, 2) = 1); otherwise member by member.  The
 * reference runs one problem per job and solves its systems one at a time
 * (src/plane_layer/PL_algebra_z_3D.f90:197-214); each member here computes
 * exactly what a single handle of the same problem computes.
 * coral_ensemble_member returns a member's handle (owned by the ensemble; do
 * not destroy it) for the state, QuickSave, diagnostics and transform calls.
 * coral_ensemble_query: what = 0 members, 1 kernels launched so far,
 * 2 substitutions batched (0/1), 3 kernels per ensemble step.
 */
typedef struct coral_ensemble coral_ensemble;
int coral_ensemble_create(int n, const char* const* equations_texts, const char* const* parameters_texts,
                          const char* scheme, int device, coral_ensemble** out);
void coral_ensemble_destroy(coral_ensemble* e);
const char* coral_ensemble_last_error(const coral_ensemble* e);
int coral_ensemble_member(coral_ensemble* e, int i, coral_handle** member);
int coral_ensemble_march(coral_ensemble* e, double dt, int nsteps);
int coral_ensemble_synchronize(coral_ensemble* e);
int coral_ensemble_query(coral_ensemble* e, int what, long long* value);

/*
 * Autotuner (no counterpart in the reference): times the kernel variants of the
 * step on this handle's problem at dt -- the FFT plans of the x passes (two or
 * three passes), the forward y pass (persistent pipelined or one CTA per tile),
 * the operator tile kernels (compiled group layouts or run-time forms), the
 * band substitution (compiled or run-time band), the fused z pass (forward
 * batches of 9 or 6 lines), the inverse x pass (persistent pipelined or one
 * CTA per tile), the inverse y pass (single-term build or term loop) and the
 * y-chunked pipeline of a stage's inverse x, z and
 * forward x passes (bands of y rows on three streams, or whole passes; timed
 * over whole steps) -- each over `repeats` eager
 * steps (CUDA events on the handle's stream, best time of the phases it
 * affects), keeps the fastest of each, and restores the state (the tuning steps
 * leave it unchanged).  All variants compute the same arithmetic.  report (may
 * be NULL) receives the timings and choices, at most n bytes.
 */
int coral_autotune(coral_handle* h, double dt, int repeats, char* report, int n);

/*
 * Sets one kernel variant of the autotuner by its knob name ("x_fft_plan",
 * "fwd_y_pass", "operator_tiles", "band_substitution", "z_pass",
 * "inv_x_pass", "inv_y_pass", "y_pipeline"), or of the band factorisation ("band_factor": shared-memory
 * window or in place; refactorises at once when factors exist): value 0 the
 * default, 1 the alternative named in the autotuner's report -- to re-apply an
 * earlier tuning without timing it again.  The variants compute the same
 * arithmetic.  CORAL_EBADARG for an unknown knob or a value other than 0 or 1.
 */
int coral_set_variant(coral_handle* h, const char* knob, int value);

/*
 * Learned subgrid closure (no counterpart in the reference).  A stencil network
 * (5 inputs -- u, v, w, T scaled by in_scale and z' -- at the 27 points of a
 * 3 x 3 x 3 stencil, three tanh layers of 64, 9 outputs) predicts, on a coarse
 * grid, the subgrid part tau_q of every quadratic variable; with a network
 * attached to a handle (coral_closure_attach) every stage adds tau_q to the
 * products before their forward transform, so the subgrid fluxes reach K_hat
 * through the recipe's own NL terms (src/plane_layer/PL_IMEX_timestepping_marching.f90:279-352
 * has only the products).  Weights BF16 with FP32 master copies, FP32
 * accumulation; forward, backward and Adam are CUDA kernels.
 *   train: inputs [nsnap][4][NYAA][NXAA][NZAA] and targets [nsnap][9][...] (float,
 *   device), points (device) = snapshot * NYAA NXAA NZAA + linear grid index;
 *   accumulates the gradient of the mean squared error (targets divided by
 *   out_scale) over the points and, with apply != 0, takes one Adam step
 *   (lr; beta1 = 0.9, beta2 = 0.999, eps = 1e-8) and clears the gradient.
 *   infer: fields = 4 full variables [f][NYAA][NXAA][NZAA] (double, device) ->
 *   tau [9][NYAA][NXAA][NZAA] (double, device), queued on stream.
 */
typedef struct coral_closure coral_closure;
int coral_closure_create(int device, unsigned long long seed, coral_closure** out);
void coral_closure_destroy(coral_closure* c);
const char* coral_closure_last_error(const coral_closure* c);
int coral_closure_param_count(void);
int coral_closure_set_scales(coral_closure* c, const float* in_scale4, const float* out_scale9);
int coral_closure_get_params(coral_closure* c, float* params, int n);
int coral_closure_set_params(coral_closure* c, const float* params, int n);
int coral_closure_get_gradient(coral_closure* c, float* grad, int n);
int coral_closure_zero_gradient(coral_closure* c);
int coral_closure_train(coral_closure* c, const float* inputs, const float* targets, int nsnap, int NXAA, int NYAA,
                        int NZAA, const long long* points, long long npts, float lr, int apply, double* loss);
int coral_closure_infer(coral_closure* c, const double* fields, int NXAA, int NYAA, int NZAA, double* tau,
                        void* stream);
/* Attach a network to a handle (NULL detaches): the full variables must be u, v,
 * w, T (4) and the quadratic variables 9.  The handle does not own the network. */
int coral_closure_attach(coral_handle* h, coral_closure* c);

#ifdef __cplusplus
}
#endif

#endif /* CORAL_B200_H */
