/*
 * fz.h -- C ABI of the B200-native FASES time-domain stepper (libfz.so).
 *
 * The reference solver (vitorotri/fases, F.A.S.E.S v0.9) has no library or plugin API: its
 * boundary is the process contract of the `fases3D` executable (argv + project files + stdout),
 * driven by `common/gui.py` through `subprocess.Popen`. This header is the function-level form
 * of that contract. Every entry point below names the piece of `fases3D` it replaces
 * (paths relative to the reference project root).
 *
 * Conventions
 *   - Every function returns an int status: FZ_OK (0) or a negative FZ_E* code. Nothing in the
 *     library calls exit(); the reference calls std::exit inside read_fit_file
 *     (common/filterABC.h:24-29,44-48). The text of the last error is returned by
 *     fz_last_error() (per handle) or fz_global_error() (for calls without a handle).
 *   - Host arrays are owned by the caller and copied on entry; fz_get_* copy into caller buffers.
 *     No device pointer ever escapes the library.
 *   - Grid arrays passed across the ABI use the reference layout: cell (i,j,k) at
 *     i + Nx*(j + Ny*k), x fastest (3D-solver/core/functions3D.cuh:48-50). The device layout is
 *     private (rows padded and aligned to 128 bytes).
 *   - One CUDA stream per handle. A handle is not thread-safe; distinct handles may run
 *     concurrently on one GPU. Only fz_sync and fz_get_* wait for the device, and every wait is
 *     a bounded poll that returns FZ_ETIMEOUT instead of hanging.
 */
#ifndef FZ_H
#define FZ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FZ_ABI_VERSION 2

/* status codes */
#define FZ_OK 0
#define FZ_EINVAL -1       /* bad argument */
#define FZ_ENOMEM -2       /* host or device allocation failed */
#define FZ_ECUDA -3        /* CUDA runtime error (text in fz_last_error) */
#define FZ_EIO -4          /* file could not be opened, read or written */
#define FZ_EPARSE -5       /* malformed config / .fit / poles / src / rec file */
#define FZ_ESTATE -6       /* call out of order (e.g. fz_run before geometry) */
#define FZ_ETIMEOUT -7     /* a bounded device wait gave up */
#define FZ_ENONFINITE -8   /* health check found NaN/Inf in the state */
#define FZ_ENODEV -9       /* no usable CUDA device */
#define FZ_EBOUNDS -10     /* the bounds-checked build (libfz_checked.so) caught an out-of-range index */

/* precision modes */
#define FZ_FP32 0  /* FP32 field state; FP64 ADE state, receiver samples and energy (default) */
#define FZ_FP64 1  /* every field and state in FP64 */

/* source waveform types: config.txt line 16 (3D-solver/core/main3D.cu:968) */
#define FZ_SRC_PCS 0
#define FZ_SRC_RICKER 1
#define FZ_SRC_SINE 2

typedef struct fz_handle fz_handle;

/* Solver parameters. Replaces the scalar part of main3D.cu's setup:
 * h = config[0] (main3D.cu:132); c, rho (454-456); dt = CFL*h/c (729-730);
 * PML keys U D R L F B = config[6..11] (155-160); PML_CELLS (functions3D.cuh:12-14);
 * tol = 3h (main3D.cu:224). */
typedef struct fz_params {
  int32_t abi_version; /* must be FZ_ABI_VERSION */
  int32_t precision;   /* FZ_FP32 or FZ_FP64 */
  int32_t device;      /* CUDA device ordinal */
  int32_t pml_cells;   /* cPML thickness in cells (reference: 20) */
  int32_t pml[6];      /* face flags in reference order U,D,R,L,F,B = z-hi,z-lo,x-hi,x-lo,y-hi,y-lo */
  double h;            /* grid spacing [m] */
  double c;            /* speed of sound [m/s] */
  double rho;          /* air density [kg/m^3] */
  double dt;           /* time step [s] */
  double tol_cells;    /* immersed blending band in cells: tol = tol_cells*h (reference: 3) */
  int32_t two_d;       /* 1: planar solve -- the grid has exactly one updated z-plane (Nz = 7 with
                          the ghost cells), no z fluxes and no z cPML; the 3D scheme restricted to
                          2D (config 1 of the benchmarks). 0: 3D. */
  int32_t batch;       /* independent field sets stepped together (0 or 1: one). Members share the
                          geometry, materials, cPML faces and receiver cells; each has its own
                          fields, ADE and cPML states and its own sources (fz_set_source_members).
                          Replaces the one-process-per-source runs of the auralization mode
                          (main3D.cu:1278, driven per source by common/gui.py). Host-side arrays of
                          fz_set_fields / fz_get_fields hold batch grids one after another; receiver
                          traces are [batch][n_rec][n_steps]. */
  /* cPML profile (functions3D.cuh:689-723; the reference's constants are the defaults):
   * sigma = (m+1) c ln(1/R0) / (2 d h) x^m, kappa = 1 + (kappa_max - 1) x^m,
   * alpha = alpha_max (0.1 + 0.9 (1 - x)), x = depth / d, m = pml_order. */
  double pml_R0;        /* target reflection (1e-7) */
  double pml_kappa_max; /* (5) */
  double pml_alpha_max; /* (20 pi) */
  double pml_order;     /* m (2) */
} fz_params;

/* Fills p with the reference defaults: FP32, device 0, 20 PML cells, no PML faces, h = 0.02,
 * T = 20 degC -> c = sqrt(1.4*287.05*293.15), rho = 1.225, CFL 0.5, tol = 3h, cPML R0 = 1e-7,
 * kappa_max = 5, alpha_max = 20 pi, order 2. */
int fz_params_init(fz_params* p);

/* Creates a solver on p->device. Replaces main3D.cu:235-293 (device probe) and the allocation
 * block 755-843. Device memory is allocated later, by fz_load_geometry_raw. */
int fz_create(const fz_params* p, fz_handle** out);
void fz_destroy(fz_handle* h);

/* Immersed geometry, as the reference caches it in output/S.bin (float32 signed distance, positive
 * in air) and output/oid.bin (uint8 material id, 0xFF = none) (main3D.cu:350-364, 410-421).
 * Nx,Ny,Nz are the padded grid (room + 3 ghost cells per side, parsing3D.h:128).
 * Builds the cell-class bytes, the compact band list in build_boundary_map order
 * (common/filterABC.h:95-108) with its precomputed probe geometry
 * (functions3D.cuh:483-512), and zeroes all fields (main3D.cu:755-802). */
int fz_load_geometry_raw(fz_handle* h, const float* S, const uint8_t* oid, int32_t Nx, int32_t Ny,
                         int32_t Nz);

/* Free and total device memory of a CUDA device (the --estimate pre-flight, main3D.cu:505-525). */
int fz_device_memory(int32_t device, int64_t* free_bytes, int64_t* total_bytes);

/* Scene geometry from an OBJ file (replaces parse_obj3d + build_sdf + build_oid_dense,
 * 3D-solver/include/parsing3D.h:150-288, 389-452, 574-661, 815-1154, run by main3D.cu:300-428):
 * fz_scene_dims gives the padded grid (mesh shifted so its minimum corner sits at 3h; domain
 * [0, max + 3h]; N = ceil(L/h) per axis) and the domain size L (may be NULL), host only.
 * fz_build_scene fills S (float32 signed distance, positive in air, exact within 8h of the
 * surface and +-8h beyond) and oid (material id = OBJ group index + 1 in order of first face,
 * for band cells 0 <= S <= tol_cells*h; 0xFF elsewhere) in the reference layout, computed on
 * `device`; cap = cells available in each array. These are the arrays fz_load_geometry_raw takes
 * and the reference caches in output/S.bin and output/oid.bin. */
int fz_scene_dims(const char* obj_path, double h, int32_t* dims, double* L);
int fz_build_scene(const char* obj_path, double h, double tol_cells, int32_t device, float* S, uint8_t* oid,
                   int64_t cap);

/* ADE materials. Replaces read_fit_file per layer (common/filterABC.h:31-90) plus the device
 * copies (main3D.cu:639-658). Arrays use the reference's flat(k, m, K) = m*K + k layout:
 * Rinf[nMat], A/zeta[nMat*K], B/C/alpha/beta[nMat*L]. Material m is oid m+1. */
int fz_set_materials(fz_handle* h, int32_t nMat, int32_t K, int32_t L, const double* Rinf,
                     const double* A, const double* zeta, const double* B, const double* C,
                     const double* alpha, const double* beta);

/* Point sources. cell_ijk[3*n] are grid cells ((int)(x/h)+3 per axis, main3D.cu:874-876);
 * sval[n] the scaled source strengths (main3D.cu:1071-1110); u_s[n_us] the shared waveform at
 * dt/2 spacing (length >= 2*Nt+1, main3D.cu:963-1124); for FZ_SRC_SINE freq[n] are per-source
 * frequencies and u_s may be NULL. Replaces kernel_inject_src_SSP (functions3D.cuh:1039-1047). */
int fz_set_sources(fz_handle* h, int32_t n, const int32_t* cell_ijk, const double* sval,
                   int32_t src_opt, const double* freq, const double* u_s, int64_t n_us);

/* Batched solves (fz_params.batch > 1): member[n] assigns each source of the last fz_set_sources
 * call to one member (0 .. batch-1), or to every member (-1, the default). No counterpart in the
 * reference, which runs one process per source position. */
int fz_set_source_members(fz_handle* h, int32_t n, const int32_t* member);

/* Receivers at grid cells cell_ijk[3*n] ((int)(x/h)+3, main3D.cu:938-940). Samples p and
 * (u,v,w) after every step into a device buffer of capacity_steps samples per receiver
 * (replaces the per-step cudaMemcpy at main3D.cu:1399-1414). */
int fz_set_receivers(fz_handle* h, int32_t n, const int32_t* cell_ijk, int64_t capacity_steps);

/* Animation slices (main3D.cu:1152-1237, 1326-1394): after every step whose index is a multiple of
 * anim_step (the first step included), the pressure on the planes x = i0, y = j0, z = k0 and the
 * in-plane components of the unit energy-flow direction sign(p) u/|u| are stored in device memory,
 * up to max_frames frames (0 turns slicing off). Set before the first step, single-member solves.
 * fz_get_slices copies the frames taken so far (*frames = their count; out may be NULL to ask):
 * per frame pX[Ny*Nz] pY[Nx*Nz] pZ[Nx*Ny] IyX IzX IxY IzY IxZ IyZ, each plane in the reference's
 * order (j + Ny*k, i + Nx*k, i + Nx*j); fz_write_outputs writes them as pressure{X,Y,Z}.bin and
 * I{y,z}_X.bin, I{x,z}_Y.bin, I{x,y}_Z.bin with the frame count in header.txt. */
int fz_set_slices(fz_handle* h, int32_t i0, int32_t j0, int32_t k0, int64_t anim_step, int64_t max_frames);
int fz_get_slices(fz_handle* h, float* out, int64_t cap, int64_t* frames);

/* Initial fields in the reference layout (any pointer may be NULL = zero). The reference always
 * starts quiescent (main3D.cu:1134-1135); this is the Gaussian-pulse initial condition of the
 * synthetic benchmarks and the hook the tests use. A new initial state: the other two field
 * sets and the ADE and cPML auxiliary states are zeroed and the health word cleared (the step
 * counter and the receiver traces recorded so far are kept). */
int fz_set_fields(fz_handle* h, const double* p, const double* u, const double* v, const double* w);

/* Enqueues nsteps SSP-RK3 steps on the handle's stream and returns. One step is the reference
 * time-loop body main3D.cu:1280-1319 + 1399-1414: three fused stage kernels (WENO-Z, Godunov
 * flux, RK combination, cPML, source), each followed by the immersed ADE band update, then the
 * receiver gather. */
int fz_run(fz_handle* h, int64_t nsteps);

/* fz_run bracketed by CUDA events on the handle's stream, followed by a bounded wait; *ms gets
 * the device time of the nsteps steps. */
int fz_run_timed(fz_handle* h, int64_t nsteps, double* ms);

/* Finalises the set-up (band list, cPML tables, TMA descriptors) and instantiates the CUDA graphs
 * fz_run launches (one per buffer parity) without running a step, then waits; the first fz_run
 * after it launches graphs only. fz_autotune and fz_set_z_schedule discard the graphs, so call it
 * after them. No counterpart in the reference, which launches every kernel of every step from the
 * host (main3D.cu:1280-1319). */
int fz_prepare(fz_handle* h);

/* Progress protocol: fz_run in slices of every_percent % of nsteps (the reference prints "NN%"
 * every 5 %, functions3D.cuh:1431-1439, parsed by common/gui.py:6713), a bounded wait after each
 * slice, then cb(steps_done_in_this_call, nsteps, user) on the calling thread (cb may be NULL).
 * A nonzero return from cb stops the run after that slice (returns FZ_OK). */
typedef int (*fz_progress_fn)(int64_t done, int64_t total, void* user);
int fz_run_progress(fz_handle* h, int64_t nsteps, int32_t every_percent, fz_progress_fn cb, void* user);

/* Bounded wait for all enqueued work (timeout_ms <= 0: 600000 ms). */
int fz_sync(fz_handle* h, int64_t timeout_ms);

/* Checkpoint / resume (no counterpart in the reference, whose time loop cannot be resumed): the
 * complete state of a solver -- all three field sets, the ADE states, the cPML psi tiles, the step
 * counter, the receiver traces so far and the animation frames -- copied into a caller-owned host
 * buffer of fz_state_bytes bytes, and back. Loading needs a solver set up the same way (geometry,
 * precision, batch, materials' pole counts, receivers and capacity, cPML faces and thickness,
 * slices) and with the same physics (h, c, rho, dt, blending band, cPML profile, geometry values,
 * material coefficients and sources, compared through a hash saved with the state); the run then
 * continues exactly as the saved one would have (same results bit for bit). */
int fz_state_bytes(fz_handle* h, int64_t* bytes);
int fz_state_save(fz_handle* h, void* buf, int64_t cap);
int fz_state_load(fz_handle* h, const void* buf, int64_t len);

/* Health of the current state (no counterpart in the reference, which never checks its fields):
 * counts NaN/Inf values over every field of the state into *nonfinite (may be NULL) and returns
 * FZ_ENONFINITE if there are any. Independently of this call, every step's receiver gather flags a
 * non-finite sample in the device error word, which the next fz_sync (and every call that waits)
 * reports as FZ_ENONFINITE; fz_set_fields starts a new state and clears the word. */
int fz_check_health(fz_handle* h, int64_t* nonfinite);

/* Steps completed so far (after fz_sync). */
int fz_steps_done(fz_handle* h, int64_t* n);

/* Groups: several handles (rooms) on one device advanced together. fz_group_run enqueues nsteps
 * steps of every member. When every member is a 3D room of the group's precision without animation
 * slices and there are at most 64 of them, the members share their launches: per stage one band
 * launch over all members and one stage launch per 28 members (their CTAs laid end to end, each CTA
 * reading its room's arguments from a table in device memory; the rooms' TMA descriptors travel as
 * kernel parameters), then one receiver launch, whatever the member count; otherwise each member's
 * own launches run as parallel branches. Runs of 10
 * steps are CUDA graphs either way. Members keep their own state and stay usable alone (fz_get_ir,
 * fz_sync, fz_run); they must all be on one device, must outlive the group, and are finalised
 * (materials, sources, receivers fixed) by fz_group_create. Results are those of each member run
 * alone, bit for bit. No counterpart in the reference (one process per room). */
typedef struct fz_group fz_group;
int fz_group_create(fz_handle* const* members, int32_t n, fz_group** out);
int fz_group_run(fz_group* g, int64_t nsteps);
/* fz_group_run bracketed by CUDA events on the group's stream, then a bounded wait. */
int fz_group_run_timed(fz_group* g, int64_t nsteps, double* ms);
int fz_group_sync(fz_group* g, int64_t timeout_ms);
void fz_group_destroy(fz_group* g);
/* *shared = 1 when the group steps its members with shared launches (above), 0 when each
 * member's own launches run as graph branches; *branches (may be NULL) gets the number of
 * concurrent branches: shared launches run as branches of rooms of about equal cells (one stream
 * each), so that one branch's band and receiver launches overlap another's stage launches. */
int fz_group_info(fz_group* g, int32_t* shared, int32_t* branches);
/* Sets the launch arrangement: branches >= 1: shared launches in that many concurrent branches (at
 * most min(n, 16)); -1: each member's own launches as graph branches; 0: the default (shared
 * launches in 4 branches for 16 rooms or more, 2 for 4 or more, else 1, where the members can share
 * launches). fz_group_autotune times the arrangements with the tile depths and keeps the fastest.
 * Results do not depend on it. */
int fz_group_set_branches(fz_group* g, int32_t branches);

/* Launch-shape autotuner. A stage-kernel CTA covers 32 x 16 columns by one z chunk of planes;
 * the chunk lengths set how many CTAs a stage launches and how whole waves of SMs fill. fz_autotune
 * times the three stage kernels on this room for the heuristic depth, up to eight other uniform
 * depths and (single rooms) guided schedules -- long chunks first, short ones for the last waves --
 * (reps steps' worth each, after one warm-up) and keeps the fastest; the state is left as it was
 * (the call does not advance the solve). kz_chunk gets the chosen (longest) chunk, ms_per_step the
 * stage kernels' time per step; fz_get_z_schedule lists the chunks. fz_group_autotune does the
 * same for all members at once, timing their kernels side by side with one uniform depth for every
 * member (clamped to each room; 0 = each member's heuristic). Results do not depend on the depth (each CTA recomputes its boundary centres).
 * The reference launches fixed TP(32,4,4) blocks (main3D.cu:1280-1306). */
int fz_autotune(fz_handle* h, int32_t reps, int32_t* kz_chunk, double* ms_per_step);
int fz_group_autotune(fz_group* g, int32_t reps, int32_t* kz_chunk, double* ms_per_step);
/* Sets the depth directly (0 = the heuristic), e.g. from a cache of earlier tuning results. */
int fz_set_kz_chunk(fz_handle* h, int32_t kz_chunk);
int fz_get_kz_chunk(fz_handle* h, int32_t* kz_chunk, int32_t* heuristic);
/* The z chunks the stage kernels use now (lengths in planes, longest first; the tuner may pick a
 * guided schedule: long chunks first, short ones for the last waves). n gets their number; at most
 * cap lengths are written to sizes (may be NULL). */
int fz_get_z_schedule(fz_handle* h, int32_t* sizes, int32_t cap, int32_t* n);
/* Sets the z chunks directly (n lengths >= 1 summing to the interior planes Nz - 6, n <= 256),
 * e.g. a schedule fz_get_z_schedule reported for this room before. */
int fz_set_z_schedule(fz_handle* h, const int32_t* sizes, int32_t n);

/* Gradient of the receiver misfit J = sum_r sum_{n < nsteps} (IR_r[n] - target[r][n])^2 (IR_r[n] = p
 * at receiver r after step n+1, FP64) with respect to every ADE coefficient of every material, by
 * the discrete adjoint of the stepping scheme (WENO-Z weights linearised, Godunov flux, RK stages,
 * cPML, immersed band and ADE recursion). Runs nsteps forward from the handle's current state
 * (which must be at step 0; cells no kernel writes are first set to zero in every field set),
 * saving a checkpoint every segment_steps steps, then recomputes each segment while storing its
 * stage states and sweeps it backwards. target is [n_rec][target_steps] (target_steps >= nsteps).
 * grad gets [nMat][1 + 2K + 4L] = Rinf, A[K], zeta[K], B[L], C[L], alpha[L], beta[L] per material,
 * in the layout of fz_set_materials (K, L as fz_material_layout reports them). ms[2] (may be
 * NULL) gets the device time of the forward pass and of the backward pass. On return the handle
 * holds the state after nsteps and the forward receiver traces. Device memory: about
 * (nsteps/segment_steps + 1) states + segment_steps x 3 field sets + 50 field arrays; FZ_ENOMEM
 * (nothing allocated) when it does not fit. 3D, batch 1, sources in updated cells only. No
 * counterpart in the reference (its material fit, common/fminconFIT.py:239-348, works on octave
 * absorption and never differentiates the solver). */
int fz_misfit_gradient(fz_handle* h, int64_t nsteps, int32_t segment_steps, const double* target,
                       int64_t target_steps, double* J, double* grad, int64_t grad_cap, double* ms);

/* Outputs of fz_misfit_gradient_ex; every pointer may be NULL (not computed), each *_cap is its
 * element count and must hold the size given. */
typedef struct fz_gradients {
  int32_t cotangent;     /* 0: J = sum (IR - target)^2 as fz_misfit_gradient. 1: target holds a
                            cotangent g[r][n] of the receiver traces; J = sum g IR and every
                            gradient is the vector-Jacobian product sum g dIR/dtheta */
  double* materials;     /* [nMat][1 + 2K + 4L], as fz_misfit_gradient's grad */
  int64_t materials_cap;
  double* source_sval;   /* [nsrc]: d J / d sval[q] (fz_set_sources' source strengths) */
  int64_t source_sval_cap;
  double* source_wave;   /* [nsrc][n_us]: d J / d u_s[nn] through source q (PCS / Ricker waveforms;
                            summing over q gives the gradient of the shared waveform) */
  int64_t source_wave_cap;
  double* pml;           /* [4]: d J / d (pml_R0, pml_kappa_max, pml_alpha_max) and 0 for pml_order */
  int64_t pml_cap;
  double* initial;       /* [4][Nx*Ny*Nz]: d J / d (p, u, v, w) of the step-0 state in the reference
                            layout; 0 at cells no kernel writes (solid interior) */
  int64_t initial_cap;
} fz_gradients;

/* fz_misfit_gradient with the gradients of fz_gradients: the ADE coefficients, the source
 * strengths and waveform samples, the cPML profile parameters and the initial fields, from one
 * forward pass with checkpoints and one reverse sweep. Same conditions, schedule and memory as
 * fz_misfit_gradient, plus one psi-tile set per segment step when the cPML gradient is asked for. */
int fz_misfit_gradient_ex(fz_handle* h, int64_t nsteps, int32_t segment_steps, const double* target,
                          int64_t target_steps, double* J, fz_gradients* out, double* ms);

/* Material table layout after setup: number of materials (>= 1) and the real-pole / complex-pair
 * counts K, L (each >= 1, zero-padded as read_fit_file pads, common/filterABC.h:52-89). */
int fz_material_layout(fz_handle* h, int32_t* nMat, int32_t* K, int32_t* L);

/* Receiver traces [n_rec][n_steps] (float32, as IR<r>_<s>.bin, main3D.cu:1403-1404) and
 * [n_rec][n_steps][3] velocities (as VEL<r>_<s>.bin, main3D.cu:1408-1412). cap = elements. */
int fz_get_ir(fz_handle* h, float* out, int64_t cap);
int fz_get_ir64(fz_handle* h, double* out, int64_t cap);
int fz_get_vel(fz_handle* h, float* out, int64_t cap);

/* Current state (the reference's U0 after the swap, main3D.cu:1312-1315), reference layout. */
int fz_get_fields(fz_handle* h, double* p, double* u, double* v, double* w);

/* FP64 acoustic energy 0.5*sum(p^2/(rho c^2) + rho |u|^2) * h^3 over the grid (the unused
 * host diagnostic functions3D.cuh:111-129, evaluated on the device in FP64). */
int fz_energy(fz_handle* h, double* E);

/* Writes output_dir/IR<r>_<src_idx>.bin and VEL<r>_<src_idx>.bin (main3D.cu:1251-1256) and
 * output_dir/header.txt (main3D.cu:1441-1449) from the samples taken so far. */
int fz_write_outputs(fz_handle* h, const char* output_dir, int32_t src_idx, const char* scene_name);

/* Grid and band facts: dims[3], n_band, n_update (cells the stage kernels write). */
int fz_info(fz_handle* h, int32_t* dims, int64_t* n_band, int64_t* n_update);

/* Per-kernel-kind device time. When enabled, every launch in fz_run is bracketed by CUDA events
 * on the handle's stream; fz_profile_read returns accumulated milliseconds and launch counts for
 * kinds 0..2 = stage kernels 0,1,2; 3 = band kernels; 4 = receiver gather. */
int fz_profile_enable(fz_handle* h, int32_t on);
int fz_profile_read(fz_handle* h, double* ms, int64_t* launches, int32_t nkinds);

/* Whole reference project: config/config.txt, config/poles.txt, input/fit/<layer>.fit,
 * src.txt, rec.txt (main3D.cu:66-160, 587-634, 861-959) with the geometry from the reference's
 * scene cache output/S.bin + output/oid.bin + output/scene_cache.txt (main3D.cu:334-380).
 * Creates the handle, loads geometry, materials, sources (with the PCS/Ricker/sine waveform and
 * its scaling, main3D.cu:963-1124), receivers, and writes config/p_ref.bin (main3D.cu:1096-1108)
 * and output/pre_header.txt (main3D.cu:527-532). n_steps_out receives Nt (main3D.cu:752). */
int fz_load_project(const char* scene_path, const char* config_path, const char* src_path,
                    const char* rec_path, int32_t precision, int32_t device, fz_handle** out,
                    int64_t* n_steps_out);

/* Source waveform exactly as main3D.cu:963-1124 computes it: u_s[0..2Nt] (double) for
 * src_opt PCS or Ricker, and the radiated reference pulse p_ref[0..2Nt] per unit source
 * (main3D.cu:1084-1090) with its peak. */
int fz_source_waveform(int32_t src_opt, double glob_f, double f_cutoff, double dt, int64_t Nt,
                       double h, double rho, double* u_s, double* p_ref, double* p_peak);

int fz_last_error(fz_handle* h, char* buf, size_t cap);
int fz_global_error(char* buf, size_t cap);

/* Allocation-free energy of caller-owned FP32 device fields. No counterpart in the reference.
 *
 * For callers that cannot allocate device memory (their fields live in a pool they manage, or
 * they run where a cudaMalloc -- which may synchronise the device -- is not allowed). The caller
 * passes device arrays p, u, v, w of n elements each and a device slot *out; the function
 * enqueues two kernels on `stream` (a cudaStream_t, NULL = default stream) that write
 * 0.5 * sum(p^2/(rho c^2) + rho |u|^2), accumulated in FP64, to *out, and returns without
 * waiting. It calls no cudaMalloc/cudaFree: its scratch is a fixed device array of
 * FZ_NOALLOC_MAX_BLOCKS doubles (32 KB) in the library, held by every GPU that loads it until
 * the process exits. n may be at most FZ_NOALLOC_MAX_CELLS; larger n returns FZ_EINVAL.
 * The first call on a device looks up that array's device address (with the device current),
 * and looks it up again when the device's context has been re-created (cudaDeviceReset);
 * make that first call before any stream capture. All calls share the array: calls that overlap
 * on the GPU race and give wrong results; order them (one stream, or events). */
#define FZ_NOALLOC_MAX_BLOCKS 4096
#define FZ_NOALLOC_MAX_CELLS (4096LL * 16384LL)
int fz_energy_noalloc(const float* p, const float* u, const float* v, const float* w, int64_t n, double rho,
                      double c, double* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FZ_H */
