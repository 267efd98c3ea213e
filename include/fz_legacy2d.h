/*
 * fz_legacy2d.h -- C ABI of the 2D legacy scheme (libfz.so).
 *
 * The reference's 2D solver (`2D-solver/`, executable `phases2D`) steps a node grid of
 * Nx x Ny points (i,j at x = i h, y = j h, flat index j*Nx + i; `2D-solver/include/parsing.h:
 * 288-299`) with its own scheme, which differs from the 3D one:
 *   - WENO5 with Jiang-Shu weights alpha_r = d_r / (beta_r + eps)^2
 *     (`2D-solver/core/functions.cuh:1029-1180`; eps = 1e-7, `main.cu:591`);
 *   - Godunov fluxes on the reconstructed states (`functions.cuh:199-213`);
 *   - SSP-RK3 in three stage kernels (`functions.cuh:1182-1390`) over buffers U0, U1, U2, with
 *     U0 <- U1 copied after every step (`main.cu:816-836`);
 *   - a multiplicative "simple" PML, q -= s q after each stage, with cubic ramps over 15 % of the
 *     smaller grid dimension on the faces switched on (`functions.cuh:936-965`);
 *   - zero-gradient copies of p and v into the three ghost rows at the bottom and top after each
 *     stage (`periodic_BC`, `functions.cuh:268-298`); u's ghost rows and the three ghost columns
 *     at each x end are never written;
 *   - the immersed ADE boundary at band cells (oid 1..254) with a bicubic probe at distance
 *     s + h from the wall and the cell centre at (i h, j h) (`functions.cuh:635-783`).
 * The reference runs the ghost-row copy inside the stage kernels from interior rows that other
 * threads of the same launch are still writing, so which values reach the ghost rows depends on
 * thread scheduling there. This library makes it deterministic: the ghost rows of a column get
 * the values its rows 3 (bottom) and Ny-4, Ny-5 (top) hold after the stage update and the PML,
 * before the boundary blend -- what the reference produces whenever the copying threads run after
 * the writers -- and a column is copied only if it has a cell with S >= h (the reference's
 * copying threads are those cells).
 *
 * Status codes, precision modes and error handling are those of fz.h. One CUDA stream per
 * handle; every wait is bounded.
 */
#ifndef FZ_LEGACY2D_H
#define FZ_LEGACY2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fz_l2d fz_l2d;

/* Scalar set-up of `2D-solver/core/main.cu:53-82, 386-404, 591`. */
typedef struct {
  int Nx, Ny;        /* node grid including the 3 ghost rows/columns at each end (>= 10 each) */
  double h;          /* grid spacing [m] (config line 1) */
  double dt;         /* time step [s]: C_CFL h / c in the reference (main.cu:392) */
  double rho, c;     /* air density, speed of sound (main.cu:384-386; T in kelvin) */
  double eps;        /* WENO-JS epsilon, 1e-7 */
  double tol;        /* band width: 3 h (main.cu:82) */
  int pml_n, pml_s, pml_e, pml_w; /* sPML faces y-high, y-low, x-high, x-low (config lines 7-10) */
  int precision;     /* FZ_FP32 (every array FP32, as the reference) or FZ_FP64 */
  int device;        /* CUDA device ordinal */
} fz_l2d_params;

/* Defaults, as the reference computes them in float: h = 0.005, c = sqrt(1.4 * 287.05 * (22 +
 * 273.15)) = 344.40, rho = 1.225, dt = 0.2 h / c, eps = 1e-7, tol = 3 h; sPML on the y faces only
 * (the shipped 2D-solver/config/config.txt); FZ_FP32; device 0. The grid size is left 0 and must
 * be set. */
void fz_l2d_params_init(fz_l2d_params* p);

int fz_l2d_create(const fz_l2d_params* p, fz_l2d** out);
int fz_l2d_destroy(fz_l2d* h);

/* Signed distances S (float, > 0 in the fluid) and object ids oid (1..nmat at band cells, 0 or 255
 * elsewhere) of the node grid: the arrays the reference writes to output/S.bin and output/oid.bin
 * (main.cu:104-134). Builds the band list in raster order (common/filterABC.h:95-108). Like
 * fz_l2d_set_materials, it resets the solve to zero fields at step 0: set the fields after both. */
int fz_l2d_load_geometry(fz_l2d* h, const float* S, const uint8_t* oid);

/* ADE coefficients of nmat (1..254) materials with K real and L complex pole pairs each
 * (zero-padded, material-major: A[m*K + k]; common/filterABC.h:31-90, main.cu:231-295);
 * 0 <= K, L <= 64. */
int fz_l2d_set_materials(fz_l2d* h, int nmat, int K, int L, const double* Rinf, const double* A,
                         const double* zeta, const double* B, const double* C, const double* alpha,
                         const double* beta);

/* Starts the solve over from the given fields at t = 0 (each Nx*Ny; NULL = zeros): U0 gets them
 * at every node, ghost nodes included, U1, U2 and the ADE states are zero, the step count and the
 * recorded trace restart (main.cu:455-473, 595-620). The reference's raised-cosine plane wave is
 * one such set of fields. */
int fz_l2d_set_fields(fz_l2d* h, const double* p, const double* u, const double* v);

/* The receiver node (i,j) with 3 <= i < Nx-3, 3 <= j < Ny-3, and the number of samples to keep:
 * p at that node after every step (main.cu:478-499, 846). The trace restarts here. */
int fz_l2d_set_receiver(fz_l2d* h, int i, int j, int64_t nsamples);

/* Enqueues nsteps steps (3 launches each, replayed from CUDA graphs) and waits for them with a
 * bounded poll. Replaces the WENO/SSP-RK3 loop of main.cu:795-858. */
int fz_l2d_run(fz_l2d* h, int64_t nsteps);

/* fz_l2d_run, and the device time of its launches in *ms (CUDA events on the handle's stream). */
int fz_l2d_run_timed(fz_l2d* h, int64_t nsteps, double* ms);

int64_t fz_l2d_step_count(const fz_l2d* h);

/* Receiver samples recorded since the last fz_l2d_set_receiver / fz_l2d_set_fields (at most the
 * number asked for in fz_l2d_set_receiver). */
int64_t fz_l2d_samples(const fz_l2d* h);

/* The first n recorded receiver samples (n <= fz_l2d_samples). */
int fz_l2d_get_ir(fz_l2d* h, double* out, int64_t n);

/* The current fields (U0 after the last step; each Nx*Ny; NULL skips a field). */
int fz_l2d_get_fields(fz_l2d* h, double* p, double* u, double* v);

/* Number of band cells of the loaded geometry. */
int64_t fz_l2d_band_cells(const fz_l2d* h);

int fz_l2d_last_error(const fz_l2d* h, char* buf, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* FZ_LEGACY2D_H */
