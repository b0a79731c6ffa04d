/*
 * phipict_b200 C ABI: the B200 (sm_100a) PISO/MHD step behind phiPICT's backend
 * protocol. Every entry point takes plain pointers and sizes, launches on the given
 * CUDA stream, never synchronises the device and returns 0 on success or a negative
 * phb_status code. No torch type crosses this boundary.
 *
 * Each declaration names the phiPICT binding it replaces (csrc/phipict/bindings.cpp
 * and the kernel it wraps). The Python mirror of the reference API lives in
 * phipict_b200/_C.py; phipict_b200/_lib.py binds this header with ctypes.
 *
 * Data layout (all device memory):
 *   - cells of all instances are concatenated: instance i owns cells
 *     [insts[i].cellOff, insts[i].cellOff + insts[i].ncells), blocks x-fastest inside;
 *     a batch of B environments of one domain is B instances, so scalar fields are
 *     [B][ncells] and vector fields [B][dims][ncells], as in phiPICT.
 *   - matrices are stored as stencils: value[slot][cell], slot 0 the diagonal,
 *     slot f+1 the neighbour across face f (-x,+x,-y,+y,-z,+z); prescribed faces hold 0.
 *     CSR (phiPICT's CSRmatrix) is produced on demand by phb_csr_pattern/phb_csr_gather.
 *   - cell metrics are SoA: metrics[k * metric_stride + m], k over {M (d*d), Minv (d*d), det}.
 */
#ifndef PHIPICT_B200_H
#define PHIPICT_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void *phb_stream; /* cudaStream_t */

enum phb_status {
	PHB_OK = 0,
	PHB_ERR_ARG = -1,      /* invalid argument (null pointer, bad size or dtype) */
	PHB_ERR_CUDA = -2,     /* a CUDA runtime call failed; see phb_last_error() */
	PHB_ERR_RANGE = -3,    /* a size exceeds a documented maximum */
	PHB_ERR_STATE = -4     /* an object was used before it was initialised */
};

enum phb_dtype { PHB_F32 = 0, PHB_F64 = 1 };

/* record sizes (int32 words) */
#define PHB_BREC 48   /* block record  */
#define PHB_FREC 16   /* fixed-face record */
#define PHB_IREC 8    /* instance record */
#define PHB_TILE 256  /* threads per CTA of the per-cell kernels */
#define PHB_TILE_CELLS 1024 /* cells per tile: one CTA, 4 cells per thread */

/* Domain descriptor: device pointers produced by Domain.PrepareSolve(). It plays the
 * part of phiPICT's DomainGPU/BlockGPU atlas (domain/domain_structs_gpu.h:168-447). */
typedef struct phb_domain {
	int32_t dims;           /* 2 or 3 */
	int32_t dtype;          /* phb_dtype of fields and metrics */
	int32_t nblocks, ninst, ntiles, nfixed;
	int64_t ncells;         /* cells of all instances */
	int64_t metric_stride;  /* cells in the metric array */
	int64_t face_metric_stride;
	const int32_t *blocks;  /* [nblocks][PHB_BREC] */
	const int32_t *tiles;   /* [ntiles][2] = (block, first local cell), PHB_TILE_CELLS cells each */
	const int32_t *fixed;   /* [nfixed][PHB_FREC] */
	const int32_t *insts;   /* [ninst][PHB_IREC] */
	const void *metrics;    /* [2d^2+1][metric_stride] */
	const void *face_metrics; /* [2d^2+1][face_metric_stride] */
	const void *fvel;       /* fixed-face velocities */
	const void *fpot;       /* fixed-face potential values */
	const void *fcw;        /* [nfixed] wall conductance ratio */
	const int8_t *fmask;    /* fixed-face potential BC masks */
	const double *dt;       /* [ninst] time step */
	const double *nu;       /* [ninst] viscosity */
	int32_t scheme;         /* advection scheme (AdvectionScheme): 0 CENTRAL, 1 LINEAR_UPWIND */
	int32_t nonortho;       /* non-orthogonal flag bits (PHB_NON_ORTHO_*) of the matrix and
	                           right-hand-side builders; 0 assembles the orthogonal terms only */
} phb_domain;

const char *phb_last_error(void);
int phb_version(void);

/* --- grid metrics ------------------------------------------------------------------
 * Replaces CoordsToTransforms / CoordsToFaceTransforms (grid/grid_gen.cu:299-396,
 * 398-496, bound through Block::setVertexCoordinates, domain/block.cpp:1005-1010).
 * coords: [dims][vz][vy][vx] vertices of one block. cell_out: SoA metric slice of the
 * block (stride metric_stride); face_out: SoA metrics of the cells of one face. */
int phb_cell_metrics(int dims, int dtype, int nx, int ny, int nz, const void *coords,
                     void *cell_out, int64_t stride, phb_stream stream);
int phb_face_metrics(int dims, int dtype, int nx, int ny, int nz, const void *coords, int face,
                     void *face_out, int64_t stride, phb_stream stream);

/* --- assembly (one launch each, all instances) ------------------------------------- */
/* The advection kernels follow phb_domain.scheme: with LINEAR_UPWIND a face whose downwind
 * and far-upwind cells lie in the same block is first-order upwind in the matrix and gets the
 * linear-upwind part as an explicit correction on the right-hand side (advection.cu:125-144,
 * :892-934); other faces stay central.
 * SetupAdvectionMatrix (bindings.cpp:639, advection.cu:27-305 PISO_build_matrix).
 * u: block velocity [inst][dims][cells]; C: stencil [2d+1][ncells]; Adiag [ncells].
 * C_lo (optional, may be NULL): float32 copy of C for mixed-precision inner solves. */
int phb_advection_matrix(const phb_domain *dom, const void *u, void *C, void *Adiag, float *C_lo, phb_stream stream);
/* SetupAdvectionVelocity (bindings.cpp:645, advection.cu:800-954). src: velocity source,
 * src_mode 0 none, 1 static per instance [inst][dims], 2 per cell [inst][dims][cells]. */
int phb_advection_rhs(const phb_domain *dom, const void *u, const void *src, int src_mode, void *rhs, phb_stream stream);
/* SetupPressureMatrix (pressure.cu:26-191). P: stencil [2d+1][ncells]. */
int phb_pressure_matrix(const phb_domain *dom, const void *Adiag, void *P, float *P_lo, phb_stream stream);
/* SetupPressureRHS (pressure.cu:350-521, then :756-801): HbyA [inst][dims][cells] and its
 * flux divergence div [ncells]. ustar: current velocity iterate (velocityResult). */
int phb_pressure_rhs(const phb_domain *dom, const void *C, const void *Adiag, const void *u, const void *ustar,
                     const void *src, int src_mode, void *hbya, phb_stream stream);
int phb_divergence(const phb_domain *dom, const void *field, void *div, phb_stream stream);
/* CorrectVelocity version 1 (velocity_correction.cu:27-60): u = HbyA - grad(p)/A. */
int phb_correct_velocity(const phb_domain *dom, const void *p, const void *hbya, const void *Adiag, void *u, phb_stream stream);
/* SetupEpotMatrix (mhd/potential.cu:30-233). */
int phb_epot_matrix(const phb_domain *dom, void *E, float *E_lo, phb_stream stream);
/* ComputeEpotRHS (mhd/potential.cu:273-366) fused with u x e_b (simulation/mhd.py:276-355):
 * writes uxb [inst][3][cells] and rhs [ncells]. e_b: [inst][3] (double). */
/* ComputeEpotRHS of a given in-plane field [inst][dims][cells] (bindings.cpp:667-689). */
int phb_epot_rhs(const phb_domain *dom, const void *field, void *rhs, phb_stream stream);
int phb_uxb_epot_rhs(const phb_domain *dom, const void *u, const double *e_b, void *uxb, void *rhs, phb_stream stream);
/* ComputeCurrentDensityFaceBased (mhd/potential.cu:718-916) fused with the Lorentz force
 * of simulation/mhd.py:543-595: J [inst][3][cells]; src[inst][dims][cells] =
 * N (J x e_b)[:dims] + (accumulate ? src : 0). stuart: [inst] (double). */
int phb_current_lorentz(const phb_domain *dom, const void *phi, const void *uxb, const double *e_b,
                        const double *stuart, void *J, void *src, int accumulate, phb_stream stream);

/* --- passive scalar transport ------------------------------------------------------ */
/* Scalar fields are [inst][channels][cells]. Fixed-face data per fixed record r (records as
 * in phb_domain.fixed): types[r * channels + c] (0 Dirichlet value, 1 Neumann gradient
 * dphi/dn) and the value of channel c at face cell fc, values[offsets[r] + c] when
 * statics[r], else values[offsets[r] + c * facecells_r + fc] (domain dtype). The scalar
 * diffusivity is nu[0] (nu_count 1), nu[c] (nu_count = channels), or the velocity viscosity
 * of the instance (nu_count 0, the reference's default without scalarViscosity). */
typedef struct phb_scalar {
	int32_t channels;
	int32_t nu_count;
	const double *nu;
	const int8_t *types;
	const void *values;
	const int64_t *offsets;
	const int8_t *statics;
} phb_scalar;
/* SetupAdvectionMatrix(forPassiveScalar=True, passiveScalarChannel=channel) (bindings.cpp:639,
 * advection.cu:27-305): the advection-diffusion row with the scalar diffusivity of `channel`
 * and its fixed-face types (a Neumann face adds no wall diffusion). Outputs as
 * phb_advection_matrix. */
int phb_scalar_matrix(const phb_domain *dom, const void *u, const phb_scalar *sc, int channel, void *C, void *Adiag,
                      float *C_lo, phb_stream stream);
/* SetupAdvectionScalar (advection.cu:545-698 kPISO_build_scalar_advection_RHS, orthogonal):
 * rhs [inst][channels][cells] from the block scalar phi (same layout); u, the block velocity,
 * gives the face fluxes of the LINEAR_UPWIND correction (may be NULL with CENTRAL). */
int phb_scalar_rhs(const phb_domain *dom, const void *phi, const void *u, const phb_scalar *sc, void *rhs,
                   phb_stream stream);

/* --- non-orthogonal grids ---------------------------------------------------------- */
/* Flag bits of phb_domain.nonortho, the nonOrthoFlags / nonOrthoMode argument of the
 * reference's Setup* calls (piso/non_ortho_flags.h:23-27). With CENTER_MATRIX and
 * DIRECT_MATRIX, phb_advection_matrix, phb_scalar_matrix and phb_pressure_matrix add the
 * cross terms det Minv[n] . Minv[t] of curvilinear grids to the diagonal and the face
 * neighbours (advection.cu:176-240, pressure.cu:103-156; the interpolation of
 * nonortho_laplace.cuh:52-129). DIAGONAL_MATRIX is accepted and, as in the reference, adds
 * nothing. phb_epot_matrix ignores the flags (the potential's own flags default to 0). */
#define PHB_NON_ORTHO_DIRECT_MATRIX 1
#define PHB_NON_ORTHO_DIRECT_RHS 2
#define PHB_NON_ORTHO_DIAGONAL_MATRIX 4
#define PHB_NON_ORTHO_DIAGONAL_RHS 8
#define PHB_NON_ORTHO_CENTER_MATRIX 16
enum { PHB_NONORTHO_VELOCITY = 0, PHB_NONORTHO_SCALAR = 1, PHB_NONORTHO_PRESSURE = 2 };
/* The explicit cross terms of a result field with DIRECT_RHS / DIAGONAL_RHS
 * (nonortho_rhs.cuh:27-180, corner values of block_data.cuh:501-620), applied in place to a
 * right-hand side built by the call named:
 *   PHB_NONORTHO_VELOCITY: field = velocity result [inst][dims][cells]; rhs (phb_advection_rhs)
 *     -= S / det, S weighted with the viscosity (advection.cu:936-937);
 *   PHB_NONORTHO_SCALAR: field = scalar result [inst][channels][cells]; rhs (phb_scalar_rhs)
 *     -= S nu_c / det per channel (advection.cu:684-689); sc as for phb_scalar_rhs;
 *   PHB_NONORTHO_PRESSURE: field = pressure result [ncells]; rhs (the divergence of
 *     phb_divergence) += S weighted with 1/Adiag (pressure.cu:839-860).
 * Does nothing when dom->nonortho has neither right-hand-side bit. */
int phb_nonortho_rhs(const phb_domain *dom, int kind, const void *field, const phb_scalar *sc, const void *Adiag,
                     void *rhs, phb_stream stream);

/* --- diagnostics -------------------------------------------------------------------- */
/* Self-test of the bounded grid-barrier wait of the persistent solvers: a cooperative launch
 * of `ctas` CTAs takes `rounds` grid barriers with a spin limit of `spin_limit` polls
 * (>= 1024). With absent_cta >= 0 that CTA leaves at once, so the other CTAs' waits run out
 * and the launch ends with the barrier error flag set instead of waiting for good (the
 * persistent solvers then leave their systems unconverged). scratch: >= 272 bytes of device
 * memory on a 16-byte boundary. Outputs (host): bar_err (1 when a wait ran out) and
 * rounds_done (barriers CTA 0 passed). Synchronises the stream. */
int phb_barrier_selftest(int ctas, int rounds, int absent_cta, unsigned int spin_limit, void *scratch, int *bar_err,
                         int *rounds_done, phb_stream stream);

/* --- vectors ------------------------------------------------------------------------ */
/* Per-instance reductions use a caller-owned scratch of phb_scratch_doubles() doubles whose
 * first word must be zero before the first call (each call leaves it zero again).
 * subtract_env_mean / _subtract_env_mean (piso_simulation.py:68-89, mhd.py:112-121):
 * x[inst][comps][cells] -= the mean of each instance's component. */
int64_t phb_scratch_doubles(const phb_domain *dom, int comps);
int phb_subtract_mean(const phb_domain *dom, void *x, int comps, double *scratch, phb_stream stream);
/* RMS of each instance's slice of v over all comps (the right-hand-side scale ||b||/sqrt(n)
 * of SolverTolerance, solvers/tolerance.py:116-140); out: [ninst] */
int phb_rms(const phb_domain *dom, const void *v, int comps, double *scratch, double *out, phb_stream stream);

/* --- CSR export (phiPICT CSRmatrix view of a stencil matrix) ----------------------- */
/* Row pointers and columns of the shared pattern of instance 0's geometry, entries sorted
 * by column as PISO_build_matrix writes them; perm[k] = slot*ncells + cell of entry k.
 * row: [ncells+1] (filled on device), col/perm: [nnz]. */
int phb_csr_row_sizes(const phb_domain *dom, int32_t *rowsize, phb_stream stream);
int phb_csr_pattern(const phb_domain *dom, const int32_t *row, int32_t *col, int32_t *perm, phb_stream stream);
int phb_csr_gather(int dtype, int64_t nnz, const int32_t *perm, const void *stencil, void *value, phb_stream stream);

/* --- Krylov solvers (SolveLinear, solvers/linear_solve.cu:22-162 and the fused kernels
 *     of solvers/krylov/krylov.cu:252-1186) ----------------------------------------- */
/* Tolerance of a solve, in the units of the stop test ||r||_2/sqrt(n) < tol.
 * mode 0: the constant atol for every system (phiPICT's plain float tolerance);
 * mode 1: SolverTolerance.resolve (solvers/tolerance.py:180-257) per instance, from the
 *         right-hand side b of the solve: tol = max(rtol*s, atol, floor_eps*s), s =
 *         ||b_inst||_2/sqrt(n_inst*nrhs), and `fallback` when that is 0 (rtol or atol <= 0
 *         means "not given");
 * mode 2: per-system values from `values` [ninst*nrhs]. */
typedef struct phb_tolerance {
	int32_t mode;
	int32_t pad;
	double rtol, atol, floor_eps, fallback;
	const double *values;
} phb_tolerance;

/* --- aggregation multigrid preconditioner -------------------------------------------
 * Replaces phiPICT's AMG hierarchy (solvers/amg.py:450-712 hierarchy_for /
 * galerkin_refresh, built with pyamg on the host) and its device V-cycle
 * (solvers/krylov/krylov.cu:1248-1546, bound as amg_pcg_solve, solvers/amg.py:1544).
 * Every level is a multi-block stencil grid: level l+1 halves each block of level l along
 * every axis longer than one cell (ceil), keeps the block topology, and its operator is the
 * Galerkin product P^T A_l P with piecewise-constant P, times coarse_scale. The coarsest
 * level is solved with a dense generalised inverse per instance (FP64), and the whole cycle
 * below a small level T (at most 1024 cells per instance) is folded into one dense operator
 * C_T = S~ + W C_{T+1} W^T (W = (I - S A) P, S = omega D^-1, S~ = 2S - S A S), so that a
 * cycle reaches level T and applies C_T in one step. The host builds the level descriptors
 * and buffers; phb_amg_setup fills the coarse operators from levels[0].A on the device. One
 * V-cycle: a damped Jacobi sweep from zero, restriction, the coarse cycle, prolongation, a
 * damped Jacobi sweep: symmetric, so it can precondition CG. */
#define PHB_AMG_MAX_LEVELS 12
typedef struct phb_amg_level {
	phb_domain dom;       /* blocks, tiles, insts of the level (level 0: the domain's own) */
	float *A;             /* stencil [2d+1][ncells]; level 0: the float32 system matrix */
	float *b;             /* restricted residual [ncells] (levels >= 1) */
	float *x;             /* correction [ncells] (levels >= 1); level 0: z of phb_amg_vcycle */
	float *wdinv;         /* omega / diagonal [ncells], written by phb_amg_setup */
	int32_t inst_cells;   /* cells of the largest instance on this level */
	int32_t pad;
} phb_amg_level;
typedef struct phb_amg {
	int32_t nlevels;      /* 2..PHB_AMG_MAX_LEVELS */
	int32_t coarse_n;     /* row stride of the coarsest inverses, >= cells of any instance (<= 1024) */
	float omega;          /* damping of the Jacobi sweeps */
	float coarse_scale;   /* factor on every Galerkin product (1: plain Galerkin) */
	int32_t tail_level;   /* T: the cycle below level T is applied as one dense operator per
	                         instance (1..nlevels-1; 0 means nlevels-1: the coarsest inverse) */
	int32_t pad;
	double *coarse_inv;   /* [ninst][coarse_n][coarse_n]: the dense operator of level T,
	                         coarse_n >= levels[T].inst_cells; written by phb_amg_setup */
	double *work;         /* setup scratch of phb_amg_work_doubles() doubles */
	int64_t work_doubles;
	phb_amg_level levels[PHB_AMG_MAX_LEVELS];
} phb_amg;
/* Doubles of setup scratch a hierarchy needs (the dense operators of levels T..nlevels-1). */
int64_t phb_amg_work_doubles(const phb_amg *amg);
/* Galerkin products of levels 1.., dense coarsest operators and their inverses. */
int phb_amg_setup(const phb_amg *amg, phb_stream stream);
/* Only the finest level follows a new level-0 matrix (its smoother omega / diagonal); the coarse
 * operators and dense inverses of the last phb_amg_setup are kept (galerkin_refresh with
 * coarse=False, solvers/amg.py:749, between the full refreshes of coarse_refresh_interval,
 * core/piso_simulation.py:2268-2297). */
int phb_amg_refresh_fine(const phb_amg *amg, phb_stream stream);
/* z = one V-cycle applied to r (both [ncells] of level 0, float32). */
int phb_amg_vcycle(const phb_amg *amg, const float *r, float *z, phb_stream stream);

typedef struct phb_solve {
	int32_t kind;         /* 0 CG, 1 BiCGStab */
	int32_t vec_dtype;    /* phb_dtype of the Krylov vectors */
	int32_t mat_dtype;    /* phb_dtype of the stencil matrix */
	int32_t nrhs;         /* right-hand sides per instance sharing its matrix (1..3) */
	int32_t maxit;
	int32_t return_best;  /* CG only: keep the iterate with the lowest residual */
	int32_t use_graph;    /* 2 (or 3): persistent cooperative kernel; 1: conditional-WHILE CUDA graph; 0: host loop */
	int32_t check_every;  /* host loop only: iterations between completion checks */
	phb_tolerance tol;
	const void *A;        /* stencil [2d+1][ncells] */
	const void *b;        /* [inst][nrhs][cells] */
	void *x;              /* in: initial guess, out: solution */
	void *work;           /* >= phb_solve_work_bytes() bytes, 256-byte aligned */
	void *state;          /* >= phb_solve_state_bytes() bytes */
	const phb_amg *amg;   /* optional (CG, float32, nrhs 1): precondition with one V-cycle of
	                         this hierarchy (set up for A); its level-0 x holds z */
	int32_t ctas_per_sm;  /* persistent kernels (use_graph 2, 3): resident CTAs per SM to launch, at
	                         most what fits; 0: as many as fit (the grid never exceeds the tile count) */
	int32_t pad;
} phb_solve;

/* per-system result, mirrors LinearSolverResultInfo (bindings.cpp:727-732) */
typedef struct phb_solve_result {
	double final_residual;
	int32_t used_iterations;
	int32_t converged;
	int32_t finite;
	int32_t status;       /* 1 converged, 2 non-finite, 3 max iterations, 4 rising */
	int32_t inner_iterations; /* refinement: inner Krylov iterations of all sweeps */
	int32_t pad;
} phb_solve_result;

int64_t phb_solve_work_bytes(const phb_domain *dom, int kind, int vec_dtype, int nrhs);
int64_t phb_solve_state_bytes(const phb_domain *dom, int nrhs);
int phb_solve_run(const phb_domain *dom, const phb_solve *s, phb_stream stream);
/* copies the per-system results to host (synchronises the stream) */
int phb_solve_results(const phb_domain *dom, const phb_solve *s, phb_solve_result *out, phb_stream stream);
/* drops cached solver graphs (ReleaseKrylovWorkspaces, bindings.cpp:775) */
int phb_release_graphs(void);

/* Projected initial guesses (no phiPICT counterpart: phiPICT starts the pressure from zero
 * or its warm start and the potential from its previous result,
 * core/piso_simulation.py:2135 _pressure_initial_guess, simulation/mhd.py:801
 * _epot_initial_guess). phb_stencil_apply: Y[v] = A X[v] for nvec float64 vectors of
 * ncells values, stride >= ncells values apart (a multiple of 4; A, X and Y 32-byte aligned),
 * A a float64 stencil matrix of the domain.
 * phb_projection_solve: alpha = G^-1 c for the m x m (m <= 16, row-major) Gram matrix of a
 * guess basis, Jacobi-scaled with the diagonal raised by reg; rows whose pivot vanishes, or
 * all rows when the result is not finite, get coefficient 0. Both are stream-ordered. */
int phb_stencil_apply(const phb_domain *dom, const double *A, const double *X, double *Y, int32_t nvec, int64_t stride,
                      phb_stream stream);
/* G = V Y^T (m x m, row-major) and c = V b for m <= 16 float64 rows of n values, stride
 * values apart (V and Y alike), b contiguous: the Gram matrix and right-hand side of a
 * projected guess, with Y = A V from phb_stencil_apply */
int phb_projection_gram(const double *V, const double *Y, const double *b, int32_t m, int64_t n, int64_t stride,
                        double *G, double *c, phb_stream stream);
int phb_projection_solve(const double *G, const double *c, int32_t m, double reg, double *alpha, phb_stream stream);

/* Mixed precision: FP64 outer iterative refinement around FP32 inner Krylov solves.
 * A64/A32: the system in float64 and its float32 copy; b/x float64. The outer loop stops
 * when ||b - A64 x||/sqrt(n) < tol for every system or after max_outer sweeps; inner
 * solves run to inner_rtol relative to their own right-hand side. */
typedef struct phb_refine {
	int32_t kind;         /* inner solver: 0 CG, 1 BiCGStab */
	int32_t nrhs;
	int32_t max_outer;
	int32_t inner_maxit;
	int32_t use_graph;    /* 2: graph outer loop, persistent inner solves; 3: host outer loop, persistent inner
	                         solves (profilers see every launch); 1: nested graph loops; 0: host loops */
	int32_t ctas_per_sm;  /* the inner persistent solves' phb_solve::ctas_per_sm */
	double inner_rtol;
	phb_tolerance tol;    /* outer tolerance, on the float64 residual */
	const double *A64;
	const float *A32;
	const double *b;
	double *x;
	void *work;           /* >= phb_refine_work_bytes() */
	void *state;          /* >= phb_solve_state_bytes() */
	const phb_amg *amg;   /* optional (inner CG, nrhs 1): AMG-preconditioned inner solves, set up for A32 */
} phb_refine;
int64_t phb_refine_work_bytes(const phb_domain *dom, int kind, int nrhs);
/* out (optional): per-system outer results, as phb_refine_results (synchronises) */
int phb_refine_run(const phb_domain *dom, const phb_refine *r, phb_solve_result *out, int *outer_used, phb_stream stream);
/* per-system outer results of the last refinement (synchronises the stream) */
int phb_refine_results(const phb_domain *dom, const phb_refine *r, phb_solve_result *out, int *outer_used, phb_stream stream);

/* --- solve without device allocation ------------------------------------------------
 * No counterpart in phiPICT. CG (as phb_solve_run with kind 0, host-polled, no CUDA graph)
 * whose workspace lives in a static device array of PHB_NOALLOC_SCRATCH_BYTES inside this
 * library, for hosts that cannot give the library device memory: programs that carve the
 * GPU into fixed slices at start-up and allow no later allocation, or plugin hosts whose
 * allocator is not reachable through a C ABI. It calls no allocator. The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) with that device
 * current, so make that first call before any stream capture; later calls whose stream is
 * not capturing look it up again, so a context reset (which may move the array) is
 * followed. An empty domain (no cells) reports every system converged after 0 iterations.
 * Sizes whose workspace
 * (phb_cg_noalloc_bytes) exceeds the array are rejected with PHB_ERR_RANGE. All calls share
 * the one array: calls that overlap on the GPU (two streams, two host threads) race.
 * out (optional): per-system results, read back with synchronous copies. */
#define PHB_NOALLOC_SCRATCH_BYTES (32u << 20)
int64_t phb_cg_noalloc_bytes(const phb_domain *dom, int dtype, int nrhs);
int phb_cg_solve_noalloc(const phb_domain *dom, int dtype, int nrhs, const void *A, const void *b, void *x,
                         const phb_tolerance *tol, int maxit, int return_best, phb_solve_result *out, phb_stream stream);

/* --- AMG-preconditioned CG on CSR matrices ----------------------------------------------
 * Replaces AMGPCGSolve (bindings.cpp:764-776, solvers/krylov/krylov.cu:1248-1612) for callers
 * that bring an algebraic hierarchy (phiPICT's solvers/amg.py builds one with pyamg). Level l
 * holds its operator A_l (values per environment when a_val_stride > 0), the inverse diagonal
 * (per environment likewise), R_l (coarse x fine) and P_l (fine x coarse) with shared values;
 * the level below the last is solved with coarse_pinv ([coarse_n]^2, or one per environment
 * when coarse_batched). dtype: the system and the CG vectors; hdtype: the hierarchy. Environments
 * share the pattern and are solved independently, each to its own tolerance (tolerances, or
 * tol for all). `levels` is a host array; every other pointer is device memory. */
typedef struct phb_csr_level {
	const int32_t *a_row, *a_col;
	const void *a_val;
	int64_t a_val_stride; /* values per environment, or 0 when shared */
	const void *dinv;     /* [n] or [nenv][n] with a_val_stride */
	const int32_t *r_row, *r_col;
	const void *r_val;
	const int32_t *p_row, *p_col;
	const void *p_val;
	int32_t n;            /* rows of A_l */
	int32_t pad;
} phb_csr_level;
typedef struct phb_csr_pcg {
	int32_t dtype, hdtype;
	int32_t n, nenv, nlevels, coarse_n, coarse_batched;
	int32_t maxit, normalized, return_best, project_constant, pre_sweeps, post_sweeps, pad;
	double tol, omega;
	const double *tolerances;  /* host, [nenv], or NULL */
	const int32_t *row, *col;  /* the system matrix (the finest level's operator) */
	const void *val;
	int64_t val_stride;
	const phb_csr_level *levels; /* host array [nlevels] */
	const void *coarse_pinv;
	const void *b;
	void *x;                   /* initial guess, overwritten with the solution */
	void *work;                /* >= phb_csr_pcg_work_bytes() */
} phb_csr_pcg;
int64_t phb_csr_pcg_work_bytes(const phb_csr_pcg *a);
/* out[nenv]: per-environment results (synchronises the stream) */
int phb_csr_pcg_solve(const phb_csr_pcg *a, phb_solve_result *out, phb_stream stream);

/* --- adjoint of the step (float64 domains) ------------------------------------------
 * Replace phiPICT's *Grad kernels (piso/advection.cu:310-544,958-1195; pressure.cu:196-345,
 * 525-750; velocity_correction.cu:301-375; mhd/potential.cu:981-1329, bound at
 * bindings.cpp:781-814) and the solve adjoint pieces of core/piso_diff.py:1154-1421
 * (LinearSolveFunction, SparseOuterProduct, csrTranspose). Every *bar output is
 * accumulated (+=): zero it before the first contribution. ubbar has the layout of the
 * fixed-face velocity buffer (phb_domain::fvel). */
/* CT = C^T as a stencil (the adjoint momentum solve, SolveLinear's transposeA); C and CT hold
 * the domain's value type (float64 or float32) */
int phb_transpose_stencil(const phb_domain *dom, const void *C, void *CT, phb_stream stream);
/* Mbar[s][i] += scale * sum_k lam[i,k] x[nb_s(i),k] (ncomp 1 or dims): the adjoint of a
 * solve M x = b with respect to M is -lam (x)^T on the stencil, lam = M^-T xbar */
int phb_adj_outer(const phb_domain *dom, int ncomp, const double *lam, const double *x, double scale, double *Mbar,
                  phb_stream stream);
/* phb_advection_matrix: Cbar (slot 0 including the adjoint of Adiag) -> ubar; u = the forward velocity
 * (needed with LINEAR_UPWIND, whose upwinded faces follow the sign of its fluxes; may be NULL for CENTRAL) */
int phb_adj_advection_matrix(const phb_domain *dom, const double *Cbar, const double *u, double *ubar, phb_stream stream);
/* phb_advection_rhs (per-cell source): rhsbar -> ubar, srcbar (may be NULL), ubbar (may be NULL); u = the
 * forward velocity (LINEAR_UPWIND's deferred correction; may be NULL for CENTRAL) */
int phb_adj_advection_rhs(const phb_domain *dom, const double *rhsbar, const double *u, double *ubar, double *srcbar,
                          double *ubbar, phb_stream stream);
/* phb_scalar_rhs: rhsbar [inst][channels][cells] -> phibar (same layout), valuesbar (the layout of
 * sc->values; may be NULL), ubbar (fixed-face velocities; may be NULL); phi = the forward scalar field;
 * with LINEAR_UPWIND also ubar through the fluxes of u, the forward velocity (both required then) */
int phb_adj_scalar_rhs(const phb_domain *dom, const phb_scalar *sc, const double *phi, const double *u,
                       const double *rhsbar, double *phibar, double *valuesbar, double *ubar, double *ubbar,
                       phb_stream stream);
/* phb_pressure_rhs: hbar -> ubar, ustarbar, Cbar (off-diagonal slots), Abar, srcbar, ubbar; h = the forward HbyA;
 * u = the forward velocity (LINEAR_UPWIND's deferred correction; may be NULL for CENTRAL) */
int phb_adj_pressure_rhs(const phb_domain *dom, const double *C, const double *Adiag, const double *u, const double *ustar,
                         const double *h,
                         const double *hbar, double *ubar, double *ustarbar, double *Cbar, double *Abar, double *srcbar,
                         double *ubbar, phb_stream stream);
/* phb_divergence: dbar -> fbar (the field) and ubbar (fixed faces) */
int phb_adj_divergence(const phb_domain *dom, const double *dbar, double *fbar, double *ubbar, phb_stream stream);
/* phb_correct_velocity: ubar -> hbar, pbar, Abar */
int phb_adj_correct_velocity(const phb_domain *dom, const double *p, const double *Adiag, const double *ubar, double *hbar,
                             double *pbar, double *Abar, phb_stream stream);
/* phb_pressure_matrix: Pbar -> Abar */
int phb_adj_pressure_matrix(const phb_domain *dom, const double *Adiag, const double *Pbar, double *Abar, phb_stream stream);
/* phb_uxb_epot_rhs: rbar (may be NULL) -> xbar (+= the flux transpose; xbar may already hold
 * the adjoint of the u x e_b output), then xbar -> ubar */
int phb_adj_uxb_epot_rhs(const phb_domain *dom, const double *e_b, const double *rbar, double *xbar, double *ubar,
                         phb_stream stream);
/* phb_current_lorentz with accumulate = 0: srcbar -> phibar, xbar (u x e_b), stuartbar [ninst] */
int phb_adj_lorentz(const phb_domain *dom, const double *phi, const double *uxb, const double *e_b, const double *stuart,
                    const double *srcbar, double *phibar, double *xbar, double *stuartbar, phb_stream stream);

#ifdef __cplusplus
}
#endif

#endif
