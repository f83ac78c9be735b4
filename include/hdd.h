/*
 * hdd.h -- C ABI of the B200 hierarchical domain-decomposition PCG Poisson solver.
 *
 * Drop-in boundary for the reference's solver API (uwgraphics/hierarchicaldd,
 * class SPGrid_Domain_Decomposition_Solver and the Test_Bench options).  Every
 * entry point returns an hdd_status; no C++ exception crosses this boundary.
 * The caller owns host buffers; the library owns all device memory.  A solver
 * handle is used from one host thread at a time.
 *
 * Dense arrays ("*_dense") cover the whole grid of size[0]*size[1]*size[2]
 * cells, x slowest and z fastest: element (i,j,k) is at (i*size[1]+j)*size[2]+k.
 * Flags use the reference bit layout (Active 0x10000, Dirichlet 0x20000, face
 * bits 0x100000<<k); cells with flag 0 are exterior.
 */
#ifndef HDD_B200_H
#define HDD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    HDD_OK = 0,
    HDD_ERR_INVALID_ARGUMENT = 1,
    HDD_ERR_CUDA = 2,
    HDD_ERR_OUT_OF_MEMORY = 3,
    HDD_ERR_NOT_INITIALIZED = 4,
    HDD_ERR_UNSUPPORTED = 5,     /* input outside what the GPU path implements */
    HDD_ERR_NOT_CONVERGED = 6,   /* max_iters reached; the solution is still returned */
    HDD_ERR_BREAKDOWN = 7,       /* non-finite scalars in PCG (e.g. NaN right-hand side) */
    HDD_ERR_TIMEOUT = 8,         /* a bounded device wait ran out */
    HDD_ERR_IO = 9,
    HDD_ERR_BUSY = 10,
    HDD_ERR_NOT_FOUND = 11,
    HDD_ERR_INTERNAL = 12
} hdd_status;

/* Precision modes of the PCG outer loop (the preconditioner is FP32 in all). */
enum {
    HDD_PRECISION_REFERENCE = 0, /* FP32 vectors, FP64 dot accumulation, FP32 alpha/beta (as the reference) */
    HDD_PRECISION_MIXED = 1      /* FP32 preconditioner and search vectors; FP64 iterate x, dots,
                                    alpha/beta and true residual r = b - A x, recomputed every
                                    true_residual_every iterations and before stopping, so the
                                    stop test holds for the true residual */
};

typedef struct {
    int size[3];            /* reference -size (cells per axis + 1) */
    int sub_size[3];        /* reference -sub_size */
    int vlevels;            /* reference -vlevels */
    int nVcycles;           /* reference -nVcycles */
    int interior_smoothing; /* reference -interior_smoothing */
    int boundary_smoothing; /* reference -boundary_smoothing */
    int sigma_levels;       /* reference -sigma_levels */
    int sigma_smoothing;    /* reference -sigma_smoothing */
    int sigma_mg;           /* reference -sigma_mg */
    double tol;             /* stop tolerance on max|r| */
    int relative_tol;       /* 1: max|r| <= tol*max|b|; 0: max|r| <= tol (reference test) */
    int max_iters;          /* reference passes 5000 */
    int min_iters;
    int precision_mode;     /* HDD_PRECISION_* */
    int true_residual_every;/* mixed mode: recompute r = b - A x every N iterations (0 = never) */
    int device;             /* CUDA device ordinal */
    int coarse_solve;       /* HDD_COARSE_* : how the coarsest interface level is solved */
    int solve_share;        /* persistent interface solves use 1/solve_share of the device's
                               resident CTAs (0 or 1 = all), leaving room for concurrent solves;
                               results do not depend on it */
    int multilevel;         /* reference -multilevel (demos/Domain_Decomposition_CPU_Only_Two_Levels,
                               SPGrid_Domain_Decomposition_Preconditioner.h:127-230): 1 = two-level
                               DD, each subdomain solved by a DD of its own at sub_size/2 (its
                               interface system and V-cycles on boxes of sub_size/2) instead of
                               V-cycles; one system per solve context */
} hdd_options;

/* Coarsest interface (sigma) level.  The reference runs 200 smoothing steps
 * there (CPU/Interface_Solver/SIGMA_MULTIGRID_SOLVER.cpp:43), a contraction
 * towards the Schur complement solve S^{-1} b. */
enum {
    HDD_COARSE_REFERENCE = 0, /* the 200 steps; replaced by one exact solve of S when they have
                                 converged (setup's estimate rho^200 <= 1e-7): same result */
    HDD_COARSE_EXACT = 1      /* always one exact solve of S: a deviation from the reference where
                                 the 200 steps have not converged (slowly contracting coarse levels) */
};

typedef struct {
    int iterations;
    int converged;
    double final_norm;        /* max|r| of the recursively updated residual */
    double b_inf;             /* max|b| over Active|Interface cells */
    double true_residual_inf; /* max|b - A x| / max|b| of the returned iterate (FP64 under
                                 HDD_PRECISION_MIXED, see hdd_get_solution_dense_f64) */
    double true_residual_l2;  /* ||b - A x||_2 / ||b||_2 of the same */
    double solve_ms;          /* device time of the PCG loop */
    double setup_ms;          /* host+device time of hdd_initialize_preconditioner */
} hdd_result;

typedef struct hdd_solver hdd_solver;

/* Defaults equal the reference Test_Bench defaults
 * (demos/Domain_Decomposition_CPU_Only/Test_Bench_3D/main.cpp:236-251) with
 * tol 1e-6 relative. */
void hdd_options_default(hdd_options* opts);

/* Replaces constructing SPGrid_Domain_Decomposition_Solver
 * (demos/Domain_Decomposition_CPU_Only/SPGrid_Domain_Decomposition_Solver/
 *  SPGrid_Domain_Decomposition_Solver.h:40). */
hdd_status hdd_create(const hdd_options* opts, hdd_solver** out);

/* Replaces Read_SPGrid / Convert (SPGrid_Domain_Decomposition_Solver.h:73-105):
 * loads cell flags and the right-hand side b. */
hdd_status hdd_set_domain_dense(hdd_solver* s, const uint32_t* flags, const float* rhs);

/* The Test_Bench "velocity" mode on a uniform grid (GPU/Test_Bench_3D/main.cpp:317-324):
 * GRID_HIERARCHY_PROJECTION::Compute_Divergence of the face velocities u, v, w
 * (Divergence_Helper, scale (1/dx)^3 * (-dx^2)) at Interior|Ghost fluid cells,
 * then Convert's flags (fluid Dirichlet 0x2 -> Dirichlet, else fluid Active 0x8
 * -> Active, else exterior; SPGrid_Convertor.h:213-236), computed on the GPU.
 * fluid_flags use the SPGrid_Fluids bits (Interior 0x1, Dirichlet 0x2, Ghost 0x4,
 * Active 0x8, face X/Y/Z valid 0x10/0x20/0x40); u[c] is the velocity on cell c's
 * -x face (v, w likewise), all dense over opts.size cells.
 * hdd_velocity_divergence_dense writes the converted flags and the right-hand
 * side to flags_out and rhs_out; hdd_set_domain_velocity_dense loads them as
 * hdd_set_domain_dense would.  The adaptive multi-level SPGrid_Fluids hierarchy
 * (its ghost-value accumulation across levels) is not implemented. */
hdd_status hdd_velocity_divergence_dense(hdd_solver* s, const uint32_t* fluid_flags, const float* u, const float* v,
                                         const float* w, float dx, uint32_t* flags_out, float* rhs_out);
hdd_status hdd_set_domain_velocity_dense(hdd_solver* s, const uint32_t* fluid_flags, const float* u, const float* v,
                                         const float* w, float dx);

/* Sparse input in SPGrid pages, for callers holding an SPGrid allocator:
 * replaces Convert / Copy (SPGrid_Domain_Decomposition_Solver.h:73-105 of the
 * CPU demo), which read the flags and right-hand side channels page by page.
 * A page is 4 x 8 x 8 cells (the 4 KB page of a 16-byte cell struct with
 * 4-byte channels, SPGrid_Mask<4,2,3>); page_origin[3*p + a] is the cell
 * index of page p's first cell (a multiple of 4, 8, 8 per axis), and cell
 * (x, y, z) of page p is element 256*p + (x*8 + y)*8 + z of flags / rhs / x.
 * Cells of pages outside options.size are ignored; cells in no page are
 * exterior (flag 0).  A negative or misaligned origin, or a page listed twice,
 * gives HDD_ERR_INVALID_ARGUMENT. */
hdd_status hdd_set_domain_pages(hdd_solver* s, long long n_pages, const int32_t* page_origin,
                                const uint32_t* flags, const float* rhs);
/* Replaces the right-hand side only (zero outside the pages given). */
hdd_status hdd_set_rhs_pages(hdd_solver* s, long long n_pages, const int32_t* page_origin, const float* rhs);
/* Copies the solution of the last solve into the pages given (0 outside the grid). */
hdd_status hdd_get_solution_pages(hdd_solver* s, long long n_pages, const int32_t* page_origin, float* x);

/* Reads the reference's SPGrid directory format (size, block_offset, flags,
 * data) written by SPGRID_READ_WRITE::Write_SPGrid
 * (demos/SPGrid_Create_Simple_Domain/SPGRID_READ_WRITE.h:43-51). */
hdd_status hdd_load_spgrid_dir(hdd_solver* s, const char* directory);

/* Interface-matrix dump modes of Initialize_Preconditioner's iomode argument
 * (demos/Domain_Decomposition_CPU_Only/SPGrid_Domain_Decomposition_Solver/
 *  SPGrid_Domain_Decomposition_Solver.h:121-161, Test_Bench -iomode). */
enum {
    HDD_IOMODE_NEITHER = 0, /* assemble, write nothing (this library's default) */
    HDD_IOMODE_OUTPUT = 1,  /* assemble, then write the matrices to the directory */
    HDD_IOMODE_INPUT = 2    /* read the matrices from the directory instead of assembling */
};

/* Sets the iomode and dump directory used by the next
 * hdd_initialize_preconditioner.  The directory holds the reference's dump
 * layout (INTERFACE_SOLVER_DATA::Write_To_File, INTERFACE_SOLVER_DATA.h:177-212,
 * and INTERFACE_MATRIX_GENERATOR::Write_Interface_Map, :66-72): files levels and
 * number_of_subdomains, Matrix Market Aii_<l>_<s>, Air_<l>_<s>, Arr_<l>, Prr_<l>,
 * and interface_map; this library adds positions_<l> for its fill-reducing
 * ordering.  OUTPUT creates the directory if needed.  INPUT checks the dump
 * against the domain (HDD_ERR_INVALID_ARGUMENT when its levels, subdomain count,
 * sizes or interface cells differ) and reports unreadable files as HDD_ERR_IO.
 * The reference defaults to iomode "output" into "matrices_dump"; this library
 * defaults to HDD_IOMODE_NEITHER. */
hdd_status hdd_set_iomode(hdd_solver* s, int iomode, const char* directory);

/* Replaces Initialize_Preconditioner (SPGrid_Domain_Decomposition_Solver.h:121-161):
 * flags, subdomains, V-cycle topology, interface matrices and factorisations. */
hdd_status hdd_initialize_preconditioner(hdd_solver* s);

/* Replaces the right-hand side only (same domain and preconditioner). */
hdd_status hdd_set_rhs_dense(hdd_solver* s, const float* rhs);

/* Replaces Solve (SPGrid_Domain_Decomposition_Solver.h:165-197). */
hdd_status hdd_solve(hdd_solver* s, hdd_result* result);

/* Copies the solution x of the last solve. */
hdd_status hdd_get_solution_dense(hdd_solver* s, float* x);

/* The same in FP64.  Under HDD_PRECISION_MIXED the iterate is accumulated in
 * FP64 (the preconditioner stays FP32) and this returns it unrounded: a
 * solution of magnitude |x| carries an FP32 rounding error of about
 * 6e-8 |x|, which bounds the relative residual an FP32 x can show at about
 * 6e-8 ||A|| |x| / |b|; the FP64 iterate has no such floor.  Under
 * HDD_PRECISION_REFERENCE it is the FP32 solution widened. */
hdd_status hdd_get_solution_dense_f64(hdd_solver* s, double* x);

/* The convergence norm max|r| of the last solve at the start of every PCG
 * iteration, entry 0 being that of r = b: the values CONJUGATE_GRADIENT::Solve
 * logs with print_residuals
 * (PB/Public_Library/PhysBAM_Tools/Krylov_Solvers/CONJUGATE_GRADIENT.cpp:38-41).
 * Writes min(capacity, *n) entries of out; *n gets iterations + 1. */
hdd_status hdd_get_residual_history(hdd_solver* s, double* out, int capacity, int* n);

/* Test seam: z = Project(Apply_Preconditioner(r)), replacing
 * SPGrid_Domain_Decomposition_Preconditioner::Apply_Preconditioner
 * (SPGrid_Domain_Decomposition_Preconditioner.h:88-128) followed by
 * CG_SYSTEM::Project. */
hdd_status hdd_apply_preconditioner_dense(hdd_solver* s, const float* r, float* z);

/* Test seam: nV V-cycles of V_Cycle_Helper::v_cycle
 * (SPGrid_Library/SPGrid_V_Cycle_Helper.h:156-195) on the level-0 arrays u
 * (in/out) and b, with the interface values of u held fixed. */
hdd_status hdd_vcycle_dense(hdd_solver* s, float* u, const float* b, int n_vcycles);

/* Test seam: y = Project(A x), replacing CG_SYSTEM::Multiply + Project
 * (CG_SYSTEM.cpp:28-44,100-119). */
hdd_status hdd_multiply_dense(hdd_solver* s, const float* x, float* y);

/* Allocation-free y = Project(A x) plus dot = sum(x*y), for callers that
 * cannot allocate device memory when they need the operator (a framework
 * whose own allocator holds the device memory, or a loop that must not stall
 * on an allocation).  No counterpart in the reference.
 *   x, y:  DEVICE arrays in the dense layout of hdd_multiply_dense
 *          (size[0]*size[1]*size[2] floats, z fastest); cells outside the
 *          stored tiles are read as zero and left unwritten in y.
 *   dot:   DEVICE pointer to one double.
 *   stream: cudaStream_t to run on (NULL = legacy default stream); the call
 *          returns without synchronising.
 * Per-tile partial sums go to one fixed device array of 32768 doubles
 * (256 KiB, held by every GPU that loads the library); domains with more
 * stored tiles get HDD_ERR_INVALID_ARGUMENT.  The first call on a device looks
 * up that array's device address, so make it before any stream capture.
 * Calls that overlap on the GPU share the array and race.  The call runs on
 * the solver's device and leaves the calling thread's current device as it
 * found it. */
hdd_status hdd_multiply_dot_dense_device_noalloc(hdd_solver* s, const float* x, float* y, double* dot,
                                                 void* stream);

/* Test seam: one sigma V-cycle (SIGMA_MULTIGRID_SOLVER.cpp:35-47) from u = 0
 * on the level-0 interface right-hand side b0 (interface DOF order). */
hdd_status hdd_sigma_vcycle(hdd_solver* s, const float* b0, float* u0);

/* Test seam: one supernodal solve x = (A + 1e-5 I)^{-1} b on the GPU, the
 * stand-in for a PARDISO phase-33 solve of SIGMA_SMOOTHER::Smooth
 * (CPU/Interface_Solver/SIGMA_SMOOTHER.cpp:293-324): kind 0 = Arr of sigma
 * level `level`, kind 1 = Aii of every subdomain of that level with the
 * unknowns concatenated in subdomain order.  *n gets the number of unknowns;
 * with b or x NULL nothing else happens.  HDD_ERR_UNSUPPORTED for the
 * coarsest level when its smoothing steps are replaced by one solve of the
 * whole level (no separate Arr / Aii plans exist there). */
hdd_status hdd_interface_solve(hdd_solver* s, int kind, int level, const float* b, float* x, int* n);

/* Test seam: the same for nrhs (1, 2 or 4) right-hand sides at once, b and x
 * holding nrhs vectors of *n entries one after another.  One launch pair
 * reads each coefficient once for all of them; each solution is bit-identical
 * to hdd_interface_solve of its right-hand side.  HDD_ERR_UNSUPPORTED when the
 * plan's largest front leaves no shared memory for nrhs vectors. */
hdd_status hdd_interface_solve_batch(hdd_solver* s, int kind, int level, int nrhs, const float* b, float* x, int* n);

/* Interface DOF count at a sigma level and the level-0 DOF -> cell map
 * (INTERFACE_MATRIX_GENERATOR::interface_map). */
hdd_status hdd_interface_size(hdd_solver* s, int level, int* n);
hdd_status hdd_interface_map(hdd_solver* s, int* cells_xyz);

/* Assembled interface matrices for inspection (kind: 0 Arr, 1 Aii, 2 Air,
 * 3 Prr).  Call first with ptr == NULL to get rows/cols/nnz. */
hdd_status hdd_interface_matrix(hdd_solver* s, int kind, int level, int subdomain, int* rows,
                                int* cols, int* nnz, int* ptr, int* col, double* val);

/* Per-phase device timing (CUDA events on the solver stream) for profiling;
 * no reference counterpart (the reference prints wall-clock times).
 * Phases: 0 V-cycle kernel, 1 Laplacian kernel, 2 PCG vector kernels,
 * 3 interface gather/scatter, 4 sigma V-cycle (includes 6 and 7), 5 dense<->
 * tile copies, 6 supernodal forward solves, 7 supernodal backward solves.
 * Enabling clears the accumulators; ms/launches/bytes hold 8 entries.
 * hdd_get_kernel_bytes gives each phase's algorithmic bytes (the data the
 * kernels must move at minimum) for phases 0, 1, 6 and 7, 0 for the others. */
hdd_status hdd_set_kernel_timing(hdd_solver* s, int enable);
hdd_status hdd_get_kernel_timing(hdd_solver* s, double* ms, long long* launches);
hdd_status hdd_get_kernel_bytes(hdd_solver* s, double* bytes);

/* Host wall time (ms) of the last hdd_initialize_preconditioner, by phase:
 * ms[0] layout and vector uploads, ms[1] interface system (assembly, or reload
 * and dump under hdd_set_iomode), ms[2] interface solver (factorisations and
 * solve plans), ms[3] total.  No reference counterpart (the reference logs its
 * setup scopes with LOG::SCOPE). */
hdd_status hdd_get_setup_timing(hdd_solver* s, double* ms);

/* Poll budget of the bounded device waits inside the interface solves (a
 * task of a persistent supernodal solve waiting for the fronts it depends
 * on; about 0.2-0.5 us per poll).  A wait that runs out raises an error word:
 * the solve stops after that PCG iteration and returns HDD_ERR_TIMEOUT, and
 * the next call starts with the word cleared.  Default 1 << 22 polls; takes
 * effect for solves after hdd_initialize_preconditioner.  No reference
 * counterpart (the reference's host threads wait without bound,
 * GPU/Nodes/Communicator.cpp:30-33). */
hdd_status hdd_set_wait_limit(hdd_solver* s, long long polls);

/* Test seam for the bounded waits: on != 0 makes one dependency of the level-0
 * interface solve unsatisfiable (a parent front then waits for one task more
 * than its child runs), so every solve reports HDD_ERR_TIMEOUT once the wait
 * limit runs out; on == 0 restores the dependency.  No reference counterpart. */
hdd_status hdd_test_stall_dependency(hdd_solver* s, int on);

/* The PCG step lengths of the last solve, alpha[i] and beta[i] of iteration i
 * (beta[0] = 0), in the precision the solve used: the Lanczos coefficients of
 * the preconditioned operator (its extreme eigenvalues follow from them).
 * Writes min(capacity, *n) entries of each; *n gets the iteration count. */
hdd_status hdd_get_pcg_coefficients(hdd_solver* s, double* alpha, double* beta, int capacity, int* n);

/* Number of our CUDA kernel launches issued since the handle was created. */
hdd_status hdd_kernel_launch_count(hdd_solver* s, long long* count);

const char* hdd_status_string(hdd_status status);
const char* hdd_last_error(const hdd_solver* s);
void hdd_destroy(hdd_solver* s);

/* ---- Serving: concurrent solves on resident domains ------------------------
 * No counterpart in the reference, whose GPU demo solves one domain per
 * process (GPU/Test_Bench_3D/main.cpp) through one worker thread per GPU
 * (GPU/Nodes/Command.h:33-55).  A server owns `slots` worker threads.  A domain
 * added with hdd_server_add_domain is admitted, in arrival order, once its
 * estimated device footprint fits the HBM budget; a worker then runs its setup
 * (as hdd_initialize_preconditioner) and the domain stays resident until
 * removed.  Each solve request names a resident (or still setting-up) domain
 * and a right-hand side.  A resident domain keeps a pool of solve contexts (the
 * PCG and interface-solve vectors on a CUDA stream of their own, sharing the
 * domain's factors and tables), growing on demand up to `slots` while the HBM
 * budget allows; workers take the oldest request whose domain has a context
 * free, so requests on one domain and on different domains run concurrently.
 * A request's result does not depend on what else is in flight (bit-identical
 * to a solve alone).  All calls except hdd_server_destroy may be made from any
 * thread at any time. */
typedef struct hdd_server hdd_server;

typedef struct {
    int slots;                  /* worker threads = requests in flight (default 4, at most 64) */
    long long hbm_budget_bytes; /* admission budget for resident domains; 0 = 90% of free device memory */
    int device;                 /* CUDA device ordinal */
    int setup_threads;          /* OpenMP threads per domain setup; 0 = host cores / slots */
    int batch;                  /* continuous batching: requests of one domain solved together, up to this
                                   many (2 or 4) per batch; 0 or 1 = each request on its own context */
} hdd_server_options;

void hdd_server_options_default(hdd_server_options* opts);
hdd_status hdd_server_create(const hdd_server_options* opts, hdd_server** out);

/* Queues a domain for setup (flags are copied; opts as for hdd_create, its
 * device ignored).  Returns at once; HDD_ERR_OUT_OF_MEMORY when the domain's
 * estimated footprint alone exceeds the budget. */
hdd_status hdd_server_add_domain(hdd_server* srv, const hdd_options* opts, const uint32_t* flags,
                                 long long* domain_id);

/* HDD_OK once the domain is resident, HDD_ERR_BUSY while it waits for budget
 * or sets up (after waiting up to wait_ms; -1 = until settled), otherwise the
 * status its setup failed with (message via hdd_server_domain_error). */
hdd_status hdd_server_domain_status(hdd_server* srv, long long domain_id, int wait_ms);
hdd_status hdd_server_domain_error(hdd_server* srv, long long domain_id, char* message, int capacity);

/* Queues one solve of the domain for the dense right-hand side rhs (copied). */
hdd_status hdd_server_submit(hdd_server* srv, long long domain_id, const float* rhs, long long* request_id);

/* Waits up to wait_ms (-1 = until done) for a request.  HDD_ERR_BUSY while it
 * is pending.  Otherwise returns the request's own status (HDD_OK,
 * HDD_ERR_NOT_CONVERGED, or its domain's setup failure), fills result, the
 * dense solution x (if not NULL) and latency_ms = wall time from submit to
 * finish (if not NULL), and forgets the request. */
hdd_status hdd_server_poll(hdd_server* srv, long long request_id, int wait_ms, hdd_result* result, float* x,
                           double* latency_ms);

/* Waits for the domain's queued requests, then frees its device state and
 * its budget. */
hdd_status hdd_server_remove_domain(hdd_server* srv, long long domain_id);

/* Device bytes held by admitted domains (estimates until set up, then what
 * their solvers and solve contexts hold) and the budget. */
hdd_status hdd_server_memory(hdd_server* srv, long long* reserved, long long* budget);

/* Lets running setups and solves finish, stops the workers and frees every
 * domain.  Requests still queued are dropped. */
void hdd_server_destroy(hdd_server* srv);

#ifdef __cplusplus
}
#endif
#endif /* HDD_B200_H */
