/*
 * titus.h -- C ABI of the B200-native CSD energy-step library (libtitus.so).
 *
 * Drop-in boundary for the dynamical-low-rank (DLR) energy loops of TITUS
 * (CSMMLab/TITUS, code/SolverCSD.jl). The host keeps the reference's
 * Settings / SolverCSD construction (grid, P_N matrices, quadrature, Roe
 * matrices, CSD energy grid) and hands the assembled problem to this library;
 * the energy loop runs on the GPU as one persistent kernel.
 *
 * Conventions: plain pointers and sizes, FP64, row-major matrices
 * (X is n x r with row (i*ny + j) for cell (i, j), 0-based), int status
 * returns (0 = success; titus_last_error() gives the message). No C++
 * exceptions cross this boundary. A solver handle belongs to one host thread.
 */
#ifndef TITUS_H
#define TITUS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TITUS_OK 0
#define TITUS_ERR_ARG 1      /* invalid argument (sizes, null pointers) */
#define TITUS_ERR_CUDA 2     /* CUDA runtime error */
#define TITUS_ERR_DEVICE 3   /* device-side error flag (e.g. barrier timeout, breakdown) */
#define TITUS_ERR_LIMIT 4    /* size beyond what this build supports */

/* Integrators: SolverCSD.jl SolveFirstCollisionSourceDLR (:891-1120),
 * SolveFirstCollisionSourceDLRParallel (:1726-2008),
 * SolveFirstCollisionSourceDLRBUGRejection (:2011-2374),
 * SolveFirstCollisionSourceDLRHighOrder (:588-889: fixed rank, inflow on the
 * two outer layers, second-order limited sweep, RK4 K/L/S streaming with the
 * central operators; the reference never allocates its KUP buffer, this one
 * does). TITUS_DLR_HIGH_ORDER needs nx, ny >= 5. */
#define TITUS_DLR_FIXED 0
#define TITUS_PARALLEL_ADAPTIVE 1
#define TITUS_BUG_ADAPTIVE 2
#define TITUS_DLR_HIGH_ORDER 3
/* The full-rank P_N first-collision sweep (SolveFirstCollisionSource,
 * SolverCSD.jl:465-586); the method of titus_dose_adjoint. */
#define TITUS_PN_FULL 4
/* SolveFirstCollisionSourceDLRParallelRejection (SolverCSD.jl:2376-2742): the
 * parallel integrator's augmented step with the BUG loop's rejections. Where
 * the reference's next step raises a DimensionMismatch (a scattering
 * rejection after a streaming step that changed the rank, :2553, :2662-2665)
 * the solve stops with TITUS_ERR_DEVICE. Plain solves and titus_solve_from
 * only (not batched). */
#define TITUS_PARALLEL_REJECTION 5

/* Assembled problem. Replaces the fields of `SolverCSD{T}` that the energy
 * loop reads (SolverCSD.jl:20-146) plus the per-step tables the loop derives
 * from them (SigmaAtEnergy, PsiBeam). All arrays are host memory, copied by
 * titus_create. */
typedef struct titus_problem {
    int32_t nx, ny;           /* NCellsX, NCellsY */
    int32_t npn;              /* nPN; N = (nPN+1)^2 moments */
    int32_t n_moments;        /* N */
    int32_t n_ordinates;      /* q = number of reduced ordinates (idxBeam) */
    int32_t n_energies;       /* nEnergies = length(csd.eTrafo) */
    int32_t r;                /* settings.r */
    double dx, dy;            /* settings.dx, settings.dy */
    double theta;             /* settings.ϑ */
    double theta_index;       /* settings.ϑIndex */
    double c_eta;             /* settings.cη */
    const double* density;    /* n: density at cell i*ny+j */
    const double* e_trafo;    /* nE: csd.eTrafo */
    const double* stopping;   /* nE: csd.S (dose weights) */
    const double* bc_energy;  /* nE: PsiBeam energy factor at index k (scale*exp(-σE(E0-E_k)^2)*S[k]*ρmin) */
    const double* sigma;      /* nE x (npn+1): SigmaAtEnergy(csd, eGrid[k]) */
    const double* bc_space;   /* n: PsiBeam spatial factor at each cell (read on boundary cells) */
    const double* bc_angle;   /* q: PsiBeam angular factor per reduced ordinate */
    const double* omega;      /* q x 3: qReduced (Omega_x, Omega_y, Omega_z) */
    const double* m_reduced;  /* N x q: MReduced (row-major) */
    /* P_N operators as CSR (N x N): [0]=Ax, [1]=Az, [2]=|Ax|, [3]=|Az| */
    const int32_t* op_rowptr[4];
    const int32_t* op_col[4];
    const double* op_val[4];
    const int32_t* x_completion;   /* candidate cells for completing rank-deficient X bases */
    int32_t n_x_completion;
    const int32_t* w_completion;   /* candidate moments for completing rank-deficient W bases */
    int32_t n_w_completion;
    const int32_t* sweep_restore;  /* cells whose ordinate-0 value is restored after the sweep */
    int32_t n_sweep_restore;
    const double* stopping_mid;    /* nE-1: csd.SMid (stopping power at the energy midpoints, CSD.jl:88-89);
                                      read by the full-rank P_N solver only, may be NULL otherwise */
} titus_problem_t;

/* Arithmetic of the energy loop. FP64: every product in FP64 (the plain
 * mode, parity with the FP64 restatement of the reference). MIXED: the
 * operator Grams X^T L_d X and W^T A_d W of the rank-adaptive integrators
 * (streaming and S-step, SolverCSD.jl:1856-1859, :2187-2199) run on the
 * tensor cores in TF32 with a hi/lo split of each FP64 input and FP32
 * accumulation wherever the basis width is >= 32; the QR / range finders, the
 * truncation SVD, the small algebra and the dose stay FP64. MIXED applies to
 * TITUS_PARALLEL_ADAPTIVE and TITUS_BUG_ADAPTIVE (plain and batched). */
typedef enum titus_precision { TITUS_PRECISION_FP64 = 0, TITUS_PRECISION_MIXED = 1 } titus_precision_t;

typedef struct titus_options {
    int32_t team_ctas;     /* CTAs cooperating on one solve (0 = library default) */
    int32_t max_steps;     /* stop after this many loop iterations (0 = full sweep) */
    double rank_tol;       /* relative singular-value cut for numerical rank (0 = 1e-12) */
    int32_t profile;       /* 1 = record per-phase device timers (read with titus_profile) */
    int32_t precision;     /* a titus_precision_t value; 0 = FP64 */
} titus_options_t;

/* Host result buffers (caller-owned). Factors are returned raw: X (n x r_cap),
 * S (r_cap x r_cap), W (N x r_cap) in their leading `rank` columns; the
 * caller forms svd(S) to build the reference's return tuple
 * (X*U, 1/2 sqrt(gamma_0) Sigma, O*W*V, W*V, dose, psi). */
typedef struct titus_result {
    double* dose;          /* n */
    double* X;             /* n x r_cap, row-major, leading dimension r_cap */
    double* S;             /* r_cap x r_cap */
    double* W;             /* N x r_cap */
    double* psi;           /* n x q */
    int32_t r_cap;         /* capacity (columns) of X, S, W */
    int32_t rank;          /* out: rank of the returned factors */
    int32_t steps_done;    /* out: loop iterations executed */
    int32_t* rank_history; /* optional (nE): fixed / parallel: rank after the step with energy
                              index n at [n-1]; BUG and parallel rejection: rank at the start of
                              each loop iteration (repeated energies included, first nE
                              iterations); -1 if unused */
    double* eta_history;   /* optional (nE): BUG / parallel rejection: streaming eta of each
                              rejection test, in order */
    double* bound_history; /* optional (nE): the matching bound
                              c_eta * theta * max(1e-7, ||S||^theta_index) / dE with the S of the
                              streaming S-step (BUG, SolverCSD.jl:2224) or the truncated S
                              (parallel rejection, :2583) */
    double* time_history;  /* optional (nE): parallel: pseudo-time t at [n-1];
                              BUG and parallel rejection: energy index n (1-based) of each iteration */
} titus_result_t;

typedef struct titus_solver titus_solver_t;

/* Upload the problem and allocate device state (replaces the data that
 * `SolverCSD(settings)` prepares, SolverCSD.jl:63-146). problem->r is
 * settings.r: the fixed rank (TITUS_DLR_FIXED, r <= 24 in this build) or the
 * rank cap of the adaptive integrators (r <= titus_max_rank(), which start at
 * floor(r/2); a step whose rank would exceed 40 fails with TITUS_ERR_LIMIT). */
int titus_create(const titus_problem_t* problem, titus_solver_t** out);

/* Run one integrator over the energy grid on the device and copy the result
 * to host buffers (replaces `Solve*(solver)` of SolverCSD.jl:891, 1726, 2011). */
int titus_solve(titus_solver_t* solver, int32_t method, const titus_options_t* options,
                titus_result_t* result);

/* Same energy loop without the host copies: leaves the state on the device.
 * `stream` is a cudaStream_t (NULL = legacy default stream). Used for
 * device-resident timing; titus_fetch copies the state out afterwards. */
int titus_solve_device(titus_solver_t* solver, int32_t method, const titus_options_t* options,
                       void* stream);
int titus_fetch(titus_solver_t* solver, titus_result_t* result);

/* One-shot: create + solve + destroy with host buffers in and out. */
int titus_solve_problem(const titus_problem_t* problem, int32_t method,
                        const titus_options_t* options, titus_result_t* result);

/* Checkpoint / resume: replace the device state (X, S, W of the given rank,
 * psi, dose) and the next energy index `n_next` (1-based like the reference
 * loop variable n), then titus_solve_from continues the loop from there with
 * any integrator (rank <= 24 for TITUS_DLR_FIXED, <= 40 for the adaptive ones;
 * the BUG loop's pseudo-time restarts at (n_next - 2) dE). */
int titus_set_state(titus_solver_t* solver, int32_t rank, const double* X, const double* S,
                    const double* W, const double* psi, const double* dose, int32_t n_next);
int titus_solve_from(titus_solver_t* solver, int32_t method, const titus_options_t* options,
                     int32_t n_stop, titus_result_t* result);

/* Where the last solve on this handle stopped: the 1-based energy index the
 * loop would process next (the reference loop variable n; a rejected BUG step
 * repeats its n) and, for the adaptive integrators, the pseudo-time t of
 * SolverCSD.jl:1763 / :2100 (fixed rank: (n_next - 2) dE). With
 * titus_fetch's factors this is a complete checkpoint for titus_set_state.
 * `t` may be NULL. */
int titus_resume_point(titus_solver_t* solver, int32_t* n_next, double* t);

/* One pencil beam of a batched solve: its own energy grid (5 MeV -> cutoff
 * grid of the base problem replaced by this spot's) and entry profile. All
 * spots share the base problem's phantom, P_N operators, quadrature and
 * reduced ordinates. Arrays are host memory, copied by the call. */
typedef struct titus_spot {
    int32_t n_energies;        /* nE of this spot's grid */
    double d_e;                /* its tau step (e_trafo[1] - e_trafo[0]) */
    const double* stopping;    /* nE */
    const double* bc_energy;   /* nE: PsiBeam energy factor */
    const double* sigma;       /* nE x (npn+1) */
    const double* bc_space;    /* n: PsiBeam spatial factor (entry point of this spot) */
} titus_spot_t;

/* Batched pencil-beam solves (no counterpart in the reference, which solves
 * one beam per Solve* call): all `nspots` spots advance in one persistent
 * launch, options->team_ctas CTAs per spot (default 1) and as many spots at a
 * time as the GPU holds teams, which take the spots longest energy grid first
 * from a device work queue. method: TITUS_PARALLEL_ADAPTIVE or
 * TITUS_BUG_ADAPTIVE; options->max_steps bounds each spot's loop.
 * dose_out: nspots x n (row s = dose of spot s); rank_out / iters_out
 * (nspots, optional): final rank and loop iterations per spot. */
int titus_solve_batched(titus_solver_t* solver, int32_t method, const titus_options_t* options, int32_t nspots,
                        const titus_spot_t* spots, double* dose_out, int32_t* rank_out, int32_t* iters_out);

/* The same batched solve in three parts, for callers that repeat it (plan
 * optimisation loops) or time it: titus_batch_upload copies the spots' tables
 * to the device once (the handle borrows `solver`, which must outlive it);
 * titus_batch_solve_device launches the persistent kernel on `stream` (a
 * cudaStream_t, NULL = default stream) and returns without waiting;
 * titus_batch_fetch waits for the device, checks its status and copies the
 * doses (nspots x n), final ranks and iteration counts out (each may be NULL).
 * Teams take spots from a device work queue, longest energy grid first, so
 * the launch ends about when its longest spot does. */
typedef struct titus_batch titus_batch_t;
int titus_batch_upload(titus_solver_t* solver, int32_t nspots, const titus_spot_t* spots, titus_batch_t** out);
int titus_batch_solve_device(titus_batch_t* batch, int32_t method, const titus_options_t* options, void* stream);
int titus_batch_fetch(titus_batch_t* batch, double* dose_out, int32_t* rank_out, int32_t* iters_out);
/* After titus_batch_fetch: per spot, the sum over its loop iterations of the
 * rank entering each (nspots entries): the work done, for throughput accounting. */
int titus_batch_rank_sums(titus_batch_t* batch, int32_t* out);
void titus_batch_destroy(titus_batch_t* batch);

void titus_destroy(titus_solver_t* solver);

/* Copy the last error message of this thread into buf (always terminated). */
int titus_last_error(char* buf, size_t len);

/* Per-phase device timers of the last profiled solve (options.profile = 1),
 * in nanoseconds at the nominal SM clock, recorded on the first CTA. Timers are
 * exclusive (time is charged to the innermost open phase):
 * [0] barrier waits, [1] reductions, [2] Jacobi eigensolvers / SVD, [3] Cholesky,
 * [4] basis completion, [5] streaming row passes, [6] scattering and truncation
 * row passes, [7] range-finder / augmentation passes, [8] small-matrix algebra,
 * [9] everything else, [10] boundary inflow, dose half-step and sweep; then
 * event counts: [11] Jacobi SVD sweeps, [12] SVD calls, [13] eigensolver calls,
 * [14] eigensolver sweeps, [15] Cholesky calls, [16] rank-revealing and [17]
 * certified range-finder sides, [18] team barriers (adaptive integrators).
 * Returns the number of entries written (<= n). */
int titus_profile(titus_solver_t* solver, double* ns, int32_t n);

/* Fixed-rank solve (method TITUS_DLR_FIXED) that allocates nothing. No
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc, because a host framework's allocator or memory pool owns their
 * device memory or their policy forbids device allocation after start-up.
 * `problem` holds DEVICE pointers in the same layout titus_create reads from
 * host memory; dose (n), X (n x r), S (r x r), W (N x r) and psi (n x q) are
 * device output buffers owned by the caller (row-major). All intermediates live
 * in one static device array of 16 MiB that every GPU loading the library keeps
 * until the process exits. A problem fits when
 *   913 n + 580 N + 4 nE + 73728 G + 48 KiB <= 16 MiB
 * (n cells, N moments, nE energies, G <= 32 CTAs; about 16 700 cells at P21
 * with G = 16); larger ones, rank > 24 or q > 24 are rejected with
 * TITUS_ERR_LIMIT. All calls on a device share that array, so calls that
 * overlap on the GPU race: issue them one at a time per device. Each call
 * clears what must start at zero and looks the array's address up for the
 * current device. The call is synchronous: it reads e_trafo[0..1] and the status
 * words back and waits for `stream`.
 * Error text (if any) is written to err[0..err_len). */
int titus_solve_noalloc(const titus_problem_t* problem, const titus_options_t* options, double* dose,
                        double* X, double* S, double* W, double* psi, int32_t* rank_out, void* stream,
                        char* err, size_t err_len);

/* Second-order limited upwind transport flux of the uncollided ordinates,
 * replacing solveFlux!(obj, phi, flux) (code/SolverCSD.jl:295-386, limiter
 * minmod/slopefit :288-293). All arrays are DEVICE arrays: phi and flux hold
 * nx*ny*q doubles with cell (i, j), ordinate l at (i*ny + j)*q + l (i along x,
 * j along y); omega_x and omega_z hold the q ordinates' x and y components
 * (qReduced[:,1] and qReduced[:,3]). flux is written on the interior cells
 * 2 <= i < nx-2, 2 <= j < ny-2 only, like the reference's loops; its other
 * entries are left as they were. phi and flux must not overlap. The call is
 * asynchronous on `stream` (a cudaStream_t, NULL for the default stream).
 * Returns TITUS_OK, TITUS_ERR_ARG (sizes, NULL, dx or dy <= 0, overlap),
 * TITUS_ERR_LIMIT (ny*q >= 2^31) or TITUS_ERR_CUDA. */
int titus_limited_flux(int32_t nx, int32_t ny, int32_t q, double dx, double dy, const double* omega_x,
                       const double* omega_z, const double* phi, double* flux, void* stream);

/* Full-rank P_N first-collision solver (SolveFirstCollisionSource,
 * code/SolverCSD.jl:465-586): the collided flux as the whole moment matrix u
 * (n x N, row-major, row i*ny + j), advanced with the reference's explicit
 * step -- upwind sweep of the reduced ordinates with the beam inflow at
 * energy[n], uTilde = u - dE (L2x u Ax + L2y u Az + L1x u |Ax| + L1y u |Az|),
 * collision (I + dE D)^{-1}, in-scattering from psi, and the dose with csd.SMid
 * (problem->stopping_mid must be set). It is the r -> N limit the DLR
 * integrators approach. titus_pn_full_solve_device runs the whole sweep on
 * `stream` (a cudaStream_t, NULL = default) as one captured CUDA graph of two
 * kernels per energy step; options->max_steps bounds the steps (0 = all).
 * titus_pn_full_fetch waits and copies u (n x N, raw: the reference returns
 * 1/2 sqrt(gamma_0) u), the dose (n) and psi (n x q) to host buffers (each may
 * be NULL). titus_pn_full_solve does both. */
int titus_pn_full_solve_device(titus_solver_t* solver, const titus_options_t* options, void* stream);
int titus_pn_full_fetch(titus_solver_t* solver, double* u_out, double* dose_out, double* psi_out);
int titus_pn_full_solve(titus_solver_t* solver, const titus_options_t* options, double* u_out, double* dose_out,
                        double* psi_out);

/* Three-dimensional problems (no counterpart in the reference, which is 2D:
 * code/stencils.jl:7-11 builds x and y stencils only). The same scheme with a
 * z direction: cell (i, j, k) has row (k*nx + i)*ny + j (z slowest, so every
 * z layer is a 2D grid in the reference's row order); the boundary (ghost)
 * cells are those on any of the six faces; z streams with the P_N matrix Ay
 * (PNSystem.jl:142-194, unused in 2D) and its Roe |Ay|, through the
 * density-weighted stencils of stencils.jl written with dz; the uncollided
 * sweep adds (Omega_y / dz) times the upwind z difference.
 * titus_create_3d takes the 2D problem struct with every cell array (density,
 * bc_space, x_completion and sweep_restore indices) over nx ny nz cells, plus
 * this extension. A 3D handle runs the full-rank P_N solver
 * (titus_pn_full_solve*, u and psi over nx ny nz rows); the DLR entry points
 * return TITUS_ERR_ARG for it. */
typedef struct titus_problem_3d {
    int32_t nz;                   /* z layers (>= 3) */
    double dz;                    /* z spacing (> 0) */
    const int32_t* op_rowptr[2];  /* CSR (N x N) of Ay, |Ay| */
    const int32_t* op_col[2];
    const double* op_val[2];
} titus_problem_3d_t;
int titus_create_3d(const titus_problem_t* problem, const titus_problem_3d_t* ext, titus_solver_t** out);

/* Dose objective and its gradients (no counterpart in the reference, which
 * has no adjoint): J = sum_c weight[c] (dose[c] - target[c])^2 of the sweep's
 * dose, or any J whose dJ/d(dose) the caller passes in dj_ddose (then weight
 * and target are ignored and *objective_out is NaN). Returns the dose (n), J,
 * dJ/drho per cell (n) and dJ/dprofile (n): the sensitivity to PsiBeam's
 * spatial factor problem->bc_space, nonzero on boundary cells only -- for a
 * plan whose profile is sum_s w_s p_s, dJ/dw_s = p_s . dJ/dprofile. The
 * energy grid and PsiBeam's rho_min are held fixed (they follow min(rho) when
 * the problem is built). method: TITUS_PN_FULL, the exact discrete adjoint of
 * titus_pn_full_solve's sweep, transposed stencils and P_N products run from
 * the last energy step back to the first; checkpoint_every = k keeps (u, psi)
 * entering every k-th step from one forward pass and recomputes each segment
 * (0 = about sqrt(steps)); device memory about (steps/k + k + 12) n N words.
 * weight, target, dj_ddose and the outputs are host arrays (NULL weight = 1,
 * NULL target = 0, NULL outputs are skipped). Synchronous. FP64 only. */
int titus_dose_adjoint(titus_solver_t* solver, int32_t method, const titus_options_t* options, const double* weight,
                       const double* target, const double* dj_ddose, int32_t checkpoint_every, double* objective_out,
                       double* dose_out, double* grad_density, double* grad_profile);

/* Test hooks (no counterpart in the reference), for failure-detection tests
 * that fault nothing.
 * titus_debug_barrier_fault: the NEXT launch on this handle bounds every team
 * barrier wait by `spin_limit` polls (0 = default, about a second), and CTA 1
 * of the team does not arrive at barrier number `barrier` (1-based, counted from
 * the start of the launch; <= 0 = every CTA arrives). The waits run out, the
 * kernel leaves, the solve returns TITUS_ERR_DEVICE naming the barrier, and the
 * handle stays usable. Needs a team of >= 2 CTAs; applies to one launch only.
 * titus_debug_fail_alloc: the `after`-th device allocation from now (any handle)
 * fails as if cudaMalloc had returned cudaErrorMemoryAllocation; 0 = off. */
int titus_debug_barrier_fault(titus_solver_t* solver, int32_t barrier, int64_t spin_limit);
int titus_debug_fail_alloc(int32_t after);
/* titus_debug_tc_gram: the MIXED mode's tensor-core Gram run on host data, for
 * the unit test of its layouts. F (rows x (nops+1) nw, row-major) holds A in
 * columns [0, nw) and nops operator images O_d A after it; out (nops x nw x nw)
 * receives out[d][i][j] = sum_r (O_d A)[r][i] A[r][j], formed as the adaptive
 * kernel forms it (hi/lo TF32 operands, tcgen05 MMAs, FP32 accumulation in
 * TMEM). nw <= 80, nops in {1, 2, 4}. */
int titus_debug_tc_gram(const double* F, int32_t rows, int32_t nw, int32_t nops, double* out);

/* Build / capability queries. */
int titus_max_rank(void);        /* largest settings.r accepted (adaptive rank cap) */
int titus_max_ordinates(void);   /* largest q supported */
const char* titus_version(void);

#ifdef __cplusplus
}
#endif

#endif /* TITUS_H */
