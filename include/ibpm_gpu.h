/*
 * ibpm_gpu.h — C ABI of libibpm_gpu.so, a B200 (sm_100a) implementation of the
 * time step of the immersed boundary projection method (NUFgroup/IBPM.jl):
 * static bodies, a moving grid or moving bodies, its discrete adjoint and
 * batches of independent problems.  Meant to be bound from Julia with
 * `ccall`, from Python with ctypes, or from C/C++ directly.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (IBPM_OK = 0, negative = error).  The text of the last
 * error of a handle is returned by ibpm_last_error().  A handle owns all of its
 * device memory and one CUDA stream; it is not thread-safe (one thread at a
 * time per handle), like the reference's IBProblem whose working memory is
 * shared across calls (src/pre-processing/models.jl:79-106).
 *
 * Array layouts are exactly the reference's (Julia column-major):
 *   Γ, ψ, nonlin[k] : (nΓ, mg),  nΓ = (nx-1)(ny-1), index (i,j) -> i + (j-1)(nx-1)
 *   q, q0           : (nq, mg),  nq = ny(nx+1) + nx(ny+1), [qx (nx+1)×ny ; qy nx×(ny+1)]
 *   F̃b              : (nf, 1),   nf = 2 nb, [x-components of all points ; y-components]
 *   xb              : (nb, 2),   [x of all points ; y of all points]
 */
#ifndef IBPM_GPU_H
#define IBPM_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define IBPM_OK               0
#define IBPM_ERR_INVALID     -1   /* bad argument, size or handle               */
#define IBPM_ERR_CUDA        -2   /* a CUDA runtime call failed                  */
#define IBPM_ERR_NONFINITE   -3   /* CD/CL became NaN/Inf during ibpm_advance    */
#define IBPM_ERR_UNSUPPORTED -4   /* valid in the reference, not in this build   */
#define IBPM_ERR_NOMEM       -5   /* device allocation failed                    */

/* Arithmetic of the step. */
#define IBPM_PREC_FP64         0  /* plain FP64 everywhere                        */
#define IBPM_PREC_FP32_REFINED 1  /* FP32 sine transforms in the projection
                                     solve and the final vort2flux!; FP64 state,
                                     stencils, residuals, trial solve, trial
                                     vort2flux!, Schur solve and forces.  A
                                     refined solve is x = x̃ + S32(b − M x̃) with
                                     the residual in FP64 and x̃ the previous
                                     solution (iterative refinement, warm start) */

typedef struct ibpm_handle ibpm_handle;

/*
 * Problem description: the data of IBProblem(grid, bodies, dt, Re; freestream)
 * (src/pre-processing/problem-types.jl:23-41) for RigidBody{Static} bodies.
 * Grid fields are those of make_grid (src/fluid-domain/fluid-domain.jl:44-73)
 * after its rounding: h = len/nx.  nx and ny must be multiples of 4
 * (get_bc!/coarsify! of src/fluid-operators/mg-utils.jl need nx/4, ny/4).
 */
typedef struct ibpm_problem_desc {
    int32_t nx, ny, mg;        /* cells per level and number of nested levels   */
    double  h;                 /* finest grid spacing                           */
    double  offx, offy;        /* -xmin, -ymin of the finest domain             */
    double  Re, dt;            /* Reynolds number, time step                    */
    double  Ux, Uy, inclination; /* freestream at t = 0 (timestepping.jl:252-270) */
    double  beta[2];           /* explicit scheme coefficients, AB2 = {1.5,-0.5} */
    int32_t nbodies;           /* number of bodies                              */
    int32_t nb;                /* total number of boundary points               */
    const int32_t* body_npts;  /* [nbodies] points per body (in xb order)       */
    const double*  xb;         /* [nb*2] column-major (nb, 2)                   */
    const double*  ds;         /* [nb] segment lengths                          */
    int32_t precision;         /* IBPM_PREC_*                                   */
    int32_t device;            /* CUDA device ordinal                           */
    int32_t refine_sweeps;     /* FP32_REFINED: FP64-residual correction sweeps
                                  per refined solve (0 means 1; the first 32
                                  steps after create or set_state run one
                                  more); ignored for FP64                       */
} ibpm_problem_desc;

/* Library version string. */
const char* ibpm_version(void);

/*
 * Build a problem on the device: grid tables, the regularisation weights of E
 * (interface-coupling.jl:72-137), the Schur complement B column by column with
 * B_times! (laplacian.jl:98-119, 143-169) and its inverse.  Replaces
 * IBProblem(...) (problem-types.jl:23-41).  The state starts as IBState(prob)
 * (state-types.jl:25-47): zeros, with the uniform base flux q0.
 */
int ibpm_create(const ibpm_problem_desc* desc, ibpm_handle** out);

/* Release every device resource of the handle. */
int ibpm_destroy(ibpm_handle* h);

/* Text of the last error recorded on `h` (or of the last failed create). */
const char* ibpm_last_error(const ibpm_handle* h);

/* Sizes of the arrays used by get/set_state: nΓ, nq, mg, nf, nbodies. */
int ibpm_sizes(const ibpm_handle* h, int64_t* nGamma, int64_t* nq, int32_t* mg,
               int32_t* nf, int32_t* nbodies);

/*
 * Copy a state in.  Any pointer may be NULL (field left unchanged).  The
 * layouts are IBState's (state-types.jl:7-22).  q0 must be uniform per
 * level and component, as base_flux! makes it for static bodies
 * (timestepping.jl:252-270); anything else returns IBPM_ERR_UNSUPPORTED.
 * On a moving grid q0 is ignored: every step recomputes it.
 * q is stored as given: the next step's nonlinear term reads it, as the
 * reference does, even if it is not the curl of ψ.
 */
int ibpm_set_state(ibpm_handle* h, const double* Gamma, const double* q,
                   const double* q0, const double* psi, const double* nonlin1,
                   const double* nonlin2, const double* Fb);

/*
 * Turn the handle into LinearizedIBProblem(base_state, prob, dt)
 * (problem-types.jl:47-87): from now on ibpm_advance steps the linearisation
 * about the base state (Γ_B (nΓ, mg), q_B (nq, mg), with the problem's base
 * flux), whose nonlinear term is C'(Q⊗Γ_B + Q_B⊗Γ)/(4hc²) (nonlinear.jl:45-65,
 * 144-163); the state's own base flux becomes zero (timestepping.jl:236-250).
 * May be called again to change the base state.  The adjoint
 * (ibpm_adjoint_run) is that of the nonlinear step and refuses a linearised
 * handle.
 */
int ibpm_set_base_state(ibpm_handle* h, const double* Gamma_B, const double* q_B);

/* Copy the state out (NULL pointers are skipped). */
int ibpm_get_state(ibpm_handle* h, double* Gamma, double* q, double* q0,
                   double* psi, double* nonlin1, double* nonlin2, double* Fb);

/*
 * Advance the state by `nsteps` steps of advance!(state, prob, t)
 * (timestepping.jl:35-67).  t is accepted for interface parity; static bodies
 * with a fixed base flux do not depend on it.  CD_out and CL_out (may be NULL)
 * receive the per-step drag and lift coefficients of update_stress!
 * (timestepping.jl:330-354) as [nsteps][nbodies].  Returns IBPM_ERR_NONFINITE
 * if any CD/CL became non-finite (the reference's run_sim! stops on a
 * non-finite CL, src/ibpm.jl:95-97); the state is then whatever the steps
 * produced.
 */
int ibpm_advance(ibpm_handle* h, double t, int32_t nsteps, double* CD_out,
                 double* CL_out);

/*
 * Make the handle's single body move with the grid: MovingGrid(U, V, θ, θ̇)
 * (structure-domain/motion-types.jl:40-48), the motion type for which
 * advance! recomputes the base flux at the start of every step
 * (timestepping.jl:41-43) as base_flux! does (timestepping.jl:273-318):
 *   Ω = −θ̇(t), α = −θ(t),
 *   Ux0 = U cos α − V sin α + (Ux cos i − Uy sin i),
 *   Uy0 = U sin α + V cos α + (Ux sin i + Uy cos i)   (Ux, Uy, i: the desc's
 *                                                      free stream),
 *   q0 = hc (−Ω (y − yc) + Ux0) on x-fluxes, hc (Ω (x − xc) + Uy0) on y-fluxes,
 * (x, y) the face centres of each level (pre-processing/models.jl:135-153).
 * xc, yc are the IBModel keywords of that file (IBProblem leaves them 0).
 * motion0 = {U, V, θ, θ̇} at t = 0 sets the q0 reported before the first step
 * (IBState(prob) calls base_flux! at t = 0, state-types.jl:45).  The bodies'
 * E, B⁻¹ and the step are those of the static case (timestepping.jl:154-163,
 * 361-372).  Refused (IBPM_ERR_UNSUPPORTED) for more than one body
 * (models.jl:137) and for a linearised handle.  From then on the handle steps
 * only through ibpm_advance_moving; the adjoint and batches refuse it.
 */
int ibpm_set_moving_grid(ibpm_handle* h, double xc, double yc, const double* motion0);

/*
 * ibpm_advance for a moving grid: step k uses motion[4k .. 4k+3] = {U, V, θ,
 * θ̇} evaluated at that step's t (the reference's advance!(state, prob, t[k])
 * evaluates the motion's functions at t[k]).  Outputs as ibpm_advance; the
 * forces are in the body (grid) frame, as the reference's state.CD/CL.
 * ibpm_get_state's q0 is then the base flux of the last step.
 */
int ibpm_advance_moving(ibpm_handle* h, int32_t nsteps, const double* motion,
                        double* CD_out, double* CL_out);

/*
 * Make every body move with a MotionFunction (structure-domain/motion-types.jl:
 * 13-17): the body's points as created are its reference configuration x0,
 * and at the start of each step, as update_bodies! does
 * (timestepping.jl:386-398, move_body! move-body-utils.jl:86-133),
 *   xb = (x, y) + Rx x0,  ub = (ẋ, ẏ) + Ru x0,
 *   Rx = [cos θ  −sin θ; sin θ  cos θ],  Ru = θ̇ [−sin θ  −cos θ; cos θ  −sin θ],
 * then E and B⁻¹ are rebuilt for the moved points and the step solves
 * B F̃b = E(qs + q0) − ub·h (boundary_forces!, timestepping.jl:174-186).  The
 * reference applies B⁻¹ by conjugate gradients to reltol 1e-12
 * (laplacian.jl:123-141); here B is rebuilt on the device every step and
 * inverted exactly (to round-off).  Refused for a linearised handle or a
 * moving grid; the adjoint and batches refuse such a handle.  A step whose
 * moved point's 13×13 stencil would leave the finest grid ends the call with
 * IBPM_ERR_INVALID.
 */
int ibpm_set_motion_function(ibpm_handle* h);

/*
 * ibpm_advance for MotionFunction bodies: step k uses, for body j,
 * motion[6 (k nbodies + j) .. +5] = {x, y, θ, ẋ, ẏ, θ̇} evaluated at that
 * step's t (get_transformation, move-body-utils.jl:70-84).  Outputs as
 * ibpm_advance (lab-frame forces).
 */
int ibpm_advance_bodies(ibpm_handle* h, int32_t nsteps, const double* motion,
                        double* CD_out, double* CL_out);

/* The body points and their velocities as of the last step (state.xb and the
 * bodies' ub), (nb, 2) column-major each; either may be NULL.  Fixed bodies
 * report their points and zero velocities. */
int ibpm_get_body_points(ibpm_handle* h, double* xb, double* ub);

/*
 * vort2flux!(state.ψ, state.q, state.Γ, model, mg) (curl.jl:133-165): make ψ
 * and q consistent with Γ (coarsifies Γ into the coarse-level centres first).
 */
int ibpm_vort2flux(ibpm_handle* h);

/* Copy out the precomputed inverse Schur complement (nf×nf, column-major),
 * the reference's prob.Binv (laplacian.jl:118). */
int ibpm_get_binv(ibpm_handle* h, double* Binv);

/* Block until all work queued on the handle's stream is done. */
int ibpm_sync(ibpm_handle* h);

/*
 * x = Δ⁻¹ rhs on one (nx-1)×(ny-1) field with zero Dirichlet edges — the
 * operator the reference applies on every level of vort2flux!
 * (src/fluid-operators/laplacian.jl:24-41) — without allocating any device
 * memory.  No counterpart in the reference: it is for callers that cannot call
 * cudaMalloc (a host runtime that owns the device memory through its own pool,
 * an application with a fixed memory budget).  rhs and x are device pointers
 * in the reference layout (column-major, no padding); the work is queued on
 * `stream` (a cudaStream_t, or NULL for the legacy default stream) and the call
 * returns without waiting for it.  Limit: nx, ny <= 512 and in the supported
 * transform lengths; larger sizes return IBPM_ERR_INVALID.  The intermediate
 * slab and transform tables are file-scope device arrays (2.1 MB + 104 KB on
 * every GPU that loads the library, held until exit), shared by all calls:
 * calls that overlap on the GPU (other streams, other threads) race on them.
 * The first call on a device looks up their device addresses, sets kernel
 * attributes and fills the tables of every supported length (later calls
 * only read them); make that first call before any stream capture.  Errors are
 * reported by ibpm_last_error(NULL).
 */
int ibpm_lap_inv_noalloc(int32_t nx, int32_t ny, const double* rhs, double* x, void* stream);

/*
 * Objective of the discrete adjoint: the time average, over the last `window`
 * of the steps run, of the force coefficients summed over the bodies,
 *   J = (1/window) Σ_{n > nsteps-window} Σ_j (w_cd CD_j(n) + w_cl CL_j(n)),
 * CD/CL those of update_stress! (timestepping.jl:330-354).
 */
typedef struct ibpm_objective {
    int32_t window;
    double  w_cd, w_cl;
} ibpm_objective;

/*
 * Discrete adjoint of `nsteps` steps of advance! from the current state (no
 * counterpart in the reference, which has the forward step and a linearised
 * problem, problem-types.jl:47-87).  The forward run stores a checkpoint of
 * the state every `k_checkpoint` steps; the reverse sweep recomputes each
 * segment from its checkpoint and applies the transpose of the step's
 * derivative backwards.  Outputs (any may be NULL):
 *   J            the objective
 *   grad_Gamma0  ∂J/∂Γ at the start, (nΓ, mg) like Γ (Γ and q as independent)
 *   grad_q0      ∂J/∂q at the start, (nq, mg) like q
 *   grad_omega0  ∂J/∂ω for a start state built from a finest-level vorticity
 *                ω as Γ = coarsify([h²ω, 0, …]), (ψ, q) = vort2flux!: (nΓ, 1)
 *   grad_alpha   ∂J/∂α, α the freestream angle of the uniform base flux
 *   grad_xb      ∂J/∂xb, the body-point positions, (nb, 2) column-major like
 *                desc.xb (ds held fixed); B = E M E' is differentiated with E
 * The handle is left at the final state of the run, as after ibpm_advance.
 * Device memory: k tape entries (Γ and q; with grad_xb also F̃b and the
 * level-1 q of each step) and nsteps/k checkpoints.
 * The smoothed delta of interface-coupling.jl:24-61 jumps by up to ~3e-9 at
 * |r| = h, 2h, 3h (rounded coefficients); grad_xb is the derivative of the
 * pieces, so finite differences agree with it where no grid sample sits at
 * such a distance (a body point on a grid line puts samples exactly there).
 */
int ibpm_adjoint_run(ibpm_handle* h, int32_t nsteps, int32_t k_checkpoint,
                     const ibpm_objective* obj, double* J, double* grad_Gamma0,
                     double* grad_q0, double* grad_omega0, double* grad_alpha,
                     double* grad_xb);

/*
 * Device time of the adjoint of one step (after an ibpm_adjoint_run), for
 * measurement: `nsteps` graph replays, one CUDA-event pair each, L2 flushed
 * between replays when flush_l2 != 0.  step_ms receives nsteps values.
 */
int ibpm_adjoint_bench(ibpm_handle* h, int32_t nsteps, int32_t flush_l2, double* step_ms);

/*
 * Batches of independent simulations (no counterpart in the reference, which
 * runs one problem per IBProblem).  Members may differ in grid size, levels,
 * Reynolds number, time step, bodies and precision; each is an ordinary
 * handle (ibpm_batch_member) whose state is set and read with
 * ibpm_set_state / ibpm_get_state.  One batch step is one CUDA-graph launch
 * whose branches are the steps of its units spread over `lanes` concurrent
 * streams: a unit is a member, or a group of members of one grid and
 * precision stepped by shared launches (ibpm_batch_grouped).  lanes = 0
 * picks shared launches or not, the level chain, the single-slab plan and
 * the lane count (powers of two up to the number of units) by timing a few
 * steps of each, then lets each group try the other chains and plans on its
 * own; the members are reset to their created state afterwards.  Members
 * must be stepped through the batch only.
 */
typedef struct ibpm_batch ibpm_batch;
int ibpm_batch_create(int32_t n, const ibpm_problem_desc* descs, int32_t lanes, ibpm_batch** out);
int ibpm_batch_destroy(ibpm_batch* b);
ibpm_handle* ibpm_batch_member(ibpm_batch* b, int32_t i);
/* Lane count in use; set it explicitly (1 … n; the state is kept). */
int ibpm_batch_lanes(const ibpm_batch* b);
int ibpm_batch_set_lanes(ibpm_batch* b, int32_t lanes);
/* Text of the last error of the batch (or of the last failed create if b is NULL). */
const char* ibpm_batch_last_error(const ibpm_batch* b);
/* Advance every member by nsteps steps of advance! (timestepping.jl:35-67). */
int ibpm_batch_advance(ibpm_batch* b, int32_t nsteps);
/* CD/CL histories of member i over the last ibpm_batch_advance, [nsteps][nbodies_i]. */
int ibpm_batch_get_forces(const ibpm_batch* b, int32_t i, double* CD, double* CL);
/* Device time of each of nsteps batch steps (CUDA events; L2 flushed between steps if flush_l2). */
int ibpm_batch_bench(ibpm_batch* b, int32_t nsteps, int32_t flush_l2, double* step_ms);

/* Transform plan of the members' single-slab launches (IBPM_PLAN_*): the one
 * lanes = 0 chose with the lane count, or the one set; setting it sets every
 * member's and captures the batch step again (the state is kept).  lanes = 0
 * may then give a group of members of one grid another plan or level chain
 * (ibpm_get_transform_plan and ibpm_get_level_chain of a member tell). */
int ibpm_batch_plan(const ibpm_batch* b);
int ibpm_batch_set_plan(ibpm_batch* b, int32_t plan);
/* Level chain of the members (IBPM_CHAIN_*): the one lanes = 0 chose, or the
 * one set; setting it captures the batch step again (the state is kept). */
int ibpm_batch_chain(const ibpm_batch* b);
int ibpm_batch_set_chain(ibpm_batch* b, int32_t chain);
/* Shared launches (1) or not (0): members of one grid (nx, ny, mg), precision
 * and sweep count, with fixed bodies, form groups whose step fields share
 * device arenas; a group steps by launches over the slabs of all its members
 * (the body operators run per member), which computes bit for bit what each
 * member computes alone.  lanes = 0 times both; setting it captures the batch
 * step again (the state is kept).  A member is released with its batch
 * (ibpm_destroy refuses it). */
int ibpm_batch_grouped(const ibpm_batch* b);
int ibpm_batch_set_grouped(ibpm_batch* b, int32_t on);

/* Page-locked host memory for state mirrors (faster get/set_state); NULL on
 * failure.  No counterpart in the reference (Julia arrays are pageable). */
void* ibpm_host_alloc(int64_t bytes);
int ibpm_host_free(void* p);

/* ---- Measurement (no counterpart in the reference, which times runs with
 * @elapsed around run_sim!, src/ibpm.jl:71) ---------------------------- */

/* Kernel classes reported by ibpm_profile. */
#define IBPM_KERNEL_COUNT 12 /* trial_rhs, dst_x, dst_y, coarsify, curl, E_gather,
                                binv_gemv, stress, proj_src, adjoint, resid,
                                bt_chain (the line samples and edge chain of
                                the boundary-transfer vort2flux!) */

/* Name of kernel class k (0 <= k < IBPM_KERNEL_COUNT). */
const char* ibpm_kernel_name(int32_t k);

/* Plans of the 2-D sine transforms (no counterpart in the reference, which
 * calls FFTW's r2r plans, src/fluid-operators/dst-inversion.jl:10-20).  A plan
 * fixes the FFT factorisation and the threads per line pair:
 *   IBPM_PLAN_LATENCY     radix 4, N/4 threads per line pair: the shortest
 *                         chain per launch, for launches too small to fill
 *                         the GPU (a single level of one simulation);
 *   IBPM_PLAN_THROUGHPUT  radix 8, N/8 threads: about two thirds of the
 *                         instructions, for launches that fill the GPU.
 *   IBPM_PLAN_AUTO        (multi-slab launches only) the throughput plan for
 *                         launches of 4 or more slabs (the all-level
 *                         launches of a step, the columns of B,
 *                         the unit solves of moving bodies), else the
 *                         single-slab plan (the levels of one step).
 * From N = 1024 on both are the radix-8 plan.  A handle starts with the
 * latency plan for single-slab launches and IBPM_PLAN_AUTO for multi-slab
 * ones; ibpm_batch_create with lanes = 0 chooses its members' single-slab
 * plan by timing.  Results agree to rounding (the factorisations differ).
 * Setting a plan captures the step graphs again on the next advance.  B⁻¹
 * of fixed bodies is built at create with the latency plan on every launch,
 * whatever plans are set later. */
#define IBPM_PLAN_LATENCY    0
#define IBPM_PLAN_THROUGHPUT 1
#define IBPM_PLAN_AUTO       2
int ibpm_set_transform_plan(ibpm_handle* h, int32_t single_slab, int32_t multi_slab);
int ibpm_get_transform_plan(const ibpm_handle* h, int32_t* single_slab, int32_t* multi_slab);

/* How vort2flux! (src/fluid-operators/curl.jl:133-165) runs its level chain
 * (no counterpart in the reference, whose levels are solved one after another):
 *   IBPM_CHAIN_SEQUENTIAL         the reference's order, level mg first, each
 *                                 level's Δ⁻¹ after the coarser one: three
 *                                 transform launches of one level each;
 *   IBPM_CHAIN_BOUNDARY_TRANSFER  every level's interior part in one launch per
 *                                 pass and the edge values of all levels from a
 *                                 rank-k factorisation of get_bc! ∘ Δ⁻¹ ∘
 *                                 apply_bc!: fewer, wider launches, more
 *                                 transform work in all.
 * Results agree to rounding.  A handle with mg >= 2 starts with the boundary
 * transfer where its factors exist (their numerical rank below 1024), else
 * sequentially; setting the boundary transfer on a handle without factors
 * builds them (IBPM_ERR_UNSUPPORTED if they do not exist).  ibpm_batch_create
 * with lanes = 0 chooses its members' chain by timing (a batch fills the GPU
 * with its members, where the sequential chain does less work).  Setting a
 * chain captures the step graphs again on the next advance. */
#define IBPM_CHAIN_SEQUENTIAL        0
#define IBPM_CHAIN_BOUNDARY_TRANSFER 1
int ibpm_set_level_chain(ibpm_handle* h, int32_t chain);
int ibpm_get_level_chain(const ibpm_handle* h, int32_t* chain);

/* Number of kernel launches in one step (one replay of the step graph). */
int ibpm_launches_per_step(ibpm_handle* h);

/* Advance nsteps steps as graph replays and return each step's device time
 * (CUDA events on the handle's stream) in step_ms[nsteps].  With flush_l2, a
 * 512 MiB buffer is written between steps, outside the timed event pairs, so
 * each step starts with a cold L2. */
int ibpm_bench(ibpm_handle* h, int32_t nsteps, int32_t flush_l2, double* step_ms);

/* Advance nsteps steps, each a replay of a step graph captured with a CUDA
 * event pair around every kernel, and accumulate per kernel class the device
 * milliseconds, algorithmic bytes (each operand read once, each result written
 * once) and launch counts into ms_out / bytes_out / calls_out
 * [IBPM_KERNEL_COUNT].  The event nodes serialise the kernels, so the sum is a
 * little above the plain graph's step time. */
int ibpm_profile(ibpm_handle* h, int32_t nsteps, int32_t flush_l2, double* ms_out,
                 double* bytes_out, int32_t* calls_out);

#ifdef __cplusplus
}
#endif

#endif /* IBPM_GPU_H */
