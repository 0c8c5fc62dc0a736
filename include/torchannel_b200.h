/*
 * torchannel_b200 -- C ABI of the B200-native TorChannel time step.
 *
 * The reference (gmcavallazzi/torChannel) is pure Python/PyTorch and has no
 * FFI of its own; each entry point below replaces the Python function named
 * beside it, and the Python package torchannel_b200 binds them with ctypes
 * (torchannel_b200/_lib.py) behind a ChannelFlow-compatible class.
 *
 * Conventions
 *  - Every entry returns an int status (TC_OK = 0); no C++ exception crosses
 *    the ABI.  tc_last_error() gives a message for the last failure.
 *  - Array arguments are DEVICE pointers to FP64 arrays in the reference
 *    layout (C order (x, y, z), z fastest, ghosts included):
 *      u (nx+1, ny+2, nz+2), v (nx+2, ny+1, nz+2), w (nx+2, ny+2, nz+1),
 *      p (nx+2, ny+2, nz+2), cell fields such as div (nx, ny, nz).
 *    Host pointers are marked "host".
 *  - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *    stream).  Entries are asynchronous unless they return a host value.
 *  - The library never allocates device memory: the caller allocates one
 *    workspace of tc_workspace_bytes() bytes and hands it to tc_create().
 */
#ifndef TORCHANNEL_B200_H
#define TORCHANNEL_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TC_OK = 0,
  TC_ERR_ARG = 1,         /* bad argument / null pointer */
  TC_ERR_SIZE = 2,        /* unsupported grid size (nx, ny even, >= 8, factors 2 and 3 only; 4 <= nz <= 512;
                             nx * ny * (nz + 1) < 2^32) */
  TC_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  TC_ERR_WORKSPACE = 4,   /* workspace too small or misaligned */
  TC_ERR_STATE = 5,       /* call needs a state set with tc_set_state first */
  TC_ERR_NONFINITE = 6    /* non-finite value found in the state */
};

enum { TC_FP64 = 0, TC_MIXED = 1 };             /* storage precision of the fields */
enum { TC_TOP_NOSLIP = 0, TC_TOP_FREESLIP = 1 }; /* boundary_conditions.top_wall.type dirichlet / neumann */
enum { TC_RHS_SEPARATE = 0, TC_RHS_FUSED = 1 };  /* which reference code path the explicit RHS follows */
enum { TC_IMEX = 0, TC_AB2 = 1, TC_FE = 2 };     /* time.scheme */

typedef struct tc_grid_desc {
  int nx, ny, nz;          /* grid.nx, grid.ny, grid.nz */
  double Lx, Ly, Lz;       /* domain.Lx, Ly, Lz */
  double nu;               /* 1 / flow.Re */
  double U_bulk;           /* flow.U_bulk (PI forcing target) */
  int top_wall;            /* TC_TOP_* */
  int precision;           /* TC_FP64 or TC_MIXED */
  int rhs_path;            /* TC_RHS_* */
  const double* dz_f;      /* host, nz      (utils.py:42) */
  const double* dz_c;      /* host, nz + 1  (utils.py:43) */
} tc_grid_desc;

typedef struct tc_ctx tc_ctx;

/* Library version string (host). */
const char* tc_version(void);

/* Message of the last failed call in this thread (host). */
const char* tc_last_error(void);

/* Bytes of device workspace needed for this grid (includes 256 B alignment
 * slack).  Replaces the tensor allocations of ChannelFlow.__init__
 * (solver.py:215-292, initflow.py:6-9, projection_fft.py:56-86). */
int tc_workspace_bytes(const tc_grid_desc* g, size_t* bytes);

/* Create a context on the current device over a caller-owned workspace.
 * Synchronous (uploads grid tables).  Replaces initialize_fft_solver
 * (projection_fft.py:3-99) and the grid set-up of solver.py:215-234. */
int tc_create(const tc_grid_desc* g, void* workspace, size_t bytes, tc_ctx** out);

int tc_destroy(tc_ctx* ctx);

/* Load u, v, w (reference layout, device, FP64) and the bulk forcing; the
 * AB2 history is cleared (next IMEX/AB2 step is an Euler step, as after
 * ChannelFlow.__init__ / a restart, solver.py:377-383).  Ghost values are
 * ignored: periodic and wall ghosts are implied by the DOFs. */
int tc_set_state(tc_ctx* ctx, const double* u, const double* v, const double* w, double forcing, void* stream);

/* Write u, v, w, p in the reference layout with ghosts filled as
 * apply_bc_all (solver.py:23-79) and the pressure ghost fill
 * (projection_fft.py:148-163) leave them.  Any pointer may be NULL. */
int tc_get_state(tc_ctx* ctx, double* u, double* v, double* w, double* p, void* stream);

/* AB2 history r_prev (the rhs_*_prev buffers of solver.py:377-383,649-651),
 * DOFs in the u/v/w reference layouts (ghost entries written as 0).
 * tc_get_history returns TC_ERR_STATE when there is no history yet. */
int tc_get_history(tc_ctx* ctx, double* ru, double* rv, double* rw, void* stream);
int tc_set_history(tc_ctx* ctx, const double* ru, const double* rv, const double* rw, void* stream);

/* Advance n_steps steps of `scheme` with time step dt.
 *   TC_IMEX: ChannelFlow.step_imex (solver.py:580-710)
 *   TC_AB2 : step_imex with the full-diffusion RHS of
 *            compute_momentum_rhs_explicit (solver.py:498-534) and no
 *            implicit solve (docs/NUMERICAL_METHODS.md:260-284)
 *   TC_FE  : step_forward_euler (solver.py:537-576; forcing fixed at 1.0)
 * Asynchronous; u_bulk and forcing stay on the device (tc_scalars). */
int tc_step(tc_ctx* ctx, int scheme, double dt, int n_steps, void* stream);

/* Replay of captured steps: with n_steps >= 4, once the AB2 history exists
 * and the CN tables match dt, tc_step captures two consecutive steps into a
 * CUDA graph (once per scheme / dt / buffer parity) and replays it; this
 * switch turns that off (on by default).  No reference counterpart (the
 * reference captures only its Poisson solve, solver.py:389-414). */
int tc_use_graphs(tc_ctx* ctx, int on);

/* Form of the Poisson middle, the y transform, the z tridiagonal solve and
 * the inverse y transform of projection_fft.py:117-139.  on = 0 (the
 * default): three kernels with register-resident transforms; 1: one kernel
 * per kx slab on a thread-block cluster (same arithmetic up to rounding of
 * the chunked sweeps); 2: two streaming passes over each kx slab, the y
 * transform with the forward elimination and the back substitution with the
 * inverse y transform (bitwise the same results as 0; register y lengths of
 * at most 256 points).  TC_ERR_SIZE when a form is asked for a grid it does
 * not support, TC_ERR_ARG for another value.  No reference counterpart. */
int tc_use_fused_poisson(tc_ctx* ctx, int on);

/* Staging of the explicit-RHS kernel: mode 1 .. 6 (1 is the default where
 * the grid allows it: x rows a multiple of 16 bytes, nx >= 64, ny >= 16), its
 * u, v, w tiles reach shared memory by 3-D tensor copies of the tensor memory
 * accelerator, in the tile shape the mode names (planes per tile, one stage
 * per CTA or a persistent two-stage pipeline; tc_capi.cu lists them with
 * their measured times); 0: by per-thread loads.  Same arithmetic,
 * bit-identical results.  TC_ERR_SIZE when a mode is asked where tensor
 * copies are not available.  No reference counterpart. */
int tc_use_tma_rhs(tc_ctx* ctx, int on);

/* y transforms of the Poisson solve (projection_fft.py:117-139 along y):
 * on (register y lengths), the rows of X reach shared memory and return by
 * bulk copies of the tensor memory accelerator; off (the default, which
 * measures faster on B200), by per-lane loads and stores.  Same arithmetic, bit-identical results.
 * TC_ERR_SIZE when asked where not available.  No reference counterpart. */
int tc_use_bulk_ffty(tc_ctx* ctx, int on);

/* Single-precision Poisson step (TC_MIXED contexts; TC_ERR_ARG otherwise):
 * the pressure solve of every IMEX step (projection_fft.py:101-215) with an
 * FP32 spectrum -- x transform, y transforms and the z tridiagonal solves of
 * all but the lowest wavenumbers in FP32, the (kx, ky) = (0,0) mode and the
 * modes with kx < 3 and |ky| < 3 solved in FP64 -- for the increment of p
 * over the previous step's pressure p_prev: the CN kernel takes
 * dt grad p_prev out of the velocity before the divergence is formed, and
 * the projection applies the increment's gradient (the same projected
 * velocity, since the projection removes every discrete gradient).  FP32
 * rounding then scales with the change of p over one step, not with p, whose
 * FP32 rounding alone would leave a post-projection divergence of about 1e-5
 * on stretched grids.  The first `warm_steps` steps after tc_set_state (and
 * every step until a previous pressure exists, and AB2 / FE steps) use the
 * FP64 solve.  y transform, z solve and inverse y transform run as one kernel
 * per kx slab with the slab in shared memory: TC_ERR_SIZE unless nx has a
 * register transform, ny = 16 K (K <= 24) and the slab (ny * nz * 8 bytes
 * plus tables) fits one CTA's shared memory (e.g. 192 x 128).  p from
 * tc_get_state is then FP32-rounded.  No reference counterpart (the reference
 * solves in its field precision, FP64). */
int tc_use_fp32_poisson(tc_ctx* ctx, int on, int warm_steps);

/* Initial projection of a fresh field: div -> Poisson -> u -= grad p
 * (dt = 1) (solver.py:345-370). */
int tc_project_initial(tc_ctx* ctx, void* stream);

/* Device pointer to the FP64 scalar block: [0] forcing, [1] u_bulk of the
 * last step, [2] CFL 1/dt scale, [3] max|div|, [4] u-plane mean at the
 * bottom, [5] at the top, [6] non-finite flag. */
int tc_scalars(tc_ctx* ctx, double** dev_ptr);

/* Set the bulk forcing scalar (solver.py:249,252). */
int tc_set_forcing(tc_ctx* ctx, double forcing, void* stream);

/* Bulk velocity of the current state (utils.py:207-223) -> host. Syncs. */
int tc_bulk_velocity(tc_ctx* ctx, double* out_host, void* stream);

/* max over cells of the CFL sums (compute_cfl_fused, operators.py:1232-1333)
 * -> host.  Syncs. */
int tc_cfl(tc_ctx* ctx, double* dti_host, void* stream);

/* Diagnostics -> host (syncs): out[0] max|div| (utils.py:226-240),
 * out[1] u_tau (utils.py:176-204), out[2] u_bulk, out[3] forcing,
 * out[4] 1 if u, v, w or p holds a NaN/Inf (solver.py:865-868). */
int tc_diagnostics(tc_ctx* ctx, double* out_host, void* stream);

/* Divergence of the current state, (nx, ny, nz) reference layout
 * (compute_divergence, utils.py:226-240). */
int tc_divergence(tc_ctx* ctx, double* div, void* stream);

/* Operator hooks on the current state (used by the parity tests):
 * explicit RHS without forcing (compute_momentum_rhs_fused_imex /
 * separate ops, or the full-diffusion variants when full != 0), written to
 * u/v/w-shaped reference arrays with zero ghosts. */
int tc_explicit_rhs(tc_ctx* ctx, int full, double* ru, double* rv, double* rw, void* stream);

/* CN implicit z-diffusion of the current state in place
 * (solve_implicit_diffusion_u/v/w, operators.py:563-811). */
int tc_implicit_diffusion(tc_ctx* ctx, double dt, void* stream);

/* Standalone FFT Poisson solve: rhs (nx, ny, nz) reference layout, device
 * FP64 -> p (nx+2, ny+2, nz+2) with ghosts (solve_poisson_fft,
 * projection_fft.py:101-165; the (0,0) mode is gauged, so p is defined up to
 * a constant).  Uses the context's workspace; the state is not touched. */
int tc_poisson_solve(tc_ctx* ctx, const double* rhs, double* p, void* stream);

/* Same solve as tc_poisson_solve for callers that cannot allocate device
 * memory (their device memory belongs to a host application's own pool, or
 * they must not risk the device-wide synchronisation of cudaMalloc/cudaFree):
 * no context, no workspace, and no allocation of any kind.  No counterpart in
 * the reference.  dz_f (nz) and dz_c (nz+1) are DEVICE arrays; rhs and p as in
 * tc_poisson_solve; FP64; all four must be device (or managed) memory of the
 * current device, else TC_ERR_ARG before any launch.  The scratch is one
 * static 64 MiB (67108864-byte) array in device memory per GPU that loads the
 * library, held until the process exits.  A grid needs
 * nx*ny*nz*8 + (nx/2+1)*ny*nz*16 bytes plus six small tables (each region
 * rounded up to 256 bytes), about 16.1 bytes per grid point: 144x144x192
 * (64153088 bytes) and 162x128x201 (exactly 67108864) fit, 162x128x202,
 * 162x162x162 or 128x128x256 do not and get TC_ERR_SIZE before any GPU
 * work.  The first call in each CUDA context (per
 * device, and again in a context made after cudaDeviceReset) sets kernel
 * attributes and reads occupancy figures there: make that first call before
 * any stream capture.  The array's address is looked up on every call.  All
 * calls share the array, so calls that overlap on the GPU (other streams,
 * other host threads) race; serialise them. */
int tc_poisson_solve_noalloc(int nx, int ny, int nz, double Lx, double Ly, const double* dz_f,
                             const double* dz_c, const double* rhs, double* p, void* stream);

/* Velocity correction with a given p (reference layout, device)
 * (project_velocity, projection.py:143-165). */
int tc_project(tc_ctx* ctx, const double* p, double dt, void* stream);

/* Turbulence statistics (turbstats.py:20-228).  tc_stats_init picks the
 * z+ planes (turbstats.py:52-69) from z_c (host, nz+2) and clears the FP64
 * running sums; tc_stats_accumulate adds one sample of the current state;
 * tc_stats_read copies the sums to host arrays: prof (5*nz: U, uu, vv, ww, uw)
 * and spec (4*(nx/2)*(ny/2): E_uu, E_vv, E_ww, E_uw, each (nx/2, ny/2)
 * C order) and the sample count; tc_stats_write loads sums back (restart,
 * turbstats.py:364-402). */
int tc_stats_init(tc_ctx* ctx, const double* z_c, double Re_tau_target, double z_plus_target,
                  int* k_bot, int* k_top);
int tc_stats_accumulate(tc_ctx* ctx, void* stream);
int tc_stats_read(tc_ctx* ctx, double* prof_host, double* spec_host, int* n_samples);
int tc_stats_write(tc_ctx* ctx, const double* prof_host, const double* spec_host, int n_samples);

/* Per-phase timing of tc_step with CUDA events recorded between the
 * kernels on the launching stream (off by default).  Phases:
 * TC_PH_RHS (kernel a), TC_PH_CN (b), TC_PH_FFTX, TC_PH_FFTY, TC_PH_TRI,
 * TC_PH_IFFTY, TC_PH_IFFTX (c), TC_PH_PROJ, TC_PH_FIN (d).
 * tc_timing_read syncs and returns the summed milliseconds per phase over
 * the recorded steps (the last TC_TIMING_RING steps at most) and the number
 * of steps summed; it clears the record.  Has no reference counterpart (the
 * reference prints wall time only, solver.py:800-805). */
enum { TC_PH_RHS = 0, TC_PH_CN, TC_PH_FFTX, TC_PH_FFTY, TC_PH_TRI, TC_PH_IFFTY, TC_PH_IFFTX, TC_PH_PROJ,
       TC_PH_FIN, TC_NPHASE };
#define TC_TIMING_RING 64
int tc_timing_enable(tc_ctx* ctx, int on);
int tc_timing_read(tc_ctx* ctx, double* ms_host, int* n_steps);

/* Read and clear the device error word (syncs). */
int tc_error(tc_ctx* ctx, int* code_host);

/* Bounds-checked builds (the library compiled with -DTC_BOUNDS_CHECK,
 * torchannel_b200.build.build_checked): *flag = 1 when a checked access of a
 * step kernel fell outside its buffer since the last call (the access was
 * skipped), with *where = file id * 100000 + source line of the first one;
 * 0 otherwise.  Both are cleared.  In the normal build *flag = -1 (no checks
 * compiled in).  Syncs the device.  No reference counterpart. */
int tc_bounds_error(int* flag, int* where);

/* ---- Adjoint of the IMEX step (FP64 contexts; TC_ERR_ARG otherwise) ------
 * No counterpart in the reference, which has no adjoint.  Reverse-mode
 * derivatives of solver.py:580-710 for gradients of an objective of the flow
 * (e.g. a time-averaged kinetic energy) with respect to the initial field and
 * a body-force field.  Arrays are in the internal layout: u and v hold nz
 * planes of nx*ny values (x fastest), w holds nz+1 face planes whose wall
 * planes 0 and nz stay 0; buffers of tc_internal_doubles' field size
 * ((nz+1)*nx*ny) fit all three.  All calls are asynchronous on `stream`.
 *
 * tc_adjoint_scratch_bytes: size of the scratch every adjoint call takes
 *   (16-byte aligned; the CN adjoint tables are cached in it per dt).
 * tc_set_body_force: a body force F (caller-owned, internal layout) added to
 *   the explicit right-hand side of every following step (R += F); null
 *   pointers remove it.
 * tc_internal_doubles / tc_save_internal / tc_load_internal: a flat record of
 *   the step state (u, v, w, the AB2 history r_u, r_v, r_w, each
 *   (nz+1)*nx*ny doubles, then the forcing) for checkpoints.
 * tc_kinetic_energy: *acc += weight * (1/(2V)) sum W q^2 of the current state
 *   (W = cell volume dx dy dz_f for u, v; face volume dx dy dz_c for w).
 * tc_adjoint_ke_seed: lambda += weight * W q / V (the gradient of that term).
 * tc_adjoint_rhs: lambda += (nu Dxy - dA[q])^T lambda_R, the transposed
 *   linearised explicit right-hand side of operators.py:126-247, 474-548 at q.
 * tc_adjoint_cn: lambda <- (Cz^-1 Bz)^T lambda, the transposed CN solve of
 *   operators.py:563-811 for dt.
 * tc_adjoint_project: lambda <- P^T lambda, P the FFT projection
 *   (projection_fft.py, projection.py:143-165); P^T = W P W^-1.
 * tc_adjoint_step: one reverse IMEX step.  In: q (the forward state before
 *   the step), lambda (adjoint of the state after it), lambda_r (adjoint of
 *   the history the step writes), mu (device scalar, adjoint of the forcing
 *   after the step).  Out, in place: the adjoints of the state, history and
 *   forcing before the step; lambda_F (optional) accumulates the body-force
 *   gradient.  `first` marks a step taken without history (Euler start). */
int tc_adjoint_scratch_bytes(tc_ctx* ctx, size_t* bytes);
int tc_set_body_force(tc_ctx* ctx, const double* fu, const double* fv, const double* fw);
int tc_internal_doubles(tc_ctx* ctx, size_t* n);
int tc_save_internal(tc_ctx* ctx, double* dst, int* have_hist, void* stream);
int tc_load_internal(tc_ctx* ctx, const double* src, int have_hist, void* stream);
int tc_kinetic_energy(tc_ctx* ctx, double weight, double* acc, void* scratch, void* stream);
int tc_adjoint_ke_seed(tc_ctx* ctx, double weight, const double* qu, const double* qv, const double* qw,
                       double* lu, double* lv, double* lw, void* stream);
int tc_adjoint_rhs(tc_ctx* ctx, const double* qu, const double* qv, const double* qw, const double* Ru,
                   const double* Rv, const double* Rw, double* lu, double* lv, double* lw, void* stream);
int tc_adjoint_cn(tc_ctx* ctx, double dt, double* lu, double* lv, double* lw, void* scratch, void* stream);
int tc_adjoint_project(tc_ctx* ctx, double* lu, double* lv, double* lw, void* scratch, void* stream);
int tc_adjoint_step(tc_ctx* ctx, double dt, int first, const double* qu, const double* qv, const double* qw,
                    double* lu, double* lv, double* lw, double* lru, double* lrv, double* lrw,
                    double* lFu, double* lFv, double* lFw, double* mu, void* scratch, void* stream);

/* Per-step hooks for the adjoint driver (FP64 contexts; no reference
 * counterpart).  Both run inside tc_step (and its captured graphs) after the
 * projection and read their switches from device memory, so changing the
 * values needs no re-capture.
 * tc_set_ke_accumulator: after every step, *acc += (*weight_dev) * KE(state)
 *   (KE as tc_kinetic_energy; a zero weight skips the work); null acc removes
 *   it.  The scratch holds the partial sums (tc_adjoint_scratch_bytes).
 * tc_set_state_tape: after every step, when 0 <= *ctr_dev < nslots, copy
 *   u, v, w of the new state into slot *ctr_dev of `tape` (slot stride
 *   3 (nz+1) nx ny doubles) and increment *ctr_dev; null tape removes it. */
int tc_set_ke_accumulator(tc_ctx* ctx, double* acc, const double* weight_dev, void* scratch);
int tc_set_state_tape(tc_ctx* ctx, double* tape, int nslots, int* ctr_dev);

/* Tile shape of the CN solve along z: rows per chunk (1 .. 32; 0 = by nz:
 * 16 up to nz = 256, else 32).  Used by the autotuners and the ensemble
 * launches; no reference counterpart.  TC_ERR_SIZE when a column would need
 * more than 16 chunks. */
int tc_set_cn_chunk(tc_ctx* ctx, int rows);

/* ---------------------------------------------------------------------------
 * Ensembles: one launch per substep for every member.
 *
 * No reference counterpart (the reference steps one ChannelFlow at a time;
 * an ensemble there is a loop of ChannelFlow.step_imex calls,
 * solver.py:580-710).  An ensemble groups up to 64 existing contexts of one
 * precision on one device whose nx and ny are 64, 96, 128, 192 or 256; each
 * substep (RHS, CN, x / y transforms, z solve, inverse transforms,
 * projection) of every member runs as ONE launch over the concatenated work
 * of all members (the CN: one launch per chunk count; the x transforms:
 * one per transform length each; the tensor-copy RHS: one per 32 members),
 * and tc_batch_step with n_steps >= 4 replays two such steps as
 * one CUDA graph.  Each member advances exactly
 * as tc_step would advance it (same kernels' tile code; bit-identical with
 * the same CN chunk length), its scalars, statistics and state entries stay
 * per context, and members may still be stepped on their own between
 * ensemble calls (the ensemble rebuilds its tables when it notices).
 * The caller owns the member-table memory (device, 16-byte aligned, size
 * from tc_batch_table_bytes); all calls on one stream.
 * tc_batch_set_shape: CN rows per chunk (16 or 32: every member's CN
 *   chunks take that many rows and its tables follow; the deepest member's
 *   chunk count fixes the CN block, whose warps beyond a shallower member's
 *   last chunk idle) and persistent CTAs per SM (0 = occupancy limit,
 *   -1 = one CTA per work unit; the CN and x-transform launches always
 *   take one CTA per unit), the ensemble autotuner's knobs.
 * tc_batch_step: dts = host array of one dt per member; members without AB2
 *   history start with a forward step as tc_step does.  Members may carry no
 *   adjoint hooks (TC_ERR_ARG).  The RHS launch stages its tiles by tensor
 *   copies (one work unit per tile of the tensor-copy RHS) while every
 *   member has tc_use_tma_rhs mode 1 on, and by per-thread loads otherwise;
 *   switching a member rebuilds the tables at the next call.
 * tc_batch_info: shape = {cn rows, ctas per SM (-1: one CTA per work
 *   unit), tables built, CN chunk warps per block (the deepest member's
 *   chunks)}; units and
 *   grids = work units and CTAs of the seven launches (RHS, CN, x transform,
 *   y transform, z solve, inverse x transform, projection). */
typedef struct tc_batch tc_batch;
int tc_batch_table_bytes(int n_members, int precision, size_t* bytes);
int tc_batch_create(tc_ctx* const* members, int n_members, void* table, size_t table_bytes, tc_batch** out);
int tc_batch_destroy(tc_batch* b);
int tc_batch_set_shape(tc_batch* b, int cn_rows, int ctas_per_sm);
int tc_batch_use_graphs(tc_batch* b, int on);
int tc_batch_step(tc_batch* b, int scheme, const double* dts, int n_steps, void* stream);
int tc_batch_info(tc_batch* b, int* shape, int* units, int* grids);

#ifdef __cplusplus
}
#endif
#endif /* TORCHANNEL_B200_H */
