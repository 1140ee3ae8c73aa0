/*
 * fvmhd3d_b200: C-ABI of the B200 (sm_100a) fluid hot path of fvmhd3d.
 *
 * The reference has no plugin or FFI layer: its hot path is a sequence of
 * argument-free member functions of `struct system` (MPI/fvmhd3d.h:298-575)
 * called from system::fluid_update (MPI/iterate.cpp:95-113) inside
 * system::iterate_step (MPI/iterate.cpp:115-247), operating on member arrays.
 * This header exposes the same sequence over a context that owns the device
 * copies of those arrays.  Each entry point names the reference function it
 * replaces.
 *
 * Conventions
 *   - Return 0 on success, a negative FVM_E* code on error; the message is in
 *     fvm_last_error().  No C++ exception crosses this boundary and no kernel
 *     traps: kernels record failures in device counters read by the host.
 *   - Host buffers are owned by the caller and only read/written during the
 *     call.  Device buffers are owned by the context.
 *   - One host thread per context; all work is ordered on the context's
 *     CUDA stream.
 *   - Layouts are row-major, one record per cell or face:
 *       W, U      ncell x 10  (primitive / conserved, MPI/Fluid.h:9-32 order)
 *       dU        ncell x 14  (dU[10], gradPsi[3], divB; MPI/Fluid.h:163-172)
 *       wrec      ncell x 50  (w, x, y, z, t blocks; MPI/Fluid.h:147-161)
 *       pos, vel  ncell x 3   (generator position / velocity)
 *       n, c      nface x 3   (area-weighted normal s1->s2; centroid in the
 *                              periodic frame of s1; MPI/fvmhd3d.h:169-191)
 */
#ifndef FVMHD3D_B200_H
#define FVMHD3D_B200_H

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FVM_OK = 0,
  FVM_EINVAL = -1,    /* bad argument or call order */
  FVM_ECUDA = -2,     /* CUDA runtime error */
  FVM_ENOMEM = -3,    /* device allocation failed */
  FVM_ENOMESH = -4,   /* no mesh / state installed yet */
  FVM_ERANGE = -5,    /* a rung left [0, 32) or a size limit was exceeded */
  FVM_EIO = -6        /* a snapshot file could not be written */
};

enum { FVM_PREC_FP64 = 0, FVM_PREC_FP32 = 1 };

typedef struct fvm_params {
  double gamma;     /* system::gamma_gas */
  double courant;   /* system::courant_no */
  double box[3];    /* system::global_domain_size (periodic box) */
  double dtmax;     /* Scheduler(dtmax), MPI/Scheduler.h:17-30 */
  int eos;          /* 0: ideal gas (MPI/set_problem.cpp:123-137);
                       1: isothermal disk (MPI/problems/mri_disk3d.cpp:368-389) */
  double iso_GM;    /* disk: cs^2(r) = iso_GM/|r| * iso_cfac^2 */
  double iso_cfac;
  int precision;    /* FVM_PREC_FP64 (plain path) or FVM_PREC_FP32 */
  int static_mesh;  /* 0: compute_pvel moves generators with the flow
                       (MPI/compute_pvel.cpp:5-50); 1: static generators, the
                       compute_pvel1 hook that sets vel = 0 for every active
                       site (MPI/set_problem.cpp:61-72, acoustic_waves.cpp:6-16) */
} fvm_params;

typedef struct fvm_ctx fvm_ctx;

/* Creates a context on CUDA device `device`.  Replaces the construction of
 * `system` and its Scheduler (MPI/fvmhd3d.h:537-552, MPI/Scheduler.h:17-30). */
fvm_ctx *fvm_create(const fvm_params *p, int device);
void fvm_destroy(fvm_ctx *c);
const char *fvm_last_error(const fvm_ctx *c);

/* Installs the Voronoi mesh (copied to the device).  Replaces the cell_list /
 * face_list produced by system::build_mesh_active
 * (MPI/build_mesh_active.cpp:663-851).  cell_face_off has ncell+1 entries. */
int fvm_set_mesh(fvm_ctx *c, int ncell, int nface, const int *s1, const int *s2,
                 const double *n, const double *centroid, const double *cell_volume,
                 const double *cell_centroid, const long long *cell_face_off,
                 const int *cell_face_ids);

/* Generator positions pos[3n] and boundary codes bnd[n] (NULL: none) of the
 * installed mesh, and the tables built from them (face offsets, per-link
 * reconstruction and limiter weights, boundary-neighbour flags), without
 * touching the fluid state or orig_pos / orig_vel.  A host that rebuilds its
 * mesh every step (MPI/iterate.cpp:150) calls fvm_set_mesh, then this, then
 * fvm_set_state (or fvm_step_host) with the state it keeps; fvm_init_problem
 * does the same as part of setting up a problem.  fvm_set_state and
 * fvm_step_host refuse a mesh without positions (FVM_ENOMESH). */
int fvm_set_positions(fvm_ctx *c, const double *pos, const int *bnd);

/* Initial state from primitives W, following the tail of the reference's
 * set_problem (MPI/problems/mri_disk3d.cpp:832-880): Wrec=(W,0,0,0,0),
 * U=cons(W), dU=0, compute_pvel, compute_timesteps(true), rung += rung_offset,
 * tend = dt(rung).  bnd may be NULL (no boundary cells). */
int fvm_init_problem(fvm_ctx *c, const double *W, const double *pos, const int *bnd,
                     int rung_offset);

/* Full per-cell state between steps (any pointer may be NULL).  set_state also
 * sets the scheduler clock (integer ticks of dtmax/2^31). */
int fvm_get_state(fvm_ctx *c, double *pos, double *vel, double *tlast, double *tend, int *rung,
                  double *U, double *dU, double *wrec);
int fvm_set_state(fvm_ctx *c, const double *vel, const double *tlast, const double *tend,
                  const int *rung, const double *U, const double *dU, const double *wrec,
                  unsigned long long tsys_ticks);

/* Generator motion and divergence diagnostics between steps (any pointer may
 * be NULL): orig_pos / orig_vel as advanced by the reference's correct()
 * (MPI/set_problem.cpp:89-101) and divBi, the per-cell divB/dt/V that
 * collect_results keeps in single precision (MPI/distribute_work.cpp:681).
 * These feed the host's next mesh build and the snapshot writer. */
int fvm_get_motion(fvm_ctx *c, double *orig_pos, double *orig_vel, float *divb);

/* The scheduler clock: Scheduler::tsysU, system::dt_global (the interval the
 * last Scheduler::pull_active_list advanced, MPI/Scheduler.h:138-153) and
 * system::iteration (steps since fvm_init_problem, MPI/iterate.cpp:117).
 * Any pointer may be NULL. */
int fvm_clock(fvm_ctx *c, unsigned long long *tsys_ticks, double *dt_global, long long *iteration);

/* Writes the reference's single-rank snapshot, system::dump_binary
 * (MPI/dump_binary.cpp:5-99), byte for byte in its layout: a 20-word header
 * and one 26-word record per cell, each framed by its byte count, native
 * little-endian int32/float32.  idx (particle ids) and rmax (the mesh
 * builder's search radius) are host data the fluid path does not hold: NULL
 * writes idx = cell index and rmax = 0.  Cell volumes are the installed mesh's;
 * the current-density words are 0 (the hot path computes no J).  Returns
 * FVM_EIO if the file cannot be written. */
int fvm_dump_binary(fvm_ctx *c, const char *path, const int *idx, const float *rmax);

/* ---- the reference's step, one entry point per member function ---------- */

/* system::get_active_ptcl(false) + Scheduler::pull_active_list + the site
 * flags of build_mesh_active + system::get_active_faces
 * (MPI/iterate.cpp:12-93, MPI/Scheduler.h:108-154,
 * MPI/build_mesh_active.cpp:524-528).  Returns the number of active cells. */
int fvm_begin_step(fvm_ctx *c);
/* system::slope_limiter (MPI/compute_reconstruction.cpp:201-602) */
int fvm_slope_limiter(fvm_ctx *c);
/* system::compute_update (MPI/compute_update.cpp:22-499) */
int fvm_compute_update(fvm_ctx *c);
/* system::compute_pvel (MPI/compute_pvel.cpp:5-52) */
int fvm_compute_pvel(fvm_ctx *c);
/* system::compute_timesteps(false) + adjust_timesteps
 * (MPI/compute_timestep.cpp:54-207).  shared != 0 puts every active cell on
 * the rung of the global minimum (the effect of compute_timesteps(true)).
 * dt_min_out (may be NULL) receives the global minimum timestep. */
int fvm_compute_timesteps(fvm_ctx *c, int shared, double *dt_min_out);
/* system::collect_results + distribute_fluid_update_data
 * (MPI/distribute_work.cpp:537-797), one rank */
int fvm_collect_results(fvm_ctx *c);
/* system::compute_update0 (MPI/compute_update.cpp:695-970) */
int fvm_compute_update0(fvm_ctx *c);
/* system::compute_reconstruction (MPI/compute_reconstruction.cpp:24-199) */
int fvm_compute_reconstruction(fvm_ctx *c);
/* system::collect_reconstruction (MPI/distribute_work.cpp:799-864) and the
 * rung re-insertion of iterate_step (MPI/iterate.cpp:199-217) */
int fvm_end_step(fvm_ctx *c, int shared);

/* One full step: begin_step, slope_limiter, compute_update, compute_pvel,
 * compute_timesteps, collect_results, compute_update0, compute_reconstruction,
 * end_step.  Returns the number of active cells. */
int fvm_step(fvm_ctx *c, int shared);

/* fvm_set_state + fvm_step + fvm_get_state in one call: the step reads the
 * host state (vel[3n], tlast[n], tend[n], rung[n], U[10n], dU[14n],
 * wrec[50n], the system clock tsys_ticks as fvm_set_state takes it) and
 * writes the stepped state back into the same arrays.  The copies of U and
 * dU run on a second stream, overlapped with the stage kernels (in while the
 * face fluxes are computed, out while the later stages run), and the host
 * waits once, at the end.  The host arrays should be pinned.  A rung outside
 * [0, 31) on input returns FVM_ERANGE before anything is uploaded.  Always the stage
 * kernels; no counterpart in the reference (a drop-in that keeps the
 * reference's host arrays calls it once per fluid step).  Returns the active
 * cell count. */
int fvm_step_host(fvm_ctx *c, int shared, unsigned long long tsys_ticks, double *vel, double *tlast, double *tend,
                  int *rung, double *U, double *dU, double *wrec);

/* nsteps full steps replayed from one captured CUDA graph (the scheduler
 * runs on the device, so there is no host round trip between steps).
 * Returns the summed number of active cells; faces_out (may be NULL)
 * receives the summed number of active faces. */
int fvm_run(fvm_ctx *c, int nsteps, int shared, long long *faces_out);

/* ---- one domain of a partitioned mesh --------------------------------------
 * A rank that owns part of the cells installs its owned cells plus the rings
 * of neighbours around them as its mesh, and its host copies the neighbour
 * rows from their owners between steps (the reference's
 * distribute_particle_fluid_data / collect_results,
 * MPI/distribute_work.cpp:367-724). */

/* The reduction of the timestep minimum over ranks: MPI_Allreduce(MIN) of
 * compute_timesteps (MPI/compute_timestep.cpp:101).  Given this rank's
 * minimum in *dt_min, the function stores the minimum over ranks and returns
 * 0 (non-zero fails the step with FVM_EINVAL). */
typedef int (*fvm_reduce_fn)(void *user, double *dt_min);

/* Installs (fn != NULL) or removes the reduction.  While it is installed,
 * fvm_compute_timesteps, fvm_step and fvm_step_host wait for the rank's
 * minimum, call fn on the calling thread and continue with its result, and
 * fvm_init_problem calls it on the initial minimum; fvm_run, whose replayed
 * steps cannot call the host, returns FVM_EINVAL, and the persistent rung
 * kernel is not used. */
int fvm_set_reduce(fvm_ctx *c, fvm_reduce_fn fn, void *user);

/* Marks the installed mesh's copies of other ranks' cells (halo[i] != 0;
 * NULL: every cell is this rank's).  Their timesteps are computed but left
 * out of the minimum (a copy in the outer ring misses neighbours, so its
 * value is not its owner's).  Cleared by fvm_set_mesh. */
int fvm_set_halo(fvm_ctx *c, const unsigned char *halo);

/* ---- inspection ----------------------------------------------------------- */

double fvm_time(const fvm_ctx *c);                       /* system::t_global */
unsigned long long fvm_tsys_ticks(const fvm_ctx *c);     /* Scheduler::tsysU */
/* face_active_list of the current step as face ids, in the reference order
 * (MPI/iterate.cpp:58-93); *n receives the count.  ids may be NULL. */
int fvm_get_active_faces(fvm_ctx *c, int *ids, int *n);
/* Wrec of the current step as the reference holds it after slope_limiter:
 * x, y, z, t scaled by the per-cell limiter for imported cells. */
int fvm_get_limited_wrec(fvm_ctx *c, double *wrec);
/* dU_import after compute_update (ncell x 14). */
int fvm_get_step_dU(fvm_ctx *c, double *dU);
/* Per-cell timestep list of the last compute_timesteps (ncell). */
int fvm_get_dt_list(fvm_ctx *c, double *dt);
/* Device counters: [0] cells that took the failed-mass fallback of
 * compute_update, [1] cells whose thermal energy went non-positive. */
int fvm_get_counters(fvm_ctx *c, long long *out2);

/* Per-face known-answer entry: system::compute_flux
 * (MPI/compute_update.cpp:973-1095) on nface given face states, host
 * buffers in and out. */
int fvm_compute_flux(fvm_ctx *c, int nface, const double *wij, const double *Wi, const double *Wj,
                     const int *jbnd, const double *normal, double *psi, double *Bn, double *flux);

/* No counterpart in the reference.  fvm_compute_flux without device
 * allocation, for callers that must not allocate while they run: a host
 * integrator solving boundary or sub-grid face batches between steps while
 * other streams keep the GPU busy (fvm_compute_flux's per-call cudaFree waits
 * for the whole device), or a run holding most of HBM for its mesh, where a
 * per-call cudaMalloc can fail mid-run.  Same arguments and results as
 * fvm_compute_flux; the batch is staged in one fixed device array of
 * FVM_FLUX_STATIC_MAX_FACES faces (about 5 MB) that every call on a device
 * shares.  nface above the capacity returns FVM_ERANGE and does nothing.
 * Calls whose GPU work overlaps (several host threads, or several contexts on
 * one device, at once) race on that array; each call returns after its work
 * has finished, so calls made one after another are safe. */
#define FVM_FLUX_STATIC_MAX_FACES 16384
int fvm_compute_flux_static(fvm_ctx *c, int nface, const double *wij, const double *Wi, const double *Wj,
                            const int *jbnd, const double *normal, double *psi, double *Bn, double *flux);

/* ---- learned face flux (the MLP stand-in for riemann_solver) ------------- */

/* Network 16 -> 128 -> 128 -> 128 -> 8 with GELU hidden layers; parameters in
 * this order, row-major, FP32: W1[128x16], b1[128], W2[128x128], b2[128],
 * W3[128x128], b3[128], W4[8x128], b4[8].  Inference rounds the weights,
 * the inputs and the hidden activations to FP16 for the tensor cores (the
 * training products round their operands to BF16); biases stay FP32. */
#define FVM_MLP_NPARAM 36232
int fvm_mlp_set_weights(fvm_ctx *c, const float *params);

/* Known-answer entry: Y[n x 8] = network(X[n x 16]) on the tensor cores, host
 * buffers in and out (X rounded to FP16). */
int fvm_mlp_eval(fvm_ctx *c, int n, const float *X, float *Y);

/* The same network with the row count read on the device, as the flux
 * passes launch it: the grid is sized for nmax rows (X and Y hold nmax rows),
 * the kernel reads n (0 <= n <= nmax) from device memory and leaves rows n..
 * of Y as they were passed in. */
int fvm_mlp_eval_counted(fvm_ctx *c, int nmax, int n, const float *X, float *Y);

/* The FP32 master parameters (FVM_MLP_NPARAM floats). */
int fvm_mlp_get_weights(fvm_ctx *c, float *params);

/* Loss L = mean over rows and outputs of wt[k] (Y - T)^2 and its gradient with
 * respect to every parameter, by the training kernels' forward and backward
 * passes over all n rows at the current parameters (wt may be NULL: 1). */
int fvm_mlp_grad(fvm_ctx *c, int n, const float *X, const float *T, const float *wt, float *grad, float *loss);

/* Trains from the current parameters with Adam (beta 0.9 / 0.999): `steps`
 * updates on minibatches of `batch` rows drawn from the n pairs (X n x 16,
 * T n x 8) by a seeded hash; loss_out[steps] gets each minibatch loss (may
 * be NULL).  The tensor-core inference weights are refreshed at the end. */
int fvm_mlp_train(fvm_ctx *c, long long n, const float *X, const float *T, const float *wt, int batch, int steps,
                  float lr, unsigned long long seed, float *loss_out);

/* Learned-flux mode of the two flux passes.  mode 0: the exact HLLD solver on
 * every face (the default, restored by fvm_set_mesh); 1: faces that pass the
 * gate take the network (weights from fvm_mlp_set_weights), the others the
 * exact solver; 2: exact everywhere, and one gated face in `hstride` (hash
 * sampled) appends its (features, targets) to a device harvest buffer of
 * hcap rows.  Gate: ideal-gas EOS, no boundary neighbour, relative density
 * and pressure jumps at most drho and dp, normal Mach number in the face
 * frame at most mach, and the size of the face's scaled jump (density by
 * the mean density, velocities by the larger fast speed c, pressure by
 * rho c^2, tangential fields by sqrt(rho) c) at most jmax.  In mode 1 a face falls back to the exact solver when
 * the state either of its cells reaches from that face's network flux alone,
 * over the cell's step, keeps less than half of the cell's mass or thermal
 * energy (positivity of the updated state); one deferred face in `judge`
 * (0: none) is also solved exactly to record the network's error.  Resets
 * the statistics. */
int fvm_set_flux_mode(fvm_ctx *c, int mode, float drho, float dp, float mach, float jmax, int judge, int hstride,
                      long long hcap);

/* What stands in for the HLLD dissipation on the faces the gate passes, in
 * mode 1: 0 the network (the default), 1 none (the central flux alone), 2 the
 * local Lax-Friedrichs dissipation.  1 and 2 are comparisons for the
 * network; gate, fallback and judge work as in mode 1.  Has no counterpart in
 * the reference (an addition of the learned form). */
int fvm_set_flux_surrogate(fvm_ctx *c, int kind);

/* Standardisation of the network: inputs (features - mu_x) / sd_x; the scaled
 * dissipation of a face is m (mu_y + sd_y * network), m the size of the
 * face's scaled jump (16, 16, 8, 8 floats; identity by default). */
int fvm_mlp_set_norm(fvm_ctx *c, const float *mu_x, const float *sd_x, const float *mu_y, const float *sd_y);

/* Cumulative learned-flux statistics since fvm_set_flux_mode: [0] deferred
 * faces, [1] exact fallbacks, [2] judged faces, [3] sum over judged faces of
 * the L1 error of the 7 predicted scaled outputs, [4] sum of their L1 norms,
 * [5] the largest single-output error, [6] fallbacks of the positivity test
 * (counted in [1] too). */
int fvm_learn_stats(fvm_ctx *c, double *stats8);

/* Rows harvested so far (capped at hcap), and a copy of the first n of them
 * (X n x 16 features, Y n x 8 targets). */
long long fvm_harvest_count(fvm_ctx *c);
int fvm_get_harvest(fvm_ctx *c, long long n, float *X, float *Y);

/* Autotuner: picks, by timing `steps` trial steps per candidate on the
 * current state (restored after every trial, so the run is unchanged), the
 * limiter variant (face records staged in shared memory or not) and the
 * block sizes of the face kernels, the one-thread-per-cell gathers and the
 * two-threads-per-cell kernels.  choice (4 ints, may be NULL) receives
 * {staged limiter, face block, cell block, two-thread cell block}.  The
 * trial steps do not call the reduction of fvm_set_reduce. */
int fvm_autotune(fvm_ctx *c, int shared, int steps, int *choice);

/* Persistent rung kernel: in steps replayed by fvm_run with individual
 * timesteps, a step whose involved cells (the active ones and their
 * neighbours) number at most max_cells runs every stage from the slope
 * limiter to the reconstruction as one cooperative launch with grid-wide
 * barriers between the stages; larger steps take the stage kernels.  The
 * choice is made on the device each step; both give the same results.
 * 0 (the default) turns it off.  Learned-flux mode and per-kernel profiling
 * always take the stage kernels.  Has no counterpart in the reference (a
 * GPU batching of its per-rung fluid_update sequence). */
int fvm_set_fused(fvm_ctx *c, int max_cells);

/* Steps the persistent rung kernel has run since the state was installed
 * (as of the last fvm_run or fvm_step). */
long long fvm_fused_step_count(const fvm_ctx *c);

/* List building of partial steps (individual timesteps).  A step whose
 * active cells plus their links number at most max_entries builds its flags,
 * active-face list and involved-cell list from the active cells' links;
 * larger steps take the pass over every face and cell.  Both select the same
 * sites (MPI/iterate.cpp:58-113): the same involved cells in ascending order
 * and the same active faces (listed in the order they are found; each face
 * pass computes every face on its own, so the results are the same bits).
 * max_entries: -1 (the default) for 1/256 of the mesh's cells plus links
 * (at least 8192), 0 to turn the incremental form off, or a positive bound.  The
 * choice is made on the device each captured step (on the host for eager
 * steps).  Has no counterpart in the reference. */
int fvm_set_list_building(fvm_ctx *c, int max_entries);

/* Steps whose lists were built incrementally since the state was installed
 * (as of the last fvm_run or fvm_step). */
long long fvm_incremental_step_count(const fvm_ctx *c);

/* Sets the launch choices fvm_autotune picks (same 4 ints: staged limiter
 * 0/1, then block sizes 32, 64 or 128), e.g. to replay a tuned configuration
 * on another run of the same mesh. */
int fvm_set_tuning(fvm_ctx *c, const int *choice);

/* Timing helper: CUDA-event time in ms of the last fvm_step's kernels. */
float fvm_last_step_ms(const fvm_ctx *c);
/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or events after the context's kernels. */
void *fvm_stream(fvm_ctx *c);
/* Active cells and active faces of the last completed step. */
int fvm_last_step_counts(const fvm_ctx *c, int *ncell_active, int *nface_active);

/* adjust_timesteps diagnostics of the last individual-timestep step: sites
 * with a neighbour outside a factor 2, parallel replays run, and 1 if the
 * sequential sweep had to run instead (any pointer may be NULL). */
int fvm_last_adjust_stats(const fvm_ctx *c, int *dirty_sites, int *replays, int *sequential);
/* FP64 FMA throughput of the context's device in FLOP/s (2 per FMA), timed
 * on a full-occupancy grid of independent FMA chains: the measured peak
 * that FP64-bound kernels are compared with (after fvm_set_mesh).  No
 * counterpart in the reference (a measurement aid). */
int fvm_fp64_peak(fvm_ctx *c, double *flops_per_s);
/* Number of kernels this context has launched so far. */
long long fvm_launch_count(const fvm_ctx *c);
/* Per-kernel CUDA-event timing: on != 0 enables it and clears the totals. */
int fvm_set_profiling(fvm_ctx *c, int on);
/* Totals of kernel class k (0, 1, ...): name, summed ms and number of
 * timed launches.  Returns 1 while k is valid, 0 past the last class. */
int fvm_kernel_times(const fvm_ctx *c, int k, const char **name, double *total_ms, long long *calls);

#ifdef __cplusplus
}
#endif
#endif
