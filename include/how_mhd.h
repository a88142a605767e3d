/* how_mhd.h -- C ABI of the B200-native HOW-MHD time-step path.
 *
 * Drop-in for the reference's driver-level surface (jeongbhin/HOW-MHD-Kokkos,
 * paths inside that project).  Every entry point names the reference function
 * it replaces.  All calls return HOW_OK (0) or a negative HOW_ERR_* code; the
 * message of the last failure on the calling thread is how_last_error().
 * Nothing aborts the process.
 *
 * State layout at the boundary is the reference's: one stage of q is
 * 8 variables (rho, mx, my, mz, Bx, By, Bz, E) x (nx+6) x (ny+6) x (nz+6)
 * doubles with k fastest (LayoutRight of q(stage, var, i, j, k),
 * src/main.cpp:101-120); active cells are i,j,k in [3, n+2].  A face-B
 * component is (nx+6)x(ny+6)x(nz+6) doubles, bxb(i) being the x-face at i+1/2
 * (src/fluxct.cpp:27-35, 84-88).  The device keeps its own x-fastest layout;
 * conversion happens only on upload/download.
 *
 * All device work of a context is ordered on the context's CUDA stream.
 * Calls on one context are not thread-safe.  Device-side faults are reported
 * through status words (HOW_ERR_NONFINITE, ...), never by trapping.
 */
#ifndef HOW_MHD_H
#define HOW_MHD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HOW_OK 0
#define HOW_ERR_ARG (-1)        /* invalid argument or size                  */
#define HOW_ERR_PARSE (-2)      /* input.in value missing or invalid          */
#define HOW_ERR_PROBLEM (-3)    /* unknown problem name                       */
#define HOW_ERR_CUDA (-4)       /* CUDA runtime error (message has details)   */
#define HOW_ERR_NODEVICE (-5)   /* no CUDA device / extension not usable      */
#define HOW_ERR_NONFINITE (-6)  /* time or dt became non-finite               */
#define HOW_ERR_DT (-7)         /* non-positive dt (src/main.cpp:175-183)     */
#define HOW_ERR_STATE (-8)      /* call out of order (e.g. no state yet)      */

#define HOW_BC_PERIODIC 0
#define HOW_BC_OPEN 1

#define HOW_PREC_FP64 0         /* plain FP64 method (the reference's)        */
#define HOW_PREC_MIXED 1        /* FP32 eigen/projection/WENO, FP64 RK/CT/CFL */

/* Parameters: struct Parameters (src/parameters.hpp:10-76).  nx/ny/nz are the
 * global active-cell counts (the reference's gnx/gny/gnz; one device-resident
 * domain, so local == global).  px/py/pz are parsed and ignored, like the
 * reference's serial build (src/mpi_domain.cpp:87-90). */
typedef struct how_params {
    int nx, ny, nz;
    int nt, nstep, ntime;
    double xsize, ysize, zsize;
    double dx, dy, dz;
    double gam, cour, tend, rhomin, pgmin;
    int bc[3];                 /* x1bc, x2bc, x3bc */
    int px, py, pz;
    char problem[64];
    char output_format[16];
    /* keys added by this implementation; the reference parser warns on them
     * and skips the line (src/parameters.cpp:112-116), so input files that
     * use them stay readable by the reference. */
    int precision;             /* HOW_PREC_*                      (key: precision fp64|mixed) */
    int router;                /* 0 off, 1 learned WENO routing   (key: router off|on)        */
    uint64_t seed;             /* problem seed                    (key: seed)                 */
    double problem_par[8];     /* problem parameters              (keys: par0..par7)          */
    int ct_avg;                /* points of the face average of B_n v_t in the CT flux terms:
                                * 2 = the reference's (src/ssprk.cpp:976-989, default),
                                * 4 = fourth-order (-1, 9, 9, -1)/16  (key: ct_avg 2|4)      */
} how_params;

typedef struct how_ctx how_ctx;

/* Problem initialiser: fill stage 0 of q (reference layout, ghosts may be
 * left untouched) from the parameters.  Returns 0 on success. */
typedef int (*how_problem_fn)(double* q, const how_params* par, void* user);

/* ------------------------------------------------------------ parameters */
/* read_parameters + finalize_parameters_after_read
 * (src/parameters.cpp:7-118, 120-160): defaults, whitespace key/value pairs,
 * '#' comments to end of line, unknown keys warned to stderr and skipped;
 * validation (positive sizes, nt > 0, tend > 0) returns HOW_ERR_PARSE
 * instead of aborting.  dx = size / n. */
int how_params_default(how_params* p);
int how_parse_input(const char* path, how_params* p);
int how_parse_input_string(const char* text, how_params* p);
int how_finalize_params(how_params* p);

/* --------------------------------------------------------------- problems */
/* register_problem / RegisterProblem (src/problem.hpp:8-22).  Built-in
 * names: orszag_tang, blast3d, brio_wu, mhd_rotor, uniform, mpi_smooth3d
 * (the reference's), plus alfven3d, blast3d_b, turb3d (new). */
int how_register_problem(const char* name, how_problem_fn fn, void* user);
/* newline-separated registered names into buf; returns the count */
int how_list_problems(char* buf, size_t cap);
/* init_problem (src/problem.cpp:17-37) on the host, no device needed:
 * fills q_host (one stage, reference layout) from the registry. */
int how_problem_init_host(const how_params* p, double* q_host);

/* ---------------------------------------------------------------- context */
/* Allocates q(6 stages), face B(6 stages) and the CT arrays on the current
 * CUDA device (the reference allocates in main.cpp:114-120 and
 * allocate_bfield_ct, src/fluxct.cpp:27-35). */
int how_create(const how_params* p, how_ctx** out);
int how_destroy(how_ctx* ctx);
const char* how_last_error(void);
int how_get_params(const how_ctx* ctx, how_params* out);
/* Bytes of device memory the context holds. */
size_t how_device_bytes(const how_ctx* ctx);

/* init_problem + bound(q,0) + initialize_bfield_from_q (src/main.cpp:125-130) */
int how_init_problem(how_ctx* ctx);

/* ------------------------------------------------------------------ state */
/* Upload / download one stage (reference layout, host memory).  Pinned host
 * buffers make the copies asynchronous-capable; pageable also works. */
int how_set_state(how_ctx* ctx, int stage, const double* q_host);
int how_get_state(how_ctx* ctx, int stage, double* q_host);
int how_set_face_b(how_ctx* ctx, int stage, const double* bx, const double* by, const double* bz);
int how_get_face_b(how_ctx* ctx, int stage, double* bx, double* by, double* bz);

/* -------------------------------------------------------- path functions */
/* bound (src/bound.cpp:295-317): periodic/open ghost fill x, then y, then z */
int how_bound(how_ctx* ctx, int stage);
/* bound_bfield (src/fluxct.cpp:481-490) */
int how_bound_bfield(how_ctx* ctx, int stage);
/* initialize_bfield_from_q (src/fluxct.cpp:65-107): needs bound(q,0) first */
int how_init_bfield_from_q(how_ctx* ctx);
/* tstep (src/tstep.cpp:11-136): CFL dt from stage 0; returns it in *dt */
int how_tstep(how_ctx* ctx, double* dt);
/* ssprk (src/ssprk.cpp:1277-1329): one SSPRK(5,4) step with the given dt, in
 * place on stage 0 (q and face B). */
int how_ssprk(how_ctx* ctx, double dt);
/* prot (src/prot.cpp:6-54) on one stage */
int how_prot(how_ctx* ctx, int stage);
/* One directional sweep of stage 1 (src/ssprk.cpp:1000-1025, 1218-1272)
 * exactly as the reference's x_sweep/y_sweep/z_sweep would run it inside
 * stage 1 of ssprk with this dt: copies q(0) to q(1) and face B(0) to face
 * B(1) first (copy_stage, copy_bfield_stage, src/ssprk.cpp:1288-1289).
 * dir 0,1,2.  Each call fills the two CT flux arrays of its direction. */
int how_sweep(how_ctx* ctx, int dir, double dt);
/* fluxct(q, iw, k1, k3, par, ct) (src/fluxct.hpp:41-42, body
 * src/fluxct.cpp:786-899), preceded by bound_bfield(iw - 1) as ssprk runs it
 * (src/ssprk.cpp:1319-1320): corner EMFs from the CT flux arrays the last
 * sweeps filled, their smoothing, face B(iw) = k1 B(iw) + k3 B(iw-1) + the CT
 * update with the dt of the last sweeps, the ghost fill of face B(iw), and
 * the face-to-centre B into q(iw, 4..6).  No prot.  In 1-D it does nothing,
 * as the reference returns early (src/fluxct.cpp:793).  iw 1..5. */
int how_fluxct(how_ctx* ctx, int iw, double k1, double k3);
/* Download a CT flux array (0..5 = fsy fsz gsx gsz hsx hsy) in the reference
 * layout, for inspection after how_sweep / how_ssprk.  Faces the sweeps
 * compute are valid; ghost entries are not filled (the EMF kernel reads
 * across the boundary through the ghost-fill index map instead). */
int how_get_ct_array(how_ctx* ctx, int which, double* host);

/* Main loop (src/main.cpp:158-223) without output: advances from *time for
 * up to max_steps steps (max_steps < 0: no limit) towards tend, with the
 * reference's nt output intervals and dt clamp to each interval's end.
 * Updates *time and *steps.  dts (may be NULL) receives each step's dt.
 * Stops with HOW_ERR_DT on a non-positive dt (src/main.cpp:175-183) and with
 * HOW_ERR_NONFINITE when the time becomes non-finite (src/main.cpp:207-212)
 * or, before a step, when stage 0 holds a non-finite value (the CFL pass
 * checks every active cell; the reference's own reduction skips such cells).
 * how_tstep reports a non-finite state the same way. */
int how_run(how_ctx* ctx, double* time, long max_steps, long* steps, double* dts, long dts_cap);

/* Dump file of q(0), output() (src/output.cpp:555-572), in the context's
 * output_format: "dat" -> <dir>/dumpNNNNNN.dat, the ASCII table of
 * output_dat (src/output.cpp:65-224); "vtk" or "vts" -> <dir>/dumpNNNNNN.vts,
 * the binary appended-raw StructuredGrid of output_vts_binary
 * (src/output.cpp:226-552).  dir NULL means "output", the reference's
 * directory; it is created if missing.  The derived columns (velocity, gas
 * pressure, v^2, B^2, the cell-centred divB diagnostic, coordinates) are
 * formed on the device and the files equal the reference's byte for byte.
 * An unknown format returns HOW_ERR_ARG where the reference aborts;
 * output_format "none" (a mode the reference lists as a to-do) writes
 * nothing.  The
 * call returns once the file is written; it stages the data through the
 * context's own buffer, one slab of z planes at a time. */
int how_output(how_ctx* ctx, int step, double time, const char* dir);

/* The same dump, without waiting for it: the derived columns of the whole
 * domain are formed into a device buffer on the context's stream (ordered
 * after the steps already queued), copied into pinned host memory on a side
 * stream, and written by a host thread, so steps queued next run while the
 * file is copied and written.  One dump is in flight per context; a second
 * call first waits for the previous one.  The buffers (18 doubles per cell
 * for .vts, 16 for .dat, on the device and pinned on the host) are kept for
 * reuse until how_destroy.  output_format "none" writes nothing (also for
 * how_output). */
int how_output_async(how_ctx* ctx, int step, double time, const char* dir);
/* Waits for the dump in flight, if any; returns its status. */
int how_output_wait(how_ctx* ctx);

/* How the sweeps compute (HOW_PREC_*). */
int how_set_precision(how_ctx* ctx, int mode);

/* Block until the context's stream is idle. */
int how_sync(how_ctx* ctx);

/* ------------------------------------------------------ instrumentation */
/* Launches of this library's kernels since the context was created. */
long how_kernel_launches(const how_ctx* ctx);
/* The context's CUDA stream (cudaStream_t) for callers that time with events. */
void* how_stream(how_ctx* ctx);
/* CUDA-event timing of every sweep-kernel launch while enabled (no reference
 * counterpart; the reference has no timers).  Enabling clears the record. */
int how_set_kernel_timing(how_ctx* ctx, int on);
/* Summed device milliseconds and count of the timed sweep launches. */
int how_get_kernel_timing(how_ctx* ctx, double* total_ms, long* launches);
/* Failure-detection tests only (no reference counterpart): nonzero makes the
 * sweep kernels' compute threads give up their bounded tile waits at once,
 * so the next sweep ends early and the call returns HOW_ERR_CUDA with
 * "bounded TMA wait expired"; the thread that issued the tile copies still
 * waits, with its full limit, for every copy it has in flight before the
 * block exits.  0 restores the normal waits; the context stays usable. */
int how_set_wait_limit(how_ctx* ctx, int expire_at_once);
/* Mean cycles per thread block of each phase of one stage-1 sweep (the
 * how_sweep semantics) -- instrumentation, no reference counterpart.
 * out[0..10] = phases (load, primitives, cell differences, routing features,
 * routing network, routing decision, eigen-system scalars, eigenvector rows,
 * projection+WENO, back-projection+CT, update); out[11] = tiles.  A phase a
 * launch does not have adds nothing. */
int how_sweep_phase_profile(how_ctx* ctx, int dir, double dt, double* out, int nout);
/* ------------------------------------------------------ batched ensembles */
/* No counterpart in the reference (which runs one domain per job).  Many
 * independent runs (members, each with its own how_params: size, gamma,
 * problem, boundaries, tend, nt) advance together: every kernel of a time step
 * is launched once for all members (the sweeps as one persistent launch per
 * direction over every member's tiles) and the step is captured in a CUDA
 * graph that is replayed until each member has reached its tend.  A member
 * computes exactly what how_run computes for it alone.  Members need nx > 1
 * and run the plain FP64 method.  how_ensemble_member gives the member's
 * context for state access (valid until how_ensemble_destroy, which also
 * destroys the members). */
typedef struct how_ensemble how_ensemble;
int how_ensemble_create(const how_params* members, int n, how_ensemble** out);
int how_ensemble_destroy(how_ensemble* e);
int how_ensemble_size(const how_ensemble* e);
how_ctx* how_ensemble_member(how_ensemble* e, int m);
/* init_problem of every member; member times back to 0 */
int how_ensemble_init(how_ensemble* e);
/* Sweep tile shapes per direction (index into the candidate list of
 * how_ensemble_shape_info).  Without this call the first how_ensemble_run
 * autotunes: one real step per candidate, then the fastest per direction. */
int how_ensemble_set_shapes(how_ensemble* e, int sx, int sy, int sz);
int how_ensemble_get_shapes(const how_ensemble* e, int* shapes /*[3]*/, double* sweep_ms /*[3 x 3]*/);
int how_ensemble_shape_info(int dir, int shape, int* lines, int* cells);
/* Advance until every member reaches its tend (max_steps < 0) or for at most
 * max_steps steps; *steps_out = the most steps any member has taken. */
int how_ensemble_run(how_ensemble* e, long max_steps, long* steps_out);
int how_ensemble_member_status(const how_ensemble* e, int m, double* time, long* steps, int* done);
long how_ensemble_graph_launches(const how_ensemble* e);
/* The ensemble's CUDA stream (cudaStream_t), for callers that time with events. */
void* how_ensemble_stream(how_ensemble* e);

/* ------------------------------------------------------- learned routing */
/* No counterpart in the reference (an addition of this library).  A
 * 6 -> 32 -> 32 -> 1 GELU network, packed FP32 as W1[32][6], b1[32],
 * W2[32][32], b2[32], w3[32], b3 (how_router_param_count() floats), routes
 * each interface of each sweep to the full characteristic WENO5 or to a
 * component-wise linear-weight fifth-order flux; a hard jump/positivity guard
 * forces full WENO.  Inference runs on the tensor cores (BF16, FP32
 * accumulate) in a routing pass before the sweeps, whose decisions the sweep
 * kernels read; the guard is evaluated inside the sweep kernels. */
int how_router_param_count(void);
/* the built-in trained weights and logit threshold (what `router on` uses) */
int how_router_default(float* w, int n, float* threshold);
int how_router_set_weights(how_ctx* ctx, const float* w, int n);
/* mode 0 off, 1 network + guard, 2 guard only; full WENO when logit > threshold */
int how_router_configure(how_ctx* ctx, int mode, float threshold, float guard_jump, float guard_floor);
/* mode 1: the network's decisions are formed every `stages` SSPRK stages of
 * a step from its first (5 = once per step, the default; 1 = every stage), or
 * with 10 at the first stage of every second step, and reused by the sweeps
 * in between; the hard guard is evaluated at every stage in any case.  Any
 * change of the state or of the router makes the next stage form fresh ones. */
int how_router_set_refresh(how_ctx* ctx, int stages);
int how_router_stats(how_ctx* ctx, unsigned long long* full, unsigned long long* cheap, int reset);
/* ... plus the 16-interface groups whose logits came from the tensor cores and
 * those that needed no tensor-core pass (every stencil uniform -- the
 * precomputed flat logit -- or guarded) */
int how_router_stats4(how_ctx* ctx, unsigned long long* full, unsigned long long* cheap,
                      unsigned long long* mma_groups, unsigned long long* flat_groups, int reset);
/* Label collection from the plain FP64 method: records of 8 floats per
 * sampled interface -- the 6 router features (the prior-stage feature is held
 * at 0), the largest departure of the nonlinear WENO weights from the linear
 * ones over the 7 fields, and the flux departure, dt/dx |F_full - F_linear|
 * over the local size of the conserved variable (rho; rho (|v| + c);
 * sqrt(rho) c; E), largest component: what routing the face to the cheap flux
 * would change in one stage. */
int how_collect_begin(how_ctx* ctx, unsigned int capacity, unsigned int every);
int how_collect_end(how_ctx* ctx, float* out, unsigned int cap, unsigned int* n);
/* Hand-written GPU training (FP32, Adam) of w in place, its gradient, and
 * batched inference by the FP32 network and by the BF16 tensor-core path. */
int how_router_train(float* w, const float* feats, const float* labels, long n, float pos_weight, int iters,
                     int batch, float lr, unsigned long long seed, float* loss_hist);
int how_router_grad(const float* w, const float* feats, const float* labels, long n, float pos_weight,
                    float* grad_out, float* loss_out);
int how_router_infer(const float* w, const float* feats, long n, float* out_fp32, float* out_bf16);

/* ------------------------------------------------- decomposed domains */
/* One domain split into z slabs ("parts"), one context per part, each on its
 * own stream and, if `devices` lists them, on its own GPU; one host thread
 * steps all parts together.  Replaces the reference's MPI decomposition:
 * setup_mpi_domain (src/mpi_domain.cpp:54-156) for a split along z, the halo
 * exchanges of q (src/bound.cpp:132-271), face B and the CT arrays
 * (src/fluxct.cpp:287-479, 554-751), here as copies of whole z planes from a
 * part's buffers into its neighbour's ghost planes (peer-to-peer between
 * GPUs), and the dt allreduce (src/tstep.cpp:87-121), here a max over the
 * parts.  Each part fills only its physical boundaries (the reference fills
 * open boundaries on both sides of a rank with one physical side,
 * src/bound.cpp:273-291).  The parts run the single-domain kernels, so a
 * decomposed run equals the whole-domain run (how_run) bit for bit.
 * Needs nx, ny > 1 and at least 3 z planes per part; part p holds global
 * active planes kstart .. kstart + nz - 1 (how_group_part_range).
 * devices: nparts device ordinals, or NULL for the current device. */
typedef struct how_group how_group;
int how_group_create(const how_params* global, int nparts, const int* devices, how_group** out);
int how_group_destroy(how_group* g);
int how_group_size(const how_group* g);
how_ctx* how_group_part(how_group* g, int part);
int how_group_part_range(const how_group* g, int part, int* kstart, int* nz);
/* The decomposition plan of part `part` (host only, no device needed): its
 * z range, the z ghost layers it fills itself (bit 0 low, bit 1 high: its
 * physical open sides; periodic sides and sides shared with a part are
 * received), its neighbours (-1: none) and the halo planes (local padded z
 * indices of the first of `nplanes` planes): the part sends planes
 * send_up_first.. to the part above, which stores them at its recv_lo_first..,
 * and sends send_down_first.. to the part below, which stores them at its
 * recv_hi_first... */
typedef struct how_part_info {
    int kstart, nz, z_sides, lo_part, hi_part;
    int nplanes, send_up_first, recv_lo_first, send_down_first, recv_hi_first;
} how_part_info;
int how_part_plan(int nz_global, int nparts, int periodic_z, int part, how_part_info* out);
/* init_problem on the global grid (host), sliced into the parts, then bound
 * and initialize_bfield_from_q with the halos (src/main.cpp:125-130) */
int how_group_init(how_group* g);
/* the same from a global stage-0 state in the reference layout */
int how_group_set_state(how_group* g, const double* q_global);
/* the main loop (src/main.cpp:158-223) over all parts; as how_run */
int how_group_run(how_group* g, double* time, long max_steps, long* steps, double* dts, long dts_cap);
/* active cells of stage 0 / face B gathered into global reference-layout arrays */
int how_group_get_state(how_group* g, double* q_global);
int how_group_get_face_b(how_group* g, double* bx, double* by, double* bz);
/* output(q, par, step, time) of every MPI rank (src/output.cpp:555-572) for
 * the parts: part p writes <dir>/dumpNNNNNN_rankPPPPPP.dat|.vts, the piece
 * the reference's rank p of a 1 x 1 x nparts layout writes, with the same
 * header fields (rank, global and local sizes, global start index, piece
 * extent), global indices and coordinates, and the divB diagnostic over the
 * piece's own cells (wrapped or clamped at the piece's edges, as the
 * reference's per-rank writer does).  For vts/vtk it also writes
 * <dir>/dumpNNNNNN.pvts, the PStructuredGrid master file that lists the pieces
 * (a to-do of the reference, README.md:758).  how_output on a part's context
 * (how_group_part) writes that part's piece alone.  "none" writes nothing. */
int how_group_output(how_group* g, int step, double time, const char* dir);

/* ---------------------------------------------------- allocation-free use */
/* Capacity of the fixed scratch behind how_tstep_noalloc, in (i, j) lines. */
#define HOW_NOALLOC_MAX_LINES 262144

/* CFL time step of a state the caller already holds on the GPU, without
 * allocating any device memory.  No counterpart in the reference: it exists
 * for callers that cannot call cudaMalloc -- a host application whose memory
 * pool owns the whole device (Kokkos, AMReX and similar), or code running
 * under an allocator that forbids device allocation after set-up.
 *   q_dev : stage 0 in the reference layout (8 x (nx+6) x (ny+6) x (nz+6)
 *           doubles, k fastest) in device memory
 *   p     : grid sizes, box sizes, gam, cour, rhomin, pgmin are read
 *   dt_dev: one double in device memory that receives dt, computed as
 *           tstep does (src/tstep.cpp:11-136)
 *   stream: cudaStream_t to order the work on (NULL = legacy stream)
 * The reduction keeps its partial results in one fixed device array of
 * HOW_NOALLOC_MAX_LINES x 3 doubles (6 MiB); nx * ny above
 * HOW_NOALLOC_MAX_LINES is refused with HOW_ERR_ARG.  Every call looks up
 * that array's device address (cudaGetSymbolAddress) on the current device.
 * Under CUDA's default lazy module loading the array is placed on a device
 * when that lookup first runs there, so the first call on each device is
 * where those 6 MiB are taken: make it during set-up, before any stream
 * capture and before a host memory pool reserves the device (or run with
 * CUDA_MODULE_LOADING=EAGER, which places it when the library loads).  The
 * array then stays until the process exits, and later calls take no device
 * memory.  All calls share the array: calls that overlap on the GPU (other
 * streams, other threads) race and must be serialised by the caller.  The
 * call is asynchronous; read dt_dev after synchronising `stream`. */
int how_tstep_noalloc(const double* q_dev, const how_params* p, double* dt_dev, void* stream);

/* Measured FP64 FMA-pipe throughput of the current device, TFLOP/s (2 flops
 * per FMA): the roofline denominator of this FP64-bound path. */
int how_measure_fp64_peak(double* tflops, int reps);

#ifdef __cplusplus
}
#endif
#endif /* HOW_MHD_H */
