/* rmt3d_gpu.h -- C ABI of the B200 implementation of RMT3D's per-timestep
 * Eulerian fluid-structure-interaction update.
 *
 * The reference's seam for this path is the fluid_3d class driven by the
 * duck-typed stepper (Sim/stepper.hh:296-376) and built by run_sim
 * (Execs/run_sim.cc:64-141).  Every entry point below replaces one member or
 * construction step of that seam; the reference location is cited beside it.
 * Plain C types only: no torch, no C++ types, no exceptions.  Every call
 * returns an int status (RMT3D_OK == 0); the step codes keep the reference's
 * values (Utilities/defs.hh:47-50).
 *
 * Threading: one host thread per scene handle at a time.  Device memory is
 * owned by the handle and never exposed except through the export calls. */
#ifndef RMT3D_GPU_H
#define RMT3D_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define RMT3D_OK 0
#define RMT3D_REFMAP_UPDATE_ERR 1   /* F3D_CONST::REFMAP_UPDATE_ERR */
#define RMT3D_PROJECTION_ERR 2      /* F3D_CONST::PROJECTION_ERR */
#define RMT3D_STEADY_SOLN_EXIT 100  /* F3D_CONST::STEADY_SOLN_EXIT */
#define RMT3D_ERR_INVALID (-1)      /* bad argument or malformed .cfg */
#define RMT3D_ERR_UNSUPPORTED (-2)  /* object/sim type outside this path */
#define RMT3D_ERR_CUDA (-3)         /* CUDA runtime error (message via rmt3d_last_error) */
#define RMT3D_ERR_EXTRAP (-4)       /* extrapolation found no eligible samples (ex.cc:253-269) */
#define RMT3D_ERR_NAN (-5)          /* NaN in a multigrid solve (fluid_3d.cc:2227) */
#define RMT3D_ERR_IO (-6)           /* file could not be read */
#define RMT3D_ERR_OOM (-7)          /* device allocation failed */
#define RMT3D_ERR_TOO_LARGE (-8)    /* size beyond a documented maximum */

#define RMT3D_MAX_OBJ 16
#define RMT3D_MAX_VEL_PROF 8

/* sim types (Execs/run_sim.cc:13-32) */
#define RMT3D_SIM_FTEST 0
#define RMT3D_SIM_STEST 1
#define RMT3D_SIM_OBJECTS 2

/* object types (Utilities/defs.hh:64-77); this path supports the first two */
#define RMT3D_OBJ_BASIC_SPHERE 0
#define RMT3D_OBJ_SPHERE 1

/* arithmetic forms */
#define RMT3D_FP64 0   /* plain form: FP64 throughout */
#define RMT3D_MIXED 1  /* FP32 multigrid V-cycles inside FP64 iterative refinement */
/* RMT3D_MIXED plus the advection stencil in FP32: FP32 velocity face states,
 * FP32 limited slopes, half-step extrapolation, upwinding and advective
 * increment added to the FP64 velocity.  2-3% faster per single-scene step
 * at 64^3-128^3; its perturbations are larger, and over the 64 seeded scenes
 * of the batched workload after 100 steps one scene's error against FP64
 * rose from 3.4e-7 (RMT3D_MIXED) to 9.3e-6 (a discrete change of the flow
 * there), against a budget of 1e-5.  No counterpart in the reference. */
#define RMT3D_MIXED_BULK32 2

/* One object: Sim/sim_params.cc:248-288 (basic_specs, extra_specs, srho,
 * shear_mod, object_list). */
typedef struct {
    int type;
    double basic[4];  /* centre x, y, z and primary dimension (radius) */
    double extra[10]; /* object-specific; SPHERE: stretch dir, sqrt(lambda), omega0[3] */
    double rho;
    double G;
} rmt3d_object_desc;

/* Run controls of sim_params that the step does not read: output and
 * checkpoint settings of run_sim/stepper (Sim/sim_params.cc:10-22, 86-160)
 * and the restart point.  A checkpoint's recover.cfg carries them
 * (sim_params.cc:489-600). */
typedef struct {
    int suppress, display;
    int chk_num;  /* > 0: initialize restarts from recover_dirname/chk.<chk_num> */
    int chk_step; /* total step count at that checkpoint */
    int chkpt_freq;
    int omp_num_thr, debug_flag, debug_obj_id, obj_body, data_fmt, out_flag, output_dim, output_ind;
    unsigned int dump_code; /* bit 1: tracers, 4: slices, 8: checkpoints, 32: macro.dat (stepper.hh:378-610) */
    int ntracers;
    double current_time; /* simulation time at the checkpoint */
    char dirname[256];   /* output directory: the .cfg path with ".cfg" -> ".out" */
    char recover_dirname[256];
} rmt3d_run_desc;

/* Everything the reference reads from sim_params and sim_manager for this
 * path (Sim/sim_params.cc:10-410, Sim/sim_manager.hh:164-188). */
typedef struct {
    int sys_size[3];
    double bounds[6]; /* ax, bx, ay, by, az, bz */
    int periodic[3];  /* derived from the BC sums, sim_params.cc:330-364 */
    int bct[3][6];    /* [velocity component][face] BC type: 0 periodic, 1 Dirichlet, 2 Neumann */
    double bcv[3][6];
    int walls[6];
    double wall_pos[6];
    double wall_dist;
    double fmu, frho, fdt_pad;
    double dt; /* user dt ("dt" keyword); the effective dt comes from the CFL rule */
    double T;
    int frames;
    int stop_short;
    int num_iters;
    int sim_type;
    int has_exact;
    int godunov;
    int implicit_visc;
    int vel_prof_num;
    double vel_profile[2 * RMT3D_MAX_VEL_PROF];
    int n_obj;
    int nlayers;
    int max_extrap_rs;
    double wt_n, ex_visc_mult, ev_trans_mult, sdt_pad, dt_ex_pad, weight_fac, gravity;
    rmt3d_object_desc obj[RMT3D_MAX_OBJ];
    int var_den;   /* compile-time VAR_DEN in the reference (Execs/Makefile:37-42) */
    int precision; /* RMT3D_FP64, RMT3D_MIXED or RMT3D_MIXED_BULK32 */
    int mg_exact;  /* 0: the reference's V-cycle control (residual tolerance of
                      mg_probs.hh:483-518); 1: additionally iterate every
                      Poisson solve until its residual stops shrinking, so
                      results are free of tolerance-level noise */
    double mixed_rtol; /* mixed form only: a solve also ends once its max-norm
                          residual is below mixed_rtol times the max-norm of
                          its right-hand side, and skips the two insurance
                          cycles (the form's accuracy target is 1e-5 rel-L2
                          after 100 steps); 0 keeps the reference's control.
                          Default 2e-6: over the 64 seeded scenes of the
                          batched workload (32^3-96^3, 1-8 spheres, variable
                          density), 100 steps, the largest rel-L2 from the
                          FP64 form is 3.4e-7 (velocity and pressure); at
                          5e-6 it is 9.3e-6, at 1e-5 three scenes exceed
                          1e-5 (largest 4e-5); below 2e-6 nothing changes. */
    rmt3d_run_desc run;
} rmt3d_scene_desc;

typedef struct rmt3d_scene rmt3d_scene;

/* ABI check: sizeof(rmt3d_scene_desc) as compiled into the library. */
int rmt3d_desc_sizeof(void);

/* Last error message of the calling thread (static storage). */
const char *rmt3d_last_error(void);

/* Parse a .cfg file with the reference's keyword semantics
 * (Sim/sim_params.cc:10-410; unknown keywords are an error, :317-321). */
int rmt3d_desc_from_cfg(const char *cfg_path, rmt3d_scene_desc *out);

/* Fill a descriptor with the reference's defaults (sim_params.cc:10-39). */
int rmt3d_desc_defaults(rmt3d_scene_desc *out);

/* Construct: fluid_3d::fluid_3d plus sim_manager setup (fluid_3d.cc:12-77,
 * sim_manager.cc:37-81).  Allocates the device state on the current device.
 * stream may be 0 (the legacy default stream) or a cudaStream_t cast to void*. */
int rmt3d_scene_create(const rmt3d_scene_desc *desc, void *stream, rmt3d_scene **out);

/* fluid_3d::initialize (fluid_3d.cc:192-233).  With run.chk_num > 0 the
 * state comes from the checkpoint run.recover_dirname/chk.<chk_num>
 * (rmt3d_read_chk_pt); otherwise, or when a checkpoint file is missing or
 * empty, from the initial conditions with a first extrapolation and dt_reg
 * from the CFL recheck, and run.chk_num is reset to 0.  The reference's
 * return value init_err (0 restarted, 1 started from scratch) is scalar 13
 * of rmt3d_get_scalar. */
int rmt3d_initialize(rmt3d_scene *s);

/* fluid_3d::set_dt (fluid_3d.hh:454-457). */
int rmt3d_set_dt(rmt3d_scene *s, double dt);

/* stepper::stepper dt fitting to frames (Sim/stepper.hh:211-227) after
 * run_sim's min(dt_reg, dt) (run_sim.cc:100-102); writes the fitted dt and
 * the number of steps per frame.  Pure host arithmetic. */
int rmt3d_stepper_dt(const rmt3d_scene_desc *desc, double dt_reg, double *dt_out, int *steps_per_frame);

/* fluid_3d::init_iter(init_err) (fluid_3d.cc:235-287) with the init_err of
 * the last rmt3d_initialize: up to num_iters pressure pre-iterations (time
 * and step count reset to 0) when it started from scratch, then in either
 * case the stress of the current state. */
int rmt3d_init_iter(rmt3d_scene *s);

/* fluid_3d::write_chk_pt (F3D_Source/fluid_3d_chk_pt.cc:3-72): writes the
 * checkpoint files vx vy vz p X Y Z OID and recover.cfg into chk_dirname
 * (created if missing).  Each field file holds the o z-slices of the
 * domain, each a (m+1)(n+1) double buffer filled as the reference's slice
 * gather does: cell fields at i + m*j, pressure on the nodal grid at
 * i + fem_m*j; X/Y/Z/OID take the map of least level set at each cell
 * (fluid_3d_io.cc:420-434), 100 / 0 where a cell has none.  recover.cfg is
 * sim_params::write_params (Sim/sim_params.cc:489-600) with chk_num = fnum,
 * chk_step = snum and current_time = the scene's time; the scene's run
 * block takes those values too.  compress != 0 compresses each field file
 * with xz as the reference does (fluid_3d_chk_pt.cc:54-59); a failed
 * compression leaves the file uncompressed, which the reader accepts. */
int rmt3d_write_chk_pt(rmt3d_scene *s, int snum, int fnum, const char *chk_dirname, int compress);

/* fluid_3d::initialize_from_chk_point (fluid_3d_chk_pt.cc:74-163) followed
 * by the rest of initialize: reads the eight field files (an X.xz file is
 * decompressed in memory when X itself is absent), resets the scene to a
 * fresh state, loads velocities, pressure, primary maps (x = xpred = X,
 * owner = OID), exchanges periodic images, extrapolates the maps and fills
 * the velocity boundary.  time and the step count come from the scene's
 * run block (current_time, chk_step).  The pressure slices are read with
 * the reference's stride m on the nodal grid (fluid_3d_chk_pt.cc:303-316),
 * so a restart reproduces the reference's restart.  *status is the
 * reference's code: 0 read, 1 a file is missing, 2 a file is empty; the
 * scene is unchanged unless it is 0. */
int rmt3d_read_chk_pt(rmt3d_scene *s, const char *chk_dirname, int *status);

/* run_sim's whole set-up sequence: initialize, stepper dt fit, set_dt,
 * init_iter (run_sim.cc:94-106). */
int rmt3d_prepare(rmt3d_scene *s);

/* fluid_3d::step_forward (fluid_3d.cc:429-577).  *status receives the
 * reference's step code; the return value is RMT3D_OK unless the call itself
 * failed. */
int rmt3d_step(rmt3d_scene *s, int debug, int *status);

/* The first last_phase (1..9) phase groups of one step_forward, for
 * phase-by-phase inspection: 1 compute_stress; 2 normal derivatives and
 * half-time edge states; 3 face BCs and Godunov upwinding; 4 MAC projection;
 * 5 update_reference_map; 6 compute_stress; 7 compute_ustar and cell BCs;
 * 8 pp_solve; 9 full reference-map update, redraw_boundary and cell BCs.
 * These are the member calls of fluid_3d.cc:470-560 in order. */
int rmt3d_step_phases(rmt3d_scene *s, int last_phase, int *status);

/* n calls of rmt3d_step, stopping at the first non-zero status. */
int rmt3d_run(rmt3d_scene *s, int nsteps, int *status);

/* Scalars: 0 dt, 1 time, 2 dt_reg, 3 eps (transition width), 4 nt (steps
 * taken), 5 last MAC V-cycles, 6 last FEM V-cycles, 7 total MAC V-cycles,
 * 8 total FEM V-cycles, 9 extrapolated maps, 10 K_stiff, 11 vmax,
 * 12 device bytes held, 13 init_err of the last rmt3d_initialize. */
int rmt3d_get_scalar(rmt3d_scene *s, int which, double *value);

/* Grid extents of the ghosted arrays: sm+4, sn+4, so+4 and the FEM node
 * grid m,n,o (fluid_3d.cc:21-24, geometry copy for the nodal grid). */
int rmt3d_get_dims(rmt3d_scene *s, int dims[6]);

/* Field export to host memory, SoA over the ghosted (sm+4)(sn+4)(so+4)
 * array with index i + sm4*j + smn4*k (fluid_3d.cc:24,45).
 * which: 0..2 vel u,v,w; 3 p; 4 dp; 5 q; 6..8 dvel; 9..26 fvel[f][c];
 *        27..35 sigma[F][c]. */
int rmt3d_get_field(rmt3d_scene *s, int which, double *host_dst);

/* The fields `which[0..n-1]` (numbering of rmt3d_get_field) copied to the
 * host buffers host_dst[0..n-1] (ncell doubles each; pinned memory lets the
 * copies overlap compute) without waiting: the fields are copied to device
 * staging buffers in the scene's stream order, then to the host on a copy
 * stream of the scene's own, so the next step can start at once.  A later
 * snapshot waits (on the device) for the previous one to reach the host.
 * rmt3d_snapshot_wait returns once the last snapshot is in host memory.  No
 * counterpart in the reference (its fields are in host memory already). */
int rmt3d_snapshot_fields(rmt3d_scene *s, const int *which, int n, double *const *host_dst);
int rmt3d_snapshot_wait(rmt3d_scene *s);

/* Reference-map export for object slot obj (0-based): per cell the map code
 * (-1 none, 0 primary, L>0 extrapolation layer L) and x[3], xpred[3]. */
int rmt3d_get_refmap(rmt3d_scene *s, int obj, int *code, double *x, double *xpred);

/* State import from the reference's AoS arrays (struct field 360 B, struct
 * ref_map 488 B; F3D_Source/fields.hh:34-646) plus its extrapolated maps as
 * (cell index, ref_map) pairs; the inverse of fluid_3d's in-memory layout. */
int rmt3d_import_reference(rmt3d_scene *s, const void *field_aos, const void *refmap_aos,
                           const int *ext_index, const void *ext_refmaps, int n_ext,
                           double dt, double time);

/* Export in the same AoS layout (fields.hh:34-646); extrapolated maps are
 * written as (cell index, ref_map) pairs into ext_index/ext_refmaps of
 * capacity max_ext, *n_ext receives the count. */
int rmt3d_export_reference(rmt3d_scene *s, void *field_aos, void *refmap_aos,
                           int *ext_index, void *ext_refmaps, int max_ext, int *n_ext);

/* Diagnostics: 0 div_u L2 of the FEM rhs (fluid_3d_utils.cc:507-653);
 * 1 solid volume sum H(phi) dV over the primary maps and 2-4 the centroid
 * x, y, z (compute_centroid, :1348-1379); 5 total deviation of det F from 1
 * and 6 its maximum (total_dev_in_detF, :1032-1084). */
int rmt3d_diag(rmt3d_scene *s, int kind, double *value);

/* Passive tracers (Utilities/tracers.{hh,cc}), present when the run block
 * has dump_code bit 1 and ntracers > 0 (fluid_3d.cc:217-219).  Each step
 * moves them by the reference's improved Euler scheme: a predictor with the
 * velocity at the start of the step and a corrector with the velocity at
 * its end, both interpolated tricubically from the 4x4x4 cell centres
 * around the tracer (tracers.hh:222-318, tracers.cc:395-457), slowed near
 * homogeneous Dirichlet walls as tracers::dx does.  A tracer that crosses a
 * periodic face re-enters on the other side; one that crosses a wall is
 * lost.  rmt3d_initialize places them: from the checkpoint's tr.<chk_num>
 * file on a restart, else uniformly at random (SplitMix64, seed 1 -- not
 * the reference's GSL stream, so fresh placements differ from its own). */

/* tracers::print's coordinates: x y z of every tracer by id (3 * ntracers
 * floats, 0 0 0 for a lost tracer) into xyz, at most max_tracers of them;
 * *n receives ntracers (0 when the scene has none). */
int rmt3d_tracer_positions(rmt3d_scene *s, float *xyz, int max_tracers, int *n);

/* tracers::set for every tracer (the restart path of
 * tracers::init_from_chkpt_files, tracers.cc:140-168): n must be ntracers;
 * a position outside the domain leaves that tracer out. */
int rmt3d_tracer_place(rmt3d_scene *s, const double *xyz, int n);

/* tracers::print (tracers.cc:105-133): binary (int count, then float x y z
 * per tracer) or text ("%g %g %g" lines).  rmt3d_write_chk_pt also writes
 * the frame's tr.<fnum> into the checkpoint directory. */
int rmt3d_write_tracers(rmt3d_scene *s, const char *filename, int binary);

/* One frame's diagnostics, the values the reference's stepper writes to
 * macro.dat and centroid.dat (Sim/stepper.hh:378-474). */
typedef struct {
    double time;
    double div_u_max, div_u_min; /* extremes of the face-velocity divergence over the cells */
    double div_u_l2;             /* weighted L2 norm of the FEM rhs (div_u, fluid_3d_utils.cc:507-653) */
    double momentum[3];          /* total_momentum (:783-800) */
    double energy, kinetic, elastic, potential, power; /* total_energy (:806-872); energy is
                                    elastic + kinetic + potential; power is 0 (no object type of
                                    this path has active stress) */
    double max_dev_detF, dev_detF; /* total_dev_in_detF (:1032-1084) */
    int n_obj;
    double centroid[RMT3D_MAX_OBJ][3]; /* compute_v_centroid (:1290-1346): heaviside-weighted mean */
    double velocity[RMT3D_MAX_OBJ][3]; /* position and velocity of each object's primary cells */
} rmt3d_macro_data;

/* All of rmt3d_macro_data in device reductions of fixed order. */
int rmt3d_macro(rmt3d_scene *s, rmt3d_macro_data *out);

/* fluid_3d::slice (F3D_Source/fluid_3d_io.cc:98-434): output type `type`
 * (write_params numbering 0-21: vx vy vz wx wy wz |u| p phi X Y Z OID LID
 * pr_phi pr_X pr_Y pr_Z div_u div_eu rho J) on the plane `point` of axis
 * `dim`, as the reference's global slice array out[a + d1 b], the two other
 * axes in increasing order.  Types 3, 4, 5, 7 and 18 live on the nodal grid
 * (m+1 points on a non-periodic axis), the rest on the cells.  obj_id -1
 * picks the map of least level set at each cell, obj_id >= 1 that object's
 * map.  A point outside the cell range gives zeros, as the reference's
 * bounds check does (:260-264).  out may be NULL to query d1 and d2. */
int rmt3d_slice(rmt3d_scene *s, int type, int dim, int point, int obj_id, double *out, int *d1, int *d2);

/* fluid_3d::write_slice (fluid_3d_io.cc:3-91): the slice written to
 * filename as a text matrix (format 0, "%17.14g "), coordinate text lines
 * (1) or gnuplot binary floats (2).  Coordinates are cell centres; the
 * last node of a nodal axis takes the next centre position, where the
 * reference reads one past its coordinate array. */
int rmt3d_write_slice(rmt3d_scene *s, int type, int dim, int point, int obj_id, int format, const char *filename);

/* Allocation-free divergence diagnostic (no counterpart in the reference; it
 * is an addition of this library).  Same value as rmt3d_diag(s, 0, ...) for
 * a scene with the given grid, computed from caller-owned device arrays, for
 * hosts that cannot allocate device memory when they need it (a host running
 * inside a memory pool it must not grow, or a plugin only handed device
 * pointers).  The scratch is a fixed array inside the library sized for at
 * most 274,625 FEM nodes (65^3, a 64^3 box with walls); larger grids return
 * RMT3D_ERR_TOO_LARGE.  No cudaMalloc/cudaFree or allocating library call is
 * made.  Each call looks the array's device address up on the current device
 * (cudaGetSymbolAddress), copies its argument block from host memory and
 * waits for `stream` before returning the value: the call is synchronous and
 * must not be issued on a stream that is capturing.  Every call shares the
 * array: calls that overlap on the GPU race.
 *   dvel[3]: du, dv, dw over the ghosted box (sys_size+4 per axis), with the
 *   two ghost layers filled as the step leaves them (on a periodic axis they
 *   hold the periodic images, which the FEM right-hand side reads);
 *   face_normal_vel[6]: for each wall face f, fvel[f][f/2] over the same box
 *   (may be NULL for periodic faces); dt_basis: the dt the FEM basis was built
 *   with (dt_reg); stream: cudaStream_t or 0; norm_out: host result. */
int rmt3d_div_u_noalloc(const int sys_size[3], const int periodic[3], const double bounds[6],
                        double dt_basis, const double *const dvel[3],
                        const double *const face_normal_vel[6], void *stream, double *norm_out);

/* Multigrid smoother of the scene's solves (no counterpart in the reference,
 * whose PGMG smoothing is a library internal): mode 0 issues one launch per
 * colour pass of the Gauss-Seidel sweeps; mode 1 one launch per whole sweep,
 * each block staging a box with an overlapped halo in shared memory and
 * running every colour pass there.  Both give the same bits. */
int rmt3d_scene_set_smoother(rmt3d_scene *s, int mode);

/* The coarse part of every V-cycle -- the levels of at most `pts` points
 * below the finest, down to the coarsest, with their smoothing, residuals,
 * transfers and the dense coarsest solve -- as one launch of a thread-block
 * cluster (16 CTAs, or 8) instead of one full-GPU launch per phase; 0 keeps
 * per-phase launches.  No counterpart in the reference. */
int rmt3d_scene_set_coarse_cluster(rmt3d_scene *s, int pts);

/* Block shape of the bulk stencil kernels of the step (stress, edge states,
 * upwinding, projections' right-hand sides and corrections, momentum
 * update): the tile of cells one 256-thread block covers, by index --
 * 0: 32x4x2 (default), 1: 32x8x1, 2: 64x4x1, 3: 32x2x4, 4: 128x2x1.  Every
 * cell's result is independent of the shape (the same bits).  No counterpart
 * in the reference. */
#define RMT3D_BLOCK_SHAPES 5
int rmt3d_scene_set_block_shape(rmt3d_scene *s, int shape);

/* Launch timing of one kernel class for roofline measurement (no counterpart
 * in the reference, which has no device code): kernel 0 = FEM Gauss-Seidel
 * colour pass on the finest level, 1 = MAC red-black pass on the finest level,
 * -1 = off.  CUDA events are recorded on the scene's stream around each
 * launch of that class, up to max_launches launches. */
int rmt3d_profile_kernel(rmt3d_scene *s, int kernel, int max_launches);

/* Sum of the timed launches' durations (ms), their count, and their
 * algorithmic bytes (8 B per point of the level read for x, plus the updated
 * colour's r read and x write). */
int rmt3d_profile_read(rmt3d_scene *s, double *ms_total, long long *launches, double *bytes_total);

/* ---- batched form ------------------------------------------------------
 * Many independent scenes (uneven grid sizes allowed) stepped together: each
 * scene keeps its own state and stream, and a pool of host threads issues
 * their steps so the kernels of many scenes overlap on the device.  No
 * counterpart in the reference, which runs one scene per process. */
typedef struct rmt3d_batch rmt3d_batch;
int rmt3d_batch_create(const rmt3d_scene_desc *descs, int nscenes, int host_threads, rmt3d_batch **out);
/* run_sim's set-up (rmt3d_prepare) of every scene */
int rmt3d_batch_prepare(rmt3d_batch *b);
/* every scene advances nsteps steps; status[i] receives scene i's step code */
int rmt3d_batch_step(rmt3d_batch *b, int nsteps, int *status);
int rmt3d_batch_size(rmt3d_batch *b, int *n);
int rmt3d_batch_scene(rmt3d_batch *b, int i, rmt3d_scene **out);
/* choose the multigrid schedule per kind of scene (grid shape, periodicity,
 * precision, density form) by timing candidates on a probe scene: the
 * smoothing counts (v_down, v_up), as the reference's mg_opt searches them
 * (Utilities/mg_probs.hh:80-208), the cluster or per-phase launch of the
 * solves, the smoother (colour passes or tiled sweeps) and the coarse
 * levels run as one cluster launch per V-cycle (rmt3d_scene_set_coarse_cluster);
 * then, under the chosen schedule, the block shape of the bulk stencil
 * kernels (rmt3d_scene_set_block_shape).  tuned_out gets 7 ints per kind:
 * (cells, v_down, v_up, cluster, smoother, coarse cluster points, block
 * shape) */
int rmt3d_batch_autotune(rmt3d_batch *b, int probe_steps, int *tuned_out, int max_out, int *n_out);

/* rmt3d_scene_set_smoother on every scene of the batch. */
int rmt3d_batch_set_smoother(rmt3d_batch *b, int mode);
int rmt3d_batch_destroy(rmt3d_batch *b);

/* Multigrid schedule of one scene: V(v_down, v_up) smoothing counts, and the
 * largest level (points) whose whole sub-cycle runs in one thread block out of
 * shared memory (0: none; negative keeps the current value). */
int rmt3d_scene_set_schedule(rmt3d_scene *s, int v_down, int v_up, int coarse_pts);

/* How each multigrid solve is issued: 1 = the whole solve as one launch in a
 * thread-block cluster of 8 or 16 CTAs, 0 (default) = one launch per phase
 * inside a graph loop.  Same operators and control; the results agree to the
 * solver tolerance. */
int rmt3d_scene_set_mg_launch(rmt3d_scene *s, int cluster);

/* Device bytes a scene with this descriptor allocates (admission control). */
size_t rmt3d_scene_footprint(const rmt3d_scene_desc *d);

/* Sums of u^2, v^2, w^2, p^2 over the interior cells, added in a fixed order
 * (the same bits for the same state on every run): a compact fingerprint of a
 * scene's state. */
int rmt3d_scene_checksum(rmt3d_scene *s, double out[4]);

/* ---- serving loop ------------------------------------------------------ */
typedef struct {
    double arrival_s;      /* arrival time after the start of rmt3d_serve */
    int steps;             /* steps to run after the set-up */
    rmt3d_scene_desc desc;
} rmt3d_request;

typedef struct {
    double admit_s, finish_s, latency_s; /* latency = finish - arrival */
    double step_p50_ms, step_p99_ms;
    double checksum[4];                  /* rmt3d_scene_checksum of the final state */
    int steps_done;
    int status;
} rmt3d_request_result;

typedef struct {
    double wall_s;
    double request_p50_s, request_p99_s;
    double step_p50_ms, step_p99_ms;
    double cellsteps_per_s;
    int requests;
} rmt3d_serve_summary;

/* Run a request stream with continuous batching: admission when a slot
 * (max_slots concurrent scenes) is free and the request's footprint fits
 * hbm_budget bytes; admitted scenes run concurrently, each on its own stream,
 * and later arrivals join as slots and memory free up; results[i] for
 * request i. */
int rmt3d_serve(const rmt3d_request *reqs, int nreq, size_t hbm_budget, int max_slots,
                rmt3d_request_result *results, rmt3d_serve_summary *summary);

/* The same stream with requests of one kind (grid shape, periodicity, form,
 * schedule) stepped together as one group graph (batched multigrid over the
 * group), each kind's group in rounds of up to 10 steps, polled and restarted
 * as they end, with requests joining and leaving between rounds; admission in
 * arrival order by footprint and max_slots requests in the system, set-up
 * overlapped with stepping. */
int rmt3d_serve_grouped(const rmt3d_request *reqs, int nreq, size_t hbm_budget, int max_slots,
                        rmt3d_request_result *results, rmt3d_serve_summary *summary);

/* Synchronise the scene's stream. */
int rmt3d_sync(rmt3d_scene *s);

/* Number of kernel launches issued by this scene so far. */
int rmt3d_launch_count(rmt3d_scene *s, long long *count);

int rmt3d_scene_destroy(rmt3d_scene *s);

#ifdef __cplusplus
}
#endif
#endif
