/* rmt3d_fluid_3d: a drop-in problem class for the reference's stepper.
 *
 * The reference drives its solver through `template<class p_class> class
 * stepper` (Sim/stepper.hh:19-620), which calls members of a fluid_3d
 * (F3D_Source/fluid_3d.hh).  This class offers every member that stepper
 * uses, forwarding each to the C ABI of librmt3d_gpu.so (rmt3d_gpu.h), so
 * that the reference's own stepper, sim_params and run_sim sequence
 * (Execs/run_sim.cc:60-141) run unchanged on the GPU path:
 *
 *   stepper.hh:305      step_forward(int debug)          -> rmt3d_step
 *   stepper.hh:298      set_dt(double)                   -> rmt3d_set_dt
 *   stepper.hh:155,194  out, rank                        -> status string, rank 0
 *   stepper.hh:350      grid->cart                       -> an MPI communicator
 *   stepper.hh:375      time                             -> scalar 1 after each step
 *   stepper.hh:413-431  div_u, total_momentum, total_energy, total_dev_in_detF
 *                                                        -> one rmt3d_macro per frame
 *   stepper.hh:438-468  compute_v_centroid, mgmt->n_obj, mgmt->avg_*
 *                                                        -> the same rmt3d_macro
 *   stepper.hh:581-587  tr->print(file[, binary])        -> rmt3d_write_tracers
 *   stepper.hh:596-599  write_slice(write_params&, file) -> rmt3d_write_slice
 *   stepper.hh:602-608  write_chk_pt(snum, fnum, dir)    -> rmt3d_write_chk_pt
 *   stepper.hh:589-593  output_contours(file)            -> not part of this
 *                       library: a warning, no file (contour output is outside
 *                       the GPU path)
 *   stepper.hh:614-620  o (dump_all's slice loop)        -> cells along z
 * and for run_sim's sequence: the constructor (fluid_3d.cc:17-128),
 * initialize() (fluid_3d.cc:192-233), mgmt->dt_reg (run_sim.cc:100-102) and
 * init_iter(int) (fluid_3d.cc:235-287).
 *
 * Include it after the reference's stepper.hh (which brings mpi.h,
 * custom_structs.hh's double_int, write_params.hh and common.hh's
 * p_fatal_error).  Errors of the library end the program through
 * p_fatal_error, as the reference's own fatal paths do.  One rank: the
 * scene is not decomposed (the library steps one scene per GPU). */
#ifndef RMT3D_FLUID_3D_HH
#define RMT3D_FLUID_3D_HH

#include <cstdio>

#include "rmt3d_gpu.h"

class rmt3d_fluid_3d {
  public:
    /** stepper reads grid->cart (MPI_Barrier before the run). */
    struct grid_view {
        MPI_Comm cart;
    };
    /** stepper reads mgmt->n_obj and the per-object centroid and velocity
     * arrays that compute_v_centroid fills (sim_manager.hh:120-140);
     * run_sim reads mgmt->dt_reg. */
    struct manager_view {
        int n_obj = 0;
        double dt_reg = 0;
        double avg_x[RMT3D_MAX_OBJ], avg_y[RMT3D_MAX_OBJ], avg_z[RMT3D_MAX_OBJ];
        double avg_velx[RMT3D_MAX_OBJ], avg_vely[RMT3D_MAX_OBJ], avg_velz[RMT3D_MAX_OBJ];
    };
    /** stepper calls tr->print(file) and tr->print(file, false). */
    struct tracer_view {
        rmt3d_scene *s = nullptr;
        void print(const char *fn, bool binary = true) {
            if (rmt3d_write_tracers(s, fn, binary ? 1 : 0)) p_fatal_error(rmt3d_last_error(), 1);
        }
    };

    int rank = 0;
    char *out = nullptr;  // no status string: stepper prints nothing for it
    double time = 0;
    double dt = 0;
    int m = 0, n = 0, o = 0;
    grid_view *grid = &grid_;
    manager_view *mgmt = &mgmt_;
    tracer_view *tr = &tr_;

    /** fluid_3d(geometry*, sim_manager*, sim_params*): the scene of the
     * .cfg file that `spars` was read from.  mg_exact = 1 iterates every
     * Poisson solve to round-off instead of the reference's residual
     * tolerance (for comparisons with a reference run in that mode). */
    template <class params>
    rmt3d_fluid_3d(const params *spars, const char *cfg_path, int mg_exact = 0) {
        rmt3d_scene_desc d;
        if (rmt3d_desc_from_cfg(cfg_path, &d)) p_fatal_error(rmt3d_last_error(), 1);
        d.mg_exact = mg_exact;
        if (rmt3d_scene_create(&d, nullptr, &s_)) p_fatal_error(rmt3d_last_error(), 1);
        grid_.cart = MPI_COMM_WORLD;
        tr_.s = s_;
        m = d.sys_size[0];
        n = d.sys_size[1];
        o = d.sys_size[2];
        mgmt_.n_obj = d.n_obj;
        (void)spars;
    }
    ~rmt3d_fluid_3d() { rmt3d_scene_destroy(s_); }
    rmt3d_fluid_3d(const rmt3d_fluid_3d &) = delete;
    rmt3d_fluid_3d &operator=(const rmt3d_fluid_3d &) = delete;

    /** fluid_3d::initialize: 0 restarted from a checkpoint, 1 from scratch. */
    int initialize() {
        md_step_ = -1;
        double init_err = 1;
        if (rmt3d_initialize(s_) || rmt3d_get_scalar(s_, 13, &init_err) || rmt3d_get_scalar(s_, 2, &mgmt_.dt_reg) ||
            rmt3d_get_scalar(s_, 1, &time))
            p_fatal_error(rmt3d_last_error(), 1);
        return (int)init_err;
    }
    /** fluid_3d::init_iter with the init_err of the last initialize. */
    void init_iter(int) {
        md_step_ = -1;
        if (rmt3d_init_iter(s_) || rmt3d_get_scalar(s_, 1, &time)) p_fatal_error(rmt3d_last_error(), 1);
    }
    void set_dt(double dt_) {
        dt = dt_;
        if (rmt3d_set_dt(s_, dt_)) p_fatal_error(rmt3d_last_error(), 1);
    }
    /** fluid_3d::step_forward: the reference's return code. */
    int step_forward(int debug) {
        int status = 0;
        md_step_ = -1;
        if (rmt3d_step(s_, debug, &status) || rmt3d_get_scalar(s_, 1, &time)) p_fatal_error(rmt3d_last_error(), 1);
        return status;
    }

    // ---- frame diagnostics (stepper::collect_macro_data) ----
    double div_u(double_int &mx, double_int &mn) {
        macro();
        mx = double_int(md_.div_u_max, 0);
        mn = double_int(md_.div_u_min, 0);
        return md_.div_u_l2;
    }
    void total_momentum(double *mmt) {
        macro();
        for (int c = 0; c < 3; c++) mmt[c] = md_.momentum[c];
    }
    double total_energy(double &pot, double &kin, double &elas, double &pow) {
        macro();
        pot = md_.potential;
        kin = md_.kinetic;
        elas = md_.elastic;
        pow = md_.power;
        return md_.energy;
    }
    double total_dev_in_detF(double &max_dev) {
        macro();
        max_dev = md_.max_dev_detF;
        return md_.dev_detF;
    }
    void compute_v_centroid() {
        macro();
        for (int i = 0; i < md_.n_obj && i < RMT3D_MAX_OBJ; i++) {
            mgmt_.avg_x[i] = md_.centroid[i][0];
            mgmt_.avg_y[i] = md_.centroid[i][1];
            mgmt_.avg_z[i] = md_.centroid[i][2];
            mgmt_.avg_velx[i] = md_.velocity[i][0];
            mgmt_.avg_vely[i] = md_.velocity[i][1];
            mgmt_.avg_velz[i] = md_.velocity[i][2];
        }
    }

    // ---- files (stepper::write_files, dump_all) ----
    template <class wparams>
    void write_slice(wparams &wp, const char *fn) {
        if (rmt3d_write_slice(s_, wp.o_type, wp.dim, wp.point, wp.obj_id, wp.format, fn))
            p_fatal_error(rmt3d_last_error(), 1);
    }
    void write_chk_pt(int snum, int fnum, const char *dir) {
        if (rmt3d_write_chk_pt(s_, snum, fnum, dir, 1)) p_fatal_error(rmt3d_last_error(), 1);
    }
    void output_contours(const char *fn) {
        if (!warned_contours_) fprintf(stderr, "rmt3d_fluid_3d: contour output (%s) is not produced on the GPU path\n", fn);
        warned_contours_ = true;
    }

    rmt3d_scene *scene() { return s_; }

  private:
    rmt3d_scene *s_ = nullptr;
    grid_view grid_;
    manager_view mgmt_;
    tracer_view tr_;
    rmt3d_macro_data md_;
    double md_step_ = -1;  // step count the cached diagnostics belong to
    bool warned_contours_ = false;

    // one device pass for all of a frame's diagnostics, reused by the calls
    // stepper makes for the same frame
    void macro() {
        double nt = 0;
        if (rmt3d_get_scalar(s_, 4, &nt)) p_fatal_error(rmt3d_last_error(), 1);
        if (nt == md_step_) return;
        if (rmt3d_macro(s_, &md_)) p_fatal_error(rmt3d_last_error(), 1);
        md_step_ = nt;
    }
};

#endif
