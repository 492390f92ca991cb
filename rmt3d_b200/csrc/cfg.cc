// .cfg front end: the reference's keyword parser (Sim/sim_params.cc:10-410)
// and the stepper's dt fit (Sim/stepper.hh:211-227), as plain host C++.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "rmt3d_gpu.h"
#include "host_common.h"

namespace {

struct tokenizer {
    std::vector<std::string> tok;
    size_t pos = 1;
    int line;
    bool bad = false;
    const std::string &next() {
        static const std::string empty;
        if (pos >= tok.size()) {
            bad = true;
            return empty;
        }
        return tok[pos++];
    }
    int next_int() { return atoi(next().c_str()); }
    double next_double() { return atof(next().c_str()); }
};

}  // namespace

extern "C" int rmt3d_desc_sizeof(void) { return (int)sizeof(rmt3d_scene_desc); }

extern "C" int rmt3d_desc_defaults(rmt3d_scene_desc *d) {
    if (!d) return rmt3d::fail(RMT3D_ERR_INVALID, "null descriptor");
    memset(d, 0, sizeof(*d));
    // sim_params.cc:10-39
    d->godunov = 1;
    d->periodic[0] = d->periodic[1] = d->periodic[2] = 1;
    d->frames = 100;
    d->stop_short = -1;
    d->num_iters = 5;
    d->dt = 1.0;
    d->T = 1.0;
    d->bounds[0] = 0; d->bounds[1] = 1;
    d->bounds[2] = 0; d->bounds[3] = 1;
    d->bounds[4] = 0; d->bounds[5] = 1;
    for (int i = 0; i < 6; i++) d->wall_pos[i] = d->bounds[i];
    d->wall_dist = 0;
    d->frho = 1;
    d->fmu = 0.002;
    d->fdt_pad = 0.5;
    d->nlayers = 8;
    d->max_extrap_rs = 5;
    d->wt_n = 2.5;
    d->ex_visc_mult = 1.0;
    d->ev_trans_mult = 1.0;
    d->sdt_pad = 0.25;
    d->dt_ex_pad = 0.8;
    d->weight_fac = 0.25;
    d->gravity = 0;
    d->sys_size[0] = d->sys_size[1] = d->sys_size[2] = 96;
    d->sim_type = RMT3D_SIM_FTEST;
    d->precision = RMT3D_FP64;
    d->mixed_rtol = 2e-6;
    // run controls, sim_params.cc:12-22
    rmt3d_run_desc &r = d->run;
    r.chkpt_freq = 1;
    r.omp_num_thr = 1;
    r.debug_obj_id = -1;
    r.obj_body = -1;
    r.out_flag = 1 | 2 | 4 | 128;
    r.output_dim = 2;
    r.output_ind = -1;
    r.dump_code = 1 | 2;
    r.ntracers = 1000;
    return RMT3D_OK;
}

extern "C" int rmt3d_desc_from_cfg(const char *path, rmt3d_scene_desc *d) {
    rmt3d_desc_defaults(d);
    size_t len = path ? strlen(path) : 0;
    if (len < 4 || strcmp(path + len - 4, ".cfg") != 0)
        return rmt3d::fail(RMT3D_ERR_INVALID, "Filename must end in '.cfg'");
    FILE *f = fopen(path, "r");
    if (!f) return rmt3d::fail(RMT3D_ERR_IO, std::string("cannot open ") + path);
    // the output directory is the .cfg path with ".cfg" -> ".out", and the
    // recovery directory defaults to it (sim_params.cc:53-61)
    rmt3d_run_desc &r = d->run;
    if (len - 4 + 5 > sizeof(r.dirname)) {
        fclose(f);
        return rmt3d::fail(RMT3D_ERR_TOO_LARGE, "cfg path longer than 250 characters");
    }
    memcpy(r.dirname, path, len - 4);
    memcpy(r.dirname + len - 4, ".out", 5);
    memcpy(r.recover_dirname, r.dirname, sizeof(r.dirname));
    char buf[1024];
    int ln = 1;
    bool var_den = false;
    while (fgets(buf, sizeof(buf), f)) {
        for (char *bp = buf; *bp; bp++)
            if (*bp == '#') {
                *bp = 0;
                break;
            }
        tokenizer t;
        t.line = ln;
        for (char *p = strtok(buf, " \t\n\r"); p; p = strtok(nullptr, " \t\n\r")) t.tok.push_back(p);
        ln++;
        if (t.tok.empty()) continue;
        const std::string &k = t.tok[0];
        auto bc = [&](int face) {
            int ty[3];
            double va[3];
            for (int i = 0; i < 3; i++) ty[i] = t.next_int();
            for (int i = 0; i < 3; i++) va[i] = t.next_double();
            for (int i = 0; i < 3; i++) {
                d->bct[i][face] = ty[i];
                d->bcv[i][face] = va[i];
            }
        };
        if (k == "suppress") {
            r.suppress = t.next_int();
        } else if (k == "display") {
            r.display = t.next_int();
        } else if (k == "recover_dirname") {
            const std::string &v = t.next();
            snprintf(r.recover_dirname, sizeof(r.recover_dirname), "%s", v.c_str());
        } else if (k == "chk_num") {
            r.chk_num = t.next_int();
        } else if (k == "chk_step") {
            r.chk_step = t.next_int();
        } else if (k == "chkpt_freq") {
            r.chkpt_freq = t.next_int();
        } else if (k == "omp_num_thr") {
            int v = t.next_int();
            if (v > 0) r.omp_num_thr = v;
        } else if (k == "debug_flag") {
            r.debug_flag = t.next_int();
        } else if (k == "debug_obj_id") {
            r.debug_obj_id = t.next_int();
        } else if (k == "out_flag") {
            r.out_flag = t.next_int();
        } else if (k == "obj_body") {
            r.obj_body = t.next_int();
        } else if (k == "data_fmt") {
            r.data_fmt = t.next_int();
        } else if (k == "output_dim") {
            r.output_dim = t.next_int();
            if (r.output_dim < 0 || r.output_dim > 2) r.output_dim = -1;
        } else if (k == "output_ind") {
            r.output_ind = t.next_int();
            if (r.output_ind < 0 || r.output_dim < 0 || r.output_ind >= d->sys_size[r.output_dim]) r.output_ind = -1;
        } else if (k == "dump_code") {
            r.dump_code = (unsigned int)atol(t.next().c_str());
        } else if (k == "ntracers") {
            r.ntracers = t.next_int();
        } else if (k == "current_time") {
            double v = t.next_double();
            if (v > 0) r.current_time = v;
        } else if (k == "implicit") {
            d->implicit_visc = t.next_int();
        } else if (k == "godunov") {
            d->godunov = t.next_int();
        } else if (k == "x_prd") {
            d->periodic[0] = t.next_int();
        } else if (k == "y_prd") {
            d->periodic[1] = t.next_int();
        } else if (k == "z_prd") {
            d->periodic[2] = t.next_int();
        } else if (k == "has_exact") {
            d->has_exact = t.next_int();
        } else if (k == "walls") {
            for (int i = 0; i < 6; i++) d->walls[i] = t.next_int();
        } else if (k == "wall_pos") {
            for (int i = 0; i < 6; i++) d->wall_pos[i] = t.next_double();
        } else if (k == "wall_dist") {
            d->wall_dist = t.next_double();
        } else if (k == "sys_size") {
            for (int i = 0; i < 3; i++) {
                int v = t.next_int();
                if (v > 0) d->sys_size[i] = v;
            }
        } else if (k == "frames") {
            d->frames = t.next_int();
        } else if (k == "stop_short") {
            d->stop_short = t.next_int();
        } else if (k == "num_iters") {
            d->num_iters = t.next_int();
        } else if (k == "dt") {
            d->dt = t.next_double();
        } else if (k == "T") {
            double v = t.next_double();
            if (v > 0) d->T = v;
        } else if (k == "xyz_bounds") {
            for (int i = 0; i < 6; i++) d->bounds[i] = t.next_double();
        } else if (k == "fmu") {
            d->fmu = t.next_double();
        } else if (k == "fdt_pad") {
            d->fdt_pad = t.next_double();
        } else if (k == "vel_prof_num") {
            d->vel_prof_num = t.next_int();
            if (d->vel_prof_num > RMT3D_MAX_VEL_PROF) {
                fclose(f);
                return rmt3d::fail(RMT3D_ERR_TOO_LARGE, "vel_prof_num above 8");
            }
        } else if (k == "vel_profile") {
            int idx = t.next_int();
            if (idx >= 0 && idx < d->vel_prof_num) {
                int vt = t.next_int();
                d->vel_profile[2 * idx] = vt;
                if (vt != 0) d->vel_profile[2 * idx + 1] = t.next_double();
            }
        } else if (k == "n_obj") {
            d->n_obj = t.next_int();
            if (d->n_obj > RMT3D_MAX_OBJ || d->n_obj < 0) {
                fclose(f);
                return rmt3d::fail(RMT3D_ERR_TOO_LARGE, "n_obj outside 0..16");
            }
            for (int i = 0; i < d->n_obj; i++) {
                d->obj[i].type = 0;
                d->obj[i].rho = 1;
                d->obj[i].G = 1;
                d->obj[i].extra[0] = 1;
                for (int j = 1; j < 10; j++) d->obj[i].extra[j] = 0;
            }
        } else if (k == "nlayers") {
            d->nlayers = t.next_int();
        } else if (k == "max_extrap_rs") {
            d->max_extrap_rs = t.next_int();
            if (d->max_extrap_rs < 2) d->max_extrap_rs = 2;
        } else if (k == "wt_n") {
            d->wt_n = t.next_double();
        } else if (k == "ex_visc_mult") {
            d->ex_visc_mult = t.next_double();
        } else if (k == "ev_trans_mult") {
            d->ev_trans_mult = t.next_double();
        } else if (k == "sdt_pad") {
            d->sdt_pad = t.next_double();
        } else if (k == "dt_ex_pad") {
            d->dt_ex_pad = t.next_double();
        } else if (k == "weight_fac") {
            d->weight_fac = t.next_double();
        } else if (k == "gravity") {
            d->gravity = t.next_double();
        } else if (k == "bc_xl") {
            bc(0);
        } else if (k == "bc_xh") {
            bc(1);
        } else if (k == "bc_yl") {
            bc(2);
        } else if (k == "bc_yh") {
            bc(3);
        } else if (k == "bc_zl") {
            bc(4);
        } else if (k == "bc_zh") {
            bc(5);
        } else if (k == "basic_specs") {
            int idx = t.next_int();
            if (idx >= 0 && idx < d->n_obj)
                for (int i = 0; i < 4; i++) d->obj[idx].basic[i] = t.next_double();
        } else if (k == "extra_specs") {
            int idx = t.next_int();
            if (idx >= 0 && idx < d->n_obj)
                for (int i = 0; i < 10; i++) d->obj[idx].extra[i] = t.next_double();
        } else if (k == "srho") {
            int idx = t.next_int();
            if (idx >= 0 && idx < d->n_obj) d->obj[idx].rho = t.next_double();
        } else if (k == "shear_mod") {
            int idx = t.next_int();
            if (idx >= 0 && idx < d->n_obj) d->obj[idx].G = t.next_double();
        } else if (k == "object_list") {
            int idx = t.next_int();
            if (idx >= 0 && idx < d->n_obj) d->obj[idx].type = t.next_int();
        } else if (k == "sim_type") {
            const std::string &v = t.next();
            if (v == "ftest") d->sim_type = RMT3D_SIM_FTEST;
            else if (v == "stest") d->sim_type = RMT3D_SIM_STEST;
            else if (v == "objects") d->sim_type = RMT3D_SIM_OBJECTS;
            else {
                fclose(f);
                return rmt3d::fail(RMT3D_ERR_UNSUPPORTED, "sim_type " + v + " is outside this path");
            }
        } else if (k == "var_den") {
            // extension keyword: selects the reference's VAR_DEN build semantics
            d->var_den = t.next_int();
        } else if (k == "precision") {
            // extension keyword: 0 FP64, 1 FP32 V-cycles inside FP64 refinement,
            // 2 that and the advection stencil in FP32
            d->precision = t.next_int();
        } else if (k == "mixed_rtol") {
            // extension keyword: relative solve tolerance of the mixed form
            d->mixed_rtol = t.next_double();
        } else {
            fclose(f);
            return rmt3d::fail(RMT3D_ERR_INVALID, "Unrecognized keyword '" + k + "' at line " + std::to_string(t.line));
        }
        if (t.bad) {
            fclose(f);
            return rmt3d::fail(RMT3D_ERR_INVALID, "Not enough arguments at input line " + std::to_string(t.line));
        }
    }
    fclose(f);
    (void)var_den;

    // derived quantities, sim_params.cc:324-372
    for (int a = 0; a < 3; a++) {
        int s = d->bct[0][2 * a] + d->bct[1][2 * a] + d->bct[2][2 * a];
        if (s >= 0 && s < 3) {
            for (int c = 0; c < 3; c++) d->bct[c][2 * a] = d->bct[c][2 * a + 1] = 0;
            d->periodic[a] = 1;
        } else {
            d->periodic[a] = 0;
        }
    }
    for (int a = 0; a < 3; a++)
        if (!d->periodic[a]) d->walls[2 * a] = d->walls[2 * a + 1] = 1;
    double dx = (d->bounds[1] - d->bounds[0]) / d->sys_size[0];
    double dy = (d->bounds[3] - d->bounds[2]) / d->sys_size[1];
    double dz = (d->bounds[5] - d->bounds[4]) / d->sys_size[2];
    double mdh = dx < dy ? dx : dy;
    mdh = mdh < dz ? mdh : dz;
    d->wall_dist = mdh > d->wall_dist ? mdh : d->wall_dist;
    if (r.output_ind == -1 && r.output_dim >= 0) r.output_ind = d->sys_size[r.output_dim] / 2;
    // a restart needs recover_dirname/chk.<chk_num>/recover.cfg, else it is
    // dropped (sim_params.cc:374-397)
    if (r.chk_num > 0) {
        char probe[600];
        snprintf(probe, sizeof(probe), "%s/chk.%05d/recover.cfg", r.recover_dirname, r.chk_num);
        FILE *fh = fopen(probe, "rb");
        if (fh) fclose(fh);
        else r.chk_num = r.chk_step = 0;
    }
    if (d->sim_type != RMT3D_SIM_OBJECTS) d->n_obj = 0;
    return RMT3D_OK;
}

extern "C" int rmt3d_stepper_dt(const rmt3d_scene_desc *d, double dt_reg, double *dt_out, int *steps_out) {
    if (!d || !dt_out) return rmt3d::fail(RMT3D_ERR_INVALID, "null argument");
    // run_sim.cc:100-102
    double dt = d->dt;
    if (dt_reg < dt) dt = dt_reg;
    // stepper.hh:220-225
    double df = d->T / (d->frames - 1);
    int steps = (int)(df / dt);
    double rem = df - steps * dt;
    if (rem > 0) dt -= (dt - rem) / (++steps);
    *dt_out = dt;
    if (steps_out) *steps_out = steps;
    return RMT3D_OK;
}
