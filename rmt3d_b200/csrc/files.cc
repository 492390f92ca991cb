// Output files in the reference's formats, host side only (the values are
// computed on the device):
//  * checkpoints (F3D_Source/fluid_3d_chk_pt.cc:3-163): eight raw double
//    files of o z-slices each, optionally xz-compressed, and the
//    recover.cfg parameter file (Sim/sim_params.cc:489-600);
//  * slice files (fluid_3d_io.cc:3-91): text matrix, coordinate text or
//    gnuplot binary;
//  * tracer files (Utilities/tracers.cc:105-170): the count and float
//    coordinates in binary, or coordinate text.
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <spawn.h>
#include <string>
#include <sys/stat.h>
#include <sys/wait.h>
#include <unistd.h>
#include <vector>

#include "rmt3d_gpu.h"
#include "host_common.h"

extern char **environ;

namespace rmt3d {

// write_params::default_names of output types 0,1,2,7,9,10,11,12
// (IO/write_params.cc:3), the fields write_chk_pt writes in this order
const char *const kChkNames[kChkFields] = {"vx", "vy", "vz", "p", "X", "Y", "Z", "OID"};

namespace {

bool exists(const std::string &p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

// runs argv[0] from PATH with stdout sent to out_fd (or inherited when < 0);
// returns the exit status, or -1 when it could not be started
int run(const char *const argv[], int out_fd) {
    posix_spawn_file_actions_t fa;
    posix_spawn_file_actions_init(&fa);
    if (out_fd >= 0) posix_spawn_file_actions_adddup2(&fa, out_fd, 1);
    pid_t pid;
    int e = posix_spawnp(&pid, argv[0], &fa, nullptr, const_cast<char *const *>(argv), environ);
    posix_spawn_file_actions_destroy(&fa);
    if (e != 0) return -1;
    if (out_fd >= 0) close(out_fd);
    int st = 0;
    while (waitpid(pid, &st, 0) < 0)
        if (errno != EINTR) return -1;
    return WIFEXITED(st) ? WEXITSTATUS(st) : -1;
}

// the decompressed bytes of an .xz file, read through `xz -dc`
bool read_xz(const std::string &path, std::vector<char> &out) {
    int fds[2];
    if (pipe(fds) != 0) return false;
    posix_spawn_file_actions_t fa;
    posix_spawn_file_actions_init(&fa);
    posix_spawn_file_actions_adddup2(&fa, fds[1], 1);
    posix_spawn_file_actions_addclose(&fa, fds[0]);
    const char *argv[] = {"xz", "-dc", path.c_str(), nullptr};
    pid_t pid;
    int e = posix_spawnp(&pid, "xz", &fa, nullptr, const_cast<char *const *>(argv), environ);
    posix_spawn_file_actions_destroy(&fa);
    close(fds[1]);
    if (e != 0) {
        close(fds[0]);
        return false;
    }
    char buf[1 << 16];
    for (;;) {
        ssize_t n = read(fds[0], buf, sizeof(buf));
        if (n < 0 && errno == EINTR) continue;
        if (n <= 0) break;
        out.insert(out.end(), buf, buf + n);
    }
    close(fds[0]);
    int st = 0;
    while (waitpid(pid, &st, 0) < 0)
        if (errno != EINTR) return false;
    return WIFEXITED(st) && WEXITSTATUS(st) == 0;
}

// one field file's bytes; false when neither it nor its .xz exists or the
// .xz cannot be decompressed (fluid_3d_chk_pt.cc:107-120)
bool load(const std::string &path, std::vector<char> &out) {
    if (exists(path)) {
        FILE *f = fopen(path.c_str(), "rb");
        if (!f) return false;
        char buf[1 << 16];
        size_t n;
        while ((n = fread(buf, 1, sizeof(buf), f)) > 0) out.insert(out.end(), buf, buf + n);
        fclose(f);
        return true;
    }
    return exists(path + ".xz") && read_xz(path + ".xz", out);
}

}  // namespace

int chk_make_dir(const char *dir) {
    if (mkdir(dir, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH) != 0 && errno != EEXIST)
        return fail(RMT3D_ERR_IO, std::string("cannot create directory ") + dir);
    return 0;
}

int chk_write_files(const char *dir, const double *buf, size_t slice_len, int nslices, int compress) {
    const size_t per_file = slice_len * (size_t)nslices;
    for (int f = 0; f < kChkFields; f++) {
        std::string path = std::string(dir) + "/" + kChkNames[f];
        FILE *fh = fopen(path.c_str(), "wb");
        if (!fh) return fail(RMT3D_ERR_IO, "cannot write " + path);
        size_t w = fwrite(buf + f * per_file, sizeof(double), per_file, fh);
        fclose(fh);
        if (w != per_file) return fail(RMT3D_ERR_IO, "short write to " + path);
        if (compress) {
            // `xz -f` replaces an older .xz, as the reference's rm + xz does
            const char *argv[] = {"xz", "-f", path.c_str(), nullptr};
            if (run(argv, -1) != 0) fprintf(stderr, "rmt3d_write_chk_pt: xz of %s failed; left uncompressed\n", path.c_str());
        }
    }
    return 0;
}

int chk_read_files(const char *dir, double *buf, size_t slice_len, int nslices, int *status) {
    // one slice buffer reused across slices and fields, as the reference's
    // u_global (fluid_3d_chk_pt.cc:96-140): a short read leaves the rest of
    // the slice from the previous one
    std::vector<double> ug(slice_len, 0.0);
    const size_t per_file = slice_len * (size_t)nslices;
    *status = 0;
    for (int f = 0; f < kChkFields; f++) {
        std::vector<char> bytes;
        if (!load(std::string(dir) + "/" + kChkNames[f], bytes)) {
            *status = 1;
            return 0;
        }
        size_t pos = 0;
        for (int k = 0; k < nslices; k++) {
            size_t avail = (bytes.size() - pos) / sizeof(double);
            size_t n = avail < slice_len ? avail : slice_len;
            if (n == 0) *status = 2;
            memcpy(ug.data(), bytes.data() + pos, n * sizeof(double));
            pos += n * sizeof(double);
            memcpy(buf + f * per_file + k * slice_len, ug.data(), slice_len * sizeof(double));
        }
    }
    return 0;
}

int chk_write_recover_cfg(const char *dir, const rmt3d_scene_desc &d, double dt) {
    std::string path = std::string(dir) + "/recover.cfg";
    FILE *fh = fopen(path.c_str(), "w");
    if (!fh) return fail(RMT3D_ERR_IO, "cannot write " + path);
    const rmt3d_run_desc &r = d.run;
    static const char *types[] = {"ftest", "stest", "objects"};
    const char *st = (d.sim_type >= 0 && d.sim_type <= 2) ? types[d.sim_type] : "ftest";
    // line for line the layout of sim_params::write_params
    fprintf(fh, "#Keyword                  Input(default)           Type\n");
    fprintf(fh, "#System parameters\n");
    fprintf(fh, "suppress                  %d#(0)                   bool\n", r.suppress);
    fprintf(fh, "display                   %d#(0)                   bool\n", r.display);
    fprintf(fh, "implicit                  %d#(0)                   bool\n", d.implicit_visc);
    fprintf(fh, "godunov                   %d#(0)                   bool\n", d.godunov);
    fprintf(fh, "x_prd                     %d#(0)                   bool\n", d.periodic[0]);
    fprintf(fh, "y_prd                     %d#(0)                   bool\n", d.periodic[1]);
    fprintf(fh, "z_prd                     %d#(0)                   bool\n", d.periodic[2]);
    fprintf(fh, "has_exact                 %d#(0)                   bool\n", d.has_exact);
    fprintf(fh, "recover_dirname           %s#                      string\n", r.dirname);
    fprintf(fh, "chk_num                   %d#(0)                   int\n", r.chk_num);
    fprintf(fh, "chk_step                  %d#(0)                   int\n", r.chk_step);
    fprintf(fh, "sys_size                  %d %d %d#({96,96,96})    int\n", d.sys_size[0], d.sys_size[1],
            d.sys_size[2]);
    fprintf(fh, "frames                    %d#(96)                  int\n", d.frames);
    fprintf(fh, "stop_short                %d#(96)                  int\n", d.stop_short);
    fprintf(fh, "chkpt_freq                %d#(1)                   int\n", r.chkpt_freq);
    fprintf(fh, "omp_num_thr               %d#(1)                   int\n", r.omp_num_thr);
    fprintf(fh, "debug_flag                %d#(0)                   int\n", r.debug_flag);
    fprintf(fh, "debug_obj_id              %d#(-1)                   int\n", r.debug_obj_id);
    fprintf(fh, "obj_body                  %d#(-1)                  int\n", r.obj_body);
    fprintf(fh, "data_fmt                  %d#(0)                   int\n", r.data_fmt);
    fprintf(fh, "out_flag                  %d#(135)                 int\n", r.out_flag);
    fprintf(fh, "output_dim                %d#0/1/2(2)              int\n", r.output_dim);
    fprintf(fh, "output_ind                %d#(48)                  int\n", r.output_ind);
    fprintf(fh, "dump_code                 %u#(3)                   unsigned int\n", r.dump_code);
    fprintf(fh, "ntracers                  %d#(1000)                int\n", r.ntracers);
    fprintf(fh, "num_iters                 %d#(5)                   int\n", d.num_iters);
    fprintf(fh, "dt                        %g#(1.)                  double\n", dt);
    fprintf(fh, "T                         %g#(1.)                  double\n", d.T);
    fprintf(fh, "current_time              %g#(0.)                  double\n", r.current_time);
    fprintf(fh, "xyz_bounds                %g %g %g %g %g %g\n", d.bounds[0], d.bounds[1], d.bounds[2],
            d.bounds[3], d.bounds[4], d.bounds[5]);
    fprintf(fh, "                          #(0 1 0 1 0 1)         doubles\n");
    fprintf(fh, "# SIMULATION TYPE CONFIGURATIONS\n");
    fprintf(fh, "sim_type                  %s#(\"ftest\")           string\n", st);
    fprintf(fh, "# FLUID PROPERTIES\n");
    fprintf(fh, "fmu                       %g#(0.002)               double\n", d.fmu);
    fprintf(fh, "fdt_pad                   %g#(0.5)                 double\n", d.fdt_pad);
    fprintf(fh, "# SOLID PROPERTIES\n");
    fprintf(fh, "n_obj                     %d#(0)                   int\n", d.n_obj);
    fprintf(fh, "nlayers                   %d#(8)                   int\n", d.nlayers);
    fprintf(fh, "wt_n                      %g#(2.5)                 double\n", d.wt_n);
    fprintf(fh, "ex_visc_mult              %g#(1.)                  double\n", d.ex_visc_mult);
    fprintf(fh, "ev_trans_mult             %g#(1.)                  double\n", d.ev_trans_mult);
    fprintf(fh, "sdt_pad                   %g#(0.25)                double\n", d.sdt_pad);
    fprintf(fh, "dt_ex_pad                 %g#(0.8)                 double\n", d.dt_ex_pad);
    fprintf(fh, "gravity                   %g#(10.)                 double\n", d.gravity);
    fprintf(fh, "# SOLIDS CONFIGURATIONS\n");
    for (int i = 0; i < d.n_obj; i++) fprintf(fh, "object_list               %d %d\n", i, d.obj[i].type);
    for (int i = 0; i < d.n_obj; i++) {
        fprintf(fh, "basic_specs               %d ", i);
        for (int j = 0; j < 4; j++) fprintf(fh, "%g ", d.obj[i].basic[j]);
        fprintf(fh, "\n");
    }
    for (int i = 0; i < d.n_obj; i++) {
        fprintf(fh, "extra_specs               %d ", i);
        for (int j = 0; j < 10; j++) fprintf(fh, "%g ", d.obj[i].extra[j]);
        fprintf(fh, "\n");
    }
    for (int i = 0; i < d.n_obj; i++) fprintf(fh, "srho                      %d %g\n", i, d.obj[i].rho);
    for (int i = 0; i < d.n_obj; i++) fprintf(fh, "shear_mod                 %d %g\n", i, d.obj[i].G);
    fprintf(fh, "vel_prof_num              %d#(1)                   int\n", d.vel_prof_num);
    for (int i = 0; i < d.vel_prof_num; i++)
        fprintf(fh, "vel_profile               %d %d %g\n", i, (int)d.vel_profile[2 * i], d.vel_profile[2 * i + 1]);
    fprintf(fh, "# DOMAIN BOUNDARY CONDITIONS\n");
    static const char *faces[6] = {"bc_xl", "bc_xh", "bc_yl", "bc_yh", "bc_zl", "bc_zh"};
    for (int f = 0; f < 6; f++)
        fprintf(fh, "%-26s%d %d %d %g %g %g\n", faces[f], d.bct[0][f], d.bct[1][f], d.bct[2][f], d.bcv[0][f],
                d.bcv[1][f], d.bcv[2][f]);
    fprintf(fh, "# WALL BOUNDARIES\n");
    fprintf(fh, "walls                     %d %d %d %d %d %d\n", d.walls[0], d.walls[1], d.walls[2], d.walls[3],
            d.walls[4], d.walls[5]);
    fprintf(fh, "wall_pos                  %g %g %g %g %g %g\n", d.wall_pos[0], d.wall_pos[1], d.wall_pos[2],
            d.wall_pos[3], d.wall_pos[4], d.wall_pos[5]);
    fprintf(fh, "wall_dist                 %g\n", d.wall_dist);
    fclose(fh);
    return 0;
}

int slice_write_file(const char *filename, const double *u, int d1, int d2, int format, const double *c1,
                     const double *c2, int m) {
    FILE *fh = fopen(filename, "w");
    if (!fh) return fail(RMT3D_ERR_IO, std::string("cannot write ") + filename);
    if (format == 0) {
        // save_matrix (fluid_3d_io.cc:58-63)
        for (int j = 0; j < d2; j++) {
            for (int i = 0; i < d1; i++) fprintf(fh, "%17.14g ", u[i + j * d1]);
            fputc('\n', fh);
        }
    } else if (format == 1) {
        // save_text (:65-71)
        for (int j = 0; j < d2; j++) {
            for (int i = 0; i < d1; i++) fprintf(fh, "%17.14f %17.14f %17.14f\n", c1[i], c2[j], u[i + j * d1]);
            fputc('\n', fh);
        }
    } else {
        // save_gnuplot (:73-91): a row of (m, x coordinates), then per line
        // (y coordinate, values), all as floats
        std::vector<float> buf(d1 + 1);
        buf[0] = (float)m;
        for (int i = 0; i < d1; i++) buf[i + 1] = (float)c1[i];
        fwrite(buf.data(), sizeof(float), d1 + 1, fh);
        for (int j = 0; j < d2; j++) {
            buf[0] = (float)c2[j];
            for (int i = 0; i < d1; i++) buf[i + 1] = (float)u[i + j * d1];
            fwrite(buf.data(), sizeof(float), d1 + 1, fh);
        }
    }
    fclose(fh);
    return 0;
}

int tracer_write_file(const char *filename, const float *pos, int n, int binary) {
    FILE *fh = fopen(filename, binary ? "wb" : "w");
    if (!fh) return fail(RMT3D_ERR_IO, std::string("cannot write ") + filename);
    if (binary) {
        fwrite(&n, sizeof(int), 1, fh);
        fwrite(pos, sizeof(float), 3 * (size_t)n, fh);
    } else {
        for (int t = 0; t < n; t++) fprintf(fh, "%g %g %g\n", pos[3 * t], pos[3 * t + 1], pos[3 * t + 2]);
    }
    fclose(fh);
    return 0;
}

int tracer_read_file(const char *filename, int n, std::vector<float> &pos) {
    FILE *fh = fopen(filename, "rb");
    if (!fh) return fail(RMT3D_ERR_IO, std::string("cannot read tracer file ") + filename);
    int lnum = 0;
    size_t got = fread(&lnum, sizeof(int), 1, fh);
    if (got == 1 && lnum == n) {
        pos.assign(3 * (size_t)n, 0.f);
        got = fread(pos.data(), sizeof(float), 3 * (size_t)n, fh);
    } else {
        got = 0;
    }
    fclose(fh);
    if (lnum != n || got != 3 * (size_t)n)
        return fail(RMT3D_ERR_IO, std::string("tracer file ") + filename +
                                      ": reading failed, or its count differs from ntracers");
    return 0;
}

}  // namespace rmt3d
