/* Oracle driver (test infrastructure): runs the reference solver's own code
 * path -- sim_params -> geometry -> sim_manager -> fluid_3d::initialize ->
 * stepper -> fluid_3d::init_iter -> stepper::run -- exactly as
 * Execs/run_sim.cc:39-141 does, then writes the full solver state in the
 * reference's own AoS layout (struct field, struct ref_map; fields.hh:34-646)
 * plus the extrapolated-map list, for the parity tests.
 *
 * Usage: ref_driver <file.cfg> <steps> <out.bin>
 *   steps = 0 writes the state after init_iter, before the first step.
 *        ref_driver <file.cfg> <steps> <prefix> phases
 *   runs <steps> steps, writes <prefix>_P0.bin, then runs the next step as
 *   the nine phase groups of fluid_3d::step_forward (fluid_3d.cc:429-577),
 *   calling the same members in the same order, and writes <prefix>_P<k>.bin
 *   after group k.
 *        ref_driver <file.cfg> <steps> <prefix> fields <k1,k2,...>
 *   steps the scene with stepper::step (the body of stepper::run's loop) and
 *   writes <prefix>_s<k>.f64 after step k for every listed k <= steps: the
 *   compact form below (velocity components and pressure only), for large
 *   grids whose full state would be hundreds of MB per dump.
 *
 * Compact layout: char[4] "RMTF"; int32 version=1; int32 m,n,o, sm4,sn4,so4,
 *   steps_done; double dt, time; then u, v, w, p as double[sm4*sn4*so4] each.
 *
 * Output layout (little endian):
 *   char[4] "RMTD"; int32 version=1;
 *   int32 m,n,o, sm4,sn4,so4, steps_done, n_extraps, sizeof(field), sizeof(ref_map);
 *   double dt, time;
 *   field[sm4*sn4*so4]; ref_map[sm4*sn4*so4];
 *   n_extraps x { int32 index, int32 pad, ref_map }.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>

#include "fluid_3d.hh"
#include "geometry.hh"
#include "sim_manager.hh"
#include "sim_params.hh"
#include "stepper.hh"

static sim_manager *alloc_manager(sim_params *spars) {
    const char *type = spars->sim_type;
    if (strcmp(type, "ftest") == 0) return new sim_ftest(spars);
    if (strcmp(type, "stest") == 0) return new sim_stest(spars);
    if (strcmp(type, "objects") == 0) return new sim_objects(spars);
    fprintf(stderr, "ref_driver: unsupported sim_type %s\n", type);
    exit(1);
}

static void dump(fluid_3d &f3d, int steps_done, const char *fn) {
    FILE *fh = fopen(fn, "wb");
    if (!fh) {
        perror(fn);
        exit(1);
    }
    const int ncell = f3d.sm4 * f3d.sn4 * f3d.so4;
    int n_ext = 0;
    for (int i = 0; i < ncell; i++) n_ext += f3d.extraps.n[i];
    fwrite("RMTD", 1, 4, fh);
    int hdr[11] = {1, f3d.m, f3d.n, f3d.o, f3d.sm4, f3d.sn4, f3d.so4, steps_done, n_ext,
                   (int)sizeof(field), (int)sizeof(ref_map)};
    fwrite(hdr, sizeof(int), 11, fh);
    double sc[2] = {f3d.dt, f3d.time};
    fwrite(sc, sizeof(double), 2, fh);
    fwrite(f3d.u_mem, sizeof(field), ncell, fh);
    fwrite(f3d.rm_mem, sizeof(ref_map), ncell, fh);
    for (int i = 0; i < ncell; i++) {
        for (int j = 0; j < f3d.extraps.n[i]; j++) {
            int rec[2] = {i, 0};
            fwrite(rec, sizeof(int), 2, fh);
            fwrite(f3d.extraps.f[i] + j, sizeof(ref_map), 1, fh);
        }
    }
    fclose(fh);
}

static void dump_fields(fluid_3d &f3d, int steps_done, const char *fn) {
    FILE *fh = fopen(fn, "wb");
    if (!fh) {
        perror(fn);
        exit(1);
    }
    const int ncell = f3d.sm4 * f3d.sn4 * f3d.so4;
    fwrite("RMTF", 1, 4, fh);
    int hdr[8] = {1, f3d.m, f3d.n, f3d.o, f3d.sm4, f3d.sn4, f3d.so4, steps_done};
    fwrite(hdr, sizeof(int), 8, fh);
    double sc[2] = {f3d.dt, f3d.time};
    fwrite(sc, sizeof(double), 2, fh);
    double *buf = new double[ncell];
    for (int c = 0; c < 4; c++) {
        for (int i = 0; i < ncell; i++) buf[i] = c < 3 ? f3d.u_mem[i].vel[c] : f3d.u_mem[i].p;
        fwrite(buf, sizeof(double), ncell, fh);
    }
    delete[] buf;
    fclose(fh);
}

int main(int argc, char *argv[]) {
    MPI_Init(&argc, &argv);
    if (argc < 4) {
        fprintf(stderr, "usage: %s <file.cfg> <steps> <out.bin>\n", argv[0]);
        return 1;
    }
    const int nsteps = atoi(argv[2]);
    sim_params spars(argv[1]);
    geometry gm(spars.sys_size[0], spars.sys_size[1], spars.sys_size[2], spars.x_prd, spars.y_prd, spars.z_prd);
    sim_manager *mgmt = alloc_manager(&spars);
    mkdir(spars.dirname, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);

    fluid_3d f3d(&gm, mgmt, &spars);
    int init_err = f3d.initialize();
    if (mgmt->dt_reg < spars.dt) spars.dt = mgmt->dt_reg;
    if (nsteps > 0) spars.stop_short = nsteps;
    stepper sim(spars, f3d);
    f3d.dt = sim.dt;
    f3d.init_iter(init_err);

    if (argc > 5 && strcmp(argv[4], "fields") == 0) {
        // the wanted step counts, ascending
        bool want[1 << 16] = {false};
        for (char *t = strtok(argv[5], ","); t; t = strtok(nullptr, ",")) {
            const int k = atoi(t);
            if (k >= 0 && k < (1 << 16)) want[k] = true;
        }
        char fn[1024];
        f3d.set_dt(sim.dt);
        if (want[0]) {
            snprintf(fn, sizeof(fn), "%s_s0.f64", argv[3]);
            dump_fields(f3d, 0, fn);
        }
        for (int k = 1; k <= nsteps; k++) {
            const int err = sim.step(f3d);
            if (err != NORMAL_EXIT) {
                fprintf(stderr, "ref_driver: step %d returned %d\n", k, err);
                return 2;
            }
            if (want[k]) {
                snprintf(fn, sizeof(fn), "%s_s%d.f64", argv[3], k);
                dump_fields(f3d, k, fn);
            }
        }
        printf("# ref_driver: V-cycles fem %ld mac %ld\n", f3d.mg_pres->ncycles, f3d.mg_mac->ncycles);
        return 0;
    }
    const bool phases = argc > 4 && strcmp(argv[4], "phases") == 0;
    double t0 = MPI_Wtime();
    if (nsteps > 0) sim.run(f3d);
    if (phases) {
        char fn[1024];
        auto out = [&](int k) {
            snprintf(fn, sizeof(fn), "%s_P%d.bin", argv[3], k);
            dump(f3d, nsteps, fn);
        };
        f3d.set_dt(sim.dt);
        out(0);
        f3d.nt++;
        f3d.compute_stress(false);
        out(1);
        f3d.normal_derivatives_velocity(f3d.dt, false);
        f3d.normal_derivatives_refmap(f3d.dt, false);
        f3d.compute_half_time_edge_velocities(f3d.dt, false);
        f3d.compute_half_time_edge_refmap(f3d.dt, false);
        f3d.time += 0.5 * f3d.dt;
        out(2);
        f3d.fill_boundary_cf(false);
        f3d.godunov_upwinding_set(false, false);
        f3d.fill_boundary_cf(false);
        out(3);
        f3d.mac_solve(f3d.dt, false);
        f3d.fill_boundary_cf(false);
        out(4);
        int err = f3d.update_reference_map(f3d.dt, false);
        if (err) printf("# ref_driver: update_reference_map error %d\n", err);
        out(5);
        f3d.compute_stress(false);
        out(6);
        f3d.compute_ustar(f3d.dt, false);
        f3d.fill_boundary_cc(false);
        f3d.communicate<2048>();
        f3d.time += 0.5 * f3d.dt;
        out(7);
        f3d.pp_solve(false);
        out(8);
        f3d.update_reference_map_full(false);
        f3d.redraw_boundary(false);
        f3d.fill_boundary_cc(false);
        f3d.communicate<2048>();
        out(9);
        printf("# ref_driver: phases written\n");
        delete mgmt;
        return 0;
    }
    double t1 = MPI_Wtime();
    printf("# ref_driver: %d steps in %.6f s (dt %.17g)\n", nsteps, t1 - t0, f3d.dt);
    f3d.watch.report();
    printf("# ref_driver: V-cycles fem %ld mac %ld\n", f3d.mg_pres->ncycles, f3d.mg_mac->ncycles);
    dump(f3d, nsteps, argv[3]);
    gm.free();
    f3d.free();
    delete mgmt;
    MPI_Finalize();
    return 0;
}
