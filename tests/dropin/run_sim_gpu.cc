/* run_sim on the GPU path: the reference's driver sequence (Execs/run_sim.cc:
 * 39-141) with its own sim_params and its unchanged stepper (Sim/stepper.hh),
 * and rmt3d_fluid_3d (include/rmt3d_fluid_3d.hh) in place of fluid_3d.
 * Test infrastructure: it shows the drop-in compiling and running against
 * the reference's own headers.  RMT3D_MG_EXACT=1 in the environment iterates
 * every Poisson solve to round-off (the oracle's exact mode).
 *
 * Usage: run_sim_gpu <file.cfg> */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sys/stat.h>
#include <sys/types.h>

#include "sim_params.hh"
#include "stepper.hh"
#include "rmt3d_fluid_3d.hh"

int main(int argc, char *argv[]) {
    MPI_Init(&argc, &argv);
    if (argc < 2) {
        printf("Usage: run_sim_gpu sample_sim.cfg\n");
        MPI_Finalize();
        return 0;
    }
    sim_params spars(argv[1]);
    mkdir(spars.dirname, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
    const char *ex = getenv("RMT3D_MG_EXACT");
    rmt3d_fluid_3d f3d(&spars, argv[1], ex && ex[0] == '1');
    int init_err = f3d.initialize();
    if (f3d.mgmt->dt_reg < spars.dt) spars.dt = f3d.mgmt->dt_reg;
    stepper sim(spars, f3d);
    f3d.set_dt(sim.dt);
    f3d.init_iter(init_err);
    printf("# Simulating to T = %0.3g with dt = %.10e\n", spars.T, sim.dt);
    sim.run(f3d);
    MPI_Finalize();
    return 0;
}
