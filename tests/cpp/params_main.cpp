// Prints the parameters a configuration file gives through the C++ surface
// (spooky_b200::Parameters), one "name value" pair per line; on an error it
// prints "error <code> <message>".  With --run N it also builds a Supervisor,
// advances N steps on the GPU and prints the time, step count and energies;
// with --snap DIR it runs the main loop to t_final writing snapshots under
// DIR/data and restarts a second Supervisor from the most recent one.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cstring>
#include <string>

#include "spooky_b200.hpp"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s spooky.cfg [--run N]\n", argv[0]);
        return 2;
    }
    try {
        spooky_b200::Parameters p(argv[1]);
        std::printf("nx %d\nny %d\nnz %d\nlx %.17g\nly %.17g\nlz %.17g\n", p.nx, p.ny, p.nz, p.lx, p.ly, p.lz);
        std::printf("incompressible %d\nmhd %d\nboussinesq %d\nnu %.17g\nnu_m %.17g\ncfl %.17g\nt_final %.17g\n",
                    p.incompressible, p.mhd, p.boussinesq, p.nu, p.nu_m, p.cfl, p.t_final);
        if (argc >= 4 && std::strcmp(argv[2], "--run") == 0) {
            const long n = std::atol(argv[3]);
            spooky_b200::Supervisor sup(p);
            // a solenoidal single mode u_x(k_y = 1) so that the run is not trivial
            std::vector<double> U(2 * (size_t)sup.fields->num_fields * sup.fields->n_complex, 0.0);
            const size_t kk = (size_t)p.nz / 2 + 1;
            U[2 * (1 * kk)] = 0.25 * p.nx * p.ny * p.nz;   // field 0 (vx), i = 0, j = 1, k = 0
            sup.fields->set(U.data(), false);
            const long taken = sup.executeMainLoop(n);
            const spk_budgets_t b = sup.fields->budgets();
            std::printf("steps %ld\nstep %d\ntime %.17g\nenergy0 %.17g\n", taken, sup.timestep->current_step,
                        sup.timestep->current_time, b.energy[0]);
        }
        if (argc >= 4 && std::strcmp(argv[2], "--snap") == 0) {
            // the main loop with snapshots in DIR/data, then a restart from the most recent one
            const std::string dir = argv[3];
            std::vector<double> U;
            {
                spooky_b200::Supervisor sup(p, nullptr, dir);
                U.assign(2 * (size_t)sup.fields->num_fields * sup.fields->n_complex, 0.0);
                const size_t kk = (size_t)p.nz / 2 + 1;
                U[2 * (1 * kk)] = 0.25 * p.nx * p.ny * p.nz;
                sup.fields->set(U.data(), false);
                sup.initialDataDump();
                const long taken = sup.executeMainLoop();
                std::printf("steps %ld\nnum_save %d\ntime %.17g\nlast %d\n", taken, sup.inout->num_save,
                            sup.timestep->current_time, sup.inout->fileCounter());
            }
            spooky_b200::Supervisor again(p, nullptr, dir, -1);
            again.timestep->refresh();
            const spk_budgets_t b = again.fields->budgets();
            std::printf("restart_num_save %d\nrestart_time %.17g\nrestart_step %d\nrestart_lastsnap %.17g\n"
                        "restart_energy0 %.17g\n", again.inout->num_save, again.timestep->current_time,
                        again.timestep->current_step, again.inout->t_lastsnap, b.energy[0]);
        }
    } catch (const spooky_b200::Error& e) {
        std::printf("error %d %s\n", e.code, e.what());
        return 0;
    }
    return 0;
}
