// ref_driver.cu -- times the reference's own CUDA build (LorenzoLMP/spooky-git,
// cuFFT + cuBLAS, FP64) on its main-loop body, in place of its src/main.cu
// (which needs the argparse library, absent here).
//
//   spooky_ref <input_dir> <state_in.bin> <warmup> <steps> [state_out.bin]
//
// It builds the reference's objects exactly as main.cu does (Supervisor,
// init_plan, init_cublas, Fields::allocate_and_move_to_gpu), then replaces
// the initial condition by the spectral state in state_in.bin
// ([F][NX][NY][NZ/2+1] complex FP64, the reference's d_all_fields layout),
// cleans its divergence, and runs `warmup` + `steps` iterations of the body
// of Supervisor::executeMainLoop (supervisor.cu:179-192: CleanFieldDivergence,
// TimeStepping::HydroMHDAdvance) without the output checks.  The timed steps
// lie between two CUDA events on the legacy stream, with a device
// synchronisation on each side.  One JSON line goes to stdout; the final
// state goes to state_out.bin when given.
// MEASUREMENT INFRASTRUCTURE: compiled with the reference's sources by
// oracle/refbuild/Makefile, never part of the library.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "common.hpp"
#include "cufft_routines.hpp"
#include "cublas_routines.hpp"
#include "fields.hpp"
#include "parameters.hpp"
#include "supervisor.hpp"
#include "timestepping.hpp"

Variables vars;
Grid grid;
Parser parser;
int threadsPerBlock{512};

#define CKR(x)                                                                              \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) {                                                            \
            std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));                   \
            return 4;                                                                       \
        }                                                                                   \
    } while (0)

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s input_dir state_in.bin warmup steps [state_out.bin]\n", argv[0]);
        return 2;
    }
    parser.input_dir = argv[1];
    parser.restart_num = -2;
    parser.stats_frequency = -1;
    const int warmup = std::atoi(argv[3]);
    const int steps = std::atoi(argv[4]);

    Supervisor spooky;
    init_plan(grid.FFT_SIZE);
    init_cublas();
    spooky.fields_ptr->allocate_and_move_to_gpu();

    const size_t n = (size_t)vars.NUM_FIELDS * grid.NTOTAL_COMPLEX;
    std::vector<data_type> U(n);
    FILE* f = std::fopen(argv[2], "rb");
    if (!f || std::fread(U.data(), sizeof(data_type), n, f) != n) {
        std::fprintf(stderr, "cannot read %zu complex values from %s\n", n, argv[2]);
        return 2;
    }
    std::fclose(f);
    CKR(cudaMemcpy(spooky.fields_ptr->d_all_fields, U.data(), sizeof(data_type) * n, cudaMemcpyHostToDevice));
    spooky.fields_ptr->CleanFieldDivergence();

    for (int i = 0; i < warmup; i++) {
        spooky.fields_ptr->CleanFieldDivergence();
        spooky.timestep_ptr->HydroMHDAdvance(spooky.fields_ptr);
    }
    cudaEvent_t e0, e1;
    CKR(cudaEventCreate(&e0));
    CKR(cudaEventCreate(&e1));
    CKR(cudaDeviceSynchronize());
    const unsigned ffts0 = spooky.NumFFTs;
    CKR(cudaEventRecord(e0, 0));
    for (int i = 0; i < steps; i++) {
        spooky.fields_ptr->CleanFieldDivergence();
        spooky.timestep_ptr->HydroMHDAdvance(spooky.fields_ptr);
    }
    CKR(cudaEventRecord(e1, 0));
    CKR(cudaDeviceSynchronize());
    float ms = 0.f;
    CKR(cudaEventElapsedTime(&ms, e0, e1));
    CKR(cudaGetLastError());

    if (argc > 5) {
        CKR(cudaMemcpy(U.data(), spooky.fields_ptr->d_all_fields, sizeof(data_type) * n, cudaMemcpyDeviceToHost));
        FILE* g = std::fopen(argv[5], "wb");
        if (!g || std::fwrite(U.data(), sizeof(data_type), n, g) != n) {
            std::fprintf(stderr, "cannot write %s\n", argv[5]);
            return 2;
        }
        std::fclose(g);
    }
    std::printf("{\"ms_total\": %.6f, \"steps\": %d, \"warmup\": %d, \"ms_per_step\": %.6f, "
                "\"steps_per_s\": %.6f, \"t\": %.17g, \"step\": %u, \"dt\": %.17g, \"ffts_per_step\": %.3f, "
                "\"nx\": %zu, \"ny\": %zu, \"nz\": %zu, \"fields\": %d}\n",
                ms, steps, warmup, ms / steps, 1000.0 * steps / ms, spooky.timestep_ptr->current_time,
                spooky.timestep_ptr->current_step, spooky.timestep_ptr->current_dt,
                steps > 0 ? (double)(spooky.NumFFTs - ffts0) / steps : 0.0, grid.NX, grid.NY, grid.NZ,
                vars.NUM_FIELDS);
    spooky.fields_ptr->clean_gpu();
    finish_cufft();
    finish_cublas();
    return 0;
}
