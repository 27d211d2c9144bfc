/* spooky_b200.hpp -- C++ surface of the B200 SPOOKY path with the reference's
 * class names, forwarding to the C ABI of spooky_b200.h.
 *
 * Reference = LorenzoLMP/spooky-git:
 *   Parameters    src/parameters/parameters.hpp   (spooky.cfg reader)
 *   Fields        src/fields/fields.hpp           (the spectral state)
 *   TimeStepping  src/timestepping/timestepping.hpp:15-56
 *   RKLegendre    src/rkl/rkl.hpp
 *   Supervisor    src/supervisor/supervisor.hpp:24-84 (executeMainLoop)
 * One Supervisor owns one spk_ctx (device state, pass buffers, CUDA graphs);
 * Fields, TimeStepping and RKLegendre are views of it.  Errors that the
 * reference prints and continues past throw spooky_b200::Error here. */
#pragma once
#include <sys/stat.h>

#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "spooky_b200.h"

namespace spooky_b200 {

struct Error : std::runtime_error {
    int code;
    Error(int rc, const std::string& msg) : std::runtime_error(msg), code(rc) {}
};

inline void check(int rc, const spk_ctx* ctx) {
    if (rc != SPK_OK) {
        const char* m = spk_last_error(ctx);
        throw Error(rc, m ? m : "spooky_b200 error");
    }
}

/* Parameters: the members of spk_params_t carry the reference's names (lx, nu,
 * cfl, t_final, mhd, ...; grid.NX[] is nx, ny, nz). */
class Parameters : public spk_params_t {
public:
    Parameters() { spk_params_default(this); }
    /* Parameters::Parameters(Supervisor&, char* configfile) */
    explicit Parameters(const std::string& configfile) { check(spk_params_from_file(configfile.c_str(), this), nullptr); }
    static Parameters from_string(const std::string& text) {
        Parameters p;
        check(spk_params_from_string(text.c_str(), &p), nullptr);
        return p;
    }
};

class Supervisor;

/* The spectral state U[f][i][j][k] (k < nz/2+1), complex FP64, held on the device. */
class Fields {
public:
    explicit Fields(spk_ctx* ctx) : ctx_(ctx) { check(spk_sizes(ctx_, &num_fields, &n_complex), ctx_); }
    int num_fields = 0;
    size_t n_complex = 0;
    /* U: 2 * num_fields * n_complex doubles (interleaved complex), host or device */
    void set(const double* U, bool device) { check(spk_set_state(ctx_, U, device ? 0 : 1), ctx_); }
    void get(double* U, bool device) { check(spk_get_state(ctx_, U, device ? 0 : 1), ctx_); }
    std::vector<double> get_host() {
        std::vector<double> v(2 * (size_t)num_fields * n_complex);
        get(v.data(), false);
        return v;
    }
    /* Fields::CleanFieldDivergence */
    void CleanFieldDivergence() { check(spk_clean_divergence(ctx_), ctx_); }
    /* Supervisor::Complex2RealFields into a device buffer of num_fields*nx*ny*nz doubles */
    void Complex2RealFields(double* R_device) { check(spk_to_real(ctx_, R_device), ctx_); }
    /* energy and dissipation per field (FP64) */
    spk_budgets_t budgets() {
        spk_budgets_t b;
        check(spk_budgets(ctx_, &b), ctx_);
        return b;
    }

private:
    spk_ctx* ctx_;
};

class TimeStepping {
public:
    explicit TimeStepping(spk_ctx* ctx) : ctx_(ctx) {}
    double current_dt = 0.0, dt_hyp = 0.0, dt_par = 0.0, dt_sts = 0.0, current_time = 0.0;
    int current_step = 0;
    /* TimeStepping::compute_dt(complexFields, realBuffer) on the context state */
    void compute_dt() { check(spk_compute_dt(ctx_, &dt_hyp, &dt_par, &dt_sts, &current_dt), ctx_); }
    /* ... and on a caller's device array (the reference's d_all_fields); the real buffer is the library's */
    void compute_dt(const double* complexFields, double* /*realBuffer*/) {
        check(spk_compute_dt_fields(ctx_, complexFields, &dt_hyp, &dt_par, &dt_sts, &current_dt), ctx_);
    }
    /* TimeStepping::RungeKutta3(complex_Fields, real_Buffer) in place on a caller's
     * device array, with the dt of the last compute_dt */
    void RungeKutta3(double* complex_Fields, double* /*real_Buffer*/) { check(spk_rk3_fields(ctx_, complex_Fields), ctx_); }
    /* TimeStepping::HydroMHDAdvance on a caller's device array (with the
     * CleanFieldDivergence of the main loop), nsteps times, asynchronously */
    void HydroMHDAdvance(double* complex_Fields, int nsteps) { check(spk_advance_fields(ctx_, complex_Fields, nsteps), ctx_); }
    /* TimeStepping::compute_dfield(complex_Fields, real_Buffer, complex_dFields):
     * device pointers; the real buffer is the library's own and may be null */
    void compute_dfield(const double* complex_Fields, double* /*real_Buffer*/, double* complex_dFields) {
        check(spk_compute_dfield(ctx_, complex_Fields, complex_dFields), ctx_);
    }
    /* TimeStepping::HydroMHDAdvance (with the CleanFieldDivergence that
     * Supervisor::executeMainLoop calls before it), nsteps times, asynchronously */
    void HydroMHDAdvance(int nsteps = 1) { check(spk_advance(ctx_, nsteps), ctx_); }
    /* host copies of time, dt and step count (synchronises) */
    void refresh() {
        check(spk_synchronize(ctx_), ctx_);
        check(spk_get_time(ctx_, &current_time, &current_dt, &current_step), ctx_);
    }

private:
    spk_ctx* ctx_;
};

class RKLegendre {
public:
    explicit RKLegendre(spk_ctx* ctx) : ctx_(ctx) {}
    /* RKLegendre::compute_cycle: one cycle of the configured scheme (STS, RKL1, RKL2) with the last dt; returns the stage count */
    int compute_cycle() {
        int s = 0;
        check(spk_rkl_cycle(ctx_, &s), ctx_);
        return s;
    }
    /* RKLegendre::compute_cycle(complex_Fields, real_Buffer) on a caller's device array */
    int compute_cycle(double* complex_Fields, double* /*real_Buffer*/) {
        int s = 0;
        check(spk_rkl_cycle_fields(ctx_, complex_Fields, &s), ctx_);
        return s;
    }

private:
    spk_ctx* ctx_;
};

/* InputOutput (src/io/inputoutput.hpp): the snapshot schedule and files of
 * the main loop (check_output.cu:59-97, hdf5_io.cu:19-276).  A snapshot is
 * due when t - t_lastsnap + 1e-8 >= toutput_flow (and at t = 0); each one
 * first cleans the divergence and advances t_lastsnap by toutput_flow, which
 * the dt rule reads.  With an output directory the snapshots are written to
 * <dir>/data/snapNNNN.h5 in the reference's HDF5 layout (spk_write_snapshot). */
class InputOutput {
public:
    InputOutput(spk_ctx* ctx, const Parameters& p, std::string output_dir)
        : ctx_(ctx), p_(p), output_dir(std::move(output_dir)) {}
    double t_lastsnap = 0.0, t_lastvar = 0.0;
    int num_save = 0;
    std::string output_dir;   // empty: the schedule runs, nothing is written

    std::string snapshot_path(int num) const {
        char name[32];
        std::snprintf(name, sizeof(name), "snap%04d.h5", num);
        return output_dir + "/data/" + name;
    }
    /* fileCounter (hdf5_io.cu:255-276): the number of the most recent snapshot, -1 when none */
    int fileCounter() const {
        int n = -1;
        struct stat st;
        while (stat(snapshot_path(n + 1).c_str(), &st) == 0) n++;
        return n;
    }
    void CheckSnapshot() {
        double t = 0.0, dt = 0.0;
        int step = 0;
        check(spk_get_time(ctx_, &t, &dt, &step), ctx_);
        if (t - t_lastsnap + 1e-8 >= p_.toutput_flow || t == 0.0) {
            check(spk_clean_divergence(ctx_), ctx_);
            if (t != 0.0) {
                t_lastsnap += p_.toutput_flow;
                check(spk_set_time(ctx_, t, step, t_lastsnap), ctx_);
            }
            if (!output_dir.empty()) WriteDataFile();
            num_save++;
        }
    }
    void WriteDataFile() {
        check(spk_write_snapshot(ctx_, snapshot_path(num_save).c_str(), p_.t_initial, t_lastsnap, t_lastvar), ctx_);
    }
    /* InputOutput::ReadDataFile(restart_num): -1 (or past the last file) the most
     * recent snapshot; returns the number read, -1 when there is none */
    int ReadDataFile(int restart_num) {
        const int last = fileCounter();
        if (last < 0) return -1;
        const int num = (restart_num == -1 || restart_num > last) ? last : restart_num;
        check(spk_read_snapshot(ctx_, snapshot_path(num).c_str(), &t_lastsnap, &t_lastvar), ctx_);
        num_save = num + 1;
        return num;
    }

private:
    spk_ctx* ctx_;
    const Parameters& p_;
};

class Supervisor {
public:
    /* cuda_stream: a cudaStream_t, or null for a stream owned by the context.
     * output_dir: where snapshots go (<dir>/data), empty for none.
     * restart_num: -2 a new run, -1 the most recent snapshot, n >= 0 snap n (main.cu's -r). */
    explicit Supervisor(const Parameters& p, void* cuda_stream = nullptr, const std::string& output_dir = "",
                        int restart_num = -2)
        : param(p), restart_num(restart_num) {
        spk_ctx* c = nullptr;
        check(spk_ctx_create(&param, cuda_stream, &c), nullptr);
        ctx_.reset(c);
        fields = std::make_unique<Fields>(c);
        timestep = std::make_unique<TimeStepping>(c);
        rkl = std::make_unique<RKLegendre>(c);
        inout = std::make_unique<InputOutput>(c, param, output_dir);
        if (restart_num >= -1) Restart();
    }
    Parameters param;
    int restart_num;
    std::unique_ptr<Fields> fields;
    std::unique_ptr<TimeStepping> timestep;
    std::unique_ptr<RKLegendre> rkl;
    std::unique_ptr<InputOutput> inout;

    /* Supervisor::Restart (supervisor.cu:241-245); no snapshot on disk: a new run */
    void Restart() {
        if (inout->output_dir.empty()) throw Error(SPK_ERR_ARG, "a restart needs an output directory");
        if (inout->ReadDataFile(restart_num) < 0) restart_num = -2;
    }
    /* the snapshot of t = 0 of a new run (supervisor.cu:215-225) */
    void initialDataDump() {
        if (restart_num == -2) inout->CheckSnapshot();
    }

    /* Supervisor::executeMainLoop (src/supervisor/supervisor.cu:169-213): steps
     * until t_final (or max_steps >= 0), each followed by the snapshot check;
     * returns the steps taken.  The device time is read after every chunk of
     * `check_every` steps (1, the default, matches the reference's loop; a
     * larger chunk avoids a host round trip per step but may end with steps of
     * zero length at t_final, which still count in current_step, and may pass
     * a snapshot time). */
    long executeMainLoop(long max_steps = -1, int check_every = 1) {
        long n = 0;
        timestep->refresh();
        while (timestep->current_time < param.t_final && (max_steps < 0 || n < max_steps)) {
            int k = check_every;
            if (max_steps >= 0 && max_steps - n < k) k = (int)(max_steps - n);
            timestep->HydroMHDAdvance(k);
            n += k;
            inout->CheckSnapshot();
            timestep->refresh();
        }
        return n;
    }
    spk_ctx* context() { return ctx_.get(); }

private:
    struct Del {
        void operator()(spk_ctx* c) const { spk_ctx_destroy(c); }
    };
    std::unique_ptr<spk_ctx, Del> ctx_;
};

}  // namespace spooky_b200
