// Internal interface between the translation units of libb200ode.so
// (b200ode.cu: kernels + integrate ABI; serve.cu: the request loop).
// Host code only; not installed, not part of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>

#include "../../include/b200ode.h"
#include "mech_dev.h"

struct b200ode_handle {
    int mech = -1;
    b200::HostMech hm;
    unsigned char* d_blob = nullptr;
    b200::DevMech dm;
    b200ode_options opt;
    int device = 0, num_sms = 0;
    size_t cap = 0;   // cells
    double* d_T = nullptr;
    double* d_Y = nullptr;
    double* d_P = nullptr;
    int32_t* d_status = nullptr;
    int32_t* d_cnt = nullptr;
    unsigned long long* d_ctl = nullptr;   // [0] queue, [1..8] totals, [9] done, [10..14] phase cycles
    void* d_wg = nullptr;                    // WarpGlobal scratch (saved Jacobians, ...)
    size_t wg_bytes = 0;
    unsigned char* d_rec = nullptr;          // step-form per-cell records
    size_t rec_bytes = 0;
    unsigned long long* h_done = nullptr;    // pinned host copy of the done counter
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    int last_blocks_per_sm = 0;
    int auto_wpb = 0;                        // warps per CTA picked by occupancy (0 = not yet)
    std::map<int, int> auto_minb;            // register variant per CTA shape (see bdf_kernel)
};

namespace b200 {

// Records msg as this thread's last error (b200ode_last_error) and returns st.
b200ode_status set_error(b200ode_status st, const std::string& msg);

// Number of 64-bit words of a persistent launch's control block: [0] work-queue
// head, [1..8] call totals (nst, nfe, nje, nsetups, nni, ncfn, netf, failed
// cells), [9] unused, [10..14] phase cycles.
constexpr int kCtlWords = 16;

// Device bytes of per-warp scratch that a persistent launch of handle h over
// n cells uses (resident warps x WarpGlobal).  0 on error (message set).
size_t persistent_scratch_bytes(b200ode_handle* h, int64_t n);

// Launches the persistent BDF kernel over n cells on stream st.  ctl
// (kCtlWords words) is cleared on the stream before the launch; wg must hold
// persistent_scratch_bytes(h, n) bytes.  Does not touch the handle's own
// device buffers, so several launches of one handle may run on different
// streams at once, each with its own ctl and wg.
b200ode_status launch_persistent(b200ode_handle* h, int64_t n, const double* dP, double P_scalar,
                                 double* dT, double* dY, int32_t* dstat, double t0, double t1,
                                 unsigned long long* ctl, void* wg, cudaStream_t st);

}  // namespace b200
