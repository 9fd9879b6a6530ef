// The opaque vajra_pdhg handle and the two solver drivers.
#pragma once

#include <chrono>
#include <vector>

#include "problem.cuh"

struct vajra_pdhg {
    vajra_opts opts{};
    int device = 0;
    cudaStream_t stream = nullptr;
    vajra::DeviceLp lp;
    // host copies needed for closed-form trivial cases and post-processing sizes
    int m = 0, n = 0;
    int64_t nnz = 0;
    int sense = 0;
    double objective_offset = 0.0;
    std::vector<double> h_c, h_cl, h_cu, h_rl, h_ru;   // only kept for m == 0 / nnz == 0
    double upload_time_sec = 0.0;
    int64_t transfers = 0;
    // SpMV lane groups chosen by the first autotuned run of this handle; later runs reuse
    // them, so repeated runs of one handle sum in the same order and repeat bit for bit.
    int tuned = 0;                       // bit 0: FP32 shapes tuned, bit 1: FP64 shapes tuned
    int tuned_a32 = 8, tuned_at32 = 8;   // lane groups (0 = row-block kernel)
    int tuned_a64 = 8, tuned_at64 = 8;
    // The LP renumbered by descending row / column entry counts, built by the first HALPERN
    // run that asks for it and kept with the handle.
    bool ordered = false;
    vajra::DeviceLp lp_ordered;
    vajra::LpOrder order;
};

namespace vajra {

using Clock = std::chrono::steady_clock;
inline double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

// Elapsed time between two points of a stream's timeline (CUDA events).
struct StreamTimer {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    StreamTimer() { cudaEventCreate(&e0); cudaEventCreate(&e1); }
    ~StreamTimer() { if (e0) cudaEventDestroy(e0); if (e1) cudaEventDestroy(e1); }
    void start(cudaStream_t st) { cudaEventRecord(e0, st); }
    void stop(cudaStream_t st) { cudaEventRecord(e1, st); }
    double seconds() const {   // call after the stream passed stop()
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) return -1.0;
        return 1e-3 * ms;
    }
};

vajra_status run_reference(vajra_pdhg* h, vajra_result* r);
vajra_status run_halpern(vajra_pdhg* h, vajra_result* r);
vajra_status run_batch(int count, const vajra_lp* lps, const vajra_opts& o, vajra_result* results,
                       cudaStream_t st, double* device_time);
vajra_status run_unrolled(int count, const vajra_lp* lps, const vajra_unrolled_opts& o, const double* weights,
                          double* h_loss, double* h_x, double* h_gc, double* h_grl, double* h_gru, cudaStream_t st);

// Closed forms for LPs without rows or without nonzeros (pdhg.cpp:88-127 for m = 0 / n = 0;
// for nnz = 0 the rows decouple from the columns).  Returns true when it handled the LP.
bool solve_trivial(const vajra_pdhg* h, vajra_result* r);

void copy_out_vector(double* dst, const double* dev, int count, cudaStream_t st);

}  // namespace vajra
