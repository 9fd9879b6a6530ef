// Drop-in replacement for the reference's src/solvers/gpu/gpu_context.cpp and
// src/solvers/gpu/pdhg_cuda.cu: implements the unchanged C++ surface of
// include/indus/gpu.hpp:49-59 over libvajra_pdhg.so's C ABI (include/vajra_pdhg.h).
//
// Build it with the reference's headers (C++20: they use <span>) and link it, together
// with libvajra_pdhg.so, in place of those two files; indus::solve
// (src/engine/model.cpp:524-525), the CLI and the benchmark harness then reach the B200
// backend unmodified.  There is no CPU fallback: without a device, solve_pdhg_gpu returns
// SolveStatus::kUnsupported with the reason in status_message.
//
// Options read (same keys as the reference, include/indus/options.hpp and
// src/solvers/gpu/pdhg_cuda.cu:249-251): iteration_limit, time_limit, enable_scaling,
// "check_frequency".  The backend's own keys:
//   "vajra_algorithm"  "halpern" (default) or "reference" (the CPU PDHG's semantics, FP64)
//   "vajra_precision"  "mixed" (default) or "fp64"
//   "vajra_tolerance"  relative KKT target of "halpern" (default 1e-8)
//   "vajra_max_violation"  "halpern" also stops only when the maxima the engine's status guard
//                      checks (model.cpp:203-374, 626-664) are below this (default 5e-8, half the
//                      guard's 1e-7), so OPTIMAL results survive the guard
//   "vajra_max_abs_violation"  ... and until every row violation is below this in absolute
//                      terms (default 5e-7, half the verifier's default 1e-6)
//   "tolerance", "gap_tolerance" are used by "reference" exactly as the CPU PDHG uses them.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "indus/gpu.hpp"
#include "indus/tolerances.hpp"
#include "vajra_pdhg.h"

namespace indus::gpu {

namespace {

thread_local GpuTimingDiagnostics g_last_timing{};

SolveStatus to_status(int32_t s) {
    return static_cast<SolveStatus>(static_cast<uint8_t>(s));
}

}  // namespace

GpuDeviceInfo probe_device() noexcept {
    GpuDeviceInfo info;
    vajra_device_info d;
    if (vajra_probe_device(0, &d) != VAJRA_OK) {
        info.available = false;
        info.device_name = d.device_name;
        return info;
    }
    info.available = true;
    info.device_name = d.device_name;
    info.total_vram_bytes = static_cast<size_t>(d.total_vram_bytes);
    info.free_vram_bytes = static_cast<size_t>(d.free_vram_bytes);
    info.compute_capability_major = d.compute_capability_major;
    info.compute_capability_minor = d.compute_capability_minor;
    info.multi_processor_count = d.multi_processor_count;
    return info;
}

bool is_cuda_available() noexcept { return vajra_is_cuda_available() != 0; }

GpuTimingDiagnostics get_last_gpu_timing() noexcept { return g_last_timing; }

Solution solve_pdhg_gpu(const Model& model, const Options& options) {
    const int m = model.num_rows;
    const int n = model.num_cols;
    Solution sol;
    sol.algorithm_used = "pdhg_cuda";
    sol.col_value.assign(static_cast<size_t>(n), 0.0);
    sol.row_value.assign(static_cast<size_t>(m), 0.0);
    sol.row_dual.assign(static_cast<size_t>(m), 0.0);
    sol.col_dual.assign(static_cast<size_t>(n), 0.0);
    sol.col_basis_status.assign(static_cast<size_t>(n), BasisStatus::kUnknown);
    sol.row_basis_status.assign(static_cast<size_t>(m), BasisStatus::kUnknown);
    if (vajra_abi_version() != VAJRA_ABI_VERSION) {
        sol.status = SolveStatus::kUnsupported;
        sol.status_message = "libvajra_pdhg ABI " + std::to_string(vajra_abi_version()) +
                             " does not match this build's header (" + std::to_string(VAJRA_ABI_VERSION) + ")";
        return sol;
    }

    vajra_lp lp{};
    lp.num_rows = m;
    lp.num_cols = n;
    lp.nnz = model.A.nnz();
    lp.col_ptr = model.A.col_ptr.empty() ? nullptr : model.A.col_ptr.data();
    std::vector<int64_t> empty_ptr;
    if (!lp.col_ptr) {
        empty_ptr.assign(static_cast<size_t>(n) + 1, 0);
        lp.col_ptr = empty_ptr.data();
    }
    lp.row_idx = model.A.row_idx.data();
    lp.values = model.A.values.data();
    lp.c = model.c.data();
    lp.col_lower = model.col_lower.data();
    lp.col_upper = model.col_upper.data();
    lp.row_lower = model.row_lower.data();
    lp.row_upper = model.row_upper.data();
    lp.sense = model.sense == ObjSense::kMaximize ? 1 : 0;
    lp.objective_offset = model.objective_offset;

    vajra_opts o;
    vajra_default_opts(&o);
    const std::string algo = options.get_string("vajra_algorithm", "halpern");
    o.algorithm = algo == "reference" ? VAJRA_ALGO_REFERENCE : VAJRA_ALGO_HALPERN;
    o.precision = options.get_string("vajra_precision", "mixed") == "fp64" ? VAJRA_PREC_FP64 : VAJRA_PREC_MIXED;
    if (o.algorithm == VAJRA_ALGO_REFERENCE) {
        o.tolerance = options.get_double("tolerance", 1e-6);
        o.gap_tolerance = options.get_double("gap_tolerance", 1e-6);
        o.check_frequency = static_cast<int32_t>(options.get_int("check_frequency", 100));
    } else {
        o.tolerance = options.get_double("vajra_tolerance", 1e-8);
        // the engine re-checks every OPTIMAL result with its status guard (model.cpp:626-664,
        // 1e-7 absolute or relative); stop only once the guard's maxima are below half of that
        o.max_violation = options.get_double("vajra_max_violation", 0.5 * tol::kPrimalFeasibility);
        // and the verifier's absolute row check (verify_solution, default tolerance 1e-6)
        o.max_abs_violation = options.get_double("vajra_max_abs_violation", 5e-7);
        o.check_frequency = static_cast<int32_t>(options.get_int("check_frequency", 64));
    }
    o.iteration_limit = options.iteration_limit;
    o.time_limit = options.time_limit;
    o.enable_scaling = options.enable_scaling ? 1 : 0;

    vajra_result r{};
    r.col_value = sol.col_value.data();
    r.row_value = sol.row_value.data();
    r.row_dual = sol.row_dual.data();
    r.col_dual = sol.col_dual.data();
    const vajra_status s = vajra_pdhg_solve(&lp, &o, &r);

    vajra_timing t{};
    vajra_last_timing(&t);
    g_last_timing = {};
    g_last_timing.upload_time_sec = t.upload_time_sec;
    g_last_timing.iteration_time_sec = t.iteration_time_sec;
    g_last_timing.download_time_sec = t.download_time_sec;
    g_last_timing.total_time_sec = t.total_time_sec;
    g_last_timing.host_device_transfers = t.host_device_transfers;
    g_last_timing.iterations = t.iterations;
    g_last_timing.device_name = t.device_name;
    g_last_timing.kernel_mode = t.kernel_mode;

    sol.status_message = r.status_message;
    if (s != VAJRA_OK) {
        sol.status = s == VAJRA_ERR_NO_DEVICE ? SolveStatus::kUnsupported
                   : s == VAJRA_ERR_INVALID_ARGUMENT ? SolveStatus::kModelError : SolveStatus::kNumericalError;
        return sol;
    }
    sol.status = to_status(r.status);
    sol.iterations = r.iterations;
    sol.objective_value = r.objective_value;
    sol.best_dual_bound = r.objective_value;
    sol.solve_time_seconds = r.total_time_sec;
    // Basis-status heuristic of the reference PDHG (src/solvers/pdhg/pdhg.cpp:420-432).
    for (int j = 0; j < n; ++j) {
        const double xj = sol.col_value[static_cast<size_t>(j)];
        const double lj = model.col_lower[static_cast<size_t>(j)];
        const double uj = model.col_upper[static_cast<size_t>(j)];
        BasisStatus& b = sol.col_basis_status[static_cast<size_t>(j)];
        if (std::abs(lj - uj) <= tol::kZeroDrop) b = BasisStatus::kFixed;
        else if (std::abs(xj - lj) <= 1e-5) b = BasisStatus::kAtLower;
        else if (std::abs(xj - uj) <= 1e-5) b = BasisStatus::kAtUpper;
        else b = BasisStatus::kBasic;
    }
    sol.recompute_quality(model);
    return sol;
}

}  // namespace indus::gpu
