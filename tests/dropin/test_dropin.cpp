// Drop-in check: the reference's own engine (indus::solve, src/engine/model.cpp:376-667),
// compiled from its sources, reaching the B200 backend through
// vajra-opt_b200/shim/indus_gpu_dropin.cpp with Options::use_gpu = true, exactly as the
// reference's GPU request test does (tests/test_pdhg.cpp:405-436).  The LPs are the ones of
// tests/test_pdhg.cpp:55-314 with their known optima; results must come back OPTIMAL from
// the engine's status guard and pass the engine's verifier.
//
// Exit code 0 = all cases pass; prints one line per case.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "indus/gpu.hpp"
#include "indus/model.hpp"
#include "indus/options.hpp"
#include "indus/verifier.hpp"

namespace {

constexpr double INF = 1e20;

struct Case {
    const char* name;
    int m, n;
    std::vector<indus::la::Triplet> trips;
    std::vector<double> c, cl, cu, rl, ru;
    indus::ObjSense sense;
    double optimum;
    bool presolve;
};

indus::Model make(const Case& k) {
    indus::Model model;
    model.name = k.name;
    model.num_rows = k.m;
    model.num_cols = k.n;
    model.sense = k.sense;
    model.c = k.c;
    model.col_lower = k.cl;
    model.col_upper = k.cu;
    model.row_lower = k.rl;
    model.row_upper = k.ru;
    model.A.set_from_triplets(k.m, k.n, k.trips);
    return model;
}

int run(const Case& k, const std::string& algo, const std::string& precision) {
    indus::Model model = make(k);
    indus::Options opts;
    opts.algorithm = "pdhg_cuda";                 // field assignment (string literals bind to set(key, bool))
    opts.use_gpu = true;
    opts.enable_presolve = k.presolve;
    opts.iteration_limit = 200000;
    opts.set("vajra_algorithm", std::string(algo));
    opts.set("vajra_precision", std::string(precision));
    if (algo == "reference") opts.set("tolerance", 1e-5);
    indus::Solution sol = indus::solve(model, opts);
    const bool opt_ok = sol.status == indus::SolveStatus::kOptimal;
    const bool obj_ok = std::abs(sol.objective_value - k.optimum) <= 1e-4 * (1.0 + std::abs(k.optimum));
    auto v = indus::verifier::verify_solution(model, sol, 1e-4);
    const auto t = indus::gpu::get_last_gpu_timing();
    const bool pass = opt_ok && obj_ok && v.passed;
    std::printf("%s %-18s %-9s %-5s status=%s obj=%.9g (expected %.9g) verifier=%d iters=%lld mode=%s\n",
                pass ? "PASS" : "FAIL", k.name, algo.c_str(), precision.c_str(), indus::to_string(sol.status),
                sol.objective_value, k.optimum, v.passed ? 1 : 0, static_cast<long long>(sol.iterations),
                t.kernel_mode.c_str());
    if (!pass) std::printf("     message: %s | %s\n", sol.status_message.c_str(), v.summary.c_str());
    return pass ? 0 : 1;
}

}  // namespace

int main() {
    const auto info = indus::gpu::probe_device();
    std::printf("device: %s available=%d\n", info.device_name.c_str(), info.available ? 1 : 0);
    if (!info.available) {
        // No CPU fallback: the engine must report UNSUPPORTED instead of solving.
        Case k{"no_device", 1, 2, {{0, 0, 1.0}, {0, 1, 1.0}}, {1, 1}, {0, 0}, {10, 10}, {3}, {10},
               indus::ObjSense::kMinimize, 3.0, false};
        indus::Options opts;
        opts.use_gpu = true;
        opts.enable_presolve = false;
        indus::Solution sol = indus::solve(make(k), opts);
        std::printf("no device -> %s (%s)\n", indus::to_string(sol.status), sol.status_message.c_str());
        return sol.status == indus::SolveStatus::kUnsupported ? 0 : 1;
    }
    const std::vector<Case> cases = {
        {"two_var", 3, 2, {{0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {2, 1, 1}}, {-1, -2}, {0, 0}, {INF, INF},
         {-INF, -INF, -INF}, {4, 3, 3}, indus::ObjSense::kMinimize, -7.0, false},
        {"equality", 2, 3, {{0, 0, 1}, {0, 1, 1}, {0, 2, 1}, {1, 0, 2}, {1, 1, 1}}, {1, 2, 3}, {0, 0, 0},
         {INF, INF, INF}, {6, 5}, {6, 5}, indus::ObjSense::kMinimize, 13.0, false},
        {"row_senses", 3, 2, {{0, 0, 1}, {0, 1, 1}, {1, 0, 1}, {1, 1, -1}, {2, 0, 2}, {2, 1, 1}}, {2, 3}, {0, 0},
         {10, 10}, {2, -INF, 1}, {INF, 4, 6}, indus::ObjSense::kMinimize, 4.0, false},
        {"free_column", 1, 2, {{0, 0, 1}, {0, 1, 1}}, {2, 1}, {-10, -INF}, {10, INF}, {5}, {5},
         indus::ObjSense::kMinimize, -5.0, false},
        {"minimise", 1, 2, {{0, 0, 1}, {0, 1, 1}}, {-2, -3}, {0, 0}, {INF, INF}, {-INF}, {5},
         indus::ObjSense::kMinimize, -15.0, false},
        {"maximise", 1, 2, {{0, 0, 1}, {0, 1, 1}}, {2, 3}, {0, 0}, {INF, INF}, {-INF}, {5},
         indus::ObjSense::kMaximize, 15.0, false},
        {"presolve_fixed", 2, 3, {{0, 0, 1}, {0, 1, 1}, {1, 1, 1}}, {-1, -1, 2}, {0, 0, 5}, {INF, INF, 5},
         {-INF, -INF}, {4, 10}, indus::ObjSense::kMinimize, 6.0, true},
        {"gpu_request", 1, 2, {{0, 0, 1}, {0, 1, 1}}, {1, 1}, {0, 0}, {10, 10}, {3}, {10},
         indus::ObjSense::kMinimize, 3.0, false},
    };
    int fails = 0;
    for (const auto& k : cases) {
        fails += run(k, "halpern", "mixed");
        fails += run(k, "halpern", "fp64");
    }
    std::printf("%s: %d failure(s)\n", fails ? "FAILED" : "OK", fails);
    return fails ? 1 : 0;
}
