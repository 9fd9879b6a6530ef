// Netlib end to end through the drop-in: the reference's MPS reader, its engine (presolve ->
// indus::gpu::solve_pdhg_gpu, which the shim maps onto libvajra_pdhg.so -> postsolve and the
// status guard), its solution writer and its file verifier.
//
//   netlib_e2e pack <model_dir> <out_dir> <name>...
//       Reads <model_dir>/<name>.mps with indus::io::read_mps (src/io/mps_reader.cpp) and
//       writes the Model to <out_dir>/<name>.lpbin (a plain binary dump: dimensions, CSC arrays,
//       bounds, objective, column types, names).  Runs where the model files are; the dumps
//       are build outputs that travel to a machine without them.
//   netlib_e2e solve <pack_dir> <sol_dir> <precision> <name>=<optimum>...
//       Loads each dump, solves it with indus::solve (src/engine/model.cpp:376-667) with
//       use_gpu and presolve on, writes <sol_dir>/<name>.sol with indus::io::write_solution
//       (src/io/writer.cpp:85-157), verifies that file against the model with
//       indus::verifier::verify_solution_file (src/engine/verifier.cpp), and compares the
//       objective with the published optimum.  One line per model; exit code 0 when all pass.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "indus/gpu.hpp"
#include "indus/io.hpp"
#include "indus/model.hpp"
#include "indus/options.hpp"
#include "indus/verifier.hpp"

namespace {

constexpr char kMagic[8] = {'V', 'J', 'L', 'P', 'B', 'I', 'N', '1'};

template <typename T>
void put(std::ofstream& f, const T& v) { f.write(reinterpret_cast<const char*>(&v), sizeof(T)); }
template <typename T>
void put_vec(std::ofstream& f, const std::vector<T>& v) {
    put<uint64_t>(f, v.size());
    if (!v.empty()) f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(sizeof(T) * v.size()));
}
void put_str(std::ofstream& f, const std::string& s) {
    put<uint64_t>(f, s.size());
    f.write(s.data(), static_cast<std::streamsize>(s.size()));
}
template <typename T>
bool get(std::ifstream& f, T& v) { return static_cast<bool>(f.read(reinterpret_cast<char*>(&v), sizeof(T))); }
template <typename T>
bool get_vec(std::ifstream& f, std::vector<T>& v) {
    uint64_t k = 0;
    if (!get(f, k) || k > (uint64_t(1) << 34)) return false;
    v.resize(k);
    return k == 0 || static_cast<bool>(f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(sizeof(T) * k)));
}
bool get_str(std::ifstream& f, std::string& s) {
    uint64_t k = 0;
    if (!get(f, k) || k > (uint64_t(1) << 20)) return false;
    s.resize(k);
    return k == 0 || static_cast<bool>(f.read(s.data(), static_cast<std::streamsize>(k)));
}

bool dump(const indus::Model& m, const std::string& path) {
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    f.write(kMagic, sizeof(kMagic));
    put<int32_t>(f, m.num_rows);
    put<int32_t>(f, m.num_cols);
    put<int32_t>(f, m.sense == indus::ObjSense::kMaximize ? 1 : 0);
    put<double>(f, m.objective_offset);
    put_str(f, m.name);
    put_vec(f, m.A.col_ptr);
    put_vec(f, m.A.row_idx);
    put_vec(f, m.A.values);
    put_vec(f, m.c);
    put_vec(f, m.row_lower);
    put_vec(f, m.row_upper);
    put_vec(f, m.col_lower);
    put_vec(f, m.col_upper);
    std::vector<uint8_t> types(m.col_type.size());
    for (size_t j = 0; j < types.size(); ++j) types[j] = static_cast<uint8_t>(m.col_type[j]);
    put_vec(f, types);
    put<uint64_t>(f, m.row_names.size());
    for (const auto& s : m.row_names) put_str(f, s);
    put<uint64_t>(f, m.col_names.size());
    for (const auto& s : m.col_names) put_str(f, s);
    return static_cast<bool>(f);
}

bool load(const std::string& path, indus::Model& m) {
    std::ifstream f(path, std::ios::binary);
    char magic[8];
    if (!f || !f.read(magic, sizeof(magic)) || std::memcmp(magic, kMagic, sizeof(kMagic)) != 0) return false;
    int32_t rows = 0, cols = 0, sense = 0;
    if (!get(f, rows) || !get(f, cols) || !get(f, sense) || !get(f, m.objective_offset) || !get_str(f, m.name)) return false;
    m.num_rows = rows;
    m.num_cols = cols;
    m.sense = sense ? indus::ObjSense::kMaximize : indus::ObjSense::kMinimize;
    m.A.m = rows;
    m.A.n = cols;
    std::vector<uint8_t> types;
    if (!get_vec(f, m.A.col_ptr) || !get_vec(f, m.A.row_idx) || !get_vec(f, m.A.values) || !get_vec(f, m.c) ||
        !get_vec(f, m.row_lower) || !get_vec(f, m.row_upper) || !get_vec(f, m.col_lower) || !get_vec(f, m.col_upper) ||
        !get_vec(f, types))
        return false;
    m.col_type.resize(types.size());
    for (size_t j = 0; j < types.size(); ++j) m.col_type[j] = static_cast<indus::VarType>(types[j]);
    uint64_t k = 0;
    if (!get(f, k) || k > static_cast<uint64_t>(rows)) return false;
    m.row_names.resize(k);
    for (auto& s : m.row_names) if (!get_str(f, s)) return false;
    if (!get(f, k) || k > static_cast<uint64_t>(cols)) return false;
    m.col_names.resize(k);
    for (auto& s : m.col_names) if (!get_str(f, s)) return false;
    return m.A.col_ptr.size() == static_cast<size_t>(cols) + 1 && m.c.size() == static_cast<size_t>(cols);
}

int pack(int argc, char** argv) {
    const std::string dir = argv[2], out = argv[3];
    int fails = 0;
    for (int i = 4; i < argc; ++i) {
        const std::string name = argv[i];
        try {
            indus::Model m = indus::io::read_mps(dir + "/" + name + ".mps");
            if (!dump(m, out + "/" + name + ".lpbin")) throw std::runtime_error("write failed");
            std::printf("packed %-10s %6d rows %6d cols %8lld nonzeros\n", name.c_str(), m.num_rows, m.num_cols,
                        static_cast<long long>(m.A.nnz()));
        } catch (const std::exception& e) {
            std::printf("FAILED %s: %s\n", name.c_str(), e.what());
            ++fails;
        }
    }
    return fails ? 1 : 0;
}

int solve(int argc, char** argv) {
    const std::string dir = argv[2], sol_dir = argv[3], precision = argv[4];
    const auto info = indus::gpu::probe_device();
    std::printf("device: %s available=%d precision=%s\n", info.device_name.c_str(), info.available ? 1 : 0,
                precision.c_str());
    int fails = 0;
    for (int i = 5; i < argc; ++i) {
        const std::string arg = argv[i];
        const size_t eq = arg.find('=');
        const std::string name = arg.substr(0, eq);
        const double optimum = std::strtod(arg.c_str() + eq + 1, nullptr);
        indus::Model model;
        if (eq == std::string::npos || !load(dir + "/" + name + ".lpbin", model)) {
            std::printf("FAIL %-10s cannot read %s/%s.lpbin\n", name.c_str(), dir.c_str(), name.c_str());
            ++fails;
            continue;
        }
        indus::Options opts;
        opts.algorithm = "pdhg_cuda";                 // field assignment (a literal binds to set(key, bool))
        opts.use_gpu = true;
        opts.enable_presolve = true;
        opts.iteration_limit = 2000000;
        opts.time_limit = 60.0;
        opts.set("vajra_precision", std::string(precision));
        indus::Solution sol = indus::solve(model, opts);
        const std::string sol_path = sol_dir + "/" + name + ".sol";
        indus::io::write_solution(sol, model, sol_path);
        const auto v = indus::verifier::verify_solution_file(model, sol_path, 1e-6);
        const auto t = indus::gpu::get_last_gpu_timing();
        const double rel = std::abs(sol.objective_value - optimum) / (1.0 + std::abs(optimum));
        const bool pass = sol.status == indus::SolveStatus::kOptimal && rel <= 1e-6 && v.passed;
        std::printf("%s %-10s status=%s obj=%.11g published=%.11g rel_err=%.2e verifier=%d iters=%lld "
                    "gpu_iter_s=%.4f mode=%s\n",
                    pass ? "PASS" : "FAIL", name.c_str(), indus::to_string(sol.status), sol.objective_value, optimum,
                    rel, v.passed ? 1 : 0, static_cast<long long>(sol.iterations), t.iteration_time_sec,
                    t.kernel_mode.c_str());
        if (!pass) std::printf("     message: %s | %s\n", sol.status_message.c_str(), v.summary.c_str());
        fails += pass ? 0 : 1;
    }
    std::printf("%s: %d failure(s)\n", fails ? "FAILED" : "OK", fails);
    return fails ? 1 : 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc >= 4 && std::strcmp(argv[1], "pack") == 0) return pack(argc, argv);
    if (argc >= 5 && std::strcmp(argv[1], "solve") == 0) return solve(argc, argv);
    std::fprintf(stderr, "usage: %s pack <model_dir> <out_dir> <name>... | solve <pack_dir> <sol_dir> <mixed|fp64> "
                         "<name>=<optimum>...\n", argv[0]);
    return 2;
}
