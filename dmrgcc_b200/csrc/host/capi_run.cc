// C ABI of the sweep engine: runs a reference input file end to end, and
// exposes the model layer (MPO, quantum tables) for inspection.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "dmrg_b200.h"
#include "host/engine.h"
#include "host/input.h"
#include "host/model.h"

using namespace dmrg;

namespace {

struct ModelSpec {
    std::unique_ptr<QuantumSpace> space;
    std::unique_ptr<MpoHamiltonian> ham;
};

// The lattice and filling a model can be built for.  The reference takes these
// keys as given; outside these ranges its quantum-number tables come out empty
// or inconsistent, so the library rejects them before building anything.
void check_sizes(int nx, int ny, int d, std::initializer_list<int> bosons) {
    if (nx < 1 || ny < 1) throw std::runtime_error("num_site_x and num_site_y must be at least 1");
    if (d < 2) throw std::runtime_error("physics_dim must be at least 2 (n_max = physics_dim - 1 >= 1)");
    const long long cap = (long long)(d - 1) * nx * ny;
    for (int n : bosons)
        if (n < 0 || n > cap)
            throw std::runtime_error("boson number " + std::to_string(n) + " outside [0, (physics_dim - 1) * sites = " +
                                     std::to_string(cap) + "]");
}

// The model executables' main() (model/real_spinless_bose_square_model.cc:11-35):
// read the model keys and build the space and the Hamiltonian.
ModelSpec make_model(InputGroup& input, const std::string& model) {
    ModelSpec m;
    if (model == "real_spinful_bose_square" || model == "complex_spinful_bose_square") {
        // model/complex_spinful_bose_square_model.cc:11-45 (same keys); the real
        // form needs flux 0, the complex one is the reference's model
        const int nx = input.getInt("num_site_x");
        const int ny = input.getInt("num_site_y");
        const int d = input.getInt("physics_dim", 2);
        const bool px = input.getBool("period_x");
        const bool py = input.getBool("period_y");
        const int nb[2] = {input.getInt("Nup"), input.getInt("Ndown")};
        const double flux = input.getDouble("flux");
        const double jx = input.getDouble("Jx");
        const double jy = input.getDouble("Jy");
        const double mu = input.getDouble("mu");
        const double u[3] = {input.getDouble("U_uu"), input.getDouble("U_dd"), input.getDouble("U_ud")};
        check_sizes(nx, ny, d, {nb[0], nb[1]});
        m.space.reset(new RealSpinfulBoseSquareSpace(nx, ny, nb, d));
        if (model == "complex_spinful_bose_square")
            m.ham.reset(new ComplexSpinfulBoseSquareHamiltonian(nx, ny, d, flux, jx, jy, u, mu, px, py));
        else
            m.ham.reset(new RealSpinfulBoseSquareHamiltonian(nx, ny, d, flux, jx, jy, u, mu, px, py));
        return m;
    }
    if (model != "real_spinless_bose_square" && model != "complex_spinless_bose_square")
        throw std::runtime_error("unknown model '" + model +
                                 "' (supported: real_spinless_bose_square, complex_spinless_bose_square, "
                                 "real_spinful_bose_square, complex_spinful_bose_square)");
    // model/real_spinless_bose_square_model.cc:11-42, or its complex twin
    // model/complex_spinless_bose_square_model.cc (same keys, same space; the
    // Hamiltonian's operators complex, so the run is ComplexTensorRundmrg's)
    const int nx = input.getInt("num_site_x");
    const int ny = input.getInt("num_site_y");
    const int nb = input.getInt("num_boson");
    const int d = input.getInt("physics_dim", 2);
    const double flux = input.getDouble("flux");
    const double jx = input.getDouble("Jx");
    const double jy = input.getDouble("Jy");
    const double u = input.getDouble("U");
    const double mu = input.getDouble("mu");
    const bool px = input.getBool("period_x");
    const bool py = input.getBool("period_y");
    check_sizes(nx, ny, d, {nb});
    m.space.reset(new RealSpinlessBoseSquareSpace(nx, ny, nb, d));
    const double flux_value = flux * 3.14159265358979323846;
    if (model == "complex_spinless_bose_square")
        m.ham.reset(new ComplexSpinlessBoseSquareHamiltonian(nx, ny, d, flux_value, jx, jy, u, mu, px, py));
    else
        m.ham.reset(new RealSpinlessBoseSquareHamiltonian(nx, ny, d, flux_value, jx, jy, u, mu, px, py));
    return m;
}

}  // namespace

struct dmrg_run_s {
    std::unique_ptr<Engine> engine;
    double total_seconds = 0.0;
};

struct dmrg_model_s {
    ModelSpec spec;
};

extern "C" {

int dmrg_run_create(dmrg_ctx_t ctx, const char* input_path, const char* model, const dmrg_run_options_t* opt,
                    dmrg_run_t* out) {
    if (!ctx || !input_path || !out) return set_error(DMRG_E_ARG, "null argument");
    *out = nullptr;
    try {
        RunOptions o;
        if (opt) {
            o.precision = opt->precision;
            if (o.precision != DMRG_PREC_FP64 && o.precision != DMRG_PREC_TF32X3 && o.precision != DMRG_PREC_BF16X3)
                return set_error(DMRG_E_ARG, "unsupported precision %d (DMRG_PREC_FP64, _TF32X3 or _BF16X3)",
                                 o.precision);
            o.verbose = opt->verbose;
            o.seed = opt->seed ? opt->seed : 1;
            o.stop_after_half_sweeps = opt->stop_after_half_sweeps;
            if (opt->lanczos_precision > 0) o.lanczos_precision = opt->lanczos_precision;
            o.two_site = opt->two_site != 0;
            o.lanczos_graph = opt->lanczos_graph == 0 ? -1 : (opt->lanczos_graph > 0 ? 1 : 0);
        }
        InputGroup input(input_path, "input", o.verbose != 0);
        ModelSpec m = make_model(input, model ? model : "real_spinless_bose_square");
        AllocScope pool(ctx->stream);  // the run's tensors come from the stream-ordered pool
        std::unique_ptr<dmrg_run_s> r(new dmrg_run_s());
        r->engine.reset(new Engine(ctx, std::move(m.space), std::move(m.ham), input, o));
        *out = r.release();
        return DMRG_OK;
    } catch (const StatusError& e) {
        return set_error(e.status, "%s", e.what());
    } catch (const std::exception& e) {
        return set_error(DMRG_E_ARG, "%s", e.what());
    }
}

int dmrg_run_execute(dmrg_run_t r) {
    if (!r) return set_error(DMRG_E_ARG, "null run");
    try {
        DMRG_CUDA_TRY(cudaSetDevice(r->engine->device()));
        AllocScope pool(r->engine->stream());
        return r->engine->Run();
    } catch (const std::exception& e) {  // no exception crosses the C ABI
        return set_error(DMRG_E_STATE, "%s", e.what());
    }
}

int dmrg_run_execute_many(dmrg_run_t* runs, int n, int threads, int* status) {
    if (!runs || n < 0 || !status) return set_error(DMRG_E_ARG, "null argument");
    for (int i = 0; i < n; ++i)
        if (!runs[i]) return set_error(DMRG_E_ARG, "run %d is null", i);
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            if (runs[i]->engine->stream() == runs[j]->engine->stream())
                return set_error(DMRG_E_ARG, "runs %d and %d share a stream (give each its own context)", i, j);
    // side by side, a run's Lanczos calls go launch by launch unless it asked for graphs
    for (int i = 0; i < n; ++i)
        if (runs[i]->engine->lanczos_graph() < 0) runs[i]->engine->set_lanczos_graph(0);
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    threads = std::min(threads, n);
    std::atomic<int> next{0};
    std::vector<std::string> errors(n);
    auto worker = [&] {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) return;
            status[i] = dmrg_run_execute(runs[i]);
            if (status[i] != DMRG_OK) errors[i] = dmrg_last_error();
        }
    };
    std::vector<std::thread> pool;
    try {
        for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    } catch (const std::system_error&) {
        // fewer threads: the calling thread and those started take all runs
    }
    worker();
    for (auto& t : pool) t.join();
    for (int i = 0; i < n; ++i)
        if (status[i] != DMRG_OK) return set_error(status[i], "run %d: %s", i, errors[i].c_str());
    return DMRG_OK;
}

int dmrg_run_destroy(dmrg_run_t r) {
    delete r;
    return DMRG_OK;
}

int dmrg_run_half_sweeps(dmrg_run_t r, int cap, double* energies, double* seconds, int* count) {
    if (!r || !count) return set_error(DMRG_E_ARG, "null argument");
    const auto& e = r->engine->half_sweep_energies();
    const auto& s = r->engine->half_sweep_seconds();
    *count = (int)e.size();
    for (int i = 0; i < (int)e.size() && i < cap; ++i) {
        if (energies) energies[i] = e[i];
        if (seconds) seconds[i] = s[i];
    }
    return DMRG_OK;
}

int dmrg_run_steps(dmrg_run_t r, int cap, int* half_sweep, int* site, double* energy, int* lanczos_dim,
                   double* discarded, int64_t* psi_dim, double* seconds, int* count) {
    if (!r || !count) return set_error(DMRG_E_ARG, "null argument");
    const auto& rec = r->engine->records();
    *count = (int)rec.size();
    for (int i = 0; i < (int)rec.size() && i < cap; ++i) {
        if (half_sweep) half_sweep[i] = rec[i].half_sweep;
        if (site) site[i] = rec[i].site;
        if (energy) energy[i] = rec[i].energy;
        if (lanczos_dim) lanczos_dim[i] = rec[i].lanczos_dim;
        if (discarded) discarded[i] = rec[i].discarded;
        if (psi_dim) psi_dim[i] = rec[i].psi_dim;
        if (seconds) seconds[i] = rec[i].seconds;
    }
    return DMRG_OK;
}

int dmrg_run_phases(dmrg_run_t r, int cap, double* seconds, int* svd_sweeps, int* count) {
    if (!r || !count) return set_error(DMRG_E_ARG, "null argument");
    const auto& ph = r->engine->half_sweep_phases();
    const auto& sw = r->engine->half_sweep_svd_sweeps();
    *count = (int)ph.size();
    for (int i = 0; i < (int)ph.size() && i < cap; ++i) {
        if (seconds)
            for (int k = 0; k < Engine::kPhases; ++k) seconds[(size_t)i * Engine::kPhases + k] = ph[i][k];
        if (svd_sweeps) svd_sweeps[i] = sw[i];
    }
    return DMRG_OK;
}

int dmrg_run_options_from_input(const char* input_path, dmrg_run_options_t* opt) {
    if (!input_path || !opt) return set_error(DMRG_E_ARG, "null argument");
    try {
        InputGroup input(input_path, "input", false);
        dmrg_run_options_t o{};
        o.precision = DMRG_PREC_FP64;
        o.verbose = 1;
        o.seed = 1;
        o.stop_after_half_sweeps = -1;
        o.lanczos_precision = 0.0;
        o.two_site = 0;
        o.lanczos_graph = 0;
        const std::string prec = input.getString("precision", "");
        if (prec == "tf32x3") o.precision = DMRG_PREC_TF32X3;
        else if (prec == "bf16x3") o.precision = DMRG_PREC_BF16X3;
        else if (!prec.empty() && prec != "fp64")
            throw std::runtime_error("precision = " + prec + ": fp64, tf32x3 or bf16x3");
        const std::string mode = input.getString("mode", "");
        if (mode == "twosite") o.two_site = 1;
        else if (!mode.empty() && mode != "onesite") throw std::runtime_error("mode = " + mode + ": onesite or twosite");
        const int seed = input.getInt("seed", 1);
        if (seed < 0) throw std::runtime_error("seed = " + std::to_string(seed) + ": must be >= 0");
        o.seed = (unsigned)seed;
        const double tol = input.getDouble("lanczos_tol", 0.0);
        if (!(tol >= 0.0) || !std::isfinite(tol)) throw std::runtime_error("lanczos_tol must be >= 0");
        o.lanczos_precision = tol;
        const int graph = input.getInt("lanczos_graph", 0);
        if (graph < -1 || graph > 1) throw std::runtime_error("lanczos_graph must be -1, 0 or 1");
        o.lanczos_graph = graph;
        *opt = o;
        return DMRG_OK;
    } catch (const std::exception& e) {
        return set_error(DMRG_E_ARG, "%s", e.what());
    }
}

int dmrg_model_create(const char* input_path, const char* model, dmrg_model_t* out) {
    if (!input_path || !out) return set_error(DMRG_E_ARG, "null argument");
    *out = nullptr;
    try {
        InputGroup input(input_path, "input", false);
        auto* m = new dmrg_model_s();
        m->spec = make_model(input, model ? model : "real_spinless_bose_square");
        m->spec.ham->DefineTensorHamiltonian();
        *out = m;
        return DMRG_OK;
    } catch (const std::exception& e) {
        return set_error(DMRG_E_ARG, "%s", e.what());
    }
}

int dmrg_model_destroy(dmrg_model_t m) {
    delete m;
    return DMRG_OK;
}

int dmrg_model_info(dmrg_model_t m, int* num_site, int* physics_dim, int* num_quantum) {
    if (!m) return set_error(DMRG_E_ARG, "null model");
    if (num_site) *num_site = m->spec.space->num_site();
    if (physics_dim) *physics_dim = m->spec.space->physics_dim();
    if (num_quantum) *num_quantum = m->spec.space->num_quantum();
    return DMRG_OK;
}

int dmrg_model_mpo(dmrg_model_t m, int site, int* left_bond, int* right_bond, int cap, double* W) {
    if (!m || !left_bond || !right_bond) return set_error(DMRG_E_ARG, "null argument");
    const MpoHamiltonian& h = *m->spec.ham;
    if (site < 0 || site >= h.num_site()) return set_error(DMRG_E_ARG, "site out of range");
    *left_bond = h.left_bond(site);
    *right_bond = h.right_bond(site);
    const int d = h.physics_dim(site);
    const int64_t n = (int64_t)*left_bond * *right_bond * d * d * (h.is_complex() ? 2 : 1);
    const double* v = h.values(site);
    if (W)
        for (int64_t i = 0; i < n && i < cap; ++i) W[i] = v[i];
    return DMRG_OK;
}

int dmrg_model_is_complex(dmrg_model_t m, int* is_complex) {
    if (!m || !is_complex) return set_error(DMRG_E_ARG, "null argument");
    *is_complex = m->spec.ham->is_complex() ? 1 : 0;
    return DMRG_OK;
}

int dmrg_model_quantum_table(dmrg_model_t m, int which, int bond, int cap, int* values, int* rows) {
    if (!m || !rows) return set_error(DMRG_E_ARG, "null argument");
    if (which != 0 && which != 1) return set_error(DMRG_E_ARG, "which must be 0 (MPS bonds) or 1 (MPO bonds)");
    if (bond < 0 || bond > m->spec.space->num_site()) return set_error(DMRG_E_ARG, "bond out of range");
    const auto& t = which == 0 ? m->spec.space->table(bond) : m->spec.ham->quantum_table(bond);
    *rows = (int)t.size();
    int k = 0;
    for (const auto& row : t)
        for (int q : row) {
            if (values && k < cap) values[k] = q;
            ++k;
        }
    return DMRG_OK;
}

}  // extern "C"
