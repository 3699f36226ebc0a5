// Test infrastructure: instrumented run of the unmodified reference's complex
// DMRG (the spinful model executable, model/complex_spinful_bose_square_model.cc,
// whose y-bond Peierls phases make the Hamiltonian complex; with Ndown = 0 it is
// the Bose-Hubbard-Hofstadter model).  The linker's --wrap routes the complex
// hot-path members through the __wrap_* functions below, which serialise inputs
// and outputs at the requested call indices and call the real member:
//   ComplexTensorLanczos::LanczosMethod              complex_tensor_lanczos.cc:14
//   ComplexTensorContraction::Left/RightCompute...   complex_tensor_contraction.cc:800,977
//   ComplexTensorLattice::Left/RightCanonical...     complex_tensor_lattice.cc (zgesdd)
// Complex arrays are written as interleaved (re, im) doubles.
//
// Usage: probe_zdump <input file>
//   PROBE_OUT=dir, PROBE_HEFF=i,..., PROBE_ENV=i,..., PROBE_CANON=i,..., PROBE_STOP=n
//   as probe_dump.
// Always writes PROBE_OUT/steps.txt (call, site, niter, psi_dim, energy, seconds).
#include "probe_common.h"

using probe::NacWriter;

static std::string g_out = ".";
static std::vector<int> g_heff, g_env, g_canon;
static int g_stop = -1;
static FILE* g_steps = nullptr;
static int n_lanczos = 0, n_env = 0, n_canon = 0;

static std::vector<int> parse_list(const char* s) {
    std::vector<int> v;
    if (!s) return v;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ',')) if (!tok.empty()) v.push_back(std::atoi(tok.c_str()));
    return v;
}
static bool wanted(const std::vector<int>& v, int i) {
    for (int x : v) if (x == i || x == -1) return true;
    return false;
}

static void zwrite_block(NacWriter& w, const std::string& p, ComplexMatrixBlock* b) {
    std::vector<int> li, ri, rows, cols;
    std::vector<double> data;
    const int nb = b ? b->num_block_ : 0;
    for (int k = 0; k < nb; ++k) {
        ComplexMatrix* m = b->matrix_block_[k];
        li.push_back(b->left_index_[k]);
        ri.push_back(b->right_index_[k]);
        rows.push_back(m->row_);
        cols.push_back(m->column_);
        for (int e = 0; e < m->total_element_num_; ++e) {
            data.push_back(m->matrix_element_[e].real_);
            data.push_back(m->matrix_element_[e].imag_);
        }
    }
    w.ints(p + ".left", li);
    w.ints(p + ".right", ri);
    w.ints(p + ".rows", rows);
    w.ints(p + ".cols", cols);
    w.dbls(p + ".data", data);
}

static void zwrite_lattice(NacWriter& w, const std::string& p, ComplexTensorLattice* t) {
    w.scalar_i(p + ".physics_dim", t->physics_dim_);
    w.ints(p + ".left_dim", std::vector<int>(t->left_dim_, t->left_dim_ + t->num_left_block_));
    w.ints(p + ".right_dim", std::vector<int>(t->right_dim_, t->right_dim_ + t->num_right_block_));
    std::vector<int> phys;
    for (int i = 0; i < t->num_left_block_; ++i)
        for (int j = 0; j < t->num_right_block_; ++j) phys.push_back(t->physics_index_[i][j]);
    w.ints(p + ".physics_index", phys);
    zwrite_block(w, p + ".ket", t->ket_tensor_);
}

static void zwrite_operator(NacWriter& w, const std::string& p, ComplexTensorOperator* op) {
    const int d = op->physics_dim_, lb = op->left_bond_, rb = op->right_bond_;
    w.ints(p + ".dims", {d, lb, rb});
    std::vector<double> v;
    for (int a = 0; a < lb; ++a)
        for (int b = 0; b < rb; ++b)
            for (int p1 = 0; p1 < d; ++p1)
                for (int p2 = 0; p2 < d; ++p2) {
                    Complex c = op->tensor_operator_[a][b]->get_matrix_element(p1, p2);
                    v.push_back(c.real_);
                    v.push_back(c.imag_);
                }
    w.dbls(p + ".W", v);
}

static void zwrite_env(NacWriter& w, const std::string& p, ComplexMatrixBlock** env, int bond) {
    w.scalar_i(p + ".bond", bond);
    for (int o = 0; o < bond; ++o) zwrite_block(w, p + "." + std::to_string(o), env[o]);
}

extern "C" {
void __real__ZN20ComplexTensorLanczos13LanczosMethodEiiRd(ComplexTensorLanczos*, int, int, double&);
void __real__ZN24ComplexTensorContraction28LeftComputeTensorContractionEP20ComplexTensorLatticeP21ComplexTensorOperatorPS_(
    ComplexTensorContraction*, ComplexTensorLattice*, ComplexTensorOperator*, ComplexTensorContraction*);
void __real__ZN24ComplexTensorContraction29RightComputeTensorContractionEP20ComplexTensorLatticeP21ComplexTensorOperatorPS_(
    ComplexTensorContraction*, ComplexTensorLattice*, ComplexTensorOperator*, ComplexTensorContraction*);

void __wrap__ZN20ComplexTensorLanczos13LanczosMethodEiiRd(ComplexTensorLanczos* self, int niter, int site,
                                                          double& result) {
    const int call = n_lanczos++;
    ComplexTensorLattice* lat = self->space_->get_tensor_lattice(site);
    ComplexTensorOperator* op = self->hamiltonian_->get_tensor_hamiltonian(site);
    ComplexTensorContraction* con = self->network_->get_tensor_contraction(site);
    const int psi_dim = lat->ComputeKetTensorDim();
    if (wanted(g_heff, call)) {
        NacWriter w(g_out + "/zheff_" + std::to_string(call) + ".nac");
        w.scalar_i("site", site);
        w.scalar_i("niter", niter);
        zwrite_lattice(w, "lattice", lat);
        zwrite_operator(w, "op", op);
        zwrite_env(w, "L", con->left_contraction_tensor_, op->left_bond_);
        zwrite_env(w, "R", con->right_contraction_tensor_, op->right_bond_);
        std::vector<Complex> out(psi_dim, Complex(0.0, 0.0));
        con->MultiplyEffectHamilton(lat, op, out.data());
        std::vector<double> flat;
        for (const Complex& c : out) {
            flat.push_back(c.real_);
            flat.push_back(c.imag_);
        }
        w.dbls("heff_out", flat);
    }
    const double t0 = GetWallTime();
    __real__ZN20ComplexTensorLanczos13LanczosMethodEiiRd(self, niter, site, result);
    const double t1 = GetWallTime();
    if (wanted(g_heff, call)) {
        NacWriter w(g_out + "/zlanczos_" + std::to_string(call) + ".nac");
        w.scalar_d("energy", result);
        zwrite_lattice(w, "lattice", lat);
    }
    std::fprintf(g_steps, "%d %d %d %d %.15e %.6f\n", call, site, niter, psi_dim, result, t1 - t0);
    std::fflush(g_steps);
    if (call == g_stop) std::exit(0);
}

static void zenv_common(bool left, ComplexTensorContraction* self, ComplexTensorLattice* lat,
                        ComplexTensorOperator* op, ComplexTensorContraction* next) {
    const int call = n_env++;
    NacWriter* w = wanted(g_env, call) ? new NacWriter(g_out + "/zenv_" + std::to_string(call) + ".nac") : nullptr;
    if (w) {
        w->scalar_i("left", left ? 1 : 0);
        zwrite_lattice(*w, "lattice", lat);
        zwrite_operator(*w, "op", op);
        if (left) zwrite_env(*w, "env_in", self->left_contraction_tensor_, op->left_bond_);
        else zwrite_env(*w, "env_in", self->right_contraction_tensor_, op->right_bond_);
    }
    if (left)
        __real__ZN24ComplexTensorContraction28LeftComputeTensorContractionEP20ComplexTensorLatticeP21ComplexTensorOperatorPS_(
            self, lat, op, next);
    else
        __real__ZN24ComplexTensorContraction29RightComputeTensorContractionEP20ComplexTensorLatticeP21ComplexTensorOperatorPS_(
            self, lat, op, next);
    if (w) {
        if (left) zwrite_env(*w, "env_out", next->left_contraction_tensor_, op->right_bond_);
        else zwrite_env(*w, "env_out", next->right_contraction_tensor_, op->left_bond_);
        delete w;
    }
}
void __wrap__ZN24ComplexTensorContraction28LeftComputeTensorContractionEP20ComplexTensorLatticeP21ComplexTensorOperatorPS_(
    ComplexTensorContraction* self, ComplexTensorLattice* lat, ComplexTensorOperator* op,
    ComplexTensorContraction* next) {
    zenv_common(true, self, lat, op, next);
}
void __wrap__ZN24ComplexTensorContraction29RightComputeTensorContractionEP20ComplexTensorLatticeP21ComplexTensorOperatorPS_(
    ComplexTensorContraction* self, ComplexTensorLattice* lat, ComplexTensorOperator* op,
    ComplexTensorContraction* next) {
    zenv_common(false, self, lat, op, next);
}

void __real__ZN20ComplexTensorLattice26LeftCanonicalTensorLatticeEid(ComplexTensorLattice*, int, double);
void __real__ZN20ComplexTensorLattice27RightCanonicalTensorLatticeEid(ComplexTensorLattice*, int, double);

static void zcanon_common(bool left, ComplexTensorLattice* self, int max_dim, double canpre) {
    const int call = n_canon++;
    NacWriter* w = wanted(g_canon, call) ? new NacWriter(g_out + "/zcanon_" + std::to_string(call) + ".nac") : nullptr;
    if (w) {
        w->scalar_i("left", left ? 1 : 0);
        w->scalar_i("max_dim", max_dim);
        w->scalar_d("canpre", canpre);
        zwrite_lattice(*w, "before", self);
    }
    if (left) __real__ZN20ComplexTensorLattice26LeftCanonicalTensorLatticeEid(self, max_dim, canpre);
    else __real__ZN20ComplexTensorLattice27RightCanonicalTensorLatticeEid(self, max_dim, canpre);
    if (w) {
        zwrite_lattice(*w, "after", self);
        if (self->canonical_tensor_) {
            zwrite_block(*w, "after.canonical", self->canonical_tensor_);
            const int n = self->canonical_tensor_->num_block_;
            w->ints("after.match_dim", std::vector<int>(self->match_dim_, self->match_dim_ + n));
        }
        delete w;
    }
}
void __wrap__ZN20ComplexTensorLattice26LeftCanonicalTensorLatticeEid(ComplexTensorLattice* self, int m, double c) {
    zcanon_common(true, self, m, c);
}
void __wrap__ZN20ComplexTensorLattice27RightCanonicalTensorLatticeEid(ComplexTensorLattice* self, int m, double c) {
    zcanon_common(false, self, m, c);
}
}  // extern "C"

int main(int argc, char* argv[]) {
    if (argc != 2) {
        std::printf("Usage: %s inputfile\n", argv[0]);
        return 1;
    }
    if (const char* o = std::getenv("PROBE_OUT")) g_out = o;
    g_heff = parse_list(std::getenv("PROBE_HEFF"));
    g_env = parse_list(std::getenv("PROBE_ENV"));
    g_canon = parse_list(std::getenv("PROBE_CANON"));
    if (const char* s = std::getenv("PROBE_STOP")) g_stop = std::atoi(s);
    g_steps = std::fopen((g_out + "/steps.txt").c_str(), "w");
    // model/complex_spinful_bose_square_model.cc:11-45
    auto input = InputGroup(argv[1], "input");
    const int nx = input.getInt("num_site_x");
    const int ny = input.getInt("num_site_y");
    const int d = input.getInt("physics_dim", 2);
    const bool px = input.getBool("period_x");
    const bool py = input.getBool("period_y");
    int nb[2] = {input.getInt("Nup"), input.getInt("Ndown")};
    double flux[2], jx[2], jy[2], mu[2], u[3];
    for (int t = 0; t < 2; ++t) {
        flux[t] = input.getDouble("flux");
        jx[t] = input.getDouble("Jx");
        jy[t] = input.getDouble("Jy");
        mu[t] = input.getDouble("mu");
    }
    u[0] = input.getDouble("U_uu");
    u[1] = input.getDouble("U_dd");
    u[2] = input.getDouble("U_ud");
    auto* space = new ComplexSpinfulBoseSquareSpace(nx, ny, nb, d);
    auto* ham = new ComplexSpinfulBoseSquareHamiltonian(nx, ny, d, flux, jx, jy, u, mu, px, py);
    auto* run = new ComplexTensorRundmrg(space, ham, input);
    run->Run();
    std::fclose(g_steps);
    return 0;
}
