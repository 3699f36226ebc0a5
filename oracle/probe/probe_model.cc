// Test infrastructure: dumps the MPO and the quantum-number tables of the
// reference's spinful model (ComplexSpinfulBoseSquareSpace /
// ComplexSpinfulBoseSquareHamiltonian, model/space/complex_spinful_bose_square_space.cc,
// model/hamiltonian/complex_spinful_bose_square_hamiltonian.cc), built from an
// input file exactly as model/complex_spinful_bose_square_model.cc:11-45 does
// and ComplexTensorRundmrg's constructor then defines it
// (src/dmrg/complexdmrg/complex_tensor_rundmrg.cc:53).
//
// With a third argument "spinless" it dumps the reference's complex spinless
// model instead (ComplexSpinlessBoseSquareSpace /
// ComplexSpinlessBoseSquareHamiltonian, built as
// model/complex_spinless_bose_square_model.cc:11-40 does).
//
// Usage: probe_model <input file> <out.nac> [spinless]
// Writes num_site; per site i "op<i>.dims" (d, left bond, right bond),
// "op<i>.W" (real parts) and "op<i>.Wi" (imaginary parts) in [l][r][p1][p2]
// order; per bond b "sq<b>" (space) and "hq<b>" (MPO) quantum tables, flattened.
#include "probe_common.h"

int main(int argc, char** argv) {
    if (argc != 3 && !(argc == 4 && std::strcmp(argv[3], "spinless") == 0)) {
        std::fprintf(stderr, "usage: %s inputfile out.nac [spinless]\n", argv[0]);
        return 1;
    }
    auto input = InputGroup(argv[1], "input");
    ComplexTensorSpace* space = nullptr;
    ComplexTensorHamiltonian* ham = nullptr;
    if (argc == 4) {
        int nx = input.getInt("num_site_x");
        int ny = input.getInt("num_site_y");
        int nb = input.getInt("num_boson");
        int d = input.getInt("physics_dim", 2);
        double flux_value = input.getDouble("flux") * PI;
        double jx = input.getDouble("Jx");
        double jy = input.getDouble("Jy");
        double u = input.getDouble("U");
        double mu = input.getDouble("mu");
        bool px = input.getBool("period_x");
        bool py = input.getBool("period_y");
        space = new ComplexSpinlessBoseSquareSpace(nx, ny, nb, d);
        ham = new ComplexSpinlessBoseSquareHamiltonian(nx, ny, d, flux_value, jx, jy, u, mu, px, py);
    } else {
        int nx = input.getInt("num_site_x");
        int ny = input.getInt("num_site_y");
        int d = input.getInt("physics_dim", 2);
        bool px = input.getBool("period_x");
        bool py = input.getBool("period_y");
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
        space = new ComplexSpinfulBoseSquareSpace(nx, ny, nb, d);
        ham = new ComplexSpinfulBoseSquareHamiltonian(nx, ny, d, flux, jx, jy, u, mu, px, py);
    }
    ham->DefineTensorHamiltonian();

    probe::NacWriter w(argv[2]);
    const int n = ham->num_site_;
    w.scalar_i("num_site", n);
    for (int i = 0; i < n; ++i) {
        ComplexTensorOperator* op = ham->tensor_hamiltonian_[i];
        const int lb = op->left_bond_, rb = op->right_bond_, pd = op->physics_dim_;
        w.ints("op" + std::to_string(i) + ".dims", {pd, lb, rb});
        std::vector<double> re, im;
        for (int a = 0; a < lb; ++a)
            for (int b = 0; b < rb; ++b)
                for (int p1 = 0; p1 < pd; ++p1)
                    for (int p2 = 0; p2 < pd; ++p2) {
                        Complex c = op->tensor_operator_[a][b]->get_matrix_element(p1, p2);
                        re.push_back(c.real_);
                        im.push_back(c.imag_);
                    }
        w.dbls("op" + std::to_string(i) + ".W", re);
        w.dbls("op" + std::to_string(i) + ".Wi", im);
    }
    for (int b = 0; b <= n; ++b) {
        std::vector<int> hq, sq;
        for (int j = 0; j < ham->num_table_[b]; ++j)
            for (int k = 0; k < ham->num_quantum_; ++k) hq.push_back(ham->quantum_table_[b][j][k]);
        for (int j = 0; j < space->num_table_[b]; ++j)
            for (int k = 0; k < space->num_quantum_; ++k) sq.push_back(space->quantum_table_[b][j][k]);
        w.ints("hq" + std::to_string(b), hq);
        w.ints("sq" + std::to_string(b), sq);
    }
    return 0;
}
