// Test infrastructure / CPU baseline: times the reference's own
// RealTensorContraction::MultiplyEffectHamilton (src/dmrg/realdmrg/
// real_tensor_contraction.cc:1223-1291, dgemm through OpenBLAS) on one H_eff
// problem read from a .nac file.
//
// Usage: probe_heff <problem.nac> <reps> [seed] [out.nac]
//   Values: the file's own (lattice.ket.data, L.<o>.data, R.<o>.data) when
//   present, else the splitmix64 stream of `seed`: psi takes elements
//   [0, psi_dim), L the next |L| (bond-major, block order), R the next |R|.
//   PROBE_WARMUP=n runs n untimed calls first.
//   Prints one line: seconds per call (best and mean), algorithmic GFLOP per call
//   counted over the reference loop, psi_dim.  With out.nac, writes the result of
//   one call on a zero state as "heff_out".
#include "probe_common.h"

using probe::NacArray;

static const std::vector<int>& I(std::map<std::string, NacArray>& d, const std::string& k) {
    auto it = d.find(k);
    if (it == d.end()) {
        std::fprintf(stderr, "missing array %s\n", k.c_str());
        std::exit(2);
    }
    return it->second.i;
}

static RealMatrixBlock* make_blocks(std::map<std::string, NacArray>& d, const std::string& p, probe::SplitMix* rng,
                                    size_t* consumed) {
    const auto& l = I(d, p + ".left");
    const auto& r = I(d, p + ".right");
    const auto& rows = I(d, p + ".rows");
    const auto& cols = I(d, p + ".cols");
    int n = (int)l.size();
    std::vector<int> li(l), ri(r);
    RealMatrixBlock* b = new RealMatrixBlock(n, li.data(), ri.data());
    const std::vector<double>* data = nullptr;
    auto it = d.find(p + ".data");
    if (it != d.end()) data = &it->second.d;
    size_t pos = 0;
    for (int k = 0; k < n; ++k) {
        RealMatrix m(rows[k], cols[k]);
        for (int e = 0; e < rows[k] * cols[k]; ++e) {
            double v = data ? (*data)[pos + e] : rng->next();
            m.get_matrix_element()[e] = v;
        }
        pos += (size_t)rows[k] * cols[k];
        delete b->matrix_block_[k];
        b->matrix_block_[k] = new RealMatrix(&m);
    }
    *consumed += pos;
    return b;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s problem.nac reps [seed] [out.nac]\n", argv[0]);
        return 1;
    }
    auto d = probe::nac_read(argv[1]);
    int reps = std::atoi(argv[2]);
    uint64_t seed = argc > 3 ? std::strtoull(argv[3], nullptr, 10) : 1234;
    probe::SplitMix rng(seed);
    size_t consumed = 0;

    const auto& ldim = I(d, "lattice.left_dim");
    const auto& rdim = I(d, "lattice.right_dim");
    const auto& phys = I(d, "lattice.physics_index");
    const auto& dims = I(d, "op.dims");
    int pd = dims[0], lb = dims[1], rb = dims[2];
    int nl = (int)ldim.size(), nr = (int)rdim.size();

    RealTensorLattice* lat = new RealTensorLattice(pd);
    std::vector<int> lblk(nl), rblk(nr), ld(ldim), rd(rdim);
    for (int i = 0; i < nl; ++i) lblk[i] = i;
    for (int i = 0; i < nr; ++i) rblk[i] = i;
    lat->DefineTensorLattice(nl, nr, lblk.data(), rblk.data(), ld.data(), rd.data());
    for (int i = 0; i < nl; ++i)
        for (int j = 0; j < nr; ++j) lat->physics_index_[i][j] = phys[(size_t)i * nr + j];
    lat->ket_tensor_ = make_blocks(d, "lattice.ket", &rng, &consumed);

    RealTensorOperator* op = new RealTensorOperator(pd);
    op->left_bond_ = lb;
    op->right_bond_ = rb;
    op->DefineTensorOperator();
    const auto& W = d["op.W"].d;
    for (int a = 0; a < lb; ++a)
        for (int b = 0; b < rb; ++b)
            for (int p1 = 0; p1 < pd; ++p1)
                for (int p2 = 0; p2 < pd; ++p2)
                    op->tensor_operator_[a][b]->set_matrix_element(p1, p2, W[(((size_t)a * rb + b) * pd + p1) * pd + p2]);

    RealTensorContraction* con = new RealTensorContraction(lb, rb);
    for (int o = 0; o < lb; ++o) con->left_contraction_tensor_[o] = make_blocks(d, "L." + std::to_string(o), &rng, &consumed);
    for (int o = 0; o < rb; ++o) con->right_contraction_tensor_[o] = make_blocks(d, "R." + std::to_string(o), &rng, &consumed);

    // Algorithmic FLOPs over the reference loop (real_tensor_contraction.cc:1243-1285).
    double flops = 0.0;
    {
        RealMatrixBlock* ket = lat->ket_tensor_;
        for (int o2 = 0; o2 < rb; ++o2) {
            RealMatrixBlock* Ro = con->right_contraction_tensor_[o2];
            for (int i = 0; i < Ro->num_block_; ++i) {
                int ldx = Ro->left_index_[i], jdx = Ro->right_index_[i];
                RealMatrix* Rm = Ro->matrix_block_[i];
                if (Rm->row_ == 0) continue;
                for (int pos = 0; pos < ket->num_block_; ++pos) {
                    if (ket->right_index_[pos] != ldx) continue;
                    int kdx = ket->left_index_[pos];
                    int p2 = lat->physics_index_[kdx][ldx];
                    if (!op->RightCheckZero(o2, p2)) continue;
                    int ak = ket->matrix_block_[pos]->row_, bl = ket->matrix_block_[pos]->column_;
                    flops += 2.0 * ak * bl * Rm->column_;
                    for (int pos2 = 0; pos2 < ket->num_block_; ++pos2) {
                        if (ket->right_index_[pos2] != jdx) continue;
                        int idx = ket->left_index_[pos2];
                        int p1 = lat->physics_index_[idx][jdx];
                        for (int o1 = 0; o1 < lb; ++o1) {
                            if (op->tensor_operator_[o1][o2]->get_matrix_element(p1, p2) == 0.0) continue;
                            int q = con->left_contraction_tensor_[o1]->FindMatrixBlock(idx, kdx);
                            if (q == -1) continue;
                            flops += 2.0 * con->left_contraction_tensor_[o1]->matrix_block_[q]->row_ * ak * Rm->column_;
                        }
                    }
                }
            }
        }
    }

    int psi_dim = lat->ComputeKetTensorDim();
    std::vector<double> state(psi_dim, 0.0);
    const char* wu = std::getenv("PROBE_WARMUP");
    for (int r = 0, n = wu ? std::atoi(wu) : 0; r < n; ++r) con->MultiplyEffectHamilton(lat, op, state.data());
    double best = 1e30, total = 0.0;
    for (int r = 0; r < reps; ++r) {
        std::fill(state.begin(), state.end(), 0.0);
        double t0 = GetWallTime();
        con->MultiplyEffectHamilton(lat, op, state.data());
        double dt = GetWallTime() - t0;
        best = dt < best ? dt : best;
        total += dt;
    }
    std::printf("{\"best_s\": %.9f, \"mean_s\": %.9f, \"gflop\": %.9f, \"psi_dim\": %d, \"reps\": %d, "
                "\"threads\": %d}\n",
                best, total / (reps > 0 ? reps : 1), flops * 1e-9, psi_dim, reps, omp_get_max_threads());
    if (argc > 4) {
        std::fill(state.begin(), state.end(), 0.0);
        con->MultiplyEffectHamilton(lat, op, state.data());
        probe::NacWriter w(argv[4]);
        w.dbls("heff_out", state);
        w.scalar_d("gflop", flops * 1e-9);
    }
    return 0;
}
