// Test program for the C++ classes of include/dmrg_b200.hpp.
//
//   layer_host <quicksort_cases.txt> <truncate_cases.txt> <input file> <model> [--device]
//
// Host part (no GPU): the reference's QuickSort on every golden case, the
// truncation dimensions of every case in the truncation file, and the model
// layer (MPO of every site, quantum tables) of an input file, printed for the
// Python test to compare with the C ABI's results and the golden orders.
// Without a GPU it also prints the status that constructing a Context gives.
// --device instead builds every device-side class on a tiny one-site problem
// (one 1x1 block, identity environments, W = [[2]]): H_eff psi, the Lanczos
// energy, both environment updates, both canonicalisations and a whole run of
// the input file; it prints their results.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "dmrg_b200.hpp"

using namespace dmrgcc_b200;

static void quicksort_cases(const char* path) {
    std::ifstream f(path);
    std::string in, out;
    while (std::getline(f, in) && std::getline(f, out)) {
        std::istringstream s(in);
        int n = 0, flag = 0;
        s >> n >> flag;
        std::vector<double> v(n);
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i) {
            s >> v[i];
            idx[i] = i;
        }
        QuickSort(v.data(), idx.data(), 0, n - 1, flag);
        std::printf("quicksort");
        for (int i : idx) std::printf(" %d", i);
        std::printf("\n");
    }
}

// QuickSort's edge cases: a flag other than 0 or 1 and an empty or one-element
// range leave both arrays as they are; a sub-range sorts only that range.
static void quicksort_edges() {
    double v[5] = {0.3, 0.9, 0.1, 0.9, 0.5};
    int idx[5] = {0, 1, 2, 3, 4};
    QuickSort(v, idx, 0, 4, 2);
    QuickSort(v, idx, 3, 3, 0);
    QuickSort(v, idx, 4, 3, 0);
    QuickSort(v, idx, 1, 3, 1);  // ascending on v[1..3]
    std::printf("quicksort_edges");
    for (int i = 0; i < 5; ++i) std::printf(" %d:%.17g", idx[i], v[i]);
    std::printf("\n");
}

// Each line: nsec max_dim canpre, then per sector its count and its values.
static void truncate_cases(const char* path) {
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream s(line);
        int nsec = 0, max_dim = 0;
        double canpre = 0;
        s >> nsec >> max_dim >> canpre;
        std::vector<std::vector<double>> sv(nsec);
        for (auto& v : sv) {
            int c = 0;
            s >> c;
            v.resize(c);
            for (double& x : v) s >> x;
        }
        const std::vector<int> t = RealTensorLattice::ComputeTruncateDim(max_dim, canpre, sv);
        std::printf("truncate");
        for (int x : t) std::printf(" %d", x);
        std::printf(" |");
        for (const auto& v : sv)
            for (double x : v) std::printf(" %.17g", x);
        std::printf("\n");
    }
}

static void model(const char* input, const char* name) {
    TensorModel m(input, name);
    std::printf("model %d %d %d %d\n", m.num_site(), m.physics_dim(), m.num_quantum(), m.is_complex() ? 1 : 0);
    for (int site = 0; site < m.num_site(); ++site) {
        int lb = 0, rb = 0;
        const std::vector<double> w = m.TensorOperator(site, lb, rb);
        std::printf("mpo %d %d %d", site, lb, rb);
        for (double x : w) std::printf(" %.17g", x);
        std::printf("\n");
    }
    for (int which = 0; which < 2; ++which)
        for (int bond = 0; bond <= m.num_site(); ++bond) {
            int rows = 0;
            const std::vector<int> q = m.QuantumTable(which, bond, rows);
            std::printf("quantum %d %d %d", which, bond, rows);
            for (int x : q) std::printf(" %d", x);
            std::printf("\n");
        }
}

// Every device-side class on a one-block problem: left and right sector 0 of
// dimension 1, physics index 0, d = 1, MPO bond 1 with W = [[2]], environments
// the 1x1 identity.  H_eff psi = 2 psi.
static int device_classes(const char* input, const char* name) {
    Context ctx(0);
    SiteTensor site;
    site.num_left_sector = site.num_right_sector = 1;
    site.physics_index = {0};
    site.ket.push_back(0, 0, 1, 1);
    site.physics_dim = site.left_bond = site.right_bond = 1;
    site.W = {2.0};
    BlockList env;
    env.push_back(0, 0, 1, 1);
    const double one = 1.0;
    RealTensorContraction h(ctx, site, {env}, {env});
    h.SetEnvironment(&one, &one);
    double psi = 0.5, state = 0.0;
    h.MultiplyEffectHamilton(&psi, &state);
    std::printf("heff %.17g %lld\n", state, (long long)h.PsiDim());
    RealTensorLanczos lz(h);
    double e = 0.0, v = 1.0;
    lz.LanczosMethod(10, &v, e);
    std::printf("lanczos %.17g %d\n", e, lz.KrylovDim());
    std::vector<double> out;
    const std::vector<BlockList> lb = RealTensorContraction::LeftComputeTensorContraction(ctx, site, {env}, &psi,
                                                                                          &one, out);
    std::printf("left_env %zu %.17g\n", lb.size(), out.empty() ? 0.0 : out[0]);
    const std::vector<BlockList> rb = RealTensorContraction::RightComputeTensorContraction(ctx, site, {env}, &psi,
                                                                                           &one, out);
    std::printf("right_env %zu %.17g\n", rb.size(), out.empty() ? 0.0 : out[0]);
    RealTensorLattice lat(ctx, {1}, {1}, site.ket);
    lat.LeftCanonicalTensorLattice(4, 1e-12, &psi);
    std::printf("left_canon %d %.17g %.17g\n", lat.TruncateDim()[0], lat.Ket()[0], lat.Canonical()[0]);
    lat.RightCanonicalTensorLattice(4, 1e-12, &psi);
    std::printf("right_canon %d %.17g %.17g\n", lat.TruncateDim()[0], lat.Ket()[0], lat.Canonical()[0]);
    dmrg_run_options_t opt = RealTensorRundmrg::DefaultOptions();
    opt.verbose = 0;
    RealTensorRundmrg run(ctx, input, name, opt);
    run.Run();
    const std::vector<double> es = run.HalfSweepEnergies();
    std::printf("run %zu %.17g\n", es.size(), es.empty() ? 0.0 : es.back());
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s quicksort_cases truncate_cases input model [--device]\n", argv[0]);
        return 2;
    }
    try {
        if (argc > 5 && std::strcmp(argv[5], "--device") == 0) return device_classes(argv[3], argv[4]);
        quicksort_cases(argv[1]);
        quicksort_edges();
        truncate_cases(argv[2]);
        model(argv[3], argv[4]);
        try {
            Context ctx(0);
            std::printf("context ok\n");
        } catch (const Error& e) {
            std::printf("context error %d\n", e.status());
        }
    } catch (const Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
