// The DMRG sweep engine: the reference's lattice / space / contraction /
// network / Lanczos / sweep-driver classes (src/dmrg/realdmrg/*) with every
// tensor resident on the device.  Host code keeps the sector bookkeeping (block
// maps, truncation, the glibc rand() stream of the initial MPS and of the
// subspace expansion) identical to the reference; all arithmetic runs in
// libdmrg_b200's kernels.
#pragma once

#include <array>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "blockops.cuh"
#include "blocksparse.h"
#include "common.cuh"
#include "host/grand.h"
#include "host/input.h"
#include "host/model.h"
#include "vec.cuh"

namespace dmrg {

// A failure raised while building a run, carrying the DMRG_E_* status that the
// C-ABI returns for it (an unreadable checkpoint file is DMRG_E_IO).
struct StatusError : std::runtime_error {
    int status;
    StatusError(int st, const std::string& what) : std::runtime_error(what), status(st) {}
};

// RealMatrixBlock (ComplexMatrixBlock) with its values on the device (packed,
// list order; a complex value is two doubles, offsets count elements).
struct DevBlocks {
    BlockListDesc d;
    DeviceBuffer buf;
    double* ptr() const { return buf.as<double>(); }
    int alloc(cudaStream_t st, bool zero, int ew = 1);  // ew: doubles per element
    void set_shape_zero() {  // ResetMatrixBlock: every block 0 x 0
        for (int k = 0; k < d.count(); ++k) d.rows[k] = d.cols[k] = 0;
        d.size = 0;
        for (int k = 0; k < d.count(); ++k) d.off[k] = 0;
    }
};

// RealTensorLattice (real_tensor_lattice.h:10-42).
struct TensorLattice {
    int physics_dim = 0;
    std::vector<int> left_block, left_dim, right_block, right_dim;
    std::vector<int> phys;  // [num_left x num_right], -1: no block
    DevBlocks ket;
    bool has_canonical = false;
    DevBlocks canonical;
    std::vector<int> match_dim;
    int nl() const { return (int)left_block.size(); }
    int nr() const { return (int)right_block.size(); }
    int p(int l, int r) const { return phys[(size_t)l * nr() + r]; }
    int64_t psi_dim() const { return ket.d.size; }
};

// One environment (all MPO bond indices of one side), packed index-major.
struct EnvData {
    EnvDesc desc;
    DeviceBuffer buf;
    double* ptr() const { return buf.as<double>(); }
};

// RealTensorContraction (real_tensor_contraction.h:8-16): left/right environments.
struct TensorContraction {
    int left_bond = 0, right_bond = 0;
    EnvData L, R;
};

struct SweepRecord {  // one site step
    int half_sweep, site, direction;  // direction 0: left->right
    double energy;
    int lanczos_dim;
    double discarded;
    int64_t psi_dim;
    double seconds;
};

struct RunOptions {
    int precision = DMRG_PREC_FP64;
    int verbose = 1;
    double lanczos_precision = 1e-15;  // hard-coded in the reference (real_tensor_lanczos.cc:29-30)
    double zero_tolerance = 1e-15;
    unsigned seed = 1;                  // glibc rand() seed; 1 = the reference's implicit seed
    int stop_after_half_sweeps = -1;    // run only this many half-sweeps (-1: all)
    int two_site = 0;                   // 1: two-site sweeps (RunTwoSite) instead of the reference's single-site ones
    // Lanczos loop as one CUDA-graph launch per call (dmrg_heff_set_graph): 1 on,
    // 0 off, -1 the operator's default.  Runs executed side by side turn it off:
    // every site step captures and instantiates a new graph, and those host calls
    // serialise across threads on one device.
    int lanczos_graph = -1;
};

class Engine {
public:
    // A complex Hamiltonian (ham->is_complex()) runs the complexdmrg twin of
    // every step (ComplexTensorRundmrg, src/dmrg/complexdmrg/*): complex site
    // tensors and environments, complex kernels.
    Engine(dmrg_ctx_t ctx, std::unique_ptr<QuantumSpace> space, std::unique_ptr<MpoHamiltonian> ham,
           InputGroup& input, const RunOptions& opt);
    ~Engine();
    // RealTensorRundmrg::Run (real_tensor_rundmrg.cc:115-245), or RunTwoSite
    // when the options ask for two-site sweeps.
    int Run();
    // Two-site sweeps over the same sweep table (host/twosite.cc); no reference
    // counterpart.
    int RunTwoSite();
    const std::vector<SweepRecord>& records() const { return records_; }
    double last_energy() const { return energy_; }
    const std::vector<double>& half_sweep_energies() const { return half_energies_; }
    const std::vector<double>& half_sweep_seconds() const { return half_seconds_; }
    // Per half-sweep: seconds in each phase (kPhases order) and Jacobi SVD sweeps.
    static constexpr int kPhases = 5;  // Lanczos, expansion, canonicalisation, environment, match + merge
    const std::vector<std::array<double, kPhases>>& half_sweep_phases() const { return half_phases_; }
    const std::vector<int>& half_sweep_svd_sweeps() const { return half_svd_sweeps_; }
    TensorLattice& lattice(int i) { return *lat_[i]; }
    TensorContraction& contraction(int i) { return *con_[i]; }
    int num_site() const { return n_; }
    bool is_complex() const { return cplx_; }
    void set_lanczos_graph(int enable) { opt_.lanczos_graph = enable; }
    int lanczos_graph() const { return opt_.lanczos_graph; }
    cudaStream_t stream() const { return st_; }
    int device() const { return ctx_->device; }

    // building blocks (public for the C ABI and tests)
    int Initialize();
    int DefineTensorSpace(int initial_block, int initial_dim);
    int CanonicalTensorSpace(int leigh, int site, double* discarded = nullptr);
    int MergeTensorSpace(int leigh, int site);
    int ExpanTensorSpace(int leigh, int site);
    int MatchTensorSpace(int leigh, int site);
    // ExpanTensorNetwork = PlanExpanTensorNetwork (host only: the expanded
    // lattice, the products to form and their rand() matrices; no CUDA call)
    // followed by ExecuteExpanTensorNetwork (the device products).
    int ExpanTensorNetwork(int leigh, int site);
    int PlanExpanTensorNetwork(int leigh, int site);
    int ExecuteExpanTensorNetwork();
    int ComputeTensorNetwork(int leigh, int site);
    int LanczosMethod(int niter, int site, double& energy, int& dim);
    // One two-site step at bond (j, j+1): merge, Lanczos, split, environment;
    // adds its phase times to `ph` (0 Lanczos, 2 split, 3 environment, 4 merge).
    int TwoSiteStep(bool l2r, int j, int niter, double& energy, int& dim, double& discarded, int64_t& theta_dim,
                    std::array<double, kPhases>& ph);
    // RealTensorSpace::WriteTensorSpace / ReadTensorSpace (real_tensor_space.cc:
    // 182-277): the MPS in the reference's binary checkpoint format.
    int WriteTensorSpace(const std::string& path);
    int ReadTensorSpace(const std::string& path);

private:
    // bookkeeping (host)
    void ComputeLatticeBlock(int site, std::vector<int>& left_block, std::vector<int>& right_block);
    void ComputeTensorIndex(int site, std::vector<int>& li, std::vector<int>& ri, std::vector<int>& pi);
    void DefineLatticeSectors(TensorLattice& t, const std::vector<int>& lb, const std::vector<int>& rb,
                              const std::vector<int>& ld, const std::vector<int>& rd);
    int DefineLatticeBlocks(TensorLattice& t, const std::vector<int>& li, const std::vector<int>& ri,
                            const std::vector<int>& pi, int row, int column, bool device = true);
    void ComputeExpanTensorLattice(int leigh, int site, std::vector<std::vector<int>>& mapping);
    int LeftExpanTensorContraction(int site, const std::vector<std::vector<int>>& mapping);
    int RightExpanTensorContraction(int site, const std::vector<std::vector<int>>& mapping);
    int ExpanLattice(int leigh, TensorLattice& t, const TensorLattice& origin, const TensorLattice* expan);
    int64_t add_random(int d0, int d1, double wre, double wim);
    int Normalize(TensorLattice& t);
    void Trace(const char* tag, int leigh, int site);
    void DefineTensorNetwork();
    int ResetEnv(int leigh, int site);

    dmrg_ctx_t ctx_;
    cudaStream_t st_;
    RunOptions opt_;
    std::unique_ptr<QuantumSpace> space_;
    std::unique_ptr<MpoHamiltonian> ham_;
    bool cplx_ = false;  // complex run
    int ew_ = 1;         // doubles per tensor element (2 when complex)
    int n_ = 0;
    std::vector<std::unique_ptr<TensorLattice>> lat_;
    std::vector<std::unique_ptr<TensorContraction>> con_;
    std::unique_ptr<TensorLattice> expan_;
    // the planned half of the current subspace expansion
    struct ExpanWork {
        struct First {  // one (m x k) * (k x n) product: L*K (left) or K*R (right)
            int64_t a_off, b_off;
            int m, k, n;
            int64_t off;
        };
        struct Contrib {  // one random matrix (d0 x d1) applied to product `first`
            int first;
            int d0, d1;
            int64_t rnd;
        };
        bool active = false, compute = false;
        int leigh = 0, site = 0;
        std::vector<First> firsts;
        std::vector<std::vector<Contrib>> contrib;  // per block of the expanded lattice
        std::vector<double> rnd;
        int64_t first_size = 0;
        BlockListDesc packed;
    };
    ExpanWork xw_;
    // sweep table (real_tensor_rundmrg.cc:70-113)
    int num_sweep_ = 0;
    std::vector<int> max_dim_, max_block_, num_iter_;
    std::vector<double> canpre_, noise_;
    int first_block_ = 0, first_dim_ = 0;
    // checkpoints (cache_record / cache_resume, real_tensor_rundmrg.cc:16-23,44-51,229-233)
    bool cache_record_ = false, cache_resume_ = false;
    std::string cache_name_ = ".", record_name_ = "record.dat", resume_name_;
    // current parameters (RealTensorSpace::DefineTensorSpaceParameter)
    int p_max_block_ = 0, p_max_dim_ = -1;
    double p_canpre_ = 1e-30, p_noise_ = 10.0;
    // scratch
    DeviceBuffer copy_tasks_, scratch_, scratch2_, norm_;
    ReduceScratch rs_;
    std::vector<SweepRecord> records_;
    std::vector<double> half_energies_, half_seconds_;
    std::vector<std::array<double, kPhases>> half_phases_;
    std::vector<int> half_svd_sweeps_;
    int svd_sweeps_ = 0;  // Jacobi sweeps of the canonicalisations of the current half-sweep
    double energy_ = 0.0;
    int half_sweep_ = 0;
    int lanczos_calls_ = 0;
    FILE* trace_ = nullptr;  // DMRG_TRACE=<file>: structure trace, one line per step operation
    GlibcRand rng_;          // the reference's rand() stream (seeded with opt.seed)
    long long rand_draws_ = 0;
};

}  // namespace dmrg
