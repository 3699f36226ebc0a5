/*
 * dmrg_b200.hpp - C++ classes over the C ABI of libdmrg_b200 (dmrg_b200.h),
 * named after the reference's classes and members, for a dmrgcc maintainer who
 * replaces its MKL path class by class.
 *
 * Header only (C++17); link with -ldmrg_b200.  Each class owns its C handle and
 * the device storage it allocates (RAII, move-only).  Each member calls the C
 * entry point that stands in for the reference member it is named after (cited
 * per member).  Where the reference prints and calls exit(-1), these classes
 * throw dmrgcc_b200::Error, which carries the DMRG_E_* status and the
 * library's message.
 *
 * Storage is the reference's: a block list is RealMatrixBlock's ordered list of
 * row-major blocks packed back to back (VectorizeMatrixBlock order,
 * src/tensor/real_matrix_block.cc:173-194), an environment is one block list
 * per MPO bond index, packed index-major, and W is dense [left_bond][right_bond][d][d].
 * Values given as host pointers are copied; "Device" members take pointers to
 * the context's device memory.
 *
 * Members that only do host bookkeeping (QuickSort,
 * RealTensorLattice::ComputeTruncateDim, TensorModel) work without a GPU; every
 * other member needs the B200 and throws Error(DMRG_E_CUDA) without one.
 */
#ifndef DMRG_B200_HPP_
#define DMRG_B200_HPP_

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dmrg_b200.h"

namespace dmrgcc_b200 {

/* A failed call: status() is the DMRG_E_* code, what() names the call and gives
 * dmrg_last_error(). */
class Error : public std::runtime_error {
   public:
    Error(int status, const std::string& where)
        : std::runtime_error(where + ": " + dmrg_last_error()), status_(status) {}
    Error(int status, const std::string& where, const std::string& message)
        : std::runtime_error(where + ": " + message), status_(status) {}
    int status() const { return status_; }

   private:
    int status_;
};

inline void check(int rc, const char* where) {
    if (rc != DMRG_OK) throw Error(rc, where);
}

/* The shape of a RealMatrixBlock (src/tensor/real_matrix_block.h:6-40): block k
 * has the sector pair (left[k], right[k]) and is rows[k] x cols[k]. */
struct BlockList {
    std::vector<int> left, right, rows, cols;

    void push_back(int l, int r, int m, int n) {
        left.push_back(l);
        right.push_back(r);
        rows.push_back(m);
        cols.push_back(n);
    }
    int num_block() const { return (int)left.size(); }
    int64_t num_element() const {
        int64_t s = 0;
        for (size_t k = 0; k < rows.size(); ++k) s += (int64_t)rows[k] * cols[k];
        return s;
    }
    dmrg_blocks_t view() const { return {num_block(), left.data(), right.data(), rows.data(), cols.data()}; }
};

inline std::vector<dmrg_blocks_t> views(const std::vector<BlockList>& lists) {
    std::vector<dmrg_blocks_t> v;
    v.reserve(lists.size());
    for (const BlockList& b : lists) v.push_back(b.view());
    return v;
}

inline int64_t num_element(const std::vector<BlockList>& lists) {
    int64_t s = 0;
    for (const BlockList& b : lists) s += b.num_element();
    return s;
}

/* One GPU and the stream every call on it is ordered on (dmrg_ctx_*). */
class Context {
   public:
    explicit Context(int device = 0) { check(dmrg_ctx_create(device, &h_), "dmrg_ctx_create"); }
    ~Context() {
        if (h_) dmrg_ctx_destroy(h_);
    }
    Context(Context&& o) noexcept : h_(std::exchange(o.h_, nullptr)) {}
    Context& operator=(Context&& o) noexcept {
        std::swap(h_, o.h_);
        return *this;
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;

    dmrg_ctx_t get() const { return h_; }
    /* Orders the context's work on `stream` (a cudaStream_t; NULL = its own). */
    void SetStream(void* stream) { check(dmrg_ctx_set_stream(h_, stream), "dmrg_ctx_set_stream"); }
    /* Waits for the context's stream; reports a device-side failure. */
    void Synchronize() { check(dmrg_ctx_sync(h_), "dmrg_ctx_sync"); }

   private:
    dmrg_ctx_t h_ = nullptr;
};

/* n doubles of device memory owned by a context (dmrg_malloc / dmrg_free). */
class DeviceVector {
   public:
    DeviceVector() = default;
    DeviceVector(Context& ctx, size_t n) : ctx_(ctx.get()), n_(n) {
        if (n) {
            void* p = nullptr;
            check(dmrg_malloc(ctx_, n * sizeof(double), &p), "dmrg_malloc");
            p_ = static_cast<double*>(p);
        }
    }
    ~DeviceVector() {
        if (p_) dmrg_free(ctx_, p_);
    }
    DeviceVector(DeviceVector&& o) noexcept
        : ctx_(o.ctx_), p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
    DeviceVector& operator=(DeviceVector&& o) noexcept {
        std::swap(ctx_, o.ctx_);
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        return *this;
    }
    DeviceVector(const DeviceVector&) = delete;
    DeviceVector& operator=(const DeviceVector&) = delete;

    double* data() const { return p_; }
    size_t size() const { return n_; }
    /* Copies n_ doubles in or out; both wait for the copy. */
    void Upload(const double* host) {
        if (n_) check(dmrg_memcpy_h2d(ctx_, p_, host, n_ * sizeof(double)), "dmrg_memcpy_h2d");
    }
    void Download(double* host) const {
        if (n_) check(dmrg_memcpy_d2h(ctx_, host, p_, n_ * sizeof(double)), "dmrg_memcpy_d2h");
    }
    std::vector<double> Download() const {
        std::vector<double> v(n_);
        Download(v.data());
        return v;
    }

   private:
    dmrg_ctx_t ctx_ = nullptr;
    double* p_ = nullptr;
    size_t n_ = 0;
};

/* One site of the lattice as the contractions see it: the sector counts, the
 * physics index of each sector pair (num_left_sector * num_right_sector
 * entries, -1 = no block: RealTensorSpace's physics index), the site tensor's
 * block list and the MPO site tensor W[left_bond][right_bond][d][d]. */
struct SiteTensor {
    int num_left_sector = 0, num_right_sector = 0;
    std::vector<int> physics_index;
    BlockList ket;
    int physics_dim = 0, left_bond = 0, right_bond = 0;
    std::vector<double> W;
};

/* RealTensorContraction (src/dmrg/realdmrg/real_tensor_contraction.h:76-92): the
 * effective Hamiltonian of one site between its environments L[0..left_bond)
 * ((bra, ket) sector pairs) and R[0..right_bond) ((ket, bra) pairs), and the
 * environment updates that carry an environment to the next site. */
class RealTensorContraction {
   public:
    RealTensorContraction(Context& ctx, SiteTensor site, std::vector<BlockList> L, std::vector<BlockList> R,
                          int precision = DMRG_PREC_FP64)
        : ctx_(&ctx), site_(std::move(site)), L_(std::move(L)), R_(std::move(R)) {
        if ((int)L_.size() != site_.left_bond || (int)R_.size() != site_.right_bond)
            throw Error(DMRG_E_ARG, "RealTensorContraction", "one block list per MPO bond index");
        const dmrg_blocks_t kb = site_.ket.view();
        const std::vector<dmrg_blocks_t> lv = views(L_), rv = views(R_);
        check(dmrg_heff_create(ctx.get(), site_.num_left_sector, site_.num_right_sector, site_.physics_index.data(),
                               &kb, site_.physics_dim, site_.left_bond, site_.right_bond, site_.W.data(), lv.data(),
                               rv.data(), precision, &h_),
              "dmrg_heff_create");
        int64_t l = 0, r = 0;
        const int rc = dmrg_heff_sizes(h_, &psi_dim_, &l, &r);
        if (rc != DMRG_OK) {
            Error err(rc, "dmrg_heff_sizes");
            dmrg_heff_destroy(h_);
            throw err;
        }
    }
    ~RealTensorContraction() {
        if (h_) dmrg_heff_destroy(h_);
    }
    RealTensorContraction(const RealTensorContraction&) = delete;
    RealTensorContraction& operator=(const RealTensorContraction&) = delete;

    dmrg_heff_t get() const { return h_; }
    Context& context() const { return *ctx_; }
    const SiteTensor& site() const { return site_; }
    int64_t PsiDim() const { return psi_dim_; }
    /* FLOPs of one MultiplyEffectHamilton over the reference loop
     * (real_tensor_contraction.cc:1243-1285). */
    double Flops() const {
        double a = 0, e = 0;
        check(dmrg_heff_flops(h_, &a, &e), "dmrg_heff_flops");
        return a;
    }

    /* Environments from host values (packed L, packed R), kept on the device by
     * this object. */
    void SetEnvironment(const double* L_host, const double* R_host) {
        Lv_ = DeviceVector(*ctx_, (size_t)num_element(L_));
        Rv_ = DeviceVector(*ctx_, (size_t)num_element(R_));
        Lv_.Upload(L_host);
        Rv_.Upload(R_host);
        SetEnvironmentDevice(Lv_.data(), Rv_.data());
    }
    /* Environments already on the device; they must outlive their use here. */
    void SetEnvironmentDevice(const double* L_dev, const double* R_dev) {
        check(dmrg_heff_set_env(h_, L_dev, R_dev), "dmrg_heff_set_env");
    }

    /* MultiplyEffectHamilton(lattice, op, state) (real_tensor_contraction.h:91-92,
     * .cc:1223-1291): state += H_eff * ket, both PsiDim() doubles in host memory. */
    void MultiplyEffectHamilton(const double* ket, double* state) {
        check(dmrg_heff_apply_host(h_, ket, state, 1), "dmrg_heff_apply_host");
    }
    /* The same on device vectors (asynchronous); accumulate = false overwrites. */
    void MultiplyEffectHamiltonDevice(const double* ket_dev, double* state_dev, bool accumulate = true) {
        check(dmrg_heff_apply(h_, ket_dev, state_dev, accumulate ? 1 : 0), "dmrg_heff_apply");
    }

    /* LeftComputeTensorContraction(lattice, op, next) (real_tensor_contraction.h:76-77,
     * .cc:782-940): the left environment of the next site from this site's ket and
     * left environment L_in (one block list per left MPO bond index).  Host values
     * in and out; returns the new environment's block lists (one per right MPO
     * bond index) and fills `L_out` with its packed values. */
    static std::vector<BlockList> LeftComputeTensorContraction(Context& ctx, const SiteTensor& site,
                                                               const std::vector<BlockList>& L_in,
                                                               const double* ket, const double* L_in_values,
                                                               std::vector<double>& L_out,
                                                               int precision = DMRG_PREC_FP64) {
        return update(ctx, 0, site, L_in, ket, L_in_values, L_out, precision);
    }
    /* RightComputeTensorContraction (real_tensor_contraction.h:81-82, .cc:959-1119):
     * the right environment of the previous site from R_in (one block list per
     * right MPO bond index); returns one block list per left MPO bond index. */
    static std::vector<BlockList> RightComputeTensorContraction(Context& ctx, const SiteTensor& site,
                                                                const std::vector<BlockList>& R_in,
                                                                const double* ket, const double* R_in_values,
                                                                std::vector<double>& R_out,
                                                                int precision = DMRG_PREC_FP64) {
        return update(ctx, 1, site, R_in, ket, R_in_values, R_out, precision);
    }

   private:
    static std::vector<BlockList> update(Context& ctx, int side, const SiteTensor& site,
                                         const std::vector<BlockList>& in, const double* ket,
                                         const double* in_values, std::vector<double>& out_values, int precision) {
        const dmrg_blocks_t kb = site.ket.view();
        const std::vector<dmrg_blocks_t> iv = views(in);
        dmrg_env_t e = nullptr;
        check(dmrg_env_create(ctx.get(), side, site.num_left_sector, site.num_right_sector,
                              site.physics_index.data(), &kb, site.physics_dim, site.left_bond, site.right_bond,
                              site.W.data(), iv.data(), precision, &e),
              "dmrg_env_create");
        struct Guard {
            dmrg_env_t e;
            ~Guard() { dmrg_env_destroy(e); }
        } guard{e};
        int bond = 0;
        int64_t size = 0;
        check(dmrg_env_out_info(e, &bond, &size), "dmrg_env_out_info");
        std::vector<BlockList> out(bond);
        for (int o = 0; o < bond; ++o) {
            int n = 0;
            check(dmrg_env_out_blocks(e, o, 0, &n, nullptr, nullptr, nullptr, nullptr), "dmrg_env_out_blocks");
            BlockList& b = out[o];
            b.left.resize(n);
            b.right.resize(n);
            b.rows.resize(n);
            b.cols.resize(n);
            if (n)
                check(dmrg_env_out_blocks(e, o, n, &n, b.left.data(), b.right.data(), b.rows.data(), b.cols.data()),
                      "dmrg_env_out_blocks");
        }
        DeviceVector k(ctx, (size_t)site.ket.num_element()), i(ctx, (size_t)num_element(in)), r(ctx, (size_t)size);
        k.Upload(ket);
        i.Upload(in_values);
        check(dmrg_env_apply(e, k.data(), i.data(), r.data()), "dmrg_env_apply");
        out_values.resize((size_t)size);
        r.Download(out_values.data());
        return out;
    }

    Context* ctx_;
    SiteTensor site_;
    std::vector<BlockList> L_, R_;
    dmrg_heff_t h_ = nullptr;
    int64_t psi_dim_ = 0;
    DeviceVector Lv_, Rv_;
};

/* RealTensorLanczos (src/dmrg/realdmrg/real_tensor_lanczos.h:18-23) over one
 * site's effective Hamiltonian. */
class RealTensorLanczos {
   public:
    explicit RealTensorLanczos(RealTensorContraction& h) : h_(&h) {}

    /* LanczosMethod(int num_iter, int site, double& result) (real_tensor_lanczos.h:23,
     * .cc:14-201): `psi` (PsiDim() doubles, host) is the start vector and receives
     * the ground vector; `result` the lowest eigenvalue.  Stops like the reference
     * (beta < zero_tol, |dE| < precision, both 1e-15 there, or num_iter
     * iterations); psi_dim < 100 takes the dense exact branch. */
    void LanczosMethod(int num_iter, double* psi, double& result, double precision = 1e-15,
                       double zero_tol = 1e-15) {
        DeviceVector v(h_->context(), (size_t)h_->PsiDim());
        v.Upload(psi);
        LanczosMethodDevice(num_iter, v.data(), result, precision, zero_tol);
        v.Download(psi);
    }
    void LanczosMethodDevice(int num_iter, double* psi_dev, double& result, double precision = 1e-15,
                             double zero_tol = 1e-15) {
        check(dmrg_lanczos(h_->get(), psi_dev, num_iter, precision, zero_tol, &result, &dim_), "dmrg_lanczos");
    }
    /* Krylov dimension of the last call (0 for the dense branch). */
    int KrylovDim() const { return dim_; }

   private:
    RealTensorContraction* h_;
    int dim_ = 0;
};

/* The reference's QuickSort with index (src/util/general.h:56,
 * general.ih:7-65) on array[left..right]: flag 0 descending, 1 ascending, with
 * the reference's tie order; index is permuted along with the values.  Any
 * other flag leaves both arrays as they are, as the reference's does. */
inline void QuickSort(double* array, int* index, int left, int right, int flag = 0) {
    if (left >= right || (flag != 0 && flag != 1)) return;
    check(dmrg_quicksort_index(array + left, index + left, right - left + 1, flag == 0 ? 1 : 0),
          "dmrg_quicksort_index");
}

/* RealTensorLattice's canonicalisation (src/dmrg/realdmrg/real_tensor_lattice.h:
 * 182-194) of one site tensor: per sector SVD, truncation, the new ket blocks
 * and the canonical tensor that the merge multiplies into the next site. */
class RealTensorLattice {
   public:
    /* left_dim / right_dim: the lattice's sector dimensions; ket: its blocks. */
    RealTensorLattice(Context& ctx, std::vector<int> left_dim, std::vector<int> right_dim, BlockList ket)
        : ctx_(&ctx), left_dim_(std::move(left_dim)), right_dim_(std::move(right_dim)), ket_(std::move(ket)) {}
    ~RealTensorLattice() { release(); }
    RealTensorLattice(const RealTensorLattice&) = delete;
    RealTensorLattice& operator=(const RealTensorLattice&) = delete;

    /* ComputeTruncateDim(max_dim, canonical_precision, ...) (real_tensor_lattice.h:
     * 182-183, .cc:501-555): the kept dimension of each sector from its singular
     * values (sorted descending), which are modified in place as the reference's
     * array is.  Host only. */
    static std::vector<int> ComputeTruncateDim(int max_dim, double canonical_precision,
                                               std::vector<std::vector<double>>& singular_value) {
        const int nsec = (int)singular_value.size();
        std::vector<int> counts(nsec), tdim(nsec);
        std::vector<double> flat;
        for (int i = 0; i < nsec; ++i) {
            counts[i] = (int)singular_value[i].size();
            flat.insert(flat.end(), singular_value[i].begin(), singular_value[i].end());
        }
        check(dmrg_truncate_dims(nsec, counts.data(), flat.data(), max_dim, canonical_precision, tdim.data()),
              "dmrg_truncate_dims");
        size_t pos = 0;
        for (int i = 0; i < nsec; ++i)
            for (double& s : singular_value[i]) s = flat[pos++];
        return tdim;
    }

    /* LeftCanonicalTensorLattice(max_dim, canonical_precision) (real_tensor_lattice.h:186,
     * .cc:558-676): `ket` holds the block values (host); afterwards Ket() is the
     * left-canonical site tensor (U slices) and Canonical() one block per right
     * sector, diag(S) V^T. */
    void LeftCanonicalTensorLattice(int max_dim, double canonical_precision, const double* ket) {
        canonicalise(0, max_dim, canonical_precision, ket);
    }
    /* RightCanonicalTensorLattice (real_tensor_lattice.h:194, .cc:794-911): the
     * right-canonical site tensor (V^T slices) and one block per left sector,
     * U diag(S). */
    void RightCanonicalTensorLattice(int max_dim, double canonical_precision, const double* ket) {
        canonicalise(1, max_dim, canonical_precision, ket);
    }

    /* Results of the last canonicalisation.  Sectors are right sectors after the
     * left one, left sectors after the right one. */
    const std::vector<int>& TruncateDim() const { return tdim_; }
    double DiscardedWeight() const { return discarded_; }
    int JacobiSweeps() const { return sweeps_; }
    /* New ket: the input's blocks in the same order with their truncated shapes. */
    const BlockList& KetBlocks() const { return new_ket_; }
    const std::vector<double>& Ket() const { return ket_values_; }
    /* Canonical tensor: block s belongs to sector s (rows x cols as listed). */
    const std::vector<int>& CanonicalRows() const { return canon_rows_; }
    const std::vector<int>& CanonicalCols() const { return canon_cols_; }
    const std::vector<double>& Canonical() const { return canon_values_; }
    std::vector<double> SingularValues(int sector) const {
        int n = 0;
        check(dmrg_canon_singular_values(h_, sector, 0, nullptr, &n), "dmrg_canon_singular_values");
        std::vector<double> s(n);
        if (n) check(dmrg_canon_singular_values(h_, sector, n, s.data(), &n), "dmrg_canon_singular_values");
        return s;
    }

   private:
    void release() {
        if (h_) dmrg_canon_destroy(h_);
        h_ = nullptr;
    }
    void canonicalise(int side, int max_dim, double canpre, const double* ket) {
        release();
        const dmrg_blocks_t kb = ket_.view();
        check(dmrg_canon_create(ctx_->get(), side, (int)left_dim_.size(), (int)right_dim_.size(), left_dim_.data(),
                                right_dim_.data(), &kb, &h_),
              "dmrg_canon_create");
        const size_t nsec = side == 0 ? right_dim_.size() : left_dim_.size();
        DeviceVector in(*ctx_, (size_t)ket_.num_element());
        in.Upload(ket);
        tdim_.assign(nsec, 0);
        check(dmrg_canon_run(h_, in.data(), max_dim, canpre, tdim_.data(), &discarded_), "dmrg_canon_run");
        int64_t ket_size = 0, canon_size = 0;
        check(dmrg_canon_out_info(h_, &ket_size, &canon_size, &sweeps_), "dmrg_canon_out_info");
        new_ket_ = ket_;
        canon_rows_.assign(nsec, 0);
        canon_cols_.assign(nsec, 0);
        std::vector<int> match(nsec);
        check(dmrg_canon_out_blocks(h_, new_ket_.rows.data(), new_ket_.cols.data(), canon_rows_.data(),
                                    canon_cols_.data(), match.data()),
              "dmrg_canon_out_blocks");
        DeviceVector k(*ctx_, (size_t)ket_size), c(*ctx_, (size_t)canon_size);
        check(dmrg_canon_write(h_, in.data(), k.data(), c.data()), "dmrg_canon_write");
        ket_values_ = k.Download();
        canon_values_ = c.Download();
    }

    Context* ctx_;
    std::vector<int> left_dim_, right_dim_;
    BlockList ket_, new_ket_;
    dmrg_canon_t h_ = nullptr;
    std::vector<int> tdim_, canon_rows_, canon_cols_;
    double discarded_ = 0.0;
    int sweeps_ = 0;
    std::vector<double> ket_values_, canon_values_;
};

/* RealTensorRundmrg (src/dmrg/realdmrg/real_tensor_rundmrg.h:41-54): a whole run
 * of a reference input file (its model keys, RealTensorRundmrg keys and sweep
 * table) on the device. */
class RealTensorRundmrg {
   public:
    static dmrg_run_options_t DefaultOptions() {
        dmrg_run_options_t o{};
        o.precision = DMRG_PREC_FP64;
        o.verbose = 1;
        o.seed = 1;
        o.stop_after_half_sweeps = -1;
        o.lanczos_precision = 0.0;
        o.two_site = 0;
        o.lanczos_graph = 0;
        return o;
    }
    /* model: "real_spinless_bose_square" (the reference's
     * model/real_spinless_bose_square_model.cc), "real_spinful_bose_square" or
     * "complex_spinful_bose_square". */
    RealTensorRundmrg(Context& ctx, const std::string& input_file,
                      const std::string& model = "real_spinless_bose_square",
                      const dmrg_run_options_t& opt = DefaultOptions())
        : opt_(opt) {
        check(dmrg_run_create(ctx.get(), input_file.c_str(), model.c_str(), &opt_, &h_), "dmrg_run_create");
    }
    ~RealTensorRundmrg() {
        if (h_) dmrg_run_destroy(h_);
    }
    RealTensorRundmrg(const RealTensorRundmrg&) = delete;
    RealTensorRundmrg& operator=(const RealTensorRundmrg&) = delete;

    dmrg_run_t get() const { return h_; }
    /* Run() (real_tensor_rundmrg.h:54, .cc:115-245): every sweep of the table. */
    void Run() { check(dmrg_run_execute(h_), "dmrg_run_execute"); }
    /* The energy after each half-sweep (the reference's "right/left energy ="). */
    std::vector<double> HalfSweepEnergies() const {
        int n = 0;
        check(dmrg_run_half_sweeps(h_, 0, nullptr, nullptr, &n), "dmrg_run_half_sweeps");
        std::vector<double> e(n);
        if (n) check(dmrg_run_half_sweeps(h_, n, e.data(), nullptr, &n), "dmrg_run_half_sweeps");
        return e;
    }

   private:
    dmrg_run_options_t opt_;
    dmrg_run_t h_ = nullptr;
};

/* The model layer of an input file, host only: the MPO of
 * RealSpinlessBoseSquareHamiltonian::DefineTensorHamiltonian
 * (model/hamiltonian/real_spinless_bose_square_hamiltonian.cc:171-228) or of the
 * spinful classes, and the quantum-number tables of RealTensorSpace (which 0)
 * and RealTensorHamiltonian (which 1). */
class TensorModel {
   public:
    TensorModel(const std::string& input_file, const std::string& model = "real_spinless_bose_square") {
        check(dmrg_model_create(input_file.c_str(), model.c_str(), &h_), "dmrg_model_create");
        check(dmrg_model_info(h_, &num_site_, &physics_dim_, &num_quantum_), "dmrg_model_info");
        int z = 0;
        check(dmrg_model_is_complex(h_, &z), "dmrg_model_is_complex");
        complex_ = z != 0;
    }
    ~TensorModel() {
        if (h_) dmrg_model_destroy(h_);
    }
    TensorModel(const TensorModel&) = delete;
    TensorModel& operator=(const TensorModel&) = delete;

    int num_site() const { return num_site_; }
    int physics_dim() const { return physics_dim_; }
    int num_quantum() const { return num_quantum_; }
    bool is_complex() const { return complex_; }
    /* The MPO site tensor W[left_bond][right_bond][d][d] of `site` (interleaved
     * (re, im) pairs for a complex model). */
    std::vector<double> TensorOperator(int site, int& left_bond, int& right_bond) const {
        check(dmrg_model_mpo(h_, site, &left_bond, &right_bond, 0, nullptr), "dmrg_model_mpo");
        std::vector<double> w((size_t)left_bond * right_bond * physics_dim_ * physics_dim_ * (complex_ ? 2 : 1));
        check(dmrg_model_mpo(h_, site, &left_bond, &right_bond, (int)w.size(), w.data()), "dmrg_model_mpo");
        return w;
    }
    /* Quantum numbers of bond `bond`: rows x num_quantum(), row-major. */
    std::vector<int> QuantumTable(int which, int bond, int& rows) const {
        check(dmrg_model_quantum_table(h_, which, bond, 0, nullptr, &rows), "dmrg_model_quantum_table");
        std::vector<int> v((size_t)rows * num_quantum_);
        if (!v.empty())
            check(dmrg_model_quantum_table(h_, which, bond, (int)v.size(), v.data(), &rows),
                  "dmrg_model_quantum_table");
        return v;
    }

   private:
    dmrg_model_t h_ = nullptr;
    int num_site_ = 0, physics_dim_ = 0, num_quantum_ = 0;
    bool complex_ = false;
};

}  // namespace dmrgcc_b200

#endif /* DMRG_B200_HPP_ */
