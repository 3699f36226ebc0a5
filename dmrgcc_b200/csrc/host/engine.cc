// DMRG sweep engine (see engine.h).  Each member names the reference routine
// whose bookkeeping it reproduces.
#include "host/engine.h"

#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <stdexcept>
#include <system_error>
#include <thread>

#include <nvtx3/nvToolsExt.h>

#include "gemm.cuh"
#include "zgemm.cuh"

extern "C" {
int dmrg_canon_create(dmrg_ctx_t, int, int, int, const int*, const int*, const dmrg_blocks_t*, dmrg_canon_t*);
int dmrg_canon_destroy(dmrg_canon_t);
int dmrg_canon_run(dmrg_canon_t, const double*, int, double, int*, double*);
int dmrg_canon_out_info(dmrg_canon_t, int64_t*, int64_t*, int*);
int dmrg_canon_out_blocks(dmrg_canon_t, int*, int*, int*, int*, int*);
int dmrg_canon_write(dmrg_canon_t, const double*, double*, double*);
int dmrg_zcanon_create(dmrg_ctx_t, int, int, int, const int*, const int*, const dmrg_blocks_t*, dmrg_zcanon_t*);
int dmrg_zcanon_destroy(dmrg_zcanon_t);
int dmrg_zcanon_run(dmrg_zcanon_t, const double*, int, double, int*, double*);
int dmrg_zcanon_out_info(dmrg_zcanon_t, int64_t*, int64_t*, int*);
int dmrg_zcanon_out_blocks(dmrg_zcanon_t, int*, int*, int*, int*, int*);
int dmrg_zcanon_write(dmrg_zcanon_t, const double*, double*, double*);
}

namespace dmrg {

namespace {

double wall_time() {
    timeval t;
    gettimeofday(&t, nullptr);
    return t.tv_sec + t.tv_usec * 1e-6;
}

dmrg_blocks_t as_blocks(const BlockListDesc& b) {
    return dmrg_blocks_t{b.count(), b.left.data(), b.right.data(), b.rows.data(), b.cols.data()};
}

// RealMatrix::RandomMatrix (src/tensor/real_matrix.cc:201-208): column-major
// draws of 0.01 * (rand() % 100) into a rows x cols row-major block; `draws`
// counts them (trace output).
void random_block(GlibcRand& rng, long long& draws, std::vector<double>& out, size_t off, int rows, int cols) {
    draws += (long long)rows * cols;
    for (int j = 0; j < cols; ++j)
        for (int i = 0; i < rows; ++i) out[off + (size_t)i * cols + j] = 0.01 * (rng.next() % 100);
}

// ComplexMatrix::RandomMatrix (src/tensor/complex_matrix.cc:201-209): the same
// column-major walk, each element Complex(0.01 * (rand() % 100), 0.01 *
// (rand() % 100)); the reference's compiler (g++, x86-64) evaluates the
// constructor's arguments right to left, so the imaginary part takes the
// first draw.  Interleaved (re, im) into a rows x cols row-major block.
void random_block_complex(GlibcRand& rng, long long& draws, std::vector<double>& out, size_t off, int rows,
                          int cols) {
    draws += 2LL * rows * cols;
    for (int j = 0; j < cols; ++j)
        for (int i = 0; i < rows; ++i) {
            const double im = 0.01 * (rng.next() % 100);
            const double re = 0.01 * (rng.next() % 100);
            out[2 * (off + (size_t)i * cols + j)] = re;
            out[2 * (off + (size_t)i * cols + j) + 1] = im;
        }
}

int find_value(const std::vector<int>& v, int x) {
    for (int i = 0; i < (int)v.size(); ++i)
        if (v[i] == x) return i;
    return -1;
}

}  // namespace

int DevBlocks::alloc(cudaStream_t st, bool zero, int ew) {
    DMRG_TRY(buf.alloc((size_t)std::max<int64_t>(d.size, 1) * ew * sizeof(double)));
    if (zero && d.size) DMRG_CUDA_TRY(cudaMemsetAsync(buf.ptr, 0, (size_t)d.size * ew * sizeof(double), st));
    return DMRG_OK;
}

// ---------------------------------------------------------------------------
// construction: RealTensorRundmrg::RealTensorRundmrg + Sweep (real_tensor_rundmrg.cc:3-113)
// ---------------------------------------------------------------------------
Engine::Engine(dmrg_ctx_t ctx, std::unique_ptr<QuantumSpace> space, std::unique_ptr<MpoHamiltonian> ham,
               InputGroup& input, const RunOptions& opt)
    : ctx_(ctx), st_(ctx->stream), opt_(opt), space_(std::move(space)), ham_(std::move(ham)) {
    n_ = space_->num_site();
    cplx_ = ham_->is_complex();
    ew_ = cplx_ ? 2 : 1;
    if (cplx_ && (opt_.two_site || opt_.precision != DMRG_PREC_FP64))
        throw StatusError(DMRG_E_ARG, "a complex run has single-site FP64 sweeps only");
    // disk_cache (tensors swapped to files between uses) is read for compatibility
    // and ignored: every tensor stays resident.  cache_record / cache_resume
    // write and read the reference's checkpoint file (real_tensor_rundmrg.cc:16-23).
    input.getBool("disk_cache", false);
    cache_name_ = input.getString("cache_name", ".");
    cache_record_ = input.getBool("cache_record", false);
    record_name_ = input.getString("record_name", "record.dat");
    cache_resume_ = input.getBool("cache_resume", false);
    if (cache_resume_) resume_name_ = input.getString("resume_name", "");
    first_block_ = input.getInt("first_block");
    first_dim_ = input.getInt("first_dim");
    const int num_sweep = input.getInt("num_sweep");
    num_sweep_ = 2 * num_sweep;
    InputGroup table(input, "sweeps");
    if (!table.GotoGroup()) throw InputError("Couldn't find table " + table.name());
    table.SkipLine();
    max_dim_.assign(num_sweep_, 0);
    max_block_.assign(num_sweep_, 0);
    num_iter_.assign(num_sweep_, 0);
    canpre_.assign(num_sweep_, 0.0);
    noise_.assign(num_sweep_, 0.0);
    int nlast = num_sweep_;
    for (int i = 0; i < num_sweep_; ++i) {
        table.file() >> max_dim_[i] >> max_block_[i] >> num_iter_[i] >> canpre_[i] >> noise_[i];
        if (max_dim_[i] == 0) {
            nlast = i - 1;
            break;
        }
    }
    if (nlast < 0) throw InputError("the sweep table starts with maxm = 0");
    for (int i = nlast + 1; i < num_sweep_; ++i) {
        max_dim_[i] = max_block_[nlast];  // the reference copies maxb into maxm here (:94)
        max_block_[i] = max_block_[nlast];
        num_iter_[i] = num_iter_[nlast];
        canpre_[i] = canpre_[nlast];
        noise_[i] = noise_[nlast];
    }
    if (opt_.verbose) {
        std::printf("Sweeps:\n");
        for (int i = 0; i < num_sweep_; ++i)
            std::printf("%d Maxm=%d, Maxb=%d, Niter=%d, Canon=%g, Noise=%g\n", i + 1, max_dim_[i], max_block_[i],
                        num_iter_[i], canpre_[i], noise_[i]);
    }
    for (int i = 0; i < num_sweep_; ++i) noise_[i] = std::pow(0.1, noise_[i]);

    rs_.alloc(2 * ctx_->num_sms, 1);
    if (const char* tp = std::getenv("DMRG_TRACE")) trace_ = std::fopen(tp, "w");
    lat_.resize(n_);
    for (int i = 0; i < n_; ++i) {
        lat_[i].reset(new TensorLattice());
        lat_[i]->physics_dim = space_->physics_dim();
    }
    rng_.seed_with(opt_.seed);
    rand_draws_ = 0;
    // a resumed run starts from the recorded MPS instead of the random one (and so
    // draws no random numbers before its first expansion), like the reference (:44-51)
    int rc = cache_resume_ ? ReadTensorSpace(resume_name_) : DefineTensorSpace(first_block_, first_dim_);
    if (rc != DMRG_OK)
        throw StatusError(rc, std::string(cache_resume_ ? "ReadTensorSpace: " : "DefineTensorSpace: ") +
                                  dmrg_last_error());
    ham_->DefineTensorHamiltonian();
    con_.resize(n_ + 1);
    for (int i = 0; i <= n_; ++i) {
        con_[i].reset(new TensorContraction());
        if (i < n_) {
            con_[i]->left_bond = ham_->left_bond(i);
            con_[i]->right_bond = ham_->right_bond(i);
        } else {
            con_[i]->left_bond = ham_->right_bond(n_ - 1);
            con_[i]->right_bond = ham_->left_bond(0);
        }
        con_[i]->L.desc.o.assign(con_[i]->left_bond, BlockListDesc());
        con_[i]->L.desc.rebase();
        con_[i]->R.desc.o.assign(con_[i]->right_bond, BlockListDesc());
        con_[i]->R.desc.rebase();
    }
}

Engine::~Engine() {
    if (trace_) std::fclose(trace_);
}

// Sector dimensions of a site after an operation (same format as the reference
// probe's trace, for step-by-step comparison).
void Engine::Trace(const char* tag, int leigh, int site) {
    if (!trace_) return;
    const TensorLattice& t = *lat_[site];
    std::fprintf(trace_, "%s %d %d L:", tag, leigh, site);
    for (int d : t.left_dim) std::fprintf(trace_, "%d,", d);
    std::fprintf(trace_, " R:");
    for (int d : t.right_dim) std::fprintf(trace_, "%d,", d);
    auto fetch = [&](const DevBlocks& b, std::vector<double>& h) {
        h.assign((size_t)b.d.size * ew_, 0.0);
        if (!h.empty() &&
            (cudaMemcpyAsync(h.data(), b.ptr(), h.size() * sizeof(double), cudaMemcpyDeviceToHost, st_) != cudaSuccess ||
             cudaStreamSynchronize(st_) != cudaSuccess))
            h.assign(h.size(), 0.0);
    };
    std::vector<double> h;
    fetch(t.ket, h);
    double norm2 = 0.0;
    for (double v : h) norm2 += v * v;
    std::fprintf(trace_, " P:%lld N:%.10e Q:%lld", (long long)t.psi_dim(), norm2, rand_draws_);
    if (tag[0] == 'C' && t.has_canonical) {  // per-block squared norms of S V^T (or U S)
        fetch(t.canonical, h);
        std::fprintf(trace_, " S:");
        for (int k = 0; k < t.canonical.d.count(); ++k) {
            double s2 = 0.0;
            for (int64_t i = 0; i < (int64_t)t.canonical.d.rows[k] * t.canonical.d.cols[k] * ew_; ++i)
                s2 += h[t.canonical.d.off[k] * ew_ + i] * h[t.canonical.d.off[k] * ew_ + i];
            std::fprintf(trace_, "%.8e,", s2);
        }
    }
    std::fprintf(trace_, "\n");
    std::fflush(trace_);
}

// ---------------------------------------------------------------------------
// sector bookkeeping (RealTensorSpace, real_tensor_space.cc)
// ---------------------------------------------------------------------------
void Engine::ComputeLatticeBlock(int site, std::vector<int>& left_block, std::vector<int>& right_block) {
    const auto& lq = space_->table(site);
    const auto& rq = space_->table(site + 1);
    if (site == 0) left_block = {0};
    else left_block = lat_[site - 1]->right_block;
    right_block.clear();
    for (int r = 0; r < (int)rq.size(); ++r) {
        for (int l = 0; l < (int)left_block.size(); ++l)
            if (space_->CheckQuantumTable(site, lq[left_block[l]], rq[r]) != -1) {
                right_block.push_back(r);
                break;
            }
        if ((int)right_block.size() == p_max_block_) break;
    }
}

void Engine::ComputeTensorIndex(int site, std::vector<int>& li, std::vector<int>& ri, std::vector<int>& pi) {
    const TensorLattice& t = *lat_[site];
    const auto& lq = space_->table(site);
    const auto& rq = space_->table(site + 1);
    li.clear();
    ri.clear();
    pi.clear();
    for (int i = 0; i < t.nl(); ++i)
        for (int j = 0; j < t.nr(); ++j) {
            const int info = space_->CheckQuantumTable(site, lq[t.left_block[i]], rq[t.right_block[j]]);
            if (info != -1) {
                li.push_back(i);
                ri.push_back(j);
                pi.push_back(info);
            }
        }
}

// RealTensorLattice::DefineTensorLattice(sectors) (real_tensor_lattice.cc:285-325)
void Engine::DefineLatticeSectors(TensorLattice& t, const std::vector<int>& lb, const std::vector<int>& rb,
                                  const std::vector<int>& ld, const std::vector<int>& rd) {
    t.left_block = lb;
    t.right_block = rb;
    t.left_dim = ld;
    t.right_dim = rd;
    t.phys.assign((size_t)lb.size() * rb.size(), -1);
}

// RealTensorLattice::DefineTensorLattice(blocks, row, column) (:328-343): every
// block row x column, random from the glibc stream.
int Engine::DefineLatticeBlocks(TensorLattice& t, const std::vector<int>& li, const std::vector<int>& ri,
                                const std::vector<int>& pi, int row, int column, bool device) {
    t.ket = DevBlocks();
    for (size_t k = 0; k < li.size(); ++k) {
        t.phys[(size_t)li[k] * t.nr() + ri[k]] = pi[k];
        t.ket.d.push(li[k], ri[k], row, column);
    }
    std::vector<double> host((size_t)std::max<int64_t>(t.ket.d.size, 0) * ew_);
    for (size_t k = 0; k < li.size(); ++k) {
        if (cplx_) random_block_complex(rng_, rand_draws_, host, (size_t)t.ket.d.off[k], row, column);
        else random_block(rng_, rand_draws_, host, (size_t)t.ket.d.off[k], row, column);
    }
    if (!device) return DMRG_OK;  // the draws only advance the stream (the caller discards the values)
    DMRG_TRY(t.ket.alloc(st_, false, ew_));
    if (!host.empty())
        DMRG_CUDA_TRY(cudaMemcpyAsync(t.ket.ptr(), host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice,
                                      st_));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
    return DMRG_OK;
}

// RealTensorSpace::DefineTensorSpace (real_tensor_space.cc:68-134)
int Engine::DefineTensorSpace(int initial_block, int initial_dim) {
    if (opt_.verbose) std::printf("Initial Block = %d, Intial Dimension = %d\n", initial_block, initial_dim);
    p_max_block_ = initial_block;
    p_max_dim_ = -1;
    p_noise_ = 10;
    p_canpre_ = 1e-30;
    for (int i = 0; i < n_; ++i) {
        std::vector<int> lb, rb;
        ComputeLatticeBlock(i, lb, rb);
        std::vector<int> ld(lb.size(), i == 0 ? 1 : initial_dim), rd(rb.size(), i == n_ - 1 ? 1 : initial_dim);
        DefineLatticeSectors(*lat_[i], lb, rb, ld, rd);
    }
    for (int i = 0; i < n_; ++i) {
        std::vector<int> li, ri, pi;
        ComputeTensorIndex(i, li, ri, pi);
        const int row = i == 0 ? 1 : initial_dim;
        const int column = i == n_ - 1 ? 1 : initial_dim;
        DMRG_TRY(DefineLatticeBlocks(*lat_[i], li, ri, pi, row, column));
        DMRG_TRY(CanonicalTensorSpace(0, i));
        if (i > 0) DMRG_TRY(MergeTensorSpace(0, i));
    }
    return DMRG_OK;
}

// ---------------------------------------------------------------------------
// canonicalisation and merge (device)
// ---------------------------------------------------------------------------
int Engine::CanonicalTensorSpace(int leigh, int site, double* discarded) {
    TensorLattice& t = *lat_[site];
    dmrg_blocks_t kb = as_blocks(t.ket.d);
    dmrg_canon_t c = nullptr;
    dmrg_zcanon_t zc = nullptr;  // complex run: ComplexTensorLattice::Left/RightCanonicalTensorLattice
    if (cplx_) DMRG_TRY(dmrg_zcanon_create(ctx_, leigh, t.nl(), t.nr(), t.left_dim.data(), t.right_dim.data(), &kb, &zc));
    else DMRG_TRY(dmrg_canon_create(ctx_, leigh, t.nl(), t.nr(), t.left_dim.data(), t.right_dim.data(), &kb, &c));
    const int nsec = leigh == 0 ? t.nr() : t.nl();
    std::vector<int> tdim(nsec);
    double disc = 0.0;
    int rc = cplx_ ? dmrg_zcanon_run(zc, t.ket.ptr(), p_max_dim_, p_canpre_, tdim.data(), &disc)
                   : dmrg_canon_run(c, t.ket.ptr(), p_max_dim_, p_canpre_, tdim.data(), &disc);
    int64_t ks = 0, cs = 0;
    int sweeps = 0;
    if (rc == DMRG_OK) rc = cplx_ ? dmrg_zcanon_out_info(zc, &ks, &cs, &sweeps) : dmrg_canon_out_info(c, &ks, &cs, &sweeps);
    svd_sweeps_ += sweeps;
    const int nb = t.ket.d.count();
    std::vector<int> kr(std::max(nb, 1)), kc(std::max(nb, 1)), cr(nsec), cc(nsec), md(nsec);
    if (rc == DMRG_OK)
        rc = cplx_ ? dmrg_zcanon_out_blocks(zc, kr.data(), kc.data(), cr.data(), cc.data(), md.data())
                   : dmrg_canon_out_blocks(c, kr.data(), kc.data(), cr.data(), cc.data(), md.data());
    DevBlocks nk, can;
    if (rc == DMRG_OK) {
        for (int k = 0; k < nb; ++k) nk.d.push(t.ket.d.left[k], t.ket.d.right[k], kr[k], kc[k]);
        for (int s = 0; s < nsec; ++s) can.d.push(s, s, cr[s], cc[s]);
        rc = nk.alloc(st_, false, ew_);
        if (rc == DMRG_OK) rc = can.alloc(st_, false, ew_);
        if (rc == DMRG_OK)
            rc = cplx_ ? dmrg_zcanon_write(zc, t.ket.ptr(), nk.ptr(), can.ptr())
                       : dmrg_canon_write(c, t.ket.ptr(), nk.ptr(), can.ptr());
        if (rc == DMRG_OK) {
            cudaError_t e = cudaStreamSynchronize(st_);
            if (e != cudaSuccess) rc = set_error(DMRG_E_CUDA, "canonical write: %s", cudaGetErrorString(e));
        }
    }
    if (cplx_) dmrg_zcanon_destroy(zc);
    else dmrg_canon_destroy(c);
    DMRG_TRY(rc);
    t.ket = std::move(nk);
    t.canonical = std::move(can);
    t.has_canonical = true;
    t.match_dim = md;
    if (leigh == 0) t.right_dim = tdim;
    else t.left_dim = tdim;
    if (discarded) *discarded = disc;
    Trace("C", leigh, site);
    return DMRG_OK;
}

int Engine::Normalize(TensorLattice& t) {
    if (t.ket.d.size == 0) return DMRG_OK;
    DMRG_TRY(norm_.alloc(8 * sizeof(double)));
    // the norm of a complex vector is that of its interleaved doubles
    const int64_t n = t.ket.d.size * ew_;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 2 * ctx_->num_sms);
    return vec_normalize(t.ket.ptr(), n, norm_.as<double>(), rs_, blocks, st_);
}

// RealTensorSpace::MergeTensorSpace -> RealTensorLattice::Left/RightMergeTensorLattice
// (real_tensor_lattice.cc:914-977): neighbour's canonical block times this site's blocks.
int Engine::MergeTensorSpace(int leigh, int site) {
    if (!(leigh == 0 && site > 0) && !(leigh == 1 && site < n_ - 1)) return DMRG_OK;
    TensorLattice& t = *lat_[site];
    TensorLattice& o = *lat_[leigh == 0 ? site - 1 : site + 1];
    if (!o.has_canonical) return set_error(DMRG_E_STATE, "Canonical tensor is nullptr in MergeTensorLattice");
    DevBlocks nk;
    GemmSchedule s;
    const int nb = t.ket.d.count();
    for (int k = 0; k < nb; ++k) {
        const int l = t.ket.d.left[k], r = t.ket.d.right[k];
        const int sec = leigh == 0 ? l : r;
        const int cr = o.canonical.d.rows[sec], cc = o.canonical.d.cols[sec];
        const int kr = t.ket.d.rows[k], kc = t.ket.d.cols[k];
        if (leigh == 0) {
            if (cc != kr) return set_error(DMRG_E_ARG, "Matrix indeces do not match in LeftMergeTensorLattice");
            nk.d.push(l, r, cr, kc);
        } else {
            if (kc != cr) return set_error(DMRG_E_ARG, "Matrix indeces do not match in RightMergeTensorLattice");
            nk.d.push(l, r, kr, cc);
        }
    }
    DMRG_TRY(nk.alloc(st_, true, ew_));
    ZGemmSchedule zs;  // complex run: ComplexMatrix::MultiplyToMatrix (zgemm)
    for (int k = 0; k < nb; ++k) {
        const int sec = leigh == 0 ? t.ket.d.left[k] : t.ket.d.right[k];
        if (nk.d.rows[k] == 0 || nk.d.cols[k] == 0) continue;
        if (cplx_) {
            zs.add_group(nk.d.off[k], nk.d.cols[k], nk.d.rows[k], nk.d.cols[k]);
            if (leigh == 0)
                zs.add_term(o.canonical.d.off[sec], o.canonical.d.cols[sec], t.ket.d.off[k], t.ket.d.cols[k],
                            o.canonical.d.cols[sec], 1.0, 0.0);
            else
                zs.add_term(t.ket.d.off[k], t.ket.d.cols[k], o.canonical.d.off[sec], o.canonical.d.cols[sec],
                            t.ket.d.cols[k], 1.0, 0.0);
            continue;
        }
        s.add_group(nk.d.off[k], nk.d.cols[k], nk.d.rows[k], nk.d.cols[k]);
        if (leigh == 0)
            s.add_term(o.canonical.d.off[sec], o.canonical.d.cols[sec], t.ket.d.off[k], t.ket.d.cols[k],
                       o.canonical.d.cols[sec], 1.0);
        else
            s.add_term(t.ket.d.off[k], t.ket.d.cols[k], o.canonical.d.off[sec], o.canonical.d.cols[sec],
                       t.ket.d.cols[k], 1.0);
    }
    if (cplx_) {
        if (leigh == 0) DMRG_TRY(zs.check_bounds(o.canonical.d.size, t.ket.d.size, nk.d.size));
        else DMRG_TRY(zs.check_bounds(t.ket.d.size, o.canonical.d.size, nk.d.size));
        DMRG_TRY(zs.finalize(st_));
        if (leigh == 0) DMRG_TRY(launch_zgemm(zs, o.canonical.ptr(), t.ket.ptr(), nk.ptr(), false, st_));
        else DMRG_TRY(launch_zgemm(zs, t.ket.ptr(), o.canonical.ptr(), nk.ptr(), false, st_));
    } else {
        if (leigh == 0) DMRG_TRY(s.check_bounds(o.canonical.d.size, t.ket.d.size, nk.d.size));
        else DMRG_TRY(s.check_bounds(t.ket.d.size, o.canonical.d.size, nk.d.size));
        DMRG_TRY(s.finalize(64, 64, 16, st_));
        if (leigh == 0) DMRG_TRY(launch_gemm_f64(s, o.canonical.ptr(), t.ket.ptr(), nk.ptr(), false, st_));
        else DMRG_TRY(launch_gemm_f64(s, t.ket.ptr(), o.canonical.ptr(), nk.ptr(), false, st_));
    }
    DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
    // sector dims follow the canonical blocks
    if (leigh == 0)
        for (int l = 0; l < t.nl(); ++l) t.left_dim[l] = o.canonical.d.rows[l];
    else
        for (int r = 0; r < t.nr(); ++r) t.right_dim[r] = o.canonical.d.cols[r];
    t.ket = std::move(nk);
    DMRG_TRY(Normalize(t));
    Trace("M", leigh, site);
    o.has_canonical = false;
    o.canonical = DevBlocks();
    o.match_dim.clear();
    return DMRG_OK;
}

// ---------------------------------------------------------------------------
// re-layout of a site tensor: Left/RightExpanTensorLattice (real_tensor_lattice.cc:979-1149)
// ---------------------------------------------------------------------------
int Engine::ExpanLattice(int leigh, TensorLattice& t, const TensorLattice& origin, const TensorLattice* expan) {
    struct Part {
        int src;  // 0 origin, 1 expan
        int q;    // block in the source
        int at;   // column (leigh 0) or row (leigh 1) offset in the new block
    };
    const int nb = t.ket.d.count();
    std::vector<std::vector<Part>> parts(nb);
    BlockListDesc nd;
    for (int k = 0; k < nb; ++k) {
        const int l = t.ket.d.left[k], r = t.ket.d.right[k];
        int e0, e1 = -1;
        if (leigh == 0) {
            e0 = find_value(origin.right_block, t.right_block[r]);
            if (expan) e1 = find_value(expan->right_block, t.right_block[r]);
        } else {
            e0 = find_value(origin.left_block, t.left_block[l]);
            if (expan) e1 = find_value(expan->left_block, t.left_block[l]);
        }
        int rows = 0, cols = 0;
        if (e0 != -1) {
            const int q = leigh == 0 ? origin.ket.d.find(l, e0) : origin.ket.d.find(e0, r);
            if (q != -1 && origin.ket.d.rows[q] * origin.ket.d.cols[q] > 0) {
                rows = origin.ket.d.rows[q];
                cols = origin.ket.d.cols[q];
                parts[k].push_back(Part{0, q, 0});
            }
        }
        if (e1 != -1) {
            const int q = leigh == 0 ? expan->ket.d.find(l, e1) : expan->ket.d.find(e1, r);
            if (q != -1 && expan->ket.d.rows[q] * expan->ket.d.cols[q] > 0) {
                const int er = expan->ket.d.rows[q], ec = expan->ket.d.cols[q];
                if (rows == 0) {  // AddToMatrix into an empty block: a copy
                    rows = er;
                    cols = ec;
                    parts[k].push_back(Part{1, q, 0});
                } else if (leigh == 0) {  // ExpanMatrix(1, .): column concatenation
                    if (er != rows) return set_error(DMRG_E_ARG, "row or column dimension is not match in ExpanMatrix");
                    parts[k].push_back(Part{1, q, cols});
                    cols += ec;
                } else {  // ExpanMatrix(0, .): row concatenation
                    if (ec != cols) return set_error(DMRG_E_ARG, "row or column dimension is not match in ExpanMatrix");
                    parts[k].push_back(Part{1, q, rows});
                    rows += er;
                }
            }
        }
        if (e0 != -1 && e1 == -1) {  // zero padding up to the sector dimension
            if (leigh == 0) {
                const int add = t.right_dim[r] - cols;
                if (add < 0) return set_error(DMRG_E_ARG, "expan_dim < 0 in LeftExpanTensorLattice");
                if (add > 0 || t.left_dim[l] > 0) {
                    if (rows != t.left_dim[l])
                        return set_error(DMRG_E_ARG, "row or column dimension is not match in ExpanMatrix");
                    cols += add;
                }
            } else {
                const int add = t.left_dim[l] - rows;
                if (add < 0) return set_error(DMRG_E_ARG, "expan_dim < 0 in RightExpanTensorLattice");
                if (add > 0 || t.right_dim[r] > 0) {
                    if (cols != t.right_dim[r])
                        return set_error(DMRG_E_ARG, "row or column dimension is not match in ExpanMatrix");
                    rows += add;
                }
            }
        }
        if (e0 == -1 && e1 == -1 && rows == 0) {  // AddToMatrix(zeros(left_dim, right_dim))
            rows = t.left_dim[l];
            cols = t.right_dim[r];
            if ((int64_t)rows * cols == 0) rows = cols = 0;
        }
        nd.push(l, r, rows, cols);
    }
    DevBlocks nk;
    nk.d = nd;
    DMRG_TRY(nk.alloc(st_, true, ew_));
    // a complex block row-major is a real one of twice the columns
    std::vector<RectCopy> from_origin, from_expan;
    for (int k = 0; k < nb; ++k)
        for (const Part& p : parts[k]) {
            const TensorLattice& src = p.src == 0 ? origin : *expan;
            const int sr = src.ket.d.rows[p.q], sc = src.ket.d.cols[p.q];
            RectCopy c{src.ket.d.off[p.q] * ew_, (nd.off[k] + (leigh == 0 ? p.at : (int64_t)p.at * nd.cols[k])) * ew_,
                       sc * ew_, nd.cols[k] * ew_, sr, sc * ew_, 1.0};
            (p.src == 0 ? from_origin : from_expan).push_back(c);
        }
    DMRG_TRY(launch_rect_copies(from_origin, origin.ket.ptr(), origin.ket.d.size * ew_, nk.ptr(), nd.size * ew_,
                                copy_tasks_, st_));
    if (!from_expan.empty()) {
        DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
        DMRG_TRY(launch_rect_copies(from_expan, expan->ket.ptr(), expan->ket.d.size * ew_, nk.ptr(), nd.size * ew_,
                                    copy_tasks_, st_));
    }
    DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
    t.ket = std::move(nk);
    return DMRG_OK;
}

static bool expansion_enabled(int max_block, int max_dim, double noise) {
    return !(max_block < 0 || max_dim < 0 || noise > 1);
}

// Sorted union of two sector lists with summed dimensions (CombineTensorLattice,
// real_tensor_lattice.cc:361-478).
static void combine_sectors(const std::vector<int>& b0, const std::vector<int>& d0, const std::vector<int>& b1,
                            const std::vector<int>& d1, std::vector<int>& out_b, std::vector<int>& out_d) {
    out_b = b0;
    for (int x : b1)
        if (find_value(b0, x) == -1) out_b.push_back(x);
    std::sort(out_b.begin(), out_b.end());
    out_d.assign(out_b.size(), 0);
    for (size_t i = 0; i < out_b.size(); ++i) {
        int j = find_value(b0, out_b[i]);
        if (j != -1) out_d[i] += d0[j];
        j = find_value(b1, out_b[i]);
        if (j != -1) out_d[i] += d1[j];
    }
}

// One expansion random matrix (d0 x d1) appended to the plan: the reference's
// RandomMatrix draws (real or complex), then 0.1 * W on its diagonal
// (real_tensor_contraction.cc:396-399, complex twin :396-399).  Returns its
// offset in elements.
int64_t Engine::add_random(int d0, int d1, double wre, double wim) {
    std::vector<double>& rnd = xw_.rnd;
    const int64_t ro = (int64_t)rnd.size() / ew_;
    rnd.resize(rnd.size() + (size_t)d0 * d1 * ew_);
    if (cplx_) {
        random_block_complex(rng_, rand_draws_, rnd, (size_t)ro, d0, d1);
        for (int q = 0; q < std::min(d0, d1); ++q) {
            rnd[2 * (ro + (size_t)q * d1 + q)] = 0.1 * wre;
            rnd[2 * (ro + (size_t)q * d1 + q) + 1] = 0.1 * wim;
        }
    } else {
        random_block(rng_, rand_draws_, rnd, (size_t)ro, d0, d1);
        for (int q = 0; q < std::min(d0, d1); ++q) rnd[ro + (size_t)q * d1 + q] = 0.1 * wre;
    }
    return ro;
}

// RealTensorSpace::ExpanTensorSpace (real_tensor_space.cc:319-387)
int Engine::ExpanTensorSpace(int leigh, int site) {
    if (!expansion_enabled(p_max_block_, p_max_dim_, p_noise_)) return DMRG_OK;
    if (!expan_) return set_error(DMRG_E_STATE, "expan_tensor_lattice is nullptr!");
    TensorLattice origin;
    {
        TensorLattice& t = *lat_[site];
        origin.physics_dim = t.physics_dim;
        origin.left_block = t.left_block;
        origin.left_dim = t.left_dim;
        origin.right_block = t.right_block;
        origin.right_dim = t.right_dim;
        origin.phys = t.phys;
        origin.ket = std::move(t.ket);
    }
    TensorLattice& t = *lat_[site];
    std::vector<int> lb = origin.left_block, ld = origin.left_dim, rb = origin.right_block, rd = origin.right_dim;
    if (leigh == 0) combine_sectors(origin.right_block, origin.right_dim, expan_->right_block, expan_->right_dim, rb, rd);
    else combine_sectors(origin.left_block, origin.left_dim, expan_->left_block, expan_->left_dim, lb, ld);
    DefineLatticeSectors(t, lb, rb, ld, rd);
    std::vector<int> li, ri, pi;
    ComputeTensorIndex(site, li, ri, pi);
    DMRG_TRY(DefineLatticeBlocks(t, li, ri, pi, 1, 1));
    t.ket.set_shape_zero();
    if (trace_) {  // the expansion term, block by block, before it is merged
        const DevBlocks& eb = expan_->ket;
        std::vector<double> h((size_t)eb.d.size * ew_);
        if (!h.empty()) {
            DMRG_CUDA_TRY(cudaMemcpyAsync(h.data(), eb.ptr(), h.size() * sizeof(double), cudaMemcpyDeviceToHost, st_));
            DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
        }
        std::fprintf(trace_, "Y %d %d", leigh, site);
        for (int k = 0; k < eb.d.count(); ++k) {
            double s2 = 0.0;
            for (int64_t i = 0; i < (int64_t)eb.d.rows[k] * eb.d.cols[k] * ew_; ++i)
                s2 += h[eb.d.off[k] * ew_ + i] * h[eb.d.off[k] * ew_ + i];
            std::fprintf(trace_, " %d.%d:%dx%d=%.8e", eb.d.left[k], eb.d.right[k], eb.d.rows[k], eb.d.cols[k], s2);
        }
        std::fprintf(trace_, "\n");
    }
    DMRG_TRY(ExpanLattice(leigh, t, origin, expan_.get()));
    expan_.reset();
    return DMRG_OK;
}

// RealTensorSpace::MatchTensorSpace (real_tensor_space.cc:389-440)
int Engine::MatchTensorSpace(int leigh, int site) {
    if (!expansion_enabled(p_max_block_, p_max_dim_, p_noise_)) return DMRG_OK;
    TensorLattice& t = *lat_[site];
    TensorLattice origin;
    origin.physics_dim = t.physics_dim;
    origin.left_block = t.left_block;
    origin.left_dim = t.left_dim;
    origin.right_block = t.right_block;
    origin.right_dim = t.right_dim;
    origin.phys = t.phys;
    origin.ket = std::move(t.ket);
    std::vector<int> lb, ld, rb, rd;
    if (leigh == 0 && site > 0) {
        lb = lat_[site - 1]->right_block;
        ld = lat_[site - 1]->match_dim;
        rb = origin.right_block;
        rd = origin.right_dim;
    } else if (leigh == 1 && site < n_ - 1) {
        lb = origin.left_block;
        ld = origin.left_dim;
        rb = lat_[site + 1]->left_block;
        rd = lat_[site + 1]->match_dim;
    }
    DefineLatticeSectors(t, lb, rb, ld, rd);
    std::vector<int> li, ri, pi;
    ComputeTensorIndex(site, li, ri, pi);
    DMRG_TRY(DefineLatticeBlocks(t, li, ri, pi, 1, 1));
    t.ket.set_shape_zero();
    if (leigh == 0 && site > 0) DMRG_TRY(ExpanLattice(1, t, origin, nullptr));
    else if (leigh == 1 && site < n_ - 1) DMRG_TRY(ExpanLattice(0, t, origin, nullptr));
    return DMRG_OK;
}

// RealTensorSpace::ComputeExpanTensorLattice (real_tensor_space.cc:552-706)
void Engine::ComputeExpanTensorLattice(int leigh, int site, std::vector<std::vector<int>>& mapping) {
    const TensorLattice& t = *lat_[site];
    const auto& lq = space_->table(site);
    const auto& rq = space_->table(site + 1);
    const auto& leigh_table = space_->table(site + leigh);
    const auto& op_table = ham_->quantum_table(site + leigh);
    const std::vector<int>& old = leigh == 0 ? t.left_block : t.right_block;
    mapping.assign(op_table.size(), std::vector<int>(old.size(), -1));
    std::vector<char> flag(leigh_table.size(), 0);
    for (size_t i = 0; i < op_table.size(); ++i)
        for (size_t j = 0; j < old.size(); ++j) {
            const std::vector<int> m = space_->MergeQuantumTable(op_table[i], leigh_table[old[j]]);
            for (size_t k = 0; k < leigh_table.size(); ++k)
                if (m == leigh_table[k]) flag[k] = 1;
        }
    std::vector<int> leigh_block;
    for (size_t i = 0; i < leigh_table.size(); ++i)
        if (flag[i]) {
            leigh_block.push_back((int)i);
            if ((int)leigh_block.size() == p_max_block_) break;
        }
    for (size_t i = 0; i < op_table.size(); ++i)
        for (size_t j = 0; j < old.size(); ++j) {
            const std::vector<int> m = space_->MergeQuantumTable(op_table[i], leigh_table[old[j]]);
            for (size_t k = 0; k < leigh_block.size(); ++k)
                if (m == leigh_table[leigh_block[k]]) {
                    mapping[i][j] = (int)k;
                    break;
                }
        }
    expan_.reset(new TensorLattice());
    TensorLattice& e = *expan_;
    e.physics_dim = t.physics_dim;
    std::vector<int> lb = leigh == 0 ? leigh_block : t.left_block;
    std::vector<int> rb = leigh == 1 ? leigh_block : t.right_block;
    DefineLatticeSectors(e, lb, rb, std::vector<int>(lb.size(), 1), std::vector<int>(rb.size(), 1));
    std::vector<int> li, ri, pi;
    for (int i = 0; i < (int)lb.size(); ++i)
        for (int j = 0; j < (int)rb.size(); ++j) {
            const int info = space_->CheckQuantumTable(site, lq[lb[i]], rq[rb[j]]);
            if (info != -1) {
                li.push_back(i);
                ri.push_back(j);
                pi.push_back(info);
            }
        }
    DefineLatticeBlocks(e, li, ri, pi, 1, 1, false);  // draws from rand() like the reference; values unused
    e.ket.set_shape_zero();
}

// ---------------------------------------------------------------------------
// subspace expansion: Left/RightExpanTensorContraction (real_tensor_contraction.cc:169-765)
// ---------------------------------------------------------------------------
int Engine::LeftExpanTensorContraction(int site, const std::vector<std::vector<int>>& mapping) {
    const TensorLattice& t = *lat_[site];
    const MpoHamiltonian& H = *ham_;
    const TensorContraction& con = *con_[site];
    TensorLattice& e = *expan_;
    const int lb = H.left_bond(site), rb = H.right_bond(site);
    auto same_left = t.ket.d.by_sector(0, t.nl());
    const bool compute = expansion_enabled(p_max_block_, p_max_dim_, p_noise_);
    xw_.active = true;
    xw_.compute = compute;
    // pass 1: which expanded right sectors receive something
    std::vector<char> exist(e.nr(), 0);
    for (int o1 = 0; o1 < lb; ++o1) {
        const BlockListDesc& Lo = con.L.desc.o[o1];
        for (int i = 0; i < Lo.count(); ++i) {
            const int idx = Lo.left[i], kdx = Lo.right[i];
            if (Lo.rows[i] == 0) continue;
            for (int pos : same_left[kdx]) {
                const int jdx = t.ket.d.right[pos];
                const int p2 = t.p(kdx, jdx);
                if (!H.MixedCheckZero(site, o1, p2)) continue;
                for (int o2 = 0; o2 < rb; ++o2) {
                    const int ldx = mapping[o2][jdx];
                    const int position = e.ket.d.find(idx, ldx);
                    if (ldx != -1 && position != -1 && H.w_nonzero(site, o1, o2, e.p(idx, ldx), p2)) exist[ldx] = 1;
                }
            }
        }
    }
    std::vector<int> keep;
    for (int i = 0; i < e.nr(); ++i)
        if (exist[i]) keep.push_back(i);
    std::vector<std::vector<int>> table(rb, std::vector<int>(t.nr(), -1));
    for (int o2 = 0; o2 < rb; ++o2)
        for (int r = 0; r < t.nr(); ++r) {
            const int ldx = mapping[o2][r];
            if (ldx == -1) continue;
            for (int i = 0; i < (int)keep.size(); ++i)
                if (e.right_block[ldx] == e.right_block[keep[i]]) {
                    table[o2][r] = i;
                    break;
                }
        }
    // rebuild the expanded lattice on the kept right sectors; blocks start empty
    std::vector<int> nrb, nphys((size_t)e.nl() * keep.size(), -1);
    for (size_t k = 0; k < keep.size(); ++k) {
        nrb.push_back(e.right_block[keep[k]]);
        for (int l = 0; l < e.nl(); ++l) nphys[(size_t)l * keep.size() + k] = e.p(l, keep[k]);
    }
    e.right_block = nrb;
    e.right_dim.assign(nrb.size(), 0);
    e.left_dim = t.left_dim;
    e.phys = nphys;
    BlockListDesc eb;
    for (int l = 0; l < e.nl(); ++l)
        for (int k = 0; k < e.nr(); ++k)
            if (e.p(l, k) != -1) eb.push(l, k, 0, 0);
    // pass 2: contributions, in the reference's order; rand() draws for each
    using First = ExpanWork::First;
    using Contrib = ExpanWork::Contrib;
    std::vector<First>& firsts = xw_.firsts;
    std::vector<std::vector<Contrib>>& contrib = xw_.contrib;
    contrib.assign(eb.count(), {});
    int64_t& first_size = xw_.first_size;
    for (int o1 = 0; o1 < lb; ++o1) {
        const BlockListDesc& Lo = con.L.desc.o[o1];
        for (int i = 0; i < Lo.count(); ++i) {
            const int idx = Lo.left[i], kdx = Lo.right[i];
            if (Lo.rows[i] == 0) continue;
            for (int pos : same_left[kdx]) {
                const int jdx = t.ket.d.right[pos];
                const int p2 = t.p(kdx, jdx);
                if (!H.MixedCheckZero(site, o1, p2)) continue;
                const int fm = Lo.rows[i], fk = Lo.cols[i], fn = t.ket.d.cols[pos];
                if (fk != t.ket.d.rows[pos]) return set_error(DMRG_E_ARG, "Matrix indeces do not match (expansion)");
                int d0 = fn;
                int d1 = (int)std::sqrt((double)fn) * t.physics_dim * t.physics_dim;
                d1 = std::min(std::max(d1, 1), 25);
                int fidx = -1;
                for (int o2 = 0; o2 < rb; ++o2) {
                    const int ldx = table[o2][jdx];
                    const int position = eb.find(idx, ldx);
                    if (ldx == -1 || position == -1) continue;
                    const int pe = nphys[(size_t)idx * keep.size() + ldx];
                    if (!H.w_nonzero(site, o1, o2, pe, p2)) continue;
                    const int64_t ro = add_random(d0, d1, H.wre(site, o1, o2, pe, p2), H.wim(site, o1, o2, pe, p2));
                    if (fidx < 0) {
                        fidx = (int)firsts.size();
                        firsts.push_back(First{con.L.desc.base[o1] + Lo.off[i], t.ket.d.off[pos], fm, fk, fn,
                                               first_size});
                        first_size += (int64_t)fm * fn;
                    }
                    contrib[position].push_back(Contrib{fidx, d0, d1, ro});
                }
            }
        }
    }
    // block shapes: rows of the L*K product, columns concatenated in order
    for (int b = 0; b < eb.count(); ++b) {
        int rows = 0, cols = 0;
        for (const Contrib& c : contrib[b]) {
            if (rows && rows != firsts[c.first].m)
                return set_error(DMRG_E_ARG, "row or column dimension is not match in ExpanMatrix");
            rows = firsts[c.first].m;
            cols += c.d1;
        }
        eb.rows[b] = rows;
        eb.cols[b] = cols;
    }
    // right_dim = widest block; empty blocks become zeros(left_dim[r], right_dim[r])
    // (the real reference indexes left_dim by r; the complex one by l, and pads
    // every other block with zero columns to right_dim, complex_tensor_contraction.cc:436-464)
    for (int r = 0; r < e.nr(); ++r) {
        e.right_dim[r] = 0;
        for (int l = 0; l < e.nl(); ++l) {
            const int b = eb.find(l, r);
            if (b != -1) e.right_dim[r] = std::max(e.right_dim[r], eb.cols[b]);
        }
        for (int l = 0; l < e.nl(); ++l) {
            const int b = eb.find(l, r);
            if (b == -1) continue;
            if (eb.rows[b] == 0) {
                const int li = cplx_ ? l : r;
                const int rr = li < (int)e.left_dim.size() ? e.left_dim[li] : 0;
                if ((int64_t)rr * e.right_dim[r] > 0) {
                    eb.rows[b] = rr;
                    eb.cols[b] = e.right_dim[r];
                }
            } else if (cplx_) {
                eb.cols[b] = e.right_dim[r];  // zero columns after the products
            }
        }
    }
    BlockListDesc& packed = xw_.packed;
    packed = BlockListDesc();
    for (int b = 0; b < eb.count(); ++b) packed.push(eb.left[b], eb.right[b], eb.rows[b], eb.cols[b]);
    return DMRG_OK;
}

int Engine::RightExpanTensorContraction(int site, const std::vector<std::vector<int>>& mapping) {
    const TensorLattice& t = *lat_[site];
    const MpoHamiltonian& H = *ham_;
    const TensorContraction& con = *con_[site];
    TensorLattice& e = *expan_;
    const int lb = H.left_bond(site), rb = H.right_bond(site);
    auto same_right = t.ket.d.by_sector(1, t.nr());
    const bool compute = expansion_enabled(p_max_block_, p_max_dim_, p_noise_);
    xw_.active = true;
    xw_.compute = compute;
    std::vector<char> exist(e.nl(), 0);
    for (int o2 = 0; o2 < rb; ++o2) {
        const BlockListDesc& Ro = con.R.desc.o[o2];
        for (int i = 0; i < Ro.count(); ++i) {
            const int kdx = Ro.left[i], idx = Ro.right[i];
            if (Ro.rows[i] == 0) continue;
            for (int pos : same_right[kdx]) {
                const int jdx = t.ket.d.left[pos];
                const int p2 = t.p(jdx, kdx);
                if (!H.RightCheckZero(site, o2, p2)) continue;
                for (int o1 = 0; o1 < lb; ++o1) {
                    const int ldx = mapping[o1][jdx];
                    const int position = e.ket.d.find(ldx, idx);
                    if (ldx != -1 && position != -1 && H.w_nonzero(site, o1, o2, e.p(ldx, idx), p2)) exist[ldx] = 1;
                }
            }
        }
    }
    std::vector<int> keep;
    for (int i = 0; i < e.nl(); ++i)
        if (exist[i]) keep.push_back(i);
    std::vector<std::vector<int>> table(lb, std::vector<int>(t.nl(), -1));
    for (int o1 = 0; o1 < lb; ++o1)
        for (int l = 0; l < t.nl(); ++l) {
            const int ldx = mapping[o1][l];
            if (ldx == -1) continue;
            for (int i = 0; i < (int)keep.size(); ++i)
                if (e.left_block[ldx] == e.left_block[keep[i]]) {
                    table[o1][l] = i;
                    break;
                }
        }
    std::vector<int> nlb, nphys(keep.size() * (size_t)e.nr(), -1);
    for (size_t k = 0; k < keep.size(); ++k) {
        nlb.push_back(e.left_block[keep[k]]);
        for (int r = 0; r < e.nr(); ++r) nphys[k * e.nr() + r] = e.p(keep[k], r);
    }
    e.left_block = nlb;
    e.left_dim.assign(nlb.size(), 0);
    e.right_dim = t.right_dim;
    e.phys = nphys;
    BlockListDesc eb;
    for (int l = 0; l < e.nl(); ++l)
        for (int r = 0; r < e.nr(); ++r)
            if (e.p(l, r) != -1) eb.push(l, r, 0, 0);
    using First = ExpanWork::First;
    using Contrib = ExpanWork::Contrib;
    std::vector<First>& firsts = xw_.firsts;
    std::vector<std::vector<Contrib>>& contrib = xw_.contrib;
    contrib.assign(eb.count(), {});
    int64_t& first_size = xw_.first_size;
    for (int o2 = 0; o2 < rb; ++o2) {
        const BlockListDesc& Ro = con.R.desc.o[o2];
        for (int i = 0; i < Ro.count(); ++i) {
            const int kdx = Ro.left[i], idx = Ro.right[i];
            if (Ro.rows[i] == 0) continue;
            for (int pos : same_right[kdx]) {
                const int jdx = t.ket.d.left[pos];
                const int p2 = t.p(jdx, kdx);
                if (!H.RightCheckZero(site, o2, p2)) continue;
                const int fm = t.ket.d.rows[pos], fk = t.ket.d.cols[pos], fn = Ro.cols[i];
                if (fk != Ro.rows[i]) return set_error(DMRG_E_ARG, "Matrix indeces do not match (expansion)");
                const int d1 = fm;
                int d0 = (int)std::sqrt((double)fm) * t.physics_dim * t.physics_dim;
                d0 = std::min(std::max(d0, 1), 25);
                int fidx = -1;
                for (int o1 = 0; o1 < lb; ++o1) {
                    const int ldx = table[o1][jdx];
                    const int position = eb.find(ldx, idx);
                    if (ldx == -1 || position == -1) continue;
                    const int pe = nphys[(size_t)ldx * e.nr() + idx];
                    if (!H.w_nonzero(site, o1, o2, pe, p2)) continue;
                    const int64_t ro = add_random(d0, d1, H.wre(site, o1, o2, pe, p2), H.wim(site, o1, o2, pe, p2));
                    if (fidx < 0) {
                        fidx = (int)firsts.size();
                        firsts.push_back(First{t.ket.d.off[pos], con.R.desc.base[o2] + Ro.off[i], fm, fk, fn,
                                               first_size});
                        first_size += (int64_t)fm * fn;
                    }
                    contrib[position].push_back(Contrib{fidx, d0, d1, ro});
                }
            }
        }
    }
    for (int b = 0; b < eb.count(); ++b) {
        int rows = 0, cols = 0;
        for (const Contrib& c : contrib[b]) {
            if (cols && cols != firsts[c.first].n)
                return set_error(DMRG_E_ARG, "row or column dimension is not match in ExpanMatrix");
            cols = firsts[c.first].n;
            rows += c.d0;
        }
        eb.rows[b] = rows;
        eb.cols[b] = cols;
    }
    for (int l = 0; l < e.nl(); ++l) {
        e.left_dim[l] = 0;
        for (int r = 0; r < e.nr(); ++r) {
            const int b = eb.find(l, r);
            if (b != -1) e.left_dim[l] = std::max(e.left_dim[l], eb.rows[b]);
        }
        for (int r = 0; r < e.nr(); ++r) {
            const int b = eb.find(l, r);
            if (b == -1) continue;
            if (eb.rows[b] == 0) {
                // the real reference builds zeros(left_dim[r], right_dim[r]) here, the
                // complex one zeros(left_dim[l], right_dim[r]) and pads every other
                // block with zero rows to left_dim[l] (complex_tensor_contraction.cc:752-781)
                const int li = cplx_ ? l : r;
                const int rr = li < (int)e.left_dim.size() ? e.left_dim[li] : 0;
                const int cc = e.right_dim[r];
                if ((int64_t)rr * cc > 0) {
                    eb.rows[b] = rr;
                    eb.cols[b] = cc;
                }
            } else if (cplx_) {
                eb.rows[b] = e.left_dim[l];  // zero rows after the products
            }
        }
    }
    BlockListDesc& packed = xw_.packed;
    packed = BlockListDesc();
    for (int b = 0; b < eb.count(); ++b) packed.push(eb.left[b], eb.right[b], eb.rows[b], eb.cols[b]);
    return DMRG_OK;
}

// The device half of the planned expansion: the expanded lattice's blocks, then
// F = L K (K R) per product and each block's column (row) ranges = noise * F Rand
// (Rand K R), in the reference's order of contributions.
int Engine::ExecuteExpanTensorNetwork() {
    if (!xw_.active) return DMRG_OK;
    if (!expan_) return set_error(DMRG_E_STATE, "expan_tensor_lattice is nullptr!");
    TensorLattice& e = *expan_;
    const BlockListDesc& packed = xw_.packed;
    e.ket = DevBlocks();
    e.ket.d = packed;
    DMRG_TRY(e.ket.alloc(st_, true, ew_));
    if (!xw_.compute || xw_.firsts.empty()) return DMRG_OK;  // rand() stream advanced; products unused
    const TensorLattice& t = *lat_[xw_.site];
    const TensorContraction& con = *con_[xw_.site];
    const std::vector<double>& rnd = xw_.rnd;
    const int64_t first_size = xw_.first_size;
    const int64_t rnd_size = (int64_t)rnd.size() / ew_;  // elements
    DMRG_TRY(scratch_.alloc((size_t)std::max<int64_t>(first_size, 1) * ew_ * sizeof(double)));
    DMRG_TRY(scratch2_.alloc(std::max<size_t>(rnd.size(), 1) * sizeof(double)));
    DMRG_CUDA_TRY(cudaMemcpyAsync(scratch2_.ptr, rnd.data(), rnd.size() * sizeof(double), cudaMemcpyHostToDevice, st_));
    // the same products in both fields: GemmSchedule (FP64) or ZGemmSchedule (complex)
    GemmSchedule sf, ss;
    ZGemmSchedule zf, zss;
    auto group = [&](bool second, int64_t c_off, int ldc, int m, int n) {
        if (cplx_) (second ? zss : zf).add_group(c_off, ldc, m, n);
        else (second ? ss : sf).add_group(c_off, ldc, m, n);
    };
    auto term = [&](bool second, int64_t a_off, int lda, int64_t b_off, int ldb, int k, double scale) {
        if (cplx_) (second ? zss : zf).add_term(a_off, lda, b_off, ldb, k, scale, 0.0);
        else (second ? ss : sf).add_term(a_off, lda, b_off, ldb, k, scale);
    };
    for (const ExpanWork::First& f : xw_.firsts) {
        group(false, f.off, f.n, f.m, f.n);
        term(false, f.a_off, f.k, f.b_off, f.n, f.k, 1.0);
    }
    for (int b = 0; b < packed.count(); ++b) {
        int at = 0;
        for (const ExpanWork::Contrib& c : xw_.contrib[b]) {
            const ExpanWork::First& f = xw_.firsts[c.first];
            if (xw_.leigh == 0) {  // columns [at, at + d1) of the block = (L K) * Rand
                group(true, packed.off[b] + at, packed.cols[b], f.m, c.d1);
                term(true, f.off, f.n, c.rnd, c.d1, c.d0, p_noise_);
                at += c.d1;
            } else {  // rows [at, at + d0) of the block = Rand * (K R)
                group(true, packed.off[b] + (int64_t)at * packed.cols[b], packed.cols[b], c.d0, f.n);
                term(true, c.rnd, c.d1, f.off, f.n, c.d1, p_noise_);
                at += c.d0;
            }
        }
    }
    const double* A1 = xw_.leigh == 0 ? con.L.ptr() : t.ket.ptr();
    const double* B1 = xw_.leigh == 0 ? t.ket.ptr() : con.R.ptr();
    const double* A2 = xw_.leigh == 0 ? scratch_.as<double>() : scratch2_.as<double>();
    const double* B2 = xw_.leigh == 0 ? scratch2_.as<double>() : scratch_.as<double>();
    const int64_t a1 = xw_.leigh == 0 ? con.L.desc.size : t.ket.d.size;
    const int64_t b1 = xw_.leigh == 0 ? t.ket.d.size : con.R.desc.size;
    const int64_t a2 = xw_.leigh == 0 ? first_size : rnd_size;
    const int64_t b2 = xw_.leigh == 0 ? rnd_size : first_size;
    if (cplx_) {
        DMRG_TRY(zf.check_bounds(a1, b1, first_size));
        DMRG_TRY(zss.check_bounds(a2, b2, packed.size));
        DMRG_TRY(zf.finalize(st_));
        DMRG_TRY(zss.finalize(st_));
        DMRG_TRY(launch_zgemm(zf, A1, B1, scratch_.as<double>(), false, st_));
        DMRG_TRY(launch_zgemm(zss, A2, B2, e.ket.ptr(), false, st_));
    } else {
        DMRG_TRY(sf.check_bounds(a1, b1, first_size));
        DMRG_TRY(ss.check_bounds(a2, b2, packed.size));
        DMRG_TRY(sf.finalize(64, 64, 16, st_));
        DMRG_TRY(ss.finalize(64, 64, 16, st_));
        DMRG_TRY(launch_gemm_f64(sf, A1, B1, scratch_.as<double>(), false, st_));
        DMRG_TRY(launch_gemm_f64(ss, A2, B2, e.ket.ptr(), false, st_));
    }
    DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
    return DMRG_OK;
}

// RealTensorNetwork::ExpanTensorNetwork (real_tensor_network.cc:116-140)
int Engine::ExpanTensorNetwork(int leigh, int site) {
    DMRG_TRY(PlanExpanTensorNetwork(leigh, site));
    return ExecuteExpanTensorNetwork();
}

int Engine::PlanExpanTensorNetwork(int leigh, int site) {
    std::vector<std::vector<int>> mapping;
    xw_ = ExpanWork();
    xw_.leigh = leigh;
    xw_.site = site;
    ComputeExpanTensorLattice((leigh + 1) % 2, site, mapping);
    if (leigh == 0 && site < n_ - 1) return LeftExpanTensorContraction(site, mapping);
    if (leigh == 1 && site > 0) return RightExpanTensorContraction(site, mapping);
    return DMRG_OK;
}

}  // namespace dmrg

// ---------------------------------------------------------------------------
// environments: RealTensorNetwork (real_tensor_network.cc) + contraction kernels
// ---------------------------------------------------------------------------
extern "C" {
int dmrg_env_create(dmrg_ctx_t, int, int, int, const int*, const dmrg_blocks_t*, int, int, int, const double*,
                    const dmrg_blocks_t*, int, dmrg_env_t*);
int dmrg_env_destroy(dmrg_env_t);
int dmrg_env_out_info(dmrg_env_t, int*, int64_t*);
int dmrg_env_out_blocks(dmrg_env_t, int, int, int*, int*, int*, int*, int*);
int dmrg_env_apply(dmrg_env_t, const double*, const double*, double*);
int dmrg_heff_create(dmrg_ctx_t, int, int, const int*, const dmrg_blocks_t*, int, int, int, const double*,
                     const dmrg_blocks_t*, const dmrg_blocks_t*, int, dmrg_heff_t*);
int dmrg_heff_destroy(dmrg_heff_t);
int dmrg_heff_set_env(dmrg_heff_t, const double*, const double*);
int dmrg_lanczos(dmrg_heff_t, double*, int, double, double, double*, int*);
int dmrg_heff_set_graph(dmrg_heff_t, int);
int dmrg_zenv_create(dmrg_ctx_t, int, int, int, const int*, const dmrg_blocks_t*, int, int, int, const double*,
                     const dmrg_blocks_t*, dmrg_env_t*);
int dmrg_zenv_apply(dmrg_env_t, const double*, const double*, double*);
int dmrg_zheff_create(dmrg_ctx_t, int, int, const int*, const dmrg_blocks_t*, int, int, int, const double*,
                      const dmrg_blocks_t*, const dmrg_blocks_t*, dmrg_zheff_t*);
int dmrg_zheff_destroy(dmrg_zheff_t);
int dmrg_zheff_set_env(dmrg_zheff_t, const double*, const double*);
int dmrg_zlanczos(dmrg_zheff_t, double*, int, double, double, double*, int*);
}

namespace dmrg {

static std::vector<dmrg_blocks_t> env_blocks(const EnvDesc& e) {
    std::vector<dmrg_blocks_t> v;
    for (const auto& b : e.o) v.push_back(as_blocks(b));
    if (v.empty()) v.push_back(dmrg_blocks_t{0, nullptr, nullptr, nullptr, nullptr});
    return v;
}

// RealTensorNetwork::DefineTensorNetwork + RealTensorContraction::DefineTensorContraction
// (real_tensor_contraction.cc:111-137): 1x1 identity blocks at both chain ends.
void Engine::DefineTensorNetwork() {
    auto define = [&](EnvData& env, int bond) {
        env.desc.o.assign(bond, BlockListDesc());
        for (int o = 0; o < bond; ++o) env.desc.o[o].push(0, 0, 1, 1);
        env.desc.rebase();
        env.buf.alloc((size_t)std::max<int64_t>(env.desc.size, 1) * ew_ * sizeof(double));
        std::vector<double> ones((size_t)env.desc.size * ew_, 1.0);
        if (cplx_)  // Complex(1, 0)
            for (size_t i = 1; i < ones.size(); i += 2) ones[i] = 0.0;
        if (!ones.empty())
            cudaMemcpyAsync(env.buf.ptr, ones.data(), ones.size() * sizeof(double), cudaMemcpyHostToDevice, st_);
        cudaStreamSynchronize(st_);
    };
    define(con_[0]->L, con_[0]->left_bond);
    define(con_[n_ - 1]->R, con_[n_ - 1]->right_bond);
}

// ResetTensorContraction: all blocks of one side become 0 x 0.
int Engine::ResetEnv(int leigh, int site) {
    EnvData& env = leigh == 0 ? con_[site]->L : con_[site]->R;
    for (auto& b : env.desc.o)
        for (int k = 0; k < b.count(); ++k) {
            b.rows[k] = b.cols[k] = 0;
            b.off[k] = 0;
        }
    for (auto& b : env.desc.o) b.size = 0;
    env.desc.rebase();
    env.buf.release();
    return DMRG_OK;
}

// RealTensorNetwork::ComputeTensorNetwork (real_tensor_network.cc:142-154)
int Engine::ComputeTensorNetwork(int leigh, int site) {
    TensorLattice& t = *lat_[site];
    const MpoHamiltonian& H = *ham_;
    const TensorContraction& src = *con_[site];
    TensorContraction& dst = *con_[leigh == 0 ? site + 1 : (site - 1 + n_ + 1) % (n_ + 1)];
    const EnvData& in = leigh == 0 ? src.L : src.R;
    EnvData& out = leigh == 0 ? dst.L : dst.R;
    std::vector<dmrg_blocks_t> ib = env_blocks(in.desc);
    dmrg_blocks_t kb = as_blocks(t.ket.d);
    dmrg_env_t e = nullptr;
    if (cplx_)  // ComplexTensorContraction::Left/RightComputeTensorContraction
        DMRG_TRY(dmrg_zenv_create(ctx_, leigh, t.nl(), t.nr(), t.phys.data(), &kb, H.physics_dim(site),
                                  H.left_bond(site), H.right_bond(site), H.values(site), ib.data(), &e));
    else
        DMRG_TRY(dmrg_env_create(ctx_, leigh, t.nl(), t.nr(), t.phys.data(), &kb, H.physics_dim(site),
                                 H.left_bond(site), H.right_bond(site), H.values(site), ib.data(), DMRG_PREC_FP64,
                                 &e));
    int bond = 0;
    int64_t size = 0;
    int rc = dmrg_env_out_info(e, &bond, &size);
    EnvDesc od;
    od.o.assign(bond, BlockListDesc());
    for (int o = 0; rc == DMRG_OK && o < bond; ++o) {
        int nb = 0;
        rc = dmrg_env_out_blocks(e, o, 0, &nb, nullptr, nullptr, nullptr, nullptr);
        std::vector<int> l(std::max(nb, 1)), r(std::max(nb, 1)), rr(std::max(nb, 1)), cc(std::max(nb, 1));
        if (rc == DMRG_OK) rc = dmrg_env_out_blocks(e, o, nb, &nb, l.data(), r.data(), rr.data(), cc.data());
        for (int k = 0; rc == DMRG_OK && k < nb; ++k) od.o[o].push(l[k], r[k], rr[k], cc[k]);
    }
    od.rebase();
    DeviceBuffer buf;
    if (rc == DMRG_OK) rc = buf.alloc((size_t)std::max<int64_t>(od.size, 1) * ew_ * sizeof(double));
    if (rc == DMRG_OK)
        rc = cplx_ ? dmrg_zenv_apply(e, t.ket.ptr(), in.ptr(), buf.as<double>())
                   : dmrg_env_apply(e, t.ket.ptr(), in.ptr(), buf.as<double>());
    if (rc == DMRG_OK) {
        cudaError_t err = cudaStreamSynchronize(st_);
        if (err != cudaSuccess) rc = set_error(DMRG_E_CUDA, "env update: %s", cudaGetErrorString(err));
    }
    dmrg_env_destroy(e);
    DMRG_TRY(rc);
    out.desc = od;
    std::swap(out.buf.ptr, buf.ptr);
    std::swap(out.buf.bytes, buf.bytes);
    return DMRG_OK;
}

// RealTensorLanczos::LanczosMethod through the device solver.
int Engine::LanczosMethod(int niter, int site, double& energy, int& dim) {
    TensorLattice& t = *lat_[site];
    const MpoHamiltonian& H = *ham_;
    const TensorContraction& c = *con_[site];
    std::vector<dmrg_blocks_t> lb = env_blocks(c.L.desc), rb = env_blocks(c.R.desc);
    dmrg_blocks_t kb = as_blocks(t.ket.d);
    if (cplx_) {  // ComplexTensorLanczos::LanczosMethod
        dmrg_zheff_t zh = nullptr;
        const double z0 = wall_time();
        DMRG_TRY(dmrg_zheff_create(ctx_, t.nl(), t.nr(), t.phys.data(), &kb, H.physics_dim(site), H.left_bond(site),
                                   H.right_bond(site), H.values(site), lb.data(), rb.data(), &zh));
        int rc = dmrg_zheff_set_env(zh, c.L.ptr(), c.R.ptr());
        const double z1 = wall_time();
        if (rc == DMRG_OK)
            rc = dmrg_zlanczos(zh, t.ket.ptr(), niter, opt_.lanczos_precision, opt_.zero_tolerance, &energy, &dim);
        const double z2 = wall_time();
        dmrg_zheff_destroy(zh);
        if (trace_)
            std::fprintf(trace_, "L %d %.3f %.3f %.3f %d %lld\n", site, 1e3 * (z1 - z0), 1e3 * (z2 - z1),
                         1e3 * (wall_time() - z2), dim, (long long)t.psi_dim());
        return rc;
    }
    dmrg_heff_t h = nullptr;
    const double t0 = wall_time();
    DMRG_TRY(dmrg_heff_create(ctx_, t.nl(), t.nr(), t.phys.data(), &kb, H.physics_dim(site), H.left_bond(site),
                              H.right_bond(site), H.values(site), lb.data(), rb.data(), opt_.precision, &h));
    if (opt_.lanczos_graph >= 0) dmrg_heff_set_graph(h, opt_.lanczos_graph);
    int rc = dmrg_heff_set_env(h, c.L.ptr(), c.R.ptr());
    const double t1 = wall_time();
    if (rc == DMRG_OK)
        rc = dmrg_lanczos(h, t.ket.ptr(), niter, opt_.lanczos_precision, opt_.zero_tolerance, &energy, &dim);
    const double t2 = wall_time();
    dmrg_heff_destroy(h);
    if (trace_)  // set-up / solve / tear-down times of this call
        std::fprintf(trace_, "L %d %.3f %.3f %.3f %d\n", site, 1e3 * (t1 - t0), 1e3 * (t2 - t1),
                     1e3 * (wall_time() - t2), dim);
    return rc;
}

// RealTensorRundmrg::Initialize (real_tensor_rundmrg.cc:247-287)
int Engine::Initialize() {
    DefineTensorNetwork();
    for (int i = n_ - 1; i > 0; --i) {
        DMRG_TRY(CanonicalTensorSpace(1, i));
        DMRG_TRY(ComputeTensorNetwork(1, i));
        DMRG_TRY(MergeTensorSpace(1, i - 1));
    }
    DMRG_TRY(CanonicalTensorSpace(1, 0));
    return DMRG_OK;
}

// RealTensorRundmrg::Run (real_tensor_rundmrg.cc:115-245)
int Engine::Run() {
    if (opt_.two_site) return RunTwoSite();
    const double t0 = wall_time();
    DMRG_TRY(Initialize());
    const int halves = opt_.stop_after_half_sweeps >= 0 ? std::min(opt_.stop_after_half_sweeps, num_sweep_)
                                                        : num_sweep_;
    for (int h = 0; h < halves; ++h) {
        half_sweep_ = h;
        const double th = wall_time();
        p_max_block_ = max_block_[h];
        p_max_dim_ = max_dim_[h];
        p_canpre_ = canpre_[h];
        p_noise_ = noise_[h];
        const bool l2r = (h % 2) == 0;
        std::array<double, kPhases> ph{};
        svd_sweeps_ = 0;
        // phase clock: every phase ends with its stream drained.  Each phase is
        // also an NVTX range (the names of dmrg_run_phases) for CUDA tools that
        // read them (ncu --nvtx); without such a tool the calls do nothing.
        static const char* const kPhaseName[kPhases] = {"lanczos", "expansion", "canonicalisation",
                                                         "environment", "match_merge"};
        double tp = wall_time();
        auto lap = [&](int k) -> int {
            DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
            nvtxRangePop();
            const double now = wall_time();
            ph[k] += now - tp;
            tp = now;
            if (k + 1 < kPhases) nvtxRangePushA(kPhaseName[k + 1]);
            return DMRG_OK;
        };
        if (l2r && opt_.verbose) std::printf("------------------------ sweep=%d ------------------------\n", h / 2);
        for (int k = 0; k < n_ - 1; ++k) {
            const int j = l2r ? k : n_ - 1 - k;
            const double ts = wall_time();
            int dim = 0;
            const int64_t psi_dim = lat_[j]->psi_dim();  // at the Lanczos call, like the reference's log
            tp = wall_time();
            nvtxRangePushA(kPhaseName[0]);
            // The expansion's host half (its lattice, its products and their
            // rand() matrices) depends only on block structures that the Lanczos
            // leaves as they are, so a second host thread plans it while the
            // device solves.  No CUDA call is made on that thread.
            int plan_rc = DMRG_OK;
            std::string plan_err;
            expan_.reset();  // a disabled expansion leaves its lattice: free its device blocks on this thread
            auto plan = [&] {
                plan_rc = PlanExpanTensorNetwork(l2r ? 0 : 1, j);
                if (plan_rc != DMRG_OK) plan_err = dmrg_last_error();
            };
            std::thread planner;
            try {
                planner = std::thread(plan);
            } catch (const std::system_error&) {
                plan();  // no thread to be had: plan first (same draws, same results)
            }
            const int lanczos_rc = LanczosMethod(num_iter_[h], j, energy_, dim);
            if (planner.joinable()) planner.join();
            DMRG_TRY(lanczos_rc);
            if (plan_rc != DMRG_OK) return set_error(plan_rc, "%s", plan_err.c_str());
            DMRG_TRY(lap(0));
            if (trace_) std::fprintf(trace_, "E %d %d P:%lld %.12e\n", lanczos_calls_, j, (long long)psi_dim, energy_);
            ++lanczos_calls_;
            DMRG_TRY(ResetEnv(l2r ? 1 : 0, j));
            DMRG_TRY(ExecuteExpanTensorNetwork());
            DMRG_TRY(ExpanTensorSpace(l2r ? 0 : 1, j));
            DMRG_TRY(lap(1));
            Trace("X", l2r ? 0 : 1, j);
            double disc = 0.0;
            tp = wall_time();
            DMRG_TRY(CanonicalTensorSpace(l2r ? 0 : 1, j, &disc));
            DMRG_TRY(lap(2));
            DMRG_TRY(ComputeTensorNetwork(l2r ? 0 : 1, j));
            DMRG_TRY(lap(3));
            const int nxt = l2r ? j + 1 : j - 1;
            DMRG_TRY(MatchTensorSpace(l2r ? 0 : 1, nxt));
            Trace("T", l2r ? 0 : 1, nxt);
            DMRG_TRY(MergeTensorSpace(l2r ? 0 : 1, nxt));
            DMRG_TRY(lap(4));
            records_.push_back(SweepRecord{h, j, l2r ? 0 : 1, energy_, dim, disc, psi_dim, wall_time() - ts});
        }
        half_energies_.push_back(energy_);
        half_seconds_.push_back(wall_time() - th);
        half_phases_.push_back(ph);
        half_svd_sweeps_.push_back(svd_sweeps_);
        if (opt_.verbose) std::printf("%s energy = %.12f\n", l2r ? "right" : "left", energy_);
        // after every full sweep, like the reference (:229-233)
        if (!l2r && cache_record_) DMRG_TRY(WriteTensorSpace(cache_name_ + "/" + record_name_));
    }
    if (opt_.verbose) std::printf("Total Time : %.12f s\n", wall_time() - t0);
    return DMRG_OK;
}

// ---------------------------------------------------------------------------
// checkpoint file: RealTensorSpace::WriteTensorSpace / ReadTensorSpace
// (real_tensor_space.cc:182-277), RealTensorLattice::Write/ReadTensorLattice
// (real_tensor_lattice.cc:218-300), RealMatrixBlock::Write/ReadMatrixBlock
// (real_matrix_block.cc:227-285), RealMatrix::Write/ReadMatrix
// (real_matrix.cc:139-180).  Native-endian binary, in this order:
//   int num_site, num_site + 1, num_site - 1, num_quantum;
//   int num_table[b] for the num_site + 1 bonds; int quantum_table[b][j][k];
//   per site: int physics_dim; int nl; (int left_block, int left_dim) x nl;
//     int nr; (int right_block, int right_dim) x nr; int physics_index[nl][nr];
//     int num_block; per block: int left, right, rows, cols, rows*cols;
//     double values[rows * cols] (row-major);
//   int max_block, max_dim; double canonical_precision, noise_factor.
// ---------------------------------------------------------------------------
namespace {
struct BinOut {
    std::FILE* f;
    bool ok = true;
    template <class T>
    void put(const T& v) { ok = ok && std::fwrite(&v, sizeof(T), 1, f) == 1; }
    void put_n(const double* v, size_t n) { ok = ok && (n == 0 || std::fwrite(v, sizeof(double), n, f) == n); }
};
struct BinIn {
    std::FILE* f;
    bool ok = true;
    template <class T>
    T get() {
        T v{};
        ok = ok && std::fread(&v, sizeof(T), 1, f) == 1;
        return v;
    }
    void get_n(double* v, size_t n) { ok = ok && (n == 0 || std::fread(v, sizeof(double), n, f) == n); }
};
}  // namespace

int Engine::WriteTensorSpace(const std::string& path) {
    if (cplx_) return set_error(DMRG_E_ARG, "checkpoints of complex runs are not supported");
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return set_error(DMRG_E_IO, "cannot open %s for writing", path.c_str());
    BinOut o{f};
    const int nq = space_->num_quantum();
    o.put(n_);
    o.put(n_ + 1);
    o.put(n_ - 1);
    o.put(nq);
    for (int b = 0; b <= n_; ++b) o.put((int)space_->table(b).size());
    for (int b = 0; b <= n_; ++b)
        for (const auto& row : space_->table(b))
            for (int k = 0; k < nq; ++k) o.put(row[k]);
    std::vector<double> host;
    int rc = DMRG_OK;
    for (int i = 0; i < n_ && o.ok && rc == DMRG_OK; ++i) {
        const TensorLattice& t = *lat_[i];
        o.put(t.physics_dim);
        o.put(t.nl());
        for (int l = 0; l < t.nl(); ++l) {
            o.put(t.left_block[l]);
            o.put(t.left_dim[l]);
        }
        o.put(t.nr());
        for (int r = 0; r < t.nr(); ++r) {
            o.put(t.right_block[r]);
            o.put(t.right_dim[r]);
        }
        for (int l = 0; l < t.nl(); ++l)
            for (int r = 0; r < t.nr(); ++r) o.put(t.p(l, r));
        const BlockListDesc& d = t.ket.d;
        host.assign((size_t)std::max<int64_t>(d.size, 0), 0.0);
        if (d.size > 0) {
            cudaError_t e = cudaMemcpyAsync(host.data(), t.ket.ptr(), (size_t)d.size * sizeof(double),
                                            cudaMemcpyDeviceToHost, st_);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
            if (e != cudaSuccess) rc = set_error(DMRG_E_CUDA, "site tensor download: %s", cudaGetErrorString(e));
        }
        o.put(d.count());
        for (int k = 0; k < d.count() && rc == DMRG_OK; ++k) {
            o.put(d.left[k]);
            o.put(d.right[k]);
            o.put(d.rows[k]);
            o.put(d.cols[k]);
            o.put(d.rows[k] * d.cols[k]);
            o.put_n(host.data() + d.off[k], (size_t)d.rows[k] * d.cols[k]);
        }
    }
    o.put(p_max_block_);
    o.put(p_max_dim_);
    o.put(p_canpre_);
    o.put(p_noise_);
    const bool closed = std::fclose(f) == 0;
    DMRG_TRY(rc);
    if (!o.ok || !closed) return set_error(DMRG_E_IO, "write to %s failed", path.c_str());
    return DMRG_OK;
}

int Engine::ReadTensorSpace(const std::string& path) {
    if (cplx_) return set_error(DMRG_E_ARG, "checkpoints of complex runs are not supported");
    std::FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return set_error(DMRG_E_IO, "cannot open %s", path.c_str());
    BinIn in{f};
    auto fail = [&](const char* what) {
        std::fclose(f);
        return set_error(DMRG_E_IO, "%s: %s", path.c_str(), what);
    };
    const int nq = space_->num_quantum();
    const int ns = in.get<int>(), nspp = in.get<int>(), nsmm = in.get<int>(), fq = in.get<int>();
    if (!in.ok || ns != n_ || nspp != n_ + 1 || nsmm != n_ - 1 || fq != nq)
        return fail("number of sites or quantum numbers differs from the model");
    std::vector<int> ntab(n_ + 1);
    for (int b = 0; b <= n_; ++b) ntab[b] = in.get<int>();
    for (int b = 0; b <= n_ && in.ok; ++b) {
        if (ntab[b] != (int)space_->table(b).size()) return fail("quantum table differs from the model");
        for (int j = 0; j < ntab[b]; ++j)
            for (int k = 0; k < nq; ++k)
                if (in.get<int>() != space_->table(b)[j][k]) return fail("quantum table differs from the model");
    }
    std::vector<double> host;
    for (int i = 0; i < n_; ++i) {
        TensorLattice& t = *lat_[i];
        const int pd = in.get<int>();
        const int nl = in.get<int>();
        if (!in.ok || pd != space_->physics_dim() || nl < 0 || nl > 1 << 20) return fail("malformed site header");
        std::vector<int> lb(nl), ld(nl);
        for (int l = 0; l < nl; ++l) {
            lb[l] = in.get<int>();
            ld[l] = in.get<int>();
        }
        const int nr = in.get<int>();
        if (!in.ok || nr < 0 || nr > 1 << 20) return fail("malformed site header");
        std::vector<int> rb(nr), rd(nr);
        for (int r = 0; r < nr; ++r) {
            rb[r] = in.get<int>();
            rd[r] = in.get<int>();
        }
        for (int l = 0; l < nl; ++l)
            if (lb[l] < 0 || lb[l] >= ntab[i] || ld[l] < 0) return fail("left sector out of range");
        for (int r = 0; r < nr; ++r)
            if (rb[r] < 0 || rb[r] >= ntab[i + 1] || rd[r] < 0) return fail("right sector out of range");
        DefineLatticeSectors(t, lb, rb, ld, rd);
        t.physics_dim = pd;
        for (int l = 0; l < nl; ++l)
            for (int r = 0; r < nr; ++r) {
                const int p = in.get<int>();
                if (p < -1 || p >= pd) return fail("physics index out of range");
                t.phys[(size_t)l * nr + r] = p;
            }
        const int nb = in.get<int>();
        if (!in.ok || nb < 0 || nb > nl * nr) return fail("malformed block list");
        DevBlocks ket;
        host.clear();
        for (int k = 0; k < nb; ++k) {
            const int l = in.get<int>(), r = in.get<int>(), rows = in.get<int>(), cols = in.get<int>();
            const int total = in.get<int>();
            if (!in.ok || l < 0 || l >= nl || r < 0 || r >= nr || rows < 0 || cols < 0 ||
                (int64_t)rows * cols != total || t.p(l, r) < 0)
                return fail("malformed block");
            ket.d.push(l, r, rows, cols);
            const size_t at = host.size();
            host.resize(at + (size_t)total);
            in.get_n(host.data() + at, (size_t)total);
        }
        if (!in.ok) return fail("truncated block values");
        t.has_canonical = false;
        t.match_dim.clear();
        int rc = ket.alloc(st_, false);
        if (rc == DMRG_OK && !host.empty()) {
            cudaError_t e = cudaMemcpyAsync(ket.ptr(), host.data(), host.size() * sizeof(double),
                                            cudaMemcpyHostToDevice, st_);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st_);
            if (e != cudaSuccess) rc = set_error(DMRG_E_CUDA, "site tensor upload: %s", cudaGetErrorString(e));
        }
        if (rc != DMRG_OK) {
            std::fclose(f);
            return rc;
        }
        t.ket = std::move(ket);
    }
    p_max_block_ = in.get<int>();
    p_max_dim_ = in.get<int>();
    p_canpre_ = in.get<double>();
    p_noise_ = in.get<double>();
    if (!in.ok) return fail("truncated parameters");
    std::fclose(f);
    return DMRG_OK;
}

}  // namespace dmrg
