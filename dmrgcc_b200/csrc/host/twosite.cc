// Two-site DMRG sweep on the device (Engine::RunTwoSite).
//
// The reference sweeps one site at a time and grows the bond by a randomised
// subspace expansion (RealTensorRundmrg::Run, src/dmrg/realdmrg/
// real_tensor_rundmrg.cc:115-245).  This mode optimises two neighbouring sites
// at once instead, with no expansion: per bond (j, j+1)
//   1. Theta = K_j K_{j+1}, on every (left, middle, right) sector triple the
//      quantum numbers allow (middle sectors from the bond's full quantum table,
//      so sectors absent from the current MPS can appear); blocks without a
//      product start at zero;
//   2. the Lanczos ground state of the two-site H_eff = L_j (W_j W_{j+1}) R_{j+1}
//      (dmrg_heff_create_blocks: the single-site operator with a combined
//      physics index and the two-site MPO);
//   3. per middle sector, the SVD of Theta's sector matrix; a global truncation
//      to the sweep table's maxm (and canpre) sets the new bond;
//   4. left to right: K_j = U, K_{j+1} = S V^T, then L_{j+1}; right to left:
//      K_j = U S, K_{j+1} = V^T, then R_j (the single-site environment
//      updates, RealTensorContraction::Left/RightComputeTensorContraction).
// Left to right the bonds are visited j = 0 .. n-2, right to left n-2 .. 0.
// The sweep table's maxm, niter and canpre apply per half-sweep; maxb and the
// noise column are not used (no expansion).  The starting MPS, its right
// canonicalisation and the environments are those of the single-site engine
// (RealTensorRundmrg::Initialize, :247-287).
#include <sys/time.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>

#include "gemm.cuh"
#include "host/engine.h"
#include "ortho.cuh"
#include "twosite.cuh"

extern "C" {
int dmrg_heff_create_blocks(dmrg_ctx_t, int, int, const int*, const dmrg_blocks_t*, int, int, int, const double*,
                            const dmrg_blocks_t*, const dmrg_blocks_t*, int, dmrg_heff_t*);
int dmrg_heff_destroy(dmrg_heff_t);
int dmrg_heff_set_env(dmrg_heff_t, const double*, const double*);
int dmrg_lanczos(dmrg_heff_t, double*, int, double, double, double*, int*);
}

namespace dmrg {

namespace {

double now_s() {
    timeval t;
    gettimeofday(&t, nullptr);
    return t.tv_sec + t.tv_usec * 1e-6;
}

dmrg_blocks_t list_of(const BlockListDesc& b) {
    return dmrg_blocks_t{b.count(), b.left.data(), b.right.data(), b.rows.data(), b.cols.data()};
}

std::vector<dmrg_blocks_t> lists_of(const EnvDesc& e) {
    std::vector<dmrg_blocks_t> v;
    for (const auto& b : e.o) v.push_back(list_of(b));
    if (v.empty()) v.push_back(dmrg_blocks_t{0, nullptr, nullptr, nullptr, nullptr});
    return v;
}

// Named-array container (.nac: int32 name length, name, dtype char 'i' | 'd',
// int32 ndim, int32 shape[ndim], little-endian data), the format the Python
// side reads (dmrgcc_b200/problem.py).
struct NacOut {
    std::FILE* f;
    void header(const std::string& name, char dt, int n) {
        const int len = (int)name.size(), nd = 1;
        std::fwrite(&len, 4, 1, f);
        std::fwrite(name.data(), 1, name.size(), f);
        std::fwrite(&dt, 1, 1, f);
        std::fwrite(&nd, 4, 1, f);
        std::fwrite(&n, 4, 1, f);
    }
    void ints(const std::string& name, const std::vector<int>& v) {
        header(name, 'i', (int)v.size());
        if (!v.empty()) std::fwrite(v.data(), 4, v.size(), f);
    }
    void doubles(const std::string& name, const std::vector<double>& v) {
        header(name, 'd', (int)v.size());
        if (!v.empty()) std::fwrite(v.data(), 8, v.size(), f);
    }
    void blocks(const std::string& p, const BlockListDesc& b) {
        ints(p + ".left", b.left);
        ints(p + ".right", b.right);
        ints(p + ".rows", b.rows);
        ints(p + ".cols", b.cols);
    }
};

// DMRG_TWOSITE_DUMP=<half-sweep>:<bond>:<path>: the block structure (no values)
// of that step's two-site H_eff problem, for benchmarks of the two-site matvec.
void dump_twosite(const std::string& path, int nl, int nr, const std::vector<int>& ldim,
                  const std::vector<int>& rdim, const BlockListDesc& theta, const std::vector<int>& bphys, int D,
                  int lb, int rb, const std::vector<double>& w2, const EnvDesc& L, const EnvDesc& R) {
    std::FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return;
    NacOut o{f};
    o.ints("lattice.left_dim", ldim);
    o.ints("lattice.right_dim", rdim);
    (void)nl;
    (void)nr;
    o.blocks("lattice.ket", theta);
    o.ints("lattice.block_phys", bphys);
    o.ints("op.dims", {D, lb, rb});
    o.doubles("op.W", w2);
    for (int i = 0; i < lb; ++i) o.blocks("L." + std::to_string(i), L.o[i]);
    for (int i = 0; i < rb; ++i) o.blocks("R." + std::to_string(i), R.o[i]);
    std::fclose(f);
}

}  // namespace

// W2[o1][o2][p1 d + p2][q1 d + q2] = sum_o W_j[o1][o](p1, q1) W_{j+1}[o][o2](p2, q2)
std::vector<double> two_site_mpo(const RealTensorOperator& a, const RealTensorOperator& b) {
    const int d = a.get_physics_dim(), lb = a.get_left_bond(), mb = a.get_right_bond(), rb = b.get_right_bond();
    const int D = d * d;
    std::vector<double> w2((size_t)lb * rb * D * D, 0.0);
    for (int o1 = 0; o1 < lb; ++o1)
        for (int o = 0; o < mb; ++o)
            for (int p1 = 0; p1 < d; ++p1)
                for (int q1 = 0; q1 < d; ++q1) {
                    const double wa = a.w(o1, o, p1, q1);
                    if (wa == 0.0) continue;
                    for (int o2 = 0; o2 < rb; ++o2)
                        for (int p2 = 0; p2 < d; ++p2)
                            for (int q2 = 0; q2 < d; ++q2) {
                                const double wb = b.w(o, o2, p2, q2);
                                if (wb == 0.0) continue;
                                w2[(((size_t)o1 * rb + o2) * D + p1 * d + p2) * D + q1 * d + q2] += wa * wb;
                            }
                }
    return w2;
}

int Engine::TwoSiteStep(bool l2r, int j, int niter, double& energy, int& dim, double& discarded,
                        int64_t& theta_dim, std::array<double, kPhases>& ph) {
    TensorLattice& A = *lat_[j];
    TensorLattice& B = *lat_[j + 1];
    const RealTensorHamiltonian& rh = static_cast<const RealTensorHamiltonian&>(*ham_);  // two-site runs are real
    const RealTensorOperator& Wa = rh.get_tensor_hamiltonian(j);
    const RealTensorOperator& Wb = rh.get_tensor_hamiltonian(j + 1);
    const int d = Wa.get_physics_dim();
    const auto& lq = space_->table(j);
    const auto& mq = space_->table(j + 1);
    const auto& rq = space_->table(j + 2);
    double tp = now_s();
    auto lap = [&](int k) -> int {
        DMRG_CUDA_TRY(cudaStreamSynchronize(st_));
        const double t = now_s();
        ph[k] += t - tp;
        tp = t;
        return DMRG_OK;
    };

    // ---- 1. Theta's blocks: per candidate middle sector c, every allowed (k, l)
    struct Mid {
        int c;                         // quantum-table index of the middle sector
        std::vector<int> ks, p1, row0; // left sectors, their physics index, first row in M_c
        std::vector<int> ls, p2, col0;
        int m = 0, n = 0;
    };
    std::vector<Mid> mids;
    for (int c = 0; c < (int)mq.size(); ++c) {
        Mid M;
        M.c = c;
        for (int k = 0; k < A.nl(); ++k) {
            const int p = space_->CheckQuantumTable(j, lq[A.left_block[k]], mq[c]);
            if (p == -1) continue;
            M.ks.push_back(k);
            M.p1.push_back(p);
            M.row0.push_back(M.m);
            M.m += A.left_dim[k];
        }
        for (int l = 0; l < B.nr(); ++l) {
            const int p = space_->CheckQuantumTable(j + 1, mq[c], rq[B.right_block[l]]);
            if (p == -1) continue;
            M.ls.push_back(l);
            M.p2.push_back(p);
            M.col0.push_back(M.n);
            M.n += B.right_dim[l];
        }
        if (!M.ks.empty() && !M.ls.empty()) mids.push_back(std::move(M));
    }
    BlockListDesc theta;
    std::vector<int> bphys;
    std::vector<SplitBlock> split;
    GemmSchedule prod;
    for (int s = 0; s < (int)mids.size(); ++s) {
        const Mid& M = mids[s];
        const int m_old = std::find(A.right_block.begin(), A.right_block.end(), M.c) - A.right_block.begin();
        const bool exists = m_old < A.nr() && m_old < B.nl() && B.left_block[m_old] == M.c;
        for (size_t a = 0; a < M.ks.size(); ++a)
            for (size_t b = 0; b < M.ls.size(); ++b) {
                const int k = M.ks[a], l = M.ls[b];
                const int pos = theta.count();
                theta.push(k, l, A.left_dim[k], B.right_dim[l]);
                bphys.push_back(M.p1[a] * d + M.p2[b]);
                split.push_back(SplitBlock{theta.off[pos], theta.rows[pos], theta.cols[pos], s, M.row0[a], M.col0[b]});
                if (!exists) continue;
                const int ka = A.ket.d.find(k, m_old), kb = B.ket.d.find(m_old, l);
                if (ka < 0 || kb < 0 || theta.rows[pos] == 0 || theta.cols[pos] == 0) continue;
                const int inner = A.ket.d.cols[ka];
                if (inner == 0) continue;
                if (A.ket.d.rows[ka] != theta.rows[pos] || B.ket.d.cols[kb] != theta.cols[pos] ||
                    B.ket.d.rows[kb] != inner)
                    return set_error(DMRG_E_ARG, "two-site merge: block shapes of sites %d, %d disagree", j, j + 1);
                prod.add_group(theta.off[pos], theta.cols[pos], theta.rows[pos], theta.cols[pos]);
                prod.add_term(A.ket.d.off[ka], inner, B.ket.d.off[kb], theta.cols[pos], inner, 1.0);
            }
    }
    theta_dim = theta.size;
    if (theta.size == 0) return set_error(DMRG_E_STATE, "two-site tensor at bond %d has no allowed block", j);
    DevBlocks th;
    th.d = theta;
    DMRG_TRY(th.alloc(st_, true));
    DMRG_TRY(prod.check_bounds(A.ket.d.size, B.ket.d.size, theta.size));
    DMRG_TRY(prod.finalize(64, 64, 16, st_));
    DMRG_TRY(launch_gemm_f64(prod, A.ket.ptr(), B.ket.ptr(), th.ptr(), false, st_));
    DMRG_TRY(norm_.alloc(8 * sizeof(double)));
    const int vb = (int)std::min<int64_t>((theta.size + 255) / 256, 2 * ctx_->num_sms);
    DMRG_TRY(vec_normalize(th.ptr(), theta.size, norm_.as<double>(), rs_, vb, st_));
    DMRG_TRY(lap(4));

    // ---- 2. two-site Lanczos
    const std::vector<double> w2 = two_site_mpo(Wa, Wb);
    const TensorContraction& cl = *con_[j];
    const TensorContraction& cr = *con_[j + 1];
    std::vector<dmrg_blocks_t> lb = lists_of(cl.L.desc), rb = lists_of(cr.R.desc);
    dmrg_blocks_t tb = list_of(theta);
    if (const char* dump = std::getenv("DMRG_TWOSITE_DUMP")) {
        int hs = -1, bond = -1, used = 0;
        if (std::sscanf(dump, "%d:%d:%n", &hs, &bond, &used) == 2 && hs == half_sweep_ && bond == j)
            dump_twosite(dump + used, A.nl(), B.nr(), A.left_dim, B.right_dim, theta, bphys, d * d,
                         Wa.get_left_bond(), Wb.get_right_bond(), w2, cl.L.desc, cr.R.desc);
    }
    dmrg_heff_t h = nullptr;
    DMRG_TRY(dmrg_heff_create_blocks(ctx_, A.nl(), B.nr(), bphys.data(), &tb, d * d, Wa.get_left_bond(),
                                     Wb.get_right_bond(), w2.data(), lb.data(), rb.data(), opt_.precision, &h));
    int rc = dmrg_heff_set_env(h, cl.L.ptr(), cr.R.ptr());
    if (rc == DMRG_OK)
        rc = dmrg_lanczos(h, th.ptr(), niter, opt_.lanczos_precision, opt_.zero_tolerance, &energy, &dim);
    dmrg_heff_destroy(h);
    DMRG_TRY(rc);
    DMRG_TRY(lap(0));

    // ---- 3. per-middle-sector SVD and truncation
    std::vector<int> sm(mids.size()), sn(mids.size());
    for (size_t s = 0; s < mids.size(); ++s) {
        sm[s] = mids[s].m;
        sn[s] = mids[s].n;
    }
    BatchedSvd svd;
    DMRG_TRY(svd.plan(sm, sn, st_));
    DeviceBuffer d_split, d_writes;
    DMRG_TRY(twosite_gather(svd, svd.index, th.ptr(), split, d_split, st_));
    int sweeps = 0;
    if (!svd.probs.empty()) DMRG_TRY(svd.run(st_, &sweeps));
    svd_sweeps_ += sweeps;
    std::vector<std::vector<double>> sv;
    DMRG_TRY(svd.singular_values(sv, st_));
    const std::vector<int> t = truncate_twosite(p_max_dim_, p_canpre_, sv);
    double all = 0.0, kept = 0.0;
    for (size_t s = 0; s < sv.size(); ++s)
        for (size_t i = 0; i < sv[s].size(); ++i) {
            all += sv[s][i] * sv[s][i];
            if ((int)i < t[s]) kept += sv[s][i] * sv[s][i];
        }
    discarded = std::max(0.0, all - kept);

    // ---- 4. the two new site tensors
    std::vector<int> keep;  // kept middle sectors (batch index), quantum-table order
    for (int s = 0; s < (int)mids.size(); ++s)
        if (t[s] > 0) keep.push_back(s);
    if (keep.empty()) return set_error(DMRG_E_NUMERIC, "two-site truncation at bond %d kept nothing", j);
    std::vector<int> mid_block, mid_dim;
    for (int s : keep) {
        mid_block.push_back(mids[s].c);
        mid_dim.push_back(t[s]);
    }
    const int nk = (int)keep.size();
    DevBlocks na, nb;
    std::vector<int> aphys((size_t)A.nl() * nk, -1), bphys2((size_t)nk * B.nr(), -1);
    std::vector<SplitWrite> writes;
    for (int k = 0; k < A.nl(); ++k)
        for (int q = 0; q < nk; ++q) {
            const Mid& M = mids[keep[q]];
            const auto it = std::find(M.ks.begin(), M.ks.end(), k);
            if (it == M.ks.end()) continue;
            const size_t a = it - M.ks.begin();
            aphys[(size_t)k * nk + q] = M.p1[a];
            na.d.push(k, q, A.left_dim[k], t[keep[q]]);
            const int pos = na.d.count() - 1;
            writes.push_back(SplitWrite{na.d.off[pos], na.d.rows[pos], na.d.cols[pos], keep[q], M.row0[a], 0, -1, -1});
        }
    std::vector<SplitWrite> writes_b;
    for (int q = 0; q < nk; ++q) {
        const Mid& M = mids[keep[q]];
        for (int l = 0; l < B.nr(); ++l) {
            const auto it = std::find(M.ls.begin(), M.ls.end(), l);
            if (it == M.ls.end()) continue;
            const size_t b = it - M.ls.begin();
            bphys2[(size_t)q * B.nr() + l] = M.p2[b];
            nb.d.push(q, l, t[keep[q]], B.right_dim[l]);
            const int pos = nb.d.count() - 1;
            writes_b.push_back(SplitWrite{nb.d.off[pos], nb.d.rows[pos], nb.d.cols[pos], keep[q], M.col0[b], 1, -1, -1});
        }
    }
    writes.insert(writes.end(), writes_b.begin(), writes_b.end());
    // the canonical factor (U left to right, V^T right to left) orthonormal: where
    // it is the working matrix's normalised columns, orthonormalise them and take
    // the other factor as the projection of M_c on them
    KetOrtho ortho;
    DeviceBuffer d_a, d_p;
    std::vector<int64_t> p_of(svd.probs.size(), -1);
    {
        std::vector<int> kept(svd.probs.size(), 0);
        std::vector<std::vector<double>> svp(svd.probs.size());
        for (int s : keep) {
            const int pi = svd.index[s];
            if (pi < 0) continue;
            const SvdProblem& p = svd.probs[pi];
            const bool wside = l2r ? !p.transposed : p.transposed != 0;
            if (!wside) continue;
            kept[pi] = t[s];
            svp[pi] = sv[s];
        }
        DMRG_TRY(ortho.plan(svd, kept, svp, st_, ctx_->num_sms));
        if (!ortho.empty()) {
            int64_t wsz = 0, psz = 0;
            for (const SvdProblem& p : svd.probs) wsz += (int64_t)p.rows * p.cols;
            GemmSchedule sp;
            sp.tb = true;
            for (int pi = 0; pi < (int)svd.probs.size(); ++pi) {
                const int64_t ko = ortho.k_off(pi);
                if (ko < 0) continue;
                const SvdProblem& p = svd.probs[pi];
                const int tk = kept[pi];
                p_of[pi] = psz;
                if (l2r) {  // S V^T = K^T M (t x n); M column-major (W layout) is the transposed B
                    sp.add_group(psz, p.n, tk, p.n);
                    sp.add_term(ko, p.rows, p.w_off, p.rows, p.rows, 1.0);
                    psz += (int64_t)tk * p.n;
                } else {    // U S = M K (m x t); M^T column-major = M row-major (ld n); K the transposed B
                    sp.add_group(psz, tk, p.m, tk);
                    sp.add_term(p.w_off, p.rows, ko, p.rows, p.rows, 1.0);
                    psz += (int64_t)p.m * tk;
                }
            }
            DMRG_TRY(d_a.alloc(std::max<int64_t>(wsz, 1) * sizeof(double)));
            DMRG_TRY(d_p.alloc(std::max<int64_t>(psz, 1) * sizeof(double)));
            if (l2r)
                DMRG_TRY(sp.check_bounds(ortho.k_size(), wsz, psz));
            else
                DMRG_TRY(sp.check_bounds(wsz, ortho.k_size(), psz));
            DMRG_TRY(sp.finalize(64, 64, 16, st_, ctx_->num_sms));
            DeviceBuffer d_split2;
            DMRG_TRY(twosite_gather(svd, svd.index, th.ptr(), split, d_split2, st_, d_a.as<double>()));
            DMRG_TRY(ortho.run(svd, st_));
            if (l2r)
                DMRG_TRY(launch_gemm_f64(sp, ortho.k(), d_a.as<double>(), d_p.as<double>(), false, st_));
            else
                DMRG_TRY(launch_gemm_f64(sp, d_a.as<double>(), ortho.k(), d_p.as<double>(), false, st_));
            const int canonical_part = l2r ? 0 : 1;
            for (SplitWrite& w : writes) {
                const int pi = svd.index[w.sector];
                if (pi < 0 || ortho.k_off(pi) < 0) continue;
                if (w.part == canonical_part)
                    w.k_off = ortho.k_off(pi);
                else
                    w.p_off = p_of[pi];
            }
        }
    }
    DMRG_TRY(na.alloc(st_, false));
    DMRG_TRY(nb.alloc(st_, false));
    DMRG_TRY(twosite_write(svd, svd.index, writes, d_writes, na.ptr(), nb.ptr(), !l2r, st_, ortho.k(), d_p.as<double>()));
    A.ket = std::move(na);
    A.right_block = mid_block;
    A.right_dim = mid_dim;
    A.phys = aphys;
    A.has_canonical = false;
    B.ket = std::move(nb);
    B.left_block = mid_block;
    B.left_dim = mid_dim;
    B.phys = bphys2;
    B.has_canonical = false;
    DMRG_TRY(lap(2));

    // ---- 5. the environment on the side the sweep moves away from
    if (l2r) DMRG_TRY(ComputeTensorNetwork(0, j));
    else DMRG_TRY(ComputeTensorNetwork(1, j + 1));
    DMRG_TRY(lap(3));
    return DMRG_OK;
}

int Engine::RunTwoSite() {
    const double t0 = now_s();
    DMRG_TRY(Initialize());
    if (n_ < 2) return set_error(DMRG_E_ARG, "two-site sweeps need at least two sites");
    const int halves = opt_.stop_after_half_sweeps >= 0 ? std::min(opt_.stop_after_half_sweeps, num_sweep_)
                                                        : num_sweep_;
    for (int hs = 0; hs < halves; ++hs) {
        half_sweep_ = hs;
        const double th = now_s();
        p_max_block_ = max_block_[hs];
        p_max_dim_ = max_dim_[hs];
        p_canpre_ = canpre_[hs];
        p_noise_ = noise_[hs];
        const bool l2r = (hs % 2) == 0;
        std::array<double, kPhases> ph{};
        svd_sweeps_ = 0;
        if (l2r && opt_.verbose) std::printf("------------------------ sweep=%d ------------------------\n", hs / 2);
        for (int k = 0; k < n_ - 1; ++k) {
            const int j = l2r ? k : n_ - 2 - k;
            const double ts = now_s();
            int dim = 0;
            double disc = 0.0;
            int64_t tdim = 0;
            DMRG_TRY(TwoSiteStep(l2r, j, num_iter_[hs], energy_, dim, disc, tdim, ph));
            ++lanczos_calls_;
            records_.push_back(SweepRecord{hs, j, l2r ? 0 : 1, energy_, dim, disc, tdim, now_s() - ts});
        }
        half_energies_.push_back(energy_);
        half_seconds_.push_back(now_s() - th);
        half_phases_.push_back(ph);
        half_svd_sweeps_.push_back(svd_sweeps_);
        if (opt_.verbose) std::printf("%s energy = %.12f\n", l2r ? "right" : "left", energy_);
    }
    if (opt_.verbose) std::printf("Total Time : %.12f s\n", now_s() - t0);
    return DMRG_OK;
}

}  // namespace dmrg
