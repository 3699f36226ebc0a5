// The complex path's canonicalisation: ComplexTensorLattice::Left/Right
// CanonicalTensorLattice (src/dmrg/complexdmrg/complex_tensor_lattice.cc, per
// sector a thin SVD by zgesdd, ComplexMatrix::SVDMatrix,
// src/tensor/complex_matrix.cc:601-638, then ComputeTruncateDim).
//
// Each complex sector matrix A = Ar + i Ai (m x n, blocks stacked as in canon.cu)
// goes through the real batched Jacobi SVD as its real form
//     [ Ar  -Ai ]
//     [ Ai   Ar ]   (2m x 2n),
// whose singular values are those of A, each twice, with singular vectors
// [x; y] <-> x + i y: a real singular pair (u, v) of the real form gives the
// complex triplet (sigma, x_u + i y_u, x_v + i y_v) of A, and the two real
// vectors of one complex value differ by a factor i.  The complex triplets are
// recovered on the host: runs of equal singular values (to 1e-9 of the
// largest) are one complex eigenspace, in which the real columns, taken as
// complex vectors of the side that becomes the new ket (U for a left, V for a
// right canonicalisation) and first orthogonalised against every vector kept
// so far, are taken in order by Gram-Schmidt with complex coefficients whenever
// more than half a vector's norm remains, until the run's complex dimension
// (half its length) is reached; a degenerate run that falls short is filled
// with the largest remainders.  Truncation is the reference's rule on the
// complex singular values; the new ket takes U (left) or V^H (right) rows, the
// canonical tensor the projection U^H A = S V^H or A V = U S, like the
// reference.
// The signs (phases) of singular vectors are free, as with zgesdd; only
// gauge-invariant products are comparable.
#include <algorithm>
#include <cmath>
#include <complex>

#include "blocksparse.h"
#include "svd.cuh"
#include "truncate.h"

using namespace dmrg;
using cplx = std::complex<double>;

namespace {

struct ZCopyTask {
    int64_t blk_off;  // complex elements
    int rows, cols;
    int problem;
    int off;          // first row (left) / column (right) of the block in the sector matrix
};

// complex block -> the real form of its sector matrix in W (column-major; W is
// the real form, or its transpose when the batch transposed it)
__global__ void zgather_kernel(const double2* __restrict__ ket, const ZCopyTask* __restrict__ tasks,
                               const SvdProblem* __restrict__ probs, double* __restrict__ W, int side) {
    const ZCopyTask t = tasks[blockIdx.x];
    const SvdProblem p = probs[t.problem];
    const int m = p.m / 2, n = p.n / 2;  // complex shape
    const double2* src = ket + t.blk_off;
    double* w = W + p.w_off;
    const int64_t total = (int64_t)t.rows * t.cols;
    for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
        const int i = (int)(e / t.cols), j = (int)(e % t.cols);
        const int ai = side == 0 ? t.off + i : i;
        const int aj = side == 0 ? j : t.off + j;
        if (ai >= m || aj >= n) continue;
        const double2 v = src[e];
        const int r[4] = {ai, ai, m + ai, m + ai};
        const int c[4] = {aj, n + aj, aj, n + aj};
        const double x[4] = {v.x, -v.y, v.y, v.x};
#pragma unroll
        for (int q = 0; q < 4; ++q)
            w[p.transposed ? (int64_t)r[q] * p.n + c[q] : (int64_t)c[q] * p.m + r[q]] = x[q];
    }
}

}  // namespace

struct dmrg_zcanon_s {
    dmrg_ctx_t ctx = nullptr;
    int side = 0, nl = 0, nr = 0, nsec = 0;
    std::vector<int> left_dim, right_dim;
    BlockListDesc ket;
    std::vector<std::vector<int>> members;
    std::vector<int> sec_m, sec_n;  // complex stacked shapes
    BatchedSvd svd;
    std::vector<ZCopyTask> copies;
    DeviceBuffer d_copies;
    bool ran = false;
    int sweeps = 0;
    std::vector<std::vector<double>> sv;  // complex singular values per sector (reference semantics)
    std::vector<std::vector<cplx>> U, V;  // per sector: m x r and n x r, column-major (column k contiguous)
    std::vector<int> rank;                // complex triplets recovered per sector
    std::vector<int> tdim;
    std::vector<std::vector<double>> forced;  // kept values after the truncation rule (forced zeros)
    BlockListDesc new_ket, canonical;
    std::vector<int> match_dim;
    double discarded = 0.0;
};

namespace {

// Complex triplets of one sector from its real-form SVD (see the file comment).
int recover_triplets(dmrg_zcanon_s& c, int s, cudaStream_t st) {
    const SvdProblem& p = c.svd.problem(s);
    const int m = c.sec_m[s], n = c.sec_n[s], r2 = p.cols, r = std::min(m, n);
    std::vector<double> W((size_t)p.rows * p.cols), Q((size_t)p.cols * p.cols), sig(r2), sgn(r2);
    std::vector<int> perm(r2);
    DMRG_CUDA_TRY(cudaMemcpyAsync(W.data(), c.svd.d_w.as<double>() + p.w_off, W.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(Q.data(), c.svd.d_q.as<double>() + p.q_off, Q.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(sig.data(), c.svd.d_s.as<double>() + p.s_off, r2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(sgn.data(), c.svd.d_sign.as<double>() + p.s_off, r2 * sizeof(double),
                                  cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(perm.data(), c.svd.d_perm.as<int>() + p.perm_off, r2 * sizeof(int),
                                  cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    // real singular pair j of the real form: u (2m), v (2n)
    auto real_pair = [&](int j, std::vector<double>& u, std::vector<double>& v) {
        const int k = perm[j];
        const double sj = sig[j];
        u.assign(2 * m, 0.0);
        v.assign(2 * n, 0.0);
        if (!p.transposed) {  // W = real form (2m x 2n): columns u_k s_k; Q = V
            for (int i = 0; i < 2 * m; ++i) u[i] = sj > 0.0 ? W[(size_t)k * p.rows + i] / sj : 0.0;
            for (int i = 0; i < 2 * n; ++i) v[i] = Q[(size_t)k * p.cols + i];
        } else {              // W = its transpose: columns v_k s_k; Q = U
            for (int i = 0; i < 2 * n; ++i) v[i] = sj > 0.0 ? W[(size_t)k * p.rows + i] / sj : 0.0;
            for (int i = 0; i < 2 * m; ++i) u[i] = Q[(size_t)k * p.cols + i];
        }
    };
    // the side that becomes the new ket (U for a left, V for a right
    // canonicalisation) is made orthonormal; the canonical factor is then the
    // projection of the sector matrix on it (dmrg_zcanon_write)
    const bool left = c.side == 0;
    const int d = left ? m : n;
    std::vector<cplx>& P = left ? c.U[s] : c.V[s];
    (left ? c.V[s] : c.U[s]).clear();
    P.assign((size_t)d * r, cplx(0.0, 0.0));
    std::vector<double>& out = c.sv[s];
    out.assign(r, 0.0);
    int kept = 0;
    const double tol = 1e-9 * std::max(sig.empty() ? 0.0 : sig[0], 1e-300);
    std::vector<double> u, v;
    // removes from x its components along the kept vectors [from, to)
    // (plain real arithmetic: std::complex's product guards against NaN/inf
    // operands at a large cost in this inner loop)
    auto project = [&](std::vector<cplx>& x, int from, int to) {
        double* xv = reinterpret_cast<double*>(x.data());
        for (int q = from; q < to; ++q) {
            const double* pv = reinterpret_cast<const double*>(&P[(size_t)q * d]);
            double ar = 0.0, ai = 0.0;  // a = <p_q, x> = sum conj(p) x
            for (int i = 0; i < d; ++i) {
                ar += pv[2 * i] * xv[2 * i] + pv[2 * i + 1] * xv[2 * i + 1];
                ai += pv[2 * i] * xv[2 * i + 1] - pv[2 * i + 1] * xv[2 * i];
            }
            for (int i = 0; i < d; ++i) {  // x -= a p_q
                const double pr = pv[2 * i], pi = pv[2 * i + 1];
                xv[2 * i] -= ar * pr - ai * pi;
                xv[2 * i + 1] -= ar * pi + ai * pr;
            }
        }
    };
    // kept vectors far in value from a candidate are complex-orthogonal to it
    // to eps ||A|| / gap already: a candidate is projected only against the
    // kept vectors within kWindow * sigma_max of its value
    constexpr double kWindow = 1e-3;
    auto project_near = [&](std::vector<cplx>& x, double value) {
        const double w = kWindow * (sig.empty() ? 0.0 : sig[0]);
        int q0 = 0;
        while (q0 < kept && out[q0] > value + w) ++q0;  // out descending
        int q1 = q0;
        while (q1 < kept && out[q1] >= value - w) ++q1;
        project(x, q0, q1);
    };
    for (int j0 = 0; j0 < r2 && kept < r;) {
        int j1 = j0 + 1;
        while (j1 < r2 && sig[j1 - 1] - sig[j1] <= tol) ++j1;
        const int want = std::min(r - kept, (j1 - j0 + 1) / 2);
        // the run's real singular vectors as complex vectors, orthogonalised (two
        // passes) against every vector kept so far: vectors of nearby runs are
        // complex-orthogonal only to eps ||A|| / gap
        std::vector<std::vector<cplx>> cx;
        std::vector<double> cs;
        for (int j = j0; j < j1; ++j) {
            if (sig[j] <= 0.0) break;
            real_pair(j, u, v);
            const std::vector<double>& x = left ? u : v;
            cx.emplace_back(d);
            for (int i = 0; i < d; ++i) cx.back()[i] = cplx(x[i], x[d + i]);
            cs.push_back(sig[j]);
            for (int pass = 0; pass < 2; ++pass) project_near(cx.back(), sig[j]);
        }
        // in descending order, a candidate whose remainder keeps more than half
        // its norm is a new complex direction (the other real vector of a
        // complex pair is the i-multiple of the first: remainder ~0); should a
        // degenerate run not reach its complex dimension that way, the largest
        // remainders fill it (pivoted Gram-Schmidt)
        std::vector<char> taken(cx.size(), 0);
        const int first = kept;
        auto norm2 = [&](int k) {
            double x = 0.0;
            for (int i = 0; i < d; ++i) x += std::norm(cx[k][i]);
            return x;
        };
        auto take = [&](int k, double nrm2) {
            taken[k] = 1;
            const double nrm = std::sqrt(nrm2);
            for (int i = 0; i < d; ++i) P[(size_t)kept * d + i] = cx[k][i] / nrm;
            out[kept] = cs[k];
            ++kept;
            for (size_t k2 = 0; k2 < cx.size(); ++k2)
                if (!taken[k2])
                    for (int pass = 0; pass < 2; ++pass) project(cx[k2], kept - 1, kept);
        };
        for (size_t k = 0; k < cx.size() && kept - first < want; ++k) {
            const double x = norm2((int)k);
            if (x > 0.5) take((int)k, x);
        }
        while (kept - first < want) {
            int best = -1;
            double bn = 0.0;
            for (size_t k = 0; k < cx.size(); ++k) {
                if (taken[k]) continue;
                const double x = norm2((int)k);
                if (x > bn) {
                    bn = x;
                    best = (int)k;
                }
            }
            if (best < 0 || bn <= 1e-6) break;  // no further independent direction in the run
            take(best, bn);
        }
        // the run's vectors in descending order of their values
        std::vector<int> ord(kept - first);
        for (int k = 0; k < kept - first; ++k) ord[k] = first + k;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return out[x] > out[y]; });
        std::vector<cplx> tp((size_t)(kept - first) * d);
        std::vector<double> to(kept - first);
        for (int k = 0; k < kept - first; ++k) {
            std::copy_n(&P[(size_t)ord[k] * d], d, &tp[(size_t)k * d]);
            to[k] = out[ord[k]];
        }
        std::copy(tp.begin(), tp.end(), P.begin() + (size_t)first * d);
        std::copy(to.begin(), to.end(), out.begin() + first);
        j0 = j1;
    }
    c.rank[s] = kept;
    return DMRG_OK;
}

}  // namespace

extern "C" {

int dmrg_zcanon_create(dmrg_ctx_t ctx, int side, int nl, int nr, const int* left_dim, const int* right_dim,
                       const dmrg_blocks_t* ket, dmrg_zcanon_t* out) {
    if (!ctx || !out || !ket || !left_dim || !right_dim || nl <= 0 || nr <= 0 || (side != 0 && side != 1))
        return set_error(DMRG_E_ARG, "invalid canonicalisation arguments");
    *out = nullptr;
    DMRG_CUDA_TRY(cudaSetDevice(ctx->device));
    auto* c = new dmrg_zcanon_s();
    c->ctx = ctx;
    c->side = side;
    c->nl = nl;
    c->nr = nr;
    c->left_dim.assign(left_dim, left_dim + nl);
    c->right_dim.assign(right_dim, right_dim + nr);
    if (!c->ket.assign(*ket)) {
        delete c;
        return set_error(DMRG_E_ARG, "invalid ket block list");
    }
    for (int k = 0; k < c->ket.count(); ++k)
        if (c->ket.left[k] < 0 || c->ket.left[k] >= nl || c->ket.right[k] < 0 || c->ket.right[k] >= nr) {
            delete c;
            return set_error(DMRG_E_ARG, "ket block %d sectors out of range", k);
        }
    c->nsec = side == 0 ? nr : nl;
    c->members = c->ket.by_sector(side == 0 ? 1 : 0, c->nsec);
    c->sec_m.assign(c->nsec, 0);
    c->sec_n.assign(c->nsec, 0);
    std::vector<int> rm(c->nsec), rn(c->nsec);
    for (int s = 0; s < c->nsec; ++s) {
        int acc = 0;
        for (int p : c->members[s]) acc += side == 0 ? c->ket.rows[p] : c->ket.cols[p];
        c->sec_m[s] = side == 0 ? acc : c->left_dim[s];
        c->sec_n[s] = side == 0 ? c->right_dim[s] : acc;
        rm[s] = 2 * c->sec_m[s];
        rn[s] = 2 * c->sec_n[s];
    }
    int rc = c->svd.plan(rm, rn, ctx->stream);
    if (rc == DMRG_OK) {
        for (int s = 0; s < c->nsec; ++s) {
            if (!c->svd.active(s)) continue;
            int acc = 0;
            for (int p : c->members[s]) {
                c->copies.push_back(ZCopyTask{c->ket.off[p], c->ket.rows[p], c->ket.cols[p], c->svd.index[s], acc});
                acc += side == 0 ? c->ket.rows[p] : c->ket.cols[p];
            }
        }
        rc = upload(c->d_copies, c->copies, ctx->stream);
    }
    if (rc != DMRG_OK) {
        delete c;
        return rc;
    }
    *out = c;
    return DMRG_OK;
}

int dmrg_zcanon_destroy(dmrg_zcanon_t c) {
    delete c;
    return DMRG_OK;
}

int dmrg_zcanon_run(dmrg_zcanon_t c, const double* ket_dev, int max_dim, double canpre, int* tdim_out,
                    double* discarded) {
    if (!c || (!ket_dev && c->ket.size)) return set_error(DMRG_E_ARG, "null argument");
    cudaStream_t st = c->ctx->stream;
    BatchedSvd& svd = c->svd;
    c->sv.assign(c->nsec, {});
    c->U.assign(c->nsec, {});
    c->V.assign(c->nsec, {});
    c->rank.assign(c->nsec, 0);
    if (!svd.probs.empty()) {
        int64_t wsize = 0;
        for (const auto& p : svd.probs) wsize += (int64_t)p.rows * p.cols;
        DMRG_CUDA_TRY(cudaMemsetAsync(svd.d_w.ptr, 0, wsize * sizeof(double), st));
        if (!c->copies.empty())
            DMRG_LAUNCH zgather_kernel<<<(int)c->copies.size(), 256, 0, st>>>(
                reinterpret_cast<const double2*>(ket_dev), c->d_copies.as<ZCopyTask>(), svd.d_probs.as<SvdProblem>(),
                svd.d_w.as<double>(), c->side);
        DMRG_CUDA_TRY(cudaGetLastError());
        DMRG_TRY(svd.run(st, &c->sweeps));
        for (int s = 0; s < c->nsec; ++s)
            if (svd.active(s)) DMRG_TRY(recover_triplets(*c, s, st));
    }
    std::vector<std::vector<double>> s = c->sv;
    for (int i = 0; i < c->nsec; ++i)
        if (!svd.active(i)) s[i].assign(1, 0.0);  // the reference's empty-sector case
    c->sv = s;
    c->tdim = compute_truncate_dim(max_dim, canpre, s);  // s: kept values, forced zeros in place
    c->forced = s;
    double all = 0.0, kept = 0.0;
    for (int i = 0; i < c->nsec; ++i) {
        for (double v : c->sv[i]) all += v * v;
        for (int j = 0; j < c->tdim[i] && j < (int)s[i].size(); ++j) kept += s[i][j] * s[i][j];
    }
    c->discarded = all - kept;
    c->new_ket = BlockListDesc();
    for (int k = 0; k < c->ket.count(); ++k) {
        const int l = c->ket.left[k], r = c->ket.right[k];
        if (c->side == 0) c->new_ket.push(l, r, c->ket.rows[k], svd.active(r) ? c->tdim[r] : c->ket.cols[k]);
        else c->new_ket.push(l, r, svd.active(l) ? c->tdim[l] : c->ket.rows[k], c->ket.cols[k]);
    }
    c->canonical = BlockListDesc();
    c->match_dim.assign(c->nsec, 0);
    for (int sct = 0; sct < c->nsec; ++sct) {
        if (c->side == 0) {
            c->match_dim[sct] = c->sec_n[sct];
            c->canonical.push(sct, sct, c->tdim[sct], c->sec_n[sct]);
        } else {
            c->match_dim[sct] = c->sec_m[sct];
            c->canonical.push(sct, sct, c->sec_m[sct], c->tdim[sct]);
        }
    }
    if (tdim_out)
        for (int i = 0; i < c->nsec; ++i) tdim_out[i] = c->tdim[i];
    if (discarded) *discarded = c->discarded;
    c->ran = true;
    return DMRG_OK;
}

int dmrg_zcanon_out_info(dmrg_zcanon_t c, int64_t* ket_size, int64_t* canonical_size, int* sweeps) {
    if (!c || !c->ran) return set_error(DMRG_E_STATE, "dmrg_zcanon_run has not been called");
    if (ket_size) *ket_size = c->new_ket.size;
    if (canonical_size) *canonical_size = c->canonical.size;
    if (sweeps) *sweeps = c->sweeps;
    return DMRG_OK;
}

int dmrg_zcanon_out_blocks(dmrg_zcanon_t c, int* ket_rows, int* ket_cols, int* canon_rows, int* canon_cols,
                           int* match_dim) {
    if (!c || !c->ran) return set_error(DMRG_E_STATE, "dmrg_zcanon_run has not been called");
    for (int k = 0; k < c->new_ket.count(); ++k) {
        if (ket_rows) ket_rows[k] = c->new_ket.rows[k];
        if (ket_cols) ket_cols[k] = c->new_ket.cols[k];
    }
    for (int s = 0; s < c->nsec; ++s) {
        if (canon_rows) canon_rows[s] = c->canonical.rows[s];
        if (canon_cols) canon_cols[s] = c->canonical.cols[s];
        if (match_dim) match_dim[s] = c->match_dim[s];
    }
    return DMRG_OK;
}

int dmrg_zcanon_singular_values(dmrg_zcanon_t c, int sector, int cap, double* values, int* count) {
    if (!c || !c->ran || !count) return set_error(DMRG_E_STATE, "dmrg_zcanon_run has not been called");
    if (sector < 0 || sector >= c->nsec) return set_error(DMRG_E_ARG, "sector %d out of range", sector);
    const auto& s = c->sv[sector];
    *count = (int)s.size();
    if (values)
        for (int i = 0; i < (int)s.size() && i < cap; ++i) values[i] = s[i];
    return DMRG_OK;
}

int dmrg_zcanon_write(dmrg_zcanon_t c, const double* ket_dev, double* new_ket_dev, double* canonical_dev) {
    if (!c || !c->ran) return set_error(DMRG_E_STATE, "dmrg_zcanon_run has not been called");
    cudaStream_t st = c->ctx->stream;
    std::vector<cplx> nk((size_t)c->new_ket.size), can((size_t)c->canonical.size, cplx(0.0, 0.0));
    std::vector<cplx> old((size_t)c->ket.size);
    if (c->ket.size)
        DMRG_CUDA_TRY(cudaMemcpyAsync(old.data(), ket_dev, old.size() * sizeof(cplx), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    for (int sct = 0; sct < c->nsec; ++sct) {
        const bool act = c->svd.active(sct);
        const int t = c->tdim[sct], m = c->sec_m[sct], n = c->sec_n[sct], rk = act ? c->rank[sct] : 0;
        const bool left = c->side == 0;
        const auto& P = left ? c->U[sct] : c->V[sct];  // orthonormal ket-side vectors, column k contiguous
        const int d = left ? m : n;
        auto pv = [&](int i, int k) { return k < rk ? P[(size_t)k * d + i] : cplx(0.0, 0.0); };
        // the sector matrix A (m x n, row-major; blocks stacked, short blocks zero-padded)
        std::vector<cplx> A;
        if (act) A.assign((size_t)m * n, cplx(0.0, 0.0));
        int acc = 0;
        for (int pos : c->members[sct]) {
            const int64_t o = c->new_ket.off[pos], oo = c->ket.off[pos];
            const int rows = c->new_ket.rows[pos], cols = c->new_ket.cols[pos];
            const int krows = c->ket.rows[pos], kcols = c->ket.cols[pos];
            if (act)
                for (int i = 0; i < krows; ++i)
                    for (int j = 0; j < kcols; ++j)
                        A[left ? (size_t)(acc + i) * n + j : (size_t)i * n + acc + j] = old[(size_t)oo + (size_t)i * kcols + j];
            for (int i = 0; i < rows; ++i)
                for (int j = 0; j < cols; ++j) {
                    cplx x;
                    if (!act) x = old[(size_t)oo + (size_t)i * cols + j];  // untouched (empty sector)
                    else if (left) x = pv(acc + i, j);                    // U rows of the block
                    else x = std::conj(pv(acc + j, i));                   // V^H columns of the block
                    nk[(size_t)o + (size_t)i * cols + j] = x;
                }
            acc += left ? krows : kcols;
        }
        const int64_t co = c->canonical.off[sct];
        const auto& f = c->forced[sct];
        if (!act) continue;  // zero block
        // canonical factor: U^H A (t x n) or A V (m x t), i.e. S V^H or U S; rows
        // (columns) whose value the truncation forced to zero stay zero
        if (left)
            for (int k = 0; k < t; ++k) {
                if (f[k] == 0.0) continue;
                for (int j = 0; j < n; ++j) {
                    cplx x(0.0, 0.0);
                    for (int i = 0; i < m; ++i) x += std::conj(pv(i, k)) * A[(size_t)i * n + j];
                    can[(size_t)co + (size_t)k * n + j] = x;
                }
            }
        else
            for (int i = 0; i < m; ++i)
                for (int k = 0; k < t; ++k) {
                    if (f[k] == 0.0) continue;
                    cplx x(0.0, 0.0);
                    for (int j = 0; j < n; ++j) x += A[(size_t)i * n + j] * pv(j, k);
                    can[(size_t)co + (size_t)i * t + k] = x;
                }
    }
    if (!nk.empty())
        DMRG_CUDA_TRY(cudaMemcpyAsync(new_ket_dev, nk.data(), nk.size() * sizeof(cplx), cudaMemcpyHostToDevice, st));
    if (!can.empty())
        DMRG_CUDA_TRY(
            cudaMemcpyAsync(canonical_dev, can.data(), can.size() * sizeof(cplx), cudaMemcpyHostToDevice, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    return DMRG_OK;
}

}  // extern "C"
