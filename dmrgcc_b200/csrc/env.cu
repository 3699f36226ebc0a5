// a2/a3: environment updates.
//
// Left (RealTensorContraction::LeftComputeTensorContraction,
// src/dmrg/realdmrg/real_tensor_contraction.cc:782-940):
//   L'[o2](i,j) += W[o1][o2](p(k,i), p(l,j)) * B(k,i)^T L[o1](k,l) K(l,j)
// stage 1: F = B(k,i)^T L[o1](k,l)      (transposed-A grouped GEMM)
// stage 2: L'[o2](i,j) += W * F K(l,j)   (one group per output block)
// Right (RightComputeTensorContraction, :959-1119):
//   R'[o1](j,i) += W[o1][o2](p(i,k), p(j,l)) * K(j,l) R[o2](l,k) B(i,k)^T
// stage 1: G = K(j,l) R[o2](l,k)
// stage 2: R'[o1](j,i) += W * G B(i,k)^T (transposed-B)
// The output block lists follow the reference's zero_flag pass (:797-883,
// :974-1060): per output bond index, blocks in row-major (first, second) sector
// order, present wherever some contribution has a nonzero W.
#include <algorithm>

#include "blocksparse.h"
#include "gemm.cuh"
#include "zgemm.cuh"

using namespace dmrg;

struct dmrg_env_s {
    dmrg_ctx_t ctx = nullptr;
    int side = 0;
    int precision = DMRG_PREC_FP64;
    SiteDesc site;
    EnvDesc in, out;
    GemmSchedule s1, s2;
    SplitPlan p1, p2;  // split precisions: the same two stages on the tcgen05 path
    // the complex path (dmrg_zenv_create): the same stages on complex blocks
    bool cplx = false;
    ZGemmSchedule z1, z2;
    DeviceBuffer scratch;
    int64_t scratch_size = 0;
    double flops_alg = 0, flops_exec = 0;
};

namespace {

struct Stage2Term {
    int out_o, out_pos;
    int scratch_index;  // which stage-1 product
    int ket_pos;        // K block (left) or B block (right)
    double w;
};

struct Stage1Task {
    int ket_pos;
    int o_in, blk_in;
    int m, n, k;
    int64_t off;
};

int build_left(dmrg_env_s& e) {
    const SiteDesc& s = e.site;
    const BlockListDesc& ket = s.ket;
    auto same_left = ket.by_sector(0, s.nl);
    // zero_flag pass -> output structure
    std::vector<char> flag((size_t)s.rb * s.nr * s.nr, 0);
    std::vector<int> dim_r(s.nr, -1);  // column count of the ket blocks with right sector r
    for (int k = 0; k < ket.count(); ++k) {
        int r = ket.right[k];
        if (dim_r[r] == -1) dim_r[r] = ket.cols[k];
        else if (dim_r[r] != ket.cols[k])
            return set_error(DMRG_E_ARG, "ket blocks of right sector %d have different widths", r);
    }
    for (int o1 = 0; o1 < s.lb; ++o1) {
        const BlockListDesc& Lo = e.in.o[o1];
        for (int i = 0; i < Lo.count(); ++i) {
            const int kdx = Lo.left[i], ldx = Lo.right[i];
            if (kdx < 0 || kdx >= s.nl || ldx < 0 || ldx >= s.nl)
                return set_error(DMRG_E_ARG, "L[%d] block %d sectors out of range", o1, i);
            if (Lo.rows[i] == 0) continue;
            for (int pk : same_left[kdx]) {
                const int idx = ket.right[pk];
                const int p1 = s.p(kdx, idx);
                if (!s.left_nonzero(o1, p1)) continue;
                for (int pl : same_left[ldx]) {
                    const int jdx = ket.right[pl];
                    const int p2 = s.p(ldx, jdx);
                    for (int o2 = 0; o2 < s.rb; ++o2)
                        if (s.w(o1, o2, p1, p2) != 0.0) flag[((size_t)o2 * s.nr + idx) * s.nr + jdx] = 1;
                }
            }
        }
    }
    e.out.o.assign(s.rb, BlockListDesc());
    for (int o2 = 0; o2 < s.rb; ++o2)
        for (int i = 0; i < s.nr; ++i)
            for (int j = 0; j < s.nr; ++j)
                if (flag[((size_t)o2 * s.nr + i) * s.nr + j]) e.out.o[o2].push(i, j, dim_r[i], dim_r[j]);
    e.out.rebase();

    std::vector<Stage1Task> tasks;
    std::vector<Stage2Term> terms;
    double f1_alg = 0, f2_alg = 0, f1_exec = 0, f2_exec = 0;
    e.scratch_size = 0;
    for (int o1 = 0; o1 < s.lb; ++o1) {
        const BlockListDesc& Lo = e.in.o[o1];
        for (int i = 0; i < Lo.count(); ++i) {
            const int kdx = Lo.left[i], ldx = Lo.right[i];
            const int lr = Lo.rows[i], lc = Lo.cols[i];
            if (lr == 0) continue;
            for (int pk : same_left[kdx]) {
                const int idx = ket.right[pk];
                const int p1 = s.p(kdx, idx);
                if (!s.left_nonzero(o1, p1)) continue;
                const int a_k = ket.rows[pk], b_i = ket.cols[pk];
                if (a_k != lr) return set_error(DMRG_E_ARG, "ket block %d rows %d != L rows %d", pk, a_k, lr);
                f1_alg += 2.0 * b_i * a_k * lc;
                const int t_index = (int)tasks.size();
                bool used = false;
                for (int pl : same_left[ldx]) {
                    const int jdx = ket.right[pl];
                    const int p2 = s.p(ldx, jdx);
                    if (ket.rows[pl] != lc) return set_error(DMRG_E_ARG, "ket block %d rows != L cols", pl);
                    f2_alg += 2.0 * b_i * lc * ket.cols[pl];
                    for (int o2 = 0; o2 < s.rb; ++o2) {
                        const double w = s.w(o1, o2, p1, p2);
                        if (w == 0.0) continue;
                        const int q = e.out.o[o2].find(idx, jdx);
                        terms.push_back(Stage2Term{o2, q, t_index, pl, w});
                        f2_exec += 2.0 * b_i * lc * ket.cols[pl];
                        used = true;
                    }
                }
                if (used) {
                    tasks.push_back(Stage1Task{pk, o1, i, b_i, lc, a_k, e.scratch_size});
                    e.scratch_size += (int64_t)b_i * lc;
                    f1_exec += 2.0 * b_i * a_k * lc;
                }
            }
        }
    }
    // stage 1: F = B^T L  (A = ket block stored a_k x b_i -> transposed)
    e.s1.reset();
    e.s1.ta = true;
    for (const Stage1Task& t : tasks) {
        e.s1.add_group(t.off, t.n, t.m, t.n);
        e.s1.add_term(ket.off[t.ket_pos], ket.cols[t.ket_pos], e.in.base[t.o_in] + e.in.o[t.o_in].off[t.blk_in],
                      t.n, t.k, 1.0);
    }
    // stage 2: out += w F K, grouped per output block
    e.s2.reset();
    std::vector<int64_t> first(e.out.o.size() + 1, 0);
    for (size_t o = 0; o < e.out.o.size(); ++o) first[o + 1] = first[o] + e.out.o[o].count();
    std::vector<std::vector<int>> bucket(first.back());
    for (int i = 0; i < (int)terms.size(); ++i) bucket[first[terms[i].out_o] + terms[i].out_pos].push_back(i);
    for (size_t o = 0; o < e.out.o.size(); ++o) {
        const BlockListDesc& Oo = e.out.o[o];
        for (int q = 0; q < Oo.count(); ++q) {
            const auto& b = bucket[first[o] + q];
            if (b.empty()) continue;
            e.s2.add_group(e.out.base[o] + Oo.off[q], Oo.cols[q], Oo.rows[q], Oo.cols[q]);
            for (int ti : b) {
                const Stage2Term& t = terms[ti];
                const Stage1Task& st = tasks[t.scratch_index];
                e.s2.add_term(st.off, st.n, ket.off[t.ket_pos], ket.cols[t.ket_pos], st.n, t.w);
            }
        }
    }
    e.flops_alg = f1_alg + f2_alg;
    e.flops_exec = f1_exec + f2_exec;
    return DMRG_OK;
}

int build_right(dmrg_env_s& e) {
    const SiteDesc& s = e.site;
    const BlockListDesc& ket = s.ket;
    auto same_right = ket.by_sector(1, s.nr);
    std::vector<char> flag((size_t)s.lb * s.nl * s.nl, 0);
    std::vector<int> dim_l(s.nl, -1);
    for (int k = 0; k < ket.count(); ++k) {
        int l = ket.left[k];
        if (dim_l[l] == -1) dim_l[l] = ket.rows[k];
        else if (dim_l[l] != ket.rows[k])
            return set_error(DMRG_E_ARG, "ket blocks of left sector %d have different heights", l);
    }
    for (int o2 = 0; o2 < s.rb; ++o2) {
        const BlockListDesc& Ro = e.in.o[o2];
        for (int i = 0; i < Ro.count(); ++i) {
            const int ldx = Ro.left[i], kdx = Ro.right[i];
            if (ldx < 0 || ldx >= s.nr || kdx < 0 || kdx >= s.nr)
                return set_error(DMRG_E_ARG, "R[%d] block %d sectors out of range", o2, i);
            if (Ro.rows[i] == 0) continue;
            for (int pl : same_right[ldx]) {
                const int jdx = ket.left[pl];
                const int p2 = s.p(jdx, ldx);
                if (!s.right_nonzero(o2, p2)) continue;
                for (int pk : same_right[kdx]) {
                    const int idx = ket.left[pk];
                    const int p1 = s.p(idx, kdx);
                    for (int o1 = 0; o1 < s.lb; ++o1)
                        if (s.w(o1, o2, p1, p2) != 0.0) flag[((size_t)o1 * s.nl + jdx) * s.nl + idx] = 1;
                }
            }
        }
    }
    e.out.o.assign(s.lb, BlockListDesc());
    for (int o1 = 0; o1 < s.lb; ++o1)
        for (int j = 0; j < s.nl; ++j)
            for (int i = 0; i < s.nl; ++i)
                if (flag[((size_t)o1 * s.nl + j) * s.nl + i]) e.out.o[o1].push(j, i, dim_l[j], dim_l[i]);
    e.out.rebase();

    std::vector<Stage1Task> tasks;
    std::vector<Stage2Term> terms;
    double f1_alg = 0, f2_alg = 0, f1_exec = 0, f2_exec = 0;
    e.scratch_size = 0;
    for (int o2 = 0; o2 < s.rb; ++o2) {
        const BlockListDesc& Ro = e.in.o[o2];
        for (int i = 0; i < Ro.count(); ++i) {
            const int ldx = Ro.left[i], kdx = Ro.right[i];
            const int rr = Ro.rows[i], rc = Ro.cols[i];
            if (rr == 0) continue;
            for (int pl : same_right[ldx]) {
                const int jdx = ket.left[pl];
                const int p2 = s.p(jdx, ldx);
                if (!s.right_nonzero(o2, p2)) continue;
                const int a_j = ket.rows[pl], b_l = ket.cols[pl];
                if (b_l != rr) return set_error(DMRG_E_ARG, "ket block %d cols %d != R rows %d", pl, b_l, rr);
                f1_alg += 2.0 * a_j * b_l * rc;
                const int t_index = (int)tasks.size();
                bool used = false;
                for (int pk : same_right[kdx]) {
                    const int idx = ket.left[pk];
                    const int p1 = s.p(idx, kdx);
                    if (ket.cols[pk] != rc) return set_error(DMRG_E_ARG, "ket block %d cols != R cols", pk);
                    f2_alg += 2.0 * a_j * rc * ket.rows[pk];
                    for (int o1 = 0; o1 < s.lb; ++o1) {
                        const double w = s.w(o1, o2, p1, p2);
                        if (w == 0.0) continue;
                        const int q = e.out.o[o1].find(jdx, idx);
                        terms.push_back(Stage2Term{o1, q, t_index, pk, w});
                        f2_exec += 2.0 * a_j * rc * ket.rows[pk];
                        used = true;
                    }
                }
                if (used) {
                    tasks.push_back(Stage1Task{pl, o2, i, a_j, rc, b_l, e.scratch_size});
                    e.scratch_size += (int64_t)a_j * rc;
                    f1_exec += 2.0 * a_j * b_l * rc;
                }
            }
        }
    }
    // stage 1: G = K R
    e.s1.reset();
    for (const Stage1Task& t : tasks) {
        e.s1.add_group(t.off, t.n, t.m, t.n);
        e.s1.add_term(ket.off[t.ket_pos], ket.cols[t.ket_pos], e.in.base[t.o_in] + e.in.o[t.o_in].off[t.blk_in],
                      t.n, t.k, 1.0);
    }
    // stage 2: out += w G B^T (B block stored a_i x b_k -> transposed)
    e.s2.reset();
    e.s2.tb = true;
    std::vector<int64_t> first(e.out.o.size() + 1, 0);
    for (size_t o = 0; o < e.out.o.size(); ++o) first[o + 1] = first[o] + e.out.o[o].count();
    std::vector<std::vector<int>> bucket(first.back());
    for (int i = 0; i < (int)terms.size(); ++i) bucket[first[terms[i].out_o] + terms[i].out_pos].push_back(i);
    for (size_t o = 0; o < e.out.o.size(); ++o) {
        const BlockListDesc& Oo = e.out.o[o];
        for (int q = 0; q < Oo.count(); ++q) {
            const auto& b = bucket[first[o] + q];
            if (b.empty()) continue;
            e.s2.add_group(e.out.base[o] + Oo.off[q], Oo.cols[q], Oo.rows[q], Oo.cols[q]);
            for (int ti : b) {
                const Stage2Term& t = terms[ti];
                const Stage1Task& st = tasks[t.scratch_index];
                e.s2.add_term(st.off, st.n, ket.off[t.ket_pos], ket.cols[t.ket_pos], st.n, t.w);
            }
        }
    }
    e.flops_alg = f1_alg + f2_alg;
    e.flops_exec = f1_exec + f2_exec;
    return DMRG_OK;
}

}  // namespace

extern "C" {

int dmrg_env_create(dmrg_ctx_t ctx, int side, int nl, int nr, const int* phys, const dmrg_blocks_t* ket, int d,
                    int lb, int rb, const double* W, const dmrg_blocks_t* env_in, int precision, dmrg_env_t* out) {
    if (!ctx || !out || !env_in) return set_error(DMRG_E_ARG, "null argument");
    if (side != 0 && side != 1) return set_error(DMRG_E_ARG, "side must be 0 (left) or 1 (right)");
    if (precision != DMRG_PREC_FP64 && precision != DMRG_PREC_TF32X3 && precision != DMRG_PREC_BF16X3)
        return set_error(DMRG_E_ARG, "unknown precision %d", precision);
    *out = nullptr;
    DMRG_CUDA_TRY(cudaSetDevice(ctx->device));
    auto* e = new dmrg_env_s();
    e->ctx = ctx;
    e->side = side;
    e->precision = precision;
    int rc = build_site_desc(e->site, nl, nr, phys, ket, d, lb, rb, W);
    if (rc == DMRG_OK && !e->in.assign(env_in, side == 0 ? lb : rb))
        rc = set_error(DMRG_E_ARG, "invalid input environment");
    if (rc == DMRG_OK) rc = side == 0 ? build_left(*e) : build_right(*e);
    cudaStream_t st = ctx->stream;
    if (rc == DMRG_OK) rc = e->s1.check_bounds(e->site.ket.size, e->in.size, e->scratch_size);
    if (rc == DMRG_OK) rc = e->s2.check_bounds(e->scratch_size, e->site.ket.size, e->out.size);
    if (rc == DMRG_OK) rc = e->s1.finalize(64, 64, 16, st);
    if (rc == DMRG_OK) rc = e->s2.finalize(64, 64, 16, st, ctx->num_sms);
    if (rc == DMRG_OK) rc = e->scratch.alloc((size_t)std::max<int64_t>(e->scratch_size, 1) * sizeof(double));
    if (rc == DMRG_OK && precision != DMRG_PREC_FP64) {
        const int fmt = precision == DMRG_PREC_BF16X3 ? kFmtBF16 : kFmtTF32;
        rc = e->p1.build(e->s1, fmt, e->site.ket.size, e->in.size, e->scratch_size, st, ctx->num_sms);
        if (rc == DMRG_OK) rc = e->p2.build(e->s2, fmt, e->scratch_size, e->site.ket.size, e->out.size, st, ctx->num_sms);
    }
    if (rc != DMRG_OK) {
        delete e;
        return rc;
    }
    *out = e;
    return DMRG_OK;
}

int dmrg_env_destroy(dmrg_env_t e) {
    delete e;
    return DMRG_OK;
}

int dmrg_env_out_info(dmrg_env_t e, int* bond, int64_t* size) {
    if (!e) return set_error(DMRG_E_ARG, "null env");
    if (bond) *bond = (int)e->out.o.size();
    if (size) *size = e->out.size;
    return DMRG_OK;
}

int dmrg_env_out_blocks(dmrg_env_t e, int o, int cap, int* nblocks, int* left, int* right, int* rows, int* cols) {
    if (!e || !nblocks) return set_error(DMRG_E_ARG, "null argument");
    if (o < 0 || o >= (int)e->out.o.size()) return set_error(DMRG_E_ARG, "bond index %d out of range", o);
    const BlockListDesc& b = e->out.o[o];
    *nblocks = b.count();
    if (cap < b.count()) return cap == 0 ? DMRG_OK : set_error(DMRG_E_ARG, "capacity %d < %d", cap, b.count());
    for (int k = 0; k < b.count(); ++k) {
        if (left) left[k] = b.left[k];
        if (right) right[k] = b.right[k];
        if (rows) rows[k] = b.rows[k];
        if (cols) cols[k] = b.cols[k];
    }
    return DMRG_OK;
}

int dmrg_env_flops(dmrg_env_t e, double* alg, double* exec) {
    if (!e) return set_error(DMRG_E_ARG, "null env");
    if (alg) *alg = e->flops_alg;
    if (exec) *exec = e->flops_exec;
    return DMRG_OK;
}

int dmrg_env_apply(dmrg_env_t e, const double* ket_dev, const double* env_in_dev, double* env_out_dev) {
    if (!e) return set_error(DMRG_E_ARG, "null env");
    cudaStream_t st = e->ctx->stream;
    if (e->out.size) DMRG_CUDA_TRY(cudaMemsetAsync(env_out_dev, 0, (size_t)e->out.size * sizeof(double), st));
    // Both sides: stage 1 reads (ket, env_in) into scratch, stage 2 reads
    // (scratch, ket) into the output; the transposes live in the schedules.
    if (e->cplx) return set_error(DMRG_E_STATE, "a complex environment update runs through dmrg_zenv_apply");
    if (e->precision != DMRG_PREC_FP64) {  // tcgen05 split products, FP64 sums and FP64 storage
        DMRG_TRY(e->p1.run(ket_dev, env_in_dev, e->scratch.as<double>(), false, e->ctx->d_status, st));
        DMRG_TRY(e->p2.run(e->scratch.as<double>(), ket_dev, env_out_dev, true, e->ctx->d_status, st));
        return DMRG_OK;
    }
    DMRG_TRY(launch_gemm_f64(e->s1, ket_dev, env_in_dev, e->scratch.as<double>(), false, st));
    DMRG_TRY(launch_gemm_f64(e->s2, e->scratch.as<double>(), ket_dev, env_out_dev, true, st));
    return DMRG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// The complex path: ComplexTensorContraction::Left/RightComputeTensorContraction
// (src/dmrg/complexdmrg/complex_tensor_contraction.cc:800-975, 977-1150) have
// the real structure with the bra block Hermitian-conjugated
// (HermitianConjugateMatrix, :929, :1113) and a complex MPO.  The real builder
// runs on a surrogate MPO whose nonzero entries are the (1-based) positions of
// the complex entries that are nonzero (|w| != 0 exactly where the complex
// reference takes the term), so the output block maps follow the same
// zero_flag pass; its terms then become complex terms whose scale is the
// complex entry at that position, with the conjugation on the bra operand.
// ---------------------------------------------------------------------------
extern "C" {

int dmrg_zenv_create(dmrg_ctx_t ctx, int side, int nl, int nr, const int* phys, const dmrg_blocks_t* ket, int d,
                     int lb, int rb, const double* W, const dmrg_blocks_t* env_in, dmrg_env_t* out) {
    if (!W || lb <= 0 || rb <= 0 || d <= 0 || !out) return set_error(DMRG_E_ARG, "null argument");
    const size_t nw = (size_t)lb * rb * d * d;
    std::vector<double> ids(nw, 0.0);
    for (size_t i = 0; i < nw; ++i)
        if (W[2 * i] != 0.0 || W[2 * i + 1] != 0.0) ids[i] = (double)(i + 1);
    DMRG_TRY(dmrg_env_create(ctx, side, nl, nr, phys, ket, d, lb, rb, ids.data(), env_in, DMRG_PREC_FP64, out));
    dmrg_env_s* e = *out;
    auto convert = [&](const GemmSchedule& s, ZGemmSchedule& z, bool stage2, int conj) {
        z.reset();
        z.ta = s.ta;
        z.tb = s.tb;
        for (const GemmGroup& g : s.groups) {
            z.add_group(g.c_off, g.ldc, g.m, g.n);
            for (int t = g.t0; t < g.t1; ++t) {
                const GemmTerm& x = s.terms[t];
                double re = x.scale, im = 0.0;
                if (stage2) {
                    const size_t pos = (size_t)x.scale - 1;
                    re = W[2 * pos];
                    im = W[2 * pos + 1];
                }
                z.add_term(x.a_off, x.lda, x.b_off, x.ldb, x.k, re, im, conj);
            }
        }
    };
    // left: stage 1 B^dagger L (conjugated A), stage 2 w F K;  right: stage 1 K R, stage 2 w G B^dagger
    convert(e->s1, e->z1, false, side == 0 ? 1 : 0);
    convert(e->s2, e->z2, true, side == 0 ? 0 : 2);
    int rc = e->z1.check_bounds(e->site.ket.size, e->in.size, e->scratch_size);
    if (rc == DMRG_OK) rc = e->z2.check_bounds(e->scratch_size, e->site.ket.size, e->out.size);
    if (rc == DMRG_OK) rc = e->z1.finalize(ctx->stream);
    if (rc == DMRG_OK) rc = e->z2.finalize(ctx->stream);
    if (rc == DMRG_OK) rc = e->scratch.alloc((size_t)std::max<int64_t>(e->scratch_size, 1) * 2 * sizeof(double));
    if (rc != DMRG_OK) {
        delete e;
        *out = nullptr;
        return rc;
    }
    e->cplx = true;
    e->flops_alg *= 4.0;  // a complex product is four real ones
    e->flops_exec *= 4.0;
    return DMRG_OK;
}

int dmrg_zenv_apply(dmrg_env_t e, const double* ket_dev, const double* env_in_dev, double* env_out_dev) {
    if (!e || !e->cplx) return set_error(DMRG_E_ARG, "not a complex environment update (dmrg_zenv_create)");
    cudaStream_t st = e->ctx->stream;
    if (e->out.size) DMRG_CUDA_TRY(cudaMemsetAsync(env_out_dev, 0, (size_t)e->out.size * 2 * sizeof(double), st));
    DMRG_TRY(launch_zgemm(e->z1, ket_dev, env_in_dev, e->scratch.as<double>(), false, st));
    DMRG_TRY(launch_zgemm(e->z2, e->scratch.as<double>(), ket_dev, env_out_dev, true, st));
    return DMRG_OK;
}

}  // extern "C"
