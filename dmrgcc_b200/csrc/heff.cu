// a1: block-sparse H_eff * psi.
//
// The reference (RealTensorContraction::MultiplyEffectHamilton,
// src/dmrg/realdmrg/real_tensor_contraction.cc:1223-1291) walks
//   o2 -> R block (l -> j) -> K block (k, l) with RightCheckZero(o2, p(k,l))
//      -> T = K(k,l) R[o2](l,j)
//      -> psi block (i, j) -> o1 with W[o1][o2](p(i,j), p(k,l)) != 0 and L[o1](i,k)
//      -> out(i,j) += W * L[o1](i,k) T
// issuing one MKL dgemm per product.  Here the same walk is done once per site,
// on the host, to build two grouped launches:
//   stage A: every T needed by at least one term, one group each (C = scratch);
//   stage B: one group per output block (i, j) holding all of its
//            (W, L block, T) terms, summed in registers by the tile owner.
#include <algorithm>
#include <cstdlib>
#include <map>

#include "heff.cuh"

using namespace dmrg;



namespace {

int build_heff(dmrg_heff_s& h) {
    const SiteDesc& s = h.site;
    const BlockListDesc& ket = s.ket;
    auto same_right = ket.by_sector(1, s.nr);
    // Validate environment sector indices.
    for (int o = 0; o < s.lb; ++o)
        for (int q = 0; q < h.L.o[o].count(); ++q)
            if (h.L.o[o].left[q] < 0 || h.L.o[o].left[q] >= s.nl || h.L.o[o].right[q] < 0 ||
                h.L.o[o].right[q] >= s.nl)
                return set_error(DMRG_E_ARG, "L[%d] block %d has sectors outside %d", o, q, s.nl);
    for (int o = 0; o < s.rb; ++o)
        for (int q = 0; q < h.R.o[o].count(); ++q)
            if (h.R.o[o].left[q] < 0 || h.R.o[o].left[q] >= s.nr || h.R.o[o].right[q] < 0 ||
                h.R.o[o].right[q] >= s.nr)
                return set_error(DMRG_E_ARG, "R[%d] block %d has sectors outside %d", o, q, s.nr);

    struct TermB {
        int out_pos;
        int64_t l_off;
        int lda;
        int t_index;
        int k;
        double w;
    };
    std::vector<TermB> termsB;
    struct TaskA {
        int pos;       // ket block
        int64_t r_off; // R block offset
        int b_l, b_j, a_k;
        int64_t t_off;
    };
    std::vector<TaskA> tasks;
    h.t_size = 0;
    double fa_alg = 0, fb = 0, fa_exec = 0;

    for (int o2 = 0; o2 < s.rb; ++o2) {
        const BlockListDesc& Ro = h.R.o[o2];
        for (int i = 0; i < Ro.count(); ++i) {
            const int ldx = Ro.left[i], jdx = Ro.right[i];
            const int rr = Ro.rows[i], rc = Ro.cols[i];
            if (rr == 0) continue;  // the reference skips empty blocks
            for (int pos : same_right[ldx]) {
                const int kdx = ket.left[pos];
                const int p2 = s.pb(pos);
                if (!s.right_nonzero(o2, p2)) continue;
                const int a_k = ket.rows[pos], b_l = ket.cols[pos];
                if (b_l != rr)
                    return set_error(DMRG_E_ARG, "ket block %d is %dx%d but R[%d] block %d is %dx%d", pos, a_k,
                                     b_l, o2, i, rr, rc);
                fa_alg += 2.0 * a_k * b_l * rc;
                if (a_k == 0 || b_l == 0 || rc == 0) continue;  // empty product
                const int t_index = (int)tasks.size();
                bool used = false;
                for (int pos2 : same_right[jdx]) {
                    const int idx = ket.left[pos2];
                    const int p1 = s.pb(pos2);
                    for (int o1 = 0; o1 < s.lb; ++o1) {
                        const double w = s.w(o1, o2, p1, p2);
                        if (w == 0.0) continue;
                        const int q = h.L.o[o1].find(idx, kdx);
                        if (q == -1) continue;
                        const int lr = h.L.o[o1].rows[q], lc = h.L.o[o1].cols[q];
                        if (lc != a_k || lr != ket.rows[pos2] || rc != ket.cols[pos2])
                            return set_error(DMRG_E_ARG,
                                             "shape mismatch: L[%d] block %d %dx%d, K %dx%d, R %dx%d, out %dx%d", o1,
                                             q, lr, lc, a_k, b_l, rr, rc, ket.rows[pos2], ket.cols[pos2]);
                        if (lr == 0) continue;
                        termsB.push_back(TermB{pos2, h.L.base[o1] + h.L.o[o1].off[q], lc, t_index, a_k, w});
                        fb += 2.0 * lr * lc * rc;
                        used = true;
                    }
                }
                if (used) {
                    tasks.push_back(TaskA{pos, h.R.base[o2] + Ro.off[i], b_l, rc, a_k, h.t_size});
                    h.t_size += (int64_t)a_k * rc;
                    fa_exec += 2.0 * a_k * b_l * rc;
                }
            }
        }
    }

    // Stage A: one group per T.
    h.sa.reset();
    for (const TaskA& t : tasks) {
        h.sa.add_group(t.t_off, t.b_j, t.a_k, t.b_j);
        h.sa.add_term(ket.off[t.pos], t.b_l, t.r_off, t.b_j, t.b_l, 1.0);
    }
    // Stage B: one group per output block, terms in generation order.
    h.sb.reset();
    std::vector<std::vector<int>> per_out(ket.count());
    for (int i = 0; i < (int)termsB.size(); ++i) per_out[termsB[i].out_pos].push_back(i);
    for (int pos2 = 0; pos2 < ket.count(); ++pos2) {
        if (per_out[pos2].empty()) continue;
        h.sb.add_group(ket.off[pos2], ket.cols[pos2], ket.rows[pos2], ket.cols[pos2]);
        for (int i : per_out[pos2]) {
            const TermB& t = termsB[i];
            const TaskA& ta = tasks[t.t_index];
            h.sb.add_term(t.l_off, t.lda, ta.t_off, ta.b_j, t.k, t.w);
        }
    }
    h.flops_alg = fa_alg + fb;
    h.flops_exec = fa_exec + fb;
    DMRG_TRY(h.sa.check_bounds(ket.size, h.R.size, h.t_size));
    DMRG_TRY(h.sb.check_bounds(h.L.size, h.t_size, ket.size));
    cudaStream_t st = h.ctx->stream;
    DMRG_TRY(h.sa.finalize(64, 64, 16, st));
    DMRG_TRY(h.sb.finalize(64, 64, 16, st, h.ctx->num_sms));
    if (is_split(h.precision)) {
        const int fmt = split_fmt(h.precision);
        h.pk_psi.fmt = h.pk_L.fmt = h.pk_R.fmt = h.pa.fmt = h.pb.fmt = fmt;
        // operand images: psi blocks and L blocks in the A role, R blocks (transposed)
        // in the B role, and the K*R intermediates written directly as B-role images
        std::vector<int64_t> psi_img(ket.count());
        for (int pos = 0; pos < ket.count(); ++pos)
            psi_img[pos] = h.pk_psi.add(ket.off[pos], ket.rows[pos], ket.cols[pos], ket.cols[pos], false);
        std::map<int64_t, int64_t> r_img, l_img;
        const int tk = pack_k(fmt);
        auto slices = [tk](int k) { return (k + tk - 1) / tk; };
        std::vector<int64_t> t_img(tasks.size());
        h.pa.reset();
        h.pa.out_mode = 1;
        h.t_img_bytes = 0;
        for (size_t i = 0; i < tasks.size(); ++i) {
            const TaskA& t = tasks[i];
            auto it = r_img.find(t.r_off);
            if (it == r_img.end())
                it = r_img.emplace(t.r_off, h.pk_R.add(t.r_off, t.b_j, t.b_l, t.b_j, true)).first;
            t_img[i] = h.t_img_bytes;
            h.t_img_bytes += image_bytes(t.b_j, slices(t.a_k));
            PackedGroup g{};
            g.t0 = (int)h.pa.terms.size();
            g.m = t.a_k;
            g.n = t.b_j;
            g.t_img = t_img[i];
            g.t_slices = slices(t.a_k);
            h.pa.terms.push_back(PackedTerm{psi_img[t.pos], it->second, slices(t.b_l), 0, 1.0});
            g.t1 = (int)h.pa.terms.size();
            h.pa.groups.push_back(g);
        }
        h.pb.reset();
        h.pb.out_mode = 0;
        for (int pos2 = 0; pos2 < ket.count(); ++pos2) {
            if (per_out[pos2].empty()) continue;
            PackedGroup g{};
            g.t0 = (int)h.pb.terms.size();
            g.m = ket.rows[pos2];
            g.n = ket.cols[pos2];
            g.c_off = ket.off[pos2];
            g.ldc = ket.cols[pos2];
            for (int i : per_out[pos2]) {
                const TermB& t = termsB[i];
                auto it = l_img.find(t.l_off);
                if (it == l_img.end())
                    it = l_img.emplace(t.l_off, h.pk_L.add(t.l_off, ket.rows[pos2], t.k, t.lda, false)).first;
                h.pb.terms.push_back(PackedTerm{it->second, t_img[t.t_index], slices(t.k), 0, t.w});
            }
            g.t1 = (int)h.pb.terms.size();
            h.pb.groups.push_back(g);
        }
        DMRG_TRY(h.pa.check_bounds(h.pk_psi.bytes, h.pk_R.bytes, 0, h.t_img_bytes));
        DMRG_TRY(h.pb.check_bounds(h.pk_L.bytes, h.t_img_bytes, ket.size, 0));
        DMRG_TRY(h.pk_psi.finalize(st));
        DMRG_TRY(h.pk_L.finalize(st));
        DMRG_TRY(h.pk_R.finalize(st));
        DMRG_TRY(h.pa.finalize(st, h.ctx->num_sms));
        DMRG_TRY(h.pb.finalize(st, h.ctx->num_sms));
        DMRG_TRY(h.img_psi.alloc((size_t)std::max<int64_t>(h.pk_psi.bytes, 16)));
        DMRG_TRY(h.img_L.alloc((size_t)std::max<int64_t>(h.pk_L.bytes, 16)));
        DMRG_TRY(h.img_R.alloc((size_t)std::max<int64_t>(h.pk_R.bytes, 16)));
        DMRG_TRY(h.img_T.alloc((size_t)std::max<int64_t>(h.t_img_bytes, 16)));
    }
    DMRG_TRY(h.T.alloc((size_t)std::max<int64_t>(h.t_size, 1) * sizeof(double)));
    return DMRG_OK;
}

}  // namespace

int dmrg::heff_apply_fp64(dmrg_heff_s& h, const double* psi, double* out, bool accumulate) {
    if ((!h.L_dev && h.L.size) || (!h.R_dev && h.R.size))
        return set_error(DMRG_E_STATE, "dmrg_heff_set_env was not called");
    cudaStream_t st = h.ctx->stream;
    if (!accumulate && h.site.ket.size)
        DMRG_CUDA_TRY(cudaMemsetAsync(out, 0, (size_t)h.site.ket.size * sizeof(double), st));
    DMRG_TRY(launch_gemm_f64(h.sa, psi, h.R_dev, h.T.as<double>(), false, st));
    DMRG_TRY(launch_gemm_f64(h.sb, h.L_dev, h.T.as<double>(), out, true, st));
    return DMRG_OK;
}

int dmrg::heff_apply_internal(dmrg_heff_s& h, const double* psi, double* out, bool accumulate) {
    if (!is_split(h.precision)) return heff_apply_fp64(h, psi, out, accumulate);
    if ((!h.L_dev && h.L.size) || (!h.R_dev && h.R.size))
        return set_error(DMRG_E_STATE, "dmrg_heff_set_env was not called");
    cudaStream_t st = h.ctx->stream;
    if (!accumulate && h.site.ket.size)
        DMRG_CUDA_TRY(cudaMemsetAsync(out, 0, (size_t)h.site.ket.size * sizeof(double), st));
    DMRG_TRY(launch_pack(h.pk_psi, psi, h.img_psi.as<unsigned char>(), st));
    DMRG_TRY(launch_gemm_split(h.pa, h.img_psi.as<unsigned char>(), h.img_R.as<unsigned char>(), nullptr,
                                h.img_T.as<unsigned char>(), false, h.ctx->d_status, st));
    DMRG_TRY(launch_gemm_split(h.pb, h.img_L.as<unsigned char>(), h.img_T.as<unsigned char>(), out, nullptr, true,
                                h.ctx->d_status, st));
    return DMRG_OK;
}

extern "C" {

static int heff_create(dmrg_ctx_t ctx, int nl, int nr, const int* phys, bool per_block, const dmrg_blocks_t* ket,
                       int d, int lb, int rb, const double* W, const dmrg_blocks_t* L, const dmrg_blocks_t* R,
                       int precision, dmrg_heff_t* out) {
    if (!ctx || !out || !L || !R) return set_error(DMRG_E_ARG, "null argument");
    if (precision != DMRG_PREC_FP64 && !is_split(precision))
        return set_error(DMRG_E_ARG, "unsupported precision %d (DMRG_PREC_FP64, _TF32X3 or _BF16X3)", precision);
    *out = nullptr;
    DMRG_CUDA_TRY(cudaSetDevice(ctx->device));
    auto* h = new dmrg_heff_s();
    h->ctx = ctx;
    h->precision = precision;
    if (const char* g = std::getenv("DMRG_LANCZOS_GRAPH")) h->use_graph = std::atoi(g) != 0;  // A/B switch
    int rc = per_block ? build_site_desc_blocks(h->site, nl, nr, phys, ket, d, lb, rb, W)
                       : build_site_desc(h->site, nl, nr, phys, ket, d, lb, rb, W);
    if (rc == DMRG_OK && !h->L.assign(L, lb)) rc = set_error(DMRG_E_ARG, "invalid L block lists");
    if (rc == DMRG_OK && !h->R.assign(R, rb)) rc = set_error(DMRG_E_ARG, "invalid R block lists");
    if (rc == DMRG_OK) rc = build_heff(*h);
    if (rc != DMRG_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return DMRG_OK;
}

int dmrg_heff_create(dmrg_ctx_t ctx, int nl, int nr, const int* phys, const dmrg_blocks_t* ket, int d, int lb,
                     int rb, const double* W, const dmrg_blocks_t* L, const dmrg_blocks_t* R, int precision,
                     dmrg_heff_t* out) {
    return heff_create(ctx, nl, nr, phys, false, ket, d, lb, rb, W, L, R, precision, out);
}

int dmrg_heff_create_blocks(dmrg_ctx_t ctx, int nl, int nr, const int* block_phys, const dmrg_blocks_t* ket, int d,
                            int lb, int rb, const double* W, const dmrg_blocks_t* L, const dmrg_blocks_t* R,
                            int precision, dmrg_heff_t* out) {
    return heff_create(ctx, nl, nr, block_phys, true, ket, d, lb, rb, W, L, R, precision, out);
}

int dmrg_heff_destroy(dmrg_heff_t h) {
    delete h;
    return DMRG_OK;
}

int dmrg_heff_sizes(dmrg_heff_t h, int64_t* psi_dim, int64_t* lsize, int64_t* rsize) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    if (psi_dim) *psi_dim = h->site.ket.size;
    if (lsize) *lsize = h->L.size;
    if (rsize) *rsize = h->R.size;
    return DMRG_OK;
}

int dmrg_heff_flops(dmrg_heff_t h, double* alg, double* exec) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    if (alg) *alg = h->flops_alg;
    if (exec) *exec = h->flops_exec;
    return DMRG_OK;
}

int dmrg_heff_set_env(dmrg_heff_t h, const double* L_dev, const double* R_dev) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    if ((!L_dev && h->L.size) || (!R_dev && h->R.size)) return set_error(DMRG_E_ARG, "null environment pointer");
    h->L_dev = L_dev;
    h->R_dev = R_dev;
    if (is_split(h->precision)) {  // environment images, kept until the next call
        DMRG_TRY(launch_pack(h->pk_L, L_dev, h->img_L.as<unsigned char>(), h->ctx->stream));
        DMRG_TRY(launch_pack(h->pk_R, R_dev, h->img_R.as<unsigned char>(), h->ctx->stream));
    }
    return DMRG_OK;
}

int dmrg_heff_apply(dmrg_heff_t h, const double* psi, double* out, int accumulate) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    return heff_apply_internal(*h, psi, out, accumulate != 0);
}

int dmrg_heff_profile(dmrg_heff_t h, const double* psi, double* out, double* ms_stage_a, double* ms_stage_b) {
    if (!h || !ms_stage_a || !ms_stage_b) return set_error(DMRG_E_ARG, "null argument");
    if ((!h->L_dev && h->L.size) || (!h->R_dev && h->R.size))
        return set_error(DMRG_E_STATE, "dmrg_heff_set_env was not called");
    cudaStream_t st = h->ctx->stream;
    cudaEvent_t ev[3];
    for (auto& e : ev) DMRG_CUDA_TRY(cudaEventCreate(&e));
    const bool split = is_split(h->precision);
    DMRG_CUDA_TRY(cudaEventRecord(ev[0], st));
    int rc = DMRG_OK;
    if (split) {  // stage A includes packing psi
        rc = launch_pack(h->pk_psi, psi, h->img_psi.as<unsigned char>(), st);
        if (rc == DMRG_OK)
            rc = launch_gemm_split(h->pa, h->img_psi.as<unsigned char>(), h->img_R.as<unsigned char>(), nullptr,
                                    h->img_T.as<unsigned char>(), false, h->ctx->d_status, st);
    } else {
        rc = launch_gemm_f64(h->sa, psi, h->R_dev, h->T.as<double>(), false, st);
    }
    cudaEventRecord(ev[1], st);
    if (rc == DMRG_OK)
        rc = split ? launch_gemm_split(h->pb, h->img_L.as<unsigned char>(), h->img_T.as<unsigned char>(), out,
                                        nullptr, true, h->ctx->d_status, st)
                   : launch_gemm_f64(h->sb, h->L_dev, h->T.as<double>(), out, true, st);
    cudaEventRecord(ev[2], st);
    cudaError_t err = cudaEventSynchronize(ev[2]);
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, ev[0], ev[1]);
    cudaEventElapsedTime(&b, ev[1], ev[2]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc != DMRG_OK) return rc;
    if (err != cudaSuccess) return set_error(DMRG_E_CUDA, "profile: %s", cudaGetErrorString(err));
    *ms_stage_a = a;
    *ms_stage_b = b;
    return DMRG_OK;
}

int dmrg_heff_apply_host(dmrg_heff_t h, const double* psi_host, double* out_host, int accumulate) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    const size_t bytes = (size_t)h->site.ket.size * sizeof(double);
    DMRG_TRY(h->io_psi.alloc(std::max<size_t>(bytes, 8)));
    DMRG_TRY(h->io_out.alloc(std::max<size_t>(bytes, 8)));
    cudaStream_t st = h->ctx->stream;
    if (bytes) {
        DMRG_CUDA_TRY(cudaMemcpyAsync(h->io_psi.ptr, psi_host, bytes, cudaMemcpyHostToDevice, st));
        if (accumulate) DMRG_CUDA_TRY(cudaMemcpyAsync(h->io_out.ptr, out_host, bytes, cudaMemcpyHostToDevice, st));
    }
    DMRG_TRY(dmrg_heff_apply(h, h->io_psi.as<double>(), h->io_out.as<double>(), accumulate));
    if (bytes) DMRG_CUDA_TRY(cudaMemcpyAsync(out_host, h->io_out.ptr, bytes, cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    if (is_split(h->precision)) return take_device_status(h->ctx);  // bounded tensor-core waits
    return DMRG_OK;
}

}  // extern "C"
