// a6/a7: canonicalisation of a site tensor by per-sector SVD and truncation.
//
// Left (RealTensorLattice::LeftCanonicalTensorLattice, src/dmrg/realdmrg/
// real_tensor_lattice.cc:558-676): for every right sector r the blocks K(l, r)
// are stacked vertically (list order) into A_r (sum of rows x right_dim[r]),
// A_r = U S V^T; the truncation keeps t_r values (ComputeTruncateDim, :501-555,
// on the host with the reference's QuickSort); K(l, r) <- its rows of U[:, :t_r];
// canonical[r] = diag(S[:t_r]) V^T[:t_r, :]; right_dim[r] <- t_r.
// Right (:794-911) mirrors it: blocks K(l, .) stacked horizontally into
// A_l (left_dim[l] x sum of cols), K(l, r) <- its columns of V^T[:t_l, :],
// canonical[l] = U[:, :t_l] diag(S[:t_l]); left_dim[l] <- t_l.
// Sectors without rows (left) / columns (right) keep the reference's special
// case: one singular value 0, a zero canonical block, the ket untouched.
//
// The kept columns on the ket's side are orthonormal to FP64 rounding, as the
// reference's dgesvd gives them: where the ket side is the one the Jacobi SVD
// leaves as the working matrix's normalised columns, they are orthonormalised
// (KetOrtho, ortho.cuh) and the canonical block is the projection of the sector
// matrix on them (K^T A left, A K right), zero in the rows / columns whose
// singular value the truncation forced to 0.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <numeric>

#include "blocksparse.h"
#include "gemm.cuh"
#include "ortho.cuh"
#include "svd.cuh"
#include "truncate.h"

using namespace dmrg;

namespace {

struct CopyTask {
    int64_t blk_off;  // ket block offset
    int rows, cols;   // ket block shape
    int problem;      // svd problem index
    int off;          // row0 (left) or col0 (right) inside the stacked sector matrix
};

struct WriteTask {
    int64_t out_off;  // new ket block offset
    int rows, cols;   // new ket block shape
    int problem;
    int off;          // row0 / col0
    int64_t k_off;    // the sector's orthonormalised kept columns in the K buffer (-1: none)
};

struct CanonTask {
    int64_t out_off;
    int rows, cols;   // canonical block shape
    int problem;      // -1: zero block
    int64_t sig_off;  // offset of the forced singular values of this sector
    int projected;    // 1: written as a projection (GEMM), only the forced zeros here
    int pad_;
};

// The kernels below move blocks in 32x32 tiles, one tile per CTA of 256
// threads (grid y = the block's tile, CTAs beyond a block's tiles return), so
// that both the row-major ket / canonical blocks and the column-major working
// matrices are read and written along their contiguous direction (a transpose
// goes through shared memory).
constexpr int kTile = 32;
__host__ __device__ inline int tiles_of(int rows, int cols) {
    return ((rows + kTile - 1) / kTile) * ((cols + kTile - 1) / kTile);
}

// Writes tile blockIdx.y of the row-major rows x cols block at out (ld cols):
// element (i, j) = value(i, j).  With `down` the source is contiguous along i
// (a column-major matrix): lanes read along i into shared memory and write
// along j.
template <class F>
__device__ __forceinline__ void write_tile(double* __restrict__ out, int rows, int cols, bool down, F value) {
    __shared__ double tile[kTile][kTile + 1];
    const int tc = (cols + kTile - 1) / kTile;
    const int i0 = (blockIdx.y / tc) * kTile, j0 = (blockIdx.y % tc) * kTile;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    if (down) {
        for (int c = ty; c < kTile; c += 8) {
            const int i = i0 + tx, j = j0 + c;
            tile[tx][c] = (i < rows && j < cols) ? value(i, j) : 0.0;
        }
        __syncthreads();
        for (int r = ty; r < kTile; r += 8) {
            const int i = i0 + r, j = j0 + tx;
            if (i < rows && j < cols) out[(int64_t)i * cols + j] = tile[r][tx];
        }
    } else {
        for (int r = ty; r < kTile; r += 8) {
            const int i = i0 + r, j = j0 + tx;
            if (i < rows && j < cols) out[(int64_t)i * cols + j] = value(i, j);
        }
    }
}

// gather: stacked A (m x n) into W (column-major; W = A or W = A^T).  Tile
// blockIdx.y of ket block blockIdx.x; block element (i, j) is A(ai, aj) with
// ai = off + i, aj = j (left) or ai = i, aj = off + j (right).
__global__ void __launch_bounds__(256) gather_kernel(const double* __restrict__ ket, const CopyTask* __restrict__ tasks,
                                                     const SvdProblem* __restrict__ probs, double* __restrict__ W,
                                                     int side) {
    __shared__ double tile[kTile][kTile + 1];
    const CopyTask t = tasks[blockIdx.x];
    if ((int)blockIdx.y >= tiles_of(t.rows, t.cols)) return;
    const SvdProblem p = probs[t.problem];
    const double* src = ket + t.blk_off;
    double* w = W + p.w_off;
    const int tc = (t.cols + kTile - 1) / kTile;
    const int i0 = (blockIdx.y / tc) * kTile, j0 = (blockIdx.y % tc) * kTile;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < kTile; r += 8) {
        const int i = i0 + r, j = j0 + tx;
        tile[r][tx] = (i < t.rows && j < t.cols) ? src[(int64_t)i * t.cols + j] : 0.0;
    }
    __syncthreads();
    if (p.transposed) {  // W = A^T: w[ai * n + aj], contiguous along the block's columns
        for (int r = ty; r < kTile; r += 8) {
            const int i = i0 + r, j = j0 + tx;
            const int ai = side == 0 ? t.off + i : i, aj = side == 0 ? j : t.off + j;
            if (i < t.rows && j < t.cols && ai < p.m && aj < p.n) w[(int64_t)ai * p.n + aj] = tile[r][tx];
        }
    } else {  // W = A: w[aj * m + ai], contiguous along the block's rows
        for (int c = ty; c < kTile; c += 8) {
            const int i = i0 + tx, j = j0 + c;
            const int ai = side == 0 ? t.off + i : i, aj = side == 0 ? j : t.off + j;
            if (i < t.rows && j < t.cols && ai < p.m && aj < p.n) w[(int64_t)aj * p.m + ai] = tile[tx][c];
        }
    }
}

// new ket blocks: left -> rows of U[:, :t]; right -> columns of V^T[:t, :]
__global__ void __launch_bounds__(256) write_ket_kernel(const WriteTask* __restrict__ tasks,
                                                        const SvdProblem* __restrict__ probs,
                                                        const double* __restrict__ W, const double* __restrict__ Q,
                                                        const double* __restrict__ sig, const int* __restrict__ perm,
                                                        const double* __restrict__ sgn, const double* __restrict__ K,
                                                        double* __restrict__ out, int side) {
    const WriteTask t = tasks[blockIdx.x];
    if ((int)blockIdx.y >= tiles_of(t.rows, t.cols)) return;
    const SvdProblem p = probs[t.problem];
    const double* w = W + p.w_off;
    const double* q = Q + p.q_off;
    double* o = out + t.out_off;
    // left: U columns are contiguous along the block's rows; right: V columns along its columns
    const bool down = side == 0;
    if (t.k_off >= 0) {  // orthonormalised columns: U[row0 + i][j] (left) or V^T[i][col0 + j] (right)
        const double* k = K + t.k_off;
        write_tile(o, t.rows, t.cols, down, [&](int i, int j) {
            return side == 0 ? k[(int64_t)j * p.rows + t.off + i] : k[(int64_t)i * p.rows + t.off + j];
        });
        return;
    }
    write_tile(o, t.rows, t.cols, down, [&](int i, int j) {
        double v;
        if (side == 0) {  // U[row0 + i][j]
            const int kc = perm[p.perm_off + j];
            const int row = t.off + i;
            if (!p.transposed) {
                const double s = sig[p.s_off + j];
                v = s > 0.0 ? w[(int64_t)kc * p.m + row] / s : 0.0;
            } else {
                v = q[(int64_t)kc * p.m + row];
            }
            v *= sgn[p.s_off + j];
        } else {  // V^T[i][col0 + j] = v_i[col0 + j]
            const int kc = perm[p.perm_off + i];
            const int col = t.off + j;
            if (!p.transposed) {
                v = q[(int64_t)kc * p.n + col];
            } else {
                const double s = sig[p.s_off + i];
                v = s > 0.0 ? w[(int64_t)kc * p.n + col] / s : 0.0;
            }
            v *= sgn[p.s_off + i];
        }
        return v;
    });
}

// canonical blocks: left -> diag(s_forced) V^T[:t, :] (t x n); right -> U[:, :t] diag(s_forced) (m x t)
__global__ void __launch_bounds__(256) write_canonical_kernel(const CanonTask* __restrict__ tasks,
                                                              const SvdProblem* __restrict__ probs,
                                                              const double* __restrict__ W, const double* __restrict__ Q,
                                                              const double* __restrict__ sig, const int* __restrict__ perm,
                                                              const double* __restrict__ forced,
                                                              const double* __restrict__ sgn, double* __restrict__ out,
                                                              int side) {
    const CanonTask t = tasks[blockIdx.x];
    if ((int)blockIdx.y >= tiles_of(t.rows, t.cols)) return;
    double* o = out + t.out_off;
    const int tc = (t.cols + kTile - 1) / kTile;
    const int i0 = (blockIdx.y / tc) * kTile, j0 = (blockIdx.y % tc) * kTile;
    if (t.problem < 0 || t.projected) {
        // a zero block; or one that is K^T A / A K already: zero the rows / columns forced to 0
        for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
            const int i = i0 + e / kTile, j = j0 + e % kTile;
            if (i >= t.rows || j >= t.cols) continue;
            if (t.problem < 0 || forced[t.sig_off + (side == 0 ? i : j)] == 0.0) o[(int64_t)i * t.cols + j] = 0.0;
        }
        return;
    }
    const SvdProblem p = probs[t.problem];
    const double* w = W + p.w_off;
    const double* q = Q + p.q_off;
    // left: rows of V^T are contiguous along the block's columns; right: U columns along its rows
    write_tile(o, t.rows, t.cols, side == 1, [&](int i, int j) {
        double v;
        if (side == 0) {  // s_i * v_i[j]
            const int kc = perm[p.perm_off + i];
            const double sf = forced[t.sig_off + i];
            if (!p.transposed) {
                v = sf * q[(int64_t)kc * p.n + j];
            } else {
                const double s = sig[p.s_off + i];
                v = s > 0.0 ? sf * w[(int64_t)kc * p.n + j] / s : 0.0;
            }
            v *= sgn[p.s_off + i];
        } else {  // u_j[i] * s_j
            const int kc = perm[p.perm_off + j];
            const double sf = forced[t.sig_off + j];
            if (!p.transposed) {
                const double s = sig[p.s_off + j];
                v = s > 0.0 ? sf * w[(int64_t)kc * p.m + i] / s : 0.0;
            } else {
                v = sf * q[(int64_t)kc * p.m + i];
            }
            v *= sgn[p.s_off + j];
        }
        return v;
    });
}

}  // namespace

struct dmrg_canon_s {
    dmrg_ctx_t ctx = nullptr;
    int side = 0;
    int nl = 0, nr = 0;
    std::vector<int> left_dim, right_dim;
    BlockListDesc ket;
    int nsec = 0;
    std::vector<std::vector<int>> members;  // ket positions of each sector, list order
    std::vector<int> sec_m, sec_n;          // stacked shape of each sector
    BatchedSvd svd;
    std::vector<CopyTask> copies;
    DeviceBuffer d_copies, d_writes, d_canons, d_forced;
    int gather_tiles = 1, write_tiles = 1, canon_tiles = 1;  // grid y of the tile kernels
    // orthonormalisation of the kept ket columns taken from the working matrix
    KetOrtho ortho;
    DeviceBuffer d_a;                       // the sector matrices again (working-matrix layout)
    GemmSchedule sc;                        // the projected canonical blocks
    // results
    bool ran = false;
    std::vector<std::vector<double>> sv;  // singular values per sector (reference semantics)
    std::vector<int> tdim;
    BlockListDesc new_ket, canonical;
    std::vector<int> match_dim;
    double discarded = 0.0;
    int sweeps = 0;
};

namespace {

// The orthonormalisation of a run (sectors whose ket side is the working
// matrix's columns) and the GEMM schedule of the projected canonical blocks.
int plan_ortho(dmrg_canon_s* c, cudaStream_t st) {
    BatchedSvd& svd = c->svd;
    std::vector<int> kept(svd.probs.size(), 0);
    std::vector<std::vector<double>> sv(svd.probs.size());
    int64_t wsz = 0;
    for (const SvdProblem& p : svd.probs) wsz += (int64_t)p.rows * p.cols;
    for (int sct = 0; sct < c->nsec; ++sct) {
        if (!svd.active(sct)) continue;
        const SvdProblem& p = svd.problem(sct);
        const bool wside = c->side == 0 ? !p.transposed : p.transposed != 0;
        if (!wside || c->tdim[sct] <= 0) continue;
        kept[svd.index[sct]] = c->tdim[sct];
        sv[svd.index[sct]] = c->sv[sct];
    }
    DMRG_TRY(c->ortho.plan(svd, kept, sv, st, c->ctx->num_sms));
    if (c->ortho.empty()) return DMRG_OK;
    DMRG_TRY(c->d_a.alloc(std::max<int64_t>(wsz, 1) * sizeof(double)));
    GemmSchedule& sc = c->sc;
    sc.reset();
    sc.tb = true;
    for (int sct = 0; sct < c->nsec; ++sct) {
        if (!svd.active(sct)) continue;
        const int pi = svd.index[sct];
        const int64_t ko = c->ortho.k_off(pi);
        if (ko < 0) continue;
        const SvdProblem& p = svd.probs[pi];
        const int t = c->tdim[sct];
        if (c->side == 0) {
            // C (t x n) = K^T A; A (m x n) is held column-major (W layout), i.e. the transposed B
            sc.add_group(c->canonical.off[sct], p.n, t, p.n);
            sc.add_term(ko, p.rows, p.w_off, p.rows, p.rows, 1.0);
        } else {
            // C (m x t) = A K; A is held as A^T column-major = A row-major (ld n); K the transposed B
            sc.add_group(c->canonical.off[sct], t, p.m, t);
            sc.add_term(p.w_off, p.rows, ko, p.rows, p.rows, 1.0);
        }
    }
    const int64_t ksz = c->ortho.k_size();
    if (c->side == 0)
        DMRG_TRY(sc.check_bounds(ksz, wsz, c->canonical.size));
    else
        DMRG_TRY(sc.check_bounds(wsz, ksz, c->canonical.size));
    DMRG_TRY(sc.finalize(64, 64, 16, st, c->ctx->num_sms));
    return DMRG_OK;
}

// Orthonormalised ket columns and the projected canonical blocks.
int run_ortho(dmrg_canon_s* c, const double* ket_dev, double* canonical_dev, cudaStream_t st) {
    if (c->ortho.empty()) return DMRG_OK;
    BatchedSvd& svd = c->svd;
    DMRG_CUDA_TRY(cudaMemsetAsync(c->d_a.ptr, 0, c->d_a.bytes, st));
    if (!c->copies.empty())
        DMRG_LAUNCH gather_kernel<<<dim3((int)c->copies.size(), c->gather_tiles), 256, 0, st>>>(
            ket_dev, c->d_copies.as<CopyTask>(), svd.d_probs.as<SvdProblem>(), c->d_a.as<double>(), c->side);
    DMRG_CUDA_TRY(cudaGetLastError());
    DMRG_TRY(c->ortho.run(svd, st));
    if (c->side == 0)
        DMRG_TRY(launch_gemm_f64(c->sc, c->ortho.k(), c->d_a.as<double>(), canonical_dev, false, st));
    else
        DMRG_TRY(launch_gemm_f64(c->sc, c->d_a.as<double>(), c->ortho.k(), canonical_dev, false, st));
    return DMRG_OK;
}

}  // namespace

extern "C" {

int dmrg_canon_create(dmrg_ctx_t ctx, int side, int nl, int nr, const int* left_dim, const int* right_dim,
                      const dmrg_blocks_t* ket, dmrg_canon_t* out) {
    if (!ctx || !out || !ket || !left_dim || !right_dim || nl <= 0 || nr <= 0 || (side != 0 && side != 1))
        return set_error(DMRG_E_ARG, "invalid canonicalisation arguments");
    *out = nullptr;
    DMRG_CUDA_TRY(cudaSetDevice(ctx->device));
    auto* c = new dmrg_canon_s();
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
    c->nsec = side == 0 ? nr : nl;
    c->members = c->ket.by_sector(side == 0 ? 1 : 0, c->nsec);
    c->sec_m.assign(c->nsec, 0);
    c->sec_n.assign(c->nsec, 0);
    for (int s = 0; s < c->nsec; ++s) {
        int acc = 0;
        for (int p : c->members[s]) acc += side == 0 ? c->ket.rows[p] : c->ket.cols[p];
        if (side == 0) {
            c->sec_m[s] = acc;
            c->sec_n[s] = c->right_dim[s];
        } else {
            c->sec_m[s] = c->left_dim[s];
            c->sec_n[s] = acc;
        }
    }
    for (int k = 0; k < c->ket.count(); ++k) {
        const int l = c->ket.left[k], r = c->ket.right[k];
        if (l < 0 || l >= nl || r < 0 || r >= nr) {
            delete c;
            return set_error(DMRG_E_ARG, "ket block %d sectors out of range", k);
        }
    }
    int rc = c->svd.plan(c->sec_m, c->sec_n, ctx->stream);
    if (rc == DMRG_OK) {
        for (int s = 0; s < c->nsec; ++s) {
            if (!c->svd.active(s)) continue;
            int acc = 0;
            for (int p : c->members[s]) {
                c->copies.push_back(CopyTask{c->ket.off[p], c->ket.rows[p], c->ket.cols[p], c->svd.index[s], acc});
                c->gather_tiles = std::max(c->gather_tiles, tiles_of(c->ket.rows[p], c->ket.cols[p]));
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

int dmrg_canon_destroy(dmrg_canon_t c) {
    delete c;
    return DMRG_OK;
}

int dmrg_canon_run(dmrg_canon_t c, const double* ket_dev, int max_dim, double canpre, int* tdim_out,
                   double* discarded) {
    if (!c || (!ket_dev && c->ket.size)) return set_error(DMRG_E_ARG, "null argument");
    cudaStream_t st = c->ctx->stream;
    BatchedSvd& svd = c->svd;
    if (!svd.probs.empty()) {
        int64_t wsize = 0;
        for (const auto& p : svd.probs) wsize += (int64_t)p.rows * p.cols;
        DMRG_CUDA_TRY(cudaMemsetAsync(svd.d_w.ptr, 0, wsize * sizeof(double), st));
        if (!c->copies.empty())
            DMRG_LAUNCH gather_kernel<<<dim3((int)c->copies.size(), c->gather_tiles), 256, 0, st>>>(ket_dev, c->d_copies.as<CopyTask>(),
                                                                 svd.d_probs.as<SvdProblem>(), svd.d_w.as<double>(),
                                                                 c->side);
        DMRG_CUDA_TRY(cudaGetLastError());
        DMRG_TRY(svd.run(st, &c->sweeps));
    }
    std::vector<std::vector<double>> s;
    DMRG_TRY(svd.singular_values(s, st));
    // reference semantics for empty sectors: singular_dim = 1, value 0
    for (int i = 0; i < c->nsec; ++i)
        if (!svd.active(i)) s[i].assign(1, 0.0);
    c->sv = s;
    c->tdim = compute_truncate_dim(max_dim, canpre, s);  // s is modified (forced zeros)
    // discarded weight: everything except the kept (possibly forced-to-zero) values
    double all = 0.0, kept = 0.0;
    for (int i = 0; i < c->nsec; ++i) {
        for (double v : c->sv[i]) all += v * v;
        for (int j = 0; j < c->tdim[i] && j < (int)s[i].size(); ++j) kept += s[i][j] * s[i][j];
    }
    c->discarded = all - kept;
    // new shapes
    c->new_ket = BlockListDesc();
    for (int k = 0; k < c->ket.count(); ++k) {
        const int l = c->ket.left[k], r = c->ket.right[k];
        if (c->side == 0) {
            const bool touched = svd.active(r);
            c->new_ket.push(l, r, c->ket.rows[k], touched ? c->tdim[r] : c->ket.cols[k]);
        } else {
            const bool touched = svd.active(l);
            c->new_ket.push(l, r, touched ? c->tdim[l] : c->ket.rows[k], c->ket.cols[k]);
        }
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
    // forced singular values (device) for the canonical blocks
    std::vector<double> forced;
    std::vector<CanonTask> ctasks;
    for (int sct = 0; sct < c->nsec; ++sct) {
        CanonTask t{c->canonical.off[sct], c->canonical.rows[sct], c->canonical.cols[sct],
                    svd.active(sct) ? svd.index[sct] : -1, (int64_t)forced.size(), 0, 0};
        for (int i = 0; i < c->tdim[sct]; ++i) forced.push_back(i < (int)s[sct].size() ? s[sct][i] : 0.0);
        ctasks.push_back(t);
    }
    DMRG_TRY(plan_ortho(c, st));
    for (CanonTask& t : ctasks)
        if (t.problem >= 0 && c->ortho.k_off(t.problem) >= 0) t.projected = 1;
    std::vector<WriteTask> wtasks;
    for (int sct = 0; sct < c->nsec; ++sct) {
        if (!svd.active(sct)) continue;
        int acc = 0;
        for (int p : c->members[sct]) {
            wtasks.push_back(WriteTask{c->new_ket.off[p], c->new_ket.rows[p], c->new_ket.cols[p], svd.index[sct], acc,
                                       c->ortho.k_off(svd.index[sct])});
            acc += c->side == 0 ? c->ket.rows[p] : c->ket.cols[p];
        }
    }
    c->write_tiles = c->canon_tiles = 1;
    for (const WriteTask& w : wtasks) c->write_tiles = std::max(c->write_tiles, tiles_of(w.rows, w.cols));
    for (const CanonTask& t : ctasks) c->canon_tiles = std::max(c->canon_tiles, tiles_of(t.rows, t.cols));
    DMRG_TRY(upload(c->d_forced, forced, st));
    DMRG_TRY(upload(c->d_canons, ctasks, st));
    DMRG_TRY(upload(c->d_writes, wtasks, st));
    c->ran = true;
    return DMRG_OK;
}

int dmrg_canon_out_info(dmrg_canon_t c, int64_t* ket_size, int64_t* canonical_size, int* sweeps) {
    if (!c || !c->ran) return set_error(DMRG_E_STATE, "dmrg_canon_run has not been called");
    if (ket_size) *ket_size = c->new_ket.size;
    if (canonical_size) *canonical_size = c->canonical.size;
    if (sweeps) *sweeps = c->sweeps;
    return DMRG_OK;
}

int dmrg_canon_out_blocks(dmrg_canon_t c, int* ket_rows, int* ket_cols, int* canon_rows, int* canon_cols,
                          int* match_dim) {
    if (!c || !c->ran) return set_error(DMRG_E_STATE, "dmrg_canon_run has not been called");
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

int dmrg_canon_singular_values(dmrg_canon_t c, int sector, int cap, double* values, int* count) {
    if (!c || !c->ran || !count) return set_error(DMRG_E_STATE, "dmrg_canon_run has not been called");
    if (sector < 0 || sector >= c->nsec) return set_error(DMRG_E_ARG, "sector %d out of range", sector);
    const auto& s = c->sv[sector];
    *count = (int)s.size();
    if (values)
        for (int i = 0; i < (int)s.size() && i < cap; ++i) values[i] = s[i];
    return DMRG_OK;
}

int dmrg_canon_write(dmrg_canon_t c, const double* ket_dev, double* new_ket_dev, double* canonical_dev) {
    if (!c || !c->ran) return set_error(DMRG_E_STATE, "dmrg_canon_run has not been called");
    cudaStream_t st = c->ctx->stream;
    BatchedSvd& svd = c->svd;
    // blocks of untouched (empty) sectors keep their values
    for (int s = 0; s < c->nsec; ++s) {
        if (svd.active(s)) continue;
        for (int p : c->members[s]) {
            const size_t bytes = (size_t)c->ket.rows[p] * c->ket.cols[p] * sizeof(double);
            if (bytes)
                DMRG_CUDA_TRY(cudaMemcpyAsync(new_ket_dev + c->new_ket.off[p], ket_dev + c->ket.off[p], bytes,
                                              cudaMemcpyDeviceToDevice, st));
        }
    }
    const int nw = (int)(c->d_writes.bytes / sizeof(WriteTask));
    int n_writes = 0;
    for (int s = 0; s < c->nsec; ++s)
        if (svd.active(s)) n_writes += (int)c->members[s].size();
    (void)nw;
    const double* sig = svd.d_s.as<double>();
    DMRG_TRY(run_ortho(c, ket_dev, canonical_dev, st));
    if (n_writes)
        DMRG_LAUNCH write_ket_kernel<<<dim3(n_writes, c->write_tiles), 256, 0, st>>>(c->d_writes.as<WriteTask>(), svd.d_probs.as<SvdProblem>(),
                                                   svd.d_w.as<double>(), svd.d_q.as<double>(), sig,
                                                   svd.d_perm.as<int>(), svd.d_sign.as<double>(),
                                                   c->ortho.k(), new_ket_dev, c->side);
    DMRG_LAUNCH write_canonical_kernel<<<dim3(c->nsec, c->canon_tiles), 256, 0, st>>>(c->d_canons.as<CanonTask>(), svd.d_probs.as<SvdProblem>(),
                                                    svd.d_w.as<double>(), svd.d_q.as<double>(), sig,
                                                    svd.d_perm.as<int>(), c->d_forced.as<double>(),
                                                    svd.d_sign.as<double>(), canonical_dev, c->side);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // extern "C"
