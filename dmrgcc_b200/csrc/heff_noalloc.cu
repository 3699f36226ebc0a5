// H_eff * psi for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs inside a
// host framework owning every device allocation (a memory pool with a hard
// budget), or a solver loop that must not allocate between its own setup and
// teardown.  dmrg_heff_apply_noalloc gives them the block-sparse H_eff * psi of
// dmrg_heff_apply without a dmrg_heff_t object and without any allocation:
// the grouped-GEMM schedule and the K*R intermediate live in one file-scope
// device array of kNoAllocScratchBytes, filled through cudaMemcpyAsync, and the
// schedule is assembled on the host in a static staging area of the same size.
//
// The device array exists once per GPU that loads the library and stays until
// the process exits.  Every call reuses it and leaves the previous call's
// contents behind (nothing in it needs to start at zero: the intermediate is
// overwritten by the first launch).  Calls that overlap on the GPU race on that
// array.  This function itself keeps its calls apart: a mutex guards the host
// staging area and is held until the call's own stream has finished the call's
// work, so calls from different host threads run one after the other, device
// work included; only work that reaches the array by other means can overlap.
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call before
// any stream capture.  The address is kept for the life of the process, so the
// library must not be used across a cudaDeviceReset of that device.
//
// Every argument is validated on the host before any CUDA call: sector indices
// of the ket, L and R blocks inside their sector ranges, each ket block's
// physics index inside [0, d), no negative shape.  A malformed table returns
// DMRG_E_ARG, like dmrg_heff_create.
#include <cmath>
#include <cstring>
#include <mutex>

#include "blocksparse.h"
#include "gemm.cuh"

namespace dmrg {
int launch_gemm_f64_tables(const GemmTerm* terms, const GemmGroup* groups, const GemmTile* tiles, int ntiles,
                           bool ta, bool tb, const double* A, const double* B, double* C, bool accumulate,
                           cudaStream_t st);
}

using namespace dmrg;

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;  // 16 MiB
constexpr int kMaxDevices = 64;
constexpr int kMaxOutBlocks = 4096;
constexpr int kMaxEnvBlocks = 1 << 16;  // blocks of all MPO bond indices of one environment
constexpr int kMaxBond = 512;
constexpr int kTile = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

unsigned char* g_scratch_addr[kMaxDevices] = {};
std::mutex g_mutex;
alignas(256) unsigned char g_staging[kNoAllocScratchBytes];  // host image of the tables
struct PendingTerm {
    int out_pos;
    GemmTerm term;
};
PendingTerm g_pending[kNoAllocScratchBytes / sizeof(PendingTerm) / 4];
int g_count[kMaxOutBlocks + 1];
// packed offsets (doubles) of every ket block and of every L / R block, bond by
// bond (the blocks of bond o start at index first[o]); filled once per call
int64_t g_ket_off[kMaxOutBlocks + 1];
int64_t g_L_off[kMaxEnvBlocks + 1], g_R_off[kMaxEnvBlocks + 1];
int g_L_first[kMaxBond + 1], g_R_first[kMaxBond + 1];

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Host view of the argument block lists (no copies).
struct View {
    int n;
    const int *left, *right, *rows, *cols;
};

View view(const dmrg_blocks_t& b) { return View{b.nblocks, b.left, b.right, b.rows, b.cols}; }

// Checks one block list: count, non-null arrays, sector indices in [0, nsec)
// on both sides, no negative shape.
bool valid_list(const dmrg_blocks_t& b, int nsec_left, int nsec_right) {
    if (b.nblocks < 0) return false;
    if (b.nblocks > 0 && (!b.left || !b.right || !b.rows || !b.cols)) return false;
    for (int k = 0; k < b.nblocks; ++k)
        if (b.left[k] < 0 || b.left[k] >= nsec_left || b.right[k] < 0 || b.right[k] >= nsec_right || b.rows[k] < 0 ||
            b.cols[k] < 0)
            return false;
    return true;
}

// Packed offsets of the blocks of `n` consecutive lists into off[first[o] + q];
// returns the total size, or -1 when more than `cap` blocks.
int64_t list_offsets(const dmrg_blocks_t* lists, int n, int64_t* off, int* first, int cap) {
    int64_t acc = 0;
    int idx = 0;
    for (int o = 0; o < n; ++o) {
        first[o] = idx;
        if (idx + lists[o].nblocks > cap) return -1;
        for (int q = 0; q < lists[o].nblocks; ++q) {
            off[idx++] = acc;
            acc += (int64_t)lists[o].rows[q] * lists[o].cols[q];
        }
    }
    first[n] = idx;
    off[idx] = acc;
    return acc;
}

int find(const View& v, int l, int r) {
    for (int k = 0; k < v.n; ++k)
        if (v.left[k] == l && v.right[k] == r) return k;
    return -1;
}

}  // namespace

extern "C" int dmrg_heff_apply_noalloc(int nl, int nr, const int* phys, const dmrg_blocks_t* ket, int d, int lb,
                                       int rb, const double* W, const dmrg_blocks_t* L, const dmrg_blocks_t* R,
                                       const double* L_dev, const double* R_dev, const double* psi_dev,
                                       double* out_dev, int accumulate, void* stream) {
    if (nl <= 0 || nr <= 0 || !phys || !ket || d <= 0 || lb <= 0 || rb <= 0 || !W || !L || !R || !psi_dev ||
        !out_dev)
        return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: null or empty argument");
    // ---- validate every table on the host, before any CUDA call -----------------------
    if (lb > kMaxBond || rb > kMaxBond)
        return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: MPO bond above %d", kMaxBond);
    if (ket->nblocks > kMaxOutBlocks)
        return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: %d ket blocks, at most %d", ket->nblocks,
                         kMaxOutBlocks);
    if (!valid_list(*ket, nl, nr))
        return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: invalid ket block list (sectors outside %dx%d)", nl,
                         nr);
    for (int k = 0; k < ket->nblocks; ++k) {
        const int p = phys[(size_t)ket->left[k] * nr + ket->right[k]];
        if (p < 0 || p >= d)
            return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: ket block %d (%d,%d) has physics index %d", k,
                             ket->left[k], ket->right[k], p);
    }
    for (int o = 0; o < lb; ++o)
        if (!valid_list(L[o], nl, nl))
            return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: L[%d] has sectors outside %d", o, nl);
    for (int o = 0; o < rb; ++o)
        if (!valid_list(R[o], nr, nr))
            return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: R[%d] has sectors outside %d", o, nr);

    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    DMRG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(DMRG_E_ARG, "device ordinal %d not supported", dev);
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(DMRG_E_CUDA, "cudaGetSymbolAddress(static scratch) failed: %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    unsigned char* scratch = g_scratch_addr[dev];

    const View K = view(*ket);
    int ket_first[2];
    list_offsets(ket, 1, g_ket_off, ket_first, kMaxOutBlocks);
    const int64_t Lsize = list_offsets(L, lb, g_L_off, g_L_first, kMaxEnvBlocks);
    const int64_t Rsize = list_offsets(R, rb, g_R_off, g_R_first, kMaxEnvBlocks);
    if (Lsize < 0 || Rsize < 0)
        return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: an environment has more than %d blocks",
                         kMaxEnvBlocks);
    auto Wat = [&](int o1, int o2, int p1, int p2) { return W[(((size_t)o1 * rb + o2) * d + p1) * d + p2]; };
    auto right_nonzero = [&](int o2, int p2) {
        for (int o1 = 0; o1 < lb; ++o1)
            for (int p1 = 0; p1 < d; ++p1)
                if (std::fabs(Wat(o1, o2, p1, p2)) > 1e-15) return true;
        return false;
    };
    // ---- walk the reference loop (real_tensor_contraction.cc:1243-1285) -------------
    // stage A groups/terms go straight to the staging area; stage B terms are
    // collected with their output block and bucketed afterwards.
    const size_t cap_pending = sizeof(g_pending) / sizeof(g_pending[0]);
    size_t nA = 0, nB = 0;
    int64_t t_size = 0;
    // pass 0 validates and counts; pass 1 records stage B terms and the stage A
    // groups (provisionally at the start of the staging area)
    for (int pass = 0; pass < 2; ++pass) {
        size_t tA = 0, tB = 0;
        int64_t toff = 0;
        for (int o2 = 0; o2 < rb; ++o2) {
            const View Ro = view(R[o2]);
            for (int i = 0; i < Ro.n; ++i) {
                const int ldx = Ro.left[i], jdx = Ro.right[i], rr = Ro.rows[i], rc = Ro.cols[i];
                if (rr == 0 || ldx < 0 || ldx >= nr || jdx < 0 || jdx >= nr) continue;
                for (int pos = 0; pos < K.n; ++pos) {
                    if (K.right[pos] != ldx) continue;
                    const int kdx = K.left[pos];
                    const int p2 = phys[(size_t)kdx * nr + ldx];
                    if (p2 < 0 || !right_nonzero(o2, p2)) continue;
                    const int a_k = K.rows[pos], b_l = K.cols[pos];
                    if (b_l != rr) return set_error(DMRG_E_ARG, "ket block %d width %d != R rows %d", pos, b_l, rr);
                    if (a_k == 0 || b_l == 0 || rc == 0) continue;
                    bool used = false;
                    for (int pos2 = 0; pos2 < K.n; ++pos2) {
                        if (K.right[pos2] != jdx) continue;
                        const int idx = K.left[pos2];
                        const int p1 = phys[(size_t)idx * nr + jdx];
                        for (int o1 = 0; o1 < lb; ++o1) {
                            const double w = Wat(o1, o2, p1, p2);
                            if (w == 0.0) continue;
                            const View Lo = view(L[o1]);
                            const int q = find(Lo, idx, kdx);
                            if (q == -1 || Lo.rows[q] == 0) continue;
                            if (Lo.cols[q] != a_k || Lo.rows[q] != K.rows[pos2] || rc != K.cols[pos2])
                                return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: inconsistent block shapes");
                            if (pass == 1) {
                                if (tB >= cap_pending)
                                    return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: more than %zu terms",
                                                     cap_pending);
                                g_pending[tB] = PendingTerm{pos2, GemmTerm{g_L_off[g_L_first[o1] + q], toff, a_k,
                                                                           rc, a_k, 0, w}};
                            }
                            ++tB;
                            used = true;
                        }
                    }
                    if (used) {
                        if (pass == 1) {
                            GemmGroup* groupsA = reinterpret_cast<GemmGroup*>(g_staging);
                            groupsA[tA] = GemmGroup{toff, rc, a_k, rc, (int)tA, (int)tA + 1, 0};
                        }
                        ++tA;
                        toff += (int64_t)a_k * rc;
                    }
                }
            }
        }
        nA = tA;
        nB = tB;
        t_size = toff;
        if (pass == 0 && nA * sizeof(GemmGroup) > kNoAllocScratchBytes)
            return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: schedule larger than the static scratch");
    }
    // stage A terms (one per group), stage B bucketed by output block in generation order
    // tiles of 64 x 64 for both stages
    auto tiles_of = [](int m, int n) { return (int64_t)((m + kTile - 1) / kTile) * ((n + kTile - 1) / kTile); };
    GemmGroup* groupsA_tmp = reinterpret_cast<GemmGroup*>(g_staging);
    int64_t ntA = 0;
    for (size_t g = 0; g < nA; ++g) ntA += tiles_of(groupsA_tmp[g].m, groupsA_tmp[g].n);
    for (int b = 0; b <= K.n; ++b) g_count[b] = 0;
    for (size_t t = 0; t < nB; ++t) ++g_count[g_pending[t].out_pos + 1];
    int nGB = 0;
    int64_t ntB = 0;
    for (int b = 0; b < K.n; ++b)
        if (g_count[b + 1]) {
            ++nGB;
            ntB += tiles_of(K.rows[b], K.cols[b]);
        }
    // region layout inside the device scratch (and the same offsets in the staging image)
    const size_t offTA = 0;
    const size_t offGA = align256(offTA + nA * sizeof(GemmTerm));
    const size_t offLA = align256(offGA + nA * sizeof(GemmGroup));
    const size_t offTB = align256(offLA + (size_t)ntA * sizeof(GemmTile));
    const size_t offGB = align256(offTB + nB * sizeof(GemmTerm));
    const size_t offLB = align256(offGB + (size_t)nGB * sizeof(GemmGroup));
    const size_t offT = align256(offLB + (size_t)ntB * sizeof(GemmTile));
    const size_t total = offT + (size_t)t_size * sizeof(double);
    if (total > kNoAllocScratchBytes)
        return set_error(DMRG_E_ARG,
                         "dmrg_heff_apply_noalloc: this problem needs %zu bytes of scratch; the static scratch holds "
                         "%zu (use dmrg_heff_create/dmrg_heff_apply)",
                         total, kNoAllocScratchBytes);
    // Build the image.  Stage A groups currently sit at offset 0: move them to offGA
    // first (offGA >= nA * sizeof(GemmTerm) > 0 when nA > 0, regions may overlap:
    // use memmove), then write the terms in front.
    if (nA) std::memmove(g_staging + offGA, g_staging, nA * sizeof(GemmGroup));
    GemmGroup* groupsA = reinterpret_cast<GemmGroup*>(g_staging + offGA);
    GemmTerm* termsA = reinterpret_cast<GemmTerm*>(g_staging + offTA);
    {  // the stage A terms: walk again, emitting one term per used K*R product

        size_t tA = 0;
        for (int o2 = 0; o2 < rb && tA < nA; ++o2) {
            const View Ro = view(R[o2]);
            for (int i = 0; i < Ro.n; ++i) {
                const int ldx = Ro.left[i], jdx = Ro.right[i], rr = Ro.rows[i], rc = Ro.cols[i];
                if (rr == 0 || ldx < 0 || ldx >= nr || jdx < 0 || jdx >= nr) continue;
                for (int pos = 0; pos < K.n; ++pos) {
                    if (K.right[pos] != ldx) continue;
                    const int kdx = K.left[pos];
                    const int p2 = phys[(size_t)kdx * nr + ldx];
                    if (p2 < 0 || !right_nonzero(o2, p2)) continue;
                    const int a_k = K.rows[pos], b_l = K.cols[pos];
                    if (a_k == 0 || b_l == 0 || rc == 0) continue;
                    bool used = false;
                    for (int pos2 = 0; pos2 < K.n && !used; ++pos2) {
                        if (K.right[pos2] != jdx) continue;
                        const int idx = K.left[pos2];
                        const int p1 = phys[(size_t)idx * nr + jdx];
                        for (int o1 = 0; o1 < lb && !used; ++o1) {
                            if (Wat(o1, o2, p1, p2) == 0.0) continue;
                            const View Lo = view(L[o1]);
                            const int q = find(Lo, idx, kdx);
                            if (q != -1 && Lo.rows[q] != 0) used = true;
                        }
                    }
                    if (used) {
                        termsA[tA] = GemmTerm{g_ket_off[pos], g_R_off[g_R_first[o2] + i], b_l, rc, b_l, 0, 1.0};
                        ++tA;
                    }
                }
            }
        }
    }
    GemmTile* tilesA = reinterpret_cast<GemmTile*>(g_staging + offLA);
    {
        int64_t k = 0;
        for (size_t g = 0; g < nA; ++g)
            for (int m0 = 0; m0 < groupsA[g].m; m0 += kTile)
                for (int n0 = 0; n0 < groupsA[g].n; n0 += kTile) tilesA[k++] = GemmTile{(int)g, m0, n0, 0};
    }
    GemmTerm* termsB = reinterpret_cast<GemmTerm*>(g_staging + offTB);
    GemmGroup* groupsB = reinterpret_cast<GemmGroup*>(g_staging + offGB);
    GemmTile* tilesB = reinterpret_cast<GemmTile*>(g_staging + offLB);
    {
        // counting sort of the pending terms by output block (stable)
        for (int b = 0; b < K.n; ++b) g_count[b + 1] += g_count[b];
        for (size_t t = 0; t < nB; ++t) termsB[g_count[g_pending[t].out_pos]++] = g_pending[t].term;
        // g_count[b] now holds the end of block b's range; its start is g_count[b-1] (or 0)
        int gi = 0;
        int64_t k = 0;
        for (int b = 0; b < K.n; ++b) {
            const int t0 = b == 0 ? 0 : g_count[b - 1], t1 = g_count[b];
            if (t1 == t0) continue;
            groupsB[gi] = GemmGroup{g_ket_off[b], K.cols[b], K.rows[b], K.cols[b], t0, t1, 0};
            for (int m0 = 0; m0 < K.rows[b]; m0 += kTile)
                for (int n0 = 0; n0 < K.cols[b]; n0 += kTile) tilesB[k++] = GemmTile{gi, m0, n0, 0};
            ++gi;
        }
    }
    // ---- every operand range inside its buffer (host check, before any device work) ---
    const int64_t psi_size = g_ket_off[K.n];
    auto check = [](const GemmTerm* terms, const GemmGroup* groups, size_t ng, int64_t asz, int64_t bsz,
                    int64_t csz) {
        for (size_t g = 0; g < ng; ++g) {
            const GemmGroup& gr = groups[g];
            if (gr.m <= 0 || gr.n <= 0) continue;
            if (gr.c_off + (int64_t)(gr.m - 1) * gr.ldc + gr.n > csz) return false;
            for (int t = gr.t0; t < gr.t1; ++t) {
                const GemmTerm& tm = terms[t];
                if (tm.a_off + (int64_t)(gr.m - 1) * tm.lda + tm.k > asz) return false;
                if (tm.b_off + (int64_t)(tm.k - 1) * tm.ldb + gr.n > bsz) return false;
            }
        }
        return true;
    };
    if (!check(termsA, groupsA, nA, psi_size, Rsize, t_size) ||
        !check(termsB, groupsB, (size_t)nGB, Lsize, t_size, psi_size))
        return set_error(DMRG_E_ARG, "dmrg_heff_apply_noalloc: block shapes inconsistent with their buffers");
    // ---- copy the tables into the static device array and launch --------------------
    if (offT) DMRG_CUDA_TRY(cudaMemcpyAsync(scratch, g_staging, offT, cudaMemcpyHostToDevice, st));
    const int64_t psi_dim = g_ket_off[K.n];
    if (!accumulate && psi_dim) DMRG_CUDA_TRY(cudaMemsetAsync(out_dev, 0, (size_t)psi_dim * sizeof(double), st));
    double* T = reinterpret_cast<double*>(scratch + offT);
    DMRG_TRY(launch_gemm_f64_tables(reinterpret_cast<const GemmTerm*>(scratch + offTA),
                                    reinterpret_cast<const GemmGroup*>(scratch + offGA),
                                    reinterpret_cast<const GemmTile*>(scratch + offLA), (int)ntA, false, false,
                                    psi_dev, R_dev, T, false, st));
    DMRG_TRY(launch_gemm_f64_tables(reinterpret_cast<const GemmTerm*>(scratch + offTB),
                                    reinterpret_cast<const GemmGroup*>(scratch + offGB),
                                    reinterpret_cast<const GemmTile*>(scratch + offLB), (int)ntB, false, false, L_dev,
                                    T, out_dev, true, st));
    // the staging image is reused by the next call: wait until the copy has read it
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    return DMRG_OK;
}
