// Host-side description of the block-sparse operands of one site: the site
// tensor's block list, the MPO tensor and the environments.  Built from the
// C-ABI dmrg_blocks_t arrays; used to derive GEMM schedules.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "dmrg_b200.h"

namespace dmrg {

// One RealMatrixBlock's shape plus packed offsets (list order, row-major blocks).
struct BlockListDesc {
    std::vector<int> left, right, rows, cols;
    std::vector<int64_t> off;
    int64_t size = 0;

    int count() const { return (int)left.size(); }

    // Copies a C-ABI description; returns false on a negative size.
    bool assign(const dmrg_blocks_t& b) {
        if (b.nblocks < 0) return false;
        left.assign(b.left, b.left + b.nblocks);
        right.assign(b.right, b.right + b.nblocks);
        rows.assign(b.rows, b.rows + b.nblocks);
        cols.assign(b.cols, b.cols + b.nblocks);
        off.resize(b.nblocks);
        size = 0;
        for (int k = 0; k < b.nblocks; ++k) {
            if (rows[k] < 0 || cols[k] < 0) return false;
            off[k] = size;
            size += (int64_t)rows[k] * cols[k];
        }
        return true;
    }
    void push(int l, int r, int nr, int nc) {
        left.push_back(l);
        right.push_back(r);
        rows.push_back(nr);
        cols.push_back(nc);
        off.push_back(size);
        size += (int64_t)nr * nc;
    }
    // First block with sectors (l, r) in list order, -1 if none
    // (RealMatrixBlock::FindMatrixBlock, src/tensor/real_matrix_block.cc:314-330).
    int find(int l, int r) const {
        for (int k = 0; k < count(); ++k)
            if (left[k] == l && right[k] == r) return k;
        return -1;
    }
    // Positions sharing a left (leigh 0) or right (leigh 1) sector, in list order
    // (FindMatrixBlock(num, pos, leigh, target), :332-363).
    std::vector<std::vector<int>> by_sector(int leigh, int nsec) const {
        std::vector<std::vector<int>> out(nsec > 0 ? nsec : 0);
        for (int k = 0; k < count(); ++k) {
            int s = leigh == 0 ? left[k] : right[k];
            if (s >= 0 && s < nsec) out[s].push_back(k);
        }
        return out;
    }
};

// One environment: a block list per MPO bond index, packed index-major.
struct EnvDesc {
    std::vector<BlockListDesc> o;
    std::vector<int64_t> base;
    int64_t size = 0;
    bool assign(const dmrg_blocks_t* b, int bond) {
        o.resize(bond);
        base.resize(bond);
        size = 0;
        for (int i = 0; i < bond; ++i) {
            if (!o[i].assign(b[i])) return false;
            base[i] = size;
            size += o[i].size;
        }
        return true;
    }
    void rebase() {
        base.resize(o.size());
        size = 0;
        for (size_t i = 0; i < o.size(); ++i) {
            base[i] = size;
            size += o[i].size;
        }
    }
};

// Site tensor sectors + MPO tensor.
struct SiteDesc {
    int nl = 0, nr = 0, d = 0, lb = 0, rb = 0;
    std::vector<int> phys;    // [nl * nr], -1 = no block (single-site tensors)
    std::vector<double> W;    // [lb][rb][d][d]
    BlockListDesc ket;
    // physics index of every ket block, in [0, d).  Single-site tensors have at
    // most one block per sector pair and take it from `phys`; a two-site tensor
    // has one block per (left, middle, right) sector triple, several per pair,
    // with the combined index p1 * d1 + p2.
    std::vector<int> bphys;

    int p(int l, int r) const { return phys[(size_t)l * nr + r]; }
    int pb(int k) const { return bphys[k]; }
    double w(int o1, int o2, int p1, int p2) const {
        return W[(((size_t)o1 * rb + o2) * d + p1) * d + p2];
    }
    // RealTensorOperator::LeftCheckZero / RightCheckZero
    // (src/dmrg/realdmrg/real_tensor_operator.cc:363-395): any |W| > 1e-15.
    bool left_nonzero(int o1, int p1) const {
        for (int o2 = 0; o2 < rb; ++o2)
            for (int p2 = 0; p2 < d; ++p2)
                if (std::fabs(w(o1, o2, p1, p2)) > 1e-15) return true;
        return false;
    }
    bool right_nonzero(int o2, int p2) const {
        for (int o1 = 0; o1 < lb; ++o1)
            for (int p1 = 0; p1 < d; ++p1)
                if (std::fabs(w(o1, o2, p1, p2)) > 1e-15) return true;
        return false;
    }
};

// Validates and copies the common site arguments of the C ABI.
int build_site_desc(SiteDesc& s, int nl, int nr, const int* phys, const dmrg_blocks_t* ket, int d, int lb,
                    int rb, const double* W);
// The same with a physics index per ket block (block_phys[nblocks]) instead of
// the sector-pair table; blocks may share a sector pair.
int build_site_desc_blocks(SiteDesc& s, int nl, int nr, const int* block_phys, const dmrg_blocks_t* ket, int d,
                           int lb, int rb, const double* W);

}  // namespace dmrg
