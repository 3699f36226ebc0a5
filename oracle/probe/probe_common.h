// Test infrastructure: helpers shared by the instrumented probes that are linked
// against the unmodified reference sources (see ../Makefile).  They serialise the
// reference's block lists into a small "named array" container (.nac):
//
//   repeated { int32 name_len; char name[name_len]; char dtype ('i' int32 | 'd' f64);
//              int32 ndim; int32 shape[ndim]; raw little-endian data }
//
// The same container is read by oracle/nac.py and by the tests.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include <omp.h>
#include <sys/time.h>

// Reference members are protected; the probes read them directly.  Every
// standard header the reference pulls in is included above first, so the
// redefinition only touches the reference's own class definitions.
#define protected public
#include "dmrgcc.h"
#undef protected

namespace probe {

struct NacWriter {
    FILE* f = nullptr;
    explicit NacWriter(const std::string& path) {
        f = std::fopen(path.c_str(), "wb");
        if (!f) { std::perror(path.c_str()); std::exit(2); }
    }
    ~NacWriter() { if (f) std::fclose(f); }
    void header(const std::string& name, char dt, const std::vector<int>& shape) {
        int32_t n = (int32_t)name.size();
        std::fwrite(&n, 4, 1, f);
        std::fwrite(name.data(), 1, n, f);
        std::fwrite(&dt, 1, 1, f);
        int32_t nd = (int32_t)shape.size();
        std::fwrite(&nd, 4, 1, f);
        for (int s : shape) { int32_t v = s; std::fwrite(&v, 4, 1, f); }
    }
    void ints(const std::string& name, const std::vector<int>& v) {
        header(name, 'i', {(int)v.size()});
        if (!v.empty()) std::fwrite(v.data(), 4, v.size(), f);
    }
    void dbls(const std::string& name, const std::vector<double>& v) {
        header(name, 'd', {(int)v.size()});
        if (!v.empty()) std::fwrite(v.data(), 8, v.size(), f);
    }
    void scalar_i(const std::string& name, int v) { ints(name, {v}); }
    void scalar_d(const std::string& name, double v) { dbls(name, {v}); }
};

struct NacArray {
    char dtype = 'i';
    std::vector<int> shape;
    std::vector<int> i;
    std::vector<double> d;
};

inline std::map<std::string, NacArray> nac_read(const std::string& path) {
    std::map<std::string, NacArray> out;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { std::perror(path.c_str()); std::exit(2); }
    for (;;) {
        int32_t n;
        if (std::fread(&n, 4, 1, f) != 1) break;
        std::string name(n, '\0');
        if (std::fread(&name[0], 1, n, f) != (size_t)n) break;
        NacArray a;
        if (std::fread(&a.dtype, 1, 1, f) != 1) break;
        int32_t nd;
        if (std::fread(&nd, 4, 1, f) != 1) break;
        size_t count = 1;
        for (int k = 0; k < nd; ++k) {
            int32_t s;
            if (std::fread(&s, 4, 1, f) != 1) break;
            a.shape.push_back(s);
            count *= (size_t)s;
        }
        if (a.dtype == 'i') { a.i.resize(count); if (count && std::fread(a.i.data(), 4, count, f) != count) break; }
        else { a.d.resize(count); if (count && std::fread(a.d.data(), 8, count, f) != count) break; }
        out[name] = std::move(a);
    }
    std::fclose(f);
    return out;
}

// Block list -> arrays prefix.{left,right,rows,cols,data}
inline void write_block(NacWriter& w, const std::string& p, RealMatrixBlock* b) {
    std::vector<int> li, ri, rows, cols;
    std::vector<double> data;
    int nb = b ? b->num_block_ : 0;
    for (int k = 0; k < nb; ++k) {
        RealMatrix* m = b->matrix_block_[k];
        li.push_back(b->left_index_[k]);
        ri.push_back(b->right_index_[k]);
        rows.push_back(m->row_);
        cols.push_back(m->column_);
        for (int e = 0; e < m->total_element_num_; ++e) data.push_back(m->matrix_element_[e]);
    }
    w.ints(p + ".left", li);
    w.ints(p + ".right", ri);
    w.ints(p + ".rows", rows);
    w.ints(p + ".cols", cols);
    w.dbls(p + ".data", data);
}

inline void write_lattice(NacWriter& w, const std::string& p, RealTensorLattice* t) {
    w.scalar_i(p + ".physics_dim", t->physics_dim_);
    w.ints(p + ".left_block", std::vector<int>(t->left_block_, t->left_block_ + t->num_left_block_));
    w.ints(p + ".left_dim", std::vector<int>(t->left_dim_, t->left_dim_ + t->num_left_block_));
    w.ints(p + ".right_block", std::vector<int>(t->right_block_, t->right_block_ + t->num_right_block_));
    w.ints(p + ".right_dim", std::vector<int>(t->right_dim_, t->right_dim_ + t->num_right_block_));
    std::vector<int> phys;
    for (int i = 0; i < t->num_left_block_; ++i)
        for (int j = 0; j < t->num_right_block_; ++j) phys.push_back(t->physics_index_[i][j]);
    w.ints(p + ".physics_index", phys);
    write_block(w, p + ".ket", t->ket_tensor_);
    if (t->canonical_tensor_) {
        write_block(w, p + ".canonical", t->canonical_tensor_);
        int n = t->canonical_tensor_->num_block_;
        w.ints(p + ".match_dim", std::vector<int>(t->match_dim_, t->match_dim_ + n));
    }
}

inline void write_operator(NacWriter& w, const std::string& p, RealTensorOperator* op) {
    int d = op->physics_dim_, lb = op->left_bond_, rb = op->right_bond_;
    w.ints(p + ".dims", {d, lb, rb});
    std::vector<double> v;
    for (int a = 0; a < lb; ++a)
        for (int b = 0; b < rb; ++b)
            for (int p1 = 0; p1 < d; ++p1)
                for (int p2 = 0; p2 < d; ++p2) v.push_back(op->tensor_operator_[a][b]->get_matrix_element(p1, p2));
    w.dbls(p + ".W", v);
}

inline void write_env(NacWriter& w, const std::string& p, RealMatrixBlock** env, int bond) {
    w.scalar_i(p + ".bond", bond);
    for (int o = 0; o < bond; ++o) write_block(w, p + "." + std::to_string(o), env[o]);
}

// Deterministic synthetic values: splitmix64 stream mapped to [-1, 1).
struct SplitMix {
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed) {}
    double next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z = z ^ (z >> 31);
        return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    }
};

}  // namespace probe
