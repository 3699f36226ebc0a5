// Test infrastructure: instrumented run of the unmodified reference DMRG.
//
// The reference's own sweep (RealTensorRundmrg::Run, src/dmrg/realdmrg/
// real_tensor_rundmrg.cc:115-245) runs untouched.  The linker's --wrap option
// routes its calls to four hot-path members through the __wrap_* functions
// below, which serialise inputs and outputs to .nac files at the requested call
// indices and then call the real member:
//   RealTensorLanczos::LanczosMethod              real_tensor_lanczos.cc:14
//   RealTensorContraction::Left/RightCompute...   real_tensor_contraction.cc:782,959
//   RealTensorLattice::Left/RightCanonical...     real_tensor_lattice.cc:558,794
//
// Usage: probe_dump <input file>
//   PROBE_OUT=dir          output directory (default ".")
//   PROBE_HEFF=i,j,...     Lanczos call indices whose H_eff problem is dumped
//   PROBE_STRUCT_ONLY=1    H_eff dumps carry block structure only (no values)
//   PROBE_ENV=i,j,...      environment-update call indices to dump
//   PROBE_CANON=i,j,...    canonicalisation call indices to dump
//   PROBE_MERGE=i,j,...    merge call indices to dump (Left/RightMergeTensorLattice)
//   PROBE_STOP=n           exit(0) right after Lanczos call n
// cache_resume in the input reads the checkpoint through a corrected copy of
// the reference's reader (see __wrap__ZN15RealTensorSpace15ReadTensorSpaceEPKc).
//   PROBE_GAUGE=1          fix the free signs of LAPACK's singular vectors and
//                          eigenvectors by the library's convention (see below)
//   PROBE_GAUGE_SEED=s     flip each of those signs at random instead (seed s)
//   PROBE_SYNTH=s          dumped env updates / canonicalisations run on seeded
//                          synthetic inputs (see below; with PROBE_STOP)
//   PROBE_ROUND_F32=1      dumped Lanczos calls run on float32-rounded inputs
// Always writes PROBE_OUT/steps.txt: one line per Lanczos call with the site,
// iteration cap, psi_dim and the energy the reference returned.
#include "probe_common.h"

using probe::NacWriter;

static RealTensorSpace* g_space = nullptr;
static RealTensorHamiltonian* g_ham = nullptr;
static std::string g_out = ".";
static std::vector<int> g_heff, g_env, g_canon;
static bool g_struct_only = false;
static int g_stop = -1;
static FILE* g_steps = nullptr;
static int n_lanczos = 0, n_env = 0, n_canon = 0;

static std::vector<int> parse_list(const char* s) {
    std::vector<int> v;
    if (!s) return v;
    std::stringstream ss(s);
    std::string tok;
    while (std::getline(ss, tok, ',')) if (!tok.empty()) v.push_back(std::atoi(tok.c_str()));
    return v;
}
static bool wanted(const std::vector<int>& v, int i) {
    for (int x : v) if (x == i || x == -1) return true;
    return false;
}
static int site_of(RealTensorLattice* t) {
    for (int i = 0; i < g_space->num_site_; ++i) if (g_space->tensor_lattice_[i] == t) return i;
    return -1;
}

// Structure trace (PROBE_TRACE=1): one line per canonicalisation, expansion,
// match and merge with the sector dimensions of the site afterwards; the
// device engine writes the same lines (DMRG_TRACE) for comparison.
static FILE* g_trace = nullptr;
// PROBE_GAUGE=1: LAPACK leaves the sign of every singular vector pair and
// eigenvector free.  With this switch each is fixed after the call by one
// convention, also used by libdmrg_b200: the component of largest magnitude of
// the left singular vector (the eigenvector) is positive, where components
// within a relative 1e-6 of the largest count as equal and the first of them
// decides.  The decomposition stays exact; only the free signs are pinned, so
// the two implementations follow one trajectory through the noise-driven
// subspace expansion (whose random matrices act in the gauge-dependent basis).
static bool g_gauge = false;
// PROBE_SYNTH=s (s != 0): at every dumped environment update and
// canonicalisation, the inputs (ket values, then the incoming environment
// bond by bond, blocks in list order, row-major) are first replaced by the
// splitmix64 stream seeded with s, mapped to [-1, 1) (probe::SplitMix), so that
// a fixture needs only the block structure, the seed and a digest of the
// reference's output.  The run is meaningless afterwards: use with PROBE_STOP.
static unsigned long long g_synth = 0;
// PROBE_ROUND_F32=1: at every dumped Lanczos call, the operator's environments
// and the start vector are first rounded to float32 values (stored as doubles),
// so that a fixture can keep them in float32 without changing the problem the
// reference solved.
static bool g_round_f32 = false;
static void synth_block(RealMatrixBlock* b, probe::SplitMix& rng) {
    for (int k = 0; b && k < b->num_block_; ++k) {
        RealMatrix* m = b->matrix_block_[k];
        for (int e = 0; e < m->total_element_num_; ++e) m->matrix_element_[e] = rng.next();
    }
}
static void round_block(RealMatrixBlock* b) {
    for (int k = 0; b && k < b->num_block_; ++k) {
        RealMatrix* m = b->matrix_block_[k];
        for (int e = 0; e < m->total_element_num_; ++e) m->matrix_element_[e] = (double)(float)m->matrix_element_[e];
    }
}
// PROBE_GAUGE_SEED=s (s != 0): instead, every singular pair and eigenvector
// that LAPACK returns has its sign flipped with probability 1/2, from a private
// splitmix64 stream seeded with s (glibc rand() is left untouched).  Each seed
// is another equally valid run of the reference; the spread of their final
// energies is the reference's own gauge spread.
static unsigned long long g_gauge_seed = 0;
static bool gauge_coin() {
    unsigned long long z = (g_gauge_seed += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return ((z ^ (z >> 31)) >> 63) != 0;
}
static double sign_of_column(const double* a, long n, long stride) {
    double m = 0.0;
    for (long i = 0; i < n; ++i) m = std::fabs(a[i * stride]) > m ? std::fabs(a[i * stride]) : m;
    if (m == 0.0) return 1.0;
    for (long i = 0; i < n; ++i)
        if (std::fabs(a[i * stride]) >= m * (1.0 - 1e-6)) return a[i * stride] < 0.0 ? -1.0 : 1.0;
    return 1.0;
}
extern "C" lapack_int __real_LAPACKE_dgesvd(int, char, char, lapack_int, lapack_int, double*, lapack_int, double*,
                                            double*, lapack_int, double*, lapack_int, double*);
extern "C" lapack_int __wrap_LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n, double* a,
                                            lapack_int lda, double* s, double* u, lapack_int ldu, double* vt,
                                            lapack_int ldvt, double* superb) {
    const lapack_int info = __real_LAPACKE_dgesvd(layout, jobu, jobvt, m, n, a, lda, s, u, ldu, vt, ldvt, superb);
    if (g_gauge && info == 0 && layout == LAPACK_ROW_MAJOR && jobu == 'S' && jobvt == 'S') {
        const lapack_int k = m < n ? m : n;  // (the reference's headers define min/max as macros)
        for (lapack_int c = 0; c < k; ++c)
            if (g_gauge_seed ? gauge_coin() : sign_of_column(u + c, m, ldu) < 0.0) {
                for (lapack_int i = 0; i < m; ++i) u[(long)i * ldu + c] = -u[(long)i * ldu + c];
                for (lapack_int j = 0; j < n; ++j) vt[(long)c * ldvt + j] = -vt[(long)c * ldvt + j];
            }
    }
    return info;
}
extern "C" lapack_int __real_LAPACKE_dsyevd(int, char, char, lapack_int, double*, lapack_int, double*);
extern "C" lapack_int __wrap_LAPACKE_dsyevd(int layout, char jobz, char uplo, lapack_int n, double* a, lapack_int lda,
                                            double* w) {
    const lapack_int info = __real_LAPACKE_dsyevd(layout, jobz, uplo, n, a, lda, w);
    if (g_gauge && info == 0 && layout == LAPACK_ROW_MAJOR && jobz == 'V')
        for (lapack_int c = 0; c < n; ++c)
            if (g_gauge_seed ? gauge_coin() : sign_of_column(a + c, n, lda) < 0.0)
                for (lapack_int i = 0; i < n; ++i) a[(long)i * lda + c] = -a[(long)i * lda + c];
    return info;
}

static long long g_rand_calls = 0;  // glibc rand() draws so far (the reference's only random source)
extern "C" int __real_rand(void);
extern "C" int __wrap_rand(void) {
    ++g_rand_calls;
    return __real_rand();
}
static double g_cut_gap = -1.0, g_pre_gap = -1.0;  // truncation_gap() of the step being traced
static void trace(const char* tag, int leigh, RealTensorLattice* t) {
    if (!g_trace) return;
    std::fprintf(g_trace, "%s %d %d L:", tag, leigh, site_of(t));
    for (int i = 0; i < t->num_left_block_; ++i) std::fprintf(g_trace, "%d,", t->left_dim_[i]);
    std::fprintf(g_trace, " R:");
    for (int i = 0; i < t->num_right_block_; ++i) std::fprintf(g_trace, "%d,", t->right_dim_[i]);
    double norm2 = 0.0;
    RealMatrixBlock* kb = t->ket_tensor_;
    for (int k = 0; kb && k < kb->num_block_; ++k) {
        const RealMatrix* m = kb->matrix_block_[k];
        for (long i = 0; i < (long)m->row_ * m->column_; ++i) norm2 += m->matrix_element_[i] * m->matrix_element_[i];
    }
    std::fprintf(g_trace, " P:%d N:%.10e Q:%lld", t->ComputeKetTensorDim(), norm2, g_rand_calls);
    if (tag[0] == 'C' && t->canonical_tensor_) {  // per-block squared norms of S V^T (or U S)
        std::fprintf(g_trace, " S:");
        RealMatrixBlock* cb = t->canonical_tensor_;
        for (int k = 0; k < cb->num_block_; ++k) {
            const RealMatrix* m = cb->matrix_block_[k];
            double s2 = 0.0;
            for (long i = 0; i < (long)m->row_ * m->column_; ++i) s2 += m->matrix_element_[i] * m->matrix_element_[i];
            std::fprintf(g_trace, "%.8e,", s2);
        }
    }
    if (tag[0] == 'C') std::fprintf(g_trace, " G:%.3e,%.3e", g_cut_gap, g_pre_gap);
    std::fprintf(g_trace, "\n");
}

static void write_struct_only_block(NacWriter& w, const std::string& p, RealMatrixBlock* b) {
    std::vector<int> li, ri, rows, cols;
    int nb = b ? b->num_block_ : 0;
    for (int k = 0; k < nb; ++k) {
        li.push_back(b->left_index_[k]);
        ri.push_back(b->right_index_[k]);
        rows.push_back(b->matrix_block_[k]->row_);
        cols.push_back(b->matrix_block_[k]->column_);
    }
    w.ints(p + ".left", li);
    w.ints(p + ".right", ri);
    w.ints(p + ".rows", rows);
    w.ints(p + ".cols", cols);
}

extern "C" {
void __real__ZN17RealTensorLanczos13LanczosMethodEiiRd(RealTensorLanczos*, int, int, double&);
void __real__ZN21RealTensorContraction28LeftComputeTensorContractionEP17RealTensorLatticeP18RealTensorOperatorPS_(
    RealTensorContraction*, RealTensorLattice*, RealTensorOperator*, RealTensorContraction*);
void __real__ZN21RealTensorContraction29RightComputeTensorContractionEP17RealTensorLatticeP18RealTensorOperatorPS_(
    RealTensorContraction*, RealTensorLattice*, RealTensorOperator*, RealTensorContraction*);
void __real__ZN17RealTensorLattice26LeftCanonicalTensorLatticeEid(RealTensorLattice*, int, double);
void __real__ZN17RealTensorLattice27RightCanonicalTensorLatticeEid(RealTensorLattice*, int, double);
void __real__ZN15RealTensorSpace16ExpanTensorSpaceEii(RealTensorSpace*, int, int);
void __real__ZN15RealTensorSpace16MatchTensorSpaceEii(RealTensorSpace*, int, int);
void __real__ZN17RealTensorLattice22LeftMergeTensorLatticeEPS_(RealTensorLattice*, RealTensorLattice*);
void __real__ZN17RealTensorLattice23RightMergeTensorLatticeEPS_(RealTensorLattice*, RealTensorLattice*);
void __wrap__ZN15RealTensorSpace16ExpanTensorSpaceEii(RealTensorSpace* self, int leigh, int site) {
    if (g_trace && self->expan_tensor_lattice_) {  // the expansion term, block by block, before it is merged
        RealMatrixBlock* kb = self->expan_tensor_lattice_->ket_tensor_;
        std::fprintf(g_trace, "Y %d %d", leigh, site);
        for (int k = 0; kb && k < kb->num_block_; ++k) {
            const RealMatrix* m = kb->matrix_block_[k];
            double s2 = 0.0;
            for (long i = 0; i < (long)m->row_ * m->column_; ++i) s2 += m->matrix_element_[i] * m->matrix_element_[i];
            std::fprintf(g_trace, " %d.%d:%dx%d=%.8e", kb->left_index_[k], kb->right_index_[k], m->row_, m->column_,
                         s2);
        }
        std::fprintf(g_trace, "\n");
    }
    __real__ZN15RealTensorSpace16ExpanTensorSpaceEii(self, leigh, site);
    trace("X", leigh, self->tensor_lattice_[site]);
}
void __wrap__ZN15RealTensorSpace16MatchTensorSpaceEii(RealTensorSpace* self, int leigh, int site) {
    __real__ZN15RealTensorSpace16MatchTensorSpaceEii(self, leigh, site);
    trace("T", leigh, self->tensor_lattice_[site]);
}
// RealTensorSpace::ReadTensorSpace(const char*) (real_tensor_space.cc:212-277,
// used by cache_resume) with its table allocation corrected: the reference
// sizes num_table_ and quantum_table_ by num_quantum_ where num_site_pp_ entries
// are read into them (:245,249), which overruns the heap and makes its resumed
// runs meaningless.  Same file format, same fields; the site tensors are read by
// the reference's own RealTensorLattice::ReadTensorLattice.
void __wrap__ZN15RealTensorSpace15ReadTensorSpaceEPKc(RealTensorSpace* self, const char* name) {
    std::ifstream f(name, std::ios::binary | std::ios::in);
    if (!f) {
        std::fprintf(stderr, "probe: cannot open %s\n", name);
        std::exit(2);
    }
    auto get = [&](auto& v) { f.read(reinterpret_cast<char*>(&v), sizeof(v)); };
    get(self->num_site_);
    get(self->num_site_pp_);
    get(self->num_site_mm_);
    get(self->num_quantum_);
    self->num_table_ = new int[self->num_site_pp_];
    for (int i = 0; i < self->num_site_pp_; ++i) get(self->num_table_[i]);
    self->quantum_table_ = new int**[self->num_site_pp_];
    for (int i = 0; i < self->num_site_pp_; ++i) {
        self->quantum_table_[i] = new int*[self->num_table_[i]];
        for (int j = 0; j < self->num_table_[i]; ++j) {
            self->quantum_table_[i][j] = new int[self->num_quantum_];
            for (int k = 0; k < self->num_quantum_; ++k) get(self->quantum_table_[i][j][k]);
        }
    }
    self->tensor_lattice_ = new RealTensorLattice*[self->num_site_];
    for (int i = 0; i < self->num_site_; ++i) {
        self->tensor_lattice_[i] = new RealTensorLattice();
        self->tensor_lattice_[i]->ReadTensorLattice(f);
    }
    get(self->max_block_);
    get(self->max_dim_);
    get(self->canonical_precision_);
    get(self->noise_factor_);
    if (!f) {
        std::fprintf(stderr, "probe: %s is truncated\n", name);
        std::exit(2);
    }
}
// PROBE_MERGE=i,j: merge call i writes merge_<i>.nac with the site it merges
// into before and after (lattices "before" / "after") and the lattice whose
// canonical tensor it multiplies in ("source", with its canonical blocks).
static std::vector<int> g_merge;
static int n_merge = 0;
static NacWriter* merge_begin(int side, RealTensorLattice* self, RealTensorLattice* o) {
    const int call = n_merge++;
    if (!wanted(g_merge, call)) return nullptr;
    auto* w = new NacWriter(g_out + "/merge_" + std::to_string(call) + ".nac");
    w->scalar_i("side", side);
    w->scalar_i("site", site_of(self));
    probe::write_lattice(*w, "before", self);
    probe::write_lattice(*w, "source", o);
    return w;
}
static void merge_end(NacWriter* w, RealTensorLattice* self) {
    if (!w) return;
    probe::write_lattice(*w, "after", self);
    delete w;
}
void __wrap__ZN17RealTensorLattice22LeftMergeTensorLatticeEPS_(RealTensorLattice* self, RealTensorLattice* o) {
    NacWriter* w = merge_begin(0, self, o);
    __real__ZN17RealTensorLattice22LeftMergeTensorLatticeEPS_(self, o);
    trace("M", 0, self);
    merge_end(w, self);
}
void __wrap__ZN17RealTensorLattice23RightMergeTensorLatticeEPS_(RealTensorLattice* self, RealTensorLattice* o) {
    NacWriter* w = merge_begin(1, self, o);
    __real__ZN17RealTensorLattice23RightMergeTensorLatticeEPS_(self, o);
    trace("M", 1, self);
    merge_end(w, self);
}
void __real__ZN17RealTensorLattice20CombineTensorLatticeEiRiRPiS2_PS_(RealTensorLattice*, int, int&, int*&, int*&,
                                                                      RealTensorLattice*);

// CombineTensorLattice's first counting loop bounds its inner scan by the size
// of the second list (real_tensor_lattice.cc:427-438).  Record every call whose
// count differs from the plain union of the two sector lists.
static FILE* g_combine = nullptr;
void __wrap__ZN17RealTensorLattice20CombineTensorLatticeEiRiRPiS2_PS_(RealTensorLattice* self, int leigh, int& num,
                                                                      int*& blocks, int*& dims,
                                                                      RealTensorLattice* expan) {
    const int n0 = leigh == 0 ? self->num_left_block_ : self->num_right_block_;
    const int n1 = leigh == 0 ? expan->num_left_block_ : expan->num_right_block_;
    const int* b0 = leigh == 0 ? self->left_block_ : self->right_block_;
    const int* b1 = leigh == 0 ? expan->left_block_ : expan->right_block_;
    int uni = n0;
    for (int j = 0; j < n1; ++j) {
        bool f = false;
        for (int i = 0; i < n0; ++i) f = f || b0[i] == b1[j];
        uni += !f;
    }
    __real__ZN17RealTensorLattice20CombineTensorLatticeEiRiRPiS2_PS_(self, leigh, num, blocks, dims, expan);
    if (!g_combine) g_combine = std::fopen((g_out + "/combine.txt").c_str(), "w");
    std::fprintf(g_combine, "%d %d %d %d %d%s\n", leigh, n0, n1, uni, num, uni != num ? " MISMATCH" : "");
    std::fflush(g_combine);
}

void __wrap__ZN17RealTensorLanczos13LanczosMethodEiiRd(RealTensorLanczos* self, int niter, int site,
                                                       double& result) {
    int call = n_lanczos++;
    if (call == 0) {  // the MPO and the quantum tables, once
        NacWriter w(g_out + "/model.nac");
        RealTensorHamiltonian* H = self->hamiltonian_;
        RealTensorSpace* S = self->space_;
        w.scalar_i("num_site", H->num_site_);
        for (int i = 0; i < H->num_site_; ++i) probe::write_operator(w, "op" + std::to_string(i), H->tensor_hamiltonian_[i]);
        for (int b = 0; b <= H->num_site_; ++b) {
            std::vector<int> q;
            for (int j = 0; j < H->num_table_[b]; ++j)
                for (int k = 0; k < H->num_quantum_; ++k) q.push_back(H->quantum_table_[b][j][k]);
            w.ints("hq" + std::to_string(b), q);
            std::vector<int> sq;
            for (int j = 0; j < S->num_table_[b]; ++j)
                for (int k = 0; k < S->num_quantum_; ++k) sq.push_back(S->quantum_table_[b][j][k]);
            w.ints("sq" + std::to_string(b), sq);
        }
    }
    RealTensorLattice* lat = self->space_->get_tensor_lattice(site);
    RealTensorOperator* op = self->hamiltonian_->get_tensor_hamiltonian(site);
    RealTensorContraction* con = self->network_->get_tensor_contraction(site);
    int psi_dim = lat->ComputeKetTensorDim();
    if (wanted(g_heff, call) && g_round_f32) {
        round_block(lat->ket_tensor_);
        for (int o = 0; o < op->left_bond_; ++o) round_block(con->left_contraction_tensor_[o]);
        for (int o = 0; o < op->right_bond_; ++o) round_block(con->right_contraction_tensor_[o]);
    }
    if (wanted(g_heff, call)) {
        NacWriter w(g_out + "/heff_" + std::to_string(call) + ".nac");
        w.scalar_i("site", site);
        w.scalar_i("call", call);
        w.scalar_i("niter", niter);
        if (g_struct_only) {
            w.scalar_i("physics_dim", lat->physics_dim_);
            w.ints("lattice.left_dim", std::vector<int>(lat->left_dim_, lat->left_dim_ + lat->num_left_block_));
            w.ints("lattice.right_dim", std::vector<int>(lat->right_dim_, lat->right_dim_ + lat->num_right_block_));
            std::vector<int> phys;
            for (int i = 0; i < lat->num_left_block_; ++i)
                for (int j = 0; j < lat->num_right_block_; ++j) phys.push_back(lat->physics_index_[i][j]);
            w.ints("lattice.physics_index", phys);
            write_struct_only_block(w, "lattice.ket", lat->ket_tensor_);
            probe::write_operator(w, "op", op);
            w.scalar_i("L.bond", op->left_bond_);
            for (int o = 0; o < op->left_bond_; ++o)
                write_struct_only_block(w, "L." + std::to_string(o), con->left_contraction_tensor_[o]);
            w.scalar_i("R.bond", op->right_bond_);
            for (int o = 0; o < op->right_bond_; ++o)
                write_struct_only_block(w, "R." + std::to_string(o), con->right_contraction_tensor_[o]);
        } else {
            probe::write_lattice(w, "lattice", lat);
            probe::write_operator(w, "op", op);
            probe::write_env(w, "L", con->left_contraction_tensor_, op->left_bond_);
            probe::write_env(w, "R", con->right_contraction_tensor_, op->right_bond_);
            std::vector<double> out(psi_dim, 0.0);
            con->MultiplyEffectHamilton(lat, op, out.data());
            w.dbls("heff_out", out);
            if (psi_dim < 400) {
                std::vector<double> h((size_t)psi_dim * psi_dim, 0.0);
                con->ComputeEffectHamilton(lat, op, h.data());
                w.dbls("heff_dense", h);
            }
        }
    }
    double t0 = GetWallTime();
    __real__ZN17RealTensorLanczos13LanczosMethodEiiRd(self, niter, site, result);
    double t1 = GetWallTime();
    if (wanted(g_heff, call) && !g_struct_only) {
        NacWriter w(g_out + "/lanczos_" + std::to_string(call) + ".nac");
        w.scalar_d("energy", result);
        probe::write_lattice(w, "lattice", lat);
    }
    std::fprintf(g_steps, "%d %d %d %d %.15e %.6f\n", call, site, niter, psi_dim, result, t1 - t0);
    if (g_trace) std::fprintf(g_trace, "E %d %d P:%d %.12e\n", call, site, psi_dim, result);
    std::fflush(g_steps);
    if (call == g_stop) std::exit(0);
}

static void env_common(bool left, RealTensorContraction* self, RealTensorLattice* lat, RealTensorOperator* op,
                       RealTensorContraction* next) {
    int call = n_env++;
    bool dump = wanted(g_env, call);
    std::string path = g_out + "/env_" + std::to_string(call) + ".nac";
    NacWriter* w = dump ? new NacWriter(path) : nullptr;
    if (w && g_synth) {
        probe::SplitMix rng(g_synth);
        synth_block(lat->ket_tensor_, rng);
        RealMatrixBlock** env = left ? self->left_contraction_tensor_ : self->right_contraction_tensor_;
        for (int o = 0; o < (left ? op->left_bond_ : op->right_bond_); ++o) synth_block(env[o], rng);
        w->scalar_i("synth_seed", (int)g_synth);
    }
    if (w) {
        w->scalar_i("left", left ? 1 : 0);
        w->scalar_i("site", site_of(lat));
        probe::write_lattice(*w, "lattice", lat);
        probe::write_operator(*w, "op", op);
        if (left) probe::write_env(*w, "env_in", self->left_contraction_tensor_, op->left_bond_);
        else probe::write_env(*w, "env_in", self->right_contraction_tensor_, op->right_bond_);
    }
    if (left)
        __real__ZN21RealTensorContraction28LeftComputeTensorContractionEP17RealTensorLatticeP18RealTensorOperatorPS_(
            self, lat, op, next);
    else
        __real__ZN21RealTensorContraction29RightComputeTensorContractionEP17RealTensorLatticeP18RealTensorOperatorPS_(
            self, lat, op, next);
    if (w) {
        if (left) probe::write_env(*w, "env_out", next->left_contraction_tensor_, op->right_bond_);
        else probe::write_env(*w, "env_out", next->right_contraction_tensor_, op->left_bond_);
        delete w;
    }
}

void __wrap__ZN21RealTensorContraction28LeftComputeTensorContractionEP17RealTensorLatticeP18RealTensorOperatorPS_(
    RealTensorContraction* self, RealTensorLattice* lat, RealTensorOperator* op, RealTensorContraction* next) {
    env_common(true, self, lat, op, next);
}
void __wrap__ZN21RealTensorContraction29RightComputeTensorContractionEP17RealTensorLatticeP18RealTensorOperatorPS_(
    RealTensorContraction* self, RealTensorLattice* lat, RealTensorOperator* op, RealTensorContraction* next) {
    env_common(false, self, lat, op, next);
}

// Conditioning of a canonicalisation's truncation decision, in units of the
// tensor's Frobenius norm: (cut) the distance between the last kept and the
// first dropped singular value when max_dim cuts the sorted list (-1 when it
// does not), and (pre) the smallest kept sigma / canpre over the values above
// canpre (a count of values above canpre decided by values only a few decades
// above it depends on the accuracy of the state, ~1e-8 after Lanczos).
// Sector matrices are stacked as the reference stacks them (blocks in list
// order).  A small value marks a step whose block dimensions can legitimately
// differ between two correct implementations.
static double truncation_gap(bool left, RealTensorLattice* t, int max_dim, double canpre) {
    RealMatrixBlock* kb = t->ket_tensor_;
    const int nsec = left ? t->num_right_block_ : t->num_left_block_;
    std::vector<double> all;
    double fro2 = 0.0;
    for (int sct = 0; sct < nsec; ++sct) {
        int m = 0, n = 0;
        std::vector<int> members;
        for (int k = 0; kb && k < kb->num_block_; ++k)
            if ((left ? kb->right_index_[k] : kb->left_index_[k]) == sct) members.push_back(k);
        for (int k : members) {
            const RealMatrix* b = kb->matrix_block_[k];
            if (left) { m += b->row_; n = n > b->column_ ? n : b->column_; }
            else { n += b->column_; m = m > b->row_ ? m : b->row_; }
        }
        if (left) n = n > t->right_dim_[sct] ? n : t->right_dim_[sct];
        else m = m > t->left_dim_[sct] ? m : t->left_dim_[sct];
        if ((long)m * n == 0) continue;
        std::vector<double> a((size_t)m * n, 0.0);
        int at = 0;
        for (int k : members) {
            const RealMatrix* b = kb->matrix_block_[k];
            for (int i = 0; i < b->row_; ++i)
                for (int j = 0; j < b->column_; ++j) {
                    const double v = b->matrix_element_[(long)i * b->column_ + j];
                    if (left) a[(size_t)(at + i) * n + j] = v;
                    else a[(size_t)i * n + at + j] = v;
                }
            at += left ? b->row_ : b->column_;
        }
        for (double v : a) fro2 += v * v;
        const int k = m < n ? m : n;
        std::vector<double> sv(k), sup(k > 1 ? k - 1 : 1);
        if (__real_LAPACKE_dgesvd(LAPACK_ROW_MAJOR, 'N', 'N', m, n, a.data(), n, sv.data(), nullptr, 1, nullptr, 1,
                                  sup.data()) != 0)
            return -2.0;
        all.insert(all.end(), sv.begin(), sv.end());
    }
    if (all.empty() || fro2 == 0.0) return -1.0;
    if (canpre > 1) canpre = 0.0;
    std::sort(all.begin(), all.end(), [](double x, double y) { return x > y; });
    const double fro = std::sqrt(fro2);
    g_pre_gap = 1e300;
    if (canpre > 0.0)
        for (double v : all)
            if (v > canpre && v / canpre < g_pre_gap) g_pre_gap = v / canpre;
    long above = 0;
    for (double v : all) above += v > canpre;
    if (max_dim > 0 && max_dim < above) return (all[max_dim - 1] - all[max_dim]) / fro;
    return -1.0;
}

static void canon_common(bool left, RealTensorLattice* self, int max_dim, double canpre) {
    int call = n_canon++;
    g_pre_gap = -1.0;
    g_cut_gap = g_trace ? truncation_gap(left, self, max_dim, canpre) : -1.0;
    bool dump = wanted(g_canon, call);
    NacWriter* w = dump ? new NacWriter(g_out + "/canon_" + std::to_string(call) + ".nac") : nullptr;
    if (w && g_synth) {
        probe::SplitMix rng(g_synth);
        synth_block(self->ket_tensor_, rng);
        w->scalar_i("synth_seed", (int)g_synth);
    }
    if (w) {
        w->scalar_i("left", left ? 1 : 0);
        w->scalar_i("site", site_of(self));
        w->scalar_i("max_dim", max_dim);
        w->scalar_d("canpre", canpre);
        probe::write_lattice(*w, "before", self);
    }
    if (left) __real__ZN17RealTensorLattice26LeftCanonicalTensorLatticeEid(self, max_dim, canpre);
    else __real__ZN17RealTensorLattice27RightCanonicalTensorLatticeEid(self, max_dim, canpre);
    trace("C", left ? 0 : 1, self);
    if (w) {
        probe::write_lattice(*w, "after", self);
        delete w;
    }
}
void __wrap__ZN17RealTensorLattice26LeftCanonicalTensorLatticeEid(RealTensorLattice* self, int m, double c) {
    canon_common(true, self, m, c);
}
void __wrap__ZN17RealTensorLattice27RightCanonicalTensorLatticeEid(RealTensorLattice* self, int m, double c) {
    canon_common(false, self, m, c);
}
}  // extern "C"

int main(int argc, char* argv[]) {
    if (argc != 2) {
        std::printf("Usage: %s inputfile\n", argv[0]);
        return 1;
    }
    if (const char* o = std::getenv("PROBE_OUT")) g_out = o;
    g_heff = parse_list(std::getenv("PROBE_HEFF"));
    g_env = parse_list(std::getenv("PROBE_ENV"));
    g_canon = parse_list(std::getenv("PROBE_CANON"));
    g_merge = parse_list(std::getenv("PROBE_MERGE"));
    g_struct_only = std::getenv("PROBE_STRUCT_ONLY") != nullptr;
    if (const char* s = std::getenv("PROBE_STOP")) g_stop = std::atoi(s);
    g_gauge = std::getenv("PROBE_GAUGE") != nullptr && std::atoi(std::getenv("PROBE_GAUGE")) != 0;
    if (const char* gs = std::getenv("PROBE_GAUGE_SEED")) {
        g_gauge_seed = std::strtoull(gs, nullptr, 10);
        g_gauge = g_gauge || g_gauge_seed != 0;
    }
    if (const char* sy = std::getenv("PROBE_SYNTH")) g_synth = std::strtoull(sy, nullptr, 10);
    g_round_f32 = std::getenv("PROBE_ROUND_F32") != nullptr;
    if (std::getenv("PROBE_TRACE")) g_trace = std::fopen((g_out + "/trace.txt").c_str(), "w");
    g_steps = std::fopen((g_out + "/steps.txt").c_str(), "w");

    auto input = InputGroup(argv[1], "input");
    int nx = input.getInt("num_site_x");
    int ny = input.getInt("num_site_y");
    int nb = input.getInt("num_boson");
    int d = input.getInt("physics_dim", 2);
    double flux = input.getDouble("flux");
    double Jx = input.getDouble("Jx");
    double Jy = input.getDouble("Jy");
    double U = input.getDouble("U");
    double mu = input.getDouble("mu");
    bool px = input.getBool("period_x");
    bool py = input.getBool("period_y");
    g_space = new RealSpinlessBoseSquareSpace(nx, ny, nb, d);
    g_ham = new RealSpinlessBoseSquareHamiltonian(nx, ny, d, flux * PI, Jx, Jy, U, mu, px, py);
    RealTensorRundmrg* run = new RealTensorRundmrg(g_space, g_ham, input);
    run->Run();
    std::fclose(g_steps);
    return 0;
}
