// Host-side model layer: MPO site operators, the MPO (Hamiltonian) with its
// per-bond operator quantum numbers, and the U(1) quantum-number tables of the
// MPS bonds.  Pure bookkeeping, built once on the host, exactly as the
// reference builds them (the block maps and the MPO feed the device schedules).
#pragma once

#include <string>
#include <vector>

#include "host/cplx.h"

namespace dmrg {

// Dense row-major host matrix used for the small one-time MPO algebra (T =
// double for the real models, Cplx for the complex ones).
template <class T>
struct HostMatrixT {
    int rows = 0, cols = 0;
    std::vector<T> v;
    HostMatrixT() = default;
    HostMatrixT(int r, int c) : rows(r), cols(c), v((size_t)r * c, T(0.0)) {}
    T& at(int i, int j) { return v[(size_t)i * cols + j]; }
    const T& at(int i, int j) const { return v[(size_t)i * cols + j]; }
};
using HostMatrix = HostMatrixT<double>;

// RealTensorOperator / ComplexTensorOperator (src/dmrg/realdmrg/
// real_tensor_operator.{h,cc}, complexdmrg/complex_tensor_operator.cc: the same
// code on complex values, zero tests by Norm): an MPO site tensor W[l][r](p1, p2).
template <class T>
class TensorOperatorT {
public:
    explicit TensorOperatorT(int physics_dim = 0) : d_(physics_dim) {}
    int get_physics_dim() const { return d_; }
    int get_left_bond() const { return lb_; }
    int get_right_bond() const { return rb_; }
    const T& w(int l, int r, int p1, int p2) const { return W_[idx(l, r, p1, p2)]; }
    T& w(int l, int r, int p1, int p2) { return W_[idx(l, r, p1, p2)]; }
    const std::vector<T>& data() const { return W_; }

    // Appends one term: leigh 0 (first site) grows the right bond, 1 (last site)
    // the left bond, otherwise both; the new corner is coeff * basic[op]
    // (ExpanTensorOperator, real_tensor_operator.cc:141-197).
    void ExpanTensorOperator(const std::vector<HostMatrixT<T>>& basic, int leigh, int op, const T& coeff);
    // Deparallelisation of the right bond (:199-237) / left bond (:239-275).
    void LeftParallelTensorOperator(int& num_unparallel, std::vector<int>& position, HostMatrixT<T>& transfer);
    void RightParallelTensorOperator(int& num_unparallel, std::vector<int>& position, HostMatrixT<T>& transfer);
    // Absorbs a neighbour's transfer matrix into the left (:277-319) / right (:321-361) bond.
    void LeftMergeTensorOperator(int num_unparallel, const HostMatrixT<T>& transfer);
    void RightMergeTensorOperator(int num_unparallel, const HostMatrixT<T>& transfer);
    // Any |W| > 1e-15 in the given row/column slice (:363-409).
    bool LeftCheckZero(int l, int p1) const;
    bool RightCheckZero(int r, int p2) const;
    bool MixedCheckZero(int l, int p2) const;

private:
    size_t idx(int l, int r, int p1, int p2) const { return (((size_t)l * rb_ + r) * d_ + p1) * d_ + p2; }
    void resize(int lb, int rb) {
        lb_ = lb;
        rb_ = rb;
        W_.assign((size_t)lb * rb * d_ * d_, T(0.0));
    }
    int d_ = 0, lb_ = 0, rb_ = 0;
    std::vector<T> W_;
};
using RealTensorOperator = TensorOperatorT<double>;
using ComplexTensorOperator = TensorOperatorT<Cplx>;

// RealMatrix::ParallelMatrix (src/tensor/real_matrix.cc:438-531) and its
// complex twin (complex_matrix.cc:451): removes columns (leigh 0) or rows
// (leigh 1) parallel to an earlier one.
template <class T>
void parallel_matrix(const HostMatrixT<T>& M, int leigh, int& num_unparallel, std::vector<int>& position,
                     HostMatrixT<T>& transfer);

// What the sweep engine reads of a Hamiltonian, real or complex: the MPO site
// tensors (values as doubles, complex ones interleaved (re, im)), their zero
// tests, and the operator quantum numbers of the MPO bonds.
class MpoHamiltonian {
public:
    virtual ~MpoHamiltonian() = default;
    virtual void DefineTensorHamiltonian() = 0;
    virtual bool is_complex() const = 0;
    int num_site() const { return num_site_; }
    // operator quantum numbers of MPO bond b (b = 0..num_site): rows x num_quantum
    const std::vector<std::vector<int>>& quantum_table(int b) const { return qtab_[b]; }
    int num_quantum() const { return num_quantum_; }
    virtual int physics_dim(int site) const = 0;
    virtual int left_bond(int site) const = 0;
    virtual int right_bond(int site) const = 0;
    virtual const double* values(int site) const = 0;
    virtual double wre(int site, int l, int r, int p1, int p2) const = 0;
    virtual double wim(int site, int l, int r, int p1, int p2) const = 0;
    virtual bool LeftCheckZero(int site, int l, int p1) const = 0;
    virtual bool RightCheckZero(int site, int r, int p2) const = 0;
    virtual bool MixedCheckZero(int site, int l, int p2) const = 0;
    bool w_nonzero(int site, int l, int r, int p1, int p2) const {
        return wre(site, l, r, p1, p2) != 0.0 || wim(site, l, r, p1, p2) != 0.0;
    }

protected:
    int num_site_ = 0, num_quantum_ = 1;
    std::vector<std::vector<std::vector<int>>> qtab_;
};

// RealTensorHamiltonian / ComplexTensorHamiltonian (real_tensor_hamiltonian.cc,
// complex_tensor_hamiltonian.cc): the MPO built term by term and deparallelised.
template <class T>
class TensorHamiltonianT : public MpoHamiltonian {
public:
    TensorOperatorT<T>& get_tensor_hamiltonian(int site) { return ops_[site]; }
    const TensorOperatorT<T>& get_tensor_hamiltonian(int site) const { return ops_[site]; }
    bool is_complex() const override;
    int physics_dim(int site) const override { return ops_[site].get_physics_dim(); }
    int left_bond(int site) const override { return ops_[site].get_left_bond(); }
    int right_bond(int site) const override { return ops_[site].get_right_bond(); }
    const double* values(int site) const override {
        return reinterpret_cast<const double*>(ops_[site].data().data());
    }
    double wre(int site, int l, int r, int p1, int p2) const override { return real_of(ops_[site].w(l, r, p1, p2)); }
    double wim(int site, int l, int r, int p1, int p2) const override { return imag_of(ops_[site].w(l, r, p1, p2)); }
    bool LeftCheckZero(int site, int l, int p1) const override { return ops_[site].LeftCheckZero(l, p1); }
    bool RightCheckZero(int site, int r, int p2) const override { return ops_[site].RightCheckZero(r, p2); }
    bool MixedCheckZero(int site, int l, int p2) const override { return ops_[site].MixedCheckZero(l, p2); }

protected:
    void init(int num_site, int physics_dim, int num_quantum);
    void ExpanTensorHamiltonian(int site, int op, const T& coeff, const std::vector<int>& expan_table);
    void ParallelTensorHamiltonian();
    void ParallelQuantumTable(int site, int num_unparallel, const std::vector<int>& position);

    std::vector<HostMatrixT<T>> basic_;
    std::vector<TensorOperatorT<T>> ops_;
};
using RealTensorHamiltonian = TensorHamiltonianT<double>;
using ComplexTensorHamiltonian = TensorHamiltonianT<Cplx>;

// H = sum over bonds of J (b+_p b_p' + h.c.) + sum_i [mu n + U n(n-1)]:
// RealSpinlessBoseSquareHamiltonian
// (model/hamiltonian/real_spinless_bose_square_hamiltonian.cc) for T = double,
// and ComplexSpinlessBoseSquareHamiltonian
// (model/hamiltonian/complex_spinless_bose_square_hamiltonian.cc), the same
// terms on complex operators, for T = Cplx.  Both store the flux and use none.
template <class T>
class SpinlessBoseSquareHamiltonianT : public TensorHamiltonianT<T> {
public:
    SpinlessBoseSquareHamiltonianT(int nx, int ny, int physics_dim, double flux_value, double hop_x, double hop_y,
                                   double inter_value, double chemical_value, bool period_x, bool period_y);
    void DefineTensorHamiltonian() override;

private:
    void DefineHamiltonian1(int p1, int p2, double coeff);  // b+_p1 b_p2
    void DefineHamiltonian2(int p1, int p2, double coeff);  // b_p1 b+_p2
    void DefineHamiltonian3(int p, double coeff);           // mu n + U n(n-1)
    int nx_, ny_, d_;
    double hop_x_, hop_y_, inter_, chem_;
    bool px_, py_;
};
using RealSpinlessBoseSquareHamiltonian = SpinlessBoseSquareHamiltonianT<double>;
using ComplexSpinlessBoseSquareHamiltonian = SpinlessBoseSquareHamiltonianT<Cplx>;

// Quantum-number tables of the MPS bonds (RealTensorSpace's quantum_table_ and
// its model hooks, real_tensor_space.cc:716-736 and
// model/space/real_spinless_bose_square_space.cc).
class QuantumSpace {
public:
    virtual ~QuantumSpace() = default;
    int num_site() const { return num_site_; }
    int physics_dim() const { return d_; }
    int num_quantum() const { return num_quantum_; }
    const std::vector<std::vector<int>>& table(int bond) const { return qtab_[bond]; }
    // physics index p with left + p == right, or -1
    virtual int CheckQuantumTable(int site, const std::vector<int>& left, const std::vector<int>& right) const = 0;
    virtual std::vector<int> MergeQuantumTable(const std::vector<int>& op, const std::vector<int>& space) const = 0;

protected:
    // Sorts a bond's rows by squared deviation from `mean` (ascending, the
    // reference's quicksort order) (ReorderQuantumTable).
    void ReorderQuantumTable(std::vector<std::vector<int>>& table, const std::vector<double>& mean);
    int num_site_ = 0, d_ = 0, num_quantum_ = 1;
    std::vector<std::vector<std::vector<int>>> qtab_;
};

class RealSpinlessBoseSquareSpace : public QuantumSpace {
public:
    RealSpinlessBoseSquareSpace(int nx, int ny, int num_boson, int physics_dim);
    int CheckQuantumTable(int site, const std::vector<int>& left, const std::vector<int>& right) const override;
    std::vector<int> MergeQuantumTable(const std::vector<int>& op, const std::vector<int>& space) const override;

private:
    int num_boson_;
};

// Two-component (spinful) bosons with U(1) x U(1): the species sit on
// alternating MPS sites (2 nx ny sites: species 0 of lattice site p at MPS site
// 2p, species 1 at 2p + 1), each with d = n_max + 1 states; bond quantum numbers
// are (N0, N1).  ComplexSpinfulBoseSquareSpace (model/space/
// complex_spinful_bose_square_space.cc:3-125) with real tensors.
class RealSpinfulBoseSquareSpace : public QuantumSpace {
public:
    RealSpinfulBoseSquareSpace(int nx, int ny, const int num_boson[2], int physics_dim);
    int CheckQuantumTable(int site, const std::vector<int>& left, const std::vector<int>& right) const override;
    std::vector<int> MergeQuantumTable(const std::vector<int>& op, const std::vector<int>& space) const override;

private:
    int num_boson_[2];
};

// H = sum over bonds of J_s (a+_s a_s' + h.c.) per species + sum_i [mu n + U_s/2
// n(n-1)] per species + U_ud n0 n1: ComplexSpinfulBoseSquareHamiltonian
// (model/hamiltonian/complex_spinful_bose_square_hamiltonian.cc:3-350), with
// the Peierls phase exp(i 2 pi (x+1) flux) on the y-bonds of column x (:297-331).
// T = double (RealSpinfulBoseSquareHamiltonian) needs flux 0 and rejects any
// other; T = Cplx (ComplexSpinfulBoseSquareHamiltonian) is the reference's class.
template <class T>
class SpinfulBoseSquareHamiltonianT : public TensorHamiltonianT<T> {
public:
    SpinfulBoseSquareHamiltonianT(int nx, int ny, int physics_dim, double flux, double hop_x, double hop_y,
                                  const double inter[3], double chemical, bool period_x, bool period_y);
    void DefineTensorHamiltonian() override;

private:
    void DefineHamiltonian1(int p1, int p2, const T& coeff);  // a+_p1 a_p2
    void DefineHamiltonian2(int p1, int p2, const T& coeff);  // a_p1 a+_p2
    void DefineHamiltonian3(int p, const T& coeff);           // mu n + U/2 n(n-1) of the site's species
    void DefineHamiltonian4(int p1, int p2, const T& coeff);  // n_p1 n_p2
    // the y-bond coefficients of column x: (conj(phase) J_y, phase J_y)
    void y_coeff(int x, T& first, T& second) const;
    int nx_, ny_, d_;
    double flux_, hop_x_, hop_y_, inter_[3], chem_;
    bool px_, py_;
};
using RealSpinfulBoseSquareHamiltonian = SpinfulBoseSquareHamiltonianT<double>;
using ComplexSpinfulBoseSquareHamiltonian = SpinfulBoseSquareHamiltonianT<Cplx>;

}  // namespace dmrg
