// Host-side model layer (see model.h).
#include "host/model.h"

#include <cmath>
#include <stdexcept>

#include "truncate.h"

namespace dmrg {

// ---------------------------------------------------------------------------
// RealTensorOperator
// ---------------------------------------------------------------------------
template <class T>
void TensorOperatorT<T>::ExpanTensorOperator(const std::vector<HostMatrixT<T>>& basic, int leigh, int op,
                                             const T& coeff) {
    int e0 = 1, e1 = 1;
    if (leigh == 0) e0 = 0;
    if (leigh == 1) e1 = 0;
    int nlb, nrb;
    if (lb_ == 0 && rb_ == 0) {
        nlb = 1;
        nrb = 1;
    } else {
        nlb = lb_ + e0;
        nrb = rb_ + e1;
    }
    std::vector<T> old = W_;
    const int olb = lb_, orb = rb_;
    resize(nlb, nrb);
    for (int l = 0; l < olb; ++l)
        for (int r = 0; r < orb; ++r)
            for (int p1 = 0; p1 < d_; ++p1)
                for (int p2 = 0; p2 < d_; ++p2) w(l, r, p1, p2) = old[(((size_t)l * orb + r) * d_ + p1) * d_ + p2];
    const int il = e0 * olb, ir = e1 * orb;
    for (int p1 = 0; p1 < d_; ++p1)
        for (int p2 = 0; p2 < d_; ++p2) w(il, ir, p1, p2) = coeff * basic[op].at(p1, p2);
}

namespace {

// The reference's element test for parallel columns/rows (util/general.h:
// isParallelElement): a zero reference entry must face a zero; otherwise all
// ratios must agree within 1e-8 (the first defines the prefactor).
void parallel_element(double e0, double e1, int position, int& info, double& prefactor, bool& zero) {
    if (std::fabs(e1) <= 1e-10) {
        if (std::fabs(e0) > 1e-10) {
            info = -1;
            prefactor = 1.0;
        }
    } else {
        const double factor = e0 / e1;
        if (zero) {
            info = position;
            prefactor = factor;
            zero = false;
        } else if (std::fabs(factor - prefactor) > 1e-8) {
            info = -1;
            prefactor = 1.0;
        }
    }
}


// The complex form (the Complex overload of isParallelElement, util/general.h):
// Norm in place of fabs, the reference's complex quotient.
void parallel_element(const Cplx& e0, const Cplx& e1, int position, int& info, Cplx& prefactor, bool& zero) {
    if (norm_of(e1) <= 1e-10) {
        if (norm_of(e0) > 1e-10) {
            info = -1;
            prefactor = Cplx(1.0);
        }
    } else {
        const Cplx factor = e0 / e1;
        if (zero) {
            info = position;
            prefactor = factor;
            zero = false;
        } else if (norm_of(factor - prefactor) > 1e-8) {
            info = -1;
            prefactor = Cplx(1.0);
        }
    }
}

}  // namespace

template <class S>
void parallel_matrix(const HostMatrixT<S>& M, int leigh, int& nu, std::vector<int>& pos, HostMatrixT<S>& T) {
    int info = 0;
    S prefactor = S(0.0);
    bool zero = true;
    if (leigh == 0) {
        pos.assign(M.cols, -1);
        pos[0] = 0;
        T = HostMatrixT<S>(M.cols, M.cols);
        T.at(0, 0) = S(1.0);
        nu = 1;
        for (int r = 0; r < M.cols; ++r) {
            for (int k = 0; k < nu; ++k) {
                info = nu;
                prefactor = S(0.0);
                zero = true;
                for (int l = 0; l < M.rows; ++l) {
                    parallel_element(M.at(l, r), M.at(l, pos[k]), pos[k], info, prefactor, zero);
                    if (info == -1) break;
                }
                if (info != -1) {
                    T.at(k, r) = prefactor;
                    break;
                }
            }
            if (info == -1) {
                pos[nu] = r;
                T.at(nu, r) = S(1.0);
                ++nu;
            }
        }
    } else {
        pos.assign(M.rows, -1);
        pos[0] = 0;
        T = HostMatrixT<S>(M.rows, M.rows);
        T.at(0, 0) = S(1.0);
        nu = 1;
        for (int l = 0; l < M.rows; ++l) {
            for (int k = 0; k < nu; ++k) {
                info = nu;
                prefactor = S(0.0);
                zero = true;
                for (int r = 0; r < M.cols; ++r) {
                    parallel_element(M.at(l, r), M.at(pos[k], r), pos[k], info, prefactor, zero);
                    if (info == -1) break;
                }
                if (info != -1) {
                    T.at(l, k) = prefactor;
                    break;
                }
            }
            if (info == -1) {
                pos[nu] = l;
                T.at(l, nu) = S(1.0);
                ++nu;
            }
        }
    }
}

template <class T>
void TensorOperatorT<T>::LeftParallelTensorOperator(int& nu, std::vector<int>& pos, HostMatrixT<T>& Tm) {
    HostMatrixT<T> R(lb_ * d_ * d_, rb_);
    for (int l = 0; l < lb_; ++l)
        for (int r = 0; r < rb_; ++r)
            for (int p1 = 0; p1 < d_; ++p1)
                for (int p2 = 0; p2 < d_; ++p2) R.at(p2 + (p1 + l * d_) * d_, r) = w(l, r, p1, p2);
    parallel_matrix(R, 0, nu, pos, Tm);
    resize(lb_, nu);
    for (int l = 0; l < lb_; ++l)
        for (int r = 0; r < rb_; ++r)
            for (int p1 = 0; p1 < d_; ++p1)
                for (int p2 = 0; p2 < d_; ++p2) w(l, r, p1, p2) = R.at(p2 + (p1 + l * d_) * d_, pos[r]);
}

template <class T>
void TensorOperatorT<T>::RightParallelTensorOperator(int& nu, std::vector<int>& pos, HostMatrixT<T>& Tm) {
    HostMatrixT<T> R(lb_, rb_ * d_ * d_);
    for (int l = 0; l < lb_; ++l)
        for (int r = 0; r < rb_; ++r)
            for (int p1 = 0; p1 < d_; ++p1)
                for (int p2 = 0; p2 < d_; ++p2) R.at(l, p2 + (p1 + r * d_) * d_) = w(l, r, p1, p2);
    parallel_matrix(R, 1, nu, pos, Tm);
    resize(nu, rb_);
    for (int l = 0; l < lb_; ++l)
        for (int r = 0; r < rb_; ++r)
            for (int p1 = 0; p1 < d_; ++p1)
                for (int p2 = 0; p2 < d_; ++p2) w(l, r, p1, p2) = R.at(pos[l], p2 + (p1 + r * d_) * d_);
}

template <class T>
void TensorOperatorT<T>::LeftMergeTensorOperator(int nu, const HostMatrixT<T>& Tm) {
    const int merge = Tm.cols;
    if (merge != lb_) throw std::runtime_error("merge dimension is not match in LeftMergeTensorOperator");
    std::vector<T> old = W_;
    const int orb = rb_;
    resize(nu, orb);
    for (int l = 0; l < nu; ++l)
        for (int r = 0; r < orb; ++r)
            for (int p1 = 0; p1 < d_; ++p1)
                for (int p2 = 0; p2 < d_; ++p2) {
                    T e = T(0.0);
                    for (int m = 0; m < merge; ++m)
                        e += Tm.at(l, m) * old[(((size_t)m * orb + r) * d_ + p1) * d_ + p2];
                    w(l, r, p1, p2) = e;
                }
}

template <class T>
void TensorOperatorT<T>::RightMergeTensorOperator(int nu, const HostMatrixT<T>& Tm) {
    const int merge = Tm.rows;
    if (merge != rb_) throw std::runtime_error("merge dimension is not match in RightMergeTensorOperator");
    std::vector<T> old = W_;
    const int olb = lb_, orb = rb_;
    resize(olb, nu);
    for (int l = 0; l < olb; ++l)
        for (int r = 0; r < nu; ++r)
            for (int p1 = 0; p1 < d_; ++p1)
                for (int p2 = 0; p2 < d_; ++p2) {
                    T e = T(0.0);
                    for (int m = 0; m < merge; ++m)
                        e += Tm.at(m, r) * old[(((size_t)l * orb + m) * d_ + p1) * d_ + p2];
                    w(l, r, p1, p2) = e;
                }
}

template <class T>
bool TensorOperatorT<T>::LeftCheckZero(int l, int p1) const {
    for (int r = 0; r < rb_; ++r)
        for (int p2 = 0; p2 < d_; ++p2)
            if (norm_of(w(l, r, p1, p2)) > 1e-15) return true;
    return false;
}
template <class T>
bool TensorOperatorT<T>::RightCheckZero(int r, int p2) const {
    for (int l = 0; l < lb_; ++l)
        for (int p1 = 0; p1 < d_; ++p1)
            if (norm_of(w(l, r, p1, p2)) > 1e-15) return true;
    return false;
}
template <class T>
bool TensorOperatorT<T>::MixedCheckZero(int l, int p2) const {
    for (int r = 0; r < rb_; ++r)
        for (int p1 = 0; p1 < d_; ++p1)
            if (norm_of(w(l, r, p1, p2)) > 1e-15) return true;
    return false;
}

// ---------------------------------------------------------------------------
// RealTensorHamiltonian
// ---------------------------------------------------------------------------
template <>
bool TensorHamiltonianT<double>::is_complex() const {
    return false;
}
template <>
bool TensorHamiltonianT<Cplx>::is_complex() const {
    return true;
}

template <class T>
void TensorHamiltonianT<T>::init(int num_site, int d, int num_quantum) {
    num_site_ = num_site;
    num_quantum_ = num_quantum;
    qtab_.assign(num_site + 1, {});
    ops_.assign(num_site, TensorOperatorT<T>(d));
}

template <class T>
void TensorHamiltonianT<T>::ExpanTensorHamiltonian(int site, int op, const T& coeff, const std::vector<int>& table) {
    int leigh = -1;
    if (site == 0) leigh = 0;
    if (site == num_site_ - 1) leigh = 1;
    ops_[site].ExpanTensorOperator(basic_, leigh, op, coeff);
    if (site < num_site_ - 1) qtab_[site + 1].push_back(table);
}

template <class T>
void TensorHamiltonianT<T>::ParallelQuantumTable(int site, int nu, const std::vector<int>& pos) {
    std::vector<std::vector<int>> t(nu);
    for (int i = 0; i < nu; ++i) t[i] = qtab_[site][pos[i]];
    qtab_[site] = t;
}

template <class T>
void TensorHamiltonianT<T>::ParallelTensorHamiltonian() {
    int nu;
    std::vector<int> pos;
    HostMatrixT<T> Tm;
    for (int i = 0; i < num_site_ - 1; ++i) {
        ops_[i].LeftParallelTensorOperator(nu, pos, Tm);
        ops_[i + 1].LeftMergeTensorOperator(nu, Tm);
        ParallelQuantumTable(i + 1, nu, pos);
    }
    for (int i = num_site_ - 1; i > 0; --i) {
        ops_[i].RightParallelTensorOperator(nu, pos, Tm);
        ops_[i - 1].RightMergeTensorOperator(nu, Tm);
        ParallelQuantumTable(i, nu, pos);
    }
}

template class TensorOperatorT<double>;
template class TensorOperatorT<Cplx>;
template class TensorHamiltonianT<double>;
template class TensorHamiltonianT<Cplx>;

template <class T>
SpinlessBoseSquareHamiltonianT<T>::SpinlessBoseSquareHamiltonianT(int nx, int ny, int d, double flux_value,
                                                                  double hop_x, double hop_y, double inter,
                                                                  double chem, bool px, bool py)
    : nx_(nx), ny_(ny), d_(d), hop_x_(hop_x), hop_y_(hop_y), inter_(inter), chem_(chem), px_(px), py_(py) {
    (void)flux_value;  // stored but unused by both spinless models (as in the reference)
    this->init(nx * ny, d, 1);
    // 0 = I, 1 = b+, 2 = b, 3 = n, 4 = mu n + U n(n-1)
    auto& basic = this->basic_;
    basic.assign(5, HostMatrixT<T>(d, d));
    for (int i = 0; i < d; ++i) {
        basic[0].at(i, i) = T(1.0);
        basic[3].at(i, i) = T((double)i);
        basic[4].at(i, i) = T(chem * i + inter * i * (i - 1));
    }
    for (int i = 1; i < d; ++i) {
        basic[1].at(i, i - 1) = T(std::sqrt((double)i));
        basic[2].at(i - 1, i) = T(std::sqrt((double)i));
    }
}

template <class T>
void SpinlessBoseSquareHamiltonianT<T>::DefineHamiltonian1(int p1, int p2, double coeff) {
    if (p1 >= p2) throw std::runtime_error("position1 >= position2 in DefineHamiltonian1");
    for (int i = 0; i < this->num_site_; ++i) {
        int op = 0, q = 0;
        double c = 1.0;
        if (i == p1) {
            op = 1;
            q = 1;
        }
        if (i > p1 && i < p2) q = 1;
        if (i == p2) {
            op = 2;
            c = coeff;
            q = 0;
        }
        this->ExpanTensorHamiltonian(i, op, T(c), {q});
    }
}

template <class T>
void SpinlessBoseSquareHamiltonianT<T>::DefineHamiltonian2(int p1, int p2, double coeff) {
    if (p1 >= p2) throw std::runtime_error("position1 >= position2 in DefineHamiltonian2");
    for (int i = 0; i < this->num_site_; ++i) {
        int op = 0, q = 0;
        double c = 1.0;
        if (i == p1) {
            op = 2;
            q = -1;
        }
        if (i > p1 && i < p2) q = -1;
        if (i == p2) {
            op = 1;
            c = coeff;
            q = 0;
        }
        this->ExpanTensorHamiltonian(i, op, T(c), {q});
    }
}

template <class T>
void SpinlessBoseSquareHamiltonianT<T>::DefineHamiltonian3(int p, double coeff) {
    for (int i = 0; i < this->num_site_; ++i) {
        int op = 0;
        double c = 1.0;
        if (i == p) {
            op = 4;
            c = coeff;
        }
        this->ExpanTensorHamiltonian(i, op, T(c), {0});
    }
}

template <class T>
void SpinlessBoseSquareHamiltonianT<T>::DefineTensorHamiltonian() {
    auto& qtab = this->qtab_;
    const int ns = this->num_site_;
    qtab[0] = {{0}};
    qtab[ns] = {{0}};
    for (int i = 0; i < nx_; ++i)
        for (int j = 0; j < ny_; ++j) {
            const int p0 = j + i * ny_;  // column-major site order (p = j + i * Ny)
            if (hop_x_ != 0) {
                const int p1 = j + ((i + 1) % nx_) * ny_;
                if (i + 1 < nx_) {
                    DefineHamiltonian1(p0, p1, hop_x_);
                    DefineHamiltonian2(p0, p1, hop_x_);
                } else if (nx_ > 2 && px_) {
                    DefineHamiltonian1(p1, p0, hop_x_);
                    DefineHamiltonian2(p1, p0, hop_x_);
                }
            }
            if (hop_y_ != 0) {
                const int p1 = (j + 1) % ny_ + i * ny_;
                if (j + 1 < ny_) {
                    DefineHamiltonian1(p0, p1, hop_y_);
                    DefineHamiltonian2(p0, p1, hop_y_);
                } else if (ny_ > 2 && py_) {
                    DefineHamiltonian1(p1, p0, hop_y_);
                    DefineHamiltonian2(p1, p0, hop_y_);
                }
            }
            if (chem_ != 0 || inter_ != 0) DefineHamiltonian3(p0, 1.0);
            this->ParallelTensorHamiltonian();
        }
}

template class SpinlessBoseSquareHamiltonianT<double>;
template class SpinlessBoseSquareHamiltonianT<Cplx>;

// ---------------------------------------------------------------------------
// Quantum tables of the MPS bonds
// ---------------------------------------------------------------------------
void QuantumSpace::ReorderQuantumTable(std::vector<std::vector<int>>& table, const std::vector<double>& mean) {
    const int n = (int)table.size();
    if (n == 0) return;
    std::vector<double> dev(n, 0.0);
    std::vector<int> index(n);
    for (int i = 0; i < n; ++i) {
        index[i] = i;
        for (int j = 0; j < num_quantum_; ++j) dev[i] += std::pow(table[i][j] - mean[j], 2);
    }
    quicksort_with_index(dev.data(), index.data(), n, false);
    std::vector<std::vector<int>> out(n);
    for (int k = 0; k < n; ++k) out[k] = table[index[k]];
    table = out;
}

RealSpinlessBoseSquareSpace::RealSpinlessBoseSquareSpace(int nx, int ny, int num_boson, int d)
    : num_boson_(num_boson) {
    num_site_ = nx * ny;
    d_ = d;
    num_quantum_ = 1;
    qtab_.assign(num_site_ + 1, {});
    for (int i = 0; i <= num_site_; ++i) {
        int lo, hi;
        double mean;
        if (i == 0) {
            lo = hi = 0;
            mean = 0.0;
        } else {
            const int min_left = 0, max_left = (d - 1) * i;
            const int min_right = num_boson - (num_site_ - i) * (d - 1), max_right = num_boson;
            lo = std::max(min_left, min_right);
            hi = std::min(max_left, max_right);
            mean = (double)num_boson / num_site_ * i;
        }
        std::vector<std::vector<int>> t;
        for (int q = lo; q <= hi; ++q) t.push_back({q});
        ReorderQuantumTable(t, {mean});
        qtab_[i] = t;
    }
}

int RealSpinlessBoseSquareSpace::CheckQuantumTable(int, const std::vector<int>& left,
                                                   const std::vector<int>& right) const {
    for (int i = 0; i < d_; ++i)
        if (left[0] + i == right[0]) return i;
    return -1;
}

std::vector<int> RealSpinlessBoseSquareSpace::MergeQuantumTable(const std::vector<int>& op,
                                                                const std::vector<int>& space) const {
    return {op[0] + space[0]};
}

}  // namespace dmrg

namespace dmrg {

// ---------------------------------------------------------------------------
// Spinful bosons on interleaved species sites
// ---------------------------------------------------------------------------
template <class T>
SpinfulBoseSquareHamiltonianT<T>::SpinfulBoseSquareHamiltonianT(int nx, int ny, int d, double flux, double hop_x,
                                                                double hop_y, const double inter[3], double chem,
                                                                bool px, bool py)
    : nx_(nx), ny_(ny), d_(d), flux_(flux), hop_x_(hop_x), hop_y_(hop_y), chem_(chem), px_(px), py_(py) {
    if (flux != 0.0 && !this->is_complex())
        throw std::runtime_error("the spinful model's Peierls phases (flux != 0) need complex tensors");
    for (int t = 0; t < 3; ++t) inter_[t] = inter[t];
    this->init(2 * nx * ny, d, 2);
    // 0 = I, 1 = a+, 2 = a, 3 = n, 4 = mu n + U_0/2 n(n-1), 5 = mu n + U_1/2 n(n-1)
    // (one chemical potential for both species, as the reference's operator 5
    // takes the first species' value, complex_spinful_bose_square_hamiltonian.cc:61)
    auto& basic = this->basic_;
    basic.assign(6, HostMatrixT<T>(d, d));
    for (int i = 0; i < d; ++i) {
        basic[0].at(i, i) = T(1.0);
        basic[3].at(i, i) = T((double)i);
        basic[4].at(i, i) = T(chem * i + 0.5 * inter_[0] * i * (i - 1));
        basic[5].at(i, i) = T(chem * i + 0.5 * inter_[1] * i * (i - 1));
    }
    for (int i = 1; i < d; ++i) {
        basic[1].at(i, i - 1) = T(std::sqrt((double)i));
        basic[2].at(i - 1, i) = T(std::sqrt((double)i));
    }
}

template <>
void SpinfulBoseSquareHamiltonianT<double>::y_coeff(int, double& first, double& second) const {
    first = second = hop_y_;
}

// phase = Phase(2 pi (x+1) flux); the first term of a bond takes Conj(phase) J_y,
// the second phase J_y (complex_spinful_bose_square_hamiltonian.cc:297-311)
template <>
void SpinfulBoseSquareHamiltonianT<Cplx>::y_coeff(int x, Cplx& first, Cplx& second) const {
    const Cplx phase = phase_of(2 * M_PI * (x + 1) * flux_);
    first = conj_of(phase) * hop_y_;
    second = phase * hop_y_;
}

// The operator's quantum number between p1 and p2 is carried by the species of p1.
template <class T>
void SpinfulBoseSquareHamiltonianT<T>::DefineHamiltonian1(int p1, int p2, const T& coeff) {
    if (p1 >= p2) throw std::runtime_error("position1 >= position2 in DefineHamiltonian1");
    const std::vector<int> q = p1 % 2 == 0 ? std::vector<int>{1, 0} : std::vector<int>{0, 1};
    for (int i = 0; i < this->num_site_; ++i) {
        int op = 0;
        T c = T(1.0);
        std::vector<int> t{0, 0};
        if (i == p1) {
            op = 1;
            t = q;
        }
        if (i > p1 && i < p2) t = q;
        if (i == p2) {
            op = 2;
            c = coeff;
            t = {0, 0};
        }
        this->ExpanTensorHamiltonian(i, op, c, t);
    }
}

template <class T>
void SpinfulBoseSquareHamiltonianT<T>::DefineHamiltonian2(int p1, int p2, const T& coeff) {
    if (p1 >= p2) throw std::runtime_error("position1 >= position2 in DefineHamiltonian2");
    const std::vector<int> q = p1 % 2 == 0 ? std::vector<int>{-1, 0} : std::vector<int>{0, -1};
    for (int i = 0; i < this->num_site_; ++i) {
        int op = 0;
        T c = T(1.0);
        std::vector<int> t{0, 0};
        if (i == p1) {
            op = 2;
            t = q;
        }
        if (i > p1 && i < p2) t = q;
        if (i == p2) {
            op = 1;
            c = coeff;
            t = {0, 0};
        }
        this->ExpanTensorHamiltonian(i, op, c, t);
    }
}

template <class T>
void SpinfulBoseSquareHamiltonianT<T>::DefineHamiltonian3(int p, const T& coeff) {
    for (int i = 0; i < this->num_site_; ++i) {
        int op = 0;
        T c = T(1.0);
        if (i == p) {
            op = p % 2 == 0 ? 4 : 5;
            c = coeff;
        }
        this->ExpanTensorHamiltonian(i, op, c, {0, 0});
    }
}

template <class T>
void SpinfulBoseSquareHamiltonianT<T>::DefineHamiltonian4(int p1, int p2, const T& coeff) {
    for (int i = 0; i < this->num_site_; ++i) {
        int op = 0;
        T c = T(1.0);
        if (i == p1) op = 3;
        if (i == p2) {
            op = 3;
            c = coeff;
        }
        this->ExpanTensorHamiltonian(i, op, c, {0, 0});
    }
}

// ComplexSpinfulBoseSquareHamiltonian::DefineTensorHamiltonian (:249-350): the
// same term order (it decides the MPO bond indices).
template <class T>
void SpinfulBoseSquareHamiltonianT<T>::DefineTensorHamiltonian() {
    const int n = this->num_site_;
    this->qtab_[0] = {{0, 0}};
    this->qtab_[n] = {{0, 0}};
    for (int i = 0; i < nx_; ++i)
        for (int j = 0; j < ny_; ++j) {
            const int p0 = j + i * ny_;
            for (int s = 0; s < 2 && hop_x_ != 0; ++s) {
                const int p1 = j + ((i + 1) % nx_) * ny_;
                if (i + 1 < nx_) {
                    DefineHamiltonian1(2 * p0 + s, 2 * p1 + s, T(hop_x_));
                    DefineHamiltonian2(2 * p0 + s, 2 * p1 + s, T(hop_x_));
                } else if (nx_ > 2 && px_) {
                    DefineHamiltonian1(2 * p1 + s, 2 * p0 + s, T(hop_x_));
                    DefineHamiltonian2(2 * p1 + s, 2 * p0 + s, T(hop_x_));
                }
            }
            for (int s = 0; s < 2 && hop_y_ != 0; ++s) {
                const int p1 = (j + 1) % ny_ + i * ny_;
                T first, second;
                y_coeff(i, first, second);
                if (j + 1 < ny_) {
                    DefineHamiltonian1(2 * p0 + s, 2 * p1 + s, first);
                    DefineHamiltonian2(2 * p0 + s, 2 * p1 + s, second);
                } else if (ny_ > 2 && py_) {  // the wrap adds its two terms in the other order
                    DefineHamiltonian2(2 * p1 + s, 2 * p0 + s, first);
                    DefineHamiltonian1(2 * p1 + s, 2 * p0 + s, second);
                }
            }
            if (chem_ != 0.0 || inter_[0] != 0.0) DefineHamiltonian3(2 * p0, T(1.0));
            if (chem_ != 0.0 || inter_[1] != 0.0) DefineHamiltonian3(2 * p0 + 1, T(1.0));
            if (inter_[2] != 0.0) DefineHamiltonian4(2 * p0, 2 * p0 + 1, T(inter_[2]));
            this->ParallelTensorHamiltonian();
        }
}

template class SpinfulBoseSquareHamiltonianT<double>;
template class SpinfulBoseSquareHamiltonianT<Cplx>;

// ComplexSpinfulBoseSquareSpace::DefineQuantumTable (:28-97): per bond, the
// admissible (N0, N1) with species 0 counted over the first (i+1)/2 MPS sites
// and species 1 over the first i/2, enumerated with N0 fastest, then ordered by
// squared deviation from the mean filling (ReorderQuantumTable).
RealSpinfulBoseSquareSpace::RealSpinfulBoseSquareSpace(int nx, int ny, const int num_boson[2], int d) {
    num_boson_[0] = num_boson[0];
    num_boson_[1] = num_boson[1];
    num_site_ = 2 * nx * ny;
    d_ = d;
    num_quantum_ = 2;
    qtab_.assign(num_site_ + 1, {});
    const int half = num_site_ / 2;
    for (int i = 0; i <= num_site_; ++i) {
        int lo[2] = {0, 0}, hi[2] = {0, 0};
        double mean[2] = {0.0, 0.0};
        if (i > 0) {
            const int pos[2] = {(i + 1) / 2, i / 2};
            for (int t = 0; t < 2; ++t) {
                const int min_left = 0, max_left = (d - 1) * pos[t];
                const int min_right = num_boson_[t] - (half - pos[t]) * (d - 1), max_right = num_boson_[t];
                lo[t] = std::max(min_left, min_right);
                hi[t] = std::min(max_left, max_right);
                mean[t] = (double)num_boson_[t] / half * pos[t];
            }
        }
        std::vector<std::vector<int>> t;
        for (int b = lo[1]; b <= hi[1]; ++b)
            for (int a = lo[0]; a <= hi[0]; ++a) t.push_back({a, b});
        ReorderQuantumTable(t, {mean[0], mean[1]});
        qtab_[i] = t;
    }
}

int RealSpinfulBoseSquareSpace::CheckQuantumTable(int site, const std::vector<int>& left,
                                                  const std::vector<int>& right) const {
    const int shift = site % 2;
    for (int i = 0; i < d_; ++i) {
        int p[2] = {0, 0};
        p[shift] = i;
        if (left[0] + p[0] == right[0] && left[1] + p[1] == right[1]) return i;
    }
    return -1;
}

std::vector<int> RealSpinfulBoseSquareSpace::MergeQuantumTable(const std::vector<int>& op,
                                                               const std::vector<int>& space) const {
    return {op[0] + space[0], op[1] + space[1]};
}

}  // namespace dmrg
