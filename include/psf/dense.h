// Minimal dense vector / matrix types for the headless solver interface.
//
// The reference's getters return Eigen types (Solver/abstractsolver.h:40-47);
// Eigen is not a dependency of this library, so these column-major containers stand in
// with the subset of the interface the solver uses (size, element access,
// raw data).
#pragma once

#include <cstddef>
#include <vector>

namespace psf {

template <class T>
class Vector {
public:
    Vector() = default;
    explicit Vector(std::size_t n, T v = T()) : d_(n, v) {}
    std::size_t size() const { return d_.size(); }
    std::size_t rows() const { return d_.size(); }
    void resize(std::size_t n) { d_.resize(n); }
    void setZero() { std::fill(d_.begin(), d_.end(), T()); }
    T &operator()(std::size_t i) { return d_[i]; }
    const T &operator()(std::size_t i) const { return d_[i]; }
    T &operator[](std::size_t i) { return d_[i]; }
    const T &operator[](std::size_t i) const { return d_[i]; }
    T *data() { return d_.data(); }
    const T *data() const { return d_.data(); }

private:
    std::vector<T> d_;
};

using VectorXd = Vector<double>;
using VectorXf = Vector<float>;

// Column-major like Eigen::MatrixXd.
class MatrixXd {
public:
    MatrixXd() = default;
    MatrixXd(std::size_t r, std::size_t c) : r_(r), c_(c), d_(r * c, 0.0) {}
    std::size_t rows() const { return r_; }
    std::size_t cols() const { return c_; }
    void resize(std::size_t r, std::size_t c)
    {
        r_ = r;
        c_ = c;
        d_.assign(r * c, 0.0);
    }
    double &operator()(std::size_t i, std::size_t j) { return d_[j * r_ + i]; }
    double operator()(std::size_t i, std::size_t j) const { return d_[j * r_ + i]; }
    double *data() { return d_.data(); }
    const double *data() const { return d_.data(); }

private:
    std::size_t r_ = 0, c_ = 0;
    std::vector<double> d_;
};

}  // namespace psf
