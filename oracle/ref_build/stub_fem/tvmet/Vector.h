// Stand-in for tvmet's fixed-size Vector and Matrix (oracle harness only).
// Eager arithmetic over plain arrays.  As in tvmet, assigning a single value
// (or constructing from one) fills every element, and `v = a, b, c;` assigns
// element by element; normalize() returns a new vector and leaves its
// argument as it is.
#ifndef REF_FEM_STUB_TVMET_H
#define REF_FEM_STUB_TVMET_H
#include <cmath>
#include <cstddef>
#include <ostream>

namespace tvmet {

template <class T, std::size_t N> class Vector;
template <class T, std::size_t R, std::size_t C> class Matrix;

// comma initialiser: the first value fills everything unless more follow
template <class T> class CommaInit {
public:
    CommaInit(T *d, std::size_t n, T x) : d_(d), n_(n), i_(1), single_(true) { d_[0] = x; }
    CommaInit(const CommaInit &o) : d_(o.d_), n_(o.n_), i_(o.i_), single_(o.single_) { o.single_ = false; }
    ~CommaInit() {
        if (single_)
            for (std::size_t k = 1; k < n_; k++) d_[k] = d_[0];
    }
    CommaInit &operator,(T x) {
        single_ = false;
        if (i_ < n_) d_[i_++] = x;
        return *this;
    }
private:
    T *d_;
    std::size_t n_, i_;
    mutable bool single_;
};

template <class T, std::size_t N> class Vector {
public:
    typedef T value_type;
    Vector() { for (std::size_t i = 0; i < N; i++) d_[i] = T(); }
    explicit Vector(T x) { for (std::size_t i = 0; i < N; i++) d_[i] = x; }
    Vector(T a, T b) { d_[0] = a; if (N > 1) d_[1] = b; }
    Vector(T a, T b, T c) { d_[0] = a; if (N > 1) d_[1] = b; if (N > 2) d_[2] = c; }
    CommaInit<T> operator=(T x) { return CommaInit<T>(d_, N, x); }
    T &operator()(std::size_t i) { return d_[i]; }
    const T &operator()(std::size_t i) const { return d_[i]; }
    T &operator[](std::size_t i) { return d_[i]; }
    const T &operator[](std::size_t i) const { return d_[i]; }
    static std::size_t size() { return N; }
    T *data() { return d_; }
    const T *data() const { return d_; }
    Vector &operator+=(const Vector &o) { for (std::size_t i = 0; i < N; i++) d_[i] += o.d_[i]; return *this; }
    Vector &operator-=(const Vector &o) { for (std::size_t i = 0; i < N; i++) d_[i] -= o.d_[i]; return *this; }
    Vector &operator*=(T s) { for (std::size_t i = 0; i < N; i++) d_[i] *= s; return *this; }
    Vector &operator/=(T s) { for (std::size_t i = 0; i < N; i++) d_[i] /= s; return *this; }
private:
    T d_[N];
};

template <class T, std::size_t N> Vector<T, N> operator+(const Vector<T, N> &a, const Vector<T, N> &b) { Vector<T, N> r(a); r += b; return r; }
template <class T, std::size_t N> Vector<T, N> operator-(const Vector<T, N> &a, const Vector<T, N> &b) { Vector<T, N> r(a); r -= b; return r; }
template <class T, std::size_t N> Vector<T, N> operator-(const Vector<T, N> &a) { Vector<T, N> r(a); r *= T(-1); return r; }
template <class T, std::size_t N> Vector<T, N> operator*(const Vector<T, N> &a, T s) { Vector<T, N> r(a); r *= s; return r; }
template <class T, std::size_t N> Vector<T, N> operator*(T s, const Vector<T, N> &a) { Vector<T, N> r(a); r *= s; return r; }
template <class T, std::size_t N> Vector<T, N> operator/(const Vector<T, N> &a, T s) { Vector<T, N> r(a); r /= s; return r; }
template <class T, std::size_t N> T dot(const Vector<T, N> &a, const Vector<T, N> &b) {
    T s = T(); for (std::size_t i = 0; i < N; i++) s += a(i) * b(i); return s;
}
template <class T, std::size_t N> T norm2(const Vector<T, N> &a) { return std::sqrt(dot(a, a)); }
template <class T, std::size_t N> Vector<T, N> normalize(const Vector<T, N> &a) { return a / norm2(a); }
template <class T> Vector<T, 3> cross(const Vector<T, 3> &a, const Vector<T, 3> &b) {
    return Vector<T, 3>(a(1) * b(2) - a(2) * b(1), a(2) * b(0) - a(0) * b(2), a(0) * b(1) - a(1) * b(0));
}
template <class T, std::size_t N> std::ostream &operator<<(std::ostream &o, const Vector<T, N> &a) {
    o << "[";
    for (std::size_t i = 0; i < N; i++) o << (i ? ", " : "") << a(i);
    return o << "]";
}

template <class T, std::size_t R, std::size_t C> class Matrix {
public:
    typedef T value_type;
    Matrix() { for (std::size_t i = 0; i < R * C; i++) d_[i] = T(); }
    explicit Matrix(T x) { for (std::size_t i = 0; i < R * C; i++) d_[i] = x; }
    CommaInit<T> operator=(T x) { return CommaInit<T>(d_, R * C, x); }
    T &operator()(std::size_t i, std::size_t j) { return d_[i * C + j]; }
    const T &operator()(std::size_t i, std::size_t j) const { return d_[i * C + j]; }
    static std::size_t rows() { return R; }
    static std::size_t cols() { return C; }
    T *data() { return d_; }
    const T *data() const { return d_; }
    Matrix &operator+=(const Matrix &o) { for (std::size_t i = 0; i < R * C; i++) d_[i] += o.d_[i]; return *this; }
    Matrix &operator-=(const Matrix &o) { for (std::size_t i = 0; i < R * C; i++) d_[i] -= o.d_[i]; return *this; }
    Matrix &operator*=(T s) { for (std::size_t i = 0; i < R * C; i++) d_[i] *= s; return *this; }
    Matrix &operator/=(T s) { for (std::size_t i = 0; i < R * C; i++) d_[i] /= s; return *this; }
private:
    T d_[R * C];
};

template <class T, std::size_t R, std::size_t C> Matrix<T, R, C> operator+(const Matrix<T, R, C> &a, const Matrix<T, R, C> &b) { Matrix<T, R, C> r(a); r += b; return r; }
template <class T, std::size_t R, std::size_t C> Matrix<T, R, C> operator-(const Matrix<T, R, C> &a, const Matrix<T, R, C> &b) { Matrix<T, R, C> r(a); r -= b; return r; }
template <class T, std::size_t R, std::size_t C> Matrix<T, R, C> operator-(const Matrix<T, R, C> &a) { Matrix<T, R, C> r(a); r *= T(-1); return r; }
template <class T, std::size_t R, std::size_t C> Matrix<T, R, C> operator*(const Matrix<T, R, C> &a, T s) { Matrix<T, R, C> r(a); r *= s; return r; }
template <class T, std::size_t R, std::size_t C> Matrix<T, R, C> operator*(T s, const Matrix<T, R, C> &a) { Matrix<T, R, C> r(a); r *= s; return r; }
template <class T, std::size_t R, std::size_t C> Matrix<T, R, C> operator/(const Matrix<T, R, C> &a, T s) { Matrix<T, R, C> r(a); r /= s; return r; }
template <class T, std::size_t R, std::size_t K, std::size_t C>
Matrix<T, R, C> operator*(const Matrix<T, R, K> &a, const Matrix<T, K, C> &b) {
    Matrix<T, R, C> r(T(0));
    for (std::size_t i = 0; i < R; i++)
        for (std::size_t j = 0; j < C; j++) {
            T s = T();
            for (std::size_t k = 0; k < K; k++) s += a(i, k) * b(k, j);
            r(i, j) = s;
        }
    return r;
}
template <class T, std::size_t R, std::size_t C>
Vector<T, R> operator*(const Matrix<T, R, C> &a, const Vector<T, C> &x) {
    Vector<T, R> r(T(0));
    for (std::size_t i = 0; i < R; i++) {
        T s = T();
        for (std::size_t k = 0; k < C; k++) s += a(i, k) * x(k);
        r(i) = s;
    }
    return r;
}
template <class T, std::size_t R, std::size_t C>
Matrix<T, R, C> prod(const Matrix<T, R, C> &a, const Matrix<T, R, C> &b) { return a * b; }
template <class T, std::size_t R, std::size_t C> Matrix<T, C, R> trans(const Matrix<T, R, C> &a) {
    Matrix<T, C, R> r;
    for (std::size_t i = 0; i < R; i++)
        for (std::size_t j = 0; j < C; j++) r(j, i) = a(i, j);
    return r;
}
template <class T, std::size_t N> T trace(const Matrix<T, N, N> &a) {
    T s = T(); for (std::size_t i = 0; i < N; i++) s += a(i, i); return s;
}
template <class M> M identity() {
    M r(typename M::value_type(0));
    for (std::size_t i = 0; i < M::rows() && i < M::cols(); i++) r(i, i) = typename M::value_type(1);
    return r;
}
template <class T, std::size_t R, std::size_t C> std::ostream &operator<<(std::ostream &o, const Matrix<T, R, C> &a) {
    for (std::size_t i = 0; i < R; i++) {
        for (std::size_t j = 0; j < C; j++) o << a(i, j) << " ";
        o << "\n";
    }
    return o;
}

}  // namespace tvmet
#endif
