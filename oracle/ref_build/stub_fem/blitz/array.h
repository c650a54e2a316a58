// Stand-in for Blitz++ arrays (oracle harness only): rank <= 4, value
// storage (the reference's element matrices are fresh objects per element,
// so value and reference semantics give the same results), resize, fill,
// element access.
#ifndef REF_FEM_STUB_BLITZ_ARRAY_H
#define REF_FEM_STUB_BLITZ_ARRAY_H
#include <vector>
#include <cstddef>
namespace blitz {
template <class T, int N> class Array {
public:
    Array() { for (int k = 0; k < 4; k++) n_[k] = 0; }
    explicit Array(int a, int b = 1, int c = 1, int d = 1) { resize(a, b, c, d); }
    void resize(int a, int b = 1, int c = 1, int d = 1) {
        n_[0] = a; n_[1] = N > 1 ? b : 1; n_[2] = N > 2 ? c : 1; n_[3] = N > 3 ? d : 1;
        v_.assign((size_t)n_[0] * n_[1] * n_[2] * n_[3], T());
    }
    Array &operator=(T x) { for (size_t i = 0; i < v_.size(); i++) v_[i] = x; return *this; }
    T &operator()(int i) { return v_[i]; }
    const T &operator()(int i) const { return v_[i]; }
    T &operator()(int i, int j) { return v_[(size_t)i * n_[1] + j]; }
    const T &operator()(int i, int j) const { return v_[(size_t)i * n_[1] + j]; }
    T &operator()(int i, int j, int k) { return v_[((size_t)i * n_[1] + j) * n_[2] + k]; }
    const T &operator()(int i, int j, int k) const { return v_[((size_t)i * n_[1] + j) * n_[2] + k]; }
    T &operator()(int i, int j, int k, int l) { return v_[(((size_t)i * n_[1] + j) * n_[2] + k) * n_[3] + l]; }
    const T &operator()(int i, int j, int k, int l) const { return v_[(((size_t)i * n_[1] + j) * n_[2] + k) * n_[3] + l]; }
    int size() const { return (int)v_.size(); }
    int extent(int k) const { return n_[k]; }
    int rows() const { return n_[0]; }
    int cols() const { return n_[1]; }
    T *data() { return v_.data(); }
private:
    std::vector<T> v_;
    int n_[4];
};
}  // namespace blitz
#endif
