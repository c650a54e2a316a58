// Stand-in for Epetra_Vector (oracle harness only): contiguous local
// values behind ExtractView, as the reference's body code reads them.
#ifndef REF_FEM_STUB_EPETRA_VECTOR_H
#define REF_FEM_STUB_EPETRA_VECTOR_H
#include <vector>
#include "Epetra_Map.h"
class Epetra_MultiVector {};
class Epetra_Vector : public Epetra_MultiVector {
public:
    explicit Epetra_Vector(int n = 0) : v_(n > 0 ? n : 1, 0.0), n_(n) {}
    int ExtractView(double **p) const { *p = const_cast<double *>(v_.data()); return 0; }
    int MyLength() const { return n_; }
    int GlobalLength() const { return n_; }
    double &operator[](int i) { return v_[i]; }
    const double &operator[](int i) const { return v_[i]; }
private:
    std::vector<double> v_;
    int n_;
};
#endif
