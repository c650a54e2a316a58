// Stand-in for Epetra's CRS matrices (oracle harness only).
// InsertGlobalValues records every (row, col, value) triplet in call order;
// Epetra sums repeated entries when it assembles, which is what the
// reference's element loops rely on, and the harness sums them the same way.
#ifndef REF_FEM_STUB_EPETRA_CRSMATRIX_H
#define REF_FEM_STUB_EPETRA_CRSMATRIX_H
#include <vector>
#include "Epetra_Vector.h"
class Epetra_RowMatrix {};
class Epetra_CrsMatrix : public Epetra_RowMatrix {
public:
    Epetra_CrsMatrix() {}
    virtual ~Epetra_CrsMatrix() {}
    int InsertGlobalValues(int nr, const int *rows, int nc, const int *cols, const double *vals) {
        for (int i = 0; i < nr; i++)
            for (int j = 0; j < nc; j++) {
                row.push_back(rows[i]);
                col.push_back(cols[j]);
                val.push_back(vals[i * nc + j]);
            }
        return 0;
    }
    int SumIntoGlobalValues(int nr, const int *rows, int nc, const int *cols, const double *vals) {
        return InsertGlobalValues(nr, rows, nc, cols, vals);
    }
    int GlobalAssemble() { return 0; }
    int FillComplete() { return 0; }
    std::vector<int> row, col;
    std::vector<double> val;
};
#endif
