// Stand-in for Epetra_FECrsMatrix (oracle harness only): see Epetra_CrsMatrix.h.
#ifndef REF_FEM_STUB_EPETRA_FECRSMATRIX_H
#define REF_FEM_STUB_EPETRA_FECRSMATRIX_H
#include "Epetra_CrsMatrix.h"
class Epetra_FECrsMatrix : public Epetra_CrsMatrix {};
#endif
