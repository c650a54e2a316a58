// Stand-in for Epetra_Import (oracle harness only): never constructed.
#ifndef REF_FEM_STUB_EPETRA_IMPORT_H
#define REF_FEM_STUB_EPETRA_IMPORT_H
class Epetra_Import {};
#endif
