// Stand-in for Epetra_Export (oracle harness only): never constructed.
#ifndef REF_FEM_STUB_EPETRA_EXPORT_H
#define REF_FEM_STUB_EPETRA_EXPORT_H
class Epetra_Export {};
#endif
