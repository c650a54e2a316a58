// Stand-in for Epetra_Map (oracle harness only): never constructed.
#ifndef REF_FEM_STUB_EPETRA_MAP_H
#define REF_FEM_STUB_EPETRA_MAP_H
#include "Epetra_SerialComm.h"
class Epetra_BlockMap {};
class Epetra_Map : public Epetra_BlockMap {};
#endif
