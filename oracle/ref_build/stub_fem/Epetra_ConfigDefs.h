// Stand-in for Trilinos' Epetra_ConfigDefs.h (oracle harness only).
#ifndef REF_FEM_STUB_EPETRA_CONFIGDEFS_H
#define REF_FEM_STUB_EPETRA_CONFIGDEFS_H
#include <iostream>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <string>
#endif
