/* Stand-in for mpi.h: the compiled reference sources include it but call
   no MPI function on the paths the oracle harness uses. */
#ifndef REF_FEM_STUB_MPI_H
#define REF_FEM_STUB_MPI_H
#endif
