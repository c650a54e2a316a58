// Stand-in (oracle harness only): same one-rank communicator.
#include "Epetra_SerialComm.h"
