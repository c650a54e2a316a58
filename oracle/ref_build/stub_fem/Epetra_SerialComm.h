// Stand-in for Epetra's communicators: one rank (oracle harness only).
#ifndef REF_FEM_STUB_EPETRA_COMM_H
#define REF_FEM_STUB_EPETRA_COMM_H
class Epetra_Comm {
public:
    virtual ~Epetra_Comm() {}
    int MyPID() const { return 0; }
    int NumProc() const { return 1; }
    void Barrier() const {}
};
class Epetra_SerialComm : public Epetra_Comm {};
class Epetra_MpiComm : public Epetra_Comm {};
#endif
