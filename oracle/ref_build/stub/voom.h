// Minimal stand-in for voomEP's src/voom.h, used ONLY to compile the
// reference's cell-model sources (voomEP/src/IonicModel/*.cc) unmodified
// for the test oracle.  The real header pulls in MPI, Blitz++ and tvmet,
// none of which the ionic models use; they only need the Real typedef.
#ifndef _VOOM_H_
#define _VOOM_H_
#include <vector>
#include <iostream>
#include <cmath>
namespace voom { typedef double Real; }
#endif
