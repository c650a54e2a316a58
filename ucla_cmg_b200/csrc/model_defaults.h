// model_defaults.h -- reference parameter sets and initial states (host).
#pragma once
#include <vector>

namespace ep {

// SetUpTusscherParameters / SetUpMahajan[_fail]Parameters
// (IonicModel/SetUpIonicConstants.h:88-315); TT gets a 54th entry, the
// s-gate variant (0: the reference's kinetics).
int default_consts(int model, int type, double *out);
// Tusscher.h:51-69, Mahajan.cc:25-160 (per tissue type), LR.cc:18-26;
// node-major layout of getInternalParameters.
int default_state(int model, int type, double *out);
// the model's own surface-to-volume ratio (Tusscher.h:72, Mahajan.cc:164, LR.cc:36-37)
double model_xi(int model);
// LRGateTable::makeGateTable (LRGateTable.h:66-79): 290001 x 14
void lr_gate_table(std::vector<double> &tab);

}  // namespace ep
