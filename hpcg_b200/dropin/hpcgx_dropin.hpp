// hpcgx_dropin.hpp -- state shared by the drop-in operator files.
//
// The drop-in replaces HPCG 3.1's replaceable files (CG.cpp, ComputeSPMV.cpp,
// ComputeSYMGS.cpp, ComputeMG.cpp, ComputeDotProduct.cpp, ComputeWAXPBY.cpp,
// OptimizeProblem.cpp) and is compiled against the reference's own headers,
// the way a vendor implementation is built.  OptimizeProblem uploads every
// level to libhpcgx and hangs a LevelState off each SparseMatrix's
// optimizationData (src/SparseMatrix.hpp:64); the operators then run on the
// GPU through the C ABI of include/hpcgx.h.
#ifndef HPCGX_DROPIN_HPP
#define HPCGX_DROPIN_HPP

#include <vector>

#include "SparseMatrix.hpp"
#include "hpcgx.h"

namespace hpcgx_dropin {

struct LevelState {
  hpcgx_problem *problem = nullptr;
  int level = 0;
  // diagonal values last written to the device; the host matrix may change
  // them through ReplaceMatrixDiagonal (src/TestCG.cpp:79,114)
  std::vector<double> diagonal;
};

// The problem built by the last OptimizeProblem call; the dot product and
// WAXPBY have no matrix argument and stage their vectors through it.
hpcgx_problem *current();
void set_current(hpcgx_problem *p);

// The drop-in state of a level, or nullptr if OptimizeProblem did not run.
LevelState *state(const SparseMatrix &A);

// Writes to the device the diagonal of every level from A down that the host
// copy changed since the last upload.
int sync_diagonals(const SparseMatrix &A);

// Returns rc; on failure also logs the library's message to HPCG_fout.
int report(int rc, const char *where);

// The GPU the drop-in runs on: HPCGX_DEVICE, else 0.
int device();

// Creating the CUDA context is the process's first CUDA call and takes about
// a second.  GenerateProblem starts it on a thread of its own
// (hpcgx_init_device), where it overlaps the host's problem generation, and
// OptimizeProblem waits for that thread before its first library call.  The
// thread's status is not reported: if the context cannot be made,
// OptimizeProblem's own hpcgx_create fails and says why.
void start_device_init();
void wait_device_init();

}  // namespace hpcgx_dropin

#endif
