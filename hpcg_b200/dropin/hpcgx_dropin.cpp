// hpcgx_dropin.cpp -- helpers of the drop-in operator files.
#include "hpcgx_dropin.hpp"

#include <cstdlib>
#include <fstream>
#include <thread>

#include "hpcg.hpp"

namespace hpcgx_dropin {

namespace {
hpcgx_problem *g_current = nullptr;

// Joined by wait_device_init, or at exit if the driver never optimizes.
struct DeviceInit {
  std::thread t;
  bool started = false;
  ~DeviceInit() {
    if (t.joinable()) t.join();
  }
} g_init;
}  // namespace

int device() {
  const char *dev = std::getenv("HPCGX_DEVICE");
  return dev ? std::atoi(dev) : 0;
}

void start_device_init() {
  if (g_init.started) return;
  g_init.started = true;
  const int d = device();
  g_init.t = std::thread([d] { (void)hpcgx_init_device(d); });
}

void wait_device_init() {
  if (g_init.t.joinable()) g_init.t.join();
}

hpcgx_problem *current() { return g_current; }
void set_current(hpcgx_problem *p) { g_current = p; }

LevelState *state(const SparseMatrix &A) { return static_cast<LevelState *>(A.optimizationData); }

int sync_diagonals(const SparseMatrix &A) {
  for (const SparseMatrix *m = &A; m; m = m->Ac) {
    LevelState *s = state(*m);
    if (!s) return HPCGX_ESTATE;
    const local_int_t n = m->localNumberOfRows;
    bool changed = false;
    for (local_int_t i = 0; i < n && !changed; ++i) changed = *m->matrixDiagonal[i] != s->diagonal[i];
    if (!changed) continue;
    for (local_int_t i = 0; i < n; ++i) s->diagonal[i] = *m->matrixDiagonal[i];
    int rc = hpcgx_set_diagonal_host(s->problem, s->level, s->diagonal.data());
    if (rc != HPCGX_OK) return report(rc, "ReplaceMatrixDiagonal coherence");
  }
  return HPCGX_OK;
}

int report(int rc, const char *where) {
  if (rc != HPCGX_OK) HPCG_fout << where << ": hpcgx error " << rc << ": " << hpcgx_last_error() << std::endl;
  return rc;
}

}  // namespace hpcgx_dropin
