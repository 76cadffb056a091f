// Device-resident state of a CG / BiCGSTAB solve (krylov.cu, cg_fused.cu)
// and the reference's termination test on it.
#pragma once

#include <cmath>

namespace mtlgpu {

struct SolverState {
  int done;       // nonzero: every kernel returns immediately
  int skip2;      // BiCGSTAB: second half of the iteration skipped
  int half_exit;  // BiCGSTAB: finished on ||s||
  int error;      // basic_iteration error code (0, 1)
  int status;     // mtlgpu_status (BREAKDOWN, ...)
  int iter;       // basic_iteration::i
  int max_iter;
  int hist_len;
  int hist_cap;
  int trips;      // device-side graph loop: body runs so far
  int max_trips;  //   and the bound past which the loop stops
  double tol;     // rtol * norm_r0
  double atol;
  double norm_r0;
  double resid;
  double rho, rho_1, rr, alpha_1, gamma, omega, ts, tt, ss;
  double* history;
};

// basic_iteration::finished(r) (basic_iteration.hpp:60-65 with converged()
// 85-93 and check_max() 43-48).  Called by one thread.
__device__ inline bool iter_finished(SolverState* st, double r) {
  if (st->history && st->hist_len < st->hist_cap) st->history[st->hist_len] = r;
  st->hist_len++;
  st->resid = r;
  bool conv = st->norm_r0 == 0.0 ? (r <= st->atol) : (r <= st->tol || r <= st->atol);
  if (conv) return true;
  if (st->iter >= st->max_iter) {
    st->error = 1;
    return true;
  }
  return false;
}

}  // namespace mtlgpu
