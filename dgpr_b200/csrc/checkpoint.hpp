// Binomial checkpointing for the reverse sweep through N explicit RK steps.
//
// States U_0 .. U_N; the adjoint runs from U_N back to U_0 and reversing step
// i needs U_i.  With `slots` state buffers (one of them holds U_0) the plan
// stores intermediate states and recomputes the rest from the nearest stored
// one.  The split points minimise the number of recomputed steps: with f free
// buffers besides the one holding the segment's first state, reversing t
// steps costs
//   C(t, f) = min over 1 <= m < t of  m + C(t - m, f - 1) + C(m, f),
//   C(1, f) = 0,  C(t, 0) = t (t - 1) / 2,
// which has the closed form (binomial checkpointing, Griewank 1992)
//   C(t, f) = r t - binom(s + r, s + 1),  s = f + 1,
//   r the smallest integer with binom(s + r, s) >= t.
// The plan is a flat list of operations on one work buffer:
//   FORWARD k   advance the work state by k steps
//   STORE s     copy the work state to checkpoint buffer s
//   RESTORE s   copy checkpoint buffer s to the work state
//   REVERSE i   reverse step i (the work state holds U_i), adjoint of
//               U_{i+1} -> adjoint of U_i
// The operations before the first REVERSE are the recorded forward run (they
// end with the work state at U_{N-1}; one more step gives U_N).
#pragma once

#include <vector>

namespace dgb {

enum CkOpKind : int { CK_FORWARD = 0, CK_STORE = 1, CK_RESTORE = 2, CK_REVERSE = 3 };

struct CkOp {
  int kind;
  long long arg;  // steps (FORWARD), buffer (STORE / RESTORE), step index (REVERSE)
};

struct CheckpointPlan {
  std::vector<CkOp> ops;
  long long nsteps = 0;
  int slots = 0;
  size_t first_reverse = 0;     // index of the first REVERSE in ops
  long long forward_steps = 0;  // FORWARD steps in the whole plan
  long long record_steps = 0;   // FORWARD steps before the first REVERSE
  int peak_slots = 0;           // checkpoint buffers in use at the same time
};

// Minimal recomputed steps C(t, f) (closed form above); saturates at 2^62.
long long checkpoint_cost(long long t, long long free_slots);

// Builds the plan for nsteps >= 1 and 1 <= slots (capped at nsteps); returns
// 0, or 1 on bad arguments.
int make_checkpoint_plan(long long nsteps, int slots, CheckpointPlan& plan);

}  // namespace dgb
