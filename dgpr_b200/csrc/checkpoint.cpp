// Binomial checkpoint plan (checkpoint.hpp) and its C export for checks.
#include "checkpoint.hpp"

#include "../../include/dgb200.h"

namespace dgb {

namespace {

constexpr long long kSat = 1LL << 62;

struct PlanBuilder {
  CheckpointPlan& P;
  long long work = 0;        // step index of the state in the work buffer
  std::vector<int> free_bufs;
  int in_use = 1;

  void restore(int buf, long long idx)
  {
    if (work == idx) return;
    P.ops.push_back({CK_RESTORE, buf});
    work = idx;
  }
  void forward(long long k)
  {
    if (k <= 0) return;
    P.ops.push_back({CK_FORWARD, k});
    work += k;
    P.forward_steps += k;
  }
  void reverse(long long i) { P.ops.push_back({CK_REVERSE, i}); }

  // largest split with m + C(t-m, f-1) + C(m, f) == C(t, f)
  static long long split(long long t, long long f)
  {
    if (f + 1 >= t) return 1;  // room for every state: store each one on the way
    const long long best = checkpoint_cost(t, f);
    for (long long m = t - 1; m >= 1; --m)
      if (m + checkpoint_cost(t - m, f - 1) + checkpoint_cost(m, f) == best) return m;
    return 1;
  }

  // reverse steps i+t-1 .. i; U_i sits in buffer buf_i, f buffers are free
  void segment(long long i, int buf_i, long long t, long long f)
  {
    while (t > 1) {
      if (f == 0) {
        for (long long k = t - 1; k >= 1; --k) {
          restore(buf_i, i);
          forward(k);
          reverse(i + k);
        }
        t = 1;
        break;
      }
      const long long m = split(t, f);
      restore(buf_i, i);
      forward(m);
      const int b = free_bufs.back();
      free_bufs.pop_back();
      P.ops.push_back({CK_STORE, b});
      if (++in_use > P.peak_slots) P.peak_slots = in_use;
      segment(i + m, b, t - m, f - 1);
      free_bufs.push_back(b);
      --in_use;
      t = m;
    }
    restore(buf_i, i);
    reverse(i);
  }
};

}  // namespace

long long checkpoint_cost(long long t, long long f)
{
  if (t <= 1) return 0;
  if (f <= 0) return t * (t - 1) / 2;
  const long long s = f + 1;
  if (s >= t) return t - 1;
  // b = binom(s + r, s), grown until it reaches t
  __int128 b = 1;
  long long r = 0;
  while (b < t) {
    ++r;
    b = b * (s + r) / r;
  }
  const __int128 b1 = b * r / (s + 1);  // binom(s + r, s + 1)
  const __int128 c = (__int128)r * t - b1;
  return c > kSat ? kSat : (long long)c;
}

int make_checkpoint_plan(long long nsteps, int slots, CheckpointPlan& plan)
{
  plan = CheckpointPlan();
  if (nsteps < 1 || slots < 1) return 1;
  if (slots > nsteps) slots = (int)nsteps;
  plan.nsteps = nsteps;
  plan.slots = slots;
  plan.peak_slots = 1;
  PlanBuilder B{plan};
  for (int b = slots - 1; b >= 1; --b) B.free_bufs.push_back(b);
  plan.ops.push_back({CK_STORE, 0});
  B.segment(0, 0, nsteps, slots - 1);
  plan.first_reverse = 0;
  while (plan.ops[plan.first_reverse].kind != CK_REVERSE) ++plan.first_reverse;
  for (size_t k = 0; k < plan.first_reverse; ++k)
    if (plan.ops[k].kind == CK_FORWARD) plan.record_steps += plan.ops[k].arg;
  return 0;
}

}  // namespace dgb

extern "C" int dgb_checkpoint_plan(long long nsteps, int slots, long long* ops_out, long long cap,
                                   long long* nops, long long* forward_steps, int* peak_slots)
{
  dgb::CheckpointPlan plan;
  if (dgb::make_checkpoint_plan(nsteps, slots, plan)) return DGB_ERR_ARG;
  const long long n = (long long)plan.ops.size();
  if (nops) *nops = n;
  if (forward_steps) *forward_steps = plan.forward_steps;
  if (peak_slots) *peak_slots = plan.peak_slots;
  if (ops_out) {
    if (cap < 2 * n) return DGB_ERR_ARG;
    for (long long k = 0; k < n; ++k) {
      ops_out[2 * k] = plan.ops[k].kind;
      ops_out[2 * k + 1] = plan.ops[k].arg;
    }
  }
  return DGB_OK;
}
