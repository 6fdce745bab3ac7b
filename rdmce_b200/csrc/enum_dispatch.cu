// enum_dispatch.cu -- picks the build of the enumeration kernel for a solve.
//
// enum.cu is compiled three times, for 3, 4 and 5 resident 8-warp blocks per
// SM (at most 85, 64 and 51 registers a thread; 24, 32 and 40 warps per SM).
// More registers mean fewer spills in the general and 64-bit tiers and in the
// root build; more warps hide more of the 32-bit tier's latency.  Which wins
// depends on the graph (measured on a B200: a full R-MAT 14 enumeration runs
// fastest with 24 warps per SM, the R-MAT 20 root sample with 32 or 40), so
// the choice is the autotuner's (api.cu) unless the caller fixes
// blocks_per_sm.
#include <algorithm>

#include "common.cuh"
#include "engine.h"

namespace mce {

int enum_build_for(uint32_t blocks_per_sm) {
  if (blocks_per_sm == 0) return 4;
  if (blocks_per_sm <= 3) return 3;
  return blocks_per_sm >= 5 ? 5 : 4;
}

uint32_t tune_pick(const TuneRecord &t, bool counting, uint32_t *mode) {
  static const uint32_t order[3] = {4, 5, 3};  // the default, then more warps, then more registers
  int best = -1;
  for (int i = 0; i < 3; i++) {
    const int b = (int)order[i] - 3;
    if (t.ms[b] < 0) {
      if (counting) break;
      *mode = 1;
      return order[i];
    }
    if (best < 0 || t.ms[b] < t.ms[best]) best = b;
  }
  *mode = 2;
  return best < 0 ? 4u : (uint32_t)best + 3;
}

void tune_record(TuneRecord &t, uint32_t blocks_per_sm, float ms) {
  if (blocks_per_sm >= 3 && blocks_per_sm <= 5 && ms > 0) t.ms[blocks_per_sm - 3] = ms;
}

mce_status enum_plan(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, SlotResult *slots,
                     unsigned long long *hist, EnumPlan *plan) {
  const int b = enum_build_for(cfg.blocks_per_sm);
  mce_status s = b == 3   ? enum_plan_b3(g, cfg, scr, slots, hist, plan)
                 : b == 5 ? enum_plan_b5(g, cfg, scr, slots, hist, plan)
                          : enum_plan_b4(g, cfg, scr, slots, hist, plan);
  plan->build = b;
  return s;
}

mce_status enum_launch(const EnumPlan &plan, cudaStream_t st) {
  return plan.build == 3 ? enum_launch_b3(plan, st) : plan.build == 5 ? enum_launch_b5(plan, st)
                                                                      : enum_launch_b4(plan, st);
}

mce_status enum_finish(const EnumPlan &plan, cudaStream_t st, EnumStats *stats) {
  return plan.build == 3 ? enum_finish_b3(plan, st, stats)
                         : plan.build == 5 ? enum_finish_b5(plan, st, stats) : enum_finish_b4(plan, st, stats);
}

mce_status enumerate(const DeviceGraph &g, const EnumConfig &cfg, Scratch *scr, cudaStream_t st, SlotResult *slots,
                     unsigned long long *hist, EnumStats *stats) {
  EnumPlan plan;
  MCE_TRY(enum_plan(g, cfg, scr, slots, hist, &plan));
  cudaEvent_t e0, e1;
  MCE_CUDA_TRY(cudaEventCreate(&e0));
  MCE_CUDA_TRY(cudaEventCreate(&e1));
  // device time of the launch alone: e1 is recorded right behind the kernel,
  // before the host reads the control block back (a host that is slow to
  // wake from that wait adds nothing); a deferred-root pass adds its own
  cudaEventRecord(e0, st);
  mce_status s = enum_launch(plan, st);
  cudaEventRecord(e1, st);
  EnumStats local;
  if (s == MCE_OK) s = enum_finish(plan, st, stats ? stats : &local);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (stats) {
    stats->ms_enum = ms + stats->ms_heavy;
    stats->blocks_per_sm = plan.blocks / std::max<uint32_t>(1, plan.sms);
  }
  return s;
}

}  // namespace mce
