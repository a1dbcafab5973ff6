// Internal interface between the solver (dmf_solver.cu) and the learned
// schedule picker (dmf_sched.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "dmf.h"

namespace dmfs {

constexpr int kFeatures = DMF_SCHED_FEATURES;  // 12
constexpr int kHidden = DMF_SCHED_HIDDEN;      // 64
constexpr int kActions = DMF_SCHED_ACTIONS;    // 4
// parameter layout: W1[64][12], W2[64][64], W3[4][64] (bf16, row = output unit),
// then b1[64], b2[64], b3[4] (fp32)
constexpr int kW1 = 0, kW2 = kW1 + kHidden * kFeatures, kW3 = kW2 + kHidden * kHidden;
constexpr int kNumW = kW3 + kActions * kHidden;  // 5120
constexpr int kB1 = 0, kB2 = kB1 + kHidden, kB3 = kB2 + kHidden;
constexpr int kNumB = kB3 + kActions;  // 132
static_assert(kNumW == DMF_SCHED_WEIGHTS && kNumB == DMF_SCHED_BIASES, "layout");

// Raw sums over one update batch, measured against the residual state the
// batch will be applied to (filled by the solver's feature kernel).
struct FeatAcc {
  unsigned long long valid;     // updates naming an existing arc (u != v)
  unsigned long long dec;       // capacity decreases
  unsigned long long satdec;    // decreases below the arc's current flow (create excess and deficit)
  unsigned long long incsat;    // increases on arcs with no residual left
  unsigned long long ins;       // capacity 0 -> positive
  unsigned long long del;       // positive -> 0
  unsigned long long sum_deg;   // out-degree of the updated arcs' tails
  unsigned long long max_deg;
  long long excess_created;     // sum of (flow - new capacity) over saturating decreases
  long long pad;
};

// Scalars of the solver the features are normalised by.
struct FeatScalars {
  float k, m, n;
  float last_flow;    // flow value before the batch
  float last_levels;  // BFS levels of the last solve
  float last_outer;   // global relabels of the last solve
};

}  // namespace dmfs

// Computes the 12 features from `d_acc` on the device and, when `sched` is
// non-null and trained, runs the MLP and picks the action with the lowest
// predicted time; otherwise the action is 0 (the plain schedule).  Waits for
// the stream and returns the features, the four predictions (zeros without a
// model) and the action on the host.
int dmf_sched_decide(dmf_sched *sched, const dmfs::FeatAcc *d_acc, const dmfs::FeatScalars &sc, cudaStream_t stream,
                     int device, float *h_feat, float *h_pred, int *h_action);
