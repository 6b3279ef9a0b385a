// bp_guess.h -- the learned initial guess (bp_guess.cu): a U-Net whose
// estimate of the velocity replaces the given start of the Picard loop.
#pragma once

#include <string>
#include <vector>

#include "bp_plan.h"

namespace bp {

struct GuessNet;

// Input normalisation of the network (per feature); nin is 5 or 6 (the
// sixth feature: log10 of the mean flow-law factor around the vertex).
struct GuessNorm {
  float shift[6], scale[6];
  int nin;
};

// Loads the weights file that net.UNet.save_bin writes and uploads them to
// the current device; nullptr with *err on a missing or malformed file.
GuessNet* guess_net_load(const char* path, std::string* err);
void guess_net_free(GuessNet* N);

// The network's guess of the instances `which` of a 3-D problem, written
// into x0 (node order) on stream s; *launches counts the kernels.
int guess_net_run(GuessNet* N, const HostPlan& p, const DevView& v, const std::vector<int>& which, double2* x0,
                  cudaStream_t s, int* launches);

}  // namespace bp
