// Run-time autotuner (autotune.cu).
#pragma once
#include <functional>
#include <string>
#include <vector>
#include "common.cuh"

namespace qsgw {

// The launch parameter for problem `key`: the cached choice; else, when tuning
// is on and no graph is being recorded, the fastest of `cands`, each run once
// through run(c) (which must redo the whole effect of the launch, e.g. clear an
// accumulated output first); else `heuristic`.  *tried tells whether trials ran
// (the output then holds a trial's result and must be cleared before the real run).
int tuned_choice(const std::string& key, const std::vector<int>& cands, int heuristic,
                 const std::function<int(int)>& run, cudaStream_t s, int* chosen, bool* tried);

// While one of these lives, tuned_choice runs no trials (for calls that add into
// an output the caller already holds, which a trial would clear).
struct TuneSuspend {
  TuneSuspend();
  ~TuneSuspend();
};

}  // namespace qsgw
