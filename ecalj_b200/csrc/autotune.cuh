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
// accumulated output first); else `heuristic`.
int tuned_choice(const std::string& key, const std::vector<int>& cands, int heuristic,
                 const std::function<int(int)>& run, cudaStream_t s, int* chosen);

}  // namespace qsgw
