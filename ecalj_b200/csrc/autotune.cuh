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

// Slice count of an int8 Ozaki contraction for problem `key`: the cached choice; else, unless
// trials are suspended or a graph is being recorded, the first of `cands` (ascending) whose
// error estimate err(ns, &e) is at most `tol` (the caller measures e against its most
// accurate count), or the last candidate's successor `top` when none is; else `fallback`.
// The estimates are kept for qsgw_autotune_report.
int tuned_slices(const std::string& key, const std::vector<int>& cands, int top, double tol,
                 const std::function<int(int, double*)>& err, int fallback, int* chosen);

// The cached choice for `key` into *v, if there is one (no trials).
bool tuned_lookup(const std::string& key, int* v);

// While one of these lives, tuned_choice runs no trials (for calls that add into
// an output the caller already holds, which a trial would clear).
struct TuneSuspend {
  TuneSuspend();
  ~TuneSuspend();
};

}  // namespace qsgw
