// Launch-configuration autotuner.  For a workload key (the shape of the work and the
// device), each candidate configuration is run once untimed and then timed with CUDA
// events on the caller's stream; the fastest median is kept.  Candidates are equivalent
// launches of the same arithmetic (tile edges whose k order per element is the same, or
// orders of independent tiles), so the choice changes speed only.
//
// Decisions live in a per-process table.  SP2B_TUNE=0 turns measuring off (the built-in
// rules apply); SP2B_TUNE_FILE names a text file, read on first use and appended to on
// every new decision, one "key choice ms0 ms1 ..." line per decision.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <string>
#include <vector>

namespace sp2b {

bool tune_enabled();
// The cached choice for key, or false.
bool tune_lookup(const std::string& key, int* choice);
// Records a decision (and appends it to SP2B_TUNE_FILE when set).
void tune_store(const std::string& key, int choice, const std::vector<float>& ms);
// Runs run(c) for c in [0, ncand): once untimed, then `reps` times between CUDA events on
// st (run must leave its work ordered on st).  *best receives the candidate with the
// lowest median time, ms the medians.  Returns SP2B_OK or the first failing run's status.
int tune_measure(int ncand, int reps, cudaStream_t st, const std::function<int(int)>& run,
                 std::vector<float>* ms, int* best);

}  // namespace sp2b
