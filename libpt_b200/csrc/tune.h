// Autotuner cache (tune.cpp): kernel-variant choices per problem key.
#pragma once

#include <string>
#include <vector>

namespace ptb {

std::string tune_key(int kind, int oa, int va, int ob, int vb, int precision,
                     int slices, int dtype);
// False when LIBPT_AUTOTUNE=0: plans keep their heuristic choices.
bool tune_enabled();
// LIBPT_TUNE_VERBOSE=1: print each measured candidate to stderr.
bool tune_verbose();
bool tune_lookup(const std::string &key, std::vector<int> *choice);
void tune_store(const std::string &key, const std::vector<int> &choice);
void tune_clear();

}  // namespace ptb
