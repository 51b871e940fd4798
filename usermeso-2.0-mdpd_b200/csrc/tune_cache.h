// Persisted autotuner picks (tune_cache.cpp): a JSON file of workload key -> pair-pass shapes.
#pragma once

#include <string>
#include <vector>

namespace mdpd {

struct TunePick {
    int density = 0;         // pair-once: gathers in flight; full list: threads per particle
    int force = 0;           // pair-once: 32; full list: threads per particle
    double ms_per_step = 0;  // the winning candidate's timed step
};

// the pick stored for key; false when the file or the key is absent.  Throws
// std::runtime_error("PARSE: ...") on a malformed file or entry.
bool tune_cache_get(const std::string &path, const std::string &key, TunePick &out);

// store (or replace) key's pick, keeping every other member of the file; written to a
// temporary beside it and renamed over it.  Throws on a malformed existing file (it is never
// overwritten) or a write failure.
void tune_cache_put(const std::string &path, const std::string &key, const TunePick &pick);

}  // namespace mdpd
