// Autotuner of the pipeline's launch parameters, cached on disk.
//
// Key: (k class: k <= 32 or not, sorted bins or not, batched or not, input
// size class = floor(log2(bases))).  Value: the minimizer tile (k-mer
// positions per phase-1 work chunk) and the offset applied to the phase-3
// MSD split width (sub-bucket size), each the fastest of its candidates when
// the key was first seen.  The cache is a text file of one line per key, so a
// later context -- or process -- with the same key reuses the choice without
// measuring again.
#pragma once
#include <cstdint>
#include <string>

namespace cf1 {

struct TuneKey {
  int wide = 0, sorted = 0, batched = 0, size_class = 0;
  bool operator==(const TuneKey &o) const {
    return wide == o.wide && sorted == o.sorted && batched == o.batched && size_class == o.size_class;
  }
  bool operator!=(const TuneKey &o) const { return !(*this == o); }
};

struct TuneValue {
  uint32_t sk_tile = 2048;
  int msd_delta = 0;
  double p1_ms = 0, p3_ms = 0;  // the winners' times when measured
};

constexpr uint32_t TUNE_TILES[3] = {1024, 2048, 4096};
// widest first: its scratch arrays are the largest, so the later (narrower)
// tries reuse them and no try pays for an allocation another one skipped
constexpr int TUNE_MSD_DELTAS[4] = {2, 1, 0, -1};

// Entry for `key` in the cache file at `path`; false when absent or unreadable.
bool tuner_lookup(const std::string &path, const TuneKey &key, TuneValue &out);
// Writes (or replaces) the entry for `key`; the file is rewritten through a
// temporary and renamed, so a reader never sees half a file.
void tuner_store(const std::string &path, const TuneKey &key, const TuneValue &val);

}  // namespace cf1
