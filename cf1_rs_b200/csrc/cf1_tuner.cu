// Autotuner cache file (see cf1_tuner.cuh).  Line format:
//   cf1tune 1 wide=<0|1> sorted=<0|1> batched=<0|1> size=<log2 bases> sk_tile=<t> msd_delta=<d> p1_ms=<f> p3_ms=<f>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <vector>

#include "cf1_tuner.cuh"

namespace cf1 {

namespace {

bool parse(const std::string &line, TuneKey &k, TuneValue &v) {
  std::istringstream in(line);
  std::string tag;
  int ver = 0;
  if (!(in >> tag >> ver) || tag != "cf1tune" || ver != 1) return false;
  int got = 0;
  std::string f;
  while (in >> f) {
    size_t eq = f.find('=');
    if (eq == std::string::npos) return false;
    std::string name = f.substr(0, eq), val = f.substr(eq + 1);
    try {
      if (name == "wide") k.wide = std::stoi(val), got |= 1;
      else if (name == "sorted") k.sorted = std::stoi(val), got |= 2;
      else if (name == "batched") k.batched = std::stoi(val), got |= 4;
      else if (name == "size") k.size_class = std::stoi(val), got |= 8;
      else if (name == "sk_tile") v.sk_tile = (uint32_t)std::stoul(val), got |= 16;
      else if (name == "msd_delta") v.msd_delta = std::stoi(val), got |= 32;
      else if (name == "p1_ms") v.p1_ms = std::stod(val);
      else if (name == "p3_ms") v.p3_ms = std::stod(val);
    } catch (...) {
      return false;
    }
  }
  if (got != 63) return false;
  bool tile_ok = false;
  for (uint32_t t : TUNE_TILES) tile_ok |= v.sk_tile == t;
  bool delta_ok = false;
  for (int d : TUNE_MSD_DELTAS) delta_ok |= v.msd_delta == d;
  return tile_ok && delta_ok;
}

std::string format(const TuneKey &k, const TuneValue &v) {
  char buf[256];
  std::snprintf(buf, sizeof(buf),
                "cf1tune 1 wide=%d sorted=%d batched=%d size=%d sk_tile=%u msd_delta=%d p1_ms=%.3f p3_ms=%.3f", k.wide,
                k.sorted, k.batched, k.size_class, v.sk_tile, v.msd_delta, v.p1_ms, v.p3_ms);
  return buf;
}

}  // namespace

bool tuner_lookup(const std::string &path, const TuneKey &key, TuneValue &out) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  bool found = false;
  while (std::getline(in, line)) {  // the last entry of a key wins
    TuneKey k;
    TuneValue v;
    if (parse(line, k, v) && k == key) {
      out = v;
      found = true;
    }
  }
  return found;
}

void tuner_store(const std::string &path, const TuneKey &key, const TuneValue &val) {
  std::vector<std::string> keep;
  {
    std::ifstream in(path);
    std::string line;
    while (in && std::getline(in, line)) {
      TuneKey k;
      TuneValue v;
      if (parse(line, k, v) && k != key) keep.push_back(line);
    }
  }
  keep.push_back(format(key, val));
  const std::string tmp = path + ".tmp";
  {
    std::ofstream out(tmp, std::ios::trunc);
    if (!out) return;  // an unwritable cache only costs a re-measurement
    for (const auto &l : keep) out << l << '\n';
    if (!out) return;
  }
  std::rename(tmp.c_str(), path.c_str());
}

}  // namespace cf1
