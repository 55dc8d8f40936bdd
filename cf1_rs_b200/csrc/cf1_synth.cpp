// Seeded synthetic inputs standing in for the reference's GENCODE / GRCh38
// benchmark sets (not available here).  Five workloads:
//   1  one record of 5 Mbp, i.i.d. uniform ACGT (seed 1)
//   2  transcriptome: 20k genes of 5-15 exons (lognormal length, median
//      150 bp, clipped to 50-2000; GC 45%), 100k transcripts made of ordered
//      random exon subsets, 1-8 isoforms per gene (seed 2)
//   3  genome: 200 Mbp in 24 chromosomes of 3-20 Mbp, GC 41%, 10% of the
//      sequence from 500 repeat families (consensus 0.3-6 kb, copies at 2-15%
//      substitution divergence, random strand), 1 kb poly-N every 5 Mb (seed 3)
//   4  the workload-3 generator at 1 Gbp, 30 chromosomes of 10-60 Mbp (seed 4)
//   5  3.1 Gbp in 25 chromosomes of 50-250 Mbp, GC 41%, ~50% repeats (1000
//      families of 0.3-6 kb at 2-20% divergence, plus tandem arrays of
//      5-200 bp units), 1 kb poly-N every 10 Mb (seed 5)
// `scale` multiplies every length and count (1.0 = the full workload).  The
// output is deterministic for a (workload, scale, seed) whatever the thread
// count: every chromosome / gene block has its own seeded generator.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace {

inline uint64_t splitmix(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {  // xoshiro256**
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    for (auto &v : s) v = splitmix(seed);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  uint64_t range(uint64_t lo, uint64_t hi) { return lo + next() % (hi - lo + 1); }  // inclusive
  double normal() {
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

struct BaseSampler {  // P(C) = P(G) = gc/2, P(A) = P(T) = (1-gc)/2
  uint32_t ta, tc, tg;
  explicit BaseSampler(double gc) {
    double at = (1 - gc) / 2, cg = gc / 2;
    ta = (uint32_t)(at * 65536);
    tc = (uint32_t)((at + cg) * 65536);
    tg = (uint32_t)((at + 2 * cg) * 65536);
  }
  void fill(Rng &r, uint8_t *out, uint64_t n) const {
    uint64_t i = 0;
    while (i < n) {
      uint64_t x = r.next();
      for (int j = 0; j < 4 && i < n; j++, i++) {
        uint32_t u = (uint32_t)(x >> (16 * j)) & 0xFFFF;
        out[i] = u < ta ? 'A' : u < tc ? 'C' : u < tg ? 'G' : 'T';
      }
    }
  }
};

inline uint8_t comp(uint8_t c) {
  switch (c) {
    case 'A': return 'T';
    case 'C': return 'G';
    case 'G': return 'C';
    case 'T': return 'A';
    default: return c;
  }
}

struct Output {
  std::vector<uint8_t> seq;
  std::vector<uint64_t> off{0};
  std::vector<std::string> names;
  void add(const uint8_t *s, uint64_t n, std::string name) {
    seq.insert(seq.end(), s, s + n);
    off.push_back(seq.size());
    names.push_back(std::move(name));
  }
};

// Copies src (possibly reverse-complemented) into dst with per-base
// substitutions at rate d.
void mutate_copy(Rng &r, const uint8_t *src, uint64_t n, uint8_t *dst, bool rc, double d, const BaseSampler &bs) {
  uint32_t thr = (uint32_t)(d * 4294967296.0);
  for (uint64_t i = 0; i < n; i++) {
    uint8_t c = rc ? comp(src[n - 1 - i]) : src[i];
    if ((uint32_t)r.next() < thr) {
      uint8_t alt;
      do { bs.fill(r, &alt, 1); } while (alt == c);
      c = alt;
    }
    dst[i] = c;
  }
}

struct GenomeSpec {
  double total;
  int n_chrom;
  double chr_lo, chr_hi;
  double gc;
  double repeat_frac;   // interspersed repeat families
  int n_families;
  double fam_lo, fam_hi;
  double div_lo, div_hi;
  double tandem_frac;   // tandem arrays (unit 5-200 bp)
  double polyn_every;   // 1 kb of N every this many bases
  uint64_t seed;
};

void gen_genome(const GenomeSpec &g, double scale, int nthreads, Output &out) {
  Rng top(g.seed);
  BaseSampler bs(g.gc);
  // chromosome lengths
  std::vector<double> lens(g.n_chrom);
  double sum = 0;
  for (auto &l : lens) { l = g.chr_lo + (g.chr_hi - g.chr_lo) * top.uniform(); sum += l; }
  std::vector<uint64_t> clen(g.n_chrom);
  for (int i = 0; i < g.n_chrom; i++) clen[i] = (uint64_t)std::max(1000.0, lens[i] / sum * g.total * scale);
  // repeat families
  std::vector<std::vector<uint8_t>> fam(g.n_families);
  std::vector<double> fdiv(g.n_families);
  for (int f = 0; f < g.n_families; f++) {
    uint64_t L = (uint64_t)(g.fam_lo + (g.fam_hi - g.fam_lo) * top.uniform());
    fam[f].resize(L);
    bs.fill(top, fam[f].data(), L);
    fdiv[f] = g.div_lo + (g.div_hi - g.div_lo) * top.uniform();
  }
  std::vector<std::vector<uint8_t>> chrom(g.n_chrom);
  std::atomic<int> next(0);
  auto work = [&] {
    for (;;) {
      int c = next.fetch_add(1);
      if (c >= g.n_chrom) break;
      uint64_t L = clen[c];
      Rng r(g.seed * 1000003ull + (uint64_t)c * 7919ull + 17);
      std::vector<uint8_t> &s = chrom[c];
      s.resize(L);
      bs.fill(r, s.data(), L);
      // interspersed repeats
      uint64_t want = (uint64_t)(g.repeat_frac * L), have = 0;
      std::vector<uint8_t> tmp;
      while (have < want && g.n_families > 0) {
        int f = (int)r.range(0, g.n_families - 1);
        uint64_t n = fam[f].size();
        if (n >= L) break;
        uint64_t pos = r.range(0, L - n);
        tmp.resize(n);
        mutate_copy(r, fam[f].data(), n, tmp.data(), r.next() & 1, fdiv[f], bs);
        std::memcpy(s.data() + pos, tmp.data(), n);
        have += n;
      }
      // tandem arrays
      want = (uint64_t)(g.tandem_frac * L);
      have = 0;
      while (have < want) {
        uint64_t unit = r.range(5, 200);
        uint64_t n = std::min<uint64_t>(L / 4, r.range(1000, 10000));
        if (n < unit) break;
        std::vector<uint8_t> u(unit);
        bs.fill(r, u.data(), unit);
        uint64_t pos = r.range(0, L - n);
        for (uint64_t i = 0; i < n; i++) s[pos + i] = u[i % unit];
        // 1% substitutions inside the array
        for (uint64_t i = 0; i < n / 100; i++) bs.fill(r, &s[pos + r.range(0, n - 1)], 1);
        have += n;
      }
      // poly-N stretches
      if (g.polyn_every > 0) {
        uint64_t every = (uint64_t)std::max(2000.0, g.polyn_every * scale);
        for (uint64_t p = every; p + 1000 <= L; p += every) std::memset(s.data() + p, 'N', 1000);
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < std::max(1, nthreads); t++) th.emplace_back(work);
  for (auto &x : th) x.join();
  uint64_t total = 0;
  for (auto &s : chrom) total += s.size();
  out.seq.reserve(total);
  for (int c = 0; c < g.n_chrom; c++) {
    out.add(chrom[c].data(), chrom[c].size(), "chr" + std::to_string(c + 1));
    std::vector<uint8_t>().swap(chrom[c]);
  }
}

void gen_transcriptome(double scale, uint64_t seed, int nthreads, Output &out) {
  const int n_genes = std::max(1, (int)std::lround(20000 * scale));
  const uint64_t target_tx = (uint64_t)std::max(1.0, std::round(100000 * scale));
  BaseSampler bs(0.45);
  Rng top(seed);
  std::vector<int> iso(n_genes);
  uint64_t tot = 0;
  for (auto &v : iso) { v = (int)top.range(1, 8); tot += v; }
  while (tot < target_tx) {  // top up to the transcript target, at most 8 per gene
    int g = (int)top.range(0, n_genes - 1);
    if (iso[g] < 8) { iso[g]++; tot++; }
  }
  std::vector<std::vector<std::pair<std::vector<uint8_t>, std::string>>> per(n_genes);
  std::atomic<int> next(0);
  auto work = [&] {
    for (;;) {
      int g = next.fetch_add(1);
      if (g >= n_genes) break;
      Rng r(seed * 1000003ull + (uint64_t)g * 104729ull + 5);
      int ne = (int)r.range(5, 15);
      std::vector<std::vector<uint8_t>> ex(ne);
      for (auto &e : ex) {
        double l = std::exp(std::log(150.0) + 0.7 * r.normal());
        uint64_t L = (uint64_t)std::min(2000.0, std::max(50.0, l));
        e.resize(L);
        bs.fill(r, e.data(), L);
      }
      for (int i = 0; i < iso[g]; i++) {
        std::vector<uint8_t> t;
        for (int e = 0; e < ne; e++)
          if (r.uniform() < 0.7) t.insert(t.end(), ex[e].begin(), ex[e].end());
        for (int e = 0; e < ne && t.size() < 200; e++) t.insert(t.end(), ex[e].begin(), ex[e].end());
        if (t.size() > 100000) t.resize(100000);
        per[g].emplace_back(std::move(t), "g" + std::to_string(g) + "_t" + std::to_string(i));
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < std::max(1, nthreads); t++) th.emplace_back(work);
  for (auto &x : th) x.join();
  for (auto &v : per)
    for (auto &p : v) out.add(p.first.data(), p.first.size(), p.second);
}

}  // namespace

extern "C" {

void *cf1synth_generate(int config, double scale, uint64_t seed, int nthreads) {
  Output *o = new Output();
  if (scale <= 0) scale = 1.0;
  switch (config) {
    case 1: {
      Rng r(seed ? seed : 1);
      BaseSampler bs(0.5);
      uint64_t L = (uint64_t)(5e6 * scale);
      std::vector<uint8_t> s(L);
      bs.fill(r, s.data(), L);
      o->add(s.data(), L, "seq1");
      break;
    }
    case 2:
      gen_transcriptome(scale, seed ? seed : 2, nthreads, *o);
      break;
    case 3:
      gen_genome({200e6, 24, 3e6, 20e6, 0.41, 0.10, 500, 300, 6000, 0.02, 0.15, 0.0, 5e6, seed ? seed : 3}, scale,
                 nthreads, *o);
      break;
    case 4:
      gen_genome({1e9, 30, 10e6, 60e6, 0.41, 0.10, 500, 300, 6000, 0.02, 0.15, 0.0, 5e6, seed ? seed : 4}, scale,
                 nthreads, *o);
      break;
    case 5:
      gen_genome({3.1e9, 25, 50e6, 250e6, 0.41, 0.40, 1000, 300, 6000, 0.02, 0.20, 0.10, 10e6, seed ? seed : 5}, scale,
                 nthreads, *o);
      break;
    default:
      delete o;
      return nullptr;
  }
  return o;
}

uint64_t cf1synth_len(void *h) { return ((Output *)h)->seq.size(); }
const uint8_t *cf1synth_seq(void *h) { return ((Output *)h)->seq.data(); }
uint64_t cf1synth_nrec(void *h) { return ((Output *)h)->names.size(); }
const uint64_t *cf1synth_offsets(void *h) { return ((Output *)h)->off.data(); }
size_t cf1synth_name(void *h, uint64_t i, char *buf, size_t cap) {
  const std::string &s = ((Output *)h)->names.at(i);
  if (buf && cap) {
    size_t n = std::min(cap - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return s.size();
}
int cf1synth_write_fasta(void *h, const char *path) {
  Output *o = (Output *)h;
  FILE *f = std::fopen(path, "wb");
  if (!f) return -1;
  for (size_t i = 0; i < o->names.size(); i++) {
    std::fprintf(f, ">%s\n", o->names[i].c_str());
    for (uint64_t p = o->off[i]; p < o->off[i + 1]; p += 80) {
      uint64_t n = std::min<uint64_t>(80, o->off[i + 1] - p);
      std::fwrite(o->seq.data() + p, 1, n, f);
      std::fputc('\n', f);
    }
  }
  return std::fclose(f) == 0 ? 0 : -1;
}
void cf1synth_free(void *h) { delete (Output *)h; }

}  // extern "C"
