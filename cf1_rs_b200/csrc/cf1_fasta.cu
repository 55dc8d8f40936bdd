// FASTA / FASTQ input (plain or gzip) for cf1gpu_add_fasta.  The reference
// reads records with needletail (src/classify.rs:541-546): sequence lines of
// a record are concatenated without their line ends, and the record id is
// the header line.
#include <zlib.h>

#include <string>
#include <vector>

#include "cf1_context.cuh"
#include "cf1_pipeline.cuh"

namespace cf1 {

void add_fasta(cf1gpu_ctx *c, const char *path) {
  gzFile f = gzopen(path, "rb");
  if (!f) throw Error(CF1GPU_ERR_IO, std::string("cannot open ") + path);
  gzbuffer(f, 1 << 20);
  std::string data;
  std::vector<char> buf(1 << 22);
  for (;;) {
    int n = gzread(f, buf.data(), (unsigned)buf.size());
    if (n < 0) {
      gzclose(f);
      throw Error(CF1GPU_ERR_IO, std::string("read error in ") + path);
    }
    if (n == 0) break;
    data.append(buf.data(), (size_t)n);
  }
  gzclose(f);
  size_t i = 0, n = data.size();
  auto line_end = [&](size_t p) {
    size_t e = data.find('\n', p);
    return e == std::string::npos ? n : e;
  };
  std::string seq;
  while (i < n) {
    if (data[i] == '\n' || data[i] == '\r') {
      i++;
      continue;
    }
    char tag = data[i];
    if (tag != '>' && tag != '@') throw Error(CF1GPU_ERR_IO, std::string("not FASTA/FASTQ: ") + path);
    size_t he = line_end(i);
    std::string name = data.substr(i + 1, he - i - 1);
    if (!name.empty() && name.back() == '\r') name.pop_back();
    i = he + 1;
    seq.clear();
    if (tag == '>') {
      while (i < n && data[i] != '>') {
        size_t e = line_end(i);
        size_t le = e;
        if (le > i && data[le - 1] == '\r') le--;
        seq.append(data, i, le - i);
        i = e + 1;
      }
    } else {
      while (i < n && data[i] != '+') {
        size_t e = line_end(i);
        size_t le = e;
        if (le > i && data[le - 1] == '\r') le--;
        seq.append(data, i, le - i);
        i = e + 1;
      }
      if (i < n) i = line_end(i) + 1;  // '+' line
      size_t q = 0;
      while (i < n && q < seq.size()) {
        size_t e = line_end(i);
        size_t le = e;
        if (le > i && data[le - 1] == '\r') le--;
        q += le - i;
        i = e + 1;
      }
    }
    add_record(c, name.data(), name.size(), reinterpret_cast<const uint8_t *>(seq.data()), seq.size());
  }
}

}  // namespace cf1
