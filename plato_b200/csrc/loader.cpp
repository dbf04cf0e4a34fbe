// Edge-list files in, per-vertex results out (host, OpenMP, zlib).
//
// Reading mirrors the reference's load path at one partition:
//   files   a path names one file or a directory of files
//           (plato/graph/detail.hpp:82-108); here the regular files of a
//           directory are read in name order, so the edge order is
//           reproducible.
//   gzip    names ending in ".gz" are inflated (detail.hpp:202-206).
//   lines   csv_parser (plato/graph/parsers.hpp:226-290): a line is split at
//           commas with empty fields skipped (strtok); the first field is the
//           source, the second the destination, each read the way
//           strtoul(field, 10) reads (leading white space, optional sign,
//           decimal digits up to the first other character; no digits -> 0).
//           Empty lines and lines without a second field are skipped.  A
//           value above 2^32 - 1 is an error here (the reference aborts).
//           Weighted lists (double_decoder, parsers.hpp:84-88) also need a
//           third field, read as strtod reads it (the field alone, as strtok
//           cuts it); lines without one are skipped.
//   info    edges = lines parsed; vertices = largest id + 1.  The reference
//           counts distinct ids and requires them compact
//           (plato/graph/structure.hpp:199-232, dcsc.hpp:48-49), so the two
//           agree on the input it accepts; ids that do not occur become
//           isolated vertices here.
// Each file is parsed in parallel: the buffer is cut at line ends into one
// piece per thread, and the pieces are joined in order.
//
// Writing mirrors thread_local_fs_output as the reference's examples use it
// (example/pagerank.cc:191-200, plato/util/foutput.cc:95-101): files
// `<dir>/<prefix><NNNN>.csv[.gz]`, one line `v,value` per vertex, values
// printed as `ostream << double` does by default (%g, 6 significant digits);
// here file i holds a contiguous range of vertices.
#include <dirent.h>
#include <omp.h>
#include <sys/stat.h>
#include <zlib.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "plato_b200.h"
#include "host_common.hpp"
#include "edge_list.hpp"

namespace {

using plato_b200::set_error;

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }

// strtoul(field, 10) on [p, e): returns false when the value exceeds 2^32 - 1.
bool read_id(const char* p, const char* e, uint32_t* out) {
  while (p < e && is_space(*p)) ++p;
  bool neg = false;
  if (p < e && (*p == '+' || *p == '-')) {
    neg = *p == '-';
    ++p;
  }
  uint64_t v = 0;
  bool big = false;
  for (; p < e && *p >= '0' && *p <= '9'; ++p) {
    v = v * 10 + static_cast<uint64_t>(*p - '0');
    if (v > 0xFFFFFFFFull) big = true;  // strtoul saturates or wraps far above 2^32
    if (big) v = 0xFFFFFFFFull + 1;
  }
  if (neg && v != 0) big = true;  // strtoul negates: a huge unsigned value
  if (big) return false;
  *out = static_cast<uint32_t>(v);
  return true;
}

// strtod on the field [p, e) alone.
double read_weight(const char* p, const char* e) {
  char tmp[64];
  const size_t n = std::min<size_t>(static_cast<size_t>(e - p), sizeof(tmp) - 1);
  std::memcpy(tmp, p, n);
  tmp[n] = '\0';
  if (static_cast<size_t>(e - p) < sizeof(tmp)) return std::strtod(tmp, nullptr);
  return std::strtod(std::string(p, e).c_str(), nullptr);
}

// One line [b, e) without its '\n'.  1 = edge, 0 = skipped, -1 = id too large.
// w non-null: the line needs a third field (the weight).
int parse_line(const char* b, const char* e, uint32_t* s, uint32_t* d, double* w = nullptr) {
  if (b == e) return 0;
  const char* p = b;
  while (p < e && *p == ',') ++p;  // strtok: leading delimiters
  if (p == e) return 0;
  const char* f1 = p;
  while (p < e && *p != ',') ++p;
  const char* f1e = p;
  while (p < e && *p == ',') ++p;
  if (p == e) return 0;  // no destination field
  const char* f2 = p;
  while (p < e && *p != ',') ++p;
  if (!read_id(f1, f1e, s) || !read_id(f2, p, d)) return -1;
  if (w) {
    while (p < e && *p == ',') ++p;
    if (p == e) return 0;  // no weight field: the decoder fails, the line is skipped
    const char* f3 = p;
    while (p < e && *p != ',') ++p;
    *w = read_weight(f3, p);
  }
  return 1;
}

int read_whole(const std::string& name, std::string* buf) {
  const bool gz = name.size() > 3 && name.compare(name.size() - 3, 3, ".gz") == 0;
  if (gz) {
    gzFile f = gzopen(name.c_str(), "rb");
    if (!f) return set_error(PLATO_EINVAL, "cannot open " + name);
    char chunk[1 << 16];
    for (;;) {
      const int n = gzread(f, chunk, sizeof(chunk));
      if (n < 0) {
        gzclose(f);
        return set_error(PLATO_EINVAL, "gzip error in " + name);
      }
      if (n == 0) break;
      buf->append(chunk, static_cast<size_t>(n));
    }
    gzclose(f);
    return PLATO_OK;
  }
  FILE* f = std::fopen(name.c_str(), "rb");
  if (!f) return set_error(PLATO_EINVAL, "cannot open " + name + ": " + std::strerror(errno));
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz > 0) {
    buf->resize(static_cast<size_t>(sz));
    if (std::fread(&(*buf)[0], 1, buf->size(), f) != buf->size()) {
      std::fclose(f);
      return set_error(PLATO_EINVAL, "short read of " + name);
    }
  }
  std::fclose(f);
  return PLATO_OK;
}

// Parses one file's text, appending to src/dst (and w when weighted) in line order.
int parse_buffer(const std::string& buf, const std::string& name, std::vector<uint32_t>& src,
                 std::vector<uint32_t>& dst, std::vector<double>* wts = nullptr) {
  const size_t n = buf.size();
  const int T = std::max(1, std::min(omp_get_max_threads(), static_cast<int>(n / (1 << 20)) + 1));
  std::vector<size_t> cut(T + 1, n);
  cut[0] = 0;
  for (int t = 1; t < T; ++t) {  // piece t starts after the line end at or past t*n/T
    size_t p = std::max<size_t>(std::max(cut[t - 1], n / T * t), 1);
    while (p < n && buf[p - 1] != '\n') ++p;
    cut[t] = p;
  }
  std::vector<std::vector<uint32_t>> ls(T), ld(T);
  std::vector<std::vector<double>> lw(T);
  std::vector<long long> bad(T, -1);  // first offending line start per piece
#pragma omp parallel for num_threads(T) schedule(static, 1)
  for (int t = 0; t < T; ++t) {
    const char* base = buf.data();
    size_t p = cut[t];
    const size_t end = cut[t + 1];
    ls[t].reserve((end - p) / 12 + 1);
    ld[t].reserve((end - p) / 12 + 1);
    while (p < end) {
      const char* nl = static_cast<const char*>(std::memchr(base + p, '\n', end - p));
      const size_t le = nl ? static_cast<size_t>(nl - base) : end;
      uint32_t s = 0, d = 0;
      double w = 0.0;
      const int r = parse_line(base + p, base + le, &s, &d, wts ? &w : nullptr);
      if (r == 1) {
        ls[t].push_back(s);
        ld[t].push_back(d);
        if (wts) lw[t].push_back(w);
      } else if (r < 0 && bad[t] < 0) {
        bad[t] = static_cast<long long>(p);
      }
      p = le + 1;
    }
  }
  for (int t = 0; t < T; ++t) {
    if (bad[t] >= 0) {
      const long long line = 1 + std::count(buf.begin(), buf.begin() + bad[t], '\n');
      return set_error(PLATO_EINVAL, name + ":" + std::to_string(line) + ": vertex id above 2^32-1");
    }
  }
  for (int t = 0; t < T; ++t) {
    src.insert(src.end(), ls[t].begin(), ls[t].end());
    dst.insert(dst.end(), ld[t].begin(), ld[t].end());
    if (wts) wts->insert(wts->end(), lw[t].begin(), lw[t].end());
  }
  return PLATO_OK;
}

int list_files(const std::string& path, std::vector<std::string>* files) {
  struct stat st {};
  if (stat(path.c_str(), &st) != 0) return set_error(PLATO_EINVAL, "no such file or directory: " + path);
  if (!S_ISDIR(st.st_mode)) {
    files->push_back(path);
    return PLATO_OK;
  }
  DIR* d = opendir(path.c_str());
  if (!d) return set_error(PLATO_EINVAL, "cannot list " + path);
  while (dirent* e = readdir(d)) {
    const std::string full = path + "/" + e->d_name;
    struct stat fs {};
    if (stat(full.c_str(), &fs) == 0 && S_ISREG(fs.st_mode)) files->push_back(full);
  }
  closedir(d);
  std::sort(files->begin(), files->end());
  return PLATO_OK;
}

}  // namespace

namespace {

int read_csv(const char* path, bool weighted, plato_edge_list** out) {
  if (!path || !out) return set_error(PLATO_EINVAL, "plato_edge_list_read_csv: null argument");
  *out = nullptr;
  try {
    std::vector<std::string> files;
    const int lrc = list_files(path, &files);
    if (lrc != PLATO_OK) return lrc;
    auto* el = new plato_edge_list();
    el->weighted = weighted;
    for (const std::string& f : files) {
      std::string buf;
      int rc = read_whole(f, &buf);
      if (rc == PLATO_OK) rc = parse_buffer(buf, f, el->src, el->dst, weighted ? &el->w : nullptr);
      if (rc != PLATO_OK) {
        delete el;
        return rc;
      }
    }
    uint32_t mx = 0;
    const int64_t n = static_cast<int64_t>(el->src.size());
#pragma omp parallel for reduction(max : mx) schedule(static)
    for (int64_t i = 0; i < n; ++i) mx = std::max(mx, std::max(el->src[i], el->dst[i]));
    if (n > 0 && mx == 0xFFFFFFFFu) {
      delete el;
      return set_error(PLATO_EINVAL, "plato_edge_list_read_csv: vertex id 2^32-1 leaves no room for the vertex count");
    }
    el->vertices = n > 0 ? mx + 1 : 0;
    *out = el;
    return PLATO_OK;
  } catch (const std::bad_alloc&) {
    return set_error(PLATO_ENOMEM, "plato_edge_list_read_csv: host allocation failed");
  }
}

}  // namespace

extern "C" int plato_edge_list_read_csv(const char* path, plato_edge_list** out) {
  return read_csv(path, false, out);
}

extern "C" int plato_edge_list_read_csv_weighted(const char* path, plato_edge_list** out) {
  return read_csv(path, true, out);
}

extern "C" int plato_edge_list_weights(const plato_edge_list* el, const double** weights) {
  if (!el || !weights) return set_error(PLATO_EINVAL, "plato_edge_list_weights: null argument");
  *weights = el->weighted ? el->w.data() : nullptr;
  return PLATO_OK;
}

extern "C" int plato_write_vertex_csv(const char* dir, const char* prefix, const void* values,
                                      int value_type, uint32_t n, uint32_t files, int gzip) {
  if (!dir || !values) return set_error(PLATO_EINVAL, "plato_write_vertex_csv: null argument");
  if (value_type != PLATO_VALUE_F32 && value_type != PLATO_VALUE_U32)
    return set_error(PLATO_EINVAL, "plato_write_vertex_csv: unknown value type");
  if (files == 0) return set_error(PLATO_EINVAL, "plato_write_vertex_csv: files must be >= 1");
  const std::string pre = prefix ? prefix : "";
  std::vector<int> rcs(files, PLATO_OK);
  std::vector<std::string> errs(files);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < static_cast<int64_t>(files); ++i) {
    const uint64_t v0 = static_cast<uint64_t>(n) * i / files, v1 = static_cast<uint64_t>(n) * (i + 1) / files;
    char name[64];
    std::snprintf(name, sizeof(name), "%04u.csv%s", static_cast<unsigned>(i), gzip ? ".gz" : "");
    const std::string path = std::string(dir) + "/" + pre + name;
    std::string text;
    text.reserve((v1 - v0) * 20);
    char line[64];
    for (uint64_t v = v0; v < v1; ++v) {
      int k;
      if (value_type == PLATO_VALUE_F32)
        k = std::snprintf(line, sizeof(line), "%llu,%g\n", static_cast<unsigned long long>(v),
                          static_cast<double>(static_cast<const float*>(values)[v]));
      else
        k = std::snprintf(line, sizeof(line), "%llu,%u\n", static_cast<unsigned long long>(v),
                          static_cast<const uint32_t*>(values)[v]);
      text.append(line, static_cast<size_t>(k));
    }
    bool ok;
    if (gzip) {
      gzFile f = gzopen(path.c_str(), "wb");
      ok = f != nullptr;
      for (size_t off = 0; ok && off < text.size(); off += (1u << 30)) {
        const unsigned len = static_cast<unsigned>(std::min<size_t>(1u << 30, text.size() - off));
        ok = gzwrite(f, text.data() + off, len) == static_cast<int>(len);
      }
      if (f) ok = (gzclose(f) == Z_OK) && ok;
    } else {
      FILE* f = std::fopen(path.c_str(), "wb");
      ok = f && std::fwrite(text.data(), 1, text.size(), f) == text.size();
      if (f) ok = (std::fclose(f) == 0) && ok;
    }
    if (!ok) {
      rcs[i] = PLATO_EINVAL;
      errs[i] = "cannot write " + path;
    }
  }
  for (uint32_t i = 0; i < files; ++i)
    if (rcs[i] != PLATO_OK) return set_error(rcs[i], errs[i]);
  return PLATO_OK;
}
