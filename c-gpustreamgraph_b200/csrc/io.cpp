// io.cpp -- readers for the reference's input files (host code, C ABI).
//
//   * graph edge list, "market_big": one "src dst" pair per line, optionally a
//     third weight column; the vertex count is max id + 1 and edges keep file
//     order (src/utils/parser.cpp:296-406, ReadGraphMarket_bigdata);
//   * stream sizes: one "adds dels" line per snapshot
//     (include/framework/Loader.h:27-62);
//   * update file: "a src dst [w]" inserts and "d src dst [w]" deletes, other
//     line types ignored (Loader.h:64-100, ReadWeightList).
// Blank lines and lines starting with '#' or '%' are skipped.  Unlike the
// reference's Loader (which writes m_batch_size[pos] after only reserve(10)),
// any number of snapshots is accepted.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sgs.h"

namespace sgs {
void set_last_error(const std::string &msg);
}

namespace {

struct Reader {
  std::vector<char> buf;
  size_t pos = 0;
  bool open(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize(n > 0 ? (size_t)n + 1 : 1);
    const size_t got = n > 0 ? std::fread(buf.data(), 1, (size_t)n, f) : 0;
    std::fclose(f);
    buf.resize(got + 1);
    buf[got] = '\0';
    return true;
  }
  // Next line as [b, e); false at end of file.
  bool line(const char *&b, const char *&e) {
    const size_t n = buf.size() - 1;
    while (pos < n) {
      size_t s = pos;
      while (pos < n && buf[pos] != '\n') ++pos;
      size_t t = pos;
      if (pos < n) ++pos;
      while (s < t && (buf[s] == ' ' || buf[s] == '\t' || buf[s] == '\r')) ++s;
      if (s == t || buf[s] == '#' || buf[s] == '%') continue;
      b = buf.data() + s;
      e = buf.data() + t;
      return true;
    }
    return false;
  }
};

// Parses up to `max` unsigned integers from [b, e); returns how many.
int parse_uints(const char *b, const char *e, uint64_t *out, int max) {
  int k = 0;
  const char *p = b;
  while (p < e && k < max) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    if (p >= e || *p < '0' || *p > '9') break;
    uint64_t v = 0;
    while (p < e && *p >= '0' && *p <= '9') v = v * 10 + (uint64_t)(*p++ - '0');
    out[k++] = v;
  }
  return k;
}

template <class T>
T *dup(const std::vector<T> &v) {
  T *p = (T *)std::malloc(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (!p) return nullptr;
  if (!v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
  return p;
}

int fail(int code, const std::string &msg) {
  sgs::set_last_error(msg);
  return code;
}

}  // namespace

extern "C" {

SGS_API void sgs_free(void *p) { std::free(p); }

SGS_API int sgs_read_edge_list(const char *path, uint32_t *nv, uint64_t *ne, uint32_t **src,
                               uint32_t **dst, uint32_t **w) {
  if (!path || !nv || !ne || !src || !dst) return fail(SGS_ERR_INVALID, "null argument");
  Reader r;
  if (!r.open(path)) return fail(SGS_ERR_INVALID, std::string("cannot open ") + path);
  std::vector<uint32_t> s, d, ww;
  uint64_t mx = 0, lineno = 0;
  int cols = -1;
  const char *b, *e;
  while (r.line(b, e)) {
    ++lineno;
    uint64_t x[3];
    const int k = parse_uints(b, e, x, 3);
    if (k < 2) return fail(SGS_ERR_INVALID, "malformed edge at data line " + std::to_string(lineno));
    if (x[0] >= 0xFFFFFFFFull || x[1] >= 0xFFFFFFFFull)
      return fail(SGS_ERR_INVALID, "vertex id too large at data line " + std::to_string(lineno));
    if (cols < 0) cols = k;
    s.push_back((uint32_t)x[0]);
    d.push_back((uint32_t)x[1]);
    if (cols >= 3) {
      if (k < 3) return fail(SGS_ERR_INVALID, "missing weight at data line " + std::to_string(lineno));
      ww.push_back((uint32_t)x[2]);
    }
    mx = std::max(mx, std::max(x[0], x[1]));
  }
  *nv = s.empty() ? 0u : (uint32_t)(mx + 1);
  *ne = s.size();
  *src = dup(s);
  *dst = dup(d);
  if (w) *w = cols >= 3 ? dup(ww) : nullptr;
  if (!*src || !*dst) return fail(SGS_ERR_OOM, "host allocation failed");
  return SGS_OK;
}

SGS_API int sgs_read_stream_sizes(const char *path, uint32_t *nsnap, uint64_t **adds,
                                  uint64_t **dels) {
  if (!path || !nsnap || !adds || !dels) return fail(SGS_ERR_INVALID, "null argument");
  Reader r;
  if (!r.open(path)) return fail(SGS_ERR_INVALID, std::string("cannot open ") + path);
  std::vector<uint64_t> a, d;
  const char *b, *e;
  while (r.line(b, e)) {
    uint64_t x[2];
    if (parse_uints(b, e, x, 2) < 2)
      return fail(SGS_ERR_INVALID, "malformed stream-size line " + std::to_string(a.size() + 1));
    a.push_back(x[0]);
    d.push_back(x[1]);
  }
  *nsnap = (uint32_t)a.size();
  *adds = dup(a);
  *dels = dup(d);
  return SGS_OK;
}

SGS_API int sgs_read_update_file(const char *path, uint64_t *n_add, uint32_t **add_u,
                                 uint32_t **add_v, uint32_t **add_w, uint64_t *n_del,
                                 uint32_t **del_u, uint32_t **del_v, uint32_t **del_w) {
  if (!path || !n_add || !add_u || !add_v || !n_del || !del_u || !del_v)
    return fail(SGS_ERR_INVALID, "null argument");
  Reader r;
  if (!r.open(path)) return fail(SGS_ERR_INVALID, std::string("cannot open ") + path);
  std::vector<uint32_t> au, av, aw, du, dv, dw;
  const char *b, *e;
  uint64_t lineno = 0;
  while (r.line(b, e)) {
    ++lineno;
    const char type = *b;
    const char *p = b + 1;
    if ((type != 'a' && type != 'd') || (p < e && *p != ' ' && *p != '\t')) continue;
    uint64_t x[3] = {0, 0, 0};
    const int k = parse_uints(p, e, x, 3);
    if (k < 2) return fail(SGS_ERR_INVALID, "malformed update at data line " + std::to_string(lineno));
    if (x[0] >= 0xFFFFFFFFull || x[1] >= 0xFFFFFFFFull)
      return fail(SGS_ERR_INVALID, "vertex id too large at data line " + std::to_string(lineno));
    if (type == 'a') {
      au.push_back((uint32_t)x[0]);
      av.push_back((uint32_t)x[1]);
      aw.push_back(k >= 3 ? (uint32_t)x[2] : 0u);
    } else {
      du.push_back((uint32_t)x[0]);
      dv.push_back((uint32_t)x[1]);
      dw.push_back(k >= 3 ? (uint32_t)x[2] : 0u);
    }
  }
  *n_add = au.size();
  *n_del = du.size();
  *add_u = dup(au);
  *add_v = dup(av);
  if (add_w) *add_w = dup(aw);
  *del_u = dup(du);
  *del_v = dup(dv);
  if (del_w) *del_w = dup(dw);
  return SGS_OK;
}

}  // extern "C"
