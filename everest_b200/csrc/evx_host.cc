// Host-side graph preparation behind the C ABI: edge-list parsing, stable
// sort by timestamp, vertex relabeling, CSR construction and motif decoding.
//
// Reference behaviour restated:
//  * EdgeListLoader::createEdgeListCache (src/core/cpu/data.cc:175-290):
//    "u v t" lines parsed with atoi, edges stable-sorted by t, IDS[i] = the
//    original (0-based) line index of sorted edge i.
//  * GraphDataLoader::createGraphData (src/core/gpu/data.cu:124-348): the
//    edge range [beg, end) is relabeled to vertices 0..V-1, out/in edge-id
//    lists are grouped by endpoint and ascending in edge id (a stable sort on
//    the endpoint), CSR offsets are their prefix sums, Eg is AoS {u,v,t} and
//    Euid is the IDS slice.  The vertex numbering differs from the
//    reference's (first appearance here); it changes no count and no
//    enumeration row, which carry original line ids.
//  * HostMotifData (src/core/cpu/data.cc:411-449) over
//    TemporalGraph::ReadGraph (src/core/cpu/Graph.cc:198-258): motif lines
//    stable-sorted by t, nodes numbered by first appearance (u before v).
#include <algorithm>
#include <cerrno>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <sstream>
#include <string>
#include <sys/mman.h>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>
#include <unordered_map>
#include <vector>

#include "../../include/everest_b200.h"

namespace evx {
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
}  // namespace evx

using evx::fail;

namespace {

template <typename T>
T *xmalloc(size_t n) {
  return static_cast<T *>(std::malloc(sizeof(T) * (n ? n : 1)));
}

// Parse one integer with atoi semantics (leading blanks, optional sign).
inline const char *parse_int(const char *p, const char *end, long long *out) {
  while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) p++;
  bool neg = false;
  if (p < end && (*p == '-' || *p == '+')) { neg = (*p == '-'); p++; }
  long long v = 0;
  while (p < end && *p >= '0' && *p <= '9') { v = v * 10 + (*p - '0'); p++; }
  *out = neg ? -v : v;
  return p;
}

inline bool blank_line(const char *p, const char *e) {
  for (; p < e; p++)
    if (*p != ' ' && *p != '\t' && *p != '\r') return false;
  return true;
}

// Stable LSD radix sort of indices by int32 key (two 16-bit passes).
void stable_sort_by_key(const int *key, int64_t n, std::vector<int> &order) {
  std::vector<int> tmp(n);
  order.resize(n);
  for (int64_t i = 0; i < n; i++) order[i] = (int)i;
  std::vector<int64_t> cnt(65537);
  for (int pass = 0; pass < 2; pass++) {
    std::fill(cnt.begin(), cnt.end(), 0);
    const int shift = pass * 16;
    auto digit = [&](int idx) -> unsigned {
      const unsigned k = (unsigned)key[idx] ^ 0x80000000u;  // signed order
      return (k >> shift) & 0xFFFFu;
    };
    for (int64_t i = 0; i < n; i++) cnt[digit(order[i]) + 1]++;
    for (int d = 0; d < 65536; d++) cnt[d + 1] += cnt[d];
    for (int64_t i = 0; i < n; i++) tmp[cnt[digit(order[i])]++] = order[i];
    order.swap(tmp);
  }
}

struct MotifEdge { long long u, v, t; int line; };

int decode_motif_lines(const std::vector<MotifEdge> &rows_in, int *k, int *mu, int *mv,
                       int *num_nodes) {
  std::vector<MotifEdge> rows = rows_in;
  if (rows.empty()) return fail(EVX_ERR_INVALID, "motif has no edges");
  if ((int)rows.size() > EVX_MAX_MOTIF_EDGES)
    return fail(EVX_ERR_INVALID, "motif has more than " + std::to_string(EVX_MAX_MOTIF_EDGES) + " edges");
  std::stable_sort(rows.begin(), rows.end(),
                   [](const MotifEdge &a, const MotifEdge &b) { return a.t < b.t; });
  std::vector<long long> ids;
  auto map = [&](long long x) {
    for (size_t i = 0; i < ids.size(); i++)
      if (ids[i] == x) return (int)i;
    ids.push_back(x);
    return (int)ids.size() - 1;
  };
  for (size_t j = 0; j < rows.size(); j++) {
    mu[j] = map(rows[j].u);
    mv[j] = map(rows[j].v);
  }
  *k = (int)rows.size();
  *num_nodes = (int)ids.size();
  return EVX_OK;
}

}  // namespace

extern "C" {

void evx_free(void *p) { std::free(p); }

int evx_edgelist_parse(const char *path, int64_t *num_edges, int **u, int **v, int **t,
                       int **ids) {
  if (!path || !num_edges || !u || !v || !t || !ids) return fail(EVX_ERR_INVALID, "null argument");
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) return fail(EVX_ERR_IO, std::string("cannot open ") + path + ": " + std::strerror(errno));
  struct stat st;
  if (fstat(fd, &st) != 0) { ::close(fd); return fail(EVX_ERR_IO, "cannot stat graph file"); }
  const size_t size = (size_t)st.st_size;
  const char *data = nullptr;
  if (size > 0) {
    void *m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
    if (m == MAP_FAILED) { ::close(fd); return fail(EVX_ERR_IO, "mmap failed"); }
    data = static_cast<const char *>(m);
  }
  ::close(fd);
  // split into chunks at line boundaries; parse in parallel
  unsigned nth = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if (size < (1u << 20)) nth = 1;
  std::vector<size_t> cut(nth + 1, size);
  cut[0] = 0;
  for (unsigned i = 1; i < nth; i++) {
    size_t p = size * i / nth;
    while (p < size && data[p - 1] != '\n') p++;
    cut[i] = p;
  }
  std::vector<std::vector<int>> U(nth), Vv(nth), T(nth);
  std::vector<int> bad(nth, 0);
  auto work = [&](unsigned c) {
    const char *p = data + cut[c], *end = data + cut[c + 1];
    while (p < end) {
      const char *nl = static_cast<const char *>(std::memchr(p, '\n', end - p));
      const char *le = nl ? nl : end;
      if (!blank_line(p, le)) {
        long long a, b, tt;
        const char *q = parse_int(p, le, &a);
        q = parse_int(q, le, &b);
        parse_int(q, le, &tt);
        if (a < INT_MIN || a > INT_MAX || b < INT_MIN || b > INT_MAX || tt < INT_MIN || tt > INT_MAX)
          bad[c] = 1;
        U[c].push_back((int)a);
        Vv[c].push_back((int)b);
        T[c].push_back((int)tt);
      }
      p = le + 1;
    }
  };
  std::vector<std::thread> th;
  for (unsigned c = 1; c < nth; c++) th.emplace_back(work, c);
  if (size) work(0);
  for (auto &x : th) x.join();
  if (data) munmap((void *)data, size);
  for (unsigned c = 0; c < nth; c++)
    if (bad[c]) return fail(EVX_ERR_OVERFLOW, "graph value does not fit int32");
  int64_t n = 0;
  for (unsigned c = 0; c < nth; c++) n += (int64_t)U[c].size();
  if (n >= INT_MAX) return fail(EVX_ERR_OVERFLOW, "too many edges for int32 ids");
  std::vector<int> uu(n), vv(n), tt(n);
  int64_t o = 0;
  for (unsigned c = 0; c < nth; c++) {
    std::copy(U[c].begin(), U[c].end(), uu.begin() + o);
    std::copy(Vv[c].begin(), Vv[c].end(), vv.begin() + o);
    std::copy(T[c].begin(), T[c].end(), tt.begin() + o);
    o += (int64_t)U[c].size();
  }
  std::vector<int> order;
  stable_sort_by_key(tt.data(), n, order);
  int *ou = xmalloc<int>(n), *ov = xmalloc<int>(n), *ot = xmalloc<int>(n), *oi = xmalloc<int>(n);
  if (!ou || !ov || !ot || !oi) {
    std::free(ou); std::free(ov); std::free(ot); std::free(oi);
    return fail(EVX_ERR_NOMEM, "host allocation failed");
  }
  for (int64_t i = 0; i < n; i++) {
    const int j = order[i];
    ou[i] = uu[j];
    ov[i] = vv[j];
    ot[i] = tt[j];
    oi[i] = j;
  }
  *num_edges = n;
  *u = ou; *v = ov; *t = ot; *ids = oi;
  return EVX_OK;
}

int evx_graph_build_host(const int *u, const int *v, const int *t, const int *ids, int64_t beg,
                         int64_t end, int64_t *num_edges, int64_t *num_vertices, int **eg,
                         int **out_v, int **in_v, int **out_r, int **in_r, int **euid) {
  if (!u || !v || !t || !num_edges || !num_vertices || !eg || !out_v || !in_v || !out_r || !in_r ||
      !euid)
    return fail(EVX_ERR_INVALID, "null argument");
  if (beg < 0 || end < beg) return fail(EVX_ERR_INVALID, "bad edge range");
  const int64_t E = end - beg;
  for (int64_t i = beg + 1; i < end; i++)
    if (t[i] < t[i - 1]) return fail(EVX_ERR_INVALID, "edge list is not sorted by timestamp");
  // relabel vertices by first appearance (u before v, in edge order)
  std::vector<int> nu(E), nv(E);
  int64_t V = 0;
  int lo = INT_MAX, hi = INT_MIN;
  for (int64_t i = beg; i < end; i++) {
    lo = std::min(lo, std::min(u[i], v[i]));
    hi = std::max(hi, std::max(u[i], v[i]));
  }
  if (E > 0 && (int64_t)hi - (int64_t)lo < 4 * E + (1 << 20)) {
    std::vector<int> map((size_t)((int64_t)hi - lo + 1), -1);
    for (int64_t i = 0; i < E; i++) {
      int &a = map[u[beg + i] - lo];
      if (a < 0) a = (int)V++;
      nu[i] = a;
      int &b = map[v[beg + i] - lo];
      if (b < 0) b = (int)V++;
      nv[i] = b;
    }
  } else if (E > 0) {
    std::unordered_map<int, int> map;
    map.reserve((size_t)E);
    for (int64_t i = 0; i < E; i++) {
      auto ia = map.emplace(u[beg + i], (int)V);
      if (ia.second) V++;
      nu[i] = ia.first->second;
      auto ib = map.emplace(v[beg + i], (int)V);
      if (ib.second) V++;
      nv[i] = ib.first->second;
    }
  }
  int *o_eg = xmalloc<int>(3 * E), *o_ov = xmalloc<int>(E), *o_iv = xmalloc<int>(E);
  int *o_or = xmalloc<int>(V + 1), *o_ir = xmalloc<int>(V + 1), *o_eu = xmalloc<int>(E);
  if (!o_eg || !o_ov || !o_iv || !o_or || !o_ir || !o_eu) {
    std::free(o_eg); std::free(o_ov); std::free(o_iv); std::free(o_or); std::free(o_ir);
    std::free(o_eu);
    return fail(EVX_ERR_NOMEM, "host allocation failed");
  }
  std::memset(o_or, 0, sizeof(int) * (V + 1));
  std::memset(o_ir, 0, sizeof(int) * (V + 1));
  for (int64_t i = 0; i < E; i++) {
    o_or[nu[i] + 1]++;
    o_ir[nv[i] + 1]++;
  }
  for (int64_t x = 0; x < V; x++) {
    o_or[x + 1] += o_or[x];
    o_ir[x + 1] += o_ir[x];
  }
  std::vector<int> oc(o_or, o_or + V), ic(o_ir, o_ir + V);
  for (int64_t i = 0; i < E; i++) {
    o_ov[oc[nu[i]]++] = (int)i;
    o_iv[ic[nv[i]]++] = (int)i;
    o_eg[3 * i] = nu[i];
    o_eg[3 * i + 1] = nv[i];
    o_eg[3 * i + 2] = t[beg + i];
    o_eu[i] = ids ? ids[beg + i] : (int)(beg + i);
  }
  *num_edges = E;
  *num_vertices = V;
  *eg = o_eg; *out_v = o_ov; *in_v = o_iv; *out_r = o_or; *in_r = o_ir; *euid = o_eu;
  return EVX_OK;
}

int evx_motif_parse_text(const char *text, int *k, int *mu, int *mv, int *num_nodes) {
  if (!text || !k || !mu || !mv || !num_nodes) return fail(EVX_ERR_INVALID, "null argument");
  std::istringstream in(text);
  std::string line;
  std::vector<MotifEdge> rows;
  int ln = 0;
  while (std::getline(in, line)) {
    std::istringstream sl(line);
    long long a, b, c;
    if (sl >> a >> b >> c) {
      rows.push_back({a, b, c, ln});
    } else {
      std::istringstream chk(line);
      std::string tok;
      if (chk >> tok) return fail(EVX_ERR_INVALID, "malformed motif line " + std::to_string(ln + 1));
    }
    ln++;
  }
  return decode_motif_lines(rows, k, mu, mv, num_nodes);
}

int evx_motif_parse(const char *path, int *k, int *mu, int *mv, int *num_nodes) {
  if (!path) return fail(EVX_ERR_INVALID, "null path");
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(EVX_ERR_IO, std::string("cannot open motif file ") + path);
  std::string s;
  char buf[4096];
  size_t r;
  while ((r = std::fread(buf, 1, sizeof(buf), f)) > 0) s.append(buf, r);
  std::fclose(f);
  return evx_motif_parse_text(s.c_str(), k, mu, mv, num_nodes);
}

}  // extern "C"
