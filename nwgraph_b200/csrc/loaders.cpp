// Graph file readers for the engine's inputs: Matrix Market coordinate files
// and NWGraph's binary edge lists, parsed on all host cores.
//
// The reference's driver loads its graph with load_graph
// (bench/gapbs/common.hpp:83-100): a file starting with "NW" is a serialized
// edge list (edge_list.hpp:237-280 over graph_base.hpp:72-86 and
// soa.hpp:333-373), a file starting with "%%MatrixMarket" goes through
// read_mm<directed> (io/mmio.hpp:86-103, 171-208), which parses one line at a
// time through a stringstream. Here both yield the same edge list, in the same
// order -- for Matrix Market: entry (i, j) as (i-1, j-1), followed by
// (j-1, i-1) when the file is symmetric and i != j -- so the CSR built from it
// (nwgpu_csr_from_edges) has the reference's rows.
//
// Matrix Market: the file is mapped, the data lines are split into one range
// per thread at line boundaries, each thread parses its range into local
// arrays, and the ranges are concatenated in order. Only coordinate files with
// general or symmetric symmetry are accepted (read_mm rejects the others);
// values are read as float when the field is not `pattern`.
//
// NW edge list: magic "NW Graph index_edge_list" (27 bytes), directedness
// (int), vertex count (size_t), open flag (bool), then the struct of arrays:
// edge count, array count, and per array its length, element size and data
// (sources and targets as uint32, then attributes).
//
// NW adjacency (adjacency.hpp:176-191 over compressed.hpp:377-413): vertex
// count (size_t), open flag (bool), magic "NW GRAPH indexed_struct_of_arrays"
// (34 bytes), N (8 bytes written from a 4-byte index, so only the low 4 carry
// the value), the row pointers (length, element size, data), then the struct
// of arrays of the entries (count, array count, per array length, element
// size, data: column ids, then attributes). This is a CSR already: it is read
// into row_ptr / col directly.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/nwgpu.h"

namespace nwgpu {
int  fail(int code, const char* fmt, ...);
void clear_error();
}  // namespace nwgpu

namespace {

using nwgpu::fail;

struct Mapped {
  const char* p = nullptr;
  size_t      size = 0;
  int         fd = -1;
  ~Mapped() {
    if (p && size) munmap(const_cast<char*>(p), size);
    if (fd >= 0) close(fd);
  }
};

int map_file(const char* path, Mapped* m) {
  if (!path) return fail(NWGPU_ERR_INVALID_ARG, "path is NULL");
  m->fd = open(path, O_RDONLY);
  if (m->fd < 0) return fail(NWGPU_ERR_INVALID_ARG, "cannot open %s: %s", path, strerror(errno));
  struct stat st;
  if (fstat(m->fd, &st) != 0) return fail(NWGPU_ERR_INVALID_ARG, "cannot stat %s", path);
  m->size = (size_t)st.st_size;
  if (m->size == 0) return fail(NWGPU_ERR_INVALID_GRAPH, "%s is empty", path);
  void* p = mmap(nullptr, m->size, PROT_READ, MAP_PRIVATE, m->fd, 0);
  if (p == MAP_FAILED) {
    m->size = 0;
    return fail(NWGPU_ERR_INVALID_ARG, "cannot map %s", path);
  }
  madvise(p, m->size, MADV_SEQUENTIAL);
  m->p = static_cast<const char*>(p);
  return NWGPU_OK;
}

// ---------------------------------------------------------------------------
// Matrix Market
// ---------------------------------------------------------------------------
struct MtxHeader {
  uint64_t n0 = 0, n1 = 0, entries = 0;
  bool     symmetric = false, pattern = false;
  size_t   data = 0;  // offset of the first entry line
};

size_t line_end(const char* p, size_t size, size_t at) {
  const void* nl = memchr(p + at, '\n', size - at);
  return nl ? (size_t)(static_cast<const char*>(nl) - p) : size;
}

int parse_mtx_header(const char* p, size_t size, MtxHeader* h) {
  size_t      e = line_end(p, size, 0);
  std::string first(p, e);
  char        w[5][64] = {{0}};
  const int   got = sscanf(first.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]);
  if (got < 5 || strcmp(w[0], "%%MatrixMarket") != 0) return fail(NWGPU_ERR_INVALID_GRAPH, "not a Matrix Market file");
  if (strcmp(w[2], "coordinate") != 0) return fail(NWGPU_ERR_UNSUPPORTED, "Matrix Market format '%s' (coordinate only)", w[2]);
  if (!strcmp(w[4], "symmetric"))
    h->symmetric = true;
  else if (strcmp(w[4], "general") != 0)
    return fail(NWGPU_ERR_UNSUPPORTED, "Matrix Market symmetry '%s' (general or symmetric only)", w[4]);
  h->pattern = !strcmp(w[3], "pattern");
  size_t at = e < size ? e + 1 : size;
  while (at < size && p[at] == '%') {  // comments
    e = line_end(p, size, at);
    at = e < size ? e + 1 : size;
  }
  if (at >= size) return fail(NWGPU_ERR_INVALID_GRAPH, "Matrix Market size line missing");
  e = line_end(p, size, at);
  std::string        sz(p + at, e - at);
  unsigned long long a = 0, b = 0, c = 0;
  if (sscanf(sz.c_str(), "%llu %llu %llu", &a, &b, &c) != 3)
    return fail(NWGPU_ERR_INVALID_GRAPH, "bad Matrix Market size line");
  h->n0 = a;
  h->n1 = b;
  h->entries = c;
  h->data = e < size ? e + 1 : size;
  return NWGPU_OK;
}

inline const char* skip_blank(const char* s, const char* end) {
  while (s < end && (*s == ' ' || *s == '\t' || *s == '\r')) ++s;
  return s;
}
inline bool parse_u64(const char*& s, const char* end, uint64_t* v) {
  s = skip_blank(s, end);
  if (s >= end || *s < '0' || *s > '9') return false;
  uint64_t x = 0;
  while (s < end && *s >= '0' && *s <= '9') x = x * 10 + (uint64_t)(*s++ - '0');
  *v = x;
  return true;
}

struct Chunk {
  std::vector<uint32_t> s, d;
  std::vector<float>    v;
  uint64_t              lines = 0;
  int                   err = 0;  // 1 bad line, 2 id out of range
};

void parse_range(const char* p, size_t b, size_t e, uint64_t max_lines, const MtxHeader& h, bool want_values, Chunk* c) {
  const char* s = p + b;
  const char* end = p + e;
  while (s < end && c->lines < max_lines) {
    const char* le = static_cast<const char*>(memchr(s, '\n', (size_t)(end - s)));
    if (!le) le = end;
    uint64_t    i, j;
    const char* q = s;
    if (!parse_u64(q, le, &i) || !parse_u64(q, le, &j)) {
      c->err = 1;
      return;
    }
    if (i == 0 || j == 0 || i > h.n0 || j > h.n0 || i > 0xFFFFFFFFull || j > 0xFFFFFFFFull) {
      c->err = 2;
      return;
    }
    float val = 1.0f;
    if (want_values && !h.pattern) {
      q = skip_blank(q, le);
      char buf[64];
      size_t len = std::min<size_t>((size_t)(le - q), sizeof buf - 1);
      memcpy(buf, q, len);
      buf[len] = 0;
      val = strtof(buf, nullptr);
    }
    c->s.push_back((uint32_t)(i - 1));
    c->d.push_back((uint32_t)(j - 1));
    if (want_values) c->v.push_back(val);
    if (h.symmetric && i != j) {
      c->s.push_back((uint32_t)(j - 1));
      c->d.push_back((uint32_t)(i - 1));
      if (want_values) c->v.push_back(val);
    }
    ++c->lines;
    s = le < end ? le + 1 : end;
  }
}

int read_mtx(const Mapped& f, uint32_t* src, uint32_t* dst, float* values, uint64_t capacity, uint64_t* m_out,
             int nthreads) {
  MtxHeader h;
  int       rc = parse_mtx_header(f.p, f.size, &h);
  if (rc) return rc;
  // thread ranges over the data region, cut at line starts
  const size_t b0 = h.data, total = f.size - b0;
  int          T = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  if (total < ((size_t)1 << 20)) T = 1;
  std::vector<size_t> cut(T + 1);
  cut[0] = b0;
  cut[T] = f.size;
  for (int t = 1; t < T; ++t) {
    size_t at = b0 + total * (size_t)t / (size_t)T;
    at = std::max(at, cut[t - 1]);
    const size_t e = line_end(f.p, f.size, at);
    cut[t] = e < f.size ? e + 1 : f.size;
  }
  // The ranges hold whole lines; each parses all of its lines (the entry
  // count limits the total afterwards, as read_mm reads exactly that many).
  std::vector<Chunk>       chunks(T);
  std::vector<std::thread> pool;
  for (int t = 0; t < T; ++t)
    pool.emplace_back([&, t] { parse_range(f.p, cut[t], cut[t + 1], ~0ull, h, values != nullptr, &chunks[t]); });
  for (auto& th : pool) th.join();
  uint64_t lines = 0, m = 0;
  for (int t = 0; t < T; ++t) {
    if (chunks[t].err && lines + chunks[t].lines < h.entries)
      return fail(NWGPU_ERR_INVALID_GRAPH, chunks[t].err == 1 ? "bad Matrix Market entry line"
                                                              : "Matrix Market entry outside 1..n");
    lines += chunks[t].lines;
  }
  if (lines < h.entries)
    return fail(NWGPU_ERR_INVALID_GRAPH, "Matrix Market file has %llu entries, the size line says %llu",
                (unsigned long long)lines, (unsigned long long)h.entries);
  // concatenate the first h.entries lines' edges in order
  uint64_t left = h.entries;
  for (int t = 0; t < T && left; ++t) {
    const Chunk& c = chunks[t];
    uint64_t     take_lines = std::min<uint64_t>(c.lines, left), take = 0;
    if (take_lines == c.lines) {
      take = c.s.size();
    } else {  // count the edges of the first take_lines lines
      for (uint64_t k = 0, l = 0; l < take_lines; ++l) {
        const bool two = h.symmetric && c.s[k] != c.d[k];
        k += two ? 2 : 1;
        take = k;
      }
    }
    if (m + take > capacity)
      return fail(NWGPU_ERR_INVALID_ARG, "the file yields more than %llu edges", (unsigned long long)capacity);
    memcpy(src + m, c.s.data(), take * sizeof(uint32_t));
    memcpy(dst + m, c.d.data(), take * sizeof(uint32_t));
    if (values) memcpy(values + m, c.v.data(), take * sizeof(float));
    m += take;
    left -= take_lines;
  }
  *m_out = m;
  return NWGPU_OK;
}

// ---------------------------------------------------------------------------
// NW binary edge list
// ---------------------------------------------------------------------------
constexpr char   kNwMagic[27] = "NW Graph index_edge_list";
constexpr size_t kNwHead = sizeof(kNwMagic) + sizeof(int32_t) + sizeof(uint64_t) + 1 + 2 * sizeof(uint64_t);

struct NwLayout {
  uint64_t n = 0, m = 0, arrays = 0;
  int32_t  directed = 1;
  size_t   off[3] = {0, 0, 0};   // data offsets of sources, targets, first attribute
  uint64_t attr_size = 0;        // element size of the first attribute (0: none)
};

int parse_nw(const Mapped& f, NwLayout* L) {
  const char* p = f.p;
  if (f.size < kNwHead || memcmp(p, kNwMagic, sizeof(kNwMagic)) != 0)
    return fail(NWGPU_ERR_INVALID_GRAPH, "not an NW Graph edge list");
  size_t at = sizeof(kNwMagic);
  memcpy(&L->directed, p + at, 4);
  at += 4;
  memcpy(&L->n, p + at, 8);
  at += 8 + 1;  // vertex count, open flag
  memcpy(&L->m, p + at, 8);
  memcpy(&L->arrays, p + at + 8, 8);
  at += 16;
  if (L->arrays < 2 || L->arrays > 16) return fail(NWGPU_ERR_INVALID_GRAPH, "NW edge list with %llu arrays",
                                                   (unsigned long long)L->arrays);
  for (uint64_t a = 0; a < L->arrays; ++a) {
    if (at + 16 > f.size) return fail(NWGPU_ERR_INVALID_GRAPH, "NW edge list truncated");
    uint64_t len, el;
    memcpy(&len, p + at, 8);
    memcpy(&el, p + at + 8, 8);
    at += 16;
    if (len != L->m) return fail(NWGPU_ERR_INVALID_GRAPH, "NW edge list array %llu has %llu of %llu entries",
                                 (unsigned long long)a, (unsigned long long)len, (unsigned long long)L->m);
    if (a < 2 && el != 4) return fail(NWGPU_ERR_UNSUPPORTED, "NW edge list with %llu-byte vertex ids",
                                      (unsigned long long)el);
    if (a < 3) L->off[a] = at;
    if (a == 2) L->attr_size = el;
    if (el == 0 || at + len * el > f.size) return fail(NWGPU_ERR_INVALID_GRAPH, "NW edge list truncated");
    at += len * el;
  }
  if (L->n >= 0xFFFFFFF0ull) return fail(NWGPU_ERR_INVALID_GRAPH, "NW edge list with n = %llu", (unsigned long long)L->n);
  return NWGPU_OK;
}

// ---------------------------------------------------------------------------
// NW binary adjacency
// ---------------------------------------------------------------------------
constexpr char   kNwAdjMagic[34] = "NW GRAPH indexed_struct_of_arrays";
constexpr size_t kNwAdjMagicAt = 8 + 1;

struct AdjLayout {
  uint64_t n = 0, nnz = 0, arrays = 0;
  size_t   rp = 0, col = 0, attr = 0;  // data offsets
  uint64_t attr_size = 0;
};

bool is_nw_adjacency(const Mapped& f) {
  return f.size >= kNwAdjMagicAt + sizeof(kNwAdjMagic) &&
         memcmp(f.p + kNwAdjMagicAt, kNwAdjMagic, sizeof(kNwAdjMagic)) == 0;
}

int parse_adj(const Mapped& f, AdjLayout* L) {
  const char* p = f.p;
  size_t      at = kNwAdjMagicAt + sizeof(kNwAdjMagic);
  auto        u64 = [&](uint64_t* v) {
    if (at + 8 > f.size) return false;
    memcpy(v, p + at, 8);
    at += 8;
    return true;
  };
  uint64_t N8 = 0, len = 0, el = 0;
  if (!u64(&N8) || !u64(&len) || !u64(&el)) return fail(NWGPU_ERR_INVALID_GRAPH, "NW adjacency truncated");
  L->n = N8 & 0xFFFFFFFFull;
  if (len != L->n + 1 || el != 4) return fail(NWGPU_ERR_UNSUPPORTED, "NW adjacency with %llu row pointers of %llu bytes",
                                              (unsigned long long)len, (unsigned long long)el);
  L->rp = at;
  if (at + 4 * len > f.size) return fail(NWGPU_ERR_INVALID_GRAPH, "NW adjacency truncated");
  at += 4 * len;
  if (!u64(&L->nnz) || !u64(&L->arrays) || L->arrays < 1 || L->arrays > 16)
    return fail(NWGPU_ERR_INVALID_GRAPH, "NW adjacency entries header");
  for (uint64_t a = 0; a < L->arrays; ++a) {
    if (!u64(&len) || !u64(&el)) return fail(NWGPU_ERR_INVALID_GRAPH, "NW adjacency truncated");
    if (len != L->nnz || el == 0 || at + len * el > f.size) return fail(NWGPU_ERR_INVALID_GRAPH, "NW adjacency array %llu",
                                                                       (unsigned long long)a);
    if (a == 0 && el != 4) return fail(NWGPU_ERR_UNSUPPORTED, "NW adjacency with %llu-byte column ids", (unsigned long long)el);
    if (a == 0) L->col = at;
    if (a == 1) {
      L->attr = at;
      L->attr_size = el;
    }
    at += len * el;
  }
  if (L->n >= 0xFFFFFFF0ull || L->nnz >= 0xFFFFFFF0ull) return fail(NWGPU_ERR_INVALID_GRAPH, "NW adjacency too large");
  return NWGPU_OK;
}

}  // namespace

extern "C" {

int nwgpu_adjacency_file_read(const char* path, uint32_t* row_ptr, uint32_t* col, float* values, uint64_t n_cap,
                              uint64_t nnz_cap, uint64_t* n_out, uint64_t* nnz_out) {
  nwgpu::clear_error();
  if (!n_out || !nnz_out) return fail(NWGPU_ERR_INVALID_ARG, "n / nnz is NULL");
  Mapped f;
  int    rc = map_file(path, &f);
  if (rc) return rc;
  if (!is_nw_adjacency(f)) return fail(NWGPU_ERR_INVALID_GRAPH, "not an NW Graph adjacency file");
  AdjLayout L;
  if ((rc = parse_adj(f, &L))) return rc;
  *n_out = L.n;
  *nnz_out = L.nnz;
  if (!row_ptr) return NWGPU_OK;  // sizes only
  if (L.n > n_cap || L.nnz > nnz_cap || (L.nnz && !col))
    return fail(NWGPU_ERR_INVALID_ARG, "the file holds n = %llu, nnz = %llu", (unsigned long long)L.n,
                (unsigned long long)L.nnz);
  memcpy(row_ptr, f.p + L.rp, (L.n + 1) * 4);
  if (L.nnz) memcpy(col, f.p + L.col, L.nnz * 4);
  if (values) {
    for (uint64_t e = 0; e < L.nnz; ++e) {
      if (L.attr_size == 4) {
        memcpy(values + e, f.p + L.attr + 4 * e, 4);
      } else if (L.attr_size == 8) {
        double x;
        memcpy(&x, f.p + L.attr + 8 * e, 8);
        values[e] = (float)x;
      } else {
        values[e] = 1.0f;
      }
    }
  }
  return NWGPU_OK;
}

int nwgpu_edge_file_probe(const char* path, nwgpu_edge_file* info) {
  nwgpu::clear_error();
  if (!info) return fail(NWGPU_ERR_INVALID_ARG, "info is NULL");
  memset(info, 0, sizeof(*info));
  Mapped f;
  int    rc = map_file(path, &f);
  if (rc) return rc;
  if (is_nw_adjacency(f)) {
    AdjLayout A;
    if ((rc = parse_adj(f, &A))) return rc;
    info->format = NWGPU_FILE_NW_ADJACENCY;
    info->n = A.n;
    info->max_edges = A.nnz;
    info->directed = 1;
    info->has_values = A.attr_size == 4 || A.attr_size == 8;
    return NWGPU_OK;
  }
  if (f.size >= 2 && f.p[0] == 'N' && f.p[1] == 'W') {
    NwLayout L;
    if ((rc = parse_nw(f, &L))) return rc;
    info->format = NWGPU_FILE_NW_EDGE_LIST;
    info->n = L.n;
    info->max_edges = L.m;
    info->directed = L.directed;
    info->has_values = L.attr_size == 4 || L.attr_size == 8;
    return NWGPU_OK;
  }
  MtxHeader h;
  if ((rc = parse_mtx_header(f.p, f.size, &h))) return rc;
  if (h.n0 >= 0xFFFFFFF0ull) return fail(NWGPU_ERR_INVALID_GRAPH, "n = %llu", (unsigned long long)h.n0);
  info->format = NWGPU_FILE_MATRIX_MARKET;
  info->n = h.n0;
  info->max_edges = h.symmetric ? 2 * h.entries : h.entries;
  info->directed = 1;
  info->has_values = !h.pattern;
  return NWGPU_OK;
}

int nwgpu_edge_file_read(const char* path, uint32_t* src, uint32_t* dst, float* values, uint64_t capacity,
                         uint64_t* m_out, int nthreads) {
  nwgpu::clear_error();
  if (!m_out) return fail(NWGPU_ERR_INVALID_ARG, "m is NULL");
  *m_out = 0;
  Mapped f;
  int    rc = map_file(path, &f);
  if (rc) return rc;
  if (capacity && (!src || !dst)) return fail(NWGPU_ERR_INVALID_ARG, "src / dst is NULL");
  if (f.size >= 2 && f.p[0] == 'N' && f.p[1] == 'W') {
    NwLayout L;
    if ((rc = parse_nw(f, &L))) return rc;
    if (L.m > capacity) return fail(NWGPU_ERR_INVALID_ARG, "the file holds %llu edges, capacity %llu",
                                    (unsigned long long)L.m, (unsigned long long)capacity);
    memcpy(src, f.p + L.off[0], L.m * 4);
    memcpy(dst, f.p + L.off[1], L.m * 4);
    for (uint64_t e = 0; e < L.m; ++e)
      if (src[e] >= L.n || dst[e] >= L.n) return fail(NWGPU_ERR_INVALID_GRAPH, "NW edge list: vertex id >= n");
    if (values) {
      if (L.attr_size == 4) {
        memcpy(values, f.p + L.off[2], L.m * 4);
      } else if (L.attr_size == 8) {
        for (uint64_t e = 0; e < L.m; ++e) {
          double x;
          memcpy(&x, f.p + L.off[2] + 8 * e, 8);
          values[e] = (float)x;
        }
      } else {
        for (uint64_t e = 0; e < L.m; ++e) values[e] = 1.0f;
      }
    }
    *m_out = L.m;
    return NWGPU_OK;
  }
  return read_mtx(f, src, dst, values, capacity, m_out, nthreads);
}

int nwgpu_edge_file_write_nw(const char* path, const uint32_t* src, const uint32_t* dst, uint64_t m, uint64_t n,
                             int directed) {
  nwgpu::clear_error();
  if (!path || (m && (!src || !dst))) return fail(NWGPU_ERR_INVALID_ARG, "NULL argument");
  FILE* fp = fopen(path, "wb");
  if (!fp) return fail(NWGPU_ERR_INVALID_ARG, "cannot create %s: %s", path, strerror(errno));
  const int32_t  d = directed ? 1 : 0;
  const uint8_t  open_flag = 0;
  const uint64_t arrays = 2, four = 4;
  bool ok = fwrite(kNwMagic, sizeof(kNwMagic), 1, fp) == 1 && fwrite(&d, 4, 1, fp) == 1 && fwrite(&n, 8, 1, fp) == 1 &&
            fwrite(&open_flag, 1, 1, fp) == 1 && fwrite(&m, 8, 1, fp) == 1 && fwrite(&arrays, 8, 1, fp) == 1;
  for (const uint32_t* a : {src, dst}) {
    ok = ok && fwrite(&m, 8, 1, fp) == 1 && fwrite(&four, 8, 1, fp) == 1 && (m == 0 || fwrite(a, 4, m, fp) == m);
  }
  ok = (fclose(fp) == 0) && ok;
  if (!ok) return fail(NWGPU_ERR_INVALID_ARG, "cannot write %s", path);
  return NWGPU_OK;
}

}  // extern "C"
