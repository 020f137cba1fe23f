// Graph files into the registry: NWGraph's MatrixMarket reader and its
// binary adjacency format, read on the host and uploaded once through
// nwg_graph_register / nwg_graph_register_u32off.
//
// MatrixMarket (read_mm, io/mmio.hpp:172-208 with mm_fill :60-103 in NWGraph):
//   header "%%MatrixMarket matrix coordinate <field> general|symmetric",
//   '%' comment lines, "rows cols nnz", then nnz lines "i j [value]" with
//   1-based ids.  Each line is an entry i-1 -> j-1; a symmetric file also
//   contributes j-1 -> i-1 for i != j; self-loops and duplicates are kept,
//   values are ignored.  n = max(rows, cols, largest id + 1).
// NW binary (index_adjacency::serialize, adjacency.hpp:158-162 over
//   unipartite_graph_base::serialize, graph_base.hpp:71-74, and
//   indexed_struct_of_arrays::serialize, containers/compressed.hpp:303-312):
//     u64 vertex count, u8 is_open,
//     34 bytes "NW GRAPH indexed_struct_of_arrays\0",
//     8 bytes N_ (written as sizeof(size_t) bytes from an index_t member:
//       with 4-byte offsets the high half is whatever followed it in
//       memory; its value after NWGraph's fill is N + 1, not N),
//     u64 offsets count (N + 1), u64 offset size (4 or 8), the offsets,
//     u64 entries (M), u64 arrays, then per array: u64 count, u64 element
//       size, data -- array 0 holds the target ids (4 bytes).
// Rows are sorted by target here (NWGraph's fill orders a row by an
// unstable sort; the order changes only which equal-depth parent a pull
// picks, never a depth).  The in-CSR is the transpose of the out-CSR, or the
// out-CSR itself when the file is symmetric.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "nwg_internal.cuh"

using namespace nwg;

#define NWG_API extern "C" __attribute__((visibility("default")))

namespace {

struct Csr {
  uint64_t              n = 0;
  std::vector<uint64_t> off;
  std::vector<uint32_t> col;
};

// Rows of (src[i] -> dst[i]) sorted by target, duplicates kept (counting
// sort by source, then each row sorted).
void build_rows(uint64_t n, const std::vector<uint32_t>& src, const std::vector<uint32_t>& dst, Csr& out) {
  out.n = n;
  out.off.assign(n + 1, 0);
  for (uint32_t s : src) out.off[(uint64_t)s + 1]++;
  for (uint64_t i = 0; i < n; ++i) out.off[i + 1] += out.off[i];
  out.col.resize(src.size());
  std::vector<uint64_t> pos(out.off.begin(), out.off.end() - 1);
  for (size_t i = 0; i < src.size(); ++i) out.col[pos[src[i]]++] = dst[i];
  for (uint64_t v = 0; v < n; ++v) std::sort(out.col.begin() + out.off[v], out.col.begin() + out.off[v + 1]);
}

bool read_file(const char* path, std::string& data) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  data.resize(sz > 0 ? (size_t)sz : 0);
  const size_t got = data.empty() ? 0 : std::fread(&data[0], 1, data.size(), f);
  std::fclose(f);
  return got == data.size();
}

// Scans an unsigned decimal at p (after blanks); false when there is none.
bool scan_u64(const char*& p, const char* end, uint64_t& x) {
  while (p < end && (*p == ' ' || *p == '\t')) ++p;
  if (p >= end || *p < '0' || *p > '9') return false;
  x = 0;
  while (p < end && *p >= '0' && *p <= '9') x = x * 10 + (uint64_t)(*p++ - '0');
  return true;
}

int parse_mm(const std::string& data, std::vector<uint32_t>& src, std::vector<uint32_t>& dst, uint64_t& n,
             bool& symmetric) {
  const char* p   = data.data();
  const char* end = p + data.size();
  auto        next_line = [&](const char*& q) {
    while (q < end && *q != '\n') ++q;
    if (q < end) ++q;
  };
  // header: %%MatrixMarket matrix coordinate <field> <symmetry>
  const char* h = p;
  next_line(p);
  std::string header(h, p);
  char        w[5][64] = {};
  if (std::sscanf(header.c_str(), "%63s %63s %63s %63s %63s", w[0], w[1], w[2], w[3], w[4]) < 5 ||
      std::strcmp(w[0], "%%MatrixMarket") != 0)
    return set_error(NWG_EINVAL, "not a MatrixMarket file (first line must start with %%MatrixMarket)");
  if (std::strcmp(w[2], "coordinate") != 0) return set_error(NWG_EINVAL, "only coordinate MatrixMarket files hold graphs");
  if (std::strcmp(w[4], "symmetric") == 0) symmetric = true;
  else if (std::strcmp(w[4], "general") == 0) symmetric = false;
  else return set_error(NWG_EINVAL, std::string("bad MatrixMarket symmetry: ") + w[4]);
  while (p < end && *p == '%') next_line(p);  // comments
  uint64_t n0 = 0, n1 = 0, nnz = 0;
  if (!scan_u64(p, end, n0) || !scan_u64(p, end, n1) || !scan_u64(p, end, nnz))
    return set_error(NWG_EINVAL, "MatrixMarket size line missing");
  next_line(p);
  src.reserve((symmetric ? 2 : 1) * nnz);
  dst.reserve((symmetric ? 2 : 1) * nnz);
  uint64_t maxid = 0;
  for (uint64_t i = 0; i < nnz; ++i) {
    uint64_t d0 = 0, d1 = 0;
    if (!scan_u64(p, end, d0) || !scan_u64(p, end, d1))
      return set_error(NWG_EINVAL, "MatrixMarket entry " + std::to_string(i + 1) + " of " + std::to_string(nnz) +
                                       " missing or malformed");
    if (d0 == 0 || d1 == 0 || d0 > 0xFFFFFFFEull || d1 > 0xFFFFFFFEull)
      return set_error(NWG_EINVAL, "MatrixMarket entry " + std::to_string(i + 1) + ": ids must be in 1..2^32-2");
    next_line(p);  // the value, if any, is ignored
    src.push_back((uint32_t)(d0 - 1));
    dst.push_back((uint32_t)(d1 - 1));
    if (symmetric && d0 != d1) {
      src.push_back((uint32_t)(d1 - 1));
      dst.push_back((uint32_t)(d0 - 1));
    }
    maxid = std::max(maxid, std::max(d0, d1));
  }
  n = std::max(std::max(n0, n1), maxid);
  if (n == 0 || n >= 0xFFFFFFFFull) return set_error(NWG_EINVAL, "MatrixMarket vertex count out of range");
  return NWG_OK;
}

int parse_nwbin(const std::string& data, Csr& out) {
  static const char kMagic[34] = "NW GRAPH indexed_struct_of_arrays";
  size_t            at         = 0;
  auto              get        = [&](void* dst, size_t bytes) {
    if (at + bytes > data.size()) return false;
    std::memcpy(dst, data.data() + at, bytes);
    at += bytes;
    return true;
  };
  uint64_t vcount = 0, nfield = 0, noff = 0, offsz = 0, m = 0, narrays = 0;
  uint8_t  is_open = 0;
  char     magic[34];
  if (!get(&vcount, 8) || !get(&is_open, 1) || !get(magic, 34) || std::memcmp(magic, kMagic, 34) != 0)
    return set_error(NWG_EINVAL, "not an NWGraph binary adjacency (magic missing)");
  if (!get(&nfield, 8) || !get(&noff, 8) || !get(&offsz, 8) || (offsz != 4 && offsz != 8))
    return set_error(NWG_EINVAL, "NWGraph binary: bad offset header");
  // n comes from the offsets count: N_ is not the vertex count (after
  // fill it holds N + 1), and with a 4-byte index_t only its low 4 bytes
  // are N_ at all (the other 4 are whatever followed N_ in memory).
  const uint64_t n = noff - 1;
  if (noff < 2 || n >= 0xFFFFFFFFull || vcount != n)
    return set_error(NWG_EINVAL, "NWGraph binary: offsets count does not match the vertex count");
  (void)nfield;
  out.n = n;
  out.off.resize(noff);
  if (offsz == 8) {
    if (!get(out.off.data(), noff * 8)) return set_error(NWG_EINVAL, "NWGraph binary: truncated offsets");
  } else {
    std::vector<uint32_t> o32(noff);
    if (!get(o32.data(), noff * 4)) return set_error(NWG_EINVAL, "NWGraph binary: truncated offsets");
    std::copy(o32.begin(), o32.end(), out.off.begin());
  }
  if (!get(&m, 8) || !get(&narrays, 8) || narrays == 0) return set_error(NWG_EINVAL, "NWGraph binary: bad array header");
  uint64_t cnt = 0, elsz = 0;
  if (!get(&cnt, 8) || !get(&elsz, 8) || cnt != m || elsz != 4)
    return set_error(NWG_EINVAL, "NWGraph binary: target ids must be one array of M 4-byte ids");
  out.col.resize(m);
  if (!get(out.col.data(), m * 4)) return set_error(NWG_EINVAL, "NWGraph binary: truncated target ids");
  if (out.off[0] != 0 || out.off[n] != m) return set_error(NWG_EINVAL, "NWGraph binary: offsets do not span M entries");
  for (uint64_t i = 0; i < n; ++i)
    if (out.off[i + 1] < out.off[i]) return set_error(NWG_EINVAL, "NWGraph binary: offsets not monotone");
  for (uint32_t c : out.col)
    if (c >= n) return set_error(NWG_EINVAL, "NWGraph binary: target id >= N");
  (void)is_open;
  return NWG_OK;
}

void transpose(const Csr& a, Csr& t) {
  std::vector<uint32_t> src(a.col.size()), dst(a.col.size());
  for (uint64_t u = 0; u < a.n; ++u)
    for (uint64_t e = a.off[u]; e < a.off[u + 1]; ++e) {
      src[e] = a.col[e];
      dst[e] = (uint32_t)u;
    }
  build_rows(a.n, src, dst, t);
}

}  // namespace

NWG_API int nwg_graph_read(const char* path, uint32_t flags, nwg_graph* out) {
  try {
    if (!path || !out) return set_error(NWG_EINVAL, "NULL path or out handle pointer");
    *out = nullptr;
    std::string data;
    if (!read_file(path, data)) return set_error(NWG_EINVAL, std::string("cannot read ") + path);
    Csr  g, gt;
    bool symmetric = (flags & NWG_READ_SYMMETRIC) != 0;
    if (data.compare(0, 14, "%%MatrixMarket") == 0) {
      std::vector<uint32_t> src, dst;
      uint64_t              n = 0;
      bool                  file_sym = false;
      int                   rc = parse_mm(data, src, dst, n, file_sym);
      if (rc) return rc;
      data.clear();
      data.shrink_to_fit();
      build_rows(n, src, dst, g);
      if (file_sym) symmetric = true;  // both directions of every entry are present
      else if (!symmetric) build_rows(n, dst, src, gt);
    } else {
      int rc = parse_nwbin(data, g);
      if (rc) return rc;
      data.clear();
      data.shrink_to_fit();
      for (uint64_t v = 0; v < g.n; ++v) std::sort(g.col.begin() + g.off[v], g.col.begin() + g.off[v + 1]);
      if (!symmetric) transpose(g, gt);
    }
    return nwg_graph_register(g.off.data(), g.col.data(), g.n, symmetric ? nullptr : gt.off.data(),
                              symmetric ? nullptr : gt.col.data(), 0u, out);
  } catch (const std::bad_alloc&) {
    return set_error(NWG_ENOMEM, "host allocation failed while reading a graph file");
  }
}

NWG_API int nwg_graph_write_nwbin(nwg_graph h, const char* path) {
  try {
    if (!h || !path) return set_error(NWG_EINVAL, "NULL graph or path");
    uint64_t n = 0, m = 0, in_m = 0;
    int      rc = nwg_graph_info(h, &n, &m, &in_m);
    if (rc) return rc;
    std::vector<uint64_t> off(n + 1);
    std::vector<uint32_t> col(std::max<uint64_t>(m, 1));
    rc = nwg_graph_copy_csr(h, off.data(), col.data(), nullptr, nullptr);
    if (rc) return rc;
    FILE* f = std::fopen(path, "wb");
    if (!f) return set_error(NWG_EINVAL, std::string("cannot write ") + path);
    static const char kMagic[34] = "NW GRAPH indexed_struct_of_arrays";
    const uint8_t     is_open    = 0;
    const uint64_t    noff = n + 1, offsz = 8, narrays = 1, elsz = 4;
    bool              ok = std::fwrite(&n, 8, 1, f) == 1 && std::fwrite(&is_open, 1, 1, f) == 1 &&
              std::fwrite(kMagic, 34, 1, f) == 1 && std::fwrite(&n, 8, 1, f) == 1 && std::fwrite(&noff, 8, 1, f) == 1 &&
              std::fwrite(&offsz, 8, 1, f) == 1 && std::fwrite(off.data(), 8, noff, f) == noff &&
              std::fwrite(&m, 8, 1, f) == 1 && std::fwrite(&narrays, 8, 1, f) == 1 && std::fwrite(&m, 8, 1, f) == 1 &&
              std::fwrite(&elsz, 8, 1, f) == 1 && (m == 0 || std::fwrite(col.data(), 4, m, f) == m);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return set_error(NWG_EINVAL, std::string("write failed: ") + path);
    return NWG_OK;
  } catch (const std::bad_alloc&) {
    return set_error(NWG_ENOMEM, "host allocation failed while writing a graph file");
  }
}
