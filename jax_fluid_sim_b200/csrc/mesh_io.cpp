// Mesh ingestion on the host cores: the face pairing of the hybrid mesh and the numeric sections
// of Gmsh's ASCII mesh files.
//
// Face pairing (hybrid/mesh.py:378-459 walks every (block, cell, local face) in order and pairs
// equal sorted corner keys through a dictionary): here the visits are sorted by (key, visit)
// with a parallel merge sort, equal keys form a group, and the faces come out in the reference's
// order (internal faces in the order of their second visit, then boundary faces in the order of
// their first).  (key, visit) is a total order because visits are distinct, so the result does
// not depend on the sort algorithm or on the thread count.
//
// Gmsh ASCII sections (the reference reads them with meshio, hybrid/mesh.py:182-236): the node
// and element records of MSH 2.2 and 4.1, parsed with std::from_chars.  The layout follows the
// Gmsh reference manual: MSH 2.2 nodes "id x y z", elements "id type ntags tags... nodes...";
// MSH 4.1 entity blocks "dim tag parametric count" with the node tags, then the coordinates,
// and element blocks "dim tag type count" with lines "id nodes...".

#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "dgb200.h"

namespace dgb {
int set_error(int code, const char* msg);   // defined with the plan code
}

namespace {

// Sorts idx with less: sorted chunks in threads, then pairwise merges (also in threads).
template <typename Less>
void parallel_sort(std::vector<int64_t>& idx, Less less) {
  const int64_t n = (int64_t)idx.size();
  const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const int64_t want = std::min<int64_t>(hw, std::max<int64_t>(1, n / 65536));
  int chunks = 1;
  while (chunks * 2 <= want) chunks *= 2;
  std::vector<int64_t> bound(chunks + 1);
  for (int c = 0; c <= chunks; ++c) bound[c] = n * c / chunks;
  auto it = idx.begin();
  if (chunks == 1) {
    std::sort(it, idx.end(), less);
    return;
  }
  {
    std::vector<std::thread> pool;
    for (int c = 0; c < chunks; ++c)
      pool.emplace_back([&, c] { std::sort(it + bound[c], it + bound[c + 1], less); });
    for (auto& t : pool) t.join();
  }
  for (int width = 1; width < chunks; width *= 2) {
    std::vector<std::thread> pool;
    for (int c = 0; c + width < chunks; c += 2 * width) {
      const int hi = std::min(c + 2 * width, chunks);
      pool.emplace_back([&, c, width, hi] { std::inplace_merge(it + bound[c], it + bound[c + width], it + bound[hi], less); });
    }
    for (auto& t : pool) t.join();
  }
}

// A forward cursor over a text buffer.
struct Cursor {
  const char* p;
  const char* end;
  void skip_space() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) ++p;
  }
  // spaces and tabs only: stops at the end of the line
  void skip_blank() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  }
  bool at_eol() {
    skip_blank();
    return p >= end || *p == '\n';
  }
  void next_line() {
    while (p < end && *p != '\n') ++p;
    if (p < end) ++p;
  }
  bool integer(int64_t& v) {
    skip_space();
    if (p < end && *p == '+') ++p;
    const auto r = std::from_chars(p, end, v);
    if (r.ec != std::errc()) return false;
    p = r.ptr;
    return true;
  }
  bool real(double& v) {
    skip_space();
    if (p < end && *p == '+') ++p;
    const auto r = std::from_chars(p, end, v);
    if (r.ec != std::errc()) return false;
    p = r.ptr;
    return true;
  }
};

int parse_error(const char* what, int64_t record) {
  const std::string msg = std::string("malformed Gmsh ") + what + " record " + std::to_string(record);
  return dgb::set_error(DGB_ERR_ARGUMENT, msg.c_str());
}

// The rest of the current line as node ids (an element record's node list).
int node_list(Cursor& c, int64_t rec, int64_t* nodes, int64_t cap, int64_t& used) {
  while (!c.at_eol()) {
    int64_t v;
    if (!c.integer(v)) return parse_error("element", rec);
    if (used >= cap) return dgb::set_error(DGB_ERR_ARGUMENT, "Gmsh element node lists exceed the buffer");
    nodes[used++] = v;
  }
  c.next_line();
  return DGB_OK;
}

}  // namespace

extern "C" int dgb_pair_faces(const int64_t* keys, int k, int64_t n, const int64_t* visit, int64_t* owner,
                              int64_t* neighbor, int64_t* count) {
  if (n < 0 || k < 1 || k > 8 || !count || (n > 0 && (!keys || !visit || !owner || !neighbor)))
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad face-pairing argument");
  std::vector<int64_t> idx(n);
  std::iota(idx.begin(), idx.end(), int64_t(0));
  auto same = [=](int64_t a, int64_t b) {
    return std::memcmp(keys + a * k, keys + b * k, sizeof(int64_t) * k) == 0;
  };
  parallel_sort(idx, [=](int64_t a, int64_t b) {
    const int64_t* ka = keys + a * k;
    const int64_t* kb = keys + b * k;
    for (int j = 0; j < k; ++j)
      if (ka[j] != kb[j]) return ka[j] < kb[j];
    return visit[a] < visit[b];
  });
  std::vector<int64_t> inner, outer;     // internal faces as (second, first); boundary faces as first
  for (int64_t i = 0; i < n;) {
    int64_t j = i + 1;
    while (j < n && same(idx[i], idx[j])) ++j;
    if (j - i > 2) return dgb::set_error(DGB_ERR_ARGUMENT, "A face is shared by more than two cells");
    if (j - i == 2) {
      inner.push_back(idx[i + 1]);
      inner.push_back(idx[i]);
    } else {
      outer.push_back(idx[i]);
    }
    i = j;
  }
  const int64_t ni = (int64_t)inner.size() / 2;
  std::vector<int64_t> order(ni);
  std::iota(order.begin(), order.end(), int64_t(0));
  std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return visit[inner[2 * a]] < visit[inner[2 * b]]; });
  for (int64_t f = 0; f < ni; ++f) {
    owner[f] = inner[2 * order[f] + 1];
    neighbor[f] = inner[2 * order[f]];
  }
  std::sort(outer.begin(), outer.end(), [&](int64_t a, int64_t b) { return visit[a] < visit[b]; });
  for (size_t f = 0; f < outer.size(); ++f) {
    owner[ni + f] = outer[f];
    neighbor[ni + f] = -1;
  }
  *count = ni + (int64_t)outer.size();
  return DGB_OK;
}

extern "C" int dgb_msh2_nodes(const char* text, int64_t len, int64_t n, int64_t* ids, double* xyz) {
  if (!text || len < 0 || n < 0 || (n > 0 && (!ids || !xyz)))
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad Gmsh node-section argument");
  Cursor c{text, text + len};
  for (int64_t i = 0; i < n; ++i) {
    if (!c.integer(ids[i]) || !c.real(xyz[3 * i]) || !c.real(xyz[3 * i + 1]) || !c.real(xyz[3 * i + 2]))
      return parse_error("node", i);
    c.next_line();
  }
  return DGB_OK;
}

extern "C" int dgb_msh2_elements(const char* text, int64_t len, int64_t n, int32_t* type, int32_t* phys,
                                 int64_t* offsets, int64_t* nodes, int64_t cap) {
  if (!text || len < 0 || n < 0 || !offsets || (n > 0 && (!type || !phys)) || (cap > 0 && !nodes))
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad Gmsh element-section argument");
  Cursor c{text, text + len};
  int64_t used = 0;
  offsets[0] = 0;
  for (int64_t i = 0; i < n; ++i) {
    int64_t id, t, ntags, tag = 0;
    if (!c.integer(id) || !c.integer(t) || !c.integer(ntags) || ntags < 0) return parse_error("element", i);
    for (int64_t g = 0; g < ntags; ++g) {
      int64_t v;
      if (!c.integer(v)) return parse_error("element", i);
      if (g == 0) tag = v;                 // the physical tag comes first
    }
    type[i] = (int32_t)t;
    phys[i] = (int32_t)tag;
    int rc;
    if ((rc = node_list(c, i, nodes, cap, used))) return rc;
    offsets[i + 1] = used;
  }
  return DGB_OK;
}

extern "C" int dgb_msh4_nodes(const char* text, int64_t len, int64_t n, int64_t* ids, double* xyz) {
  if (!text || len < 0 || n < 0 || (n > 0 && (!ids || !xyz)))
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad Gmsh node-section argument");
  Cursor c{text, text + len};
  int64_t blocks, total, lo, hi;
  if (!c.integer(blocks) || !c.integer(total) || !c.integer(lo) || !c.integer(hi) || blocks < 0)
    return parse_error("node-section header", 0);
  if (total != n) return dgb::set_error(DGB_ERR_ARGUMENT, "Gmsh node count differs from the section header");
  int64_t row = 0;
  for (int64_t b = 0; b < blocks; ++b) {
    int64_t dim, tag, parametric, count;
    if (!c.integer(dim) || !c.integer(tag) || !c.integer(parametric) || !c.integer(count) || count < 0 ||
        row + count > n)
      return parse_error("node block", b);
    for (int64_t k = 0; k < count; ++k)
      if (!c.integer(ids[row + k])) return parse_error("node", row + k);
    c.next_line();
    for (int64_t k = 0; k < count; ++k) {
      double* x = xyz + 3 * (row + k);
      if (!c.real(x[0]) || !c.real(x[1]) || !c.real(x[2])) return parse_error("node", row + k);
      c.next_line();                      // parametric coordinates, if any, are not kept
    }
    row += count;
  }
  if (row != n) return dgb::set_error(DGB_ERR_ARGUMENT, "Gmsh node blocks do not add up to the section header");
  return DGB_OK;
}

extern "C" int dgb_msh4_elements(const char* text, int64_t len, int64_t n, int32_t* type, int32_t* entity_dim,
                                 int32_t* entity_tag, int64_t* offsets, int64_t* nodes, int64_t cap) {
  if (!text || len < 0 || n < 0 || !offsets || (n > 0 && (!type || !entity_dim || !entity_tag)) ||
      (cap > 0 && !nodes))
    return dgb::set_error(DGB_ERR_ARGUMENT, "bad Gmsh element-section argument");
  Cursor c{text, text + len};
  int64_t blocks, total, lo, hi;
  if (!c.integer(blocks) || !c.integer(total) || !c.integer(lo) || !c.integer(hi) || blocks < 0)
    return parse_error("element-section header", 0);
  if (total != n) return dgb::set_error(DGB_ERR_ARGUMENT, "Gmsh element count differs from the section header");
  c.next_line();
  int64_t row = 0, used = 0;
  offsets[0] = 0;
  for (int64_t b = 0; b < blocks; ++b) {
    int64_t dim, tag, t, count;
    if (!c.integer(dim) || !c.integer(tag) || !c.integer(t) || !c.integer(count) || count < 0 || row + count > n)
      return parse_error("element block", b);
    c.next_line();
    for (int64_t k = 0; k < count; ++k) {
      int64_t id;
      if (!c.integer(id)) return parse_error("element", row + k);
      type[row + k] = (int32_t)t;
      entity_dim[row + k] = (int32_t)dim;
      entity_tag[row + k] = (int32_t)tag;
      int rc;
      if ((rc = node_list(c, row + k, nodes, cap, used))) return rc;
      offsets[row + k + 1] = used;
    }
    row += count;
  }
  if (row != n) return dgb::set_error(DGB_ERR_ARGUMENT, "Gmsh element blocks do not add up to the section header");
  return DGB_OK;
}
