// Host preparation, restated from the reference's ingest / canonicalize /
// graph / compress / JLA-plan stages.  Orderings, tie rules, compensated sums
// and error classes follow the cited reference functions so that retained
// masks, dimensions, checksums and semantic ranks are bit-identical.
#include "prep.h"

#include "radix.h"

#include <algorithm>
#include <omp.h>
#include <atomic>
#include <parallel/algorithm>
#include <functional>
#include <exception>
#include <thread>
#include <cstring>
#include <numeric>

namespace fevcb {

namespace {

constexpr uint32_t MISSING = 0xffffffffu;

// Stable sort of a large index range on all host cores (multiway merge sort,
// OpenMP); a stable sort's output is unique, so it equals std::stable_sort's.
template <class It, class Cmp>
void sort_rows(It first, It last, Cmp cmp) {
  if (last - first >= (1 << 16))
    __gnu_parallel::stable_sort(first, last, cmp);
  else
    std::stable_sort(first, last, cmp);
}

std::vector<uint64_t> copy_integer(const double* p, uint64_t rows, const char* label, int32_t code) {
  if (!p) fail(INVALID_INPUT, "engine_ingest", std::string(label) + " pointer is null");
  if (reinterpret_cast<uintptr_t>(p) % alignof(double))
    fail(INVALID_INPUT, "engine_ingest", std::string(label) + " pointer is not aligned for binary64 values");
  std::vector<uint64_t> out(rows);
  for (uint64_t r = 0; r < rows; ++r) {
    double v = p[r];
    if (!std::isfinite(v) || !(v > 0.0 && v <= double(MAX_EXACT_BINARY64_INTEGER)) || std::trunc(v) != v)
      fail(code, "engine_ingest",
           std::string(label) + " must be a positive exact binary64 integer at zero-based row " + std::to_string(r));
    out[r] = uint64_t(v);
  }
  return out;
}

std::vector<double> copy_finite(const double* p, uint64_t rows, const char* label) {
  if (!p) fail(INVALID_INPUT, "engine_ingest", std::string(label) + " pointer is null");
  if (reinterpret_cast<uintptr_t>(p) % alignof(double))
    fail(INVALID_INPUT, "engine_ingest", std::string(label) + " pointer is not aligned for binary64 values");
  std::vector<double> out(p, p + rows);
  for (uint64_t r = 0; r < rows; ++r)
    if (!std::isfinite(out[r]))
      fail(INVALID_INPUT, "engine_ingest", std::string(label) + " is nonfinite at zero-based row " + std::to_string(r));
  return out;
}

// Reference `redense` (problem.rs:696-745): sorted distinct levels, dense ids
// (a level's id is its rank among the distinct values).  Identifiers that span
// a range no wider than a few times the row count are relabelled through a
// presence table over the range; wider ones are radix sorted.
std::vector<uint32_t> redense(const std::vector<uint64_t>& values, std::vector<uint64_t>& levels, const char* label) {
  size_t n = values.size();
  if (n > 0xffffffffull) fail(RESOURCE_LIMIT, "canonicalize", "row count exceeds the u32 implementation limit");
  levels.clear();
  std::vector<uint32_t> dense(n);
  if (n == 0) return dense;
  uint64_t lo = values[0], hi = values[0];
  for (uint64_t v : values) {
    lo = std::min(lo, v);
    hi = std::max(hi, v);
  }
  if (hi - lo < 4 * uint64_t(n) + 1024) {
    std::vector<uint32_t> id(size_t(hi - lo) + 1, MISSING);
    for (uint64_t v : values) id[v - lo] = 0;
    for (size_t k = 0; k < id.size(); ++k)
      if (id[k] != MISSING) {
        id[k] = uint32_t(levels.size());
        levels.push_back(lo + k);
      }
    for (size_t i = 0; i < n; ++i) dense[i] = id[values[i] - lo];
  } else {
    std::vector<uint64_t> key(values);
    std::vector<uint32_t> row(n);
    std::iota(row.begin(), row.end(), 0u);
    radix_sort_pairs(key, row);
    for (size_t i = 0; i < n; ++i) {
      if (i == 0 || key[i] != key[i - 1]) levels.push_back(key[i]);
      dense[row[i]] = uint32_t(levels.size() - 1);
    }
  }
  if (levels.size() > 0xffffffffull)
    fail(RESOURCE_LIMIT, "canonicalize", std::string(label) + " cardinality exceeds the u32 implementation limit");
  return dense;
}

void hash_word(uint64_t& h, uint64_t v) {
  for (int b = 0; b < 8; ++b) {
    h ^= (v >> (8 * b)) & 0xff;
    h *= 0x00000100000001b3ull;
  }
}

// Reference `topology_checksum` (problem.rs:1213-1248): FNV-1a over the sorted
// (worker, firm, deletion, frequency) records, each word little-endian.  A
// deletion unit lies in one (worker, firm) coordinate, so the record order is
// the units ordered by (worker, firm, unit) with each unit's rows ordered by
// frequency; the units are radix sorted and the rows bucketed by unit.  When
// the inputs break that property the records are sorted directly.
uint64_t topology_checksum(const std::vector<uint32_t>& w, const std::vector<uint32_t>& f,
                           const std::vector<uint32_t>& d, const std::vector<uint64_t>& q) {
  size_t n = w.size();
  uint64_t h = 0xcbf29ce484222325ull;
  auto record = [&](size_t i) {
    hash_word(h, w[i]);
    hash_word(h, f[i]);
    hash_word(h, d[i]);
    hash_word(h, q[i]);
  };
  uint32_t units = 0;
  for (uint32_t x : d) units = std::max(units, x + 1);
  std::vector<uint32_t> uw(units, MISSING), uf(units, MISSING);
  bool functional = true;
  for (size_t i = 0; i < n && functional; ++i) {
    uint32_t u = d[i];
    if (uw[u] == MISSING) {
      uw[u] = w[i];
      uf[u] = f[i];
    } else if (uw[u] != w[i] || uf[u] != f[i]) {
      functional = false;
    }
  }
  if (!functional) {
    std::vector<size_t> order(n);
    std::iota(order.begin(), order.end(), size_t(0));
    sort_rows(order.begin(), order.end(), [&](size_t a, size_t b) {
      if (w[a] != w[b]) return w[a] < w[b];
      if (f[a] != f[b]) return f[a] < f[b];
      if (d[a] != d[b]) return d[a] < d[b];
      return q[a] < q[b];
    });
    for (size_t i : order) record(i);
    return h;
  }
  // units present, in (worker, firm, unit) order (LSD radix keeps unit order on ties)
  std::vector<uint64_t> ukey;
  std::vector<uint32_t> uid;
  for (uint32_t u = 0; u < units; ++u)
    if (uw[u] != MISSING) {
      ukey.push_back((uint64_t(uw[u]) << 32) | uf[u]);
      uid.push_back(u);
    }
  radix_sort_pairs(ukey, uid);
  // rows bucketed by unit
  std::vector<uint64_t> ptr(size_t(units) + 1, 0);
  for (uint32_t x : d) ptr[x + 1]++;
  for (uint32_t u = 0; u < units; ++u) ptr[u + 1] += ptr[u];
  std::vector<uint32_t> rows(n);
  {
    std::vector<uint64_t> cur(ptr.begin(), ptr.end() - 1);
    for (size_t i = 0; i < n; ++i) rows[cur[d[i]]++] = uint32_t(i);
  }
  for (uint32_t u : uid) {
    auto b = rows.begin() + ptr[u], e = rows.begin() + ptr[u + 1];
    if (e - b > 1) std::sort(b, e, [&](uint32_t a, uint32_t c) { return q[a] < q[c]; });
    for (auto it = b; it != e; ++it) record(*it);
  }
  return h;
}

size_t count_true(const std::vector<uint8_t>& m) {
  size_t c = 0;
  for (uint8_t v : m) c += v;
  return c;
}

// Indices of the true entries in increasing order (chunks counted and filled
// on all host cores).
std::vector<uint64_t> active_indices(const std::vector<uint8_t>& m) {
  const size_t n = m.size();
  const int threads = n >= (size_t(1) << 20) ? std::max(1, omp_get_max_threads()) : 1;
  std::vector<size_t> count(size_t(threads) + 1, 0);
  std::vector<uint64_t> out;
#pragma omp parallel num_threads(threads)
  {
    const int t = omp_get_thread_num();
    const size_t b = n * t / threads, e = n * (t + 1) / threads;
    size_t c = 0;
    for (size_t i = b; i < e; ++i) c += m[i] != 0;
    count[t + 1] = c;
#pragma omp barrier
#pragma omp single
    {
      for (int u = 0; u < threads; ++u) count[u + 1] += count[u];
      out.resize(count[threads]);
    }
    size_t at = count[t];
    for (size_t i = b; i < e; ++i)
      if (m[i]) out[at++] = i;
  }
  return out;
}

// Bipartite graph with workers 0..W-1 and firms W..W+F-1 in CSR form; an arc
// holds its head and its undirected edge id together (one cache line per
// visit in the traversals).
struct Arc {
  uint32_t to, edge;
};
struct Graph {
  size_t nodes = 0, edges = 0;
  std::vector<uint64_t> ptr;
  std::vector<Arc> arc;
};

Graph make_graph(size_t nodes, const std::vector<uint32_t>& eu, const std::vector<uint32_t>& ev) {
  Graph g;
  g.nodes = nodes;
  g.edges = eu.size();
  g.ptr.assign(nodes + 1, 0);
  for (size_t e = 0; e < eu.size(); ++e) {
    g.ptr[eu[e] + 1]++;
    g.ptr[ev[e] + 1]++;
  }
  for (size_t v = 0; v < nodes; ++v) g.ptr[v + 1] += g.ptr[v];
  g.arc.resize(2 * eu.size());
  std::vector<uint64_t> cur(g.ptr.begin(), g.ptr.end() - 1);
  for (size_t e = 0; e < eu.size(); ++e) {
    g.arc[cur[eu[e]]++] = Arc{ev[e], uint32_t(e)};
    g.arc[cur[ev[e]]++] = Arc{eu[e], uint32_t(e)};
  }
  return g;
}

void validate_mask(const Canonical& in, const std::vector<uint8_t>& active) {
  if (active.size() != in.rows()) fail(INVALID_INPUT, "graph", "active mask has the wrong length");
  if (count_true(active) == 0) fail(GRAPH_EMPTY, "graph", "active graph is empty");
}

// Reference `coordinate_graph` (graph.rs:707-760): distinct active (worker,
// firm) pairs, in (worker, firm) order.  The distinct pairs of all rows are
// indexed once at canonicalisation (Canonical::coord), so a mask selects its
// edges with one pass over the rows.
Graph coordinate_graph(const Canonical& in, const std::vector<uint8_t>& active) {
  validate_mask(in, active);
  std::vector<uint8_t> used(in.coord_worker.size(), 0);
  for (size_t r = 0; r < in.rows(); ++r)
    if (active[r]) used[in.coord[r]] = 1;
  std::vector<uint32_t> eu, ev;
  for (size_t c = 0; c < used.size(); ++c)
    if (used[c]) {
      eu.push_back(in.coord_worker[c]);
      ev.push_back(uint32_t(in.workers + in.coord_firm[c]));
    }
  return make_graph(in.workers + in.firms, eu, ev);
}

struct ComponentResult {
  std::vector<uint8_t> keep;
  size_t components = 0, retained_rows = 0;
};

// Reference `largest_component` (graph.rs:619-705): rank components by
// (firm count, physical mass); a tie for the maximum is an identification error.
ComponentResult largest_component(const Canonical& in, const std::vector<uint8_t>& active) {
  Graph g = coordinate_graph(in, active);
  std::vector<uint32_t> label(g.nodes, MISSING);
  std::vector<uint32_t> queue;
  queue.reserve(g.nodes);
  size_t comps = 0;
  for (size_t root = 0; root < g.nodes; ++root) {
    if (g.ptr[root] == g.ptr[root + 1] || label[root] != MISSING) continue;
    label[root] = uint32_t(comps);
    queue.clear();
    queue.push_back(uint32_t(root));
    for (size_t h = 0; h < queue.size(); ++h) {
      uint32_t v = queue[h];
      for (uint64_t a = g.ptr[v]; a < g.ptr[v + 1]; ++a) {
        uint32_t u = g.arc[a].to;
        if (label[u] == MISSING) {
          label[u] = uint32_t(comps);
          queue.push_back(u);
        }
      }
    }
    ++comps;
  }
  if (comps == 0) fail(GRAPH_EMPTY, "graph", "no connected worker-firm component remains");
  std::vector<uint64_t> firms(comps, 0), mass(comps, 0);
  for (size_t f = 0; f < in.firms; ++f) {
    uint32_t c = label[in.workers + f];
    if (c != MISSING) firms[c]++;
  }
  for (size_t r = 0; r < in.rows(); ++r) {
    if (!active[r]) continue;
    uint32_t c = label[in.worker[r]];
    if (c == MISSING) fail(INTERNAL_INVARIANT_FAILED, "graph", "active row has no connected-component label");
    mass[c] += in.frequency[r];
  }
  size_t best = 0;
  for (size_t c = 1; c < comps; ++c)
    if (firms[c] > firms[best] || (firms[c] == firms[best] && mass[c] > mass[best])) best = c;
  size_t winners = 0;
  for (size_t c = 0; c < comps; ++c) winners += (firms[c] == firms[best] && mass[c] == mass[best]);
  if (winners != 1)
    fail(GRAPH_UNIDENTIFIED, "graph", "multiple connected components tie for largest-component selection");
  ComponentResult out;
  out.components = comps;
  out.keep.resize(in.rows());
  for (size_t r = 0; r < in.rows(); ++r) {
    out.keep[r] = active[r] && label[in.worker[r]] == best;
    out.retained_rows += out.keep[r];
  }
  return out;
}

// Iterative Tarjan low-link over a CSR multigraph.  The parent arc is skipped
// by edge identity (not by endpoint), so parallel edges count as cycles.
// Articulation vertices and bridges are properties of the graph, independent
// of the traversal order (reference `articulation_vertices` graph.rs:872-936
// and `bridge_edges` graph.rs:1031-1088).
// edge_on: optional per-edge mask; masked-off edges are absent and a vertex
// with no edge left is not part of the graph.
void tarjan(const Graph& g, std::vector<uint8_t>* articulation, std::vector<uint8_t>* bridge,
            const std::vector<uint8_t>* edge_on = nullptr) {
  // per-vertex DFS state in one record (discovery time, low link, parent,
  // parent edge, next arc): a visit touches one cache line
  struct Node {
    uint32_t disc = 0, low = 0, parent = MISSING, parent_edge = MISSING;
    uint64_t next = 0;
  };
  const size_t n = g.nodes;
  if (n >= MISSING) fail(RESOURCE_LIMIT, "graph", "graph has too many vertices");
  std::vector<Node> st(n);
  if (articulation) articulation->assign(n, 0);
  if (bridge) bridge->assign(g.edges, 0);
  uint32_t clock = 0;
  std::vector<uint32_t> stack;
  for (size_t root = 0; root < n; ++root) {
    if (st[root].disc) continue;
    bool has_edge = false;
    for (uint64_t a = g.ptr[root]; a < g.ptr[root + 1] && !has_edge; ++a)
      has_edge = !edge_on || (*edge_on)[g.arc[a].edge];
    if (!has_edge) continue;
    st[root].disc = st[root].low = ++clock;
    st[root].next = g.ptr[root];
    uint32_t root_children = 0;
    stack.clear();
    stack.push_back(uint32_t(root));
    while (!stack.empty()) {
      uint32_t v = stack.back();
      Node& sv = st[v];
      if (sv.next < g.ptr[v + 1]) {
        const Arc arc = g.arc[sv.next++];
        if (arc.edge == sv.parent_edge || (edge_on && !(*edge_on)[arc.edge])) continue;
        Node& su = st[arc.to];
        if (!su.disc) {
          su.parent = v;
          su.parent_edge = arc.edge;
          root_children += v == root;
          su.disc = su.low = ++clock;
          su.next = g.ptr[arc.to];
          stack.push_back(arc.to);
        } else {
          sv.low = std::min(sv.low, su.disc);
        }
      } else {
        stack.pop_back();
        uint32_t p = sv.parent;
        if (p != MISSING) {
          Node& sp = st[p];
          if (bridge && sv.low > sp.disc) (*bridge)[sv.parent_edge] = 1;
          sp.low = std::min(sp.low, sv.low);
          if (articulation && sp.parent != MISSING && sv.low >= sp.disc) (*articulation)[p] = 1;
        }
      }
    }
    if (articulation) (*articulation)[root] = root_children > 1;
  }
}

// Run independent tasks on their own threads; after all finish the first
// exception in task order is rethrown (the error a sequential run reports).
void run_tasks(const std::vector<std::function<void()>>& tasks) {
  std::vector<std::exception_ptr> err(tasks.size());
  std::vector<std::thread> th;
  for (size_t i = 1; i < tasks.size(); ++i)
    th.emplace_back([&, i] {
      try {
        tasks[i]();
      } catch (...) {
        err[i] = std::current_exception();
      }
    });
  try {
    if (!tasks.empty()) tasks[0]();
  } catch (...) {
    err[0] = std::current_exception();
  }
  for (auto& t : th) t.join();
  for (auto& e : err)
    if (e) std::rethrow_exception(e);
}

// Run two independent tasks on two threads; the first exception (a's first)
// is rethrown after both finish.
template <class A, class B>
void run_side_by_side(A&& a, B&& b) {
  std::exception_ptr ea, eb;
  std::thread t([&] {
    try {
      b();
    } catch (...) {
      eb = std::current_exception();
    }
  });
  try {
    a();
  } catch (...) {
    ea = std::current_exception();
  }
  t.join();
  if (ea) std::rethrow_exception(ea);
  if (eb) std::rethrow_exception(eb);
}

// Deletion units of the canonical input (each lies in one worker-firm
// coordinate, which canonicalisation checked): worker, firm, coordinate, row
// count and physical mass.
struct UnitTable {
  std::vector<uint32_t> worker, firm, coord;
  std::vector<uint64_t> rows, mass;
};

UnitTable unit_table(const Canonical& in) {
  const size_t D = in.deletion_units;
  UnitTable u;
  u.worker.assign(D, MISSING);
  u.firm.assign(D, MISSING);
  u.coord.assign(D, MISSING);
  u.rows.assign(D, 0);
  u.mass.assign(D, 0);
  for (size_t r = 0; r < in.rows(); ++r) {
    uint32_t d = in.deletion[r];
    if (u.worker[d] == MISSING) {
      u.worker[d] = in.worker[r];
      u.firm[d] = in.firm[r];
      u.coord[d] = in.coord[r];
    }
    u.rows[d] += 1;
    u.mass[d] += in.frequency[r];
  }
  return u;
}

uint64_t active_rows(const UnitTable& u, const std::vector<uint8_t>& act) {
  uint64_t n = 0;
  for (size_t d = 0; d < act.size(); ++d)
    if (act[d]) n += u.rows[d];
  return n;
}

// The coordinate graph of all rows (edge id = coordinate) and the deletion
// multigraph of all units (edge id = unit), built once; the fixed point masks
// edges off instead of rebuilding (`coordinate_graph` of the active rows has
// exactly the coordinates of the active units).
struct UnitGraphs {
  Graph coords, units;
  std::vector<uint8_t> coord_on;
};

UnitGraphs unit_graphs(const Canonical& in, const UnitTable& u) {
  UnitGraphs g;
  std::vector<uint32_t> eu(in.coord_worker.size()), ev(in.coord_worker.size());
  for (size_t c = 0; c < eu.size(); ++c) {
    eu[c] = in.coord_worker[c];
    ev[c] = uint32_t(in.workers + in.coord_firm[c]);
  }
  g.coords = make_graph(in.workers + in.firms, eu, ev);
  eu.resize(u.worker.size());
  ev.resize(u.worker.size());
  for (size_t d = 0; d < u.worker.size(); ++d) {
    eu[d] = u.worker[d];
    ev[d] = uint32_t(in.workers + u.firm[d]);
  }
  g.units = make_graph(in.workers + in.firms, eu, ev);
  g.coord_on.assign(in.coord_worker.size(), 0);
  return g;
}

// coordinates with an active unit
void mark_coords(const UnitTable& u, const std::vector<uint8_t>& act, UnitGraphs& g) {
  std::fill(g.coord_on.begin(), g.coord_on.end(), 0);
  bool any = false;
  for (size_t d = 0; d < act.size(); ++d)
    if (act[d]) {
      g.coord_on[u.coord[d]] = 1;
      any = true;
    }
  if (!any) fail(GRAPH_EMPTY, "graph", "active graph is empty");
}

struct UnitComponents {
  std::vector<uint8_t> keep;  // per unit
  size_t components = 0;
  uint64_t retained_rows = 0;
};

// `largest_component` over the active units' rows: components by (firm count,
// physical mass), a tie for the maximum is an identification error.
UnitComponents unit_largest_component(const Canonical& in, const UnitTable& u, const std::vector<uint8_t>& act,
                                      UnitGraphs& gs) {
  mark_coords(u, act, gs);
  const Graph& g = gs.coords;
  const std::vector<uint8_t>& on = gs.coord_on;
  std::vector<uint32_t> label(g.nodes, MISSING), queue;
  queue.reserve(g.nodes);
  size_t comps = 0;
  for (size_t root = 0; root < g.nodes; ++root) {
    if (label[root] != MISSING) continue;
    bool has_edge = false;
    for (uint64_t a = g.ptr[root]; a < g.ptr[root + 1] && !has_edge; ++a) has_edge = on[g.arc[a].edge];
    if (!has_edge) continue;
    label[root] = uint32_t(comps);
    queue.clear();
    queue.push_back(uint32_t(root));
    for (size_t h = 0; h < queue.size(); ++h) {
      uint32_t v = queue[h];
      for (uint64_t a = g.ptr[v]; a < g.ptr[v + 1]; ++a)
        if (on[g.arc[a].edge] && label[g.arc[a].to] == MISSING) {
          label[g.arc[a].to] = uint32_t(comps);
          queue.push_back(g.arc[a].to);
        }
    }
    ++comps;
  }
  if (comps == 0) fail(GRAPH_EMPTY, "graph", "no connected worker-firm component remains");
  std::vector<uint64_t> firms(comps, 0), mass(comps, 0);
  for (size_t f = 0; f < in.firms; ++f) {
    uint32_t c = label[in.workers + f];
    if (c != MISSING) firms[c]++;
  }
  for (size_t d = 0; d < act.size(); ++d) {
    if (!act[d]) continue;
    uint32_t c = label[u.worker[d]];
    if (c == MISSING) fail(INTERNAL_INVARIANT_FAILED, "graph", "active row has no connected-component label");
    mass[c] += u.mass[d];
  }
  size_t best = 0;
  for (size_t c = 1; c < comps; ++c)
    if (firms[c] > firms[best] || (firms[c] == firms[best] && mass[c] > mass[best])) best = c;
  size_t winners = 0;
  for (size_t c = 0; c < comps; ++c) winners += (firms[c] == firms[best] && mass[c] == mass[best]);
  if (winners != 1)
    fail(GRAPH_UNIDENTIFIED, "graph", "multiple connected components tie for largest-component selection");
  UnitComponents out;
  out.components = comps;
  out.keep.resize(act.size());
  for (size_t d = 0; d < act.size(); ++d) {
    out.keep[d] = act[d] && label[u.worker[d]] == best;
    if (out.keep[d]) out.retained_rows += u.rows[d];
  }
  return out;
}

// `worker_articulations` of the active units' coordinate graph.
std::vector<uint8_t> unit_articulations(const Canonical& in, const UnitTable& u, const std::vector<uint8_t>& act,
                                        UnitGraphs& gs) {
  mark_coords(u, act, gs);
  std::vector<uint8_t> art;
  tarjan(gs.coords, &art, nullptr, &gs.coord_on);
  art.resize(in.workers);
  return art;
}

// `distinct_deletion_counts`: active units per worker.
std::vector<uint64_t> unit_counts(const Canonical& in, const UnitTable& u, const std::vector<uint8_t>& act) {
  std::vector<uint64_t> counts(in.workers, 0);
  for (size_t d = 0; d < act.size(); ++d)
    if (act[d]) counts[u.worker[d]]++;
  return counts;
}

// `deletion_bridges`: the active units as multigraph edges, bridges by id.
std::vector<uint32_t> unit_bridges(const std::vector<uint8_t>& act, const UnitGraphs& gs) {
  bool any = false;
  for (uint8_t a : act) any |= a != 0;
  if (!any) fail(GRAPH_EMPTY, "graph", "active graph is empty");
  std::vector<uint8_t> br;
  tarjan(gs.units, nullptr, &br, &act);
  std::vector<uint32_t> out;
  for (size_t d = 0; d < act.size(); ++d)
    if (act[d] && br[d]) out.push_back(uint32_t(d));
  return out;
}

GroupIndex grouped_rows(size_t groups, const std::vector<uint32_t>& row_group) {
  GroupIndex gi;
  gi.ptr.assign(groups + 1, 0);
  for (uint32_t g : row_group) {
    if (g >= groups) fail(INTERNAL_INVARIANT_FAILED, "compression", "row group exceeds group count");
    gi.ptr[g + 1]++;
  }
  for (size_t g = 0; g < groups; ++g) gi.ptr[g + 1] += gi.ptr[g];
  const size_t R = row_group.size();
  std::vector<uint64_t> cur(gi.ptr.begin(), gi.ptr.end() - 1);
  gi.items.resize(R);
  for (size_t r = 0; r < R; ++r) gi.items[cur[row_group[r]]++] = uint32_t(r);
  return gi;
}

GroupIndex grouped_from_order(size_t groups, const std::vector<uint32_t>& group_of, std::vector<uint32_t>&& order) {
  GroupIndex gi;
  gi.ptr.assign(groups + 1, 0);
  for (uint32_t it : order) gi.ptr[group_of[it] + 1]++;
  for (size_t g = 0; g < groups; ++g) gi.ptr[g + 1] += gi.ptr[g];
  gi.items = std::move(order);
  return gi;
}

}  // namespace

InputColumns copy_columns(uint64_t rows, const double* worker, const double* firm, const double* deletion,
                          const double* outcome, const double* frequency, const double* target,
                          const double* const* controls, uint32_t controls_count, const double* probe_order) {
  InputColumns c;
  c.controls.resize(controls_count);
  // every column is copied and checked on its own thread; the error reported
  // is the one of the first failing column in this order
  std::vector<std::function<void()>> tasks = {
      [&] { c.worker = copy_integer(worker, rows, "worker identifier", INVALID_IDENTIFIER); },
      [&] { c.firm = copy_integer(firm, rows, "firm identifier", INVALID_IDENTIFIER); },
      [&] { c.deletion = copy_integer(deletion, rows, "deletion identifier", INVALID_IDENTIFIER); },
      [&] { c.outcome = copy_finite(outcome, rows, "outcome"); },
      [&] { c.frequency = copy_integer(frequency, rows, "frequency weight", INVALID_WEIGHT); },
      [&] {
        if (!target) fail(INVALID_INPUT, "engine_ingest", "target weight pointer is null");
        c.target.assign(target, target + rows);
        for (uint64_t r = 0; r < rows; ++r)
          if (!std::isfinite(c.target[r]) || c.target[r] < 0.0)
            fail(INVALID_TARGET_WEIGHT, "engine_ingest",
                 "target weight is negative or nonfinite at zero-based row " + std::to_string(r));
      },
      [&] {
        if (controls_count == 0 && controls)
          fail(INVALID_INPUT, "engine_prepare", "zero controls require a null control-pointer array");
        if (controls_count > 0 && !controls)
          fail(INVALID_INPUT, "engine_prepare", "positive control count requires a control-pointer array");
      }};
  if (controls)
    for (uint32_t k = 0; k < controls_count; ++k)
      tasks.push_back([&, k] { c.controls[k] = copy_finite(controls[k], rows, "control"); });
  if (probe_order) tasks.push_back([&] { c.probe_order = copy_finite(probe_order, rows, "probe-order value"); });
  run_tasks(tasks);
  return c;
}

Canonical canonicalize(InputColumns&& in, bool implicit_match) {
  size_t n = in.worker.size();
  if (n == 0) fail(INVALID_INPUT, "ingest", "input sample is empty");
  if (in.firm.size() != n || in.deletion.size() != n || in.outcome.size() != n || in.frequency.size() != n ||
      in.target.size() != n)
    fail(INVALID_INPUT, "ingest", "input columns have inconsistent lengths");
  for (auto& c : in.controls)
    if (c.size() != n) fail(INVALID_INPUT, "ingest", "input columns have inconsistent lengths");
  uint64_t physical = 0;
  double target_total = 0.0;
  for (size_t r = 0; r < n; ++r) {
    if (!std::isfinite(in.outcome[r]))
      fail(INVALID_INPUT, "ingest", "outcome is nonfinite at zero-based row " + std::to_string(r));
    if (in.frequency[r] == 0) fail(INVALID_WEIGHT, "ingest", "frequency is zero at zero-based row " + std::to_string(r));
    if (!std::isfinite(in.target[r]) || in.target[r] < 0.0)
      fail(INVALID_TARGET_WEIGHT, "ingest", "target weight is invalid at zero-based row " + std::to_string(r));
    for (auto& c : in.controls)
      if (!std::isfinite(c[r])) fail(INVALID_INPUT, "ingest", "control is nonfinite at zero-based row " + std::to_string(r));
    physical += in.frequency[r];
    if (physical < in.frequency[r]) fail(RESOURCE_LIMIT, "ingest", "physical-frequency total overflow");
    if (physical > MAX_EXACT_BINARY64_INTEGER)
      fail(RESOURCE_LIMIT, "ingest", "literal physical-frequency total exceeds the exact binary64 integer range");
    target_total += in.target[r];
  }
  if (!std::isfinite(target_total) || target_total <= 0.0)
    fail(INVALID_TARGET_WEIGHT, "ingest", "target weights must have positive finite total mass");

  Canonical c;
  std::vector<uint64_t> wl, fl, dl;
  // the three identifier columns are relabelled side by side (the implicit
  // match keys need the dense worker and firm ids first)
  std::vector<std::function<void()>> tasks = {[&] { c.worker = redense(in.worker, wl, "worker"); },
                                              [&] { c.firm = redense(in.firm, fl, "firm"); }};
  if (!implicit_match) tasks.push_back([&] { c.deletion = redense(in.deletion, dl, "deletion"); });
  run_tasks(tasks);
  c.workers = wl.size();
  c.firms = fl.size();
  if (implicit_match) {
    std::vector<uint64_t> keys(n);
    for (size_t r = 0; r < n; ++r) keys[r] = uint64_t(c.worker[r]) * c.firms + c.firm[r] + 1;
    c.deletion = redense(keys, dl, "deletion");
  }
  c.deletion_units = dl.size();
  {
    std::vector<uint32_t> cw(c.deletion_units, MISSING), cf(c.deletion_units, MISSING);
    for (size_t r = 0; r < n; ++r) {
      uint32_t d = c.deletion[r];
      if (cw[d] == MISSING) {
        cw[d] = c.worker[r];
        cf[d] = c.firm[r];
      } else if (cw[d] != c.worker[r] || cf[d] != c.firm[r]) {
        fail(INVALID_IDENTIFIER, "canonicalize", "each deletion identifier must stay within one worker-firm coordinate");
      }
    }
  }
  {
    // distinct (worker, firm) coordinates in (worker, firm) order: rows
    // bucketed by worker, each worker's rows ordered by firm
    std::vector<uint64_t> ptr(c.workers + 1, 0);
    for (uint32_t w : c.worker) ptr[w + 1]++;
    for (size_t w = 0; w < c.workers; ++w) ptr[w + 1] += ptr[w];
    std::vector<uint32_t> rows(n);
    {
      std::vector<uint64_t> cur(ptr.begin(), ptr.end() - 1);
      for (size_t r = 0; r < n; ++r) rows[cur[c.worker[r]]++] = uint32_t(r);
    }
    c.coord.resize(n);
    c.coord_worker.reserve(n);
    c.coord_firm.reserve(n);
    for (size_t w = 0; w < c.workers; ++w) {
      auto b = rows.begin() + ptr[w], e = rows.begin() + ptr[w + 1];
      if (e - b > 1) std::sort(b, e, [&](uint32_t x, uint32_t y) { return c.firm[x] < c.firm[y]; });
      uint32_t last = MISSING;
      for (auto it = b; it != e; ++it) {
        uint32_t f = c.firm[*it];
        if (f != last) {
          c.coord_worker.push_back(uint32_t(w));
          c.coord_firm.push_back(f);
          last = f;
        }
        c.coord[*it] = uint32_t(c.coord_worker.size() - 1);
      }
    }
  }
  c.outcome = std::move(in.outcome);
  c.frequency = std::move(in.frequency);
  c.target = std::move(in.target);
  c.controls = std::move(in.controls);
  c.probe_order = std::move(in.probe_order);
  c.physical_total = physical;
  c.target_total = target_total;
  return c;
}

std::vector<uint8_t> select_match_graph(const Canonical& in, GraphReceipt& rc) {
  if (in.rows() == 0) fail(GRAPH_EMPTY, "graph", "command sample is empty");
  // Every step of the match fixed point keeps or drops whole deletion units
  // (components and movers by worker, articulation workers, bridge units), so
  // it runs on the units; the row mask is read off at the end.
  const UnitTable u = unit_table(in);
  UnitGraphs gs = unit_graphs(in, u);
  const size_t D = u.worker.size();
  std::vector<uint8_t> act(D, 1);
  rc = GraphReceipt{};
  rc.input_rows = in.rows();
  rc.input_physical_mass = in.physical_total;

  UnitComponents initial = unit_largest_component(in, u, act, gs);
  rc.initial_components = initial.components;
  rc.maximum_components = initial.components;
  rc.initial_component_rows = initial.retained_rows;
  act.swap(initial.keep);

  {
    auto units = unit_counts(in, u, act);
    for (size_t d = 0; d < D; ++d)
      if (act[d]) act[d] = units[u.worker[d]] > 1;
  }
  uint64_t movers = active_rows(u, act);
  rc.mover_input_rows = movers;
  if (movers == 0) fail(GRAPH_EMPTY, "graph", "no observations remain in the mover target population");
  UnitComponents mover = unit_largest_component(in, u, act, gs);
  rc.maximum_components = std::max<uint64_t>(rc.maximum_components, mover.components);
  act.swap(mover.keep);

  size_t initial_edges = count_true(act);
  rc.initial_deletion_edges = initial_edges;
  uint64_t bound = in.workers + initial_edges + 1;

  // A step that only removed workers with one unit (leaves of one connected
  // coordinate graph) cannot split it: the next component pass would keep
  // everything and report one component, so it is skipped.
  bool connected = false;
  for (;;) {
    if (rc.fixed_point_iterations > bound)
      fail(GRAPH_CERTIFICATE_FAILED, "graph", "sample fixed-point pruning exceeded its finite iteration bound");
    if (!connected) {
      UnitComponents comp = unit_largest_component(in, u, act, gs);
      rc.maximum_components = std::max<uint64_t>(rc.maximum_components, comp.components);
      act.swap(comp.keep);
    }
    connected = false;
    if (count_true(act) == 0) fail(GRAPH_EMPTY, "graph", "no component remains after fixed-point pruning");

    auto units = unit_counts(in, u, act);
    size_t removed = 0;
    for (size_t w = 0; w < in.workers; ++w) removed += units[w] == 1;
    if (removed) {
      for (size_t d = 0; d < D; ++d)
        if (act[d] && units[u.worker[d]] == 1) act[d] = 0;
      rc.insufficient_workers_removed += removed;
      rc.degree_iterations++;
      rc.fixed_point_iterations++;
      connected = true;
      continue;
    }
    // articulation workers and bridge units of the same state, side by side;
    // the bridges are used only when there is no articulation
    std::vector<uint8_t> art;
    std::vector<uint32_t> bridges;
    run_side_by_side([&] { art = unit_articulations(in, u, act, gs); }, [&] { bridges = unit_bridges(act, gs); });
    size_t arts = count_true(art);
    if (arts) {
      for (size_t d = 0; d < D; ++d)
        if (act[d] && art[u.worker[d]]) act[d] = 0;
      rc.articulation_workers_removed += arts;
      rc.articulation_iterations++;
      rc.fixed_point_iterations++;
      continue;
    }
    if (bridges.empty()) break;
    uint64_t removed_rows = 0;
    for (uint32_t d : bridges) {
      act[d] = 0;
      removed_rows += u.rows[d];
    }
    rc.bridge_units_removed += bridges.size();
    rc.bridge_rows_removed += removed_rows;
    rc.bridge_iterations++;
    rc.fixed_point_iterations++;
  }
  if (rc.fixed_point_iterations > bound)
    fail(GRAPH_CERTIFICATE_FAILED, "graph", "sample fixed-point pruning exceeded its finite iteration bound");
  // The loop leaves only from a state it has just certified: one component
  // (the pass above kept the largest and changed nothing after it), no
  // worker with a single unit, no articulation worker, no bridge unit.  The
  // reference's closing component pass and certificates recompute exactly
  // these on the same state, so they are implied here.
  uint64_t kept = active_rows(u, act);
  if (kept == 0) fail(GRAPH_EMPTY, "graph", "no component remains after fixed-point graph pruning");
  rc.retained_rows = kept;
  for (size_t d = 0; d < D; ++d)
    if (act[d]) rc.retained_physical_mass += u.mass[d];
  rc.retained_deletion_edges = count_true(act);
  std::vector<uint8_t> active(in.rows());
  for (size_t r = 0; r < in.rows(); ++r) active[r] = act[in.deletion[r]];
  return active;
}

std::vector<uint8_t> select_implicit_match_graph(const Canonical& in, GraphReceipt& rc) {
  if (in.rows() == 0) fail(GRAPH_EMPTY, "graph_implicit_match", "command sample is empty");
  std::vector<uint8_t> active(in.rows(), 1);
  Graph g = coordinate_graph(in, active);
  auto unsupported = [](const char* m) { fail(UNSUPPORTED_FEATURE, "graph_implicit_match", m); };
  if (g.edges != in.deletion_units)
    unsupported("each implicit match deletion unit must identify one distinct worker-firm coordinate");
  ComponentResult comp = largest_component(in, active);
  if (comp.components != 1) unsupported("the implicit-match graph shortcut requires one connected component");
  for (size_t w = 0; w < in.workers; ++w)
    if (g.ptr[w + 1] - g.ptr[w] <= 1)
      unsupported("the implicit-match graph shortcut requires every worker to be a mover");
  std::vector<uint8_t> art, br;
  tarjan(g, &art, &br);
  for (size_t w = 0; w < in.workers; ++w)
    if (art[w]) unsupported("the implicit-match graph shortcut does not admit worker articulations");
  for (uint8_t b : br)
    if (b) unsupported("the implicit-match graph shortcut does not admit bridge deletion units");
  rc = GraphReceipt{};
  rc.input_rows = rc.retained_rows = in.rows();
  rc.input_physical_mass = rc.retained_physical_mass = in.physical_total;
  rc.initial_components = rc.maximum_components = 1;
  rc.initial_component_rows = rc.mover_input_rows = in.rows();
  rc.initial_deletion_edges = rc.retained_deletion_edges = g.edges;
  return active;
}

std::vector<uint8_t> select_observation_graph(const Canonical& in, GraphReceipt& rc) {
  if (in.rows() == 0) fail(GRAPH_EMPTY, "graph", "command sample is empty");
  // Every step of the observation fixed point keeps or drops whole workers
  // (components, physical singletons, articulation workers), so it runs on a
  // worker mask over the coordinate graph built once; the row mask is read
  // off at the end.
  const size_t W = in.workers, R = in.rows();
  std::vector<uint64_t> wrows(W, 0), wmass(W, 0);
  for (size_t r = 0; r < R; ++r) {
    wrows[in.worker[r]] += 1;
    wmass[in.worker[r]] += in.frequency[r];
  }
  // Workers with one firm (leaves) are left out of the traversed graph: a
  // leaf shares its firm's component, is never an articulation point and
  // changes no other worker's articulation status.  Firms reached only by
  // leaves form components of their own, added after the traversal.
  std::vector<uint32_t> degree(W, 0), leaf_firm(W, MISSING);
  for (size_t c = 0; c < in.coord_worker.size(); ++c) degree[in.coord_worker[c]]++;
  for (size_t c = 0; c < in.coord_worker.size(); ++c)
    if (degree[in.coord_worker[c]] == 1) leaf_firm[in.coord_worker[c]] = in.coord_firm[c];
  Graph g;
  std::vector<uint32_t> edge_worker;  // worker of each traversed edge
  // The repeated component and articulation passes run on a copy of the
  // graph whose vertices are numbered in breadth-first order and whose edges
  // are numbered in the order that traversal first meets them, so the passes
  // walk their per-vertex and per-edge state nearly in sequence.  vnew maps a
  // vertex (worker w, firm W + f) to its number in the copy.  Components,
  // articulation points and their counts do not depend on the numbering.
  std::vector<uint32_t> vnew;
  {
    std::vector<uint32_t> eu, ev;
    for (size_t c = 0; c < in.coord_worker.size(); ++c)
      if (degree[in.coord_worker[c]] > 1) {
        eu.push_back(in.coord_worker[c]);
        ev.push_back(uint32_t(W + in.coord_firm[c]));
      }
    const size_t n = W + in.firms, E = eu.size();
    Graph g0 = make_graph(n, eu, ev);
    vnew.assign(n, MISSING);
    std::vector<uint32_t> enew(E, MISSING), queue;
    queue.reserve(n);
    uint32_t nv = 0, ne = 0;
    for (size_t root = 0; root < n; ++root) {
      if (vnew[root] != MISSING || g0.ptr[root] == g0.ptr[root + 1]) continue;
      vnew[root] = nv++;
      queue.clear();
      queue.push_back(uint32_t(root));
      for (size_t h = 0; h < queue.size(); ++h) {
        const uint32_t v = queue[h];
        for (uint64_t a = g0.ptr[v]; a < g0.ptr[v + 1]; ++a) {
          const Arc arc = g0.arc[a];
          if (enew[arc.edge] == MISSING) enew[arc.edge] = ne++;
          if (vnew[arc.to] == MISSING) {
            vnew[arc.to] = nv++;
            queue.push_back(arc.to);
          }
        }
      }
    }
    for (size_t v = 0; v < n; ++v)
      if (vnew[v] == MISSING) vnew[v] = nv++;  // vertices without a traversed edge
    std::vector<uint32_t> eu2(E), ev2(E);
    edge_worker.assign(E, 0);
    for (size_t e = 0; e < E; ++e) {
      eu2[enew[e]] = vnew[eu[e]];
      ev2[enew[e]] = vnew[ev[e]];
      edge_worker[enew[e]] = eu[e];
    }
    g = make_graph(n, eu2, ev2);
  }
  std::vector<uint8_t> wact(W, 0), on(edge_worker.size(), 0);
  for (size_t w = 0; w < W; ++w) wact[w] = wrows[w] > 0;
  auto mark = [&] {
    size_t edges = 0;
    for (size_t c = 0; c < in.coord_worker.size(); ++c) edges += wact[in.coord_worker[c]];
    for (size_t e = 0; e < on.size(); ++e) on[e] = wact[edge_worker[e]];
    if (!edges) fail(GRAPH_EMPTY, "graph", "active graph is empty");
    return edges;
  };
  auto rows_of = [&] {
    uint64_t n = 0;
    for (size_t w = 0; w < W; ++w)
      if (wact[w]) n += wrows[w];
    return n;
  };
  // `largest_component` on the active workers: (firm count, physical mass)
  auto component = [&](size_t& comps) {
    mark();
    std::vector<uint32_t> label2(g.nodes, MISSING), queue;
    queue.reserve(g.nodes);
    comps = 0;
    for (size_t root = 0; root < g.nodes; ++root) {
      if (label2[root] != MISSING) continue;
      bool has_edge = false;
      for (uint64_t a = g.ptr[root]; a < g.ptr[root + 1] && !has_edge; ++a) has_edge = on[g.arc[a].edge];
      if (!has_edge) continue;
      label2[root] = uint32_t(comps);
      queue.clear();
      queue.push_back(uint32_t(root));
      for (size_t h = 0; h < queue.size(); ++h) {
        uint32_t v = queue[h];
        for (uint64_t a = g.ptr[v]; a < g.ptr[v + 1]; ++a)
          if (on[g.arc[a].edge] && label2[g.arc[a].to] == MISSING) {
            label2[g.arc[a].to] = uint32_t(comps);
            queue.push_back(g.arc[a].to);
          }
      }
      ++comps;
    }
    std::vector<uint32_t> label(g.nodes);
    for (size_t v = 0; v < g.nodes; ++v) label[v] = label2[vnew[v]];
    for (size_t w = 0; w < W; ++w)
      if (wact[w] && degree[w] == 1) {
        uint32_t& fl = label[W + leaf_firm[w]];
        if (fl == MISSING) fl = uint32_t(comps++);  // a firm with leaves only
        label[w] = fl;
      }
    if (comps == 0) fail(GRAPH_EMPTY, "graph", "no connected worker-firm component remains");
    std::vector<uint64_t> firms(comps, 0), mass(comps, 0);
    for (size_t f = 0; f < in.firms; ++f)
      if (label[W + f] != MISSING) firms[label[W + f]]++;
    for (size_t w = 0; w < W; ++w)
      if (wact[w]) {
        if (label[w] == MISSING) fail(INTERNAL_INVARIANT_FAILED, "graph", "active row has no connected-component label");
        mass[label[w]] += wmass[w];
      }
    size_t best = 0;
    for (size_t c = 1; c < comps; ++c)
      if (firms[c] > firms[best] || (firms[c] == firms[best] && mass[c] > mass[best])) best = c;
    size_t winners = 0;
    for (size_t c = 0; c < comps; ++c) winners += (firms[c] == firms[best] && mass[c] == mass[best]);
    if (winners != 1)
      fail(GRAPH_UNIDENTIFIED, "graph", "multiple connected components tie for largest-component selection");
    for (size_t w = 0; w < W; ++w) wact[w] = wact[w] && label[w] == best;
  };
  rc = GraphReceipt{};
  rc.input_rows = R;
  rc.input_physical_mass = in.physical_total;
  size_t comps = 0;
  component(comps);
  rc.initial_components = rc.maximum_components = comps;
  rc.initial_component_rows = rows_of();
  rc.mover_input_rows = rc.initial_component_rows;
  rc.initial_deletion_edges = mark();
  uint64_t bound = W + 1;
  // A step that removed only physical singletons (one row, one coordinate:
  // leaves of one connected graph) cannot split it, so the next component
  // pass is skipped; the loop leaves from a state it has just certified, so
  // the reference's closing component pass and certificates are implied.
  bool connected = false;
  for (;;) {
    if (rc.fixed_point_iterations > bound)
      fail(GRAPH_CERTIFICATE_FAILED, "graph", "observation-deletion pruning exceeded its finite iteration bound");
    if (!connected) {
      component(comps);
      rc.maximum_components = std::max<uint64_t>(rc.maximum_components, comps);
    }
    connected = false;
    if (rows_of() == 0) fail(GRAPH_EMPTY, "graph", "no component remains after observation-deletion pruning");
    size_t removed = 0;
    for (size_t w = 0; w < W; ++w) removed += wact[w] && wmass[w] == 1;
    if (removed) {
      for (size_t w = 0; w < W; ++w)
        if (wact[w] && wmass[w] == 1) wact[w] = 0;
      rc.insufficient_workers_removed += removed;
      rc.degree_iterations++;
      rc.fixed_point_iterations++;
      connected = true;
      continue;
    }
    mark();
    std::vector<uint8_t> art2, art(W);
    tarjan(g, &art2, nullptr, &on);
    for (size_t w = 0; w < W; ++w) art[w] = art2[vnew[w]];
    size_t arts = count_true(art);
    if (arts == 0) break;
    for (size_t w = 0; w < W; ++w)
      if (art[w]) wact[w] = 0;
    rc.articulation_workers_removed += arts;
    rc.articulation_iterations++;
    rc.fixed_point_iterations++;
  }
  uint64_t kept = rows_of();
  if (kept == 0) fail(GRAPH_EMPTY, "graph", "no component remains after observation-deletion graph pruning");
  rc.retained_rows = kept;
  for (size_t w = 0; w < W; ++w)
    if (wact[w]) rc.retained_physical_mass += wmass[w];
  rc.retained_deletion_edges = mark();
  std::vector<uint8_t> active(R);
  for (size_t r = 0; r < R; ++r) active[r] = wact[in.worker[r]];
  return active;
}

Compressed compress(const Canonical& in, const std::vector<uint8_t>& active, bool implicit_match) {
  if (active.size() != in.rows()) fail(INVALID_INPUT, "compression", "active mask has the wrong length");
  Compressed p;
  if (implicit_match && count_true(active) != in.rows())
    fail(INTERNAL_INVARIANT_FAILED, "compression", "the certified implicit-match route must retain every row");
  p.retained_rows = active_indices(active);
  size_t R = p.retained_rows.size();
  if (R == 0) fail(GRAPH_EMPTY, "compression", "no rows remain after graph selection");

  auto redense_selected = [&](const std::vector<uint32_t>& values, size_t levels, size_t& count) {
    std::vector<uint32_t> map(levels, MISSING);
    if (implicit_match) {
      for (size_t l = 0; l < levels; ++l) map[l] = uint32_t(l);
      count = levels;
      return map;
    }
    std::vector<uint8_t> present(levels, 0);
#pragma omp parallel for schedule(static) if (R >= 65536)
    for (size_t i = 0; i < R; ++i) present[values[p.retained_rows[i]]] = 1;
    uint32_t next = 0;
    for (size_t l = 0; l < levels; ++l)
      if (present[l]) map[l] = next++;
    count = next;
    return map;
  };
  size_t W, F, D;
  auto wmap = redense_selected(in.worker, in.workers, W);
  auto fmap = redense_selected(in.firm, in.firms, F);
  auto dmap = redense_selected(in.deletion, in.deletion_units, D);
  p.row_worker.resize(R);
  p.row_firm.resize(R);
  p.row_deletion.resize(R);
#pragma omp parallel for schedule(static) if (R >= 65536)
  for (size_t i = 0; i < R; ++i) {
    uint64_t r = p.retained_rows[i];
    p.row_worker[i] = wmap[in.worker[r]];
    p.row_firm[i] = fmap[in.firm[r]];
    p.row_deletion[i] = dmap[in.deletion[r]];
  }
  if (F < 2) fail(GRAPH_UNIDENTIFIED, "compression", "retained graph must contain at least two firms");
  p.workers = W;
  p.firms = F;
  p.deletion_units = D;

  // cells: rows sorted by (worker, firm, source row)
  // stable radix sort of the (worker, firm) keys: equal keys keep row order
  std::vector<uint32_t> order(R);
  std::iota(order.begin(), order.end(), 0u);
  std::vector<uint64_t> key(R);
#pragma omp parallel for schedule(static) if (R >= 65536)
  for (size_t i = 0; i < R; ++i) key[i] = (uint64_t(p.row_worker[i]) << 32) | p.row_firm[i];
  {
    std::vector<uint64_t> sorted_key = key;
    radix_sort_pairs(sorted_key, order);
  }
  p.row_cell.assign(R, MISSING);
  // cell boundaries in the sorted order, then every cell's Kahan sums (in row
  // order, as a sequential walk would take them) independently
  std::vector<size_t> cell_start;
  {
    std::vector<uint8_t> first(R);
#pragma omp parallel for schedule(static) if (R >= 65536)
    for (size_t i = 0; i < R; ++i) first[i] = i == 0 || key[order[i]] != key[order[i - 1]];
    const std::vector<uint64_t> at = active_indices(first);
    cell_start.assign(at.begin(), at.end());
  }
  const size_t NC = cell_start.size();
  cell_start.push_back(R);
  p.cell_worker.resize(NC);
  p.cell_firm.resize(NC);
  p.cell_weight.resize(NC);
  p.cell_outcome_sum.resize(NC);
  p.cell_target_sum.resize(NC);
  std::atomic<bool> bad_moment{false};
#pragma omp parallel for schedule(static) if (NC >= 65536)
  for (size_t cell = 0; cell < NC; ++cell) {
    const uint64_t k = key[order[cell_start[cell]]];
    KahanSum wsum, ysum, tsum;
    for (size_t j = cell_start[cell]; j < cell_start[cell + 1]; ++j) {
      uint32_t lr = order[j];
      uint64_t src = p.retained_rows[lr];
      double wt = double(in.frequency[src]);
      double y = wt * in.outcome[src];
      if (!std::isfinite(wt) || !std::isfinite(y)) bad_moment = true;
      wsum.add(wt);
      ysum.add(y);
      tsum.add(in.target[src]);
      p.row_cell[lr] = uint32_t(cell);
    }
    p.cell_worker[cell] = uint32_t(k >> 32);
    p.cell_firm[cell] = uint32_t(k & 0xffffffffu);
    p.cell_weight[cell] = wsum.finish();
    p.cell_outcome_sum[cell] = ysum.finish();
    p.cell_target_sum[cell] = tsum.finish();
  }
  if (bad_moment) fail(INVALID_WEIGHT, "compression", "weighted cell moment is nonfinite");
  p.cell_index.ptr.assign(cell_start.begin(), cell_start.end());
  p.cell_index.items = order;
  size_t C = p.cell_worker.size();
  p.cells = C;
  {
    std::vector<uint32_t> ord(C);
    std::iota(ord.begin(), ord.end(), 0u);
    p.worker_index = grouped_from_order(W, p.cell_worker, std::move(ord));
    // cells are numbered in (worker, firm) order, so a stable counting sort by
    // firm gives the (firm, worker, cell) order
    std::vector<uint32_t> fptr(F + 1, 0), ford(C);
    for (size_t c = 0; c < C; ++c) fptr[p.cell_firm[c] + 1]++;
    for (size_t f = 0; f < F; ++f) fptr[f + 1] += fptr[f];
    {
      std::vector<uint32_t> at(fptr.begin(), fptr.end() - 1);
      for (size_t c = 0; c < C; ++c) ford[at[p.cell_firm[c]]++] = uint32_t(c);
    }
    p.firm_index = grouped_from_order(F, p.cell_firm, std::move(ford));
  }

  // exact target strata (reference `exact_target_strata`, problem.rs:900-965;
  // the certified-match variant yields the same order)
  {
    auto cmp = [&](uint32_t a, uint32_t b) -> int {
      uint64_t sa = p.retained_rows[a], sb = p.retained_rows[b];
      if (p.row_worker[a] != p.row_worker[b]) return p.row_worker[a] < p.row_worker[b] ? -1 : 1;
      if (p.row_firm[a] != p.row_firm[b]) return p.row_firm[a] < p.row_firm[b] ? -1 : 1;
      if (p.row_deletion[a] != p.row_deletion[b]) return p.row_deletion[a] < p.row_deletion[b] ? -1 : 1;
      int c = total_cmp(in.outcome[sa], in.outcome[sb]);
      if (c) return c;
      if (in.frequency[sa] != in.frequency[sb]) return in.frequency[sa] < in.frequency[sb] ? -1 : 1;
      c = total_cmp(in.target[sa], in.target[sb]);
      if (c) return c;
      for (auto& ctl : in.controls) {
        c = total_cmp(ctl[sa], ctl[sb]);
        if (c) return c;
      }
      return 0;
    };
    // the comparison leads with (worker, firm), the cell key: `order` already
    // holds the rows by cell with ties in row order, so a stable sort inside
    // every cell gives the stable sort of all rows
    std::vector<uint32_t> tord = order;
    {
      std::vector<size_t> cell_begin(C + 1, 0);
      for (size_t i = 0; i < R; ++i) cell_begin[p.row_cell[i] + 1]++;
      for (size_t c = 0; c < C; ++c) cell_begin[c + 1] += cell_begin[c];
#pragma omp parallel for schedule(dynamic, 4096) if (C >= 65536)
      for (size_t c = 0; c < C; ++c)
        if (cell_begin[c + 1] - cell_begin[c] > 1)
          std::stable_sort(tord.begin() + cell_begin[c], tord.begin() + cell_begin[c + 1],
                           [&](uint32_t a, uint32_t b) { return cmp(a, b) < 0; });
    }
    p.row_target.assign(R, MISSING);
    {
      // stratum starts compared on all host cores, then every row's stratum
      std::vector<uint8_t> first(R);
#pragma omp parallel for schedule(static) if (R >= 65536)
      for (size_t i = 0; i < R; ++i) first[i] = i == 0 || cmp(tord[i - 1], tord[i]) != 0;
      const std::vector<uint64_t> starts = active_indices(first);
      const size_t S = starts.size();
#pragma omp parallel for schedule(static) if (S >= 65536)
      for (size_t k = 0; k < S; ++k) {
        const size_t e = k + 1 < S ? starts[k + 1] : R;
        for (size_t i = starts[k]; i < e; ++i) p.row_target[tord[i]] = uint32_t(k);
      }
      p.exact_target_strata = S;
    }
    p.target_index = grouped_from_order(p.exact_target_strata, p.row_target, std::move(tord));
  }
  // the deletion index and the retained copies of the row columns are
  // independent: one thread each (a column's gather and its totals in row
  // order, as a sequential walk takes them)
  KahanSum tt;
  p.controls.resize(in.controls.size());
  std::vector<std::function<void()>> tasks = {
      [&] { p.deletion_index = grouped_rows(D, p.row_deletion); },
      [&] {
        p.outcome.resize(R);
        for (size_t i = 0; i < R; ++i) p.outcome[i] = in.outcome[p.retained_rows[i]];
      },
      [&] {
        p.frequency.resize(R);
        for (size_t i = 0; i < R; ++i) {
          p.frequency[i] = in.frequency[p.retained_rows[i]];
          p.physical_total += p.frequency[i];
        }
      },
      [&] {
        p.target.resize(R);
        for (size_t i = 0; i < R; ++i) {
          p.target[i] = in.target[p.retained_rows[i]];
          tt.add(p.target[i]);
        }
      }};
  for (size_t k = 0; k < in.controls.size(); ++k)
    tasks.push_back([&, k] {
      std::vector<double>& col = p.controls[k];
      col.resize(R);
      for (size_t i = 0; i < R; ++i) col[i] = in.controls[k][p.retained_rows[i]];
    });
  if (!in.probe_order.empty())
    tasks.push_back([&] {
      p.probe_order.resize(R);
      for (size_t i = 0; i < R; ++i) p.probe_order[i] = in.probe_order[p.retained_rows[i]];
    });
  run_tasks(tasks);
  p.target_total = tt.finish();
  if (!std::isfinite(p.target_total) || p.target_total <= 0.0)
    fail(INVALID_TARGET_WEIGHT, "compression", "retained target mass is not positive and finite");
  p.rows_physical = p.physical_total;
  return p;
}

uint64_t compressed_topology_checksum(const Compressed& p) {
  return topology_checksum(p.row_worker, p.row_firm, p.row_deletion, p.frequency);
}

JlaPlan build_plan(const Compressed& p) {
  size_t R = p.rows();
  JlaPlan plan;
  std::vector<double> per_copy(R);
  for (size_t r = 0; r < R; ++r) {
    if (p.frequency[r] == 0 || p.frequency[r] > MAX_EXACT_BINARY64_INTEGER)
      fail(INVALID_WEIGHT, "jla_plan", "frequency must be an exact positive binary64 integer");
    double v = canonical_zero(p.target[r] / double(p.frequency[r]));
    if (!std::isfinite(v) || v < 0.0)
      fail(INVALID_TARGET_WEIGHT, "jla_plan", "per-copy target mass is invalid at zero-based row " + std::to_string(r));
    per_copy[r] = v;
  }
  bool has_order = !p.probe_order.empty();
  // semantic key (reference `compare_semantic_rows`, jla.rs:523-540)
  auto sem = [&](uint32_t a, uint32_t b) -> int {
    if (p.row_worker[a] != p.row_worker[b]) return p.row_worker[a] < p.row_worker[b] ? -1 : 1;
    if (p.row_firm[a] != p.row_firm[b]) return p.row_firm[a] < p.row_firm[b] ? -1 : 1;
    if (p.row_deletion[a] != p.row_deletion[b]) return p.row_deletion[a] < p.row_deletion[b] ? -1 : 1;
    int c = ordered_f64(per_copy[a], per_copy[b]);
    if (c) return c;
    c = ordered_f64(p.outcome[a], p.outcome[b]);
    if (c) return c;
    if (has_order) return ordered_f64(p.probe_order[a], p.probe_order[b]);
    return 0;
  };
  std::vector<uint32_t> order(R);
  std::iota(order.begin(), order.end(), 0u);
  sort_rows(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    int c = sem(a, b);
    return c ? c < 0 : a < b;
  });
  plan.row_rank.assign(R, 0);
  uint64_t current = 0;
  for (size_t i = 0; i < R; ++i) {
    if (i == 0 || sem(order[i - 1], order[i]) != 0) ++current;
    plan.row_rank[order[i]] = current;
  }

  // deletion units (reference `deletion_plan`, jla.rs:574-649)
  size_t G = p.deletion_index.ptr.size() - 1;
  plan.del_cell.resize(G);
  plan.del_count.resize(G);
  plan.del_rank.resize(G);
  plan.del_outcome_sum.resize(G);
  plan.del_target_mass.resize(G);
  for (size_t g = 0; g < G; ++g) {
    uint64_t b = p.deletion_index.ptr[g], e = p.deletion_index.ptr[g + 1];
    if (b == e) fail(INTERNAL_INVARIANT_FAILED, "jla_plan", "deletion unit has no retained row");
    uint64_t phys = 0, minrank = ~uint64_t(0);
    uint32_t cell = MISSING;
    StableSum y, t;
    for (uint64_t i = b; i < e; ++i) {
      uint32_t r = p.deletion_index.items[i];
      phys += p.frequency[r];
      if (cell == MISSING) cell = p.row_cell[r];
      else if (cell != p.row_cell[r])
        fail(INVALID_IDENTIFIER, "jla_plan", "one deletion unit crosses coefficient cells");
      y.add(double(p.frequency[r]) * p.outcome[r]);
      t.add(p.target[r]);
      minrank = std::min(minrank, plan.row_rank[r]);
    }
    plan.del_cell[g] = cell;
    plan.del_count[g] = phys;
    plan.del_outcome_sum[g] = y.finish();
    plan.del_target_mass[g] = t.finish();
    plan.del_rank[g] = minrank;
  }
  {
    std::vector<uint64_t> s = plan.del_rank;
    std::sort(s.begin(), s.end());
    if (std::adjacent_find(s.begin(), s.end()) != s.end())
      fail(INTERNAL_INVARIANT_FAILED, "jla_plan", "deletion-unit semantic ranks are not unique");
  }

  // target strata (reference `target_plan`, jla.rs:651-790)
  std::vector<uint32_t> tord(R);
  std::iota(tord.begin(), tord.end(), 0u);
  sort_rows(tord.begin(), tord.end(), [&](uint32_t a, uint32_t b) {
    if (p.row_cell[a] != p.row_cell[b]) return p.row_cell[a] < p.row_cell[b];
    int c = ordered_f64(per_copy[a], per_copy[b]);
    if (c) return c < 0;
    if (plan.row_rank[a] != plan.row_rank[b]) return plan.row_rank[a] < plan.row_rank[b];
    return a < b;
  });
  for (size_t cur = 0; cur < R;) {
    size_t begin = cur;
    uint32_t cell = p.row_cell[tord[cur]];
    double pc = canonical_zero(per_copy[tord[cur]]);
    uint64_t bits;
    std::memcpy(&bits, &pc, 8);
    ++cur;
    while (cur < R) {
      double v = canonical_zero(per_copy[tord[cur]]);
      uint64_t vb;
      std::memcpy(&vb, &v, 8);
      if (p.row_cell[tord[cur]] != cell || vb != bits) break;
      ++cur;
    }
    uint64_t phys = 0, minrank = ~uint64_t(0);
    StableSum t;
    for (size_t j = begin; j < cur; ++j) {
      uint32_t r = tord[j];
      phys += p.frequency[r];
      t.add(p.target[r]);
      minrank = std::min(minrank, plan.row_rank[r]);
    }
    plan.tgt_cell.push_back(cell);
    plan.tgt_per_copy.push_back(pc);
    plan.tgt_count.push_back(phys);
    plan.tgt_mass.push_back(t.finish());
    plan.tgt_rank.push_back(minrank);
  }
  {
    std::vector<uint64_t> s = plan.tgt_rank;
    std::sort(s.begin(), s.end());
    if (std::adjacent_find(s.begin(), s.end()) != s.end())
      fail(INTERNAL_INVARIANT_FAILED, "jla_plan", "target semantic plan is incomplete or noncanonical");
  }
  return plan;
}

}  // namespace fevcb

namespace fevcb {

void build_target_strata(const Compressed& p, const std::vector<double>& per_copy, JlaPlan& plan);

// Leave-observation-out units.  Semantic ranks order rows by worker, firm,
// per-copy target mass and outcome (total order, -0.0 folded into +0.0 for
// the mass), then the controls and the probe order; the deletion identifier
// takes no part (reference `observation_row_ranks` / `compare_observation_rows`,
// generic_jla.rs:4267-4334).  Rows of one rank form a class whose physical
// copies are numbered consecutively in row order: copy c of the class draws
// bit c % 64 of Counter-V1 word c / 64 for entity = rank (reference
// `observation_classes`, generic_jla.rs:4158-4215, `observation_addresses`,
// generic_jla/statistical_batches.rs:15-54, `rademacher_copy`,
// generic_jla.rs:10322-10329).
// Rows grouped by cell, in row order inside each cell (a stable counting
// sort), and the cell offsets.  Cells are numbered in (worker, firm) order,
// so a comparison that leads with (worker, firm) or with the cell sorts all
// rows stably when every cell's range is stable-sorted by the rest of it.
static std::vector<uint32_t> rows_by_cell(const Compressed& p, std::vector<size_t>& begin) {
  const size_t R = p.rows(), C = p.cells;
  if (p.cell_index.items.size() == R && p.cell_index.ptr.size() == C + 1) {  // kept by the compression
    begin.assign(p.cell_index.ptr.begin(), p.cell_index.ptr.end());
    return p.cell_index.items;
  }
  begin.assign(C + 1, 0);
  for (size_t r = 0; r < R; ++r) begin[p.row_cell[r] + 1]++;
  for (size_t c = 0; c < C; ++c) begin[c + 1] += begin[c];
  std::vector<uint32_t> order(R);
  std::vector<size_t> at(begin.begin(), begin.end() - 1);
  for (size_t r = 0; r < R; ++r) order[at[p.row_cell[r]]++] = uint32_t(r);
  return order;
}

template <class Less>
static void sort_within_cells(std::vector<uint32_t>& order, const std::vector<size_t>& begin, Less less) {
  const size_t C = begin.size() - 1;
#pragma omp parallel for schedule(dynamic, 4096) if (C >= 65536)
  for (size_t c = 0; c < C; ++c)
    if (begin[c + 1] - begin[c] > 1) std::stable_sort(order.begin() + begin[c], order.begin() + begin[c + 1], less);
}

static void build_observation_units(const Compressed& p, const std::vector<double>& per_copy, JlaPlan& plan) {
  size_t R = p.rows();
  bool has_order = !p.probe_order.empty();
  auto sem = [&](uint32_t a, uint32_t b) -> int {
    if (p.row_worker[a] != p.row_worker[b]) return p.row_worker[a] < p.row_worker[b] ? -1 : 1;
    if (p.row_firm[a] != p.row_firm[b]) return p.row_firm[a] < p.row_firm[b] ? -1 : 1;
    int c = total_cmp(canonical_zero(per_copy[a]), canonical_zero(per_copy[b]));
    if (c) return c;
    c = total_cmp(p.outcome[a], p.outcome[b]);
    if (c) return c;
    for (auto& col : p.controls) {
      c = ordered_f64(col[a], col[b]);
      if (c) return c;
    }
    if (has_order) return ordered_f64(p.probe_order[a], p.probe_order[b]);
    return 0;
  };
  std::vector<size_t> cell_begin;
  std::vector<uint32_t> order = rows_by_cell(p, cell_begin);
  sort_within_cells(order, cell_begin, [&](uint32_t a, uint32_t b) { return sem(a, b) < 0; });
  // class starts: the rows whose semantic key differs from the previous row's
  // (compared on all host cores); rank = 1 + the class index
  std::vector<uint8_t> first(R);
#pragma omp parallel for schedule(static) if (R >= 65536)
  for (size_t i = 0; i < R; ++i) first[i] = i == 0 || sem(order[i - 1], order[i]) != 0;
  const std::vector<uint64_t> starts = active_indices(first);
  const size_t classes = starts.size();
  plan.row_rank.assign(R, 0);
  plan.row_copy_offset.assign(R, 0);
  plan.group_ptr.assign(classes + 1, 0);
  plan.group_rows.assign(order.begin(), order.end());
  plan.del_cell.assign(classes, 0);
  plan.del_count.assign(classes, 0);
  plan.del_rank.assign(classes, 0);
  plan.del_outcome_sum.assign(classes, 0.0);
  plan.del_target_mass.assign(classes, 0.0);
  std::atomic<bool> bad{false};
  // classes: rows sorted by (rank, row); the stable sort above already holds
  // equal ranks in row order.  Every class is summed in row order by one
  // thread, so the sums do not depend on the thread count.
#pragma omp parallel for schedule(dynamic, 4096) if (classes >= 65536)
  for (size_t k = 0; k < classes; ++k) {
    const size_t i = starts[k], j = k + 1 < classes ? starts[k + 1] : R;
    uint64_t phys = 0;
    StableSum y, t;
    for (size_t u = i; u < j; ++u) {
      const uint32_t r = order[u];
      plan.row_rank[r] = k + 1;
      plan.row_copy_offset[r] = phys;
      phys += p.frequency[r];
      y.add(double(p.frequency[r]) * p.outcome[r]);
      t.add(p.target[r]);
    }
    if (phys == 0 || (phys + 63) / 64 > (uint64_t(1) << 20)) bad = true;
    plan.group_ptr[k + 1] = j;
    plan.del_cell[k] = p.row_cell[order[i]];
    plan.del_count[k] = phys;
    plan.del_rank[k] = k + 1;
    plan.del_outcome_sum[k] = y.finish();
    plan.del_target_mass[k] = t.finish();
  }
  if (bad) fail(RESOURCE_LIMIT, "generic_jla_rng_preflight", "observation class has an invalid physical trial count");
}

JlaPlan build_generic_plan(const Compressed& p, Deletion deletion) {
  size_t R = p.rows();
  JlaPlan plan;
  plan.generic = true;
  std::vector<double> per_copy(R);
  for (size_t r = 0; r < R; ++r) per_copy[r] = p.target[r] / double(p.frequency[r]);
  bool has_order = !p.probe_order.empty();
  if (deletion == Deletion::Observation) {
    plan.observation = true;
    build_observation_units(p, per_copy, plan);
    build_target_strata(p, per_copy, plan);
    return plan;
  }
  // reference `compare_semantic_rows` (generic_jla.rs:3878-3900): per-copy mass
  // and outcome by total order (no zero canonicalisation), then the controls
  // and the probe order with -0.0 mapped to +0.0
  auto sem = [&](uint32_t a, uint32_t b) -> int {
    if (p.row_worker[a] != p.row_worker[b]) return p.row_worker[a] < p.row_worker[b] ? -1 : 1;
    if (p.row_firm[a] != p.row_firm[b]) return p.row_firm[a] < p.row_firm[b] ? -1 : 1;
    if (p.row_deletion[a] != p.row_deletion[b]) return p.row_deletion[a] < p.row_deletion[b] ? -1 : 1;
    int c = total_cmp(per_copy[a], per_copy[b]);
    if (c) return c;
    c = total_cmp(p.outcome[a], p.outcome[b]);
    if (c) return c;
    for (auto& col : p.controls) {
      c = ordered_f64(col[a], col[b]);
      if (c) return c;
    }
    if (has_order) return ordered_f64(p.probe_order[a], p.probe_order[b]);
    return 0;
  };
  std::vector<uint32_t> order(R);
  std::iota(order.begin(), order.end(), 0u);
  sort_rows(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return sem(a, b) < 0; });
  plan.row_rank.assign(R, 0);
  uint64_t current = 0;
  for (size_t i = 0; i < R; ++i) {
    if (i == 0 || sem(order[i - 1], order[i]) != 0) ++current;
    plan.row_rank[order[i]] = current;
  }
  // match groups (deletion units), rows stably sorted by rank
  size_t G = p.deletion_index.ptr.size() - 1;
  plan.group_ptr.assign(p.deletion_index.ptr.begin(), p.deletion_index.ptr.end());
  plan.group_rows.assign(p.deletion_index.items.begin(), p.deletion_index.items.end());
  plan.del_cell.resize(G);
  plan.del_count.resize(G);
  plan.del_rank.resize(G);
  plan.del_outcome_sum.resize(G);
  plan.del_target_mass.resize(G);
  for (size_t g = 0; g < G; ++g) {
    auto b = plan.group_rows.begin() + plan.group_ptr[g], e = plan.group_rows.begin() + plan.group_ptr[g + 1];
    if (b == e) fail(RESOURCE_LIMIT, "generic_jla_match_plan", "a match block is empty or exceeds blocksize_limit");
    std::stable_sort(b, e, [&](uint32_t x, uint32_t y) { return plan.row_rank[x] < plan.row_rank[y]; });
    uint32_t cell = p.row_cell[*b];
    uint64_t phys = 0, ent = ~uint64_t(0);
    StableSum y, t;
    for (auto it = b; it != e; ++it) {
      if (p.row_cell[*it] != cell)
        fail(INVALID_IDENTIFIER, "generic_jla_match_plan", "one match deletion unit crosses coefficient cells");
      phys += p.frequency[*it];
      ent = std::min(ent, plan.row_rank[*it]);
      y.add(double(p.frequency[*it]) * p.outcome[*it]);
      t.add(p.target[*it]);
    }
    if (phys == 0 || (phys + 63) / 64 > (uint64_t(1) << 20))
      fail(RESOURCE_LIMIT, "jla_validate", "match deletion unit trial preflight failed");
    plan.del_cell[g] = cell;
    plan.del_count[g] = phys;
    plan.del_rank[g] = ent;
    plan.del_outcome_sum[g] = y.finish();
    plan.del_target_mass[g] = t.finish();
  }
  build_target_strata(p, per_copy, plan);
  return plan;
}

// Target strata of the generic estimator: rows grouped by (cell, per-copy
// target mass), each stratum keyed by its smallest semantic rank (reference
// `target_plan`, generic_jla.rs:3902-3995).
void build_target_strata(const Compressed& p, const std::vector<double>& per_copy, JlaPlan& plan) {
  size_t R = p.rows();
  std::vector<size_t> cell_begin;
  std::vector<uint32_t> tord = rows_by_cell(p, cell_begin);
  sort_within_cells(tord, cell_begin, [&](uint32_t a, uint32_t b) {
    int c = total_cmp(canonical_zero(per_copy[a]), canonical_zero(per_copy[b]));
    if (c) return c < 0;
    return plan.row_rank[a] < plan.row_rank[b];
  });
  // strata: runs of equal (cell, per-copy mass bits), found on all host cores;
  // each stratum is summed in order by one thread
  auto bits_of = [&](uint32_t r) {
    const double v = canonical_zero(per_copy[r]);
    uint64_t b;
    std::memcpy(&b, &v, 8);
    return b;
  };
  std::vector<uint8_t> first(R);
#pragma omp parallel for schedule(static) if (R >= 65536)
  for (size_t i = 0; i < R; ++i)
    first[i] = i == 0 || p.row_cell[tord[i]] != p.row_cell[tord[i - 1]] || bits_of(tord[i]) != bits_of(tord[i - 1]);
  const std::vector<uint64_t> starts = active_indices(first);
  const size_t S = starts.size();
  plan.tgt_cell.assign(S, 0);
  plan.tgt_per_copy.assign(S, 0.0);
  plan.tgt_count.assign(S, 0);
  plan.tgt_mass.assign(S, 0.0);
  plan.tgt_rank.assign(S, 0);
#pragma omp parallel for schedule(dynamic, 4096) if (S >= 65536)
  for (size_t k = 0; k < S; ++k) {
    const size_t b = starts[k], e = k + 1 < S ? starts[k + 1] : R;
    uint64_t phys = 0, ent = ~uint64_t(0);
    StableSum t;
    for (size_t u = b; u < e; ++u) {
      const uint32_t r = tord[u];
      phys += p.frequency[r];
      t.add(p.target[r]);
      ent = std::min(ent, plan.row_rank[r]);
    }
    plan.tgt_cell[k] = p.row_cell[tord[b]];
    plan.tgt_per_copy[k] = canonical_zero(per_copy[tord[b]]);
    plan.tgt_count[k] = phys;
    plan.tgt_mass[k] = t.finish();
    plan.tgt_rank[k] = ent;
  }
}

}  // namespace fevcb
