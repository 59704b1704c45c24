// Native gate-fusion planner: circuit graph + agglomerative fusion + cost models.
//
// C++ restatement of the reference's optimiser (narix10yc/cast_simulator):
//   * CircuitGraph, rows x qubits with left-push insertion, squeeze, same-row
//     and cross-row fusion (src/circuit_graph.rs:107-504);
//   * phase 1 size-2 canonicalisation and phase 2 agglomerative fusion over
//     candidate sizes 3..size_max with a cost-model accept/rollback step
//     (src/fusion.rs:14-345);
//   * SizeOnlyCostModel and HardwareAdaptiveCostModel (src/cost_model.rs:20-44,
//     238-275), the latter with a per-gate-size crossover so that gates that run
//     on the tensor-core path are measured against the tensor pipe's ceiling.
// Unitary gates only (the state-vector path); noisy circuits are fused on the
// host-side Python mirror, which keeps the Kraus branches.
#include "../../include/cast_b200.h"
#include "internal.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <exception>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_set>
#include <vector>

namespace {

using cd = std::complex<double>;

struct HGate {
  std::vector<uint32_t> q;  // ascending
  std::vector<cd> m;        // row-major 2^k x 2^k
  std::vector<int> prov;    // source gates in application order (trajectory builder)
  uint32_t k() const { return (uint32_t)q.size(); }
};
using GatePtr = std::shared_ptr<const HGate>;

// expand_matrix: gate.rs:436-468 (identity on the union's other wires)
std::vector<cd> expand(const HGate &g, const std::vector<uint32_t> &uq) {
  const size_t ud = 1ull << uq.size(), gd = 1ull << g.k();
  if (g.q == uq) return g.m;
  std::vector<uint32_t> pos(g.k());
  size_t tmask = 0;
  for (uint32_t t = 0; t < g.k(); ++t) {
    pos[t] = (uint32_t)(std::find(uq.begin(), uq.end(), g.q[t]) - uq.begin());
    tmask |= 1ull << pos[t];
  }
  std::vector<size_t> comp(ud);
  for (size_t i = 0; i < ud; ++i) {
    size_t c = 0;
    for (uint32_t t = 0; t < g.k(); ++t) c |= ((i >> pos[t]) & 1ull) << t;
    comp[i] = c;
  }
  std::vector<cd> out(ud * ud, cd(0, 0));
  for (size_t r = 0; r < ud; ++r)
    for (size_t c = 0; c < ud; ++c)
      if (((r ^ c) & ~tmask) == 0) out[r * ud + c] = g.m[comp[r] * gd + comp[c]];
  return out;
}

// QuantumGate::matmul (unitary part): self * other on the union (gate.rs:280-284, 319)
GatePtr matmul(const HGate &a, const HGate &b) {
  auto g = std::make_shared<HGate>();
  g->prov = b.prov;  // b acts first
  g->prov.insert(g->prov.end(), a.prov.begin(), a.prov.end());
  std::set_union(a.q.begin(), a.q.end(), b.q.begin(), b.q.end(), std::back_inserter(g->q));
  const size_t d = 1ull << g->q.size();
  const std::vector<cd> ea = expand(a, g->q), eb = expand(b, g->q);
  g->m.assign(d * d, cd(0, 0));
  for (size_t r = 0; r < d; ++r)
    for (size_t t = 0; t < d; ++t) {
      const cd x = ea[r * d + t];
      if (x == cd(0, 0)) continue;
      for (size_t c = 0; c < d; ++c) g->m[r * d + c] += x * eb[t * d + c];
    }
  return g;
}

double arithmetic_intensity(const HGate &g, double ztol) {
  size_t nnz = 0;
  for (const cd &z : g.m) nnz += (std::abs(z.real()) > ztol) + (std::abs(z.imag()) > ztol);
  return (double)nnz / (double)(1ull << g.k());
}

struct Cost {
  int kind;  // 0 size-only, 1 hardware-adaptive
  uint32_t max_size;
  double zero_tol;
  double crossover;         // CUDA-core crossover AI
  double tensor_crossover;  // crossover for gates with k >= tensor_min_k (0 = none)
  uint32_t tensor_min_k;

  double of(const HGate &g) const {
    if (kind == 0) return g.k() > max_size ? 1.0 : 1e-10;
    if (g.k() > max_size) return INFINITY;
    const double xo =
        (tensor_min_k && g.k() >= tensor_min_k && tensor_crossover > 0) ? tensor_crossover : crossover;
    return std::max(1.0, arithmetic_intensity(g, zero_tol) / xo);
  }
};

// CircuitGraph (circuit_graph.rs)
struct Graph {
  uint32_t n = 0;
  std::vector<std::vector<int>> rows;
  std::vector<GatePtr> gates;

  int id_at(size_t row, uint32_t q) const {
    return row < rows.size() && q < n ? rows[row][q] : -1;
  }
  bool vacant(size_t row, const std::vector<uint32_t> &qs) const {
    for (uint32_t q : qs)
      if (q < n && rows[row][q] >= 0) return false;
    return true;
  }
  void place(size_t row, int id, const std::vector<uint32_t> &qs) {
    for (uint32_t q : qs) rows[row][q] = id;
  }
  int insert(GatePtr g) {
    size_t min_row = 0;
    for (uint32_t q : g->q)
      for (size_t r = rows.size(); r-- > 0;)
        if (rows[r][q] >= 0) {
          min_row = std::max(min_row, r + 1);
          break;
        }
    size_t row = rows.size();
    for (size_t r = min_row; r < rows.size(); ++r)
      if (vacant(r, g->q)) {
        row = r;
        break;
      }
    if (row == rows.size()) rows.emplace_back(n, -1);
    const int id = (int)gates.size();
    gates.push_back(g);
    place(row, id, g->q);
    return id;
  }
  int insert_at(size_t row, GatePtr g) {
    const int id = (int)gates.size();
    gates.push_back(g);
    place(row, id, g->q);
    return id;
  }
  GatePtr remove_at(size_t row, uint32_t q) {
    const int id = id_at(row, q);
    if (id < 0 || !gates[id]) return nullptr;
    GatePtr g = gates[id];
    for (uint32_t x : g->q) rows[row][x] = -1;
    gates[id] = nullptr;
    return g;
  }
  std::vector<int> live_ids() const {
    std::vector<int> out;
    for (const auto &r : rows) {
      std::vector<int> seen;
      for (int id : r)
        if (id >= 0 && std::find(seen.begin(), seen.end(), id) == seen.end()) seen.push_back(id);
      out.insert(out.end(), seen.begin(), seen.end());
    }
    return out;
  }
  void squeeze() {
    std::vector<std::vector<int>> nr;
    std::vector<int> last(n, -1);
    for (int id : live_ids()) {
      const auto &qs = gates[id]->q;
      size_t mr = 0;
      for (uint32_t q : qs)
        if (last[q] >= 0) mr = std::max(mr, (size_t)last[q] + 1);
      size_t row = nr.size();
      for (size_t r = mr; r < nr.size(); ++r) {
        bool ok = true;
        for (uint32_t q : qs) ok = ok && nr[r][q] < 0;
        if (ok) {
          row = r;
          break;
        }
      }
      if (row == nr.size()) nr.emplace_back(n, -1);
      for (uint32_t q : qs) {
        nr[row][q] = id;
        last[q] = (int)row;
      }
    }
    rows.swap(nr);
  }
  int fuse_same_row(size_t row, uint32_t qa, uint32_t qb) {
    const int a = id_at(row, qa), b = id_at(row, qb);
    if (a < 0 || b < 0 || a == b) return -1;
    GatePtr ga = gates[a], gb = gates[b];
    remove_at(row, qa);
    remove_at(row, qb);
    return insert_at(row, matmul(*ga, *gb));
  }
  std::pair<int, size_t> fuse_across(size_t ra, uint32_t qa, size_t rb, uint32_t qb) {
    const int a = id_at(ra, qa), b = id_at(rb, qb);
    GatePtr ga = gates[a], gb = gates[b];
    remove_at(ra, qa);
    remove_at(rb, qb);
    GatePtr f = matmul(*gb, *ga);
    size_t target;
    if (vacant(rb, f->q)) target = rb;
    else if (vacant(ra, f->q)) target = ra;
    else {
      rows.insert(rows.begin() + rb, std::vector<int>(n, -1));
      target = rb;
    }
    return {insert_at(target, f), target};
  }
};

// ── phase 1 (fusion.rs:14-134) ──────────────────────────────────────────────
bool absorb_single(Graph &g, size_t row, uint32_t q) {
  const int id = g.id_at(row, q);
  if (id < 0 || !g.gates[id] || g.gates[id]->k() != 1) return false;
  GatePtr gate = g.gates[id];
  for (size_t nr = row + 1; nr < g.rows.size(); ++nr) {
    const int nid = g.id_at(nr, q);
    if (nid < 0 || !g.gates[nid]) continue;
    GatePtr f = matmul(*g.gates[nid], *gate);
    g.remove_at(row, q);
    g.remove_at(nr, q);
    g.insert_at(nr, f);
    return true;
  }
  for (size_t pr = row; pr-- > 0;) {
    const int pid = g.id_at(pr, q);
    if (pid < 0 || !g.gates[pid]) continue;
    GatePtr f = matmul(*gate, *g.gates[pid]);
    g.remove_at(row, q);
    g.remove_at(pr, q);
    g.insert_at(pr, f);
    return true;
  }
  return false;
}

bool fuse_adjacent_two(Graph &g, size_t row, uint32_t q) {
  const int l = g.id_at(row, q);
  if (l < 0 || !g.gates[l] || g.gates[l]->k() != 2 || g.gates[l]->q[0] != q) return false;
  const int r = g.id_at(row + 1, q);
  if (r < 0 || !g.gates[r] || g.gates[r]->k() != 2 || g.gates[r]->q != g.gates[l]->q) return false;
  GatePtr f = matmul(*g.gates[r], *g.gates[l]);
  g.remove_at(row, q);
  g.remove_at(row + 1, q);
  g.insert_at(row + 1, f);
  return true;
}

void size_two_fusion(Graph &g) {
  size_t n1 = 0;
  for (size_t row = 0; row < g.rows.size(); ++row)
    for (uint32_t q = 0; q < g.n; ++q) n1 += absorb_single(g, row, q);
  if (n1) g.squeeze();
  size_t n2 = 0;
  for (size_t row = 0; row + 1 < g.rows.size(); ++row)
    for (uint32_t q = 0; q < g.n; ++q) n2 += fuse_adjacent_two(g, row, q);
  if (n2) g.squeeze();
}

// ── phase 2 (fusion.rs:168-345) ─────────────────────────────────────────────
size_t union_count(const std::vector<uint32_t> &a, const std::vector<uint32_t> &b) {
  std::vector<uint32_t> u;
  std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(u));
  return u.size();
}

size_t start_fusion(Graph &g, const Cost &cost, double margin, uint32_t cdd, size_t start_row,
                    uint32_t start_q) {
  const int seed_id = g.id_at(start_row, start_q);
  if (seed_id < 0) return 0;
  GatePtr seed = g.gates[seed_id];
  if (seed->q[0] != start_q) return 0;
  std::vector<std::pair<GatePtr, size_t>> tentative{{seed, start_row}};
  std::unordered_set<int> absorbed{seed_id};
  int prod_id = seed_id;
  size_t prod_row = start_row;
  GatePtr prod = seed;
  for (uint32_t q = start_q + 1; q < g.n; ++q) {
    const int cid = g.id_at(prod_row, q);
    if (cid < 0 || absorbed.count(cid)) continue;
    GatePtr cand = g.gates[cid];
    if (union_count(prod->q, cand->q) > cdd) continue;
    tentative.push_back({cand, prod_row});
    absorbed.insert(cid);
    prod_id = g.fuse_same_row(prod_row, prod->q[0], q);
    absorbed.insert(prod_id);
    prod = g.gates[prod_id];
  }
  for (;;) {
    const size_t nr = prod_row + 1;
    if (nr >= g.rows.size()) break;
    bool progressed = false;
    const std::vector<uint32_t> pq = prod->q;
    for (uint32_t q : pq) {
      const int cid = g.id_at(nr, q);
      if (cid < 0 || absorbed.count(cid)) continue;
      GatePtr cand = g.gates[cid];
      if (union_count(prod->q, cand->q) > cdd) continue;
      tentative.push_back({cand, nr});
      absorbed.insert(cid);
      auto res = g.fuse_across(prod_row, prod->q[0], nr, q);
      prod_id = res.first;
      prod_row = res.second;
      absorbed.insert(prod_id);
      prod = g.gates[prod_id];
      progressed = true;
      break;
    }
    if (!progressed) break;
  }
  if (tentative.size() == 1) return 0;
  double old_cost = 0;
  for (auto &t : tentative) old_cost += cost.of(*t.first);
  const double new_cost = cost.of(*prod);
  const double benefit = old_cost / (new_cost + 1e-10) - 1.0;
  if (!(benefit >= margin)) {
    g.remove_at(prod_row, prod->q[0]);
    for (auto &t : tentative) g.insert_at(t.second, t.first);
    return 0;
  }
  return tentative.size() - 1;
}

size_t gate_fusion_pass(Graph &g, const Cost &cost, double margin, uint32_t cdd) {
  size_t nf = 0;
  const size_t nrows = g.rows.size();
  for (size_t row = 0; row < nrows; ++row)
    for (uint32_t q = 0; q < g.n; ++q) nf += start_fusion(g, cost, margin, cdd, row, q);
  if (nf) g.squeeze();
  return nf;
}

// ── trajectory-program construction ─────────────────────────────────────────
// The host half of the batched trajectories, natively: the same program the
// Python builder emits (and a CPU test checks exactly as a channel sequence):
//  * unitary gates collect into a segment; a depolarizing / bit-flip /
//    phase-flip channel marks the last gate on its qubit (an identity is
//    inserted when there is none);
//  * any other channel closes the segment: the segment is fused (size-only
//    cost, width k) and every block is emitted, followed by its Pauli errors
//    moved to the block's end as U_s P U_s^dagger (U_s: the block's gates after
//    the error); amplitude damping on consecutive qubits with one rate merges
//    into one mask; other one-qubit channels are emitted with their Kraus
//    operators sqrt(p_i) K_i.
using Mat = std::vector<cd>;

Mat mat_mul(const Mat &a, const Mat &b, size_t d) {
  Mat c(d * d, cd(0, 0));
  for (size_t r = 0; r < d; ++r)
    for (size_t t = 0; t < d; ++t) {
      const cd x = a[r * d + t];
      if (x == cd(0, 0)) continue;
      for (size_t j = 0; j < d; ++j) c[r * d + j] += x * b[t * d + j];
    }
  return c;
}

Mat dagger(const Mat &a, size_t d) {
  Mat c(d * d);
  for (size_t r = 0; r < d; ++r)
    for (size_t j = 0; j < d; ++j) c[j * d + r] = std::conj(a[r * d + j]);
  return c;
}

Mat identity(size_t d) {
  Mat m(d * d, cd(0, 0));
  for (size_t i = 0; i < d; ++i) m[i * d + i] = 1.0;
  return m;
}

bool close2(const cd *a, const Mat &b, double tol) {
  for (int i = 0; i < 4; ++i)
    if (std::abs(a[i].real() - b[i].real()) > tol || std::abs(a[i].imag() - b[i].imag()) > tol)
      return false;
  return true;
}

const Mat &pauli(int i) {
  static const Mat x{0, 1, 1, 0}, y{0, cd(0, -1), cd(0, 1), 0}, z{1, 0, 0, -1};
  return i == 0 ? x : (i == 1 ? y : z);
}

struct Channel {  // a one-qubit channel: base matrix and weighted branches
  uint32_t q;
  const cd *base;
  std::vector<double> w;
  std::vector<const cd *> k;  // 2 x 2 each
};

// (p, three matrices) for a Pauli channel on an identity base, as the Python
// builder's _is_pauli_channel; empty when it is not one.
bool pauli_channel(const Channel &c, double &p, std::vector<Mat> &mats) {
  const Mat eye = identity(2);
  if (!close2(c.base, eye, 1e-9) || c.k.empty() || !close2(c.k[0], eye, 1e-9)) return false;
  const size_t ne = c.k.size() - 1;
  mats.clear();
  for (size_t i = 1; i < c.k.size(); ++i) {
    int which = -1;
    for (int j = 0; j < 3; ++j)
      if (close2(c.k[i], pauli(j), 1e-9)) which = j;
    if (which < 0) return false;
    mats.push_back(pauli(which));
  }
  if (ne == 3) {
    const double lo = std::min({c.w[1], c.w[2], c.w[3]}), hi = std::max({c.w[1], c.w[2], c.w[3]});
    if (hi - lo > 1e-12 * std::max(1.0, std::abs(c.w[1]))) return false;
    p = c.w[1] + c.w[2] + c.w[3];
    return true;
  }
  if (ne == 1) {
    p = c.w[1];
    mats = {mats[0], mats[0], mats[0]};
    return true;
  }
  return false;
}

// gamma of an amplitude-damping channel (weights p0, p1; K0 = diag(1, s),
// K1 = sqrt(gamma)|0><1| after scaling by sqrt(p)), as _damping_rate; < 0 if not.
double damping_rate(const Channel &c) {
  if (!close2(c.base, identity(2), 1e-9) || c.k.size() != 2) return -1;
  const double s0 = std::sqrt(c.w[0]), s1 = std::sqrt(c.w[1]);
  const cd k00 = s0 * c.k[0][0], k01 = s0 * c.k[0][1], k10 = s0 * c.k[0][2], k11 = s0 * c.k[0][3];
  if (std::abs(k01) > 1e-12 || std::abs(k10) > 1e-12 || std::abs(k00 - 1.0) > 1e-12) return -1;
  const double gamma = 1.0 - std::norm(k11);
  const Mat exp1{0, std::sqrt(std::max(gamma, 0.0)), 0, 0};
  Mat k1(4);
  for (int i = 0; i < 4; ++i) k1[i] = s1 * c.k[1][i];
  if (!close2(k1.data(), exp1, 1e-12)) return -1;
  return gamma;
}

struct TrajBuilder {
  void *prog;
  uint32_t n, fk;
  char *eb;
  size_t el;
  uint32_t stats[4] = {0, 0, 0, 0};  // blocks, error sites, damping ops, channels
  std::vector<GatePtr> seg;
  std::map<int, std::vector<std::tuple<uint32_t, double, std::vector<Mat>>>> markers;
  std::vector<int> last_on;
  uint32_t damp_mask = 0;
  double damp_gamma = 0;

  void fail(const char *what) {
    throw std::runtime_error(std::string(what) + ": " + (eb && el ? eb : ""));
  }
  void emit_gate(const HGate &g) {
    std::vector<cast_complex64_t> m(g.m.size());
    for (size_t e = 0; e < g.m.size(); ++e) m[e] = {g.m[e].real(), g.m[e].imag()};
    if (cast_b200_traj_add_gate(prog, m.data(), g.q.data(), g.k(), eb, el)) fail("add_gate");
    ++stats[0];
  }
  void flush_damp() {
    if (damp_mask) {
      if (cast_b200_traj_add_damping(prog, damp_mask, damp_gamma, eb, el)) fail("add_damping");
      ++stats[2];
    }
    damp_mask = 0;
  }
  void flush() {
    if (seg.empty()) return;
    Graph g;
    g.n = n;
    for (const GatePtr &x : seg) g.insert(x);
    Cost cost{0, fk, 0.0, 0.0, 0.0, 0};
    size_two_fusion(g);
    for (uint32_t cdd = 3; cdd <= fk; ++cdd)
      while (gate_fusion_pass(g, cost, 0.0, cdd) > 0) {
      }
    for (int id : g.live_ids()) {
      const HGate &blk = *g.gates[id];
      emit_gate(blk);
      bool any = false;
      for (int j : blk.prov) any = any || markers.count(j);
      if (!any) continue;
      const size_t d = 1ull << blk.k();
      std::vector<Mat> suffix(blk.prov.size());
      Mat u = identity(d);
      for (size_t pos = blk.prov.size(); pos-- > 0;) {
        suffix[pos] = u;
        u = mat_mul(u, expand(*seg[blk.prov[pos]], blk.q), d);
      }
      for (size_t pos = 0; pos < blk.prov.size(); ++pos) {
        auto it = markers.find(blk.prov[pos]);
        if (it == markers.end()) continue;
        const Mat ud = dagger(suffix[pos], d);
        for (const auto &mk : it->second) {
          std::vector<cast_complex64_t> buf;
          for (const Mat &P : std::get<2>(mk)) {
            HGate h;
            h.q = {std::get<0>(mk)};
            h.m = P;
            const Mat e = mat_mul(mat_mul(suffix[pos], expand(h, blk.q), d), ud, d);
            for (const cd &z : e) buf.push_back({z.real(), z.imag()});
          }
          if (cast_b200_traj_add_pauli_error(prog, std::get<1>(mk), buf.data(), eb, el))
            fail("add_pauli_error");
          ++stats[1];
        }
      }
    }
    seg.clear();
    markers.clear();
    std::fill(last_on.begin(), last_on.end(), -1);
  }
  void unitary(const uint32_t *q, uint32_t k, const cast_complex64_t *m) {
    flush_damp();
    auto h = std::make_shared<HGate>();
    h->q.assign(q, q + k);
    const size_t ne = 1ull << (2 * k);
    h->m.resize(ne);
    for (size_t e = 0; e < ne; ++e) h->m[e] = cd(m[e].re, m[e].im);
    const int idx = (int)seg.size();
    h->prov = {idx};
    seg.push_back(h);
    for (uint32_t b = 0; b < k; ++b) last_on[q[b]] = idx;
  }
  void channel(const Channel &c) {
    double p;
    std::vector<Mat> mats;
    if (pauli_channel(c, p, mats)) {
      flush_damp();
      if (last_on[c.q] < 0) {
        const cast_complex64_t id[4] = {{1, 0}, {0, 0}, {0, 0}, {1, 0}};
        unitary(&c.q, 1, id);
      }
      markers[last_on[c.q]].emplace_back(c.q, p, std::move(mats));
      return;
    }
    flush();  // any other channel closes the segment
    const double gamma = damping_rate(c);
    if (gamma >= 0) {
      if (damp_mask && (std::abs(gamma - damp_gamma) > 1e-15 || ((damp_mask >> c.q) & 1))) flush_damp();
      damp_mask |= 1u << c.q;
      damp_gamma = gamma;
      return;
    }
    flush_damp();
    if (c.k.size() > 4) throw std::runtime_error("trajectory mode supports one-qubit channels with <= 4 Kraus operators");
    std::vector<cast_complex64_t> kr;
    for (size_t i = 0; i < c.k.size(); ++i) {
      const double s = std::sqrt(c.w[i]);
      for (int e = 0; e < 4; ++e) kr.push_back({s * c.k[i][e].real(), s * c.k[i][e].imag()});
    }
    if (cast_b200_traj_add_channel(prog, c.q, kr.data(), (uint32_t)c.k.size(), eb, el)) fail("add_channel");
    ++stats[3];
  }
};

constexpr uint32_t kFusedMagic = 0xCB20F05Eu;
struct Fused {
  uint32_t magic = kFusedMagic;
  std::vector<GatePtr> gates;
};

}  // namespace

extern "C" {

void *cast_b200_fuse(uint32_t n_qubits, uint32_t n_gates, const uint32_t *gate_k,
                     const uint32_t *qubits, const cast_complex64_t *matrices,
                     const cast_b200_fusion_config_t *config, char *err_buf, size_t err_buf_len) {
  if ((n_gates && (!gate_k || !qubits || !matrices)) || !config) {
    cb2::write_err(err_buf, err_buf_len, "arguments must not be null");
    return nullptr;
  }
  if (config->size_max < 2 || config->size_max > cb2::kMaxGateQubits) {
    cb2::write_err(err_buf, err_buf_len, "size_max must be 2.." + std::to_string(cb2::kMaxGateQubits));
    return nullptr;
  }
  try {
    Graph g;
    g.n = n_qubits;
    size_t qo = 0, mo = 0;
    for (uint32_t i = 0; i < n_gates; ++i) {
      auto h = std::make_shared<HGate>();
      const uint32_t k = gate_k[i];
      if (k == 0 || k > cb2::kMaxGateQubits) throw std::runtime_error("gate size out of range");
      h->q.assign(qubits + qo, qubits + qo + k);
      for (uint32_t b = 0; b < k; ++b) {
        if (h->q[b] >= n_qubits) throw std::runtime_error("gate qubit out of range");
        if (b && h->q[b - 1] >= h->q[b]) throw std::runtime_error("gate qubits must be ascending");
      }
      const size_t ne = 1ull << (2 * k);
      h->m.resize(ne);
      for (size_t e = 0; e < ne; ++e) h->m[e] = cd(matrices[mo + e].re, matrices[mo + e].im);
      qo += k;
      mo += ne;
      g.insert(h);
    }
    Cost cost{(int)config->cost_kind, config->size_max, config->zero_tol, config->crossover_ai,
              config->tensor_crossover_ai, config->tensor_min_k};
    if (cost.kind == 1 && !(cost.crossover > 0)) throw std::runtime_error("crossover_ai must be > 0");
    size_two_fusion(g);
    for (uint32_t cdd = 3; cdd <= config->size_max; ++cdd)
      while (gate_fusion_pass(g, cost, config->benefit_margin, cdd) > 0) {
      }
    Fused *f = new Fused;
    for (int id : g.live_ids()) f->gates.push_back(g.gates[id]);
    cb2::clear_err(err_buf, err_buf_len);
    return f;
  } catch (const std::exception &e) {
    cb2::write_err(err_buf, err_buf_len, e.what());
    return nullptr;
  }
}

uint32_t cast_b200_fused_num_gates(const void *fused) {
  const Fused *f = static_cast<const Fused *>(fused);
  return f && f->magic == kFusedMagic ? (uint32_t)f->gates.size() : 0;
}

int cast_b200_fused_gate(const void *fused, uint32_t index, uint32_t *out_k, uint32_t *out_qubits,
                         cast_complex64_t *out_matrix) {
  const Fused *f = static_cast<const Fused *>(fused);
  if (!f || f->magic != kFusedMagic || index >= f->gates.size() || !out_k) return 1;
  const HGate &g = *f->gates[index];
  *out_k = g.k();
  if (out_qubits)
    for (uint32_t b = 0; b < g.k(); ++b) out_qubits[b] = g.q[b];
  if (out_matrix)
    for (size_t e = 0; e < g.m.size(); ++e) out_matrix[e] = {g.m[e].real(), g.m[e].imag()};
  return 0;
}

int cast_b200_program_add_fused(void *program, const void *fused, char *err_buf,
                                size_t err_buf_len) {
  const Fused *f = static_cast<const Fused *>(fused);
  if (!f || f->magic != kFusedMagic) {
    cb2::write_err(err_buf, err_buf_len, "invalid fused-circuit handle");
    return 1;
  }
  std::vector<cast_complex64_t> buf;
  for (const GatePtr &g : f->gates) {
    buf.resize(g->m.size());
    for (size_t e = 0; e < g->m.size(); ++e) buf[e] = {g->m[e].real(), g->m[e].imag()};
    if (cast_b200_program_add_gate(program, buf.data(), g->q.data(), g->k(), err_buf, err_buf_len))
      return 1;
  }
  cb2::clear_err(err_buf, err_buf_len);
  return 0;
}

void cast_b200_fused_free(void *fused) {
  Fused *f = static_cast<Fused *>(fused);
  if (!f || f->magic != kFusedMagic) return;
  f->magic = 0;
  delete f;
}

int cast_b200_traj_build(void *program, uint32_t n_items, const uint32_t *kind, const uint32_t *k,
                         const uint32_t *qubits, const cast_complex64_t *matrices,
                         const uint32_t *n_branches, const double *weights, uint32_t fusion_k,
                         uint32_t *out_stats, char *err_buf, size_t err_buf_len) {
  const uint32_t n = cast_b200_traj_num_qubits(program);
  if (!n || (n_items && (!kind || !k || !qubits || !matrices || !n_branches))) {
    cb2::write_err(err_buf, err_buf_len, "invalid trajectory program or circuit arrays");
    return 1;
  }
  if (fusion_k < 1 || fusion_k > 4) {
    cb2::write_err(err_buf, err_buf_len, "trajectory fusion width must be 1..4");
    return 1;
  }
  try {
    TrajBuilder tb{program, n, fusion_k, err_buf, err_buf_len};
    tb.last_on.assign(n, -1);
    size_t qo = 0, mo = 0, wo = 0;
    for (uint32_t i = 0; i < n_items; ++i) {
      const uint32_t kk = k[i];
      if (kk == 0 || kk > cb2::kMaxGateQubits) throw std::runtime_error("gate size out of range");
      for (uint32_t b = 0; b < kk; ++b) {
        if (qubits[qo + b] >= n) throw std::runtime_error("qubit out of range");
        if (b && qubits[qo + b - 1] >= qubits[qo + b]) throw std::runtime_error("qubits must be ascending");
      }
      if (kind[i] == 0) {
        tb.unitary(qubits + qo, kk, matrices + mo);
        mo += 1ull << (2 * kk);
      } else {
        if (kk != 1 || !weights) throw std::runtime_error("trajectory mode supports one-qubit channels");
        Channel c;
        c.q = qubits[qo];
        c.base = reinterpret_cast<const cd *>(matrices + mo);
        mo += 4;
        for (uint32_t b = 0; b < n_branches[i]; ++b) {
          c.w.push_back(weights[wo + b]);
          c.k.push_back(reinterpret_cast<const cd *>(matrices + mo));
          mo += 4;
        }
        wo += n_branches[i];
        tb.channel(c);
      }
      qo += kk;
    }
    tb.flush();
    tb.flush_damp();
    if (out_stats)
      for (int j = 0; j < 4; ++j) out_stats[j] = tb.stats[j];
    cb2::clear_err(err_buf, err_buf_len);
    return 0;
  } catch (const std::exception &e) {
    cb2::write_err(err_buf, err_buf_len, e.what());
    return 1;
  }
}

}  // extern "C"
