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
//     on the tensor-core path are judged against the tensor pipe's ceiling.
// Unitary gates only (the state-vector path); noisy circuits are fused on the
// host-side Python mirror, which keeps the Kraus branches.
#include "../../include/cast_b200.h"
#include "internal.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <exception>
#include <memory>
#include <set>
#include <unordered_set>
#include <vector>

namespace {

using cd = std::complex<double>;

struct HGate {
  std::vector<uint32_t> q;  // ascending
  std::vector<cd> m;        // row-major 2^k x 2^k
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

}  // extern "C"
