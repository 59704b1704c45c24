/*
 * CPU parity oracle for the gate-application path.  TEST INFRASTRUCTURE ONLY:
 * this file is a scalar FP64 restatement of the reference simulator's CPU
 * semantics (narix10yc/cast_simulator, a Rust crate) and is only ever loaded by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, to check results.
 * The product (cast_simulator_b200) never links, imports or calls it.
 *
 * Every routine cites the reference code it restates (path:line inside the
 * reference project).  The reference cannot be compiled here (Rust + LLVM, no
 * cargo/rustc/llvm-config), so the oracle is pinned by the reference's own
 * known-answer tests and by golden vectors derived from its QASM fixture
 * tests/assets/qft_14.qasm (see tests/golden/make_golden.py).
 *
 * Conventions (identical to the reference):
 *  - statevector: interleaved complex128 [re0, im0, re1, im1, ...]
 *    (src/cuda/statevector.rs:52-57: n_elements = 2 * 2^n);
 *  - a k-qubit gate matrix is row-major 2^k x 2^k complex, interleaved;
 *    gate qubit qubits[b] is bit b of the local matrix index
 *    (src/cpp/cuda/cuda_gen.cpp:241-246), qubits ascending.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_MAX_K 12

/* ------------------------------------------------------------------------ */
/* Seeded RNG: SplitMix64 (public-domain algorithm by S. Vigna).             */
/* The reference seeds rand 0.8.5 StdRng (ChaCha12); that stream cannot be   */
/* reproduced without a Rust toolchain, so circuits are defined on this      */
/* generator on both sides of every parity check.                            */
/* ------------------------------------------------------------------------ */
typedef struct { uint64_t s; } or_rng;

static uint64_t or_next(or_rng *r) {
  uint64_t z = (r->s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* uniform double in [0, 1) with 53 random bits */
static double or_uniform(or_rng *r) { return (double)(or_next(r) >> 11) * 0x1.0p-53; }

uint64_t or_splitmix64(uint64_t *state) {
  or_rng r = {*state};
  uint64_t v = or_next(&r);
  *state = r.s;
  return v;
}

double or_uniform_from(uint64_t *state) {
  or_rng r = {*state};
  double v = or_uniform(&r);
  *state = r.s;
  return v;
}

/* ------------------------------------------------------------------------ */
/* Named gate matrices: src/types/matrix.rs:51-215.                          */
/* ------------------------------------------------------------------------ */
enum {
  OR_I = 0, OR_X, OR_Y, OR_Z, OR_H, OR_S, OR_T, OR_RX, OR_RY, OR_RZ, OR_U3,
  OR_CX, OR_CZ, OR_CP, OR_SWAP, OR_CCX
};

static void set_c(double *m, int dim, int r, int c, double re, double im) {
  m[2 * (r * dim + c)] = re;
  m[2 * (r * dim + c) + 1] = im;
}

/* Writes the matrix of gate `kind` into `out` (interleaved, row-major) and
 * returns its qubit count.  params = {theta, phi, lambda} as needed. */
int or_named_matrix(int kind, const double *params, double *out) {
  int k = 1;
  if (kind >= OR_CX && kind <= OR_SWAP) k = 2;
  if (kind == OR_CCX) k = 3;
  const int dim = 1 << k;
  memset(out, 0, sizeof(double) * 2 * dim * dim);
  const double p0 = params ? params[0] : 0.0;
  const double p1 = params ? params[1] : 0.0;
  const double p2 = params ? params[2] : 0.0;
  switch (kind) {
  case OR_I: set_c(out, 2, 0, 0, 1, 0); set_c(out, 2, 1, 1, 1, 0); break;
  case OR_X: set_c(out, 2, 0, 1, 1, 0); set_c(out, 2, 1, 0, 1, 0); break;        /* matrix.rs:59-61 */
  case OR_Y: set_c(out, 2, 0, 1, 0, -1); set_c(out, 2, 1, 0, 0, 1); break;       /* matrix.rs:63-73 */
  case OR_Z: set_c(out, 2, 0, 0, 1, 0); set_c(out, 2, 1, 1, -1, 0); break;       /* matrix.rs:75-77 */
  case OR_H: {                                                                    /* matrix.rs:79-82 */
    const double s = 0.70710678118654752440;
    set_c(out, 2, 0, 0, s, 0); set_c(out, 2, 0, 1, s, 0);
    set_c(out, 2, 1, 0, s, 0); set_c(out, 2, 1, 1, -s, 0);
    break;
  }
  case OR_S: set_c(out, 2, 0, 0, 1, 0); set_c(out, 2, 1, 1, 0, 1); break;        /* matrix.rs:84-94 */
  case OR_T: {                                                                    /* matrix.rs:96-107 */
    const double ph = 0.78539816339744830962;
    set_c(out, 2, 0, 0, 1, 0); set_c(out, 2, 1, 1, cos(ph), sin(ph));
    break;
  }
  case OR_RX: {                                                                   /* matrix.rs:109-121 */
    const double c = cos(p0 * 0.5), s = sin(p0 * 0.5);
    set_c(out, 2, 0, 0, c, 0); set_c(out, 2, 0, 1, 0, -s);
    set_c(out, 2, 1, 0, 0, -s); set_c(out, 2, 1, 1, c, 0);
    break;
  }
  case OR_RY: {                                                                   /* matrix.rs:123-127 */
    const double c = cos(p0 * 0.5), s = sin(p0 * 0.5);
    set_c(out, 2, 0, 0, c, 0); set_c(out, 2, 0, 1, -s, 0);
    set_c(out, 2, 1, 0, s, 0); set_c(out, 2, 1, 1, c, 0);
    break;
  }
  case OR_RZ: {                                                                   /* matrix.rs:129-141 */
    const double c = cos(p0 * 0.5), s = sin(p0 * 0.5);
    set_c(out, 2, 0, 0, c, -s); set_c(out, 2, 1, 1, c, s);
    break;
  }
  case OR_U3: {                                                                   /* matrix.rs:143-158 */
    const double c = cos(p0 * 0.5), s = sin(p0 * 0.5);
    const double epr = cos(p1), epi = sin(p1);           /* e^{i phi} */
    const double elr = cos(p2), eli = sin(p2);           /* e^{i lambda} */
    const double eplr = cos(p1 + p2), epli = sin(p1 + p2);
    set_c(out, 2, 0, 0, c, 0.0);
    set_c(out, 2, 0, 1, -elr * s, -eli * s);
    set_c(out, 2, 1, 0, epr * s, epi * s);
    set_c(out, 2, 1, 1, eplr * c, epli * c);
    break;
  }
  case OR_CX:                                                                     /* matrix.rs:160-170 */
    set_c(out, 4, 0, 0, 1, 0); set_c(out, 4, 1, 3, 1, 0);
    set_c(out, 4, 2, 2, 1, 0); set_c(out, 4, 3, 1, 1, 0);
    break;
  case OR_CZ:                                                                     /* matrix.rs:172-182 */
    set_c(out, 4, 0, 0, 1, 0); set_c(out, 4, 1, 1, 1, 0);
    set_c(out, 4, 2, 2, 1, 0); set_c(out, 4, 3, 3, -1, 0);
    break;
  case OR_CP:                                                                     /* matrix.rs:184-189 */
    set_c(out, 4, 0, 0, 1, 0); set_c(out, 4, 1, 1, 1, 0);
    set_c(out, 4, 2, 2, 1, 0); set_c(out, 4, 3, 3, cos(p0), sin(p0));
    break;
  case OR_SWAP:                                                                   /* matrix.rs:191-201 */
    set_c(out, 4, 0, 0, 1, 0); set_c(out, 4, 1, 2, 1, 0);
    set_c(out, 4, 2, 1, 1, 0); set_c(out, 4, 3, 3, 1, 0);
    break;
  case OR_CCX:                                                                    /* matrix.rs:203-210 */
    for (int i = 0; i < 6; ++i) set_c(out, 8, i, i, 1, 0);
    set_c(out, 8, 6, 7, 1, 0); set_c(out, 8, 7, 6, 1, 0);
    break;
  default:
    return -1;
  }
  return k;
}

/* ------------------------------------------------------------------------ */
/* Qubit canonicalisation: src/types/gate.rs:483-521, 575-595.               */
/* Sort qubits ascending; result[i][j] = input[map(i)][map(j)] where map     */
/* scatters bit p of i to the original position of the qubit now at p.      */
/* Returns 0, or -1 when two qubits are equal (gate.rs:490-494).            */
/* ------------------------------------------------------------------------ */
int or_canonicalize(double *mat, uint32_t *qubits, uint32_t k) {
  if (k > OR_MAX_K) return -2;
  uint32_t order[OR_MAX_K];
  for (uint32_t i = 0; i < k; ++i) order[i] = i;
  /* stable insertion sort of positions by qubit */
  for (uint32_t i = 1; i < k; ++i) {
    uint32_t v = order[i];
    int j = (int)i - 1;
    while (j >= 0 && qubits[order[j]] > qubits[v]) { order[j + 1] = order[j]; --j; }
    order[j + 1] = v;
  }
  uint32_t sorted[OR_MAX_K];
  for (uint32_t i = 0; i < k; ++i) sorted[i] = qubits[order[i]];
  for (uint32_t i = 1; i < k; ++i)
    if (sorted[i - 1] >= sorted[i]) return -1;
  int identity = 1;
  for (uint32_t i = 0; i < k; ++i) identity &= (order[i] == i);
  memcpy(qubits, sorted, sizeof(uint32_t) * k);
  if (identity) return 0;
  const size_t dim = (size_t)1 << k;
  size_t *map = (size_t *)malloc(sizeof(size_t) * dim);
  double *tmp = (double *)malloc(sizeof(double) * 2 * dim * dim);
  for (size_t i = 0; i < dim; ++i) {
    size_t o = 0;
    for (uint32_t p = 0; p < k; ++p)
      if ((i >> p) & 1u) o |= (size_t)1 << order[p];
    map[i] = o;
  }
  for (size_t r = 0; r < dim; ++r)
    for (size_t c = 0; c < dim; ++c) {
      tmp[2 * (r * dim + c)] = mat[2 * (map[r] * dim + map[c])];
      tmp[2 * (r * dim + c) + 1] = mat[2 * (map[r] * dim + map[c]) + 1];
    }
  memcpy(mat, tmp, sizeof(double) * 2 * dim * dim);
  free(map);
  free(tmp);
  return 0;
}

/* Sorted union of two ascending qubit lists: gate.rs:612-648. */
static uint32_t union_qubits(const uint32_t *a, uint32_t ka, const uint32_t *b, uint32_t kb,
                             uint32_t *out) {
  uint32_t i = 0, j = 0, n = 0;
  while (i < ka || j < kb) {
    if (i == ka) out[n++] = b[j++];
    else if (j == kb) out[n++] = a[i++];
    else if (a[i] < b[j]) out[n++] = a[i++];
    else if (a[i] > b[j]) out[n++] = b[j++];
    else { out[n++] = a[i++]; ++j; }
  }
  return n;
}

/* expand_matrix: gate.rs:436-468 (identity on the union's other wires). */
static void expand_matrix(const double *m, const uint32_t *gq, uint32_t gk, const uint32_t *uq,
                          uint32_t uk, double *out) {
  const size_t udim = (size_t)1 << uk;
  uint32_t pos[OR_MAX_K];
  size_t tmask = 0;
  for (uint32_t t = 0; t < gk; ++t) {
    for (uint32_t u = 0; u < uk; ++u)
      if (uq[u] == gq[t]) pos[t] = u;
    tmask |= (size_t)1 << pos[t];
  }
  const size_t gdim = (size_t)1 << gk;
  memset(out, 0, sizeof(double) * 2 * udim * udim);
  for (size_t r = 0; r < udim; ++r)
    for (size_t c = 0; c < udim; ++c) {
      if (((r ^ c) & ~tmask) != 0) continue;
      size_t gr = 0, gc = 0;
      for (uint32_t t = 0; t < gk; ++t) {
        gr |= ((r >> pos[t]) & 1u) << t;
        gc |= ((c >> pos[t]) & 1u) << t;
      }
      out[2 * (r * udim + c)] = m[2 * (gr * gdim + gc)];
      out[2 * (r * udim + c) + 1] = m[2 * (gr * gdim + gc) + 1];
    }
}

static void cmatmul(const double *a, const double *b, size_t dim, double *out) {
  for (size_t r = 0; r < dim; ++r)
    for (size_t c = 0; c < dim; ++c) {
      double re = 0.0, im = 0.0;
      for (size_t t = 0; t < dim; ++t) {
        const double ar = a[2 * (r * dim + t)], ai = a[2 * (r * dim + t) + 1];
        const double br = b[2 * (t * dim + c)], bi = b[2 * (t * dim + c) + 1];
        re += ar * br - ai * bi;
        im += ar * bi + ai * br;
      }
      out[2 * (r * dim + c)] = re;
      out[2 * (r * dim + c) + 1] = im;
    }
}

/* QuantumGate::matmul (unitary part): gate.rs:280-284, 319.
 * out = A * B on the union of qubits (B applied first).  Returns union size. */
int or_matmul(const double *ma, const uint32_t *qa, uint32_t ka, const double *mb,
              const uint32_t *qb, uint32_t kb, double *out, uint32_t *qout) {
  uint32_t uq[2 * OR_MAX_K];
  const uint32_t uk = union_qubits(qa, ka, qb, kb, uq);
  if (uk > OR_MAX_K) return -1;
  const size_t dim = (size_t)1 << uk;
  double *ea = (double *)malloc(sizeof(double) * 2 * dim * dim);
  double *eb = (double *)malloc(sizeof(double) * 2 * dim * dim);
  expand_matrix(ma, qa, ka, uq, uk, ea);
  expand_matrix(mb, qb, kb, uq, uk, eb);
  cmatmul(ea, eb, dim, out);
  memcpy(qout, uq, sizeof(uint32_t) * uk);
  free(ea);
  free(eb);
  return (int)uk;
}

/* superoperator_of: gate.rs:662-680.  S[r,c] = U[r%d, c%d] * conj(U[r/d, c/d]). */
void or_superop_accumulate(const double *u, uint32_t k, double weight, double *s) {
  const size_t d = (size_t)1 << k, sd = d * d;
  for (size_t r = 0; r < sd; ++r)
    for (size_t c = 0; c < sd; ++c) {
      const size_t ik = r % d, ib = r / d, jk = c % d, jb = c / d;
      const double ar = u[2 * (ik * d + jk)], ai = u[2 * (ik * d + jk) + 1];
      const double br = u[2 * (ib * d + jb)], bi = -u[2 * (ib * d + jb) + 1];
      s[2 * (r * sd + c)] += weight * (ar * br - ai * bi);
      s[2 * (r * sd + c) + 1] += weight * (ar * bi + ai * br);
    }
}

/* ------------------------------------------------------------------------ */
/* Scalar gate application with bit-deposit addressing:                      */
/* CPUStatevectorData::apply_gate, src/cpu/statevector.rs:469-516, and       */
/* pdep_usize, statevector.rs:592-606.  qubits must be ascending.            */
/* ------------------------------------------------------------------------ */
static uint64_t pdep(uint64_t src, uint64_t mask) {
  uint64_t out = 0, bit = 0;
  for (int d = 0; d < 64; ++d) {
    if (!((mask >> d) & 1ull)) continue;
    if ((src >> bit) & 1ull) out |= 1ull << d;
    ++bit;
  }
  return out;
}

int or_apply_gate(double *sv, uint32_t n, const double *mat, const uint32_t *qubits, uint32_t k) {
  if (k == 0 || k > OR_MAX_K || k > n) return -1;
  for (uint32_t i = 0; i < k; ++i) {
    if (qubits[i] >= n) return -1;
    if (i && qubits[i - 1] >= qubits[i]) return -1;
  }
  uint64_t tmask = 0;
  for (uint32_t i = 0; i < k; ++i) tmask |= 1ull << qubits[i];
  const uint64_t full = (n == 64) ? ~0ull : ((1ull << n) - 1);
  const uint64_t task_mask = full ^ tmask;
  const uint64_t n_tasks = 1ull << (n - k);
  const size_t dim = (size_t)1 << k;
  uint64_t *idx = (uint64_t *)malloc(sizeof(uint64_t) * dim);
  uint64_t *off = (uint64_t *)malloc(sizeof(uint64_t) * dim);
  double *upd = (double *)malloc(sizeof(double) * 2 * dim);
  for (size_t a = 0; a < dim; ++a) off[a] = pdep(a, tmask);
  /* pdep of consecutive task ids: increment within the task mask */
  uint64_t dep = 0;
  for (uint64_t t = 0; t < n_tasks; ++t) {
    for (size_t a = 0; a < dim; ++a) idx[a] = dep | off[a];
    for (size_t r = 0; r < dim; ++r) {
      double re = 0.0, im = 0.0;
      for (size_t c = 0; c < dim; ++c) {
        const double mr = mat[2 * (r * dim + c)], mi = mat[2 * (r * dim + c) + 1];
        const double xr = sv[2 * idx[c]], xi = sv[2 * idx[c] + 1];
        re += mr * xr - mi * xi;
        im += mr * xi + mi * xr;
      }
      upd[2 * r] = re;
      upd[2 * r + 1] = im;
    }
    for (size_t r = 0; r < dim; ++r) {
      sv[2 * idx[r]] = upd[2 * r];
      sv[2 * idx[r] + 1] = upd[2 * r + 1];
    }
    dep = (dep - task_mask) & task_mask; /* next value with bits only in task_mask */
  }
  free(idx);
  free(off);
  free(upd);
  return 0;
}

/* Plain PDEP exported for tests of the addressing rule. */
uint64_t or_pdep(uint64_t src, uint64_t mask) { return pdep(src, mask); }

/* ------------------------------------------------------------------------ */
/* Sparsity classification of matrix scalars, src/cpp/cuda/cuda_gen.cpp:84-103:
 * |v| < ztol/K -> 0, |v-1| < otol/K -> 1, |v+1| < otol/K -> -1 (K = 2^k);
 * when `f32` is set the remaining immediates are rounded to float.        */
/* ------------------------------------------------------------------------ */
void or_snap_matrix(double *m, uint32_t k, double ztol, double otol, int f32) {
  const size_t dim = (size_t)1 << k;
  const double K = (double)dim;
  const double zt = ztol / K, ot = otol / K;
  for (size_t i = 0; i < 2 * dim * dim; ++i) {
    const double v = m[i];
    if (ztol > 0.0 && fabs(v) < zt) m[i] = 0.0;
    else if (otol > 0.0 && fabs(v - 1.0) < ot) m[i] = 1.0;
    else if (otol > 0.0 && fabs(v + 1.0) < ot) m[i] = -1.0;
    else if (f32) m[i] = (double)(float)v;
  }
}

/* ------------------------------------------------------------------------ */
/* States                                                                    */
/* ------------------------------------------------------------------------ */
/* Deterministic normalised state amp_i ~ (i+1, 0.5 i - 0.25):
 * tests/cpu_cuda_compare.rs:54-69. */
void or_seeded_state(double *sv, uint32_t n) {
  const uint64_t len = 1ull << n;
  double norm = 0.0;
  for (uint64_t i = 0; i < len; ++i) {
    sv[2 * i] = (double)i + 1.0;
    sv[2 * i + 1] = (double)i * 0.5 - 0.25;
    norm += sv[2 * i] * sv[2 * i] + sv[2 * i + 1] * sv[2 * i + 1];
  }
  norm = sqrt(norm);
  for (uint64_t i = 0; i < 2 * len; ++i) sv[i] /= norm;
}

/* i.i.d. N(0,1) re/im per amplitude, then normalised: the semantics of
 * CPUStatevectorData::randomize, src/cpu/statevector.rs:459-465
 * (Box-Muller on SplitMix64 instead of rand_distr's ziggurat). */
void or_random_state(double *sv, uint32_t n, uint64_t seed) {
  or_rng r = {seed};
  const uint64_t len = 1ull << n;
  double norm = 0.0;
  for (uint64_t i = 0; i < len; ++i) {
    const double u1 = 1.0 - or_uniform(&r); /* (0, 1] */
    const double u2 = or_uniform(&r);
    const double rad = sqrt(-2.0 * log(u1));
    sv[2 * i] = rad * cos(6.283185307179586477 * u2);
    sv[2 * i + 1] = rad * sin(6.283185307179586477 * u2);
    norm += sv[2 * i] * sv[2 * i] + sv[2 * i + 1] * sv[2 * i + 1];
  }
  norm = sqrt(norm);
  for (uint64_t i = 0; i < 2 * len; ++i) sv[i] /= norm;
}

/* <a|b> over `len` amplitudes. */
void or_inner(const double *a, const double *b, uint64_t len, double *out_re, double *out_im) {
  double re = 0.0, im = 0.0;
  for (uint64_t i = 0; i < len; ++i) {
    re += a[2 * i] * b[2 * i] + a[2 * i + 1] * b[2 * i + 1];
    im += a[2 * i] * b[2 * i + 1] - a[2 * i + 1] * b[2 * i];
  }
  *out_re = re;
  *out_im = im;
}

/* ------------------------------------------------------------------------ */
/* Circuit builders.  Builder gates have k <= 3: {k, qubits[3], 4x4 max}.    */
/* Qubits are canonical (ascending) after construction, as in                */
/* QuantumGate::new (gate.rs:32-45).                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint32_t k;
  uint32_t qubits[3];
  double mat[2 * 64];
} or_gate;

static int push_named(or_gate *out, uint32_t cap, uint32_t *n, int kind, const double *params,
                      uint32_t q0, uint32_t q1, uint32_t q2) {
  if (*n >= cap) { ++*n; return 0; }
  or_gate *g = &out[*n];
  memset(g, 0, sizeof(*g));
  const int k = or_named_matrix(kind, params, g->mat);
  g->k = (uint32_t)k;
  g->qubits[0] = q0; g->qubits[1] = q1; g->qubits[2] = q2;
  if (or_canonicalize(g->mat, g->qubits, g->k) != 0) return -1;
  ++*n;
  return 0;
}

/* QuantumCircuit::qft (CP form): src/types/circuit.rs:151-171.
 * For i: H(i); for j>i: CP(pi/2^(j-i), ctrl=j, targ=i); then SWAP(i, n-1-i). */
uint32_t or_build_qft_cp(uint32_t nq, int swap, or_gate *out, uint32_t cap) {
  uint32_t n = 0;
  for (uint32_t i = 0; i < nq; ++i) {
    push_named(out, cap, &n, OR_H, NULL, i, 0, 0);
    for (uint32_t j = i + 1; j < nq; ++j) {
      double th = 3.14159265358979323846 / (double)(1ull << (j - i));
      push_named(out, cap, &n, OR_CP, &th, j, i, 0);
    }
  }
  if (swap)
    for (uint32_t i = 0; i < nq / 2; ++i) push_named(out, cap, &n, OR_SWAP, NULL, i, nq - 1 - i, 0);
  return n;
}

/* QFT with each CP(theta) decomposed into CX + single-qubit phases, the
 * construction of the reference fixture tests/assets/qft_14.qasm:3-8:
 * u3(0,0,t/2) c; cx c,t; u3(0,0,-t/2) t; cx c,t; u3(0,0,t/2) t. */
uint32_t or_build_qft_cx(uint32_t nq, or_gate *out, uint32_t cap) {
  uint32_t n = 0;
  const double pi = 3.14159265358979323846;
  for (uint32_t i = 0; i < nq; ++i) {
    push_named(out, cap, &n, OR_H, NULL, i, 0, 0);
    for (uint32_t j = i + 1; j < nq; ++j) {
      const double half = pi / (double)(1ull << (j - i + 1));
      double pp[3] = {0.0, 0.0, half};
      double pm[3] = {0.0, 0.0, -half};
      push_named(out, cap, &n, OR_U3, pp, i, 0, 0);
      push_named(out, cap, &n, OR_CX, NULL, i, j, 0);
      push_named(out, cap, &n, OR_U3, pm, j, 0, 0);
      push_named(out, cap, &n, OR_CX, NULL, i, j, 0);
      push_named(out, cap, &n, OR_U3, pp, j, 0, 0);
    }
  }
  for (uint32_t i = 0; i < nq / 2; ++i) push_named(out, cap, &n, OR_SWAP, NULL, i, nq - 1 - i, 0);
  return n;
}

/* Random brickwork: each layer U3(theta, phi, lambda) on every qubit, angles
 * uniform in [0, 2pi) drawn in qubit order (theta, phi, lambda), then CZ on
 * (0,1),(2,3),... for even layers and (1,2),(3,4),... for odd layers. */
uint32_t or_build_brickwork(uint32_t nq, uint32_t depth, uint64_t seed, or_gate *out,
                            uint32_t cap) {
  or_rng r = {seed};
  uint32_t n = 0;
  const double tau = 6.283185307179586477;
  for (uint32_t l = 0; l < depth; ++l) {
    for (uint32_t q = 0; q < nq; ++q) {
      double a[3];
      a[0] = tau * or_uniform(&r);
      a[1] = tau * or_uniform(&r);
      a[2] = tau * or_uniform(&r);
      push_named(out, cap, &n, OR_U3, a, q, 0, 0);
    }
    for (uint32_t q = l & 1u; q + 1 < nq; q += 2) push_named(out, cap, &n, OR_CZ, NULL, q, q + 1, 0);
  }
  return n;
}

/* ------------------------------------------------------------------------ */
/* Density-matrix channel application: to_density_matrix_gate               */
/* (gate.rs:236-257) + prepare_gates lifting (simulator/mod.rs:605-611).     */
/* rho is the vectorised 2n-qubit state, rho[i | j<<n] = rho_{ij}.           */
/* kraus: nb matrices of 2^k x 2^k, S = sum_b w_b K_b (x) conj(K_b) on the    */
/* virtual qubits [q..., q+n...].                                           */
/* ------------------------------------------------------------------------ */
int or_dm_apply_channel(double *rho, uint32_t n, const double *kraus, const double *weights,
                        uint32_t nb, const uint32_t *qubits, uint32_t k) {
  if (2 * k > OR_MAX_K) return -1;
  const size_t d = (size_t)1 << k, sd = d * d;
  double *s = (double *)calloc(2 * sd * sd, sizeof(double));
  for (uint32_t b = 0; b < nb; ++b) or_superop_accumulate(kraus + 2 * d * d * b, k, weights[b], s);
  uint32_t vq[2 * OR_MAX_K];
  for (uint32_t i = 0; i < k; ++i) {
    vq[i] = qubits[i];
    vq[i + k] = qubits[i] + n;
  }
  const int rc = or_apply_gate(rho, 2 * n, s, vq, 2 * k);
  free(s);
  return rc;
}

/* Diagonal of the vectorised density matrix: populations (simulator/mod.rs:387-395). */
void or_dm_populations(const double *rho, uint32_t n, double *out) {
  const uint64_t dim = 1ull << n;
  for (uint64_t i = 0; i < dim; ++i) out[i] = rho[2 * (i | (i << n))];
}
