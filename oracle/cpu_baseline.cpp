// Threaded SIMD CPU baseline (timed beside the GPU numbers; TEST/BENCH
// INFRASTRUCTURE ONLY, never linked by the product).
//
// A C++ restatement of the semantics of the reference's CPU gate kernels
// (narix10yc/cast_simulator; its own LLVM-ORC JIT cannot be built here):
//  - split re/im SIMD layout: amplitude i has its real part at
//    insert_zero_to_bit(i, s) and its imaginary part at that | (1 << s)
//    (src/cpu/statevector.rs:170-186, 583-587), s = log2(lanes per register);
//  - matrix scalars within ztol of 0 are skipped and within otol of +-1 turn
//    into adds/subtracts, WITHOUT the 1/K scaling of the CUDA generator
//    (src/cpu/kernel.rs:41-62; src/cpp/cuda/cuda_gen.cpp:79-83);
//  - the task range [0, 2^(n-k)) is split into contiguous chunks, one per
//    std::thread (src/cpu/kernel.rs:371-434).
// Gates whose targets all sit at or above s run fully vectorised (one task =
// 2^s consecutive amplitudes); gates with a target below s run a scalar loop
// over the same layout.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

typedef double v4d __attribute__((vector_size(32)));
typedef float v8f __attribute__((vector_size(32)));

template <typename T> struct Lanes;
template <> struct Lanes<double> {  // 4 x f64 per 256-bit register
  static constexpr int S = 2;
  typedef v4d V;
};
template <> struct Lanes<float> {  // 8 x f32 per 256-bit register
  static constexpr int S = 3;
  typedef v8f V;
};

struct Sv {
  uint32_t n;
  int f32;
  void *data;
  size_t scalars;
};

inline uint64_t insert_zero(uint64_t x, int bit) {
  const uint64_t lo = (1ull << bit) - 1;
  return (x & lo) + ((x & ~lo) << 1);
}

inline uint64_t pdep(uint64_t src, uint64_t mask) {
  uint64_t out = 0;
  for (uint64_t bit = 1; mask; bit <<= 1) {
    const uint64_t low = mask & (~mask + 1);
    if (src & bit) out |= low;
    mask ^= low;
  }
  return out;
}

enum Kind : int8_t { kZero = 0, kOne = 1, kMinusOne = -1, kImm = 2 };

struct Entry {
  Kind kind;
  double v;
};

template <typename T> struct Mat {
  int k;
  int dim;
  std::vector<Entry> re, im;
};

template <typename T> Mat<T> classify(const double *m, int k, double ztol, double otol) {
  Mat<T> out;
  out.k = k;
  out.dim = 1 << k;
  const size_t nn = (size_t)out.dim * out.dim;
  out.re.resize(nn);
  out.im.resize(nn);
  auto cls = [&](double v) -> Entry {
    if (ztol > 0 && std::fabs(v) < ztol) return {kZero, 0.0};
    if (otol > 0 && std::fabs(v - 1.0) < otol) return {kOne, 1.0};
    if (otol > 0 && std::fabs(v + 1.0) < otol) return {kMinusOne, -1.0};
    return {kImm, (double)(T)v};
  };
  for (size_t i = 0; i < nn; ++i) {
    out.re[i] = cls(m[2 * i]);
    out.im[i] = cls(m[2 * i + 1]);
  }
  return out;
}

template <typename V> inline V mul_kind(const Entry &e, V x, V ev) {
  switch (e.kind) {
  case kOne: return x;
  case kMinusOne: return -x;
  default: return ev * x;
  }
}

// Vectorised path: all targets >= S.  One task = 2^S consecutive amplitudes.
template <typename T>
void apply_vec(T *data, uint32_t n, const Mat<T> &M, const uint32_t *qubits, uint64_t t0,
               uint64_t t1) {
  constexpr int S = Lanes<T>::S;
  constexpr int L = 1 << S;
  typedef typename Lanes<T>::V V;
  const int k = M.k, dim = M.dim;
  // task bits enumerate the amplitude-index bits that are neither targets nor
  // the S lane bits; block index b covers amplitude bits >= S.
  uint64_t tmask = 0;
  for (int i = 0; i < k; ++i) tmask |= 1ull << (qubits[i] - S);
  const uint64_t nb = n - S;
  const uint64_t task_mask = ((nb == 64) ? ~0ull : ((1ull << nb) - 1)) ^ tmask;
  std::vector<uint64_t> off(dim);
  for (int a = 0; a < dim; ++a) off[a] = pdep((uint64_t)a, tmask);
  std::vector<V> xr(dim), xi(dim);
  std::vector<V> mre(M.re.size()), mim(M.im.size());
  for (size_t i = 0; i < M.re.size(); ++i) {
    for (int l = 0; l < L; ++l) {
      mre[i][l] = (T)M.re[i].v;
      mim[i][l] = (T)M.im[i].v;
    }
  }
  for (uint64_t t = t0; t < t1; ++t) {
    const uint64_t base = pdep(t, task_mask);
    for (int a = 0; a < dim; ++a) {
      const V *blk = reinterpret_cast<const V *>(data + 2 * L * (base | off[a]));
      xr[a] = blk[0];
      xi[a] = blk[1];
    }
    for (int r = 0; r < dim; ++r) {
      V ar = {}, ai = {};
      for (int c = 0; c < dim; ++c) {
        const Entry &er = M.re[r * dim + c], &ei = M.im[r * dim + c];
        if (er.kind != kZero) {
          ar += mul_kind(er, xr[c], mre[r * dim + c]);
          ai += mul_kind(er, xi[c], mre[r * dim + c]);
        }
        if (ei.kind != kZero) {
          ar -= mul_kind(ei, xi[c], mim[r * dim + c]);
          ai += mul_kind(ei, xr[c], mim[r * dim + c]);
        }
      }
      V *blk = reinterpret_cast<V *>(data + 2 * L * (base | off[r]));
      blk[0] = ar;
      blk[1] = ai;
    }
  }
}

// Scalar path for gates with a target inside the SIMD lanes.
template <typename T>
void apply_scalar(T *data, uint32_t n, const Mat<T> &M, const uint32_t *qubits, uint64_t t0,
                  uint64_t t1) {
  constexpr int S = Lanes<T>::S;
  const int k = M.k, dim = M.dim;
  uint64_t tmask = 0;
  for (int i = 0; i < k; ++i) tmask |= 1ull << qubits[i];
  const uint64_t task_mask = ((1ull << n) - 1) ^ tmask;
  std::vector<uint64_t> off(dim);
  for (int a = 0; a < dim; ++a) off[a] = pdep((uint64_t)a, tmask);
  std::vector<T> xr(dim), xi(dim);
  std::vector<uint64_t> pos(dim);
  for (uint64_t t = t0; t < t1; ++t) {
    const uint64_t base = pdep(t, task_mask);
    for (int a = 0; a < dim; ++a) {
      pos[a] = insert_zero(base | off[a], S);
      xr[a] = data[pos[a]];
      xi[a] = data[pos[a] | (1ull << S)];
    }
    for (int r = 0; r < dim; ++r) {
      T ar = 0, ai = 0;
      for (int c = 0; c < dim; ++c) {
        const Entry &er = M.re[r * dim + c], &ei = M.im[r * dim + c];
        if (er.kind != kZero) {
          ar += (T)er.v * xr[c];
          ai += (T)er.v * xi[c];
        }
        if (ei.kind != kZero) {
          ar -= (T)ei.v * xi[c];
          ai += (T)ei.v * xr[c];
        }
      }
      data[pos[r]] = ar;
      data[pos[r] | (1ull << S)] = ai;
    }
  }
}

template <typename T>
int apply_t(Sv *sv, const double *mat, const uint32_t *qubits, uint32_t k, int nthreads) {
  constexpr int S = Lanes<T>::S;
  const double tol = sizeof(T) == 8 ? 1e-12 : 1e-6;
  Mat<T> M = classify<T>(mat, (int)k, tol, tol);
  T *data = static_cast<T *>(sv->data);
  const bool vec = qubits[0] >= (uint32_t)S && sv->n >= (uint32_t)S + k;
  const uint64_t ntasks = vec ? (1ull << (sv->n - S - k)) : (1ull << (sv->n - k));
  if (nthreads < 1) nthreads = 1;
  if ((uint64_t)nthreads > ntasks) nthreads = (int)ntasks;
  std::vector<std::thread> pool;
  const uint64_t chunk = (ntasks + nthreads - 1) / nthreads;
  for (int w = 0; w < nthreads; ++w) {
    const uint64_t t0 = w * chunk, t1 = std::min<uint64_t>(ntasks, t0 + chunk);
    if (t0 >= t1) break;
    pool.emplace_back([=, &M]() {
      if (vec) apply_vec<T>(data, sv->n, M, qubits, t0, t1);
      else apply_scalar<T>(data, sv->n, M, qubits, t0, t1);
    });
  }
  for (auto &t : pool) t.join();
  return 0;
}

} // namespace

extern "C" {

void *cb_alloc(uint32_t n, int f32) {
  Sv *sv = new Sv;
  sv->n = n;
  sv->f32 = f32;
  const int S = f32 ? Lanes<float>::S : Lanes<double>::S;
  const uint32_t e = n > (uint32_t)S ? n : (uint32_t)S;
  sv->scalars = 2ull << e;
  const size_t bytes = sv->scalars * (f32 ? 4 : 8);
  sv->data = std::aligned_alloc(64, (bytes + 63) / 64 * 64);
  if (!sv->data) { delete sv; return nullptr; }
  std::memset(sv->data, 0, bytes);
  return sv;
}

void cb_free(void *p) {
  Sv *sv = static_cast<Sv *>(p);
  if (!sv) return;
  std::free(sv->data);
  delete sv;
}

// Load interleaved complex128 amplitudes into the split layout.
void cb_load(void *p, const double *amps) {
  Sv *sv = static_cast<Sv *>(p);
  const int S = sv->f32 ? Lanes<float>::S : Lanes<double>::S;
  const uint64_t len = 1ull << sv->n;
  for (uint64_t i = 0; i < len; ++i) {
    const uint64_t b = insert_zero(i, S);
    if (sv->f32) {
      static_cast<float *>(sv->data)[b] = (float)amps[2 * i];
      static_cast<float *>(sv->data)[b | (1ull << S)] = (float)amps[2 * i + 1];
    } else {
      static_cast<double *>(sv->data)[b] = amps[2 * i];
      static_cast<double *>(sv->data)[b | (1ull << S)] = amps[2 * i + 1];
    }
  }
}

void cb_store(void *p, double *amps) {
  Sv *sv = static_cast<Sv *>(p);
  const int S = sv->f32 ? Lanes<float>::S : Lanes<double>::S;
  const uint64_t len = 1ull << sv->n;
  for (uint64_t i = 0; i < len; ++i) {
    const uint64_t b = insert_zero(i, S);
    if (sv->f32) {
      amps[2 * i] = static_cast<float *>(sv->data)[b];
      amps[2 * i + 1] = static_cast<float *>(sv->data)[b | (1ull << S)];
    } else {
      amps[2 * i] = static_cast<double *>(sv->data)[b];
      amps[2 * i + 1] = static_cast<double *>(sv->data)[b | (1ull << S)];
    }
  }
}

// Amplitudes [first, first + count) as interleaved complex128, for comparing a
// large state chunk by chunk without a second full copy on the host.
int cb_store_range(void *p, uint64_t first, uint64_t count, double *amps) {
  Sv *sv = static_cast<Sv *>(p);
  const int S = sv->f32 ? Lanes<float>::S : Lanes<double>::S;
  if (first > (1ull << sv->n) || count > (1ull << sv->n) - first) return 1;
  for (uint64_t j = 0; j < count; ++j) {
    const uint64_t b = insert_zero(first + j, S);
    if (sv->f32) {
      amps[2 * j] = static_cast<float *>(sv->data)[b];
      amps[2 * j + 1] = static_cast<float *>(sv->data)[b | (1ull << S)];
    } else {
      amps[2 * j] = static_cast<double *>(sv->data)[b];
      amps[2 * j + 1] = static_cast<double *>(sv->data)[b | (1ull << S)];
    }
  }
  return 0;
}

// Initialise |0...0>: statevector.rs:439-442 (initialize).
void cb_zero(void *p) {
  Sv *sv = static_cast<Sv *>(p);
  std::memset(sv->data, 0, sv->scalars * (sv->f32 ? 4 : 8));
  if (sv->f32) static_cast<float *>(sv->data)[0] = 1.0f;
  else static_cast<double *>(sv->data)[0] = 1.0;
}

// Apply a k-qubit gate (qubits ascending, matrix interleaved row-major).
int cb_apply(void *p, const double *mat, const uint32_t *qubits, uint32_t k, int nthreads) {
  Sv *sv = static_cast<Sv *>(p);
  if (!sv || k == 0 || k > 7 || k > sv->n) return 1;
  for (uint32_t i = 0; i < k; ++i)
    if (qubits[i] >= sv->n || (i && qubits[i - 1] >= qubits[i])) return 1;
  return sv->f32 ? apply_t<float>(sv, mat, qubits, k, nthreads)
                 : apply_t<double>(sv, mat, qubits, k, nthreads);
}

} // extern "C"
