/*
 * Extension C ABI of libcast_b200.so: entry points with no counterpart in the
 * reference's ffi_cuda.h, added beside it (the drop-in ABI is unchanged).
 * Same conventions as ffi_cuda.h: int 0 = success / 1 = failure (NULL for
 * handle-returning calls), message in err_buf, err_buf[0] = '\0' on success.
 * Statevectors are device pointers to 2^n interleaved (re, im) amplitudes of
 * the given precision (0 = F32, 1 = F64); gate matrices are host arrays of
 * 4^k cast_complex64_t, row-major, with qubits ascending and qubits[b] = bit b
 * of the matrix index (the reference convention, src/cpp/cuda/cuda_gen.cpp:241-246).
 * Each entry names the reference code whose job it takes over.
 */
#ifndef CAST_B200_H
#define CAST_B200_H

#include "ffi_types.h"

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* -- Device selection -----------------------------------------------------------
 * Makes `device` current for the calling thread in this library's CUDA runtime
 * (one process per GPU).  The reference hard-wires device 0
 * (src/cpp/cuda/cuda_exec.cpp:50). */
int cast_b200_set_device(int device, char *err_buf, size_t err_buf_len);

/* -- Stream-ordered helpers ------------------------------------------------------
 * A stream that does not synchronise with the legacy default stream (so work
 * that other threads put on stream 0 cannot invalidate a graph capture on it),
 * and a reset to |0...0> ordered on `stream` (cudaMemsetAsync plus one element
 * written by a kernel; no host copy).  The reference's cast_cuda_stream_create
 * and cast_cuda_sv_zero (src/cpp/cuda/cuda_exec.cpp:268-279, 452-479) are the
 * blocking / host-synchronous forms. */
void *cast_b200_stream_create_nonblocking(char *err_buf, size_t err_buf_len);
/* A non-blocking stream with a scheduling priority (no counterpart in the
 * reference): numerically lower is more urgent, clamped into the device's range
 * (cudaDeviceGetStreamPriorityRange: 0 is the default, negative values are more
 * urgent).  When several streams have work waiting, thread blocks of the more
 * urgent stream's kernels start first as SMs free up. */
void *cast_b200_stream_create_priority(int priority, char *err_buf, size_t err_buf_len);
int cast_b200_sv_zero_async(uint64_t dptr, size_t n_elements, uint8_t precision, void *stream,
                            char *err_buf, size_t err_buf_len);

/* -- Kernel path control ------------------------------------------------------
 * 0 = automatic (default), 1 = register kernel only, 2 = shared-memory tile
 * kernel wherever it applies.  For measurement and tests; returns the previous
 * setting.  No reference counterpart (the reference has one code generator). */
int cast_b200_set_gate_path(int path);

/* Kernel choice for one class of dense gates with k <= 4 that have a target
 * below qubit 5 (the targets a warp's contiguous loads cannot stride over).  A
 * class is (precision 0 FP32 / 1 FP64, k, low_mask = the set of targets below
 * qubit 5 as bits, 1..31 with at most k bits).  engine -1 restores the built-in
 * rule, 0 routes the class to the register kernel, 1 to the shared-memory tile
 * kernel; tile_bits 0 keeps the built-in tile size, 11 or 12 sets 2048 or 4096
 * amplitudes a tile.  Written by the kernel autotuner from measured times; takes
 * effect for launches after the call (CUDA graphs captured before it keep the
 * kernels they captured) and applies process-wide.  cast_b200_set_gate_path's
 * forced paths override it.  Returns 0, or 1 with a message for an
 * out-of-range class or value.  No reference counterpart (the reference tunes
 * one generated kernel per gate through its code generator). */
int cast_b200_set_kernel_choice(uint8_t precision, uint32_t k, uint32_t low_mask, int engine,
                                uint32_t tile_bits, char *err_buf, size_t err_buf_len);

/* -- One-call gate application ------------------------------------------------
 * Snap (ztol/otol scaled by 1/2^k, as cuda_gen.cpp:84-103) and apply one gate
 * in place on `stream`.  Takes over the compile -> load -> launch sequence of
 * CudaKernelManager::{generate,apply} (src/cuda/kernel.rs:778-924) for callers
 * that hold the matrix as data.  k <= 7; for k >= 6, and for sparse gates, the
 * matrix is staged in a device buffer owned by the library, so the call is
 * synchronous. */
int cast_b200_apply_gate(uint64_t sv_dptr, uint32_t sv_n_qubits, uint8_t precision,
                         const cast_complex64_t *matrix, const uint32_t *qubits,
                         uint32_t n_gate_qubits, double ztol, double otol, void *stream,
                         char *err_buf, size_t err_buf_len);

/* The kernel family a gate would run on in a program (split = the program's
 * split-precision mode), decided exactly as a launch decides it; touches no
 * device.  0 register kernel, 1 tile kernel (low targets), 2 staged wide-gate
 * kernel, 3 sparse CSR kernel, 4 tiled sparse CSR kernel, 5 tcgen05 tensor
 * path; -1 on an invalid gate (message in err_buf).  No counterpart in the
 * reference, whose generator emits one kernel per gate. */
int cast_b200_gate_engine(uint8_t precision, uint32_t sv_n_qubits, const cast_complex64_t *matrix,
                          const uint32_t *qubits, uint32_t n_gate_qubits, double ztol,
                          double otol, int split, char *err_buf, size_t err_buf_len);

/* -- Gate programs ---------------------------------------------------------------
 * An ordered list of gates for one statevector size and precision, uploaded
 * once and replayed many times: the device-side analogue of the reference's
 * compile_batch + apply-all + sync loop (src/simulator/mod.rs:523-562,
 * src/simulator/bench.rs:136-167).  With use_graph != 0 the launches are
 * captured once per (statevector, stream) into a CUDA graph and replayed. */
void *cast_b200_program_create(uint8_t precision, uint32_t sv_n_qubits, double ztol, double otol,
                               char *err_buf, size_t err_buf_len);
int cast_b200_program_add_gate(void *program, const cast_complex64_t *matrix,
                               const uint32_t *qubits, uint32_t n_gate_qubits, char *err_buf,
                               size_t err_buf_len);
/* Opt-in tensor-core path for complex64 programs: gates with 5 or 6 qubits added
 * afterwards run as split-BF16 tcgen05 GEMMs ([[A,-B],[B,A]] applied to
 * 128-group tiles, hi/lo operand split, three products, FP32 accumulation in
 * tensor memory; ~1e-5 relative error per pass).  Must be set before the first
 * gate. */
int cast_b200_program_set_split_precision(void *program, int enable, char *err_buf,
                                          size_t err_buf_len);
/* Reads and clears the tensor-core kernel's error word: 0 when every bounded
 * wait of every launch since the last call completed, else a bit per wait kind
 * that expired (the affected tiles were left unwritten).  Synchronizes the
 * device first, so every launch issued before the call is covered. */
int cast_b200_tensor_status(uint32_t *out_bits, char *err_buf, size_t err_buf_len);
/* Selects how the tensor-core kernel loads amplitudes: 0 or 1 = register loads
 * (the default, measured fastest), 2 = TMA bulk copies for 6-qubit gates whose
 * lowest target qubit is >= 7 when the statevector has whole 128-group tiles,
 * register loads otherwise.  Both give the same results; returns the previous
 * mode. */
int cast_b200_set_tensor_loader(int mode);
uint32_t cast_b200_program_num_gates(const void *program);
int cast_b200_program_run(void *program, uint64_t sv_dptr, void *stream, int use_graph,
                          char *err_buf, size_t err_buf_len);
void cast_b200_program_destroy(void *program);

/* -- FP64 reductions ---------------------------------------------------------------
 * <a|b> over 2^n amplitudes, FP64 accumulation; synchronous on `stream`.
 * Replaces the host loop of CPUStatevector::fidelity (src/cpu/statevector.rs:363-374)
 * for device states. */
int cast_b200_inner_product(uint64_t a_dptr, uint64_t b_dptr, uint32_t n_qubits,
                            uint8_t precision, double *out_re, double *out_im, void *stream,
                            char *err_buf, size_t err_buf_len);
/* out_p1[q] = P(qubit q = 1) for q < n (so <Z_q> = 1 - 2 out_p1[q]) and
 * *out_norm = sum |a|^2, in one FP64 pass; synchronous. */
int cast_b200_qubit_populations(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                                double *out_p1, double *out_norm, void *stream, char *err_buf,
                                size_t err_buf_len);
/* Marginal probabilities over `measured` qubits (bin index bit j = qubit
 * measured[j]), 2^n_measured bins, FP64; replaces the download-then-bin of
 * marginal_probabilities / accumulate_marginal_probs (src/simulator/mod.rs:282-291,
 * src/simulator/measure.rs:15-41).  n_measured <= 12. */
int cast_b200_marginal_probabilities(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                                     const uint32_t *measured, uint32_t n_measured,
                                     double *out_probs, void *stream, char *err_buf,
                                     size_t err_buf_len);
/* Density-matrix diagonal: out[i] = Re rho[i | i << n] for the vectorised
 * 2n-qubit state (QuantumState::populations / trace, src/simulator/mod.rs:387-413). */
int cast_b200_dm_populations(uint64_t rho_dptr, uint32_t n_physical, uint8_t precision,
                             double *out, void *stream, char *err_buf, size_t err_buf_len);
/* Shot sampling on the device (replaces the reference's host-side path:
 * marginal_probabilities downloads the statevector, src/simulator/mod.rs:282-291,
 * and batch_sample draws by the inverse CDF, src/simulator/measure.rs:49-76).
 * Draws n_shots basis states from |a_i|^2 / sum |a|^2 without copying the state
 * off the device: the CDF is an exact 64-bit fixed-point prefix sum (each
 * probability scaled by 2^62 / total), and a shot with uniform u takes the
 * first index whose inclusive prefix is > floor(u * Q), Q the integer total
 * (the last index if none).  out_keys[i] (host array of n_shots) receives the
 * sampled index, or with n_measured > 0 its bits at measured[0..m) packed into
 * bits 0..m-1; keys come in ascending order of the sampled index.
 * cast_b200_sample draws the uniforms on the device (Philox-4x32-10 keyed by
 * `seed`, sorted by construction: normalised exponential spacings);
 * cast_b200_sample_at takes them from the caller (non-decreasing, in [0, 1)).
 * Up to 36 qubits and 2^30 shots a call; synchronous on `stream`.  A pinned
 * (page-locked) out_keys takes the keys by one direct DMA; after an error its
 * contents are unspecified. */
int cast_b200_sample(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision, uint64_t n_shots,
                     uint64_t seed, const uint32_t *measured, uint32_t n_measured,
                     uint64_t *out_keys, void *stream, char *err_buf, size_t err_buf_len);
int cast_b200_sample_at(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                        const double *sorted_uniforms, uint64_t n_shots, const uint32_t *measured,
                        uint32_t n_measured, uint64_t *out_keys, void *stream, char *err_buf,
                        size_t err_buf_len);
/* Amplitude damping on the qubits of `mask` for host-driven quantum-jump
 * trajectories on the plain path (no counterpart in the reference, whose
 * ensemble loop weights branches by fixed probabilities,
 * src/simulator/trajectory.rs:180-265).  damping_sums: *out_total = sum |a_i|^2
 * and *out_weighted = sum |a_i|^2 (1 - gamma)^popc(i & mask), both FP64, so the
 * no-jump branch has probability weighted / total; synchronous on `stream`.
 * scale_popc: a_i *= scale * factor^popc(i & mask) (with factor = sqrt(1 - gamma)
 * and scale = 1 / sqrt(weighted) it applies the no-jump branch renormalised to
 * norm 1); enqueued on `stream`. */
int cast_b200_damping_sums(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision, uint64_t mask,
                           double gamma, double *out_total, double *out_weighted, void *stream,
                           char *err_buf, size_t err_buf_len);
int cast_b200_scale_popc(uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision, uint64_t mask,
                         double factor, double scale, void *stream, char *err_buf,
                         size_t err_buf_len);

/* -- Native fusion planner -----------------------------------------------------------
 * Runs the reference's optimiser - phase 1 size-2 canonicalisation and phase 2
 * agglomerative fusion for candidate sizes 3..size_max with cost-model
 * accept/rollback (src/fusion.rs:14-345 over the CircuitGraph of
 * src/circuit_graph.rs:107-504) - on a unitary gate list given in circuit
 * order (gate_k[i] qubits each, ascending, concatenated in `qubits`; 4^k
 * matrix entries each, concatenated in `matrices`).  cost_kind 0 is
 * SizeOnlyCostModel (cost_model.rs:20-44), 1 is HardwareAdaptiveCostModel
 * (cost_model.rs:238-275: cost = max(1, AI / crossover)); gates with
 * k >= tensor_min_k (when non-zero) use tensor_crossover_ai instead, the
 * crossover of the tensor-core contraction path.  The result lists the fused
 * gates in row order (the reference's gates_in_row_order). */
typedef struct cast_b200_fusion_config_t {
  uint32_t size_max;
  uint32_t cost_kind;
  double benefit_margin;
  double zero_tol;
  double crossover_ai;
  double tensor_crossover_ai;
  uint32_t tensor_min_k;
  uint32_t reserved;
} cast_b200_fusion_config_t;

void *cast_b200_fuse(uint32_t n_qubits, uint32_t n_gates, const uint32_t *gate_k,
                     const uint32_t *qubits, const cast_complex64_t *matrices,
                     const cast_b200_fusion_config_t *config, char *err_buf, size_t err_buf_len);
uint32_t cast_b200_fused_num_gates(const void *fused);
/* Copies fused gate `index`: its size, ascending qubits (<= 7) and 4^k entries. */
int cast_b200_fused_gate(const void *fused, uint32_t index, uint32_t *out_k, uint32_t *out_qubits,
                         cast_complex64_t *out_matrix);
/* Appends every fused gate to a gate program (cast_b200_program_add_gate). */
int cast_b200_program_add_fused(void *program, const void *fused, char *err_buf,
                                size_t err_buf_len);
void cast_b200_fused_free(void *fused);

/* -- Batched noisy trajectories ---------------------------------------------------
 * A trajectory program for n <= 22 qubits (complex64 amplitudes, FP64 branch
 * sums): fused unitary blocks (k <= 4), Pauli errors attached to the block they
 * follow (three k-qubit matrices U P U^dagger for X, Y, Z, each fired with
 * probability prob / 3), amplitude damping on a qubit mask, and general
 * single-qubit channels (1..4 Kraus operators, 2x2 each).  cast_b200_traj_run
 * samples n_traj Monte-Carlo quantum-jump trajectories from |0...0> in one
 * persistent kernel launch (captured once into a CUDA graph when use_graph and
 * stream is non-NULL) and returns <Z_q> per trajectory (n_traj x n doubles) and
 * one sampled bitstring per trajectory.  Replaces the deterministic ensemble
 * branching of src/simulator/trajectory.rs:180-312, whose branch weights are the
 * fixed p_i rather than ||K_i psi||^2. */
void *cast_b200_traj_create(uint32_t n_qubits, char *err_buf, size_t err_buf_len);
void cast_b200_traj_destroy(void *program);
int cast_b200_traj_add_gate(void *program, const cast_complex64_t *matrix, const uint32_t *qubits,
                            uint32_t n_gate_qubits, char *err_buf, size_t err_buf_len);
int cast_b200_traj_add_pauli_error(void *program, double prob, const cast_complex64_t *matrices,
                                   char *err_buf, size_t err_buf_len);
int cast_b200_traj_add_damping(void *program, uint32_t qubit_mask, double gamma, char *err_buf,
                               size_t err_buf_len);
int cast_b200_traj_add_channel(void *program, uint32_t qubit, const cast_complex64_t *kraus,
                               uint32_t n_kraus, char *err_buf, size_t err_buf_len);
uint32_t cast_b200_traj_num_ops(const void *program);
uint32_t cast_b200_traj_num_qubits(const void *program);
/* Builds the whole program from a circuit, natively (the trajectory
 * construction: Pauli channels moved to the end of their fused block as
 * U P U^dagger, damping merged into masks, other one-qubit channels kept).
 * Item i is a unitary gate (kind 0: k[i] ascending qubits, 4^k matrix entries)
 * or a one-qubit channel (kind 1: base matrix then n_branches[i] Kraus
 * matrices, 4 entries each, and as many weights).  Qubits, matrices and
 * weights are consumed in item order.  out_stats (4 entries, may be NULL):
 * fused blocks, Pauli error sites, damping ops, general channels. */
int cast_b200_traj_build(void *program, uint32_t n_items, const uint32_t *kind, const uint32_t *k,
                         const uint32_t *qubits, const cast_complex64_t *matrices,
                         const uint32_t *n_branches, const double *weights, uint32_t fusion_k,
                         uint32_t *out_stats, char *err_buf, size_t err_buf_len);
/* Reads op `index` back: type (0 gate, 1 Pauli error, 2 damping, 3 channel),
 * k and qubits, probability (error) or rate (damping), qubit mask (damping),
 * and its matrices (gate: 1, error: 3 on the block's qubits, channel: the
 * Kraus operators; complex64 precision) when out_mats holds enough entries. */
int cast_b200_traj_get_op(const void *program, uint32_t index, uint32_t *out_type, uint32_t *out_k,
                          uint32_t *out_qubits, double *out_prob, uint32_t *out_mask,
                          uint32_t *out_n_mats, cast_complex64_t *out_mats, size_t out_mats_len);
/* Launch shape of the trajectory kernel, a tuning knob with no counterpart in
 * the reference.  threads: threads per CTA, 512 or 1024, or 0 (the default) to
 * choose by state size.  max_ctas: CTAs, i.e. trajectories in flight (each owns
 * a 2^n-amplitude slice of the workspace), or 0 (the default) for one per SM. */
int cast_b200_traj_set_launch(void *program, uint32_t threads, uint32_t max_ctas, char *err_buf,
                              size_t err_buf_len);
int cast_b200_traj_run(void *program, uint32_t n_traj, uint64_t seed, double *out_z,
                       uint32_t *out_samples, void *stream, int use_graph, char *err_buf,
                       size_t err_buf_len);
/* Trajectories first .. first + n_traj - 1 of the same seed: trajectory i draws
 * from Philox stream (seed, i) whatever range it is run in, so ranges split over
 * ranks or calls reproduce one cast_b200_traj_run of the whole batch row for row.
 * Outputs are indexed from 0 (row j is trajectory first + j). */
int cast_b200_traj_run_range(void *program, uint32_t first, uint32_t n_traj, uint64_t seed,
                             double *out_z, uint32_t *out_samples, void *stream, int use_graph,
                             char *err_buf, size_t err_buf_len);

/* -- Many small circuits in one launch ------------------------------------------------
 * No counterpart in the reference, which runs one circuit at a time
 * (Simulator::simulate, src/simulator/mod.rs:523-547, one kernel per gate).  A
 * batch holds independent circuits of 1..20 qubits, each with its own device
 * statevector (2^n amplitudes of its precision, 16-byte aligned; circuits of a
 * batch must not share memory), its own precision and gates of 1..4 qubits
 * (qubits ascending; matrices snapped like the plain path's).  batch_run
 * executes every circuit in ONE persistent kernel - one CTA a circuit, claimed
 * from a device work counter, longest first - then writes <Z_q> (FP64) of every
 * circuit to out_z, circuit after circuit in the order they were added
 * (cast_b200_batch_num_z values); synchronous on `stream`.  The circuits'
 * statevectors hold the final states afterwards.  init_zero: start from
 * |0...0> (else from the statevector's contents).  A batch keeps its circuits
 * until batch_clear and its device buffers until batch_destroy. */
void *cast_b200_batch_create(char *err_buf, size_t err_buf_len);
void cast_b200_batch_destroy(void *batch);
int cast_b200_batch_add(void *batch, uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                        uint32_t n_gates, const uint32_t *gate_k, const uint32_t *qubits,
                        const cast_complex64_t *matrices, int init_zero, double ztol, double otol,
                        char *err_buf, size_t err_buf_len);
/* The gates of a cast_b200_fuse result (fused at size_max <= 4). */
int cast_b200_batch_add_fused(void *batch, uint64_t sv_dptr, uint32_t n_qubits, uint8_t precision,
                              const void *fused, int init_zero, double ztol, double otol,
                              char *err_buf, size_t err_buf_len);
uint32_t cast_b200_batch_num_circuits(const void *batch);
uint32_t cast_b200_batch_num_z(const void *batch);
void cast_b200_batch_clear(void *batch);
int cast_b200_batch_run(void *batch, double *out_z, void *stream, char *err_buf,
                        size_t err_buf_len);

/* -- Allocation-free norm^2 -------------------------------------------------------
 * No counterpart in the reference: an extra variant of cast_cuda_norm_squared
 * for callers that cannot let a library allocate device memory: applications
 * whose device memory is owned by a pool or arena that accounts for every byte,
 * and hosts that forbid allocations once running (cudaMalloc / cudaFree may
 * synchronise the whole device and stall their other streams).  Same result
 * (sum of squares of n_elements scalars, FP64 accumulation, written to the host
 * double *out_norm_sq; the call waits for it on `stream`, NULL = legacy default
 * stream), but the scratch is a fixed array inside the library (about 1 MiB per
 * GPU, held until the process exits) and no memory is allocated.  Limit:
 * n_elements <= 2^32 (F64) / 2^33 (F32), i.e. 32 GiB of amplitudes; larger
 * inputs are rejected with an error.  dptr must be 16-byte aligned.  The first
 * call on each device (and the first after a cudaDeviceReset) looks up the
 * array's device address; make that first call before any stream capture.
 * Calls whose kernels may overlap on the GPU share the array and race; order
 * them. */
int cast_b200_norm_squared_noalloc(uint64_t dptr, size_t n_elements, uint8_t precision,
                                   double *out_norm_sq, void *stream, char *err_buf,
                                   size_t err_buf_len);

#ifdef __cplusplus
}
#endif

#endif /* CAST_B200_H */
