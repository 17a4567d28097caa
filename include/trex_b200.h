/*
 * trex_b200 -- B200 (sm_100a) automaton-simulation engine, C ABI.
 *
 * Two groups of entry points live in libtrex_b200.so:
 *
 *  1. Drop-in replacements for the reference's ctypes C ABI. Names, argument
 *     order and meaning follow the reference exactly; each declaration cites
 *     the reference definition it replaces (paths inside the reference
 *     project). As in the reference, every pointer is caller-owned HOST
 *     memory, the library owns the device buffers, copies inputs in and
 *     results out, and keeps one engine per family (init replaces it).
 *     Return codes: 0 ok, -1 not initialised, -2 unsupported shape; this
 *     library adds the negative codes below and never exits the process.
 *
 *  2. trex_* handle entry points (no reference counterpart): many resident
 *     automata, device pointers, 64-bit offsets, explicit streams, the
 *     per-position scan, Boolean and probabilistic NFAs.
 *
 * Strings are passed CSR-style: a byte buffer plus offsets[n+1].
 */
#ifndef TREX_B200_H
#define TREX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ---------------------------------------------------------- */
#define TREX_OK 0
#define TREX_ERR_NOT_INIT (-1)    /* reference: engine not initialised        */
#define TREX_ERR_SHAPE (-2)       /* reference: unsupported shape / device    */
#define TREX_ERR_CUDA (-3)        /* a CUDA call failed; see trex_last_error  */
#define TREX_ERR_CAPACITY (-4)    /* batch larger than the init-time maximum  */
#define TREX_ERR_ARG (-5)         /* invalid argument (null, negative, bad CSR)*/
#define TREX_ERR_DEVICE (-6)      /* a kernel reported an error or a timeout  */
#define TREX_ERR_OOM (-7)         /* device allocation failed                  */

/* Message of the last error raised on the calling thread ("" if none). */
const char *trex_last_error(void);
/* Library version string. */
const char *trex_version(void);

/* Limits of the bounded device waits (no counterpart in the reference, whose
 * look-back spins without a limit, cuda/monoid_scan.cu:187-193): scan_polls =
 * polls of one look-back step of trex_dfa_scan_run, mbar_cycles = clock cycles
 * of one hand-off wait inside the tensor-core NFA kernel (trex_pnfa_run modes
 * BF16, FP16, BOOL, BOOL8). A wait that runs out sets the timeout bit (4) of
 * the run's error word and the kernel returns; the results of that run are
 * then invalid. 0 restores a default (2^24 polls; 4e9 cycles, about 2 s).
 * Process-wide, read at each launch; meant for tests of the give-up paths. */
int trex_set_wait_limits(int64_t scan_polls, int64_t mbar_cycles);

/* Launch profiler: after trex_profile_begin(n), the main kernel of each of the
 * next n runs is bracketed by CUDA events on its stream. trex_profile_end
 * stops recording, waits for the events and writes up to `capacity`
 * per-launch durations (ms) plus the number recorded. */
int trex_profile_begin(int max_launches);
int trex_profile_end(float *ms_out, int capacity, int *count);

/* ========================================================================== *
 * 1. Reference C ABI                                                          *
 * ========================================================================== */

/* ---- monoid batch engine (reference cuda/monoid_batch.cu:594-673) ---------- */
/* Replaces monoid_batch_engine_device_check (monoid_batch.cu:601-609):
 * 0 = a device is present, -1 = no device, -2 = compute capability < 7. */
int monoid_batch_engine_device_check(void);
/* Replaces monoid_batch_engine_init (monoid_batch.cu:611-628). The monoid is
 * walked as an automaton over M elements: curr = char_compose[curr*sigma_ext +
 * raw_char_map[byte]], result = accept[curr]. M <= 255. */
int monoid_batch_engine_init(int M, int sigma_ext, int identity,
                             const uint8_t *char_compose, const uint8_t *raw_char_map,
                             const uint8_t *accept, const uint8_t *monoid_compose,
                             int max_total_chars, int max_batch);
/* Replaces monoid_batch_engine_set_kgram (monoid_batch.cu:630-638). The fused
 * [M*256] table is validated against char_compose; the k-gram table is kept
 * for API compatibility. */
int monoid_batch_engine_set_kgram(const uint8_t *fused_compose, const uint8_t *kgram_compose,
                                  int kgram_k, int sigma_k, int sigma);
/* Replaces monoid_batch_engine_destroy (monoid_batch.cu:640-645). */
void monoid_batch_engine_destroy(void);
/* Replaces monoid_batch_engine_dispatch (monoid_batch.cu:647-658):
 * results[B] = 0/1, kernel_ms / total_ms from CUDA events. */
int monoid_batch_engine_dispatch(const uint8_t *raw_concat, const int *offsets, int *results,
                                 int B, int total_chars, float *kernel_ms, float *total_ms);
/* Replaces monoid_batch_engine_dispatch_prefix (monoid_batch.cu:660-671): same
 * results; long strings are split across the GPU (segment maps). */
int monoid_batch_engine_dispatch_prefix(const uint8_t *raw_concat, const int *offsets,
                                        int *results, int B, int total_chars,
                                        float *kernel_ms, float *total_ms);

/* ---- prefix compose engine (reference cuda/prefix_compose.cu:418-472) ------ */
/* Replaces prefix_engine_device_check (prefix_compose.cu:425-433). */
int prefix_engine_device_check(void);
/* Replaces prefix_engine_init (prefix_compose.cu:435-449): tmap[256*N] with
 * tmap[byte*N + s] = next state, accept[N], start state; N <= 16 in the
 * reference, N <= 256 here. K is accepted and ignored, as in the reference. */
int prefix_engine_init(const uint8_t *tmap, const uint8_t *accept, int start_state, int N,
                       int K, int max_total_chars, int max_batch);
/* Replaces prefix_engine_dispatch (prefix_compose.cu:451-462). */
int prefix_engine_dispatch(const uint8_t *raw_concat, const int *offsets, int *results,
                           int B, int total_chars, float *kernel_ms, float *total_ms);
/* Replaces prefix_engine_destroy (prefix_compose.cu:464-469). */
void prefix_engine_destroy(void);

/* ---- monoid scan engine (reference cuda/monoid_scan.cu:457-515) ------------ */
/* Replaces monoid_engine_init (monoid_scan.cu:468-478): compose[M*M] uint16 with
 * compose[c_new*M + acc_old], accept[M]. */
int monoid_engine_init(int monoid_size, int identity_idx, const uint16_t *compose_table,
                       const uint8_t *accept_table, int max_total_chars, int max_batch);
/* Replaces monoid_engine_destroy (monoid_scan.cu:480-485). */
void monoid_engine_destroy(void);
/* Replaces monoid_engine_dispatch_batch (monoid_scan.cu:492-503): chars are
 * monoid element indices (uint16), one per input character. */
int monoid_engine_dispatch_batch(const uint16_t *chars, const int *offsets, int *results,
                                 int B, int total_chars, float *kernel_ms, float *total_ms);
/* Replaces monoid_engine_device_check (monoid_scan.cu:505-513). */
int monoid_engine_device_check(void);

/* ---- NFA engine (reference cuda/nfa_tc_evolution.cu:936-1015) -------------- */
/* Replaces nfa_tc_engine_init (nfa_tc_evolution.cu:941-952): T[sigma*n*n]
 * float with T[c][dst][src] > 0.5 meaning an edge, accept[n], start[n].
 * The reference requires sigma == 2 and n == 64; here n <= 64, sigma <= 255. */
int nfa_tc_engine_init(const float *T_matrices, const float *accept_mask,
                       const float *start_vec, int n, int sigma, int max_B, int max_L);
/* Replaces nfa_tc_engine_dispatch (nfa_tc_evolution.cu:954-1010): results[B]
 * = accept flag; bytes >= sigma are skipped (the C engine's convention). */
int nfa_tc_engine_dispatch(const uint8_t *raw_concat, const int *offsets, int *results,
                           int B, int total_chars, float *kernel_ms, float *total_ms);
/* Replaces nfa_tc_engine_destroy (nfa_tc_evolution.cu:1012-1014). */
void nfa_tc_engine_destroy(void);

/* ========================================================================== *
 * 2. Handle API (device pointers, 64-bit offsets, explicit stream)            *
 * ========================================================================== */

typedef struct trex_dfa_set trex_dfa_set;

/* Upload n_dfas byte DFAs (n_dfas <= 64). DFA d has n_states[d] (1..256)
 * states, start state starts[d], transition table tmaps + sum_{e<d} 256*N_e
 * (entry [byte*N + s] = next state) and accept flags accepts + sum_{e<d} N_e. */
int trex_dfa_set_create(int n_dfas, const int32_t *n_states, const int32_t *starts,
                        const uint8_t *tmaps, const uint8_t *accepts, trex_dfa_set **out);
void trex_dfa_set_destroy(trex_dfa_set *set);

/* K-gram walking (the reference's monoid K-gram path, src/kgram.py:29-231,
 * cuda/monoid_batch.cu:103-125, re-designed): for an automaton with at most 16
 * states whose bytes fall into at most 16 distinguished bytes plus one column
 * shared by every other byte, k = 2, 4 or 8 consecutive input bytes advance
 * the state with one table lookup (the codes of the k bytes form an 8-bit
 * index: k <= 8 / bits for 1-, 2- or 4-bit codes). Windows holding any other
 * byte are walked byte by byte; results are identical for every input.
 * trex_dfa_kgram_max: the largest k automaton dfa_index allows (1: none).
 * trex_dfa_set_kgram: k = 1 (byte walk, the default), 2, 4, 8, or 0 for the
 * largest allowed; TREX_ERR_SHAPE when the automaton does not allow k. Call
 * it between runs of the set (it updates the automaton's device descriptor
 * with a synchronous copy). trex_dfa_get_kgram: the current k. */
int trex_dfa_kgram_max(const trex_dfa_set *set, int dfa_index, int *k_max);
int trex_dfa_set_kgram(trex_dfa_set *set, int dfa_index, int k);
int trex_dfa_get_kgram(const trex_dfa_set *set, int dfa_index, int *k);

/* Device scratch (bytes) needed by trex_dfa_batch_run for a batch. */
int64_t trex_dfa_batch_scratch_bytes(int64_t n_strings, int64_t total_bytes, int32_t seg_len);

/* Final state / accept flag of every string. All pointers are DEVICE
 * pointers: data[total_bytes], offsets[n+1] (int64, non-decreasing),
 * dfa_id[n] (NULL = automaton 0), outputs (each may be NULL):
 * final_state[n], accept[n] (uint8 0/1), accept_i32[n] (int 0/1).
 * scratch: at least trex_dfa_batch_scratch_bytes bytes, 16-byte aligned (as
 * cudaMalloc returns; else TREX_ERR_ARG), or NULL to use a buffer owned by the
 * set. seg_len: characters per work item (0 = default;
 * longer strings are split and their segment maps composed). stream: a
 * cudaStream_t (NULL = legacy default stream). */
int trex_dfa_batch_run(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                       const int32_t *dfa_id, int64_t n_strings, int64_t total_bytes,
                       uint8_t *final_state, uint8_t *accept, int32_t *accept_i32,
                       void *scratch, int64_t scratch_bytes, int32_t seg_len, void *stream);

/* Multi-pattern batch (the reference's PackedEngine, src/packed_engine.py:
 * 25-125 and 275-439, which packs the patterns block-diagonally and evolves
 * one state vector): every one of n_strings strings is walked by every
 * automaton of the set, reading the input once per automaton but no copy of
 * it; results are automaton-major: final_state / accept / accept_i32 hold
 * n_dfas * n_strings entries, entry d * n_strings + i for string i on
 * automaton d. Scratch: trex_dfa_batch_scratch_bytes(n_strings * n_dfas,
 * total_bytes * n_dfas, seg_len) bytes, or NULL for the set's own. */
int trex_dfa_batch_run_multi(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                             int64_t n_strings, int64_t total_bytes, uint8_t *final_state,
                             uint8_t *accept, int32_t *accept_i32, void *scratch,
                             int64_t scratch_bytes, int32_t seg_len, void *stream);

/* Error word of the last trex_dfa_batch_run that used `scratch` (NULL = the
 * set's own scratch): 0 = fine, bit 0 = malformed offsets, bit 1 = automaton
 * id out of range (the affected strings were skipped), bit 2 = offsets that
 * overlap so far that the batch needs more work items than total_bytes allows
 * for (no string of the batch was run), or a string longer than 64 GiB (that
 * string was skipped). Synchronises. */
int trex_dfa_batch_error(trex_dfa_set *set, void *scratch, int32_t *err_out);

/* The same device-pointer batch without any allocation (no counterpart in the
 * reference). Some callers cannot allocate device memory while they run: a
 * process whose device memory belongs to another allocator (a framework's
 * caching allocator, a memory pool with a fixed budget), a real-time serving
 * loop that must not enter the driver's allocator (cudaMalloc / cudaFree can
 * synchronise the device). This entry point takes no scratch argument: its
 * scratch is a file-scope device array of 8 MiB (every GPU that loads the
 * library holds it until the process exits), so a batch whose
 * trex_dfa_batch_scratch_bytes is above 8 MiB is refused with
 * TREX_ERR_CAPACITY (about 58K strings of 2 KiB at the default segment length;
 * the scratch grows with strings + total_bytes / seg_len work items). The
 * caller still passes inputs and outputs, and calls it with the set's device
 * current (else TREX_ERR_ARG). The first call on each device (and again after
 * a cudaDeviceReset, which makes a new context) looks up the array's device
 * address (cudaGetSymbolAddress); make that first call before any stream
 * capture. Every call on a device shares the one array and it keeps the last
 * call's contents (the counters it needs zeroed are cleared at the start of
 * each call), so calls whose work overlaps on the GPU -- different streams,
 * or other host threads -- race: serialise them. Errors are reported as by
 * trex_dfa_batch_run, through trex_dfa_batch_static_error: strings with
 * malformed offsets or automaton ids are skipped (their outputs are not
 * written), and offsets that overlap so far that the batch needs more work
 * items than total_bytes allows for skip the whole batch (no output is
 * written). */
int trex_dfa_batch_run_static(trex_dfa_set *set, const uint8_t *data, const int64_t *offsets,
                              const int32_t *dfa_id, int64_t n_strings, int64_t total_bytes,
                              uint8_t *final_state, uint8_t *accept, int32_t *accept_i32,
                              int32_t seg_len, void *stream);

/* Error word (bits as trex_dfa_batch_error) of the last
 * trex_dfa_batch_run_static on the set's device, read from the static array
 * with a copy from the symbol (no allocation; no counterpart in the
 * reference). Call it with the set's device current; synchronises. */
int trex_dfa_batch_static_error(trex_dfa_set *set, int32_t *err_out);

/* The same batch from HOST buffers (64-bit offsets): copies the inputs in,
 * runs, copies the requested outputs (each may be NULL) back and reports
 * kernel_ms (device work) and total_ms (copies + device work). Device staging
 * buffers are owned by the set and grow on demand. */
int trex_dfa_batch_host(trex_dfa_set *set, const uint8_t *h_data, const int64_t *h_offsets,
                        const int32_t *h_dfa_id, int64_t n_strings, int64_t total_bytes,
                        uint8_t *h_final_state, uint8_t *h_accept, int32_t *h_accept_i32,
                        int32_t seg_len, float *kernel_ms, float *total_ms);

/* Per-position states (the reference's prefix products,
 * src/simulation.py:142-153, evaluated on the start state): states[p] = the
 * state after byte p of its string, for every byte of the batch (DEVICE
 * buffers; states has total_bytes bytes and the same layout as data). Also
 * final_state[n] / accept[n] (each may be NULL). Automaton dfa_index of the
 * set must have at most 16 states. Long strings are split into tiles of
 * tile_len bytes (0 = default) scanned in one pass with a decoupled
 * look-back. scratch: trex_dfa_scan_scratch_bytes bytes (required). */
int64_t trex_dfa_scan_scratch_bytes(int64_t n_strings, int64_t total_bytes, int32_t tile_len);
int trex_dfa_scan_run(trex_dfa_set *set, int dfa_index, const uint8_t *data,
                      const int64_t *offsets, int64_t n_strings, int64_t total_bytes,
                      uint8_t *states, uint8_t *final_state, uint8_t *accept, void *scratch,
                      int64_t scratch_bytes, int32_t tile_len, void *stream);
/* Error word of the last scan that used `scratch` (same sizes as the run):
 * bit 0 malformed offsets, bit 2 a look-back wait ran out, bit 3 offsets that
 * overlap so far that the tiles exceed the scratch (no tile was scanned).
 * Synchronises. */
int trex_dfa_scan_error(void *scratch, int64_t n_strings, int64_t total_bytes, int32_t tile_len,
                        int32_t *err_out);

/* ---- Boolean NFA (<= 64 states), bit-parallel --------------------------- */
typedef struct trex_nfa trex_nfa;
/* cols[c*64 + j] = destination mask of source state j on symbol c (epsilon
 * closure folded in), c < sigma <= 255. Bytes >= sigma are skipped
 * (unknown_rejects = 0, the reference C engine) or make the string reject
 * with an empty final mask (unknown_rejects = 1, Python simulate_nfa). */
int trex_nfa_create(int n_states, int sigma, const uint64_t *cols, uint64_t start_mask,
                    uint64_t accept_mask, int unknown_rejects, trex_nfa **out);
void trex_nfa_destroy(trex_nfa *nfa);
/* DEVICE buffers; final_mask[n] (uint64), accept[n], accept_i32[n] may each be NULL. */
int trex_nfa_run(trex_nfa *nfa, const uint8_t *data, const int64_t *offsets, int64_t n_strings,
                 int64_t total_bytes, uint64_t *final_mask, uint8_t *accept, int32_t *accept_i32,
                 void *stream);
/* Error word of the last run (bit 0: malformed offsets). Synchronises. */
int trex_nfa_error(trex_nfa *nfa, int32_t *err_out);
/* Many automata in one call (a serving batch): strings group_first[g] ..
 * group_first[g+1] - 1 of offsets run on nfas[g], for n_groups <= 64 groups;
 * group_first (HOST, n_groups + 1 entries, nondecreasing from 0) gives the
 * groups. The groups run side by side: one launch per table layout, each CTA
 * loading its own group's tables. DEVICE buffers as in trex_nfa_run, indexed
 * by the string's position in offsets; scratch holds 8 * (n_groups + 1)
 * bytes (work counters, then the error word at byte 8 * n_groups: bit 0
 * malformed offsets), zeroed by the call. Asynchronous on stream. */
int trex_nfa_run_multi(trex_nfa *const *nfas, int n_groups, const int64_t *group_first,
                       const uint8_t *data, const int64_t *offsets, int64_t total_bytes,
                       uint64_t *final_mask, uint8_t *accept, int32_t *accept_i32, void *scratch,
                       void *stream);

/* ---- probabilistic NFA (<= 64 states): s' = T[c] s ----------------------
 * Replaces the reference's nfa_prob_v5_tc_kernel / nfa_prob_v6_cuda_kernel
 * (cuda/nfa_tc_evolution.cu:456-610), which are reachable only from its test
 * main and return dot(s_L, accept) > 0.5; this form returns the natural
 * log-likelihood log(dot(s_L, accept)) in FP64 as well as that flag.
 * T[c][dst][src] (row-major, sigma x n x n), start[n], accept[n]. Bytes
 * >= sigma are skipped (the reference kernels leave the state unchanged). */
typedef struct trex_pnfa trex_pnfa;
enum {
    TREX_PNFA_BF16 = 0,
    TREX_PNFA_FP16 = 1,
    TREX_PNFA_FP32 = 2,
    TREX_PNFA_BOOL = 3,
    TREX_PNFA_BF16_CC = 4,
    TREX_PNFA_FP16_CC = 5,
    TREX_PNFA_BOOL8 = 6
};
int trex_pnfa_create(int n_states, int sigma, const float *T, const float *start,
                     const float *accept, trex_pnfa **out);
void trex_pnfa_destroy(trex_pnfa *pnfa);
/* mode TREX_PNFA_BF16 / TREX_PNFA_FP16: tensor-core products (tcgen05) with
 * 16-bit operands and FP32 accumulation, sigma <= 28 (else TREX_ERR_SHAPE);
 * TREX_PNFA_FP32: FP32 on CUDA cores, any sigma. Every step renormalises the
 * state by a power of two kept as an integer exponent.
 * TREX_PNFA_BOOL: the Boolean NFA of the same tables on the tensor cores
 * (replaces the FP16 WMMA nfa_tc_binary kernels, cuda/nfa_tc_evolution.cu:
 * 59-442): every nonzero T entry is an edge, start and accept are the sets of
 * nonzero entries, and every product is thresholded to {0, 1}
 * (s' = min(T[c] s, 1), exact: operands are 0/1 in BF16, sums are small
 * integers in FP32); accept = some accepting state is active, and loglik is
 * the log of the number of active accepting states. sigma <= 28.
 * TREX_PNFA_BOOL8: the same Boolean NFA with 0/1 int8 operands and int32
 * sums (tcgen05 kind::i8: K = 32 an instruction, so half the MMA
 * instructions of TREX_PNFA_BOOL), thresholded to {0, 1} every step (exact).
 * The four tensor-core modes run with sigma <= 4 on a kernel that keeps one
 * string on each TMEM lane (the symbol folded into K: no sorting of strings by
 * symbol; 2-4x the throughput), above it on the kernel that groups strings by
 * symbol pair each step; results are the same within each mode's rounding.
 * TREX_PNFA_BF16_CC / TREX_PNFA_FP16_CC: CUDA cores with the 16-bit tables in
 * shared memory and an FP32 state, four warps per string: the low-latency form
 * for few (possibly long) strings, sigma <= 28. DEVICE buffers;
 * loglik[n] (-inf when the likelihood is 0), accept[n], accept_i32[n]
 * (dot > 0.5) may each be NULL. One run at a time per handle. */
int trex_pnfa_run(trex_pnfa *pnfa, int mode, const uint8_t *data, const int64_t *offsets,
                  int64_t n_strings, int64_t total_bytes, double *loglik, uint8_t *accept,
                  int32_t *accept_i32, void *stream);
/* Error word of the last run: bit 0 malformed offsets (those strings get no
 * result), bit 2 an internal wait ran out. Synchronises. */
int trex_pnfa_error(trex_pnfa *pnfa, int32_t *err_out);
/* Sizes every later launch of this handle for at most max_sms SMs (one CTA an
 * SM for the tensor-core and shared-memory forms, 64 warps an SM for FP32);
 * 0 restores all SMs. The kernels take strings from a work queue, so results
 * do not change, only how much of the GPU a run may hold: a server uses it to
 * leave SMs to other work beside long probabilistic chains. */
int trex_pnfa_set_sm_limit(trex_pnfa *pnfa, int max_sms);

/* ---- serving: strings from a staging buffer to their batch places ---------
 * No reference counterpart (the reference serves one static batch per call,
 * cuda/monoid_batch.cu:498-588). String i of the staging buffer,
 * src[src_offsets[i] .. src_offsets[i+1]), is copied to dst[dst_begin[i] ..].
 * DEVICE buffers: src (src_bytes), src_offsets[n+1] (nondecreasing, from 0,
 * src_offsets[n] <= src_bytes), dst (dst_bytes), dst_begin[n], err (one
 * int32 the call ORs into). A byte outside its string's source range or the
 * destination is not written and sets bit 0 of *err. Asynchronous on stream;
 * destination ranges that overlap leave those bytes unspecified. */
int trex_scatter_strings(const uint8_t *src, int64_t src_bytes, const int64_t *src_offsets,
                         int64_t n_strings, uint8_t *dst, int64_t dst_bytes,
                         const int64_t *dst_begin, int32_t *err, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TREX_B200_H */
