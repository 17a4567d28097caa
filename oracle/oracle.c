/*
 * CPU oracle for the automaton-simulation hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This file restates, in plain C, the reference
 * algorithms that the CUDA kernels must reproduce. Only the tests, the smoke
 * check and the CPU-baseline leg of the benchmark may load it, and only as a
 * checker; the product library never calls into it.
 *
 * Restated reference behaviour (paths are inside the reference project):
 *   dfa walk       src/regex_to_dfa.py:224-233 (DFA.simulate) through the byte
 *                  map of src/simulation.py:274-297 (precompute_tmap); the same
 *                  loop as cuda/prefix_compose.cu:488-516 (cpu_prefix_compose)
 *                  and cuda/monoid_batch.cu:679-699 (cpu_monoid_batch).
 *   positions      src/simulation.py:142-153 (prefix_scan_sequential): the
 *                  state after each prefix, i.e. argmax((T[i]..T[0]) start).
 *   monoid walk    src/monoid.py:174-192 / cuda/monoid_scan.cu:65-108:
 *                  acc = compose[c * M + acc].
 *   boolean nfa    src/nfa_matrices.py:133-157 (simulate_nfa): state =
 *                  min(T[c] state, 1); a symbol >= sigma rejects, or, in the
 *                  C engine's convention (cuda/nfa_tc_evolution.cu:1029-1054,
 *                  :735-737), is skipped.
 *   prob. nfa      cuda/nfa_tc_evolution.cu:506-559 without the threshold:
 *                  s' = T[c] s in FP64 with exact power-of-two rescaling,
 *                  loglik = log(accept . s_L) + sum of scale exponents * ln 2.
 *
 * Parity pin: the tests check this file against golden vectors generated by
 * importing the reference's Python modules (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

int oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- DFA over bytes ----------------------------------------------------
 * tmaps:   concatenation of per-DFA tables, table d has 256 * n_states[d]
 *          bytes at tmap_offset[d]; entry [byte * N + s] is the next state.
 * dfa_id:  per-string automaton index (NULL = all strings use automaton 0).
 */
void oracle_dfa_walk(const uint8_t *tmaps, const int64_t *tmap_offset,
                     const int32_t *n_states, const int32_t *starts,
                     const uint8_t *accepts, const int64_t *accept_offset,
                     const uint8_t *bytes, const int64_t *offsets,
                     const int32_t *dfa_id, int64_t n_strings,
                     uint8_t *final_state, uint8_t *accept_out) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_strings; i++) {
        int d = dfa_id ? dfa_id[i] : 0;
        const uint8_t *t = tmaps + tmap_offset[d];
        int N = n_states[d];
        unsigned s = (unsigned)starts[d];
        const uint8_t *p = bytes + offsets[i];
        int64_t len = offsets[i + 1] - offsets[i];
        for (int64_t k = 0; k < len; k++) s = t[(unsigned)p[k] * (unsigned)N + s];
        if (final_state) final_state[i] = (uint8_t)s;
        if (accept_out) accept_out[i] = accepts[accept_offset[d] + s];
    }
}

/* Per-position states of one string: out[k] = state after bytes[0..k]. */
void oracle_dfa_positions(const uint8_t *tmap, int N, int start,
                          const uint8_t *bytes, int64_t len, uint8_t *out) {
    unsigned s = (unsigned)start;
    for (int64_t k = 0; k < len; k++) {
        s = tmap[(unsigned)bytes[k] * (unsigned)N + s];
        out[k] = (uint8_t)s;
    }
}

/* Several strings in parallel, one output stream per string laid out like
 * the input (out has offsets[n] bytes). */
void oracle_dfa_positions_batch(const uint8_t *tmap, int N, int start,
                                const uint8_t *bytes, const int64_t *offsets,
                                int64_t n_strings, uint8_t *out) {
    #pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n_strings; i++)
        oracle_dfa_positions(tmap, N, start, bytes + offsets[i],
                             offsets[i + 1] - offsets[i], out + offsets[i]);
}

/* ---- monoid walk over uint16 element indices -------------------------- */
void oracle_monoid_walk(const uint16_t *compose, int M, int identity,
                        const uint8_t *accept, const uint16_t *chars,
                        const int64_t *offsets, int64_t n_strings,
                        int32_t *results) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n_strings; i++) {
        unsigned acc = (unsigned)identity;
        for (int64_t k = offsets[i]; k < offsets[i + 1]; k++)
            acc = compose[(unsigned)chars[k] * (unsigned)M + acc];
        results[i] = accept[acc] ? 1 : 0;
    }
}

/* ---- Boolean NFA with at most 64 states --------------------------------
 * cols[c * 64 + src] = bit mask of destinations reachable from src on c.
 * unknown_rejects: 1 = a symbol >= sigma makes the string reject
 * (Python simulate_nfa), 0 = the symbol is skipped (C engine).
 * final_mask[i] is the state mask after the string (0 when rejected early).
 */
void oracle_nfa_bool(const uint64_t *cols, int sigma, uint64_t start_mask,
                     uint64_t accept_mask, int unknown_rejects,
                     const uint8_t *bytes, const int64_t *offsets,
                     int64_t n_strings, uint64_t *final_mask,
                     uint8_t *accept_out) {
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < n_strings; i++) {
        uint64_t s = start_mask;
        int rejected = 0;
        for (int64_t k = offsets[i]; k < offsets[i + 1]; k++) {
            unsigned c = bytes[k];
            if ((int)c >= sigma) {
                if (unknown_rejects) { rejected = 1; s = 0; break; }
                continue;
            }
            const uint64_t *col = cols + (size_t)c * 64;
            uint64_t nxt = 0, rem = s;
            while (rem) {
                int src = __builtin_ctzll(rem);
                nxt |= col[src];
                rem &= rem - 1;
            }
            s = nxt;
        }
        if (final_mask) final_mask[i] = s;
        if (accept_out) accept_out[i] = (!rejected && (s & accept_mask)) ? 1 : 0;
    }
}

/* ---- Probabilistic NFA in FP64 -----------------------------------------
 * T[c][dst][src] row-major doubles (sigma * N * N), start[N], accept[N].
 * Symbols >= sigma are skipped. After every step the state is multiplied by
 * 2^-e where e is the exponent of its largest entry (frexp), and e is added
 * to the running exponent, so the stored state never under- or overflows.
 * loglik[i] = log(accept . s) + exps * ln 2 (-inf when the mass is zero).
 */
void oracle_pnfa_fp64(const double *T, int sigma, int N, const double *start,
                      const double *accept, const uint8_t *bytes,
                      const int64_t *offsets, int64_t n_strings,
                      double *loglik) {
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t i = 0; i < n_strings; i++) {
        double s[64], t[64];
        int64_t e_total = 0;
        for (int r = 0; r < N; r++) s[r] = start[r];
        for (int64_t k = offsets[i]; k < offsets[i + 1]; k++) {
            unsigned c = bytes[k];
            if ((int)c >= sigma) continue;
            const double *Tc = T + (size_t)c * N * N;
            double mx = 0.0;
            for (int r = 0; r < N; r++) {
                double acc = 0.0;
                const double *row = Tc + (size_t)r * N;
                for (int q = 0; q < N; q++) acc += row[q] * s[q];
                t[r] = acc;
                if (acc > mx) mx = acc;
            }
            if (mx > 0.0) {
                int e;
                frexp(mx, &e);
                for (int r = 0; r < N; r++) s[r] = ldexp(t[r], -e);
                e_total += e;
            } else {
                for (int r = 0; r < N; r++) s[r] = 0.0;
            }
        }
        double dot = 0.0;
        for (int r = 0; r < N; r++) dot += accept[r] * s[r];
        loglik[i] = (dot > 0.0) ? log(dot) + (double)e_total * M_LN2 : -INFINITY;
    }
}
