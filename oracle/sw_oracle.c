/*
 * Smith-Waterman oracle -- TEST INFRASTRUCTURE ONLY (loaded by tests/, smoke() and bench.py's CPU
 * legs, never by the product). A restatement, in C, of fgkl's reference port of GATK's
 * SmithWatermanJavaAligner (crates/smithwaterman/src/reference.rs:9-203): full integer score and
 * traceback matrices, affine gaps tracked per column (vertical) and per row (horizontal), ties
 * resolved diagonal first, then the horizontal gap, then the vertical one, and GATK's four overhang
 * strategies for where the alignment ends and how unaligned sequence is reported.
 *
 * Strategy codes as fgkl's JNI entry assigns them (crates/jni/src/lib.rs:290-296): 0 SoftClip,
 * 1 Indel, 2 LeadingIndel, 3 Ignore.
 */
#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { SW_SOFTCLIP = 0, SW_INDEL = 1, SW_LEADING_INDEL = 2, SW_IGNORE = 3 };

/* GATK's MATRIX_MIN_CUTOFF and lowInitValue (lib.rs:19-22). */
#define SW_MATRIX_MIN_CUTOFF (-100000000)
#define SW_LOW_INIT_VALUE (INT_MIN / 2)

/* Utils.lastIndexOf (lib.rs:602-607): start of the last occurrence of q in r, or -1. */
int or_sw_last_index_of(const uint8_t* r, int n, const uint8_t* q, int m) {
    if (m > n) return -1;
    for (int s = n - m; s >= 0; --s)
        if (memcmp(r + s, q, (size_t)m) == 0) return s;
    return -1;
}

/* calculate_matrix, reference.rs:35-111. sw and bt are (n + 1) x (m + 1), row-major by reference
 * position; bt holds 0 (diagonal), -ki (horizontal gap of ki) or kd (vertical gap of kd). */
static void sw_matrix(const uint8_t* ref, int n, const uint8_t* alt, int m, int w_match, int w_mismatch, int w_open,
                      int w_extend, int strategy, int32_t* sw, int32_t* bt) {
    const int ncol = m + 1, nrow = n + 1;
    int32_t* best_v = malloc(sizeof(int32_t) * (size_t)(ncol + 1));
    int32_t* size_v = calloc((size_t)(ncol + 1), sizeof(int32_t));
    int32_t* best_h = malloc(sizeof(int32_t) * (size_t)(nrow + 1));
    int32_t* size_h = calloc((size_t)(nrow + 1), sizeof(int32_t));
    for (int j = 0; j <= ncol; ++j) best_v[j] = SW_LOW_INIT_VALUE;
    for (int i = 0; i <= nrow; ++i) best_h[i] = SW_LOW_INIT_VALUE;
    if (strategy == SW_INDEL || strategy == SW_LEADING_INDEL) {
        int32_t cur = w_open;
        sw[1] = cur;
        for (int j = 2; j < ncol; ++j) sw[j] = (cur += w_extend);
        cur = w_open;
        sw[ncol] = cur;
        for (int i = 2; i < nrow; ++i) sw[(size_t)i * ncol] = (cur += w_extend);
    }
    for (int i = 1; i < nrow; ++i) {
        const uint8_t a = ref[i - 1];
        for (int j = 1; j < ncol; ++j) {
            const uint8_t b = alt[j - 1];
            const int32_t diag = sw[(size_t)(i - 1) * ncol + j - 1] + (a == b ? w_match : w_mismatch);
            int32_t gap = sw[(size_t)(i - 1) * ncol + j] + w_open;
            best_v[j] += w_extend;
            if (gap > best_v[j]) {
                best_v[j] = gap;
                size_v[j] = 1;
            } else {
                size_v[j] += 1;
            }
            const int32_t down = best_v[j], kd = size_v[j];
            gap = sw[(size_t)i * ncol + j - 1] + w_open;
            best_h[i] += w_extend;
            if (gap > best_h[i]) {
                best_h[i] = gap;
                size_h[i] = 1;
            } else {
                size_h[i] += 1;
            }
            const int32_t right = best_h[i], ki = size_h[i];
            const size_t c = (size_t)i * ncol + j;
            if (diag >= down && diag >= right) {
                sw[c] = diag > SW_MATRIX_MIN_CUTOFF ? diag : SW_MATRIX_MIN_CUTOFF;
                bt[c] = 0;
            } else if (right >= down) {
                sw[c] = right > SW_MATRIX_MIN_CUTOFF ? right : SW_MATRIX_MIN_CUTOFF;
                bt[c] = -ki;
            } else {
                sw[c] = down > SW_MATRIX_MIN_CUTOFF ? down : SW_MATRIX_MIN_CUTOFF;
                bt[c] = kd;
            }
        }
    }
    free(best_v);
    free(size_v);
    free(best_h);
    free(size_h);
}

static int sw_push(uint8_t* ops, uint32_t* lens, int cap, int k, uint8_t op, uint32_t len) {
    if (k < cap) {
        ops[k] = op;
        lens[k] = len;
    }
    return k + 1;
}

/*
 * align, reference.rs:9-31, with calculate_cigar, :113-203. Writes the CIGAR (in alternate order)
 * as ops ('M', 'I', 'D', 'S') and lengths, at most `cap` elements, and the reference offset of the
 * first aligned base. Returns the element count (more than `cap` when the arrays were too short),
 * or -1 for an empty sequence.
 */
int or_sw_align(const uint8_t* ref, int n, const uint8_t* alt, int m, int w_match, int w_mismatch, int w_open,
                int w_extend, int strategy, uint8_t* ops, uint32_t* lens, int cap, int32_t* offset) {
    if (n <= 0 || m <= 0) return -1;
    if (strategy == SW_SOFTCLIP || strategy == SW_IGNORE) {
        const int s = or_sw_last_index_of(ref, n, alt, m);
        if (s >= 0) {
            *offset = s;
            return sw_push(ops, lens, cap, 0, 'M', (uint32_t)m);
        }
    }
    const int N = n + 1, M = m + 1;
    int32_t* sw = calloc((size_t)N * M, sizeof(int32_t));
    int32_t* bt = calloc((size_t)N * M, sizeof(int32_t));
    sw_matrix(ref, n, alt, m, w_match, w_mismatch, w_open, w_extend, strategy, sw, bt);

    int p1 = 0, p2 = m, segment = 0;
    int32_t best = INT_MIN;
    if (strategy == SW_INDEL) {
        p1 = n;
    } else {
        for (int i = 1; i < N; ++i) {
            const int32_t cur = sw[(size_t)i * M + m];
            if (cur >= best) {
                p1 = i;
                best = cur;
            }
        }
        if (strategy != SW_LEADING_INDEL) {
            for (int j = 1; j < M; ++j) {
                const int32_t cur = sw[(size_t)n * M + j];
                if (cur > best || (cur == best && abs(n - j) < abs(p1 - p2))) {
                    p1 = n;
                    p2 = j;
                    best = cur;
                    segment = m - j;
                }
            }
        }
    }
    /* Elements are collected last to first and reversed at the end. */
    uint8_t* rops = malloc((size_t)(n + m + 4));
    uint32_t* rlens = malloc(sizeof(uint32_t) * (size_t)(n + m + 4));
    int k = 0;
    if (segment > 0 && strategy == SW_SOFTCLIP) {
        rops[k] = 'S';
        rlens[k++] = (uint32_t)segment;
        segment = 0;
    }
    uint8_t state = 'M';
    do {
        const int32_t btr = bt[(size_t)p1 * M + p2];
        uint8_t next;
        int step;
        if (btr > 0) {
            next = 'D';
            step = btr;
        } else if (btr < 0) {
            next = 'I';
            step = -btr;
        } else {
            next = 'M';
            step = 1;
        }
        if (next == 'M') {
            p1 -= 1;
            p2 -= 1;
        } else if (next == 'I') {
            p2 -= step;
        } else {
            p1 -= step;
        }
        if (next == state) {
            segment += step;
        } else {
            if (segment > 0) {
                rops[k] = state;
                rlens[k++] = (uint32_t)segment;
            }
            segment = step;
            state = next;
        }
    } while (p1 > 0 && p2 > 0);
    if (strategy == SW_SOFTCLIP) {
        rops[k] = state;
        rlens[k++] = (uint32_t)segment;
        if (p2 > 0) {
            rops[k] = 'S';
            rlens[k++] = (uint32_t)p2;
        }
        *offset = p1;
    } else if (strategy == SW_IGNORE) {
        rops[k] = state;
        rlens[k++] = (uint32_t)(segment + p2);
        *offset = p1 - p2;
    } else {
        rops[k] = state;
        rlens[k++] = (uint32_t)segment;
        if (p1 > 0) {
            rops[k] = 'D';
            rlens[k++] = (uint32_t)p1;
        } else if (p2 > 0) {
            rops[k] = 'I';
            rlens[k++] = (uint32_t)p2;
        }
        *offset = 0;
    }
    int out = 0;
    for (int e = k - 1; e >= 0; --e) out = sw_push(ops, lens, cap, out, rops[e], rlens[e]);
    free(rops);
    free(rlens);
    free(sw);
    free(bt);
    return out;
}
