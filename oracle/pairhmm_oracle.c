/*
 * CPU oracle for the PairHMM / PD-HMM likelihood path -- TEST INFRASTRUCTURE ONLY.
 *
 * Nothing in the product links or calls this file. Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark load it, and only as the checker or the timed CPU reference.
 *
 * It restates, in plain C with double precision, the reference algorithm of fgkl
 * (fulcrumgenomics/fgkl v0.2.0):
 *   - probability tables            crates/pairhmm/src/model.rs:37-106
 *   - plain scalar oracle           crates/pairhmm/src/reference.rs:20-64
 *   - partially determined oracle   crates/pairhmm/src/pd_reference.rs:29-118
 *                                   with the flag bits of crates/pairhmm/src/pd.rs:15-27
 *                                   and base_matches_pd of crates/pairhmm/src/pd.rs:99-110
 * plus an FP64 scalar adjoint (no counterpart in the reference) for the gradient of the summed
 * log10 likelihood with respect to the gap-open, gap-continuation and base-error probabilities.
 *
 * Parity of this file is pinned by the reference's own known-answer tests (model.rs:112-154,
 * reference.rs:81-114, pd_reference.rs:138-183, pd.rs flag tests), restated in tests/.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAX_QUAL 254
#define TRISTATE_CORRECTION 3.0
#define JACOBIAN_MAX_TOLERANCE 8.0
#define JACOBIAN_TABLE_STEP 0.0001

/* Transition indices, model.rs:15-21. */
enum { MM = 0, IM = 1, MI = 2, II = 3, MD = 4, DD = 5, NTRANS = 6 };

/* PD flag bits, pd.rs:15-27. */
enum { PD_SNP = 1, PD_DEL_START = 2, PD_DEL_END = 4, PD_ALT_A = 8, PD_ALT_C = 16, PD_ALT_G = 32, PD_ALT_T = 64 };

static double g_error_prob[MAX_QUAL + 1];
static double g_m2m[((MAX_QUAL + 1) * (MAX_QUAL + 2)) / 2];
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

/* MathUtils.fastRound as in model.rs:104-106: truncation after adding +-0.5. */
static int64_t fast_round(double d) { return d > 0.0 ? (int64_t)(d + 0.5) : (int64_t)(d - 0.5); }

/* log10(1 + 10^-diff) at the quantized table point, model.rs:99-102. */
static double jacobian(double diff) {
    int64_t k = fast_round(diff * (1.0 / JACOBIAN_TABLE_STEP));
    return log10(1.0 + pow(10.0, -(double)k * JACOBIAN_TABLE_STEP));
}

/* MathUtils.approximateLog10SumLog10, model.rs:87-96. */
double or_approximate_log10_sum_log10(double a, double b) {
    if (a > b) return or_approximate_log10_sum_log10(b, a);
    if (a == -INFINITY) return b;
    double diff = b - a;
    return diff < JACOBIAN_MAX_TOLERANCE ? b + jacobian(diff) : b;
}

/* Tables::new, model.rs:37-50. */
static void build_tables(void) {
    const double inv_ln10 = 1.0 / M_LN10;
    for (int q = 0; q <= MAX_QUAL; q++) g_error_prob[q] = pow(10.0, (double)q / -10.0);
    int offset = 0;
    for (int i = 0; i <= MAX_QUAL; i++) {
        for (int j = 0; j <= i; j++) {
            double log10_sum = or_approximate_log10_sum_log10(-0.1 * (double)i, -0.1 * (double)j);
            double p = pow(10.0, log10_sum);
            if (p > 1.0) p = 1.0;
            double m2m_log10 = log1p(-p) * inv_ln10;
            g_m2m[offset + j] = pow(10.0, m2m_log10);
        }
        offset += i + 1;
    }
}

static void ensure_tables(void) { pthread_once(&g_once, build_tables); }

/* Tables::error_prob, model.rs:53-55 (quals clamp at MAX_QUAL). */
double or_error_prob(int qual) {
    ensure_tables();
    if (qual > MAX_QUAL) qual = MAX_QUAL;
    if (qual < 0) qual = 0;
    return g_error_prob[qual];
}

/* Tables::match_to_match, model.rs:59-64. */
double or_match_to_match(int ins_qual, int del_qual) {
    ensure_tables();
    int a = ins_qual > MAX_QUAL ? MAX_QUAL : ins_qual;
    int b = del_qual > MAX_QUAL ? MAX_QUAL : del_qual;
    int lo = a <= b ? a : b, hi = a <= b ? b : a;
    return g_m2m[((hi * (hi + 1)) >> 1) + lo];
}

/* Tables::transitions, model.rs:67-77. */
void or_transitions(int ins_qual, int del_qual, int gcp, double* t) {
    double gap_continue = or_error_prob(gcp);
    t[MM] = or_match_to_match(ins_qual, del_qual);
    t[MI] = or_error_prob(ins_qual);
    t[MD] = or_error_prob(del_qual);
    t[IM] = 1.0 - gap_continue;
    t[II] = gap_continue;
    t[DD] = gap_continue;
}

/* Tables::priors, model.rs:80-83. */
void or_priors(int qual, double* out) {
    double e = or_error_prob(qual);
    out[0] = 1.0 - e;
    out[1] = e / TRISTATE_CORRECTION;
}

/* GATK's LoglessPairHMM.INITIAL_CONDITION = 2^1020, reference.rs:12. */
double or_initial_condition(void) { return ldexp(1.0, 1020); }

/* base_matches_pd, pd.rs:99-110. */
int or_base_matches_pd(uint8_t read_base, uint8_t flags) {
    if (!(flags & PD_SNP)) return 0;
    switch (read_base) {
        case 'A': case 'a': return (flags & PD_ALT_A) != 0;
        case 'C': case 'c': return (flags & PD_ALT_C) != 0;
        case 'G': case 'g': return (flags & PD_ALT_G) != 0;
        case 'T': case 't': return (flags & PD_ALT_T) != 0;
        default: return 0;
    }
}

/*
 * reference::log10_likelihood, reference.rs:20-64: the full-matrix FP64 LoglessPairHMM with the
 * Java operation order. Both the read and the haplotype must be non-empty.
 */
double or_log10_likelihood(const uint8_t* hap, int hap_len, const uint8_t* bases, const uint8_t* quals,
                           const uint8_t* ins, const uint8_t* del, const uint8_t* gcp, int read_len) {
    const int rows = read_len + 1, cols = hap_len + 1;
    double* m = calloc((size_t)rows * cols, sizeof(double));
    double* x = calloc((size_t)rows * cols, sizeof(double));
    double* y = calloc((size_t)rows * cols, sizeof(double));
    const double initial = or_initial_condition() / (double)hap_len;
    for (int j = 0; j < cols; j++) y[j] = initial;
    for (int i = 1; i < rows; i++) {
        double t[NTRANS], pr[2];
        or_transitions(ins[i - 1], del[i - 1], gcp[i - 1], t);
        or_priors(quals[i - 1], pr);
        const uint8_t rb = bases[i - 1];
        for (int j = 1; j < cols; j++) {
            const uint8_t hb = hap[j - 1];
            const double prior = (rb == hb || rb == 'N' || hb == 'N') ? pr[0] : pr[1];
            const size_t diag = (size_t)(i - 1) * cols + (j - 1), up = (size_t)(i - 1) * cols + j;
            const size_t left = (size_t)i * cols + (j - 1), cur = (size_t)i * cols + j;
            m[cur] = prior * (m[diag] * t[MM] + x[diag] * t[IM] + y[diag] * t[IM]);
            x[cur] = m[up] * t[MI] + x[up] * t[II];
            y[cur] = m[left] * t[MD] + y[left] * t[DD];
        }
    }
    double sum = 0.0;
    const size_t last = (size_t)(rows - 1) * cols;
    for (int j = 1; j < cols; j++) sum += m[last + j] + x[last + j];
    free(m);
    free(x);
    free(y);
    return log10(sum) - log10(or_initial_condition());
}

/*
 * pd_reference::log10_likelihood, pd_reference.rs:29-118: FP64 LoglessPDPairHMM with its three
 * branch matrices and the deletion state carried from the end of one row into the next.
 */
double or_pd_log10_likelihood(const uint8_t* hap, const uint8_t* flags, int hap_len, const uint8_t* bases,
                              const uint8_t* quals, const uint8_t* ins, const uint8_t* del, const uint8_t* gcp,
                              int read_len) {
    enum { NORMAL = 0, INSIDE_DEL = 1, AFTER_DEL = 2 };
    const int rows = read_len + 1, cols = hap_len + 1;
    const size_t n = (size_t)rows * cols;
    double* m = calloc(n, sizeof(double));
    double* x = calloc(n, sizeof(double));
    double* y = calloc(n, sizeof(double));
    double* bm = calloc(n, sizeof(double));
    double* bx = calloc(n, sizeof(double));
    double* by = calloc(n, sizeof(double));
    const double initial = or_initial_condition() / (double)hap_len;
    for (int j = 0; j < cols; j++) y[j] = initial;
    int state = NORMAL;
    for (int i = 1; i < rows; i++) {
        double t[NTRANS], pr[2];
        or_transitions(ins[i - 1], del[i - 1], gcp[i - 1], t);
        or_priors(quals[i - 1], pr);
        const uint8_t rb = bases[i - 1];
        for (int j = 1; j < cols; j++) {
            const uint8_t hb = hap[j - 1], flag = flags[j - 1];
            const double prior =
                (rb == hb || rb == 'N' || hb == 'N' || or_base_matches_pd(rb, flag)) ? pr[0] : pr[1];
            const size_t diag = (size_t)(i - 1) * cols + (j - 1), up = (size_t)(i - 1) * cols + j;
            const size_t left = (size_t)i * cols + (j - 1), cur = (size_t)i * cols + j;
            const int del_end = (flag & PD_DEL_END) != 0;
            if (state == NORMAL) {
                bm[cur] = m[left];
                by[cur] = y[left];
                bx[cur] = x[left];
                m[cur] = prior * (m[diag] * t[MM] + x[diag] * t[IM] + y[diag] * t[IM]);
                y[cur] = m[left] * t[MD] + y[left] * t[DD];
            } else if (state == INSIDE_DEL) {
                bm[cur] = bm[left];
                by[cur] = by[left];
                bx[cur] = bx[left];
                m[cur] = prior * (m[diag] * t[MM] + x[diag] * t[IM] + y[diag] * t[IM]);
                y[cur] = m[left] * t[MD] + y[left] * t[DD];
            } else {
                bm[cur] = fmax(bm[left], m[left]);
                by[cur] = fmax(by[left], y[left]);
                bx[cur] = fmax(bx[left], x[left]);
                m[cur] = prior * (fmax(bm[diag], m[diag]) * t[MM] + fmax(bx[diag], x[diag]) * t[IM] +
                                  fmax(by[diag], y[diag]) * t[IM]);
                y[cur] = fmax(bm[left], m[left]) * t[MD] + fmax(by[left], y[left]) * t[DD];
            }
            if (del_end)
                x[cur] = fmax(bm[up], m[up]) * t[MI] + fmax(bx[up], x[up]) * t[II];
            else
                x[cur] = m[up] * t[MI] + x[up] * t[II];
            if (state == AFTER_DEL) state = NORMAL;
            if (flag & PD_DEL_START) state = INSIDE_DEL;
            if (del_end) state = AFTER_DEL;
        }
    }
    double sum = 0.0;
    const size_t last = (size_t)(rows - 1) * cols;
    for (int j = 1; j < cols; j++) sum += m[last + j] + x[last + j];
    free(m); free(x); free(y); free(bm); free(bx); free(by);
    return log10(sum) - log10(or_initial_condition());
}

/* ------------------------------------------------------------------------------------------ */
/* Adjoint oracle (new; the reference has no gradient).                                       */
/*                                                                                            */
/* Continuous parameterisation per read position r (row i = r + 1):                            */
/*   dI = P(M->I), dD = P(M->D), eps = gap continuation (II = DD = eps, IM = 1 - eps),          */
/*   e = base error (match prior 1 - e, mismatch prior e / 3), MM = 1 - dI - dD.               */
/* The forward recurrence is reference.rs:49-54 with these transitions. The gradient of         */
/* log10 L with respect to each per-position parameter is sum over the DP edges that use it of  */
/* F(source) * d(weight)/d(theta) * B(dest), divided by L * ln(10).                             */
/* ------------------------------------------------------------------------------------------ */

/* Forward likelihood (log10) under the continuous parameterisation. */
double or_adj_log10_likelihood(const uint8_t* hap, int hap_len, const uint8_t* bases, int read_len,
                               const double* d_ins, const double* d_del, const double* eps,
                               const double* err) {
    const int rows = read_len + 1, cols = hap_len + 1;
    double* m = calloc((size_t)rows * cols, sizeof(double));
    double* x = calloc((size_t)rows * cols, sizeof(double));
    double* y = calloc((size_t)rows * cols, sizeof(double));
    const double initial = or_initial_condition() / (double)hap_len;
    for (int j = 0; j < cols; j++) y[j] = initial;
    for (int i = 1; i < rows; i++) {
        const int r = i - 1;
        const double mm = 1.0 - d_ins[r] - d_del[r], im = 1.0 - eps[r];
        const double pm = 1.0 - err[r], px = err[r] / 3.0;
        const uint8_t rb = bases[r];
        for (int j = 1; j < cols; j++) {
            const uint8_t hb = hap[j - 1];
            const double prior = (rb == hb || rb == 'N' || hb == 'N') ? pm : px;
            const size_t diag = (size_t)(i - 1) * cols + (j - 1), up = (size_t)(i - 1) * cols + j;
            const size_t left = (size_t)i * cols + (j - 1), cur = (size_t)i * cols + j;
            m[cur] = prior * (m[diag] * mm + x[diag] * im + y[diag] * im);
            x[cur] = m[up] * d_ins[r] + x[up] * eps[r];
            y[cur] = m[left] * d_del[r] + y[left] * eps[r];
        }
    }
    double sum = 0.0;
    const size_t last = (size_t)(rows - 1) * cols;
    for (int j = 1; j < cols; j++) sum += m[last + j] + x[last + j];
    free(m); free(x); free(y);
    return log10(sum) - log10(or_initial_condition());
}

/*
 * Gradient of log10 L with respect to dI, dD, eps and e at every read position, ADDED into
 * g_ins, g_del, g_eps, g_err (each read_len long). Returns log10 L.
 */
double or_adj_gradient(const uint8_t* hap, int hap_len, const uint8_t* bases, int read_len, const double* d_ins,
                       const double* d_del, const double* eps, const double* err, double* g_ins, double* g_del,
                       double* g_eps, double* g_err) {
    const int rows = read_len + 1, cols = hap_len + 1;
    const size_t n = (size_t)rows * cols;
    double* fm = calloc(n, sizeof(double));
    double* fx = calloc(n, sizeof(double));
    double* fy = calloc(n, sizeof(double));
    double* bm = calloc(n, sizeof(double));
    double* bx = calloc(n, sizeof(double));
    double* by = calloc(n, sizeof(double));
    const double initial = or_initial_condition() / (double)hap_len;
    for (int j = 0; j < cols; j++) fy[j] = initial;
#define PRIOR(i, j)                                                                                   \
    ((bases[(i) - 1] == hap[(j) - 1] || bases[(i) - 1] == 'N' || hap[(j) - 1] == 'N') ? 1.0 - err[(i) - 1] \
                                                                                       : err[(i) - 1] / 3.0)
#define MATCHES(i, j) (bases[(i) - 1] == hap[(j) - 1] || bases[(i) - 1] == 'N' || hap[(j) - 1] == 'N')
    for (int i = 1; i < rows; i++) {
        const int r = i - 1;
        const double mm = 1.0 - d_ins[r] - d_del[r], im = 1.0 - eps[r];
        for (int j = 1; j < cols; j++) {
            const size_t diag = (size_t)(i - 1) * cols + (j - 1), up = (size_t)(i - 1) * cols + j;
            const size_t left = (size_t)i * cols + (j - 1), cur = (size_t)i * cols + j;
            fm[cur] = PRIOR(i, j) * (fm[diag] * mm + fx[diag] * im + fy[diag] * im);
            fx[cur] = fm[up] * d_ins[r] + fx[up] * eps[r];
            fy[cur] = fm[left] * d_del[r] + fy[left] * eps[r];
        }
    }
    double total = 0.0;
    const size_t last = (size_t)(rows - 1) * cols;
    for (int j = 1; j < cols; j++) total += fm[last + j] + fx[last + j];
    /* Backward: B(state) = d(total)/d(state). */
    for (int i = rows - 1; i >= 1; i--) {
        for (int j = cols - 1; j >= 1; j--) {
            const size_t cur = (size_t)i * cols + j;
            double vm = (i == rows - 1) ? 1.0 : 0.0, vx = vm, vy = 0.0;
            if (i + 1 < rows && j + 1 < cols) {
                const size_t dn = (size_t)(i + 1) * cols + (j + 1);
                const double into = PRIOR(i + 1, j + 1) * bm[dn];
                vm += into * (1.0 - d_ins[i] - d_del[i]);
                vx += into * (1.0 - eps[i]);
                vy += into * (1.0 - eps[i]);
            }
            if (i + 1 < rows) {
                const size_t below = (size_t)(i + 1) * cols + j;
                vm += bx[below] * d_ins[i];
                vx += bx[below] * eps[i];
            }
            if (j + 1 < cols) {
                const size_t right = (size_t)i * cols + (j + 1);
                vm += by[right] * d_del[i - 1];
                vy += by[right] * eps[i - 1];
            }
            bm[cur] = vm;
            bx[cur] = vx;
            by[cur] = vy;
        }
    }
    const double norm = 1.0 / (total * M_LN10);
    for (int i = 1; i < rows; i++) {
        const int r = i - 1;
        double gi = 0.0, gd = 0.0, ge = 0.0, gq = 0.0;
        for (int j = 1; j < cols; j++) {
            const size_t diag = (size_t)(i - 1) * cols + (j - 1), up = (size_t)(i - 1) * cols + j;
            const size_t left = (size_t)i * cols + (j - 1), cur = (size_t)i * cols + j;
            const double p = PRIOR(i, j);
            const double dp = MATCHES(i, j) ? -1.0 : 1.0 / 3.0;
            const double bmc = bm[cur];
            gi += -fm[diag] * p * bmc + fm[up] * bx[cur];
            gd += -fm[diag] * p * bmc + fm[left] * by[cur];
            ge += -(fx[diag] + fy[diag]) * p * bmc + fx[up] * bx[cur] + fy[left] * by[cur];
            const double s = fm[diag] * (1.0 - d_ins[r] - d_del[r]) + (fx[diag] + fy[diag]) * (1.0 - eps[r]);
            gq += dp * s * bmc;
        }
        g_ins[r] += gi * norm;
        g_del[r] += gd * norm;
        g_eps[r] += ge * norm;
        g_err[r] += gq * norm;
    }
#undef PRIOR
#undef MATCHES
    free(fm); free(fx); free(fy); free(bm); free(bx); free(by);
    return log10(total) - log10(or_initial_condition());
}

/* ------------------------------------------------------------------------------------------ */
/* Whole-matrix drivers over the flattened layout of the JNI boundary                          */
/* (crates/jni/src/lib.rs:159-254): five concatenated read arrays delimited by read_offsets     */
/* (num_reads + 1 entries), concatenated haplotypes delimited by hap_offsets, output            */
/* out[r * num_haps + h]. Rows of the output are split over threads.                            */
/* ------------------------------------------------------------------------------------------ */

typedef struct {
    const uint8_t *bases, *quals, *ins, *del, *gcp;
    const int32_t* read_offsets;
    int num_reads;
    const uint8_t* hap_bases;
    const uint8_t* hap_flags; /* NULL for the plain PairHMM */
    const int32_t* hap_offsets;
    int num_haps;
    double* out;
    int next; /* shared work counter */
    pthread_mutex_t lock;
} matrix_job;

static void* matrix_worker(void* arg) {
    matrix_job* job = arg;
    for (;;) {
        pthread_mutex_lock(&job->lock);
        int r = job->next++;
        pthread_mutex_unlock(&job->lock);
        if (r >= job->num_reads) break;
        const int lo = job->read_offsets[r], len = job->read_offsets[r + 1] - lo;
        for (int h = 0; h < job->num_haps; h++) {
            const int hlo = job->hap_offsets[h], hlen = job->hap_offsets[h + 1] - hlo;
            double v;
            if (job->hap_flags)
                v = or_pd_log10_likelihood(job->hap_bases + hlo, job->hap_flags + hlo, hlen, job->bases + lo,
                                           job->quals + lo, job->ins + lo, job->del + lo, job->gcp + lo, len);
            else
                v = or_log10_likelihood(job->hap_bases + hlo, hlen, job->bases + lo, job->quals + lo, job->ins + lo,
                                        job->del + lo, job->gcp + lo, len);
            job->out[(size_t)r * job->num_haps + h] = v;
        }
    }
    return NULL;
}

int or_compute_matrix(const uint8_t* bases, const uint8_t* quals, const uint8_t* ins, const uint8_t* del,
                      const uint8_t* gcp, const int32_t* read_offsets, int num_reads, const uint8_t* hap_bases,
                      const uint8_t* hap_flags, const int32_t* hap_offsets, int num_haps, double* out,
                      int threads) {
    ensure_tables();
    matrix_job job;
    memset(&job, 0, sizeof job);
    job.bases = bases; job.quals = quals; job.ins = ins; job.del = del; job.gcp = gcp;
    job.read_offsets = read_offsets; job.num_reads = num_reads;
    job.hap_bases = hap_bases; job.hap_flags = hap_flags; job.hap_offsets = hap_offsets;
    job.num_haps = num_haps; job.out = out;
    pthread_mutex_init(&job.lock, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tids[256];
    for (int t = 1; t < threads; t++) pthread_create(&tids[t], NULL, matrix_worker, &job);
    matrix_worker(&job);
    for (int t = 1; t < threads; t++) pthread_join(tids[t], NULL);
    pthread_mutex_destroy(&job.lock);
    return 0;
}
