/* One lane-batched PD-HMM kernel instantiation of fgkl_cpu.c -- TEST AND BENCHMARK INFRASTRUCTURE.
 *
 * Included after fgkl_cpu_kernel.h's instantiation with the same macros (FC_E, FC_L, FC_V, FC_NAME,
 * FC_TARGET, FC_F32) plus FC_VI, the integer vector type of FC_V's shape. It restates fgkl's batched PD kernel (crates/pairhmm/src/pd_kernel.rs):
 * reads on SIMD lanes, each haplotype swept row by row; per-column deletion states resolved on the
 * host into runs of columns (first row, later rows), each run computed by the inner loop for its
 * state and DEL_END flag (pd_kernel.rs:748-920); GATK's three branch matrices kept as running
 * vectors and stored only at DEL_END columns; prefix sharing from snapshots that also hold the
 * branch values (pd_kernel.rs:535-656).
 */

#define FC_S(x) ((FC_V){} + (FC_E)(x))
#define FC_LD(p) (*(const FC_V*)(p))
#define FC_ST(p, v) (*(FC_V*)(p) = (v))
/* Lane-wise maximum by a compare mask (FC_VI: the integer vector of FC_V's shape); the operands
 * are finite and non-negative in this recurrence (simd.rs Float::max). */
#define FC_MAXV(a, b) ((FC_V)((((FC_VI)(a)) & ((FC_VI)((a) > (b)))) | (((FC_VI)(b)) & ~((FC_VI)((a) > (b))))))

#if FC_F32
#define FC_INITIAL 0x1p120f
#define FC_HAS_MIN_ACCEPTED 1
#define FC_MIN_ACCEPTED 1e-28
#define FC_LOG10_INITIAL (120.0 * 0.30102999566398119521)
#else
#define FC_INITIAL 0x1p1020
#define FC_HAS_MIN_ACCEPTED 0
#define FC_MIN_ACCEPTED 0.0
#define FC_LOG10_INITIAL (1020.0 * 0.30102999566398119521)
#endif

typedef struct {
    int rows, nsets, cols;
    size_t snap_stride; /* elements per snapshot: m, x, y, bm, bx, by rows then acc */
    FC_E *trans, *prior, *end_mul;
    uint8_t* end_rows;
    FC_E* prev[6]; /* m, x, y, bm, bx, by: [col][lane] */
    FC_E* cur[6];
    FC_E* snaps;
    int* snap_hap_len;
    int *lcp_counts, *snap_cols;
    int n_snap_cols;
    fc_run *first_runs, *later_runs;
    int n_first, n_later;
    FC_E acc[FC_L] __attribute__((aligned(64)));
    fc_buf b_trans, b_prior, b_end, b_end_rows, b_prev, b_cur, b_snaps, b_snap_len, b_lcp, b_snap_cols, b_runs;
} FC_NAME(pdws);

static FC_E* FC_NAME(pd_snap)(FC_NAME(pdws) * w, int col, int part) {
    return w->snaps + (size_t)col * w->snap_stride + (size_t)part * (w->rows + 1) * FC_L;
}

static void* FC_NAME(pdws_new)(void) {
    const size_t bytes = (sizeof(FC_NAME(pdws)) + 63) & ~(size_t)63;
    void* p = aligned_alloc(64, bytes);
    if (!p) abort();
    memset(p, 0, bytes);
    return p;
}

static void FC_NAME(pdws_free)(void* p) {
    FC_NAME(pdws)* w = p;
    if (!w) return;
    fc_buf* bufs[] = {&w->b_trans, &w->b_prior, &w->b_end, &w->b_end_rows, &w->b_prev, &w->b_cur,
                      &w->b_snaps, &w->b_snap_len, &w->b_lcp, &w->b_snap_cols, &w->b_runs};
    for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; i++) free(bufs[i]->p);
    free(w);
}

/* Workspace::prepare (pd_kernel.rs:473-533). */
static void FC_NAME(pd_prepare)(FC_NAME(pdws) * w, const fc_read* reads, int n, const fc_pdhaps* hs) {
    int rows = 0;
    for (int l = 0; l < n; l++)
        if (reads[l].len > rows) rows = reads[l].len;
    const int nsets = hs->nsets, cols = hs->max_len + 1;
    w->rows = rows;
    w->nsets = nsets;
    w->cols = cols;
    w->trans = fc_grow(&w->b_trans, (size_t)rows * 6 * FC_L * sizeof(FC_E));
    w->prior = fc_grow(&w->b_prior, (size_t)rows * nsets * FC_L * sizeof(FC_E));
    memset(w->trans, 0, (size_t)rows * 6 * FC_L * sizeof(FC_E));
    memset(w->prior, 0, (size_t)rows * nsets * FC_L * sizeof(FC_E));
    w->end_mul = fc_grow(&w->b_end, (size_t)rows * FC_L * sizeof(FC_E));
    memset(w->end_mul, 0, (size_t)rows * FC_L * sizeof(FC_E));
    w->end_rows = fc_grow(&w->b_end_rows, (size_t)rows + 1);
    memset(w->end_rows, 0, (size_t)rows + 1);
    for (int l = 0; l < n; l++) {
        const fc_read* rd = &reads[l];
        for (int r = 0; r < rd->len; r++) {
            double t[6], p[2];
            or_transitions(rd->ins[r], rd->del[r], rd->gcp[r], t);
            for (int k = 0; k < 6; k++) w->trans[((size_t)r * 6 + k) * FC_L + l] = (FC_E)t[k];
            or_priors(rd->quals[r], p);
            for (int c = 0; c < nsets; c++)
                w->prior[((size_t)r * nsets + c) * FC_L + l] = (FC_E)(fc_mset_accepts(hs->sets[c], rd->bases[r]) ? p[0] : p[1]);
        }
        w->end_mul[(size_t)(rd->len - 1) * FC_L + l] = 1;
        w->end_rows[rd->len - 1] = 1;
    }
    char* pb = fc_grow(&w->b_prev, (size_t)6 * cols * FC_L * sizeof(FC_E));
    char* cb = fc_grow(&w->b_cur, (size_t)6 * cols * FC_L * sizeof(FC_E));
    for (int a = 0; a < 6; a++) {
        w->prev[a] = (FC_E*)pb + (size_t)a * cols * FC_L;
        w->cur[a] = (FC_E*)cb + (size_t)a * cols * FC_L;
    }
    w->snap_stride = (size_t)6 * (rows + 1) * FC_L + FC_L;
    w->snaps = fc_grow(&w->b_snaps, (size_t)cols * w->snap_stride * sizeof(FC_E));
    w->snap_hap_len = fc_grow(&w->b_snap_len, (size_t)cols * sizeof(int));
    /* The virtual column before the haplotype: the initial deletion value in row zero, zero branch
     * values, recorded for a haplotype of length one. */
    memset(w->snaps, 0, w->snap_stride * sizeof(FC_E));
    FC_E* oy = FC_NAME(pd_snap)(w, 0, 2);
    for (int l = 0; l < FC_L; l++) oy[l] = FC_INITIAL;
    w->snap_hap_len[0] = 1;
    w->lcp_counts = fc_grow(&w->b_lcp, (size_t)cols * sizeof(int));
    memset(w->lcp_counts, 0, (size_t)cols * sizeof(int));
    for (int k = 1; k < hs->n; k++) w->lcp_counts[hs->lcp[k]]++;
    w->snap_cols = fc_grow(&w->b_snap_cols, (size_t)cols * sizeof(int));
}

typedef struct {
    FC_V m_diag, x_diag, y_diag, m_left, x_left, y_left;
    FC_V bm, bx, by; /* branch values at the column one back */
} FC_NAME(pdst);

/* dp_segment (pd_kernel.rs:800-920): columns lo+1..hi of the current row in one state. */
FC_TARGET static inline void FC_NAME(pd_segment)(FC_NAME(pdws) * w, FC_NAME(trans_t) * t, const FC_E* prior_row,
                                                 const uint8_t* codes, int lo, int hi, int state, int del_end, int acc,
                                                 FC_NAME(pdst) * s, FC_V* rowsum) {
    FC_E *const *pv = w->prev, *const *cu = w->cur;
    const FC_V entry_m = s->m_left, entry_x = s->x_left, entry_y = s->y_left;
    FC_V sum = *rowsum;
    for (int j = lo; j < hi; j++) {
        const size_t off = (size_t)(j + 1) * FC_L;
        const FC_V prior = FC_LD(prior_row + (size_t)codes[j] * FC_L);
        const FC_V m_up = FC_LD(pv[0] + off), x_up = FC_LD(pv[1] + off), y_up = FC_LD(pv[2] + off);
        FC_V bm, bx, by;
        if (state == FC_PD_NORMAL) {
            bm = s->m_left;
            bx = s->x_left;
            by = s->y_left;
        } else if (state == FC_PD_INSIDE_DEL) {
            bm = s->bm;
            bx = s->bx;
            by = s->by;
        } else {
            bm = FC_MAXV(s->bm, s->m_left);
            bx = FC_MAXV(s->bx, s->x_left);
            by = FC_MAXV(s->by, s->y_left);
        }
        FC_V m, y;
        if (state == FC_PD_AFTER_DEL) {
            const FC_V m_d = FC_MAXV(FC_LD(pv[3] + off - FC_L), s->m_diag);
            const FC_V x_d = FC_MAXV(FC_LD(pv[4] + off - FC_L), s->x_diag);
            const FC_V y_d = FC_MAXV(FC_LD(pv[5] + off - FC_L), s->y_diag);
            m = prior * (y_d * t->im + (x_d * t->im + m_d * t->mm));
            y = by * t->dd + bm * t->md;
        } else {
            m = prior * (s->y_diag * t->im + (s->x_diag * t->im + s->m_diag * t->mm));
            y = s->y_left * t->dd + s->m_left * t->md;
        }
        FC_V x;
        if (del_end) {
            const FC_V bm_up = FC_LD(pv[3] + off), bx_up = FC_LD(pv[4] + off);
            x = FC_MAXV(bx_up, x_up) * t->ii + FC_MAXV(bm_up, m_up) * t->mi;
        } else {
            x = x_up * t->ii + m_up * t->mi;
        }
        FC_ST(cu[0] + off, m);
        FC_ST(cu[1] + off, x);
        FC_ST(cu[2] + off, y);
        if (del_end) {
            FC_ST(cu[3] + off, bm);
            FC_ST(cu[4] + off, bx);
            FC_ST(cu[5] + off, by);
        }
        if (acc) sum = sum + (m + x);
        if (state == FC_PD_AFTER_DEL) {
            s->bm = bm;
            s->bx = bx;
            s->by = by;
        }
        s->m_diag = m_up;
        s->x_diag = x_up;
        s->y_diag = y_up;
        s->m_left = m;
        s->x_left = x;
        s->y_left = y;
    }
    if (state == FC_PD_NORMAL) {
        /* The branch values at the last column are the DP values one column before it. */
        if (hi - lo >= 2) {
            const size_t off = (size_t)(hi - 1) * FC_L;
            s->bm = FC_LD(cu[0] + off);
            s->bx = FC_LD(cu[1] + off);
            s->by = FC_LD(cu[2] + off);
        } else {
            s->bm = entry_m;
            s->bx = entry_x;
            s->by = entry_y;
        }
    }
    *rowsum = sum;
}

/* Workspace::run_hap (pd_kernel.rs:535-656): haplotype k from the snapshot at column start. */
FC_TARGET static void FC_NAME(pd_run_hap)(FC_NAME(pdws) * w, const fc_pdhaps* hs, int k, int start) {
    const int rows = w->rows, nsets = w->nsets, hap_len = hs->len[k];
    const uint8_t* codes = hs->codes + hs->code_off[k];
    w->n_first = fc_cut_runs(hs->first_row[k], hs->n_first[k], start, w->snap_cols, w->n_snap_cols, w->first_runs);
    w->n_later = fc_cut_runs(hs->later_rows[k], hs->n_later[k], start, w->snap_cols, w->n_snap_cols, w->later_runs);
    const FC_V zero = FC_S(0);
    const FC_V init = FC_S((FC_E)((double)FC_INITIAL / (double)hap_len));
    const FC_V scale = FC_S((FC_E)((double)w->snap_hap_len[start] / (double)hap_len));
    const FC_E* src[6];
    for (int a = 0; a < 6; a++) src[a] = FC_NAME(pd_snap)(w, start, a);
    const FC_E* src_acc = FC_NAME(pd_snap)(w, start, 6);
    /* Row zero: free deletions along the haplotype, zero branch values at DEL_END columns. */
    for (int j = start; j <= hap_len; j++) {
        FC_ST(w->prev[0] + (size_t)j * FC_L, zero);
        FC_ST(w->prev[1] + (size_t)j * FC_L, zero);
        FC_ST(w->prev[2] + (size_t)j * FC_L, init);
    }
    for (int d = 0; d < hs->n_del_end[k]; d++) {
        const int j = hs->del_end_cols[k][d];
        FC_ST(w->prev[3] + (size_t)j * FC_L, zero);
        FC_ST(w->prev[4] + (size_t)j * FC_L, zero);
        FC_ST(w->prev[5] + (size_t)j * FC_L, zero);
    }
    FC_V acc_v = FC_LD(src_acc) * scale;
    for (int s = 0; s < w->n_snap_cols; s++) {
        const int q = w->snap_cols[s];
        w->snap_hap_len[q] = hap_len;
        for (int a = 0; a < 6; a++) FC_ST(FC_NAME(pd_snap)(w, q, a), a == 2 ? init : zero);
        FC_ST(FC_NAME(pd_snap)(w, q, 6), acc_v);
    }
    if (start == hap_len) {
        FC_ST(w->acc, acc_v);
        return;
    }
    for (int i = 1; i <= rows; i++) {
        const int r = i - 1;
        FC_NAME(trans_t) t = FC_NAME(load_trans)(w->trans, r);
        const FC_E* prior_row = w->prior + (size_t)r * nsets * FC_L;
        FC_NAME(pdst) st;
        st.m_diag = FC_LD(src[0] + (size_t)(i - 1) * FC_L) * scale;
        st.x_diag = FC_LD(src[1] + (size_t)(i - 1) * FC_L) * scale;
        st.y_diag = FC_LD(src[2] + (size_t)(i - 1) * FC_L) * scale;
        st.m_left = FC_LD(src[0] + (size_t)i * FC_L) * scale;
        st.x_left = FC_LD(src[1] + (size_t)i * FC_L) * scale;
        st.y_left = FC_LD(src[2] + (size_t)i * FC_L) * scale;
        st.bm = FC_LD(src[3] + (size_t)i * FC_L) * scale;
        st.bx = FC_LD(src[4] + (size_t)i * FC_L) * scale;
        st.by = FC_LD(src[5] + (size_t)i * FC_L) * scale;
        for (int a = 3; a < 6; a++) FC_ST(w->prev[a] + (size_t)start * FC_L, FC_LD(src[a] + (size_t)(i - 1) * FC_L) * scale);
        const fc_run* runs = i == 1 ? w->first_runs : w->later_runs;
        const int nr = i == 1 ? w->n_first : w->n_later;
        const int ends_here = w->end_rows[r];
        FC_V rowsum = zero;
        for (int u = 0; u < nr; u++) {
            const fc_run* run = &runs[u];
            FC_NAME(pd_segment)(w, &t, prior_row, codes, run->lo, run->hi, run->state, run->del_end, ends_here, &st,
                                &rowsum);
            if (run->at_snap) {
                const int q = run->hi;
                FC_ST(FC_NAME(pd_snap)(w, q, 0) + (size_t)i * FC_L, st.m_left);
                FC_ST(FC_NAME(pd_snap)(w, q, 1) + (size_t)i * FC_L, st.x_left);
                FC_ST(FC_NAME(pd_snap)(w, q, 2) + (size_t)i * FC_L, st.y_left);
                FC_ST(FC_NAME(pd_snap)(w, q, 3) + (size_t)i * FC_L, st.bm);
                FC_ST(FC_NAME(pd_snap)(w, q, 4) + (size_t)i * FC_L, st.bx);
                FC_ST(FC_NAME(pd_snap)(w, q, 5) + (size_t)i * FC_L, st.by);
                if (ends_here) {
                    FC_E* sa = FC_NAME(pd_snap)(w, q, 6);
                    FC_ST(sa, FC_LD(w->end_mul + (size_t)r * FC_L) * rowsum + FC_LD(sa));
                }
            }
        }
        if (ends_here) acc_v = FC_LD(w->end_mul + (size_t)r * FC_L) * rowsum + acc_v;
        for (int a = 0; a < 6; a++) {
            FC_E* tmp = w->prev[a];
            w->prev[a] = w->cur[a];
            w->cur[a] = tmp;
        }
    }
    FC_ST(w->acc, acc_v);
}

/* PdRunner::run_impl (pd_kernel.rs:290-330). */
FC_TARGET static void FC_NAME(pd_run_batch_impl)(void* wsp, const fc_read* reads, int n, const void* hsp, double* out,
                                                 fc_pairs* fallback) {
    FC_NAME(pdws)* w = wsp;
    const fc_pdhaps* hs = hsp;
    FC_NAME(pd_prepare)(w, reads, n, hs);
    w->first_runs = fc_grow(&w->b_runs, sizeof(fc_run) * 2 * (size_t)(2 * w->cols + 2));
    w->later_runs = w->first_runs + 2 * w->cols + 2;
    const int nh = hs->n;
    for (int k = 0; k < nh; k++) {
        const int start = hs->lcp[k];
        if (k > 0) w->lcp_counts[start]--;
        w->n_snap_cols = 0;
        for (int q = start + 1; q <= hs->len[k]; q++)
            if (w->lcp_counts[q] > 0) w->snap_cols[w->n_snap_cols++] = q;
        FC_NAME(pd_run_hap)(w, hs, k, start);
        for (int l = 0; l < n; l++) {
            const double raw = (double)w->acc[l];
            if (FC_HAS_MIN_ACCEPTED && (isnan(raw) || raw < FC_MIN_ACCEPTED)) {
                fc_pairs_push(fallback, l, k);
                out[(size_t)l * nh + k] = NAN;
            } else {
                out[(size_t)l * nh + k] = log10(raw) - FC_LOG10_INITIAL;
            }
        }
    }
}

static void FC_NAME(pd_run_batch)(void* wsp, const fc_read* reads, int n, const void* hs, double* out,
                                  fc_pairs* fallback) {
    const unsigned saved = _mm_getcsr();
    _mm_setcsr(saved | 0x8040u);
    FC_NAME(pd_run_batch_impl)(wsp, reads, n, hs, out, fallback);
    _mm_setcsr(saved);
}

#undef FC_S
#undef FC_LD
#undef FC_ST
#undef FC_MAXV
#undef FC_INITIAL
#undef FC_HAS_MIN_ACCEPTED
#undef FC_MIN_ACCEPTED
#undef FC_LOG10_INITIAL
