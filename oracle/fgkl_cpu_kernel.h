/* One lane-batched PairHMM kernel instantiation of fgkl_cpu.c -- TEST AND BENCHMARK INFRASTRUCTURE.
 *
 * Included once per (element type, lane count, instruction set) with these macros defined:
 *   FC_E        float or double
 *   FC_L        lanes (reads per batch)
 *   FC_V        GCC vector type of FC_L FC_E elements
 *   FC_NAME(x)  x with the instantiation's suffix appended
 *   FC_TARGET   function attribute selecting the instruction set (may be empty)
 *   FC_F32      1 for single precision, 0 for double
 *
 * It restates fgkl's batched kernel (crates/pairhmm/src/kernel.rs): reads on SIMD lanes, the DP
 * matrix of each haplotype swept row by row; haplotypes in sorted order resume from the snapshot of
 * the column their common prefix ends at (kernel.rs:610-765, run_hap); the snapshot taken for one
 * haplotype length is rescaled by the ratio of lengths; backward sweeps over shared suffixes
 * (kernel.rs:797-895) whose nodes a cut haplotype joins in double precision (kernel.rs:767-795).
 * Workspace layouts follow kernel.rs:424-458: every table is lane-interleaved, element i of every
 * lane one contiguous vector.
 */

#define FC_S(x) ((FC_V){} + (FC_E)(x))
#define FC_LD(p) (*(const FC_V*)(p))
#define FC_ST(p, v) (*(FC_V*)(p) = (v))

#if FC_F32
#define FC_INITIAL 0x1p120f
#define FC_BACKWARD_SCALE 0x1p120f
#define FC_HAS_MIN_ACCEPTED 1
#define FC_MIN_ACCEPTED 1e-28
#define FC_MIN_ACCEPTED_JOINED 1e-28
#define FC_LOG10_INITIAL (120.0 * 0.30102999566398119521)
#else
#define FC_INITIAL 0x1p1020
#define FC_BACKWARD_SCALE 1.0
#define FC_HAS_MIN_ACCEPTED 0
#define FC_MIN_ACCEPTED 0.0
#define FC_MIN_ACCEPTED_JOINED 1e24
#define FC_LOG10_INITIAL (1020.0 * 0.30102999566398119521)
#endif

typedef struct {
    int rows, ncodes, cols;
    size_t snap_stride, node_stride; /* elements per snapshot / backward node */
    FC_E *trans, *prior, *end_mul;   /* [row][6][lane], [row][code][lane], [row][lane] */
    uint8_t* end_rows;
    FC_E *row_prev, *row_cur;        /* [col][m,x,y][lane] */
    FC_E* snaps;                     /* [col] { m[(rows+1)][lane], x[..], y[..], acc[lane] } */
    int* snap_hap_len;
    int *lcp_counts, *snap_cols;
    int n_snap_cols;
    FC_E *bwd_prev, *bwd_cur;        /* [col][m,x][lane] */
    FC_E* nodes;                     /* [node] { m[(rows+1)][lane], y[..], s[lane] } */
    FC_E *join_m, *join_y;           /* [(rows+1)][lane] */
    FC_E acc[FC_L] __attribute__((aligned(64)));
    double joined[FC_L];
    fc_buf b_trans, b_prior, b_end, b_end_rows, b_prev, b_cur, b_snaps, b_snap_len, b_lcp, b_snap_cols, b_bprev,
        b_bcur, b_nodes, b_jm, b_jy;
} FC_NAME(ws);

typedef struct {
    FC_V mm, im, mi, ii, md, dd;
} FC_NAME(trans_t);

FC_TARGET static inline FC_NAME(trans_t) FC_NAME(load_trans)(const FC_E* trans, int r) {
    const FC_E* t = trans + (size_t)r * 6 * FC_L;
    FC_NAME(trans_t) o;
    o.mm = FC_LD(t + FC_MM * FC_L);
    o.im = FC_LD(t + FC_IM * FC_L);
    o.mi = FC_LD(t + FC_MI * FC_L);
    o.ii = FC_LD(t + FC_II * FC_L);
    o.md = FC_LD(t + FC_MD * FC_L);
    o.dd = FC_LD(t + FC_DD * FC_L);
    return o;
}

static FC_E* FC_NAME(snap_m)(FC_NAME(ws) * w, int col) { return w->snaps + (size_t)col * w->snap_stride; }
static FC_E* FC_NAME(snap_x)(FC_NAME(ws) * w, int col) {
    return FC_NAME(snap_m)(w, col) + (size_t)(w->rows + 1) * FC_L;
}
static FC_E* FC_NAME(snap_y)(FC_NAME(ws) * w, int col) {
    return FC_NAME(snap_m)(w, col) + (size_t)2 * (w->rows + 1) * FC_L;
}
static FC_E* FC_NAME(snap_acc)(FC_NAME(ws) * w, int col) {
    return FC_NAME(snap_m)(w, col) + (size_t)3 * (w->rows + 1) * FC_L;
}
static FC_E* FC_NAME(node_m)(FC_NAME(ws) * w, int node) { return w->nodes + (size_t)node * w->node_stride; }
static FC_E* FC_NAME(node_y)(FC_NAME(ws) * w, int node) {
    return FC_NAME(node_m)(w, node) + (size_t)(w->rows + 1) * FC_L;
}
static FC_E* FC_NAME(node_s)(FC_NAME(ws) * w, int node) {
    return FC_NAME(node_m)(w, node) + (size_t)2 * (w->rows + 1) * FC_L;
}

static void* FC_NAME(ws_new)(void) {
    const size_t bytes = (sizeof(FC_NAME(ws)) + 63) & ~(size_t)63;
    void* p = aligned_alloc(64, bytes);
    if (!p) abort();
    memset(p, 0, bytes);
    return p;
}

static void FC_NAME(ws_free)(void* p) {
    FC_NAME(ws)* w = p;
    if (!w) return;
    fc_buf* bufs[] = {&w->b_trans, &w->b_prior, &w->b_end, &w->b_end_rows, &w->b_prev, &w->b_cur, &w->b_snaps,
                      &w->b_snap_len, &w->b_lcp, &w->b_snap_cols, &w->b_bprev, &w->b_bcur, &w->b_nodes, &w->b_jm,
                      &w->b_jy};
    for (size_t i = 0; i < sizeof bufs / sizeof bufs[0]; i++) free(bufs[i]->p);
    free(w);
}

/* Workspace::prepare (kernel.rs:485-580): per-read tables of the batch, buffers sized for the set. */
static void FC_NAME(prepare)(FC_NAME(ws) * w, const fc_read* reads, int n, const fc_haps* hs) {
    int rows = 0;
    for (int l = 0; l < n; l++)
        if (reads[l].len > rows) rows = reads[l].len;
    const int ncodes = hs->ncodes, cols = hs->max_len + 1;
    w->rows = rows;
    w->ncodes = ncodes;
    w->cols = cols;
    w->trans = fc_grow(&w->b_trans, (size_t)rows * 6 * FC_L * sizeof(FC_E));
    w->prior = fc_grow(&w->b_prior, (size_t)rows * ncodes * FC_L * sizeof(FC_E));
    for (int r = 0; r < rows; r++) {
        FC_E* tr = w->trans + (size_t)r * 6 * FC_L;
        FC_E* pr = w->prior + (size_t)r * ncodes * FC_L;
        for (int l = 0; l < FC_L; l++) {
            if (l >= n || r >= reads[l].len) {
                for (int k = 0; k < 6; k++) tr[k * FC_L + l] = 0;
                for (int c = 0; c < ncodes; c++) pr[c * FC_L + l] = 0;
                continue;
            }
            const fc_read* rd = &reads[l];
            double t[6], p[2];
            or_transitions(rd->ins[r], rd->del[r], rd->gcp[r], t);
            for (int k = 0; k < 6; k++) tr[k * FC_L + l] = (FC_E)t[k];
            or_priors(rd->quals[r], p);
            const uint8_t rb = rd->bases[r];
            for (int c = 0; c < ncodes; c++) {
                const uint8_t hb = hs->code_byte[c];
                const int match = rb == hb || rb == 'N' || hb == 'N';
                pr[c * FC_L + l] = (FC_E)(match ? p[0] : p[1]);
            }
        }
    }
    w->end_mul = fc_grow(&w->b_end, (size_t)rows * FC_L * sizeof(FC_E));
    memset(w->end_mul, 0, (size_t)rows * FC_L * sizeof(FC_E));
    w->end_rows = fc_grow(&w->b_end_rows, (size_t)rows + 1);
    memset(w->end_rows, 0, (size_t)rows + 1);
    for (int l = 0; l < n; l++) {
        w->end_mul[(size_t)(reads[l].len - 1) * FC_L + l] = 1;
        w->end_rows[reads[l].len - 1] = 1;
    }
    w->row_prev = fc_grow(&w->b_prev, (size_t)cols * 3 * FC_L * sizeof(FC_E));
    w->row_cur = fc_grow(&w->b_cur, (size_t)cols * 3 * FC_L * sizeof(FC_E));
    w->snap_stride = (size_t)3 * (rows + 1) * FC_L + FC_L;
    w->snaps = fc_grow(&w->b_snaps, (size_t)cols * w->snap_stride * sizeof(FC_E));
    w->snap_hap_len = fc_grow(&w->b_snap_len, (size_t)cols * sizeof(int));
    /* The virtual column before the haplotype: only the initial deletion value in row zero,
     * recorded for a haplotype of length one so that the length rescaling applies. */
    memset(w->snaps, 0, w->snap_stride * sizeof(FC_E));
    FC_E* oy = FC_NAME(snap_y)(w, 0);
    for (int l = 0; l < FC_L; l++) oy[l] = FC_INITIAL;
    w->snap_hap_len[0] = 1;
    w->lcp_counts = fc_grow(&w->b_lcp, (size_t)cols * sizeof(int));
    memset(w->lcp_counts, 0, (size_t)cols * sizeof(int));
    for (int k = 1; k < hs->n; k++)
        if (!hs->dup[k]) w->lcp_counts[hs->lcp[k]]++;
    w->snap_cols = fc_grow(&w->b_snap_cols, (size_t)cols * sizeof(int));
    if (hs->nsweeps > 0) {
        w->bwd_prev = fc_grow(&w->b_bprev, (size_t)cols * 2 * FC_L * sizeof(FC_E));
        w->bwd_cur = fc_grow(&w->b_bcur, (size_t)cols * 2 * FC_L * sizeof(FC_E));
        w->node_stride = (size_t)2 * (rows + 1) * FC_L + FC_L;
        w->nodes = fc_grow(&w->b_nodes, (size_t)hs->nodes * w->node_stride * sizeof(FC_E));
        w->join_m = fc_grow(&w->b_jm, (size_t)(rows + 1) * FC_L * sizeof(FC_E));
        w->join_y = fc_grow(&w->b_jy, (size_t)(rows + 1) * FC_L * sizeof(FC_E));
    }
    for (int l = 0; l < FC_L; l++) w->joined[l] = 0.0;
}

/* Workspace::fill_last_column_node (kernel.rs:582-606): backward node 0, the last column of every
 * haplotype, from which only trailing insertions reach the end of the read. */
FC_TARGET static void FC_NAME(fill_last_column_node)(FC_NAME(ws) * w) {
    const int rows = w->rows;
    const FC_V scale = FC_S(FC_BACKWARD_SCALE);
    memset(FC_NAME(node_m)(w, 0), 0, w->node_stride * sizeof(FC_E));
    FC_E* m = FC_NAME(node_m)(w, 0);
    FC_V x_below = FC_S(0);
    for (int i = rows; i >= 1; i--) {
        const FC_V sink = scale * FC_LD(w->end_mul + (size_t)(i - 1) * FC_L);
        FC_V mi = FC_S(0), ii = FC_S(0);
        if (i < rows) {
            FC_NAME(trans_t) t = FC_NAME(load_trans)(w->trans, i);
            mi = t.mi;
            ii = t.ii;
        }
        FC_ST(m + (size_t)i * FC_L, x_below * mi + sink);
        x_below = x_below * ii + sink;
    }
}

typedef struct {
    FC_V bm_diag, by_right, bm_last;
} FC_NAME(bstate);

/* backward_segment (kernel.rs:1046-1101): row i, columns hi-1 down to lo, from row i+1 in prev. */
FC_TARGET static inline FC_NAME(bstate)
    FC_NAME(backward_segment)(const FC_NAME(trans_t) * below, FC_V md, FC_V dd, const FC_E* prior_row,
                              const uint8_t* codes, int lo, int hi, const FC_E* prev, FC_E* cur, FC_NAME(bstate) st,
                              int with_sink, FC_V sink) {
    for (int j = hi - 1; j >= lo; j--) {
        const size_t off = (size_t)j * 2 * FC_L;
        const FC_V prior = FC_LD(prior_row + (size_t)codes[j] * FC_L);
        const FC_V bx_below = FC_LD(prev + off + FC_L);
        const FC_V bm_below = FC_LD(prev + off);
        const FC_V into_match = prior * st.bm_diag;
        const FC_V indel_to_match = into_match * below->im;
        FC_V bx = bx_below * below->ii + indel_to_match;
        const FC_V by = st.by_right * dd + indel_to_match;
        FC_V bm = st.by_right * md + (bx_below * below->mi + into_match * below->mm);
        if (with_sink) {
            bm = bm + sink;
            bx = bx + sink;
        }
        FC_ST(cur + off, bm);
        FC_ST(cur + off + FC_L, bx);
        st.bm_diag = bm_below;
        st.by_right = by;
        st.bm_last = bm;
    }
    return st;
}

/* backward_row_zero (kernel.rs:1104-1126): paths starting in row 0 move straight to the match
 * state of row 1 one column right; only their running sum is kept. */
FC_TARGET static inline FC_NAME(bstate)
    FC_NAME(backward_row_zero)(FC_V im, const FC_E* prior_row, const uint8_t* codes, int lo, int hi,
                               const FC_E* prev, FC_NAME(bstate) st, FC_V* starts_after) {
    for (int j = hi - 1; j >= lo; j--) {
        const FC_V prior = FC_LD(prior_row + (size_t)codes[j] * FC_L);
        const FC_V by = prior * st.bm_diag * im;
        *starts_after = *starts_after + by;
        st.bm_diag = FC_LD(prev + (size_t)j * 2 * FC_L);
        st.by_right = by;
    }
    return st;
}

/* Workspace::run_hap_backward (kernel.rs:797-895): one backward sweep over depths
 * resume+1..need of its haplotype, rows from the last up to 0, storing the nodes it writes. */
FC_TARGET static void FC_NAME(run_hap_backward)(FC_NAME(ws) * w, const fc_sweep* sw, const uint8_t* codes,
                                                int hap_len) {
    const int rows = w->rows, ncodes = w->ncodes;
    const int right = hap_len - sw->resume, left = hap_len - sw->need;
    const FC_E* sm = FC_NAME(node_m)(w, sw->start);
    const FC_E* sy = FC_NAME(node_y)(w, sw->start);
    const FC_E* ss = FC_NAME(node_s)(w, sw->start);
    const FC_V zero = FC_S(0), scale = FC_S(FC_BACKWARD_SCALE);
    FC_E* prev = w->bwd_prev;
    FC_E* cur = w->bwd_cur;
    for (int j = left; j < right; j++) {
        FC_ST(prev + (size_t)j * 2 * FC_L, zero);
        FC_ST(prev + (size_t)j * 2 * FC_L + FC_L, zero);
    }
    FC_V starts_after = FC_LD(ss);
    for (int i = rows; i >= 0; i--) {
        FC_NAME(trans_t) below;
        if (i < rows) {
            below = FC_NAME(load_trans)(w->trans, i);
        } else {
            below.mm = below.im = below.mi = below.ii = below.md = below.dd = zero;
        }
        const FC_E* prior_row = w->prior + (size_t)(i < rows ? i : rows - 1) * ncodes * FC_L;
        FC_V md = zero, dd = zero;
        if (i >= 1) {
            FC_NAME(trans_t) t = FC_NAME(load_trans)(w->trans, i - 1);
            md = t.md;
            dd = t.dd;
        }
        const int with_sink = i >= 1 && w->end_rows[i - 1];
        const FC_V sink = with_sink ? scale * FC_LD(w->end_mul + (size_t)(i - 1) * FC_L) : zero;
        FC_NAME(bstate) st;
        st.bm_diag = i < rows ? FC_LD(sm + (size_t)(i + 1) * FC_L) : zero;
        st.by_right = FC_LD(sy + (size_t)i * FC_L);
        st.bm_last = zero;
        int hi = right;
        for (int k = 0; k <= sw->nwrites; k++) {
            int lo, node = -1;
            if (k < sw->nwrites) {
                lo = hap_len - sw->wdepth[k];
                node = sw->wnode[k];
            } else {
                lo = left;
            }
            if (lo < hi) {
                if (i == 0)
                    st = FC_NAME(backward_row_zero)(below.im, prior_row, codes, lo, hi, prev, st, &starts_after);
                else
                    st = FC_NAME(backward_segment)(&below, md, dd, prior_row, codes, lo, hi, prev, cur, st,
                                                   with_sink, sink);
                hi = lo;
            }
            if (node >= 0) {
                FC_ST(FC_NAME(node_y)(w, node) + (size_t)i * FC_L, st.by_right);
                if (i == 0)
                    FC_ST(FC_NAME(node_s)(w, node), starts_after);
                else
                    FC_ST(FC_NAME(node_m)(w, node) + (size_t)i * FC_L, st.bm_last);
            }
        }
        if (i > 0) {
            FC_E* t = prev;
            prev = cur;
            cur = t;
        }
    }
}

typedef struct {
    FC_V m_diag, x_diag, y_diag, m_left, x_left, y_left;
} FC_NAME(cstate);

/* dp_segment (kernel.rs:975-1028): columns lo+1..hi of the current row; with acc, also sums
 * match plus insertion over them into rowsum. */
FC_TARGET static inline FC_NAME(cstate)
    FC_NAME(dp_segment)(const FC_NAME(trans_t) * t, const FC_E* prior_row, const uint8_t* codes, int lo, int hi,
                        const FC_E* prev, FC_E* cur, FC_NAME(cstate) st, int acc, FC_V* rowsum) {
    FC_V sum = *rowsum;
    for (int k = lo; k < hi; k++) {
        const size_t off = (size_t)(k + 1) * 3 * FC_L;
        const FC_V prior = FC_LD(prior_row + (size_t)codes[k] * FC_L);
        const FC_V m_up = FC_LD(prev + off), x_up = FC_LD(prev + off + FC_L), y_up = FC_LD(prev + off + 2 * FC_L);
        const FC_V m = prior * (st.y_diag * t->im + (st.x_diag * t->im + st.m_diag * t->mm));
        const FC_V x = x_up * t->ii + m_up * t->mi;
        const FC_V y = st.y_left * t->dd + st.m_left * t->md;
        FC_ST(cur + off, m);
        FC_ST(cur + off + FC_L, x);
        FC_ST(cur + off + 2 * FC_L, y);
        if (acc) sum = sum + (m + x);
        st.m_diag = m_up;
        st.x_diag = x_up;
        st.y_diag = y_up;
        st.m_left = m;
        st.x_left = x;
        st.y_left = y;
    }
    *rowsum = sum;
    return st;
}

/* Workspace::run_hap (kernel.rs:610-765): columns start+1..stop of one haplotype of length hap_len,
 * column start coming from its snapshot; records the snapshots in snap_cols and, when stopping at a
 * cut, the forward values of column stop+1 entered from column stop. */
FC_TARGET static void FC_NAME(run_hap)(FC_NAME(ws) * w, int start, int stop, int hap_len, const uint8_t* codes) {
    const int join = stop < hap_len;
    const int rows = w->rows, ncodes = w->ncodes;
    const FC_E* src_m = FC_NAME(snap_m)(w, start);
    const FC_E* src_x = FC_NAME(snap_x)(w, start);
    const FC_E* src_y = FC_NAME(snap_y)(w, start);
    const FC_E* src_acc = FC_NAME(snap_acc)(w, start);
    const FC_V zero = FC_S(0);
    const FC_V init = FC_S((FC_E)((double)FC_INITIAL / (double)hap_len));
    const FC_V scale = FC_S((FC_E)((double)w->snap_hap_len[start] / (double)hap_len));
    FC_E* prev = w->row_prev;
    FC_E* cur = w->row_cur;
    for (int j = start; j <= stop; j++) {
        FC_E* col = prev + (size_t)j * 3 * FC_L;
        FC_ST(col, zero);
        FC_ST(col + FC_L, zero);
        FC_ST(col + 2 * FC_L, init);
    }
    FC_V acc_v = FC_LD(src_acc) * scale;
    for (int s = 0; s < w->n_snap_cols; s++) {
        const int q = w->snap_cols[s];
        w->snap_hap_len[q] = hap_len;
        FC_ST(FC_NAME(snap_m)(w, q), zero);
        FC_ST(FC_NAME(snap_x)(w, q), zero);
        FC_ST(FC_NAME(snap_y)(w, q), init);
        FC_ST(FC_NAME(snap_acc)(w, q), acc_v);
    }
    if (start == stop && !join) {
        FC_ST(w->acc, acc_v);
        return;
    }
    for (int i = 1; i <= rows; i++) {
        const int r = i - 1;
        const FC_NAME(trans_t) t = FC_NAME(load_trans)(w->trans, r);
        const FC_E* prior_row = w->prior + (size_t)r * ncodes * FC_L;
        FC_NAME(cstate) st;
        st.m_diag = FC_LD(src_m + (size_t)(i - 1) * FC_L) * scale;
        st.x_diag = FC_LD(src_x + (size_t)(i - 1) * FC_L) * scale;
        st.y_diag = FC_LD(src_y + (size_t)(i - 1) * FC_L) * scale;
        st.m_left = FC_LD(src_m + (size_t)i * FC_L) * scale;
        st.x_left = FC_LD(src_x + (size_t)i * FC_L) * scale;
        st.y_left = FC_LD(src_y + (size_t)i * FC_L) * scale;
        FC_V rowsum = zero;
        if (w->end_rows[r]) {
            /* A read ends on this row: every snapshot also needs the row's sum up to its column. */
            const FC_V e = FC_LD(w->end_mul + (size_t)r * FC_L);
            int lo = start;
            for (int s = 0; s < w->n_snap_cols; s++) {
                const int q = w->snap_cols[s];
                if (q > lo) st = FC_NAME(dp_segment)(&t, prior_row, codes, lo, q, prev, cur, st, 1, &rowsum);
                FC_ST(FC_NAME(snap_m)(w, q) + (size_t)i * FC_L, st.m_left);
                FC_ST(FC_NAME(snap_x)(w, q) + (size_t)i * FC_L, st.x_left);
                FC_ST(FC_NAME(snap_y)(w, q) + (size_t)i * FC_L, st.y_left);
                FC_E* sa = FC_NAME(snap_acc)(w, q);
                FC_ST(sa, e * rowsum + FC_LD(sa));
                lo = q;
            }
            if (stop > lo) st = FC_NAME(dp_segment)(&t, prior_row, codes, lo, stop, prev, cur, st, 1, &rowsum);
            acc_v = e * rowsum + acc_v;
        } else {
            if (stop > start) st = FC_NAME(dp_segment)(&t, prior_row, codes, start, stop, prev, cur, st, 0, &rowsum);
            for (int s = 0; s < w->n_snap_cols; s++) {
                const int q = w->snap_cols[s];
                const FC_E* col = cur + (size_t)q * 3 * FC_L;
                FC_ST(FC_NAME(snap_m)(w, q) + (size_t)i * FC_L, FC_LD(col));
                FC_ST(FC_NAME(snap_x)(w, q) + (size_t)i * FC_L, FC_LD(col + FC_L));
                FC_ST(FC_NAME(snap_y)(w, q) + (size_t)i * FC_L, FC_LD(col + 2 * FC_L));
            }
        }
        if (join) {
            /* Column stop+1 as dp_segment would compute it, without its insertion value: paths
             * enter a column only through match or deletion. */
            const FC_V prior = FC_LD(prior_row + (size_t)codes[stop] * FC_L);
            const FC_V m = prior * (st.y_diag * t.im + (st.x_diag * t.im + st.m_diag * t.mm));
            const FC_V y = st.y_left * t.dd + st.m_left * t.md;
            FC_ST(w->join_m + (size_t)i * FC_L, m);
            FC_ST(w->join_y + (size_t)i * FC_L, y);
        }
        FC_E* tmp = prev;
        prev = cur;
        cur = tmp;
    }
    FC_ST(w->acc, acc_v);
}

/* Workspace::join (kernel.rs:767-795): paths ending before the cut, plus those entering the cut
 * column times their backward mass, plus those starting at the cut column or later, in double. */
FC_TARGET static void FC_NAME(join)(FC_NAME(ws) * w, int node, int hap_len) {
    double crossing[FC_L];
    for (int l = 0; l < FC_L; l++) crossing[l] = 0.0;
    const FC_E* bm = FC_NAME(node_m)(w, node);
    const FC_E* by = FC_NAME(node_y)(w, node);
    const FC_E* bs = FC_NAME(node_s)(w, node);
    for (int i = 1; i <= w->rows; i++) {
        const FC_E* fm = w->join_m + (size_t)i * FC_L;
        const FC_E* fy = w->join_y + (size_t)i * FC_L;
        const FC_E* nm = bm + (size_t)i * FC_L;
        const FC_E* ny = by + (size_t)i * FC_L;
        for (int l = 0; l < FC_L; l++)
            crossing[l] += (double)fm[l] * (double)nm[l] + (double)fy[l] * (double)ny[l];
    }
    const double init = (double)(FC_E)((double)FC_INITIAL / (double)hap_len);
    const double scale = (double)FC_BACKWARD_SCALE;
    for (int l = 0; l < FC_L; l++) {
        const double starts_after = init * (double)bs[l];
        w->joined[l] = (double)w->acc[l] + (crossing[l] + starts_after) / scale;
    }
}

/* finish_lane (kernel.rs:897-915). */
static inline double FC_NAME(finish_lane)(double raw, int has_min, double min_accepted, int lane, int k,
                                          fc_pairs* fallback) {
    if (has_min && (isnan(raw) || raw < min_accepted)) {
        fc_pairs_push(fallback, lane, k);
        return NAN;
    }
    return log10(raw) - FC_LOG10_INITIAL;
}

/* Runner::run_impl (kernel.rs:220-290): at most FC_L reads against every haplotype of the set,
 * out[lane * n + sorted hap]; lost pairs appended to fallback as (lane, sorted hap), NaN in place. */
FC_TARGET static void FC_NAME(run_batch_impl)(void* wsp, const fc_read* reads, int n, const void* hsp, double* out,
                                              fc_pairs* fallback) {
    FC_NAME(ws)* w = wsp;
    const fc_haps* hs = hsp;
    FC_NAME(prepare)(w, reads, n, hs);
    if (hs->nsweeps > 0) {
        FC_NAME(fill_last_column_node)(w);
        for (int s = 0; s < hs->nsweeps; s++) {
            const fc_sweep* sw = &hs->sweeps[s];
            FC_NAME(run_hap_backward)(w, sw, hs->codes + hs->code_off[sw->hap], hs->len[sw->hap]);
        }
    }
    const int nh = hs->n;
    for (int k = 0; k < nh; k++) {
        if (hs->dup[k]) {
            for (int l = 0; l < n; l++) {
                const double result = out[(size_t)l * nh + k - 1];
                if (isnan(result)) fc_pairs_push(fallback, l, k);
                out[(size_t)l * nh + k] = result;
            }
            continue;
        }
        const int start = hs->lcp[k];
        if (k > 0) w->lcp_counts[start]--;
        const int hap_len = hs->len[k];
        const int cut_col = hs->cut_col[k];
        const int stop = cut_col > 0 ? cut_col - 1 : hap_len;
        w->n_snap_cols = 0;
        for (int q = start + 1; q <= stop; q++)
            if (w->lcp_counts[q] > 0) w->snap_cols[w->n_snap_cols++] = q;
        FC_NAME(run_hap)(w, start, stop, hap_len, hs->codes + hs->code_off[k]);
        int has_min;
        double min_accepted;
        if (cut_col == 0) {
            for (int l = 0; l < n; l++) w->joined[l] = (double)w->acc[l];
            has_min = FC_HAS_MIN_ACCEPTED;
            min_accepted = FC_MIN_ACCEPTED;
        } else {
            FC_NAME(join)(w, hs->cut_node[k], hap_len);
            has_min = 1;
            min_accepted = FC_MIN_ACCEPTED_JOINED;
        }
        for (int l = 0; l < n; l++)
            out[(size_t)l * nh + k] = FC_NAME(finish_lane)(w->joined[l], has_min, min_accepted, l, k, fallback);
    }
}

/* The runner entry: flush subnormals to zero around the batch (simd.rs:204-228). */
static void FC_NAME(run_batch)(void* wsp, const fc_read* reads, int n, const void* hs, double* out,
                               fc_pairs* fallback) {
    const unsigned saved = _mm_getcsr();
    _mm_setcsr(saved | 0x8040u);
    FC_NAME(run_batch_impl)(wsp, reads, n, hs, out, fallback);
    _mm_setcsr(saved);
}

#undef FC_S
#undef FC_LD
#undef FC_ST
#undef FC_INITIAL
#undef FC_BACKWARD_SCALE
#undef FC_HAS_MIN_ACCEPTED
#undef FC_MIN_ACCEPTED
#undef FC_MIN_ACCEPTED_JOINED
#undef FC_LOG10_INITIAL
