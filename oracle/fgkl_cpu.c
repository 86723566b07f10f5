/* CPU restatement of fgkl's batched PairHMM -- TEST AND BENCHMARK INFRASTRUCTURE ONLY.
 *
 * The timed CPU reference of the benchmark (its reference arm and its cpu_baseline leg) and a second
 * checker in the CPU tests; the product never loads it. fgkl itself is a Rust crate and no Rust
 * toolchain exists here, so this file restates, in C, the algorithm its CPU path runs:
 *   - crates/pairhmm/src/lib.rs:346-550 (Batcher): reads sorted longest first, batches of the
 *     runner's lane count (16 FP32 lanes on AVX-512, a remainder of at most 8 on AVX2 lanes),
 *     FP32 first, lost pairs recomputed in FP64 -- a read lost against a third or more of the
 *     haplotypes with all of them in one shared sweep, other pairs one haplotype at a time -- and
 *     pairs whose joined FP64 result is too small for the backward values recomputed once more
 *     without suffix sharing;
 *   - crates/pairhmm/src/kernel.rs:34-108 (SortedHaps: sort, prior-table codes, common prefixes,
 *     duplicates), kernel.rs:220-290 and 485-1126 (the kernel, in fgkl_cpu_kernel.h);
 *   - crates/pairhmm/src/plan.rs (SuffixPlan: cut depths, backward sweeps, node numbering).
 * The numeric model (transition and prior tables) is the oracle's (pairhmm_oracle.c). Regions run
 * on a pool of threads, one region at a time per thread; every call of fgkl runs on its calling
 * thread, so a caller with many regions gets the same parallelism from its own threads.
 *
 * Instruction sets are chosen at run time: AVX-512 wide and AVX2 narrow lanes when the CPU has
 * AVX-512F, AVX2 lanes otherwise, and portable GCC vectors (8 FP32 / 4 FP64 lanes) without either.
 */
#include <immintrin.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* From pairhmm_oracle.c: GATK's tables (crates/pairhmm/src/model.rs:37-83). */
void or_transitions(int ins_qual, int del_qual, int gcp, double* t);
void or_priors(int qual, double* out);

enum { FC_MM = 0, FC_IM = 1, FC_MI = 2, FC_II = 3, FC_MD = 4, FC_DD = 5 };

/* A growable 64-byte aligned buffer; contents are not kept across growth. */
typedef struct {
    void* p;
    size_t cap;
} fc_buf;

static void* fc_grow(fc_buf* b, size_t bytes) {
    if (bytes == 0) bytes = 64;
    if (bytes > b->cap) {
        free(b->p);
        size_t cap = (bytes + 63) & ~(size_t)63;
        b->p = aligned_alloc(64, cap);
        if (!b->p) abort();
        b->cap = cap;
    }
    return b->p;
}

typedef struct {
    const uint8_t *bases, *quals, *ins, *del, *gcp;
    int len;
} fc_read;

typedef struct {
    int* v; /* (read, hap) pairs */
    size_t n, cap;
} fc_pairs;

static void fc_pairs_push(fc_pairs* p, int a, int b) {
    if (p->n == p->cap) {
        p->cap = p->cap ? 2 * p->cap : 64;
        p->v = realloc(p->v, p->cap * 2 * sizeof(int));
        if (!p->v) abort();
    }
    p->v[2 * p->n] = a;
    p->v[2 * p->n + 1] = b;
    p->n++;
}

/* One backward sweep (plan.rs:22-31): depths resume+1..need of sorted haplotype hap, starting from
 * node start, writing (depth, node) in ascending depth. */
typedef struct {
    int hap, resume, need, start;
    int nwrites;
    int *wdepth, *wnode;
} fc_sweep;

/* A sorted haplotype set with its sharing plan (kernel.rs:34-48, plan.rs:41-52). */
typedef struct {
    int n, max_len, ncodes;
    int* order; /* order[k]: caller index of sorted haplotype k */
    const uint8_t** bases;
    int* len;
    uint8_t* codes; /* concatenated per sorted haplotype, at code_off[k] */
    size_t* code_off;
    int* lcp;
    uint8_t* dup;
    uint8_t code_byte[256];
    int* cut_col; /* 0: no cut */
    int* cut_node;
    int nsweeps, nodes;
    fc_sweep* sweeps;
} fc_haps;

static int fc_cmp_bytes(const uint8_t* a, int la, const uint8_t* b, int lb) {
    const int n = la < lb ? la : lb;
    const int c = memcmp(a, b, (size_t)n);
    if (c) return c;
    return (la > lb) - (la < lb);
}

static int fc_cmp_reversed(const uint8_t* a, int la, const uint8_t* b, int lb) {
    const int n = la < lb ? la : lb;
    for (int i = 0; i < n; i++) {
        const uint8_t x = a[la - 1 - i], y = b[lb - 1 - i];
        if (x != y) return x < y ? -1 : 1;
    }
    return (la > lb) - (la < lb);
}

/* Stable insertion sort of idx[0..n) under cmp(ctx, a, b); sets are small. */
static void fc_stable_sort(int* idx, int n, int (*cmp)(const void*, int, int), const void* ctx) {
    for (int i = 1; i < n; i++) {
        const int v = idx[i];
        int j = i - 1;
        while (j >= 0 && cmp(ctx, idx[j], v) > 0) {
            idx[j + 1] = idx[j];
            j--;
        }
        idx[j + 1] = v;
    }
}

typedef struct {
    const uint8_t* const* bases;
    const int* len;
} fc_seqs;

static int fc_cmp_fwd_idx(const void* ctx, int a, int b) {
    const fc_seqs* s = ctx;
    return fc_cmp_bytes(s->bases[a], s->len[a], s->bases[b], s->len[b]);
}

static int fc_cmp_rev_idx(const void* ctx, int a, int b) {
    const fc_seqs* s = ctx;
    return fc_cmp_reversed(s->bases[a], s->len[a], s->bases[b], s->len[b]);
}

static int fc_common_suffix(const uint8_t* a, int la, const uint8_t* b, int lb) {
    int n = 0;
    while (n < la && n < lb && a[la - 1 - n] == b[lb - 1 - n]) n++;
    return n;
}

/* A backward sweep must skip at least this many forward columns to pay for its join (plan.rs:9). */
#define FC_MIN_SAVING 4

typedef struct {
    int sweep, depth, id;
} fc_node_id;

typedef struct {
    fc_node_id* v;
    int n, cap;
} fc_node_ids;

/* NodeNumbering::node_for (plan.rs:268-293): the node of depth `depth` along the suffix at position
 * r of the reversed-bases order, numbered on first request. */
static int fc_node_for(fc_node_ids* ids, const fc_sweep* sweeps, const int* sweep_at, const int* lcs, int r,
                       int depth) {
    if (depth == 0) return 0;
    int p = r, shared = INT32_MAX;
    for (;;) {
        const int s = sweep_at[p];
        if (s >= 0 && sweeps[s].resume < depth && depth <= sweeps[s].need) {
            for (int i = 0; i < ids->n; i++)
                if (ids->v[i].sweep == s && ids->v[i].depth == depth) return ids->v[i].id;
            if (ids->n == ids->cap) {
                ids->cap = ids->cap ? 2 * ids->cap : 16;
                ids->v = realloc(ids->v, (size_t)ids->cap * sizeof(fc_node_id));
                if (!ids->v) abort();
            }
            const int id = ids->n + 1;
            ids->v[ids->n++] = (fc_node_id){s, depth, id};
            return id;
        }
        if (lcs[p] < shared) shared = lcs[p];
        if (p == 0 || shared < depth) abort(); /* the plan never asks for an uncomputed depth */
        p--;
    }
}

/* SuffixPlan::new (plan.rs:62-90) for a sorted set. */
static void fc_plan_suffixes(fc_haps* h) {
    const int n = h->n;
    int* distinct = malloc(sizeof(int) * (size_t)n);
    int nd = 0;
    for (int k = 0; k < n; k++)
        if (!h->dup[k]) distinct[nd++] = k;
    /* SuffixOrder (plan.rs:124-150). */
    int* order = malloc(sizeof(int) * (size_t)(nd ? nd : 1));
    memcpy(order, distinct, sizeof(int) * (size_t)nd);
    fc_seqs seqs = {h->bases, h->len};
    fc_stable_sort(order, nd, fc_cmp_rev_idx, &seqs);
    int* lcs = calloc((size_t)(nd ? nd : 1), sizeof(int));
    for (int r = 1; r < nd; r++)
        lcs[r] = fc_common_suffix(h->bases[order[r - 1]], h->len[order[r - 1]], h->bases[order[r]], h->len[order[r]]);
    int* pos = calloc((size_t)n, sizeof(int));
    for (int r = 0; r < nd; r++) pos[order[r]] = r;
    /* cut_depths (plan.rs:160-184). */
    int* depth = calloc((size_t)n, sizeof(int));
    for (int t = 0; t < nd; t++) {
        const int k = distinct[t];
        int shared_prefix = h->lcp[k];
        if (t + 1 < nd && h->lcp[distinct[t + 1]] > shared_prefix) shared_prefix = h->lcp[distinct[t + 1]];
        const int len = h->len[k];
        if (shared_prefix < len) {
            const int r = pos[k];
            int s = lcs[r];
            if (r + 1 < nd && lcs[r + 1] > s) s = lcs[r + 1];
            const int d = s < len - shared_prefix - 1 ? s : len - shared_prefix - 1;
            if (d >= FC_MIN_SAVING) depth[k] = d;
        }
    }
    /* backward_sweeps (plan.rs:189-216). */
    h->sweeps = calloc((size_t)(nd ? nd : 1), sizeof(fc_sweep));
    h->nsweeps = 0;
    int* sweep_at = malloc(sizeof(int) * (size_t)(nd ? nd : 1));
    int reach = 0;
    for (int r = 0; r < nd; r++) {
        const int k = order[r];
        const int resume = lcs[r] < reach ? lcs[r] : reach;
        sweep_at[r] = -1;
        if (depth[k] > resume) {
            sweep_at[r] = h->nsweeps;
            h->sweeps[h->nsweeps++] = (fc_sweep){k, resume, depth[k], 0, 0, NULL, NULL};
        }
        reach = resume > depth[k] ? resume : depth[k];
    }
    fc_node_ids ids = {NULL, 0, 0};
    int* starts = malloc(sizeof(int) * (size_t)(h->nsweeps ? h->nsweeps : 1));
    for (int s = 0; s < h->nsweeps; s++)
        starts[s] = fc_node_for(&ids, h->sweeps, sweep_at, lcs, pos[h->sweeps[s].hap], h->sweeps[s].resume);
    for (int t = 0; t < nd; t++) {
        const int k = distinct[t];
        if (depth[k] > 0) {
            h->cut_node[k] = fc_node_for(&ids, h->sweeps, sweep_at, lcs, pos[k], depth[k]);
            h->cut_col[k] = h->len[k] - depth[k];
        }
    }
    for (int s = 0; s < h->nsweeps; s++) {
        fc_sweep* sw = &h->sweeps[s];
        sw->start = starts[s];
        for (int i = 0; i < ids.n; i++)
            if (ids.v[i].sweep == s) sw->nwrites++;
        sw->wdepth = malloc(sizeof(int) * (size_t)(sw->nwrites ? sw->nwrites : 1));
        sw->wnode = malloc(sizeof(int) * (size_t)(sw->nwrites ? sw->nwrites : 1));
        int m = 0;
        for (int i = 0; i < ids.n; i++)
            if (ids.v[i].sweep == s) {
                /* insertion in ascending depth */
                int j = m++;
                while (j > 0 && sw->wdepth[j - 1] > ids.v[i].depth) {
                    sw->wdepth[j] = sw->wdepth[j - 1];
                    sw->wnode[j] = sw->wnode[j - 1];
                    j--;
                }
                sw->wdepth[j] = ids.v[i].depth;
                sw->wnode[j] = ids.v[i].id;
            }
    }
    h->nodes = ids.n + 1;
    free(ids.v);
    free(starts);
    free(sweep_at);
    free(depth);
    free(pos);
    free(lcs);
    free(order);
    free(distinct);
}

static const uint8_t FC_STANDARD[5] = {'A', 'C', 'G', 'T', 'N'};

/* SortedHaps::new (kernel.rs:53-81). */
static void fc_haps_build(fc_haps* h, const uint8_t* const* bases, const int* len, const int* caller_index, int n,
                          int share_suffixes) {
    memset(h, 0, sizeof *h);
    h->n = n;
    h->order = malloc(sizeof(int) * (size_t)n);
    for (int k = 0; k < n; k++) h->order[k] = k;
    fc_seqs seqs = {bases, len};
    fc_stable_sort(h->order, n, fc_cmp_fwd_idx, &seqs);
    h->bases = malloc(sizeof(uint8_t*) * (size_t)n);
    h->len = malloc(sizeof(int) * (size_t)n);
    size_t total = 0;
    for (int k = 0; k < n; k++) {
        h->bases[k] = bases[h->order[k]];
        h->len[k] = len[h->order[k]];
        total += (size_t)h->len[k];
        if (h->len[k] > h->max_len) h->max_len = h->len[k];
    }
    if (caller_index)
        for (int k = 0; k < n; k++) h->order[k] = caller_index[h->order[k]];
    /* Prior-table codes: ACGTN, then every other byte in order of first appearance. */
    int code_of[256];
    for (int b = 0; b < 256; b++) code_of[b] = -1;
    h->ncodes = 5;
    for (int c = 0; c < 5; c++) {
        code_of[FC_STANDARD[c]] = c;
        h->code_byte[c] = FC_STANDARD[c];
    }
    for (int k = 0; k < n; k++)
        for (int j = 0; j < h->len[k]; j++) {
            const uint8_t b = h->bases[k][j];
            if (code_of[b] < 0) {
                code_of[b] = h->ncodes;
                h->code_byte[h->ncodes++] = b;
            }
        }
    h->codes = malloc(total ? total : 1);
    h->code_off = malloc(sizeof(size_t) * (size_t)(n + 1));
    size_t off = 0;
    for (int k = 0; k < n; k++) {
        h->code_off[k] = off;
        for (int j = 0; j < h->len[k]; j++) h->codes[off + (size_t)j] = (uint8_t)code_of[h->bases[k][j]];
        off += (size_t)h->len[k];
    }
    h->code_off[n] = off;
    h->lcp = calloc((size_t)n, sizeof(int));
    h->dup = calloc((size_t)n, 1);
    for (int k = 1; k < n; k++) {
        const int m = h->len[k - 1] < h->len[k] ? h->len[k - 1] : h->len[k];
        int c = 0;
        while (c < m && h->bases[k - 1][c] == h->bases[k][c]) c++;
        h->lcp[k] = c;
        h->dup[k] = h->len[k - 1] == h->len[k] && c == h->len[k];
    }
    h->cut_col = calloc((size_t)n, sizeof(int));
    h->cut_node = calloc((size_t)n, sizeof(int));
    h->nodes = 1;
    if (share_suffixes && n > 0) fc_plan_suffixes(h);
}

static void fc_haps_free(fc_haps* h) {
    for (int s = 0; s < h->nsweeps; s++) {
        free(h->sweeps[s].wdepth);
        free(h->sweeps[s].wnode);
    }
    free(h->sweeps);
    free(h->order);
    free(h->bases);
    free(h->len);
    free(h->codes);
    free(h->code_off);
    free(h->lcp);
    free(h->dup);
    free(h->cut_col);
    free(h->cut_node);
}

/* ---- PD-HMM haplotype sets (pd_kernel.rs:41-136, 186-214, 699-746) ------------------------------ */

enum { FC_PD_SNP = 1, FC_PD_DEL_START = 2, FC_PD_DEL_END = 4, FC_PD_ALTS = 8 | 16 | 32 | 64 };
enum { FC_PD_NORMAL = 0, FC_PD_INSIDE_DEL = 1, FC_PD_AFTER_DEL = 2 };

int or_base_matches_pd(uint8_t read_base, uint8_t flags); /* pairhmm_oracle.c, pd.rs:99-110 */

/* The read bases a column accepts as a match: its base and, on a SNP column, the flagged alternates. */
typedef struct {
    uint8_t base, alts;
} fc_mset;

static fc_mset fc_mset_of(uint8_t base, uint8_t flag) {
    fc_mset m = {base, (uint8_t)((flag & FC_PD_SNP) ? (flag & FC_PD_ALTS) : 0)};
    return m;
}

static int fc_mset_accepts(fc_mset m, uint8_t rb) {
    return rb == m.base || rb == 'N' || m.base == 'N' || (m.alts && or_base_matches_pd(rb, (uint8_t)(FC_PD_SNP | m.alts)));
}

/* Columns lo+1..hi in one deletion state, all with or all without DEL_END. */
typedef struct {
    int lo, hi;
    uint8_t state, del_end;
} fc_seg;

/* A run after cutting at the snapshot columns; at_snap: it ends at one. */
typedef struct {
    int lo, hi;
    uint8_t state, del_end, at_snap;
} fc_run;

/* segments (pd_kernel.rs:723-746): a row's runs starting in `state`; returns the run count and sets
 * *end to the state carried out of the last column. `out` holds len entries at most. */
static int fc_pd_segments(const uint8_t* flags, int len, int state, fc_seg* out, int* end) {
    int n = 0;
    for (int j = 0; j < len; j++) {
        const int col = j + 1, del_end = (flags[j] & FC_PD_DEL_END) != 0;
        if (n > 0 && out[n - 1].state == state && out[n - 1].del_end == del_end)
            out[n - 1].hi = col;
        else
            out[n++] = (fc_seg){j, col, (uint8_t)state, (uint8_t)del_end};
        if (state == FC_PD_AFTER_DEL) state = FC_PD_NORMAL;
        if (flags[j] & FC_PD_DEL_START) state = FC_PD_INSIDE_DEL;
        if (del_end) state = FC_PD_AFTER_DEL;
    }
    *end = state;
    return n;
}

/* The deletion state carried out of a row that starts in NORMAL. */
static int fc_pd_end_state(const uint8_t* flags, int len) {
    int state = FC_PD_NORMAL;
    for (int j = 0; j < len; j++) {
        if (state == FC_PD_AFTER_DEL) state = FC_PD_NORMAL;
        if (flags[j] & FC_PD_DEL_START) state = FC_PD_INSIDE_DEL;
        if (flags[j] & FC_PD_DEL_END) state = FC_PD_AFTER_DEL;
    }
    return state;
}

/* cut_runs (pd_kernel.rs:699-721): runs clipped to the columns after `start`, cut at snapshots. */
static int fc_cut_runs(const fc_seg* segs, int nseg, int start, const int* snap, int nsnap, fc_run* out) {
    int n = 0, next = 0;
    for (int i = 0; i < nseg; i++) {
        int lo = segs[i].lo > start ? segs[i].lo : start;
        if (lo >= segs[i].hi) continue;
        while (next < nsnap && snap[next] <= lo) next++;
        while (next < nsnap && snap[next] < segs[i].hi) {
            out[n++] = (fc_run){lo, snap[next], segs[i].state, segs[i].del_end, 1};
            lo = snap[next++];
        }
        const int at = next < nsnap && snap[next] == segs[i].hi;
        out[n++] = (fc_run){lo, segs[i].hi, segs[i].state, segs[i].del_end, (uint8_t)at};
    }
    return n;
}

/* SortedPdHaps (pd_kernel.rs:61-136): sorted by (row-end state, interleaved bases and flags). */
typedef struct {
    int n, max_len, nsets;
    int* order;
    const uint8_t** bases;
    const uint8_t** flags;
    int* len;
    uint8_t* codes; /* match-set code per column, at code_off[k] */
    size_t* code_off;
    int** del_end_cols; /* 1-based columns carrying DEL_END */
    int* n_del_end;
    fc_seg** first_row;
    int* n_first;
    fc_seg** later_rows;
    int* n_later;
    int* lcp;
    int* end_state;
    fc_mset sets[256];
} fc_pdhaps;

typedef struct {
    const uint8_t* const* bases;
    const uint8_t* const* flags;
    const int* len;
    const int* end;
} fc_pdkey;

static int fc_cmp_pd_idx(const void* ctx, int a, int b) {
    const fc_pdkey* k = ctx;
    if (k->end[a] != k->end[b]) return k->end[a] < k->end[b] ? -1 : 1;
    const int n = k->len[a] < k->len[b] ? k->len[a] : k->len[b];
    for (int j = 0; j < n; j++) {
        if (k->bases[a][j] != k->bases[b][j]) return k->bases[a][j] < k->bases[b][j] ? -1 : 1;
        if (k->flags[a][j] != k->flags[b][j]) return k->flags[a][j] < k->flags[b][j] ? -1 : 1;
    }
    return (k->len[a] > k->len[b]) - (k->len[a] < k->len[b]);
}

/* Returns 0, or -1 when the set holds more than 256 distinct match sets. */
static int fc_pdhaps_build(fc_pdhaps* h, const uint8_t* const* bases, const uint8_t* const* flags, const int* len, int n) {
    memset(h, 0, sizeof *h);
    h->n = n;
    /* The state carried out of a row, which every later row starts in, sorts the haplotypes. */
    int* end = malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int i = 0; i < n; i++) end[i] = fc_pd_end_state(flags[i], len[i]);
    h->order = malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int i = 0; i < n; i++) h->order[i] = i;
    fc_pdkey key = {bases, flags, len, end};
    fc_stable_sort(h->order, n, fc_cmp_pd_idx, &key);
    h->bases = malloc(sizeof(uint8_t*) * (size_t)(n ? n : 1));
    h->flags = malloc(sizeof(uint8_t*) * (size_t)(n ? n : 1));
    h->len = malloc(sizeof(int) * (size_t)(n ? n : 1));
    h->end_state = malloc(sizeof(int) * (size_t)(n ? n : 1));
    h->code_off = malloc(sizeof(size_t) * (size_t)(n + 1));
    h->del_end_cols = calloc((size_t)(n ? n : 1), sizeof(int*));
    h->n_del_end = calloc((size_t)(n ? n : 1), sizeof(int));
    h->first_row = calloc((size_t)(n ? n : 1), sizeof(fc_seg*));
    h->n_first = calloc((size_t)(n ? n : 1), sizeof(int));
    h->later_rows = calloc((size_t)(n ? n : 1), sizeof(fc_seg*));
    h->n_later = calloc((size_t)(n ? n : 1), sizeof(int));
    h->lcp = calloc((size_t)(n ? n : 1), sizeof(int));
    size_t total = 0;
    for (int k = 0; k < n; k++) total += (size_t)len[h->order[k]];
    h->codes = malloc(total ? total : 1);
    int rc = 0;
    size_t off = 0;
    for (int k = 0; k < n; k++) {
        const int i = h->order[k];
        h->bases[k] = bases[i];
        h->flags[k] = flags[i];
        h->len[k] = len[i];
        h->end_state[k] = end[i];
        if (len[i] > h->max_len) h->max_len = len[i];
        h->code_off[k] = off;
        for (int j = 0; j < len[i]; j++) {
            const fc_mset m = fc_mset_of(bases[i][j], flags[i][j]);
            int c = 0;
            while (c < h->nsets && (h->sets[c].base != m.base || h->sets[c].alts != m.alts)) c++;
            if (c == h->nsets) {
                if (h->nsets == 256) {
                    rc = -1;
                    c = 0;
                } else {
                    h->sets[h->nsets++] = m;
                }
            }
            h->codes[off + (size_t)j] = (uint8_t)c;
        }
        off += (size_t)len[i];
        int nd = 0;
        for (int j = 0; j < len[i]; j++) nd += (flags[i][j] & FC_PD_DEL_END) != 0;
        h->del_end_cols[k] = malloc(sizeof(int) * (size_t)(nd ? nd : 1));
        for (int j = 0, d = 0; j < len[i]; j++)
            if (flags[i][j] & FC_PD_DEL_END) h->del_end_cols[k][d++] = j + 1;
        h->n_del_end[k] = nd;
        int e1, e2;
        const size_t nseg = len[i] > 0 ? (size_t)len[i] : 1;
        h->first_row[k] = malloc(sizeof(fc_seg) * nseg);
        h->n_first[k] = fc_pd_segments(flags[i], len[i], FC_PD_NORMAL, h->first_row[k], &e1);
        h->later_rows[k] = malloc(sizeof(fc_seg) * nseg);
        h->n_later[k] = fc_pd_segments(flags[i], len[i], e1, h->later_rows[k], &e2);
    }
    h->code_off[n] = off;
    for (int k = 1; k < n; k++) {
        if (h->end_state[k - 1] != h->end_state[k]) continue;
        const int m = h->len[k - 1] < h->len[k] ? h->len[k - 1] : h->len[k];
        int c = 0;
        while (c < m && h->bases[k - 1][c] == h->bases[k][c] && h->flags[k - 1][c] == h->flags[k][c]) c++;
        h->lcp[k] = c;
    }
    free(end);
    return rc;
}

static void fc_pdhaps_free(fc_pdhaps* h) {
    for (int k = 0; k < h->n; k++) {
        free(h->del_end_cols[k]);
        free(h->first_row[k]);
        free(h->later_rows[k]);
    }
    free(h->order);
    free(h->bases);
    free(h->flags);
    free(h->len);
    free(h->end_state);
    free(h->codes);
    free(h->code_off);
    free(h->del_end_cols);
    free(h->n_del_end);
    free(h->first_row);
    free(h->n_first);
    free(h->later_rows);
    free(h->n_later);
    free(h->lcp);
}

/* ---- kernel instantiations ------------------------------------------------------------------ */

typedef float fc_f32x16 __attribute__((vector_size(64)));
typedef float fc_f32x8 __attribute__((vector_size(32)));
typedef double fc_f64x8 __attribute__((vector_size(64)));
typedef double fc_f64x4 __attribute__((vector_size(32)));
typedef int32_t fc_i32x16 __attribute__((vector_size(64)));
typedef int32_t fc_i32x8 __attribute__((vector_size(32)));
typedef int64_t fc_i64x8 __attribute__((vector_size(64)));
typedef int64_t fc_i64x4 __attribute__((vector_size(32)));

#define FC_E float
#define FC_L 16
#define FC_V fc_f32x16
#define FC_NAME(x) fc_##x##_f32x16
#define FC_TARGET __attribute__((target("avx512f,avx2,fma")))
#define FC_F32 1
#define FC_VI fc_i32x16
#include "fgkl_cpu_kernel.h"
#include "fgkl_cpu_pd_kernel.h"
#undef FC_E
#undef FC_L
#undef FC_V
#undef FC_NAME
#undef FC_TARGET
#undef FC_F32
#undef FC_VI

#define FC_E float
#define FC_L 8
#define FC_V fc_f32x8
#define FC_NAME(x) fc_##x##_f32x8
#define FC_TARGET __attribute__((target("avx2,fma")))
#define FC_F32 1
#define FC_VI fc_i32x8
#include "fgkl_cpu_kernel.h"
#include "fgkl_cpu_pd_kernel.h"
#undef FC_E
#undef FC_L
#undef FC_V
#undef FC_NAME
#undef FC_TARGET
#undef FC_F32
#undef FC_VI

#define FC_E float
#define FC_L 8
#define FC_V fc_f32x8
#define FC_NAME(x) fc_##x##_f32x8p
#define FC_TARGET
#define FC_F32 1
#define FC_VI fc_i32x8
#include "fgkl_cpu_kernel.h"
#include "fgkl_cpu_pd_kernel.h"
#undef FC_E
#undef FC_L
#undef FC_V
#undef FC_NAME
#undef FC_TARGET
#undef FC_F32
#undef FC_VI

#define FC_E double
#define FC_L 8
#define FC_V fc_f64x8
#define FC_NAME(x) fc_##x##_f64x8
#define FC_TARGET __attribute__((target("avx512f,avx2,fma")))
#define FC_F32 0
#define FC_VI fc_i64x8
#include "fgkl_cpu_kernel.h"
#include "fgkl_cpu_pd_kernel.h"
#undef FC_E
#undef FC_L
#undef FC_V
#undef FC_NAME
#undef FC_TARGET
#undef FC_F32
#undef FC_VI

#define FC_E double
#define FC_L 4
#define FC_V fc_f64x4
#define FC_NAME(x) fc_##x##_f64x4
#define FC_TARGET __attribute__((target("avx2,fma")))
#define FC_F32 0
#define FC_VI fc_i64x4
#include "fgkl_cpu_kernel.h"
#include "fgkl_cpu_pd_kernel.h"
#undef FC_E
#undef FC_L
#undef FC_V
#undef FC_NAME
#undef FC_TARGET
#undef FC_F32
#undef FC_VI

#define FC_E double
#define FC_L 4
#define FC_V fc_f64x4
#define FC_NAME(x) fc_##x##_f64x4p
#define FC_TARGET
#define FC_F32 0
#define FC_VI fc_i64x4
#include "fgkl_cpu_kernel.h"
#include "fgkl_cpu_pd_kernel.h"
#undef FC_E
#undef FC_L
#undef FC_V
#undef FC_NAME
#undef FC_TARGET
#undef FC_F32
#undef FC_VI

typedef struct {
    int lanes;
    void* (*ws_new)(void);
    void (*ws_free)(void*);
    void (*run)(void* ws, const fc_read* reads, int n, const void* hs, double* out, fc_pairs* fallback);
} fc_runner;

/* 0-5 the plain kernel, 6-11 the PD kernel: f32x16, f32x8, f32x8 portable, f64x8, f64x4, f64x4 portable. */
#define FC_NRUNNERS 12
static const fc_runner FC_RUNNERS[FC_NRUNNERS] = {
    {16, fc_ws_new_f32x16, fc_ws_free_f32x16, fc_run_batch_f32x16},
    {8, fc_ws_new_f32x8, fc_ws_free_f32x8, fc_run_batch_f32x8},
    {8, fc_ws_new_f32x8p, fc_ws_free_f32x8p, fc_run_batch_f32x8p},
    {8, fc_ws_new_f64x8, fc_ws_free_f64x8, fc_run_batch_f64x8},
    {4, fc_ws_new_f64x4, fc_ws_free_f64x4, fc_run_batch_f64x4},
    {4, fc_ws_new_f64x4p, fc_ws_free_f64x4p, fc_run_batch_f64x4p},
    {16, fc_pdws_new_f32x16, fc_pdws_free_f32x16, fc_pd_run_batch_f32x16},
    {8, fc_pdws_new_f32x8, fc_pdws_free_f32x8, fc_pd_run_batch_f32x8},
    {8, fc_pdws_new_f32x8p, fc_pdws_free_f32x8p, fc_pd_run_batch_f32x8p},
    {8, fc_pdws_new_f64x8, fc_pdws_free_f64x8, fc_pd_run_batch_f64x8},
    {4, fc_pdws_new_f64x4, fc_pdws_free_f64x4, fc_pd_run_batch_f64x4},
    {4, fc_pdws_new_f64x4p, fc_pdws_free_f64x4p, fc_pd_run_batch_f64x4p},
};

/* Instruction set: 2 = AVX-512F (+AVX2 narrow), 1 = AVX2, 0 = portable vectors. */
int fc_detect_isa(void) {
    __builtin_cpu_init();
    const int avx2 = __builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma");
    if (avx2 && __builtin_cpu_supports("avx512f")) return 2;
    return avx2 ? 1 : 0;
}

/* The wide and narrow runner of a precision (kernel.rs:165-191, lib.rs:399-413). */
static int fc_wide(int isa, int dbl) {
    if (isa == 2) return dbl ? 3 : 0;
    if (isa == 1) return dbl ? 4 : 1;
    return dbl ? 5 : 2;
}
static int fc_narrow(int isa, int dbl) {
    if (isa == 2) return dbl ? 4 : 1;
    return fc_wide(isa, dbl);
}

/* Per-thread state: one workspace per runner. */
typedef struct {
    int isa;
    void* ws[FC_NRUNNERS];
} fc_thread;

static void* fc_ws(fc_thread* t, int runner) {
    if (!t->ws[runner]) t->ws[runner] = FC_RUNNERS[runner].ws_new();
    return t->ws[runner];
}

/* ---- the batching driver (lib.rs:346-550) -------------------------------------------------- */

typedef struct {
    fc_thread* t;
    int share_suffixes, double_fallback;
    int pd; /* the haplotype sets are fc_pdhaps (PD-HMM), else fc_haps */
    int64_t fallback_pairs;
} fc_batcher;

static int fc_set_n(const fc_batcher* b, const void* hs) {
    return b->pd ? ((const fc_pdhaps*)hs)->n : ((const fc_haps*)hs)->n;
}

/* A set of sorted haplotype h alone (HapSet::single, kernel.rs:119-122, pd_kernel.rs:152-154). */
typedef union {
    fc_haps plain;
    fc_pdhaps pd;
} fc_any_haps;

static void fc_set_single(const fc_batcher* b, const void* hs, int h, fc_any_haps* out) {
    if (b->pd) {
        const fc_pdhaps* p = hs;
        fc_pdhaps_build(&out->pd, &p->bases[h], &p->flags[h], &p->len[h], 1);
    } else {
        const fc_haps* p = hs;
        fc_haps_build(&out->plain, &p->bases[h], &p->len[h], NULL, 1, 0);
    }
}

static void fc_set_free(const fc_batcher* b, fc_any_haps* s) {
    if (b->pd)
        fc_pdhaps_free(&s->pd);
    else
        fc_haps_free(&s->plain);
}

/* Runs reads in batches of the runner's lanes; lost pairs offset by first_read (lib.rs:439-461). */
static void fc_run_batches(fc_batcher* b, int runner, const fc_read* reads, int n, const void* hs, double* tmp,
                           int first_read, fc_pairs* fallback) {
    if (n == 0) return;
    const int lanes = FC_RUNNERS[runner].lanes, nh = fc_set_n(b, hs);
    fc_pairs batch = {NULL, 0, 0};
    for (int lo = 0; lo < n; lo += lanes) {
        const int hi = lo + lanes < n ? lo + lanes : n;
        batch.n = 0;
        FC_RUNNERS[runner].run(fc_ws(b->t, runner), reads + lo, hi - lo, hs, tmp + (size_t)lo * nh, &batch);
        for (size_t i = 0; i < batch.n; i++)
            fc_pairs_push(fallback, first_read + lo + batch.v[2 * i], batch.v[2 * i + 1]);
    }
    free(batch.v);
}

/* Batcher::run_pass (lib.rs:417-435): full batches on the wide runner, a remainder that fits the
 * narrow runner on it. */
static void fc_run_pass(fc_batcher* b, int dbl, const fc_read* reads, int n, const void* hs, double* tmp,
                        fc_pairs* fallback) {
    const int base = b->pd ? 6 : 0;
    const int wide = base + fc_wide(b->t->isa, dbl), narrow = base + fc_narrow(b->t->isa, dbl);
    const int rest = n % FC_RUNNERS[wide].lanes;
    const int split = (narrow != wide && rest <= FC_RUNNERS[narrow].lanes) ? n - rest : n;
    fc_run_batches(b, wide, reads, split, hs, tmp, 0, fallback);
    fc_run_batches(b, narrow, reads + split, n - split, hs, tmp + (size_t)split * fc_set_n(b, hs), split, fallback);
}

/* Batcher::recompute_in_double (lib.rs:493-549). Returns the pairs still lost in `lost`. */
static void fc_recompute_in_double(fc_batcher* b, const int* pairs, size_t npairs, const fc_read* reads, int nreads,
                                   const void* hs, double* tmp, fc_pairs* lost) {
    const int nh = fc_set_n(b, hs);
    int* per_read = calloc((size_t)nreads, sizeof(int));
    for (size_t i = 0; i < npairs; i++) per_read[pairs[2 * i]]++;
    /* Reads lost against a third or more of the haplotypes rerun against all of them, shared. */
    int* dense = malloc(sizeof(int) * (size_t)(nreads ? nreads : 1));
    int nd = 0;
    for (int r = 0; r < nreads; r++)
        if (per_read[r] > 0 && per_read[r] * 3 >= nh) dense[nd++] = r;
    if (nd > 0) {
        fc_read* batch = malloc(sizeof(fc_read) * (size_t)nd);
        for (int i = 0; i < nd; i++) batch[i] = reads[dense[i]];
        double* out = malloc(sizeof(double) * (size_t)nd * nh);
        fc_pairs dl = {NULL, 0, 0};
        fc_run_pass(b, 1, batch, nd, hs, out, &dl);
        for (size_t i = 0; i < dl.n; i++) fc_pairs_push(lost, dense[dl.v[2 * i]], dl.v[2 * i + 1]);
        int* slot = malloc(sizeof(int) * (size_t)nreads);
        for (int r = 0; r < nreads; r++) slot[r] = -1;
        for (int i = 0; i < nd; i++) slot[dense[i]] = i;
        for (size_t i = 0; i < npairs; i++) {
            const int r = pairs[2 * i], h = pairs[2 * i + 1];
            if (slot[r] >= 0) tmp[(size_t)r * nh + h] = out[(size_t)slot[r] * nh + h];
        }
        free(slot);
        free(dl.v);
        free(out);
        free(batch);
    }
    /* The other pairs, grouped by haplotype, one unshared haplotype at a time, reads in ascending
     * position (the BTreeMap orders of lib.rs:516-522). */
    const int wide = (b->pd ? 6 : 0) + fc_wide(b->t->isa, 1), narrow = (b->pd ? 6 : 0) + fc_narrow(b->t->isa, 1);
    const int lanes = FC_RUNNERS[wide].lanes;
    uint8_t* is_dense = calloc((size_t)(nreads ? nreads : 1), 1);
    for (int i = 0; i < nd; i++) is_dense[dense[i]] = 1;
    uint8_t* want = calloc((size_t)nreads * (nh ? nh : 1), 1);
    for (size_t i = 0; i < npairs; i++)
        if (!is_dense[pairs[2 * i]]) want[(size_t)pairs[2 * i] * nh + pairs[2 * i + 1]] = 1;
    int* chunk = malloc(sizeof(int) * (size_t)lanes);
    fc_read* batch = malloc(sizeof(fc_read) * (size_t)lanes);
    double out[16];
    fc_pairs none = {NULL, 0, 0};
    for (int h = 0; h < nh; h++) {
        fc_any_haps single;
        int built = 0;
        int m = 0;
        for (int r = 0; r <= nreads; r++) {
            const int take = r < nreads && want[(size_t)r * nh + h];
            if (take) chunk[m++] = r;
            if (m == lanes || (r == nreads && m > 0)) {
                if (!built) {
                    fc_set_single(b, hs, h, &single);
                    built = 1;
                }
                const int runner = (narrow != wide && m <= FC_RUNNERS[narrow].lanes) ? narrow : wide;
                for (int i = 0; i < m; i++) batch[i] = reads[chunk[i]];
                FC_RUNNERS[runner].run(fc_ws(b->t, runner), batch, m, &single, out, &none);
                for (int i = 0; i < m; i++) tmp[(size_t)chunk[i] * nh + h] = out[i];
                m = 0;
            }
        }
        if (built) fc_set_free(b, &single);
    }
    free(none.v);
    free(batch);
    free(chunk);
    free(want);
    free(is_dense);
    free(dense);
    free(per_read);
}

/* Batcher::compute (lib.rs:377-397) for one region: out[read * n_haps + hap] in caller order. A PD
 * region (hf, the haplotypes' flags, not NULL) runs the PD kernel, which shares prefixes only, so
 * its FP64 pass loses no pair (pd_kernel.rs:156-166). Returns -1 when a PD region holds more than
 * 256 distinct match sets, else 0. */
static int fc_compute_region(fc_batcher* b, int dbl, const fc_read* reads_in, int nreads, const uint8_t* const* hb,
                             const uint8_t* const* hf, const int* hl, int nh, double* out) {
    if (nreads == 0 || nh == 0) return 0;
    fc_any_haps set;
    const int* order;
    if (b->pd) {
        if (fc_pdhaps_build(&set.pd, hb, hf, hl, nh) != 0) {
            fc_pdhaps_free(&set.pd);
            return -1;
        }
        order = set.pd.order;
    } else {
        fc_haps_build(&set.plain, hb, hl, NULL, nh, b->share_suffixes);
        order = set.plain.order;
    }
    const void* hs = &set;
    /* Longest reads first, stable. */
    int* read_order = malloc(sizeof(int) * (size_t)nreads);
    for (int r = 0; r < nreads; r++) read_order[r] = r;
    for (int i = 1; i < nreads; i++) {
        const int v = read_order[i];
        int j = i - 1;
        while (j >= 0 && reads_in[read_order[j]].len < reads_in[v].len) {
            read_order[j + 1] = read_order[j];
            j--;
        }
        read_order[j + 1] = v;
    }
    fc_read* reads = malloc(sizeof(fc_read) * (size_t)nreads);
    for (int r = 0; r < nreads; r++) reads[r] = reads_in[read_order[r]];
    double* tmp = malloc(sizeof(double) * (size_t)nreads * nh);
    fc_pairs fallback = {NULL, 0, 0};
    fc_run_pass(b, dbl, reads, nreads, hs, tmp, &fallback);
    if (fallback.n > 0) {
        b->fallback_pairs += (int64_t)fallback.n;
        if (b->double_fallback) {
            /* Batcher::run_fallback (lib.rs:467-490). */
            fc_pairs lost = {NULL, 0, 0};
            if (!dbl) {
                fc_recompute_in_double(b, fallback.v, fallback.n, reads, nreads, hs, tmp, &lost);
            } else {
                for (size_t i = 0; i < fallback.n; i++) fc_pairs_push(&lost, fallback.v[2 * i], fallback.v[2 * i + 1]);
            }
            if (lost.n > 0 && !b->pd) {
                fc_haps unshared;
                fc_haps_build(&unshared, set.plain.bases, set.plain.len, NULL, nh, 0);
                fc_pairs none = {NULL, 0, 0};
                fc_recompute_in_double(b, lost.v, lost.n, reads, nreads, &unshared, tmp, &none);
                free(none.v);
                fc_haps_free(&unshared);
            }
            free(lost.v);
        }
    }
    for (int pos = 0; pos < nreads; pos++)
        for (int k = 0; k < nh; k++) out[(size_t)read_order[pos] * nh + order[k]] = tmp[(size_t)pos * nh + k];
    free(fallback.v);
    free(tmp);
    free(reads);
    free(read_order);
    fc_set_free(b, &set);
    return 0;
}

/* ---- the exported driver --------------------------------------------------------------------- */

typedef struct {
    const uint8_t *bases, *quals, *ins, *del, *gcp, *hap_bases, *hap_flags;
    const int64_t *read_offsets, *hap_offsets;
    const int64_t *read_first, *hap_first, *out_first;
    const int32_t *n_reads, *n_haps;
    int n_regions, dbl, share_suffixes, double_fallback, isa;
    double* out;
    int next;
    int64_t fallback_pairs;
    int failed; /* a PD region with more than 256 distinct match sets */
    pthread_mutex_t lock;
} fc_job;

static void* fc_worker(void* arg) {
    fc_job* job = arg;
    fc_thread t;
    memset(&t, 0, sizeof t);
    t.isa = job->isa;
    fc_batcher b = {&t, job->share_suffixes, job->double_fallback, job->hap_flags != NULL, 0};
    fc_read* reads = NULL;
    const uint8_t** hb = NULL;
    const uint8_t** hf = NULL;
    int* hl = NULL;
    int cap_r = 0, cap_h = 0;
    for (;;) {
        pthread_mutex_lock(&job->lock);
        const int g = job->next++;
        pthread_mutex_unlock(&job->lock);
        if (g >= job->n_regions) break;
        const int nr = job->n_reads[g], nh = job->n_haps[g];
        if (nr > cap_r) {
            cap_r = nr;
            reads = realloc(reads, sizeof(fc_read) * (size_t)cap_r);
        }
        if (nh > cap_h) {
            cap_h = nh;
            hb = realloc(hb, sizeof(uint8_t*) * (size_t)cap_h);
            hf = realloc(hf, sizeof(uint8_t*) * (size_t)cap_h);
            hl = realloc(hl, sizeof(int) * (size_t)cap_h);
        }
        for (int r = 0; r < nr; r++) {
            const int64_t i = job->read_first[g] + r;
            const int64_t lo = job->read_offsets[i];
            reads[r] = (fc_read){job->bases + lo, job->quals + lo, job->ins + lo, job->del + lo, job->gcp + lo,
                                 (int)(job->read_offsets[i + 1] - lo)};
        }
        for (int h = 0; h < nh; h++) {
            const int64_t i = job->hap_first[g] + h;
            hb[h] = job->hap_bases + job->hap_offsets[i];
            hf[h] = job->hap_flags ? job->hap_flags + job->hap_offsets[i] : NULL;
            hl[h] = (int)(job->hap_offsets[i + 1] - job->hap_offsets[i]);
        }
        if (fc_compute_region(&b, job->dbl, reads, nr, hb, hf, hl, nh, job->out + job->out_first[g]) != 0) {
            pthread_mutex_lock(&job->lock);
            job->failed = 1;
            pthread_mutex_unlock(&job->lock);
        }
    }
    for (int r = 0; r < FC_NRUNNERS; r++)
        if (t.ws[r]) FC_RUNNERS[r].ws_free(t.ws[r]);
    free(reads);
    free(hb);
    free(hf);
    free(hl);
    pthread_mutex_lock(&job->lock);
    job->fallback_pairs += b.fallback_pairs;
    pthread_mutex_unlock(&job->lock);
    return NULL;
}

/* Computes n_regions regions on `threads` threads; with hap_flags (per haplotype base, as the
 * bases) the PD-HMM, else the plain PairHMM. Region g holds reads read_first[g] ..
 * read_first[g] + n_reads[g] - 1 (delimited by read_offsets) and haplotypes hap_first[g] .. (by
 * hap_offsets); its n_reads x n_haps results land at out + out_first[g], read-major, in log10.
 * precision: 0 single (GKL's default), 1 double. isa: -1 detect, else 0/1/2 as fc_detect_isa
 * (capped at what the CPU has). Returns the pairs that lost precision in the first pass, -1 on
 * a bad argument, or -2 when a PD region holds more than 256 distinct match sets. */
int64_t fc_compute_regions_flags(const uint8_t* bases, const uint8_t* quals, const uint8_t* ins, const uint8_t* del,
                                 const uint8_t* gcp, const int64_t* read_offsets, const uint8_t* hap_bases,
                                 const uint8_t* hap_flags, const int64_t* hap_offsets, const int64_t* read_first,
                                 const int32_t* n_reads, const int64_t* hap_first, const int32_t* n_haps,
                                 const int64_t* out_first, int n_regions, int precision, int share_suffixes,
                                 int double_fallback, int threads, int isa, double* out) {
    if (n_regions < 0 || threads < 0) return -1;
    const int have = fc_detect_isa();
    if (isa < 0 || isa > have) isa = have;
    fc_job job;
    memset(&job, 0, sizeof job);
    job.bases = bases;
    job.quals = quals;
    job.ins = ins;
    job.del = del;
    job.gcp = gcp;
    job.hap_bases = hap_bases;
    job.hap_flags = hap_flags;
    job.read_offsets = read_offsets;
    job.hap_offsets = hap_offsets;
    job.read_first = read_first;
    job.hap_first = hap_first;
    job.out_first = out_first;
    job.n_reads = n_reads;
    job.n_haps = n_haps;
    job.n_regions = n_regions;
    job.dbl = precision != 0;
    job.share_suffixes = share_suffixes;
    job.double_fallback = double_fallback;
    job.isa = isa;
    job.out = out;
    pthread_mutex_init(&job.lock, NULL);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tids[256];
    for (int t = 1; t < threads; t++) pthread_create(&tids[t], NULL, fc_worker, &job);
    fc_worker(&job);
    for (int t = 1; t < threads; t++) pthread_join(tids[t], NULL);
    pthread_mutex_destroy(&job.lock);
    return job.failed ? -2 : job.fallback_pairs;
}

/* The plain PairHMM (no flags). */
int64_t fc_compute_regions(const uint8_t* bases, const uint8_t* quals, const uint8_t* ins, const uint8_t* del,
                           const uint8_t* gcp, const int64_t* read_offsets, const uint8_t* hap_bases,
                           const int64_t* hap_offsets, const int64_t* read_first, const int32_t* n_reads,
                           const int64_t* hap_first, const int32_t* n_haps, const int64_t* out_first, int n_regions,
                           int precision, int share_suffixes, int double_fallback, int threads, int isa, double* out) {
    return fc_compute_regions_flags(bases, quals, ins, del, gcp, read_offsets, hap_bases, NULL, hap_offsets, read_first,
                                    n_reads, hap_first, n_haps, out_first, n_regions, precision, share_suffixes,
                                    double_fallback, threads, isa, out);
}
