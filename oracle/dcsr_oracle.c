/*
 * dcsr_oracle.c -- CPU restatement of the DCSR operators (TEST INFRASTRUCTURE).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg use
 * this file; it is the checker, never the product.  See dcsr_oracle.h for the
 * layout and the pinning story.  Build: oracle/Makefile (-ffp-contract=off so
 * every add and multiply rounds exactly like the device code).
 */
#include "dcsr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- helpers */

static int64_t align_up64(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

/* Value arithmetic in the matrix type: F32 rounds every result to float. */
static double vadd(int32_t dt, double a, double b) {
  if (dt == OR_F32) return (double)((float)a + (float)b);
  return a + b;
}
static double vmul(int32_t dt, double a, double b) {
  if (dt == OR_F32) return (double)((float)a * (float)b);
  return a * b;
}
static double vround(int32_t dt, double a) { return dt == OR_F32 ? (double)(float)a : a; }

void or_default_opts(or_opts *o, int mode) {
  o->max_segs = 4;
  o->mode = mode;
  o->alpha = 4;
  o->spare_x16 = 16;
  o->min_spare = 4096;
  o->reloc_min = 2048;
  if (mode == OR_APPEND) { /* reference-tight load/compaction (load.h:207-227, :574-580) */
    o->factor_x16 = 16;
    o->min_cap = 0;
    o->align = 1;
  } else {                 /* canonical: 2x per-row slack, 16-byte aligned segments */
    o->factor_x16 = 32;
    o->min_cap = 4;
    o->align = 4;
  }
}

int64_t or_policy_cap(const or_opts *o, int64_t len) {
  int64_t c = (len * o->factor_x16 + 15) / 16;
  if (c < o->min_cap) c = o->min_cap;
  if (c < len) c = len;
  return align_up64(c, o->align);
}

int64_t or_pool_capacity(const or_opts *o, int64_t top) {
  int64_t spare = top * o->spare_x16 / 16;
  if (spare < o->min_spare) spare = o->min_spare;
  return top + spare;
}

static int64_t seg_index(const or_dcsr *m, int l, int32_t r) { return (int64_t)l * m->pitch + 2 * (int64_t)r; }

or_dcsr *or_create(int32_t n_rows, int32_t n_cols, int32_t dtype, const or_opts *o) {
  if (n_rows < 0 || n_cols < 0 || o->max_segs < 1 || o->max_segs > 4) return NULL;
  or_dcsr *m = (or_dcsr *)calloc(1, sizeof(or_dcsr));
  m->n_rows = n_rows;
  m->n_cols = n_cols;
  m->dtype = dtype;
  m->o = *o;
  m->pitch = (int32_t)align_up64(2 * (int64_t)n_rows, 32);
  m->row_sizes = (int32_t *)calloc((size_t)n_rows + 1, sizeof(int32_t));
  size_t ns = (size_t)m->pitch * o->max_segs;
  m->seg = (int32_t *)malloc((ns ? ns : 1) * sizeof(int32_t));
  for (size_t i = 0; i < ns; i++) m->seg[i] = -1;
  m->pool_cap = 0;
  m->cols = NULL;
  m->vals = NULL;
  return m;
}

void or_destroy(or_dcsr *m) {
  if (!m) return;
  free(m->row_sizes);
  free(m->seg);
  free(m->cols);
  free(m->vals);
  free(m);
}

static void set_pool(or_dcsr *m, int64_t cap) {
  m->pool_cap = cap;
  m->cols = (int32_t *)realloc(m->cols, (size_t)(cap ? cap : 1) * sizeof(int32_t));
  m->vals = (double *)realloc(m->vals, (size_t)(cap ? cap : 1) * sizeof(double));
}

/* Linked segments of row r: starts/caps, returns count (reference walk,
 * include/sparse_update.inl:77-86). */
static int row_chain(const or_dcsr *m, int32_t r, int64_t *st, int64_t *cp) {
  int n = 0;
  for (int l = 0; l < m->o.max_segs; l++) {
    int32_t s = m->seg[seg_index(m, l, r)];
    if (s < 0) break;
    st[n] = s;
    cp[n] = (int64_t)m->seg[seg_index(m, l, r) + 1] - s;
    n++;
  }
  return n;
}

/* Physical slot of logical position p of a row. */
static int64_t phys(const int64_t *st, const int64_t *cp, int ns, int64_t p) {
  for (int i = 0; i < ns; i++) {
    if (p < cp[i]) return st[i] + p;
    p -= cp[i];
  }
  return -1;
}

static void read_row(const or_dcsr *m, int32_t r, int32_t *c, double *v) {
  int64_t st[8], cp[8];
  int ns = row_chain(m, r, st, cp);
  int64_t L = m->row_sizes[r];
  for (int64_t p = 0; p < L; p++) {
    int64_t q = phys(st, cp, ns, p);
    c[p] = m->cols[q];
    v[p] = m->vals[q];
  }
}

static void write_row(or_dcsr *m, int32_t r, const int32_t *c, const double *v, int64_t L) {
  int64_t st[8], cp[8];
  int ns = row_chain(m, r, st, cp);
  for (int64_t p = 0; p < L; p++) {
    int64_t q = phys(st, cp, ns, p);
    m->cols[q] = c[p];
    m->vals[q] = v[p];
  }
}

int64_t or_nnz(const or_dcsr *m) {
  int64_t s = 0;
  for (int32_t r = 0; r < m->n_rows; r++) s += m->row_sizes[r];
  return s;
}

static int32_t max_row_len(const or_dcsr *m) {
  int32_t mx = 0;
  for (int32_t r = 0; r < m->n_rows; r++)
    if (m->row_sizes[r] > mx) mx = m->row_sizes[r];
  return mx;
}

/* ------------------------------------------------- stable counting sorts */

/* perm <- indices 0..n-1 stably sorted by key[] in [0, nkeys). */
static void counting_sort(const int32_t *key, int64_t n, int32_t nkeys, const int64_t *in, int64_t *out) {
  int64_t *cnt = (int64_t *)calloc((size_t)nkeys + 1, sizeof(int64_t));
  for (int64_t i = 0; i < n; i++) cnt[key[in[i]] + 1]++;
  for (int32_t k = 0; k < nkeys; k++) cnt[k + 1] += cnt[k];
  for (int64_t i = 0; i < n; i++) out[cnt[key[in[i]]]++] = in[i];
  free(cnt);
}

/* Stable sort of 0..n-1 by (row[,col]) -- the cusp sort_by_row /
 * sort_by_row_and_column LSD order (cusp/detail/sort.inl:38-113). */
static int64_t *stable_order(const int32_t *rows, const int32_t *cols, int64_t n, int32_t nr,
                             int32_t nc, int by_col) {
  int64_t *a = (int64_t *)malloc((size_t)(n ? n : 1) * sizeof(int64_t));
  int64_t *b = (int64_t *)malloc((size_t)(n ? n : 1) * sizeof(int64_t));
  for (int64_t i = 0; i < n; i++) a[i] = i;
  if (by_col) {
    counting_sort(cols, n, nc, a, b);
    counting_sort(rows, n, nr, b, a);
  } else {
    counting_sort(rows, n, nr, a, b);
    memcpy(a, b, (size_t)n * sizeof(int64_t));
  }
  free(b);
  return a;
}

static int check_indices(const or_dcsr *m, const int32_t *rows, const int32_t *cols, int64_t n) {
  for (int64_t i = 0; i < n; i++)
    if (rows[i] < 0 || rows[i] >= m->n_rows || cols[i] < 0 || cols[i] >= m->n_cols) return OR_BAD_INDEX;
  return OR_OK;
}

/* -------------------------------------------------------------- loading */

/* Lay out rows with policy capacities in row order (reference SetRowData,
 * include/sparse_update.inl:1078-1096, generalised by the slack policy). */
static void layout_rows(or_dcsr *m, const int64_t *len) {
  size_t ns = (size_t)m->pitch * m->o.max_segs;
  for (size_t i = 0; i < ns; i++) m->seg[i] = -1;
  int64_t off = 0;
  for (int32_t r = 0; r < m->n_rows; r++) {
    int64_t cap = or_policy_cap(&m->o, len[r]);
    m->seg[seg_index(m, 0, r)] = (int32_t)off;
    m->seg[seg_index(m, 0, r) + 1] = (int32_t)(off + cap);
    m->row_sizes[r] = (int32_t)len[r];
    off += cap;
  }
  m->row_sizes[m->n_rows] = (int32_t)off;
}

/* Canonical row content from an ordered entry list: in MERGE mode equal
 * columns of a row are summed left to right in list order. */
static int load_sorted(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals,
                       const int64_t *ord, int64_t n) {
  int64_t *len = (int64_t *)calloc((size_t)m->n_rows + 1, sizeof(int64_t));
  int32_t *oc = (int32_t *)malloc((size_t)(n ? n : 1) * sizeof(int32_t));
  double *ov = (double *)malloc((size_t)(n ? n : 1) * sizeof(double));
  int64_t w = 0;
  int32_t prow = -1, pcol = -1;
  for (int64_t i = 0; i < n; i++) {
    int64_t e = ord[i];
    int32_t r = rows[e], c = cols[e];
    double v = vround(m->dtype, vals[e]);
    if (m->o.mode == OR_MERGE && r == prow && c == pcol) {
      ov[w - 1] = vadd(m->dtype, ov[w - 1], v);
      continue;
    }
    oc[w] = c;
    ov[w] = v;
    w++;
    len[r]++;
    prow = r;
    pcol = c;
  }
  layout_rows(m, len);
  int64_t top = m->row_sizes[m->n_rows];
  set_pool(m, or_pool_capacity(&m->o, top));
  int64_t p = 0;
  for (int32_t r = 0; r < m->n_rows; r++) {
    int64_t s = m->seg[seg_index(m, 0, r)];
    for (int64_t j = 0; j < len[r]; j++) {
      m->cols[s + j] = oc[p];
      m->vals[s + j] = ov[p];
      p++;
    }
  }
  free(len);
  free(oc);
  free(ov);
  return OR_OK;
}

int or_load_coo(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals, int64_t nnz) {
  int st = check_indices(m, rows, cols, nnz);
  if (st) return st;
  int64_t *ord = stable_order(rows, cols, nnz, m->n_rows, m->n_cols, m->o.mode == OR_MERGE);
  st = load_sorted(m, rows, cols, vals, ord, nnz);
  free(ord);
  return st;
}

/* Reference LoadMatrix(dcsr, csr) include/load.h:207-227 (copy + SetRowData);
 * MERGE mode additionally canonicalises each row (sorted, duplicates summed). */
int or_load_csr(or_dcsr *m, const int32_t *row_ptr, const int32_t *cols, const double *vals) {
  int64_t nnz = row_ptr[m->n_rows];
  for (int32_t r = 0; r < m->n_rows; r++)
    if (row_ptr[r + 1] < row_ptr[r] || row_ptr[0] != 0) return OR_BAD_ARG;
  int32_t *rows = (int32_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(int32_t));
  for (int32_t r = 0; r < m->n_rows; r++)
    for (int64_t j = row_ptr[r]; j < row_ptr[r + 1]; j++) rows[j] = r;
  int st = or_load_coo(m, rows, cols, vals, nnz);
  free(rows);
  return st;
}

/* ----------------------------------------------------------- compaction */

/* Reference SortMatrixRow include/load.h:404-581 (+ CompactIndices/SetOffsets
 * include/sparse_update.inl:916-1073), with the row-ordered layout of the
 * canonical semantics instead of the bin-permuted one. */
void or_compact(or_dcsr *m) {
  int64_t n = m->n_rows;
  int64_t nnz = or_nnz(m);
  int32_t *oc = (int32_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(int32_t));
  double *ov = (double *)malloc((size_t)(nnz ? nnz : 1) * sizeof(double));
  int64_t *len = (int64_t *)malloc((size_t)(n + 1) * sizeof(int64_t));
  int64_t p = 0;
  for (int32_t r = 0; r < n; r++) {
    len[r] = m->row_sizes[r];
    read_row(m, r, oc + p, ov + p);
    p += len[r];
  }
  layout_rows(m, len);
  int64_t top = m->row_sizes[n];
  int64_t cap = or_pool_capacity(&m->o, top);
  if (cap < m->pool_cap) cap = m->pool_cap;
  free(m->cols);
  free(m->vals);
  m->cols = NULL;
  m->vals = NULL;
  set_pool(m, cap);
  p = 0;
  for (int32_t r = 0; r < n; r++) {
    int64_t s = m->seg[seg_index(m, 0, r)];
    for (int64_t j = 0; j < len[r]; j++) {
      m->cols[s + j] = oc[p];
      m->vals[s + j] = ov[p];
      p++;
    }
  }
  free(oc);
  free(ov);
  free(len);
}

void or_grow(or_dcsr *m, int64_t new_cap) {
  if (new_cap > m->pool_cap) set_pool(m, new_cap);
}

/* -------------------------------------------------------------- updates */

typedef struct {
  int32_t row;
  int64_t b0, b1;     /* range in the sorted order */
  int64_t seg_cap;    /* new segment capacity (0 = none) */
  int layer;          /* layer of the new segment */
} touched_t;

/* MERGE mode plan + apply for one batch. */
static int update_merge(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals,
                        int64_t nnz, int64_t *need_out) {
  int64_t *ord = stable_order(rows, cols, nnz, m->n_rows, m->n_cols, 1);
  int64_t nt = 0;
  touched_t *t = (touched_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(touched_t));
  for (int64_t i = 0; i < nnz; i++) {
    if (i == 0 || rows[ord[i]] != rows[ord[i - 1]]) {
      t[nt].row = rows[ord[i]];
      t[nt].b0 = i;
      nt++;
    }
    t[nt - 1].b1 = i + 1;
  }
  int32_t mx = max_row_len(m);
  int32_t *ac = (int32_t *)malloc((size_t)(mx + 1) * sizeof(int32_t));
  double *av = (double *)malloc((size_t)(mx + 1) * sizeof(double));
  int st = OR_OK;
  int64_t need = 0;
  /* plan: new length, capacity, layer, allocation size */
  for (int64_t k = 0; k < nt; k++) {
    int32_t r = t[k].row;
    int64_t L = m->row_sizes[r];
    read_row(m, r, ac, av);
    int64_t mnew = 0, ins0 = L;
    for (int64_t i = t[k].b0; i < t[k].b1; i++) {
      int32_t c = cols[ord[i]];
      if (i > t[k].b0 && c == cols[ord[i - 1]]) continue;
      int64_t lo = 0, hi = L;
      while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (ac[mid] < c) lo = mid + 1; else hi = mid;
      }
      if (lo >= L || ac[lo] != c) {
        if (mnew == 0) ins0 = lo;
        mnew++;
      }
    }
    int64_t st_[8], cp_[8];
    int ns = row_chain(m, r, st_, cp_);
    int64_t tot = 0;
    for (int i = 0; i < ns; i++) tot += cp_[i];
    int64_t nl = L + mnew;
    t[k].seg_cap = 0;
    t[k].layer = -1;
    if (mnew > 0 && L - ins0 > m->o.reloc_min) {
      /* relocation: the whole merged row goes to one fresh segment */
      t[k].seg_cap = or_policy_cap(&m->o, nl);
      t[k].layer = 8; /* marker: reset the chain to this segment */
      need += t[k].seg_cap;
    } else if (nl > tot) {
      t[k].layer = tot == 0 ? 0 : ns;
      if (t[k].layer >= m->o.max_segs) {
        /* every layer in use: relocation into one fresh segment (chain reset) */
        t[k].seg_cap = or_policy_cap(&m->o, nl);
        t[k].layer = 8;
      } else {
        t[k].seg_cap = align_up64(or_policy_cap(&m->o, nl) - tot, m->o.align);
      }
      need += t[k].seg_cap;
    }
  }
  int64_t top = m->row_sizes[m->n_rows];
  if (need_out) *need_out = top + need;
  if (st == OR_OK && top + need > m->pool_cap) st = OR_POOL_EXHAUSTED;
  if (st == OR_OK) {
    int32_t *nc = (int32_t *)malloc((size_t)(mx + nnz + 1) * sizeof(int32_t));
    double *nv = (double *)malloc((size_t)(mx + nnz + 1) * sizeof(double));
    int64_t addr = top;
    for (int64_t k = 0; k < nt; k++) {
      int32_t r = t[k].row;
      int64_t L = m->row_sizes[r];
      read_row(m, r, ac, av);
      if (t[k].layer == 8) {
        for (int l = 0; l < m->o.max_segs; l++) {
          m->seg[seg_index(m, l, r)] = -1;
          m->seg[seg_index(m, l, r) + 1] = -1;
        }
        m->seg[seg_index(m, 0, r)] = (int32_t)addr;
        m->seg[seg_index(m, 0, r) + 1] = (int32_t)(addr + t[k].seg_cap);
        addr += t[k].seg_cap;
      } else if (t[k].seg_cap > 0) {
        m->seg[seg_index(m, t[k].layer, r)] = (int32_t)addr;
        m->seg[seg_index(m, t[k].layer, r) + 1] = (int32_t)(addr + t[k].seg_cap);
        addr += t[k].seg_cap;
      }
      int64_t ia = 0, w = 0, i = t[k].b0;
      while (ia < L || i < t[k].b1) {
        int32_t cb = i < t[k].b1 ? cols[ord[i]] : 0x7fffffff;
        if (ia < L && ac[ia] < cb) {
          nc[w] = ac[ia];
          nv[w++] = av[ia++];
        } else if (ia < L && ac[ia] == cb) {
          double v = av[ia++];
          while (i < t[k].b1 && cols[ord[i]] == cb) v = vadd(m->dtype, v, vround(m->dtype, vals[ord[i++]]));
          nc[w] = cb;
          nv[w++] = v;
        } else {
          double v = vround(m->dtype, vals[ord[i++]]);
          while (i < t[k].b1 && cols[ord[i]] == cb) v = vadd(m->dtype, v, vround(m->dtype, vals[ord[i++]]));
          nc[w] = cb;
          nv[w++] = v;
        }
      }
      m->row_sizes[r] = (int32_t)w;
      write_row(m, r, nc, nv, w);
    }
    m->row_sizes[m->n_rows] = (int32_t)addr;
    free(nc);
    free(nv);
  }
  free(ac);
  free(av);
  free(t);
  free(ord);
  return st;
}

/* APPEND mode: reference UpdateMatrix_dcsr include/sparse_update.inl:16-130
 * (segment walk :77-88, empty-row branch :56-72, new segment of
 * rlB - free + alpha at layer Aoffset+1 :93-105, append :108-124), with
 * deterministic row-ordered allocation and an overflow guard. */
static int update_append(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals,
                         int64_t nnz, int64_t *need_out) {
  int64_t *ord = stable_order(rows, cols, nnz, m->n_rows, m->n_cols, 0);
  int64_t nt = 0;
  touched_t *t = (touched_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(touched_t));
  for (int64_t i = 0; i < nnz; i++) {
    if (i == 0 || rows[ord[i]] != rows[ord[i - 1]]) {
      t[nt].row = rows[ord[i]];
      t[nt].b0 = i;
      nt++;
    }
    t[nt - 1].b1 = i + 1;
  }
  int st = OR_OK;
  int64_t need = 0;
  for (int64_t k = 0; k < nt; k++) {
    int32_t r = t[k].row;
    int64_t rlA = m->row_sizes[r], rlB = t[k].b1 - t[k].b0;
    int32_t s0 = m->seg[seg_index(m, 0, r)], e0 = m->seg[seg_index(m, 0, r) + 1];
    t[k].seg_cap = 0;
    t[k].layer = -1;
    if (rlA == 0 && s0 == e0) {
      t[k].seg_cap = rlB + m->o.alpha;
      t[k].layer = 0;
    } else {
      int64_t st_[8], cp_[8];
      int ns = row_chain(m, r, st_, cp_);
      int off = 0;
      int64_t nxt;
      if (rlA > 0) {
        int64_t a = 0;
        while (a < rlA) {
          a += cp_[off];
          if (a < rlA) off++;
        }
        nxt = st_[off] + cp_[off] + rlA - a;
      } else {
        nxt = st_[0];
      }
      (void)ns;
      int64_t fr = st_[off] + cp_[off] - nxt;
      if (fr < rlB) {
        t[k].seg_cap = rlB - fr + m->o.alpha;
        t[k].layer = off + 1;
        if (t[k].layer >= m->o.max_segs) st = OR_LAYER_OVERFLOW;
      }
    }
    need += t[k].seg_cap;
  }
  int64_t top = m->row_sizes[m->n_rows];
  if (need_out) *need_out = top + need;
  if (st == OR_OK && top + need > m->pool_cap) st = OR_POOL_EXHAUSTED;
  if (st == OR_OK) {
    int64_t addr = top;
    for (int64_t k = 0; k < nt; k++) {
      int32_t r = t[k].row;
      if (t[k].seg_cap > 0) {
        m->seg[seg_index(m, t[k].layer, r)] = (int32_t)addr;
        m->seg[seg_index(m, t[k].layer, r) + 1] = (int32_t)(addr + t[k].seg_cap);
        addr += t[k].seg_cap;
      }
      int64_t st_[8], cp_[8];
      int ns = row_chain(m, r, st_, cp_);
      int64_t L = m->row_sizes[r];
      for (int64_t i = t[k].b0; i < t[k].b1; i++) {
        int64_t q = phys(st_, cp_, ns, L++);
        m->cols[q] = cols[ord[i]];
        m->vals[q] = vround(m->dtype, vals[ord[i]]);
      }
      m->row_sizes[r] = (int32_t)L;
    }
    m->row_sizes[m->n_rows] = (int32_t)addr;
  }
  free(t);
  free(ord);
  return st;
}

int or_update(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals, int64_t nnz,
              int64_t *need) {
  int st = check_indices(m, rows, cols, nnz);
  if (need) *need = m->row_sizes[m->n_rows];
  if (st) return st;
  if (nnz == 0) return OR_OK;
  if (m->o.mode == OR_APPEND) return update_append(m, rows, cols, vals, nnz, need);
  return update_merge(m, rows, cols, vals, nnz, need);
}

/* The library's repair policy for a rejected update: compact, retry; if the
 * pool is still short, grow it to the policy capacity of the requirement. */
int or_update_auto(or_dcsr *m, const int32_t *rows, const int32_t *cols, const double *vals, int64_t nnz) {
  int64_t need = 0;
  int st = or_update(m, rows, cols, vals, nnz, &need);
  if (st == OR_POOL_EXHAUSTED || st == OR_LAYER_OVERFLOW) {
    or_compact(m);
    st = or_update(m, rows, cols, vals, nnz, &need);
    if (st == OR_POOL_EXHAUSTED) {
      or_grow(m, or_pool_capacity(&m->o, need));
      st = or_update(m, rows, cols, vals, nnz, &need);
    }
  }
  return st;
}

/* --------------------------------------------------------------- export */

/* Reference LoadMatrix(csr, dcsr) include/load.h:232-253, valid in any state
 * (row order, chains followed). */
void or_export_csr(const or_dcsr *m, int32_t *row_ptr, int32_t *cols, double *vals) {
  int64_t p = 0;
  row_ptr[0] = 0;
  for (int32_t r = 0; r < m->n_rows; r++) {
    read_row(m, r, cols + p, vals + p);
    p += m->row_sizes[r];
    row_ptr[r + 1] = (int32_t)p;
  }
}

/* ---------------------------------------------------------------- SpMV */

/* Reference spmv_dcsr_bin* include/spmv.inl:364-622: per-row sum over the
 * segment chain, here in FP64 with current (not stale) row lengths. */
void or_spmv(const or_dcsr *m, const double *x, int32_t k, int64_t ldx, double *y, int64_t ldy,
             double alpha, double beta) {
  double acc[8];
  for (int32_t r = 0; r < m->n_rows; r++) {
    int64_t st[8], cp[8];
    int ns = row_chain(m, r, st, cp);
    for (int j = 0; j < k; j++) acc[j] = 0.0;
    int64_t L = m->row_sizes[r];
    for (int64_t p = 0; p < L; p++) {
      int64_t q = phys(st, cp, ns, p);
      double a = m->vals[q];
      int64_t c = m->cols[q];
      for (int j = 0; j < k; j++) acc[j] += a * x[c * ldx + j];
    }
    for (int j = 0; j < k; j++) {
      double out = alpha * acc[j];
      if (beta != 0.0) out += beta * y[r * ldy + j];
      y[r * ldy + j] = out;
    }
  }
}

void or_row_reduce(const or_dcsr *m, int32_t op, double *y) {
  for (int32_t r = 0; r < m->n_rows; r++) {
    int64_t st[8], cp[8];
    int ns = row_chain(m, r, st, cp);
    int64_t L = m->row_sizes[r];
    double acc = 0.0;
    for (int64_t p = 0; p < L; p++) {
      double a = m->vals[phys(st, cp, ns, p)];
      if (op == 0) acc += a;
      else if (op == 1) acc = (p == 0 || a > acc) ? a : acc;
      else if (op == 2) acc = (p == 0 || a < acc) ? a : acc;
    }
    if (op == 3) acc = (double)L;
    y[r] = acc;
  }
}

/* -------------------------------------------------------------- SpGEMM */

void or_spgemm_counts(const or_dcsr *A, const or_dcsr *B, int64_t *counts) {
  int32_t mx = max_row_len(A);
  int32_t *ac = (int32_t *)malloc((size_t)(mx + 1) * sizeof(int32_t));
  double *av = (double *)malloc((size_t)(mx + 1) * sizeof(double));
  for (int32_t i = 0; i < A->n_rows; i++) {
    read_row(A, i, ac, av);
    int64_t s = 0;
    for (int32_t p = 0; p < A->row_sizes[i]; p++) s += B->row_sizes[ac[p]];
    counts[i] = s;
  }
  free(ac);
  free(av);
}

typedef struct { int32_t col; int64_t pos; double v; } prod_t;
static int prod_cmp(const void *a, const void *b) {
  const prod_t *x = (const prod_t *)a, *y = (const prod_t *)b;
  if (x->col != y->col) return x->col < y->col ? -1 : 1;
  return x->pos < y->pos ? -1 : (x->pos > y->pos);
}

/* Reference spmm_dcsr_* include/spmm.inl:7-101 (expand products of row i in
 * A-order then B-order), :169-265 (sort by column, sum equal columns, keep
 * explicit zeros); all rows computed (no >2048 product gap). */
or_dcsr *or_spgemm(const or_dcsr *A, const or_dcsr *B, const or_opts *o, int *status) {
  *status = OR_OK;
  if (A->n_cols != B->n_rows || A->dtype != B->dtype) {
    *status = OR_BAD_ARG;
    return NULL;
  }
  int32_t dt = A->dtype;
  int64_t *cnt = (int64_t *)malloc((size_t)(A->n_rows + 1) * sizeof(int64_t));
  or_spgemm_counts(A, B, cnt);
  int64_t mxp = 0;
  for (int32_t i = 0; i < A->n_rows; i++)
    if (cnt[i] > mxp) mxp = cnt[i];
  prod_t *pr = (prod_t *)malloc((size_t)(mxp + 1) * sizeof(prod_t));
  int32_t mxa = max_row_len(A), mxb = max_row_len(B);
  int32_t *ac = (int32_t *)malloc((size_t)(mxa + 1) * sizeof(int32_t));
  double *av = (double *)malloc((size_t)(mxa + 1) * sizeof(double));
  int32_t *bc = (int32_t *)malloc((size_t)(mxb + 1) * sizeof(int32_t));
  double *bv = (double *)malloc((size_t)(mxb + 1) * sizeof(double));
  /* gather the output as COO in final order, then load with C's policy */
  int64_t cap = 1024, n = 0;
  int32_t *cr = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
  int32_t *cc = (int32_t *)malloc((size_t)cap * sizeof(int32_t));
  double *cv = (double *)malloc((size_t)cap * sizeof(double));
  for (int32_t i = 0; i < A->n_rows; i++) {
    read_row(A, i, ac, av);
    int64_t np = 0;
    for (int32_t p = 0; p < A->row_sizes[i]; p++) {
      int32_t k = ac[p];
      read_row(B, k, bc, bv);
      for (int32_t q = 0; q < B->row_sizes[k]; q++) {
        pr[np].col = bc[q];
        pr[np].pos = np;
        pr[np].v = vmul(dt, av[p], bv[q]);
        np++;
      }
    }
    qsort(pr, (size_t)np, sizeof(prod_t), prod_cmp);
    for (int64_t j = 0; j < np;) {
      double v = pr[j].v;
      int64_t e = j + 1;
      while (e < np && pr[e].col == pr[j].col) v = vadd(dt, v, pr[e++].v);
      if (n == cap) {
        cap *= 2;
        cr = (int32_t *)realloc(cr, (size_t)cap * sizeof(int32_t));
        cc = (int32_t *)realloc(cc, (size_t)cap * sizeof(int32_t));
        cv = (double *)realloc(cv, (size_t)cap * sizeof(double));
      }
      cr[n] = i;
      cc[n] = pr[j].col;
      cv[n] = v;
      n++;
      j = e;
    }
  }
  or_opts oo = *o;
  oo.mode = OR_MERGE;
  or_dcsr *C = or_create(A->n_rows, B->n_cols, dt, &oo);
  *status = or_load_coo(C, cr, cc, cv, n);
  free(cnt);
  free(pr);
  free(ac);
  free(av);
  free(bc);
  free(bv);
  free(cr);
  free(cc);
  free(cv);
  return C;
}

/* --------------------------------------------------- segmented primitives */

void or_count_sorted_indices(const int32_t *I, int64_t n, int32_t *X) {
  for (int64_t i = 0; i < n; i++) X[I[i]] += 1;
}

int64_t or_reduce_by_key(const int32_t *keys, const double *vals, int64_t n, int32_t dtype,
                         int32_t *out_keys, double *out_vals) {
  /* The library's stated order: a run is cut into pieces at its head and at
   * every multiple of RBK_PIECE inside it; each piece is summed left to
   * right, then the piece sums left to right.  (The reference's CTA
   * reduce-by-key, include/reduce.inl:139-308, sums in a tree order of its
   * own; it specifies none.) */
  const int64_t RBK_PIECE = 256;
  int64_t w = 0, i = 0;
  while (i < n) {
    int64_t e = i + 1;
    while (e < n && keys[e] == keys[i]) e++;
    double total = 0.0;
    for (int64_t p = i; p < e;) {
      int64_t pe = (p / RBK_PIECE + 1) * RBK_PIECE;
      if (pe > e) pe = e;
      double s = vround(dtype, vals[p]);
      for (int64_t q = p + 1; q < pe; q++) s = vadd(dtype, s, vround(dtype, vals[q]));
      total = p == i ? s : vadd(dtype, total, s);
      p = pe;
    }
    out_keys[w] = keys[i];
    out_vals[w] = total;
    w++;
    i = e;
  }
  return w;
}

void or_bin_counts(const or_dcsr *m, int64_t *counts) {
  for (int i = 0; i < 7; i++) counts[i] = 0;
  for (int32_t r = 0; r < m->n_rows; r++) {
    int32_t rl = m->row_sizes[r];
    int b = rl < 2 ? 0 : rl < 4 ? 1 : rl < 8 ? 2 : rl < 16 ? 3 : rl < 32 ? 4 : rl < 512 ? 5 : 6;
    counts[b]++;
  }
}

/* ---------------------------------------------------------- validation */

int or_validate(const or_dcsr *m) {
  int64_t top = m->row_sizes[m->n_rows];
  if (top > m->pool_cap) return -1;
  for (int32_t r = 0; r < m->n_rows; r++) {
    int64_t st[8], cp[8];
    int ns = row_chain(m, r, st, cp);
    int64_t tot = 0;
    for (int i = 0; i < ns; i++) {
      if (cp[i] < 0 || st[i] + cp[i] > top) return -2;
      tot += cp[i];
    }
    for (int l = ns; l < m->o.max_segs; l++)
      if (m->seg[seg_index(m, l, r)] != -1) return -3;
    if (m->row_sizes[r] > tot || m->row_sizes[r] < 0) return -4;
    int32_t prev = -1;
    for (int64_t p = 0; p < m->row_sizes[r]; p++) {
      int32_t c = m->cols[phys(st, cp, ns, p)];
      if (c < 0 || c >= m->n_cols) return -5;
      if (m->o.mode == OR_MERGE && c <= prev) return -6;
      prev = c;
    }
  }
  return 0;
}
