/*
 * ORACLE -- test infrastructure only (see airfoil_oracle.c).
 *
 * Sequential restatement of the product's mesh renumbering, to pin the GPU
 * implementation bit for bit:
 *
 *  - base graph (op2/src/externlib/op_renumber.cpp:274-350): targets of one
 *    element of the base map are adjacent (self map: rows are the adjacency);
 *  - base order: reverse Cuthill-McKee as the product defines it (the
 *    reference's base order comes from PT-Scotch, an unvendored library, so
 *    this part of the parity is unpinned): George-Liu pseudo-peripheral
 *    start from an unvisited vertex of minimum degree, lowest id on ties
 *    (then the min-degree vertex of the last BFS level, lowest id on ties,
 *    at most 8 rounds, stop when the
 *    eccentricity stops growing); sequential Cuthill-McKee visiting each
 *    vertex's unvisited neighbours by (degree capped at 63, id); reversed;
 *  - propagation (propagate_reordering, :72-151) in the reference's
 *    recursive order over the maps in declaration order, ties of the
 *    first-target sort broken by original index (the reference leaves them
 *    to qsort);
 *  - the result: perm[set][i] = new index of element i.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int from, to, dim;
  const int *map;
} orc_map;

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* CSR adjacency of the base map's target set (rows sorted, unique) */
static void build_graph(const orc_map *base, int nfrom, int nto, int **row_out, int **col_out) {
  int *deg = calloc((size_t)nto + 1, sizeof(int));
  int d = base->dim;
  if (base->from == base->to) {
    for (int u = 0; u < nto; u++)
      for (int a = 0; a < d; a++) {
        int v = base->map[(size_t)u * d + a];
        if (v >= 0 && v < nto && v != u) deg[u]++;
      }
  } else {
    for (int i = 0; i < nfrom; i++)
      for (int a = 0; a < d; a++) {
        int u = base->map[(size_t)i * d + a];
        if (u < 0 || u >= nto) continue;
        for (int b = 0; b < d; b++) {
          int v = base->map[(size_t)i * d + b];
          if (b != a && v != u && v >= 0 && v < nto) deg[u]++;
        }
      }
  }
  int *row = malloc(sizeof(int) * ((size_t)nto + 1));
  row[0] = 0;
  for (int u = 0; u < nto; u++) row[u + 1] = row[u] + deg[u];
  int *col = malloc(sizeof(int) * ((size_t)row[nto] + 1));
  int *fill = calloc((size_t)nto + 1, sizeof(int));
  if (base->from == base->to) {
    for (int u = 0; u < nto; u++)
      for (int a = 0; a < d; a++) {
        int v = base->map[(size_t)u * d + a];
        if (v >= 0 && v < nto && v != u) col[row[u] + fill[u]++] = v;
      }
  } else {
    for (int i = 0; i < nfrom; i++)
      for (int a = 0; a < d; a++) {
        int u = base->map[(size_t)i * d + a];
        if (u < 0 || u >= nto) continue;
        for (int b = 0; b < d; b++) {
          int v = base->map[(size_t)i * d + b];
          if (b != a && v != u && v >= 0 && v < nto) col[row[u] + fill[u]++] = v;
        }
      }
  }
  /* sort + unique rows, then compact */
  int *row2 = malloc(sizeof(int) * ((size_t)nto + 1));
  int k = 0;
  row2[0] = 0;
  for (int u = 0; u < nto; u++) {
    int *c = col + row[u];
    qsort(c, (size_t)(row[u + 1] - row[u]), sizeof(int), cmp_int);
    for (int j = 0; j < row[u + 1] - row[u]; j++)
      if (j == 0 || c[j] != c[j - 1]) col[k++] = c[j];
    row2[u + 1] = k;
  }
  free(deg);
  free(fill);
  free(row);
  *row_out = row2;
  *col_out = col;
}

static int bfs_levels(int n, const int *row, const int *col, const int *newidx, int *mark,
                      int stamp, int start, int *buf_a, int *buf_b, int **last, int *last_len) {
  int *cur = buf_a, *nxt = buf_b, len = 1, nlev = 0;
  (void)n;
  cur[0] = start;
  mark[start] = stamp;
  for (;;) {
    int nl = 0;
    nlev++;
    for (int j = 0; j < len; j++) {
      int u = cur[j];
      for (int t = row[u]; t < row[u + 1]; t++) {
        int v = col[t];
        if (newidx[v] < 0 && mark[v] != stamp) {
          mark[v] = stamp;
          nxt[nl++] = v;
        }
      }
    }
    if (nl == 0) {
      *last = cur;
      *last_len = len;
      return nlev;
    }
    int *t = cur;
    cur = nxt;
    nxt = t;
    len = nl;
  }
}

typedef struct {
  uint64_t key;
} key64;

static int cmp_u64(const void *a, const void *b) {
  uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return (x > y) - (x < y);
}

/* perm[v] = new index (reverse Cuthill-McKee) */
void orc_rcm(int n, const int *row, const int *col, int *perm) {
  int *newidx = malloc(sizeof(int) * ((size_t)n + 1));
  int *mark = calloc((size_t)n + 1, sizeof(int));
  int *a = malloc(sizeof(int) * ((size_t)n + 1));
  int *b = malloc(sizeof(int) * ((size_t)n + 1));
  uint64_t *keys = malloc(sizeof(uint64_t) * ((size_t)n + 1));
  for (int i = 0; i < n; i++) newidx[i] = -1;
  int pos = 0, stamp = 1;
  while (pos < n) {
    /* an unvisited vertex of minimum degree, lowest id on ties */
    int start = -1, sd = 0x7fffffff;
    for (int v = 0; v < n; v++)
      if (newidx[v] < 0 && row[v + 1] - row[v] < sd) {
        sd = row[v + 1] - row[v];
        start = v;
      }
    int *last, last_len;
    int ecc = bfs_levels(n, row, col, newidx, mark, stamp++, start, a, b, &last, &last_len);
    for (int round = 0; round < 8; round++) {
      int bd = 0x7fffffff, best = 0x7fffffff;
      for (int j = 0; j < last_len; j++) {
        int v = last[j], d = row[v + 1] - row[v];
        if (d < bd || (d == bd && v < best)) {
          bd = d;
          best = v;
        }
      }
      int e2 = bfs_levels(n, row, col, newidx, mark, stamp++, best, a, b, &last, &last_len);
      if (e2 <= ecc) break;
      ecc = e2;
      start = best;
    }
    /* Cuthill-McKee: level by level, new vertices keyed by
       (first parent's position in the level, min(degree, 63), id) */
    int *cur = a, *nxt = b, len = 1;
    cur[0] = start;
    newidx[start] = pos++;
    for (;;) {
      int nl = 0;
      for (int j = 0; j < len; j++) {
        int u = cur[j];
        for (int t = row[u]; t < row[u + 1]; t++) {
          int v = col[t];
          if (newidx[v] == -1) {
            newidx[v] = -2; /* discovered by its first parent */
            int d = row[v + 1] - row[v];
            if (d > 63) d = 63;
            keys[nl++] = ((uint64_t)(unsigned)j << 38) | ((uint64_t)d << 32) | (unsigned)v;
          }
        }
      }
      if (nl == 0) break;
      qsort(keys, (size_t)nl, sizeof(uint64_t), cmp_u64);
      for (int k = 0; k < nl; k++) {
        int v = (int)(keys[k] & 0xffffffffu);
        nxt[k] = v;
        newidx[v] = pos + k;
      }
      pos += nl;
      int *t = cur;
      cur = nxt;
      nxt = t;
      len = nl;
    }
  }
  for (int v = 0; v < n; v++) perm[v] = n - 1 - newidx[v];
  free(newidx);
  free(mark);
  free(a);
  free(b);
  free(keys);
}

typedef struct {
  int nsets, nmaps;
  const int *set_size;
  const orc_map *maps;
  int **perm; /* per set, NULL until derived */
} prop_ctx;

typedef struct {
  int key, idx;
} kv;

static int cmp_kv(const void *a, const void *b) {
  const kv *x = a, *y = b;
  if (x->key != y->key) return (x->key > y->key) - (x->key < y->key);
  return (x->idx > y->idx) - (x->idx < y->idx);
}

static void propagate(prop_ctx *c, int from, int to) {
  int n = c->set_size[to];
  if (n == 0) return;
  if (!c->perm[to]) {
    for (int m = 0; m < c->nmaps; m++) {
      const orc_map *mp = &c->maps[m];
      if (mp->to != from || mp->from != to) continue;
      kv *r = malloc(sizeof(kv) * (size_t)n);
      for (int i = 0; i < n; i++) {
        r[i].key = c->perm[from][mp->map[(size_t)mp->dim * i]];
        r[i].idx = i;
      }
      qsort(r, (size_t)n, sizeof(kv), cmp_kv);
      c->perm[to] = malloc(sizeof(int) * (size_t)n);
      for (int i = 0; i < n; i++) c->perm[to][r[i].idx] = i;
      free(r);
      break;
    }
  }
  if (!c->perm[to]) {
    for (int m = 0; m < c->nmaps; m++) {
      const orc_map *mp = &c->maps[m];
      if (mp->to != to || mp->from != from) continue;
      int nf = c->set_size[from];
      int *inv = malloc(sizeof(int) * ((size_t)nf + 1));
      for (int i = 0; i < nf; i++) inv[c->perm[from][i]] = i;
      int *p = malloc(sizeof(int) * (size_t)n);
      for (int i = 0; i < n; i++) p[i] = -1;
      int counter = 0;
      for (int i = 0; i < nf; i++)
        for (int d = 0; d < mp->dim; d++) {
          int idx = mp->map[(size_t)inv[i] * mp->dim + d];
          if (idx < n && p[idx] == -1) p[idx] = counter++;
        }
      free(inv);
      int onto = counter == n;
      if (!onto) {
        free(p);
        continue;
      }
      c->perm[to] = p;
      break;
    }
  }
  if (!c->perm[to]) return;
  for (int m = 0; m < c->nmaps; m++)
    if (c->maps[m].to == to && !c->perm[c->maps[m].from]) propagate(c, to, c->maps[m].from);
  for (int m = 0; m < c->nmaps; m++)
    if (c->maps[m].from == to && !c->perm[c->maps[m].to]) propagate(c, to, c->maps[m].to);
}

/* Renumbering from base map `base` over sets/maps in declaration order.
 * maps_flat: per map {from, to, dim}; map_data: per map pointer.
 * perm_out[s] (caller-allocated, set_size[s] ints) receives the permutation;
 * has_perm[s] = 1 if the set was renumbered. */
int orc_renumber(int nsets, const int *set_size, int nmaps, const int *maps_flat,
                 const int *const *map_data, int base, int **perm_out, int *has_perm) {
  orc_map *maps = malloc(sizeof(orc_map) * (size_t)nmaps);
  for (int m = 0; m < nmaps; m++) {
    maps[m].from = maps_flat[3 * m];
    maps[m].to = maps_flat[3 * m + 1];
    maps[m].dim = maps_flat[3 * m + 2];
    maps[m].map = map_data[m];
  }
  const orc_map *bm = &maps[base];
  int *row, *col;
  build_graph(bm, set_size[bm->from], set_size[bm->to], &row, &col);
  prop_ctx c = {nsets, nmaps, set_size, maps, calloc((size_t)nsets, sizeof(int *))};
  c.perm[bm->to] = malloc(sizeof(int) * ((size_t)set_size[bm->to] + 1));
  orc_rcm(set_size[bm->to], row, col, c.perm[bm->to]);
  propagate(&c, bm->to, bm->to);
  for (int s = 0; s < nsets; s++) {
    has_perm[s] = c.perm[s] != NULL;
    if (c.perm[s]) {
      memcpy(perm_out[s], c.perm[s], sizeof(int) * (size_t)set_size[s]);
      free(c.perm[s]);
    }
  }
  free(c.perm);
  free(row);
  free(col);
  free(maps);
  return 0;
}
