/*
 * mbe_oracle.c -- CPU oracle for maximal biclique enumeration.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only
 * as the checker or the timed CPU baseline.  The engine never calls it.
 *
 * Three independent enumerators over the same input, all reporting the count
 * of maximal bicliques and the canonical set hash (ids are ORIGINAL ids: U =
 * the integers on an .adj line, V = 0-based line numbers):
 *
 *   orc_brute_force  closure of V-neighbourhood intersections on tiny graphs
 *                    (|U| <= 64): the maximal bicliques are exactly the
 *                    distinct non-empty L = N(S), S a non-empty set of V rows.
 *   orc_mbea         restatement of MbeaFinder::biclique_find
 *                    (src/BicliqueFinder.cu:20-57) with the biclique emitted at
 *                    its count site (line 53).
 *   orc_gmbe         restatement of the GMBE per-root enumeration: root set-up
 *                    of IterFinderWithMultipleVertex for a one-vertex task
 *                    (src/IterFinderGpu.cu:772-887), IterProcess
 *                    (src/IterFinderGpu.cu:12-69), finder_push and finder_pop
 *                    with PRUNE_EN (src/IterFinderGpu.h:206-303).  Roots run in
 *                    parallel with OpenMP; it also counts the algorithmic bytes
 *                    of the GMBE tree used as the roofline numerator.
 *
 * Set hash (shared definition with the engine, restated here independently):
 *   key_U(u) = fmix64(2u), key_V(v) = fmix64(2v+1) (MurmurHash3 finaliser),
 *   H(L,R) = fmix64(sum key_U ^ rotl64(sum key_V, 29) ^ (|L|<<32 | |R|)),
 *   set_hash = sum of H over all maximal bicliques, mod 2^64.
 */
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct orc_result {
  uint64_t count;
  uint64_t set_hash;
  uint64_t non_maximal;
  uint64_t alg_bytes; /* algorithmic bytes of the GMBE tree (orc_gmbe only) */
  uint64_t nodes;     /* pushes (orc_gmbe) / recursive calls (orc_mbea) */
} orc_result;

static inline uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}
static inline uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
static inline uint64_t key_u(int64_t u) { return fmix64((uint64_t)u * 2u); }
static inline uint64_t key_v(int64_t v) { return fmix64((uint64_t)v * 2u + 1u); }
static inline uint64_t bic_hash(uint64_t sL, uint64_t sR, uint64_t nL, uint64_t nR) {
  return fmix64(sL ^ rotl64(sR, 29) ^ ((nL << 32) | nR));
}

/* ------------------------------------------------------------------------ */
/* Internal graph: -t swap and -o 1/2 ordering restated from                 */
/* src/BiGraph.cu:67-92, 217-277.  The result does not depend on them; they  */
/* only fix the internal root order the GMBE restatement walks.             */
typedef struct ograph {
  int32_t nU, nV;
  int64_t nE;
  int32_t *off, *adj;   /* V rows -> U */
  int32_t *roff, *radj; /* U rows -> V */
  int32_t *v_orig, *u_orig;
  int swapped;
} ograph;

static const int32_t* g_sort_off;
static const int32_t* g_sort_adj;
static const int32_t* g_sort_orig;
static int g_sort_desc;
static int cmp_rows(const void* pa, const void* pb) {
  int32_t a = *(const int32_t*)pa, b = *(const int32_t*)pb;
  int32_t sa = g_sort_off[a + 1] - g_sort_off[a], sb = g_sort_off[b + 1] - g_sort_off[b];
  if (sa != sb) return g_sort_desc ? (sa > sb ? -1 : 1) : (sa < sb ? -1 : 1);
  for (int32_t i = 0; i < sa; ++i) {
    int32_t x = g_sort_adj[g_sort_off[a] + i], y = g_sort_adj[g_sort_off[b] + i];
    if (x != y) return x < y ? -1 : 1;
  }
  return g_sort_orig[a] < g_sort_orig[b] ? -1 : (g_sort_orig[a] > g_sort_orig[b]);
}

static void transpose(const int32_t* off, const int32_t* adj, int32_t nr, int32_t nc, int32_t** toff,
                      int32_t** tadj) {
  int64_t ne = off[nr];
  int32_t* o = (int32_t*)calloc((size_t)nc + 1, sizeof(int32_t));
  int32_t* a = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ne > 0 ? ne : 1));
  int32_t* fill = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nc > 0 ? nc : 1));
  for (int64_t i = 0; i < ne; ++i) o[adj[i] + 1]++;
  for (int32_t i = 0; i < nc; ++i) o[i + 1] += o[i];
  for (int32_t i = 0; i < nc; ++i) fill[i] = o[i];
  for (int32_t r = 0; r < nr; ++r)
    for (int32_t i = off[r]; i < off[r + 1]; ++i) a[fill[adj[i]]++] = r;
  free(fill);
  *toff = o;
  *tadj = a;
}

static void ograph_free(ograph* g) {
  free(g->off);
  free(g->adj);
  free(g->roff);
  free(g->radj);
  free(g->v_orig);
  free(g->u_orig);
}

static void ograph_build(int32_t nV, int32_t nU, const int32_t* row_off, const int32_t* col,
                         int uvtrans, int order, ograph* g) {
  int64_t nE = row_off[nV];
  int32_t *voff, *vadj, *uoff, *uadj;
  voff = (int32_t*)malloc(sizeof(int32_t) * ((size_t)nV + 1));
  vadj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nE > 0 ? nE : 1));
  memcpy(voff, row_off, sizeof(int32_t) * ((size_t)nV + 1));
  memcpy(vadj, col, sizeof(int32_t) * (size_t)nE);
  transpose(voff, vadj, nV, nU, &uoff, &uadj);
  int32_t* vorig = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nV > 0 ? nV : 1));
  int32_t* uorig = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nU > 0 ? nU : 1));
  for (int32_t i = 0; i < nV; ++i) vorig[i] = i;
  for (int32_t i = 0; i < nU; ++i) uorig[i] = i;
  int swap = (uvtrans == 1 && nU < nV) || (uvtrans == 2 && nU > nV);
  if (swap) {
    int32_t t = nU; nU = nV; nV = t;
    int32_t* p;
    p = voff; voff = uoff; uoff = p;
    p = vadj; vadj = uadj; uadj = p;
    p = vorig; vorig = uorig; uorig = p;
  }
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nV > 0 ? nV : 1));
  for (int32_t i = 0; i < nV; ++i) perm[i] = i;
  if (order == 1 || order == 2) {
    g_sort_off = voff;
    g_sort_adj = vadj;
    g_sort_orig = vorig;
    g_sort_desc = order == 2;
    qsort(perm, (size_t)nV, sizeof(int32_t), cmp_rows);
  }
  g->nU = nU;
  g->nV = nV;
  g->nE = nE;
  g->swapped = swap;
  g->off = (int32_t*)malloc(sizeof(int32_t) * ((size_t)nV + 1));
  g->adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nE > 0 ? nE : 1));
  g->v_orig = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nV > 0 ? nV : 1));
  g->off[0] = 0;
  for (int32_t i = 0; i < nV; ++i) {
    int32_t s = perm[i], len = voff[s + 1] - voff[s];
    memcpy(g->adj + g->off[i], vadj + voff[s], sizeof(int32_t) * (size_t)len);
    g->off[i + 1] = g->off[i] + len;
    g->v_orig[i] = vorig[s];
  }
  g->u_orig = uorig;
  transpose(g->off, g->adj, nV, nU, &g->roff, &g->radj);
  free(perm);
  free(voff);
  free(vadj);
  free(uoff);
  free(uadj);
  free(vorig);
}

/* Hash keys of internal vertices, in original ids and original sides. */
static inline uint64_t ikey_u(const ograph* g, int32_t u) {
  return g->swapped ? key_v(g->u_orig[u]) : key_u(g->u_orig[u]);
}
static inline uint64_t ikey_v(const ograph* g, int32_t v) {
  return g->swapped ? key_u(g->v_orig[v]) : key_v(g->v_orig[v]);
}
/* Hash of a biclique given internal-side sums (sI over internal U = L side). */
static inline uint64_t ihash(const ograph* g, uint64_t sI_U, uint64_t nI_U, uint64_t sI_V,
                             uint64_t nI_V) {
  return g->swapped ? bic_hash(sI_V, sI_U, nI_V, nI_U) : bic_hash(sI_U, sI_V, nI_U, nI_V);
}

static int bsearch_i32(const int32_t* a, int32_t n, int32_t key) {
  int32_t lo = 0, hi = n - 1;
  while (lo <= hi) {
    int32_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] == key) return mid;
    if (a[mid] < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* ------------------------------------------------------------------------ */
/* Brute-force closure (|U| <= 64).                                          */
int orc_brute_force(int32_t nV, int32_t nU, const int32_t* row_off, const int32_t* col,
                    orc_result* out) {
  memset(out, 0, sizeof(*out));
  if (nU > 64 || nU < 0 || nV < 0) return -1;
  uint64_t* nb = (uint64_t*)calloc((size_t)(nV > 0 ? nV : 1), sizeof(uint64_t));
  for (int32_t v = 0; v < nV; ++v)
    for (int32_t i = row_off[v]; i < row_off[v + 1]; ++i) nb[v] |= 1ULL << col[i];
  size_t cap = 1024, n = 0;
  uint64_t* sets = (uint64_t*)malloc(cap * sizeof(uint64_t));
  /* open-addressing membership table, grown as needed */
  size_t tcap = 4096;
  uint64_t* table = (uint64_t*)calloc(tcap, sizeof(uint64_t)); /* 0 = empty (L never 0) */
#define BF_INSERT(x)                                                              \
  do {                                                                            \
    uint64_t _x = (x);                                                            \
    if (n * 2 >= tcap) {                                                          \
      size_t ncap = tcap * 2;                                                     \
      uint64_t* nt = (uint64_t*)calloc(ncap, sizeof(uint64_t));                   \
      for (size_t _i = 0; _i < n; ++_i) {                                         \
        size_t h = (size_t)(fmix64(sets[_i]) & (ncap - 1));                       \
        while (nt[h]) h = (h + 1) & (ncap - 1);                                   \
        nt[h] = sets[_i];                                                         \
      }                                                                           \
      free(table);                                                                \
      table = nt;                                                                 \
      tcap = ncap;                                                                \
    }                                                                             \
    size_t h = (size_t)(fmix64(_x) & (tcap - 1));                                 \
    int found = 0;                                                                \
    while (table[h]) {                                                            \
      if (table[h] == _x) { found = 1; break; }                                   \
      h = (h + 1) & (tcap - 1);                                                   \
    }                                                                             \
    if (!found) {                                                                 \
      table[h] = _x;                                                              \
      if (n == cap) { cap *= 2; sets = (uint64_t*)realloc(sets, cap * sizeof(uint64_t)); } \
      sets[n++] = _x;                                                             \
    }                                                                             \
  } while (0)
  for (int32_t v = 0; v < nV; ++v)
    if (nb[v]) BF_INSERT(nb[v]);
  for (size_t i = 0; i < n; ++i)
    for (int32_t v = 0; v < nV; ++v) {
      uint64_t y = sets[i] & nb[v];
      if (y) BF_INSERT(y);
    }
#undef BF_INSERT
  for (size_t i = 0; i < n; ++i) {
    uint64_t L = sets[i], sL = 0, sR = 0, nR = 0;
    for (int32_t u = 0; u < nU; ++u)
      if (L >> u & 1) sL += key_u(u);
    for (int32_t v = 0; v < nV; ++v)
      if ((nb[v] & L) == L) { sR += key_v(v); ++nR; }
    out->set_hash += bic_hash(sL, sR, (uint64_t)__builtin_popcountll(L), nR);
  }
  out->count = n;
  free(sets);
  free(table);
  free(nb);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* MbeaFinder restatement (src/BicliqueFinder.cu:20-57).                     */
typedef struct mbea_ctx {
  const ograph* g;
  orc_result* r;
} mbea_ctx;

static int32_t isect(const int32_t* a, int32_t na, const int32_t* b, int32_t nb, int32_t* out) {
  int32_t i = 0, j = 0, k = 0;
  while (i < na && j < nb) {
    if (a[i] == b[j]) { if (out) out[k] = a[i]; ++k; ++i; ++j; }
    else if (a[i] > b[j]) ++j;
    else ++i;
  }
  return k;
}

static void mbea_find(mbea_ctx* ctx, const int32_t* L, int32_t nL, const int32_t* R, int32_t nR,
                      const int32_t* C, int32_t nC, int32_t vc) {
  const ograph* g = ctx->g;
  ctx->r->nodes++;
  int32_t* Lp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nL > 0 ? nL : 1));
  int32_t nLp = isect(L, nL, g->adj + g->off[vc], g->off[vc + 1] - g->off[vc], Lp);
  if (nLp == 0) { free(Lp); return; }
  int32_t* Rp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nR + nC + 1));
  int32_t* Cp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nC + 1));
  int32_t nRp = nR, nCp = 0;
  memcpy(Rp, R, sizeof(int32_t) * (size_t)nR);
  for (int32_t k = 0; k < nC; ++k) {
    int32_t c = C[k];
    int32_t nc = isect(Lp, nLp, g->adj + g->off[c], g->off[c + 1] - g->off[c], NULL);
    if (nc == nLp) {
      if (c < vc) { ctx->r->non_maximal++; free(Lp); free(Rp); free(Cp); return; }
      Rp[nRp++] = c;
    } else if (nc != 0) {
      Cp[nCp++] = c;
    }
  }
  ctx->r->count++;
  uint64_t sU = 0, sV = 0;
  for (int32_t i = 0; i < nLp; ++i) sU += ikey_u(g, Lp[i]);
  for (int32_t i = 0; i < nRp; ++i) sV += ikey_v(g, Rp[i]);
  ctx->r->set_hash += ihash(g, sU, (uint64_t)nLp, sV, (uint64_t)nRp);
  for (int32_t k = 0; k < nCp; ++k)
    if (Cp[k] > vc) mbea_find(ctx, Lp, nLp, Rp, nRp, Cp, nCp, Cp[k]);
  free(Lp);
  free(Rp);
  free(Cp);
}

int orc_mbea(int32_t nV, int32_t nU, const int32_t* row_off, const int32_t* col, int32_t uvtrans,
             int32_t order, orc_result* out) {
  memset(out, 0, sizeof(*out));
  ograph g;
  ograph_build(nV, nU, row_off, col, uvtrans, order, &g);
  int32_t* L = (int32_t*)malloc(sizeof(int32_t) * (size_t)(g.nU > 0 ? g.nU : 1));
  int32_t* C = (int32_t*)malloc(sizeof(int32_t) * (size_t)(g.nV > 0 ? g.nV : 1));
  for (int32_t i = 0; i < g.nU; ++i) L[i] = i;
  for (int32_t i = 0; i < g.nV; ++i) C[i] = i;
  mbea_ctx ctx = {&g, out};
  for (int32_t i = 0; i < g.nV; ++i) mbea_find(&ctx, L, g.nU, NULL, 0, C, g.nV, C[i]);
  free(L);
  free(C);
  ograph_free(&g);
  return 0;
}

/* ------------------------------------------------------------------------ */
/* GMBE per-root restatement.                                                 */
#define B_FREE 0x7fff    /* candidate live at every level              */
#define B_TOUCHED 0x3fff /* marked by finder_pop's restore pass        */

typedef struct gws {
  int32_t* cnt;   /* [nV] neighbour count of a V vertex inside the root L */
  int32_t* posC;  /* [nV] index in C, or -1 */
  int32_t* touched;
  int32_t* Cv;    /* candidates (sorted internal V ids) */
  int32_t* ncnt;  /* |N(c) ∩ L_current| */
  int32_t* bound; /* level bound (reference: C_level_neighbors >> 16) */
  int32_t* Llevel;
  int32_t* stack;
  int32_t* aoff;  /* local adjacency: L position -> C positions */
  int32_t* aadj;
  size_t aadj_cap;
} gws;

typedef struct gacc {
  uint64_t count, hash, non_max, bytes, nodes;
} gacc;

static inline int64_t deg_u(const ograph* g, int32_t u) { return g->roff[u + 1] - g->roff[u]; }
static inline int64_t deg_v(const ograph* g, int32_t v) { return g->off[v + 1] - g->off[v]; }

static void gmbe_root(const ograph* g, int32_t v, int prune, gws* w, gacc* a, int64_t* stat) {
  const int32_t* L = g->adj + g->off[v];
  int32_t nL = g->off[v + 1] - g->off[v];
  if (nL == 0) return;
  int32_t nt = 0;
  uint64_t S = 0;
  for (int32_t l = 0; l < nL; ++l) {
    int32_t u = L[l];
    S += (uint64_t)deg_u(g, u);
    for (int32_t j = g->roff[u]; j < g->roff[u + 1]; ++j) {
      int32_t c = g->radj[j];
      if (w->cnt[c]++ == 0) w->touched[nt++] = c;
    }
  }
  /* maximality of the root: R[0] == v  (src/IterFinderGpu.cu:814-816) */
  int maximal = 1;
  for (int32_t k = 0; k < nt; ++k)
    if (w->cnt[w->touched[k]] == nL && w->touched[k] < v) { maximal = 0; break; }
  a->nodes++;
  if (!maximal) {
    a->non_max++;
    for (int32_t k = 0; k < nt; ++k) w->cnt[w->touched[k]] = 0;
    return;
  }
  qsort(w->touched, (size_t)nt, sizeof(int32_t), cmp_i32);
  uint64_t sRroot = 0, nRroot = 0, sL = 0;
  int32_t nC = 0;
  for (int32_t k = 0; k < nt; ++k) {
    int32_t c = w->touched[k];
    if (w->cnt[c] == nL) { sRroot += ikey_v(g, c); ++nRroot; }
    else { w->posC[c] = nC; w->Cv[nC] = c; w->ncnt[nC] = w->cnt[c]; w->bound[nC] = B_FREE; ++nC; }
  }
  for (int32_t l = 0; l < nL; ++l) sL += ikey_u(g, L[l]);
  a->count++;
  a->hash += ihash(g, sL, (uint64_t)nL, sRroot, nRroot);
  a->bytes += 4 * S + 4 * (uint64_t)nC;
  if (stat) { stat[0] = nL; stat[1] = nC; stat[2] = (int64_t)S; }
  uint64_t count0 = a->count, nodes0 = a->nodes;
  if (nL > 1 && nC > 0) {
    /* local adjacency L position -> C positions */
    uint64_t need = 0;
    for (int32_t l = 0; l < nL; ++l) need += (uint64_t)deg_u(g, L[l]);
    if (need > w->aadj_cap) {
      free(w->aadj);
      w->aadj_cap = need * 2;
      w->aadj = (int32_t*)malloc(sizeof(int32_t) * w->aadj_cap);
    }
    int32_t pos = 0;
    for (int32_t l = 0; l < nL; ++l) {
      w->aoff[l] = pos;
      int32_t u = L[l];
      for (int32_t j = g->roff[u]; j < g->roff[u + 1]; ++j) {
        int32_t p = w->posC[g->radj[j]];
        if (p >= 0) w->aadj[pos++] = p;
      }
      w->Llevel[l] = 0;
    }
    w->aoff[nL] = pos;
    /* next_id: first candidate after v in C (src/IterFinderGpu.cu:832-834) */
    int32_t next_id = 0;
    while (next_id < nC && w->Cv[next_id] < v) ++next_id;

    /* IterProcess (src/IterFinderGpu.cu:12-69) */
    int32_t level = 1;
    w->stack[0] = next_id;
    while (level != 0) {
      int32_t cur = -1;
      for (int32_t i = w->stack[level - 1]; i < nC; ++i)
        if (w->bound[i] > level - 1 && w->ncnt[i] != 0) { cur = i; break; }
      if (cur != -1) {
        /* ---- finder_push (src/IterFinderGpu.h:206-264) ---- */
        int32_t x = w->Cv[cur];
        const int32_t* Nx = g->adj + g->off[x];
        int32_t dx = g->off[x + 1] - g->off[x];
        int32_t kept = 0, removed = 0;
        uint64_t sLn = 0;
        for (int32_t l = 0; l < nL; ++l)
          if (w->Llevel[l] == level - 1) {
            if (bsearch_i32(Nx, dx, L[l]) >= 0) { w->Llevel[l] = level; ++kept; sLn += ikey_u(g, L[l]); }
            else ++removed;
          }
        int32_t nLp = kept + removed;
        /* recompute iff |L_parent| > 2 |L_new| (src/IterFinderGpu.h:230) */
        int recompute = nLp > 2 * kept;
        uint64_t dbytes = 0;
        if (recompute) {
          for (int32_t i = 0; i < nC; ++i) w->ncnt[i] = 0;
          for (int32_t l = 0; l < nL; ++l)
            if (w->Llevel[l] == level) {
              dbytes += (uint64_t)deg_u(g, L[l]);
              for (int32_t k = w->aoff[l]; k < w->aoff[l + 1]; ++k) w->ncnt[w->aadj[k]]++;
            }
        } else {
          for (int32_t l = 0; l < nL; ++l)
            if (w->Llevel[l] == level - 1) {
              dbytes += (uint64_t)deg_u(g, L[l]);
              for (int32_t k = w->aoff[l]; k < w->aoff[l + 1]; ++k) w->ncnt[w->aadj[k]]--;
            }
        }
        a->bytes += 4 * ((uint64_t)nLp + (uint64_t)dx) + 4 * dbytes + 4 * (uint64_t)nC;
        a->nodes++;
        int is_max = 1;
        uint64_t sRn = sRroot, nRn = nRroot;
        for (int32_t i = 0; i < nC; ++i)
          if (w->ncnt[i] == kept) {
            sRn += ikey_v(g, w->Cv[i]);
            ++nRn;
            if (i < cur && w->bound[i] >= level) is_max = 0;
            else if (w->bound[i] > level) w->bound[i] = level;
          }
        if (is_max) {
          a->count++;
          a->hash += ihash(g, sLn, (uint64_t)kept, sRn, nRn);
        } else {
          a->non_max++;
        }
        if (is_max && w->ncnt[cur] > 1) {
          w->stack[level - 1] = cur;
          w->stack[level] = cur + 1;
          ++level;
          continue;
        }
        w->stack[level - 1] = cur + 1;
      } else {
        --level;
        if (level == 0) break;
        cur = w->stack[level - 1];
        w->stack[level - 1] = cur + 1;
      }
      /* ---- finder_pop (src/IterFinderGpu.h:266-303) at `level` for `cur` ---- */
      uint64_t pbytes = 0;
      for (int32_t l = 0; l < nL; ++l) {
        if (w->Llevel[l] == level - 1) {
          pbytes += (uint64_t)deg_u(g, L[l]);
          for (int32_t k = w->aoff[l]; k < w->aoff[l + 1]; ++k) {
            int32_t p = w->aadj[k];
            w->ncnt[p]++;
            if (w->bound[p] >= level) w->bound[p] = B_TOUCHED;
          }
        } else if (w->Llevel[l] >= level) {
          w->Llevel[l] = level - 1;
        }
      }
      a->bytes += 4 * pbytes;
      if (prune) {
        for (int32_t i = 0; i < nC; ++i)
          if (w->bound[i] >= level)
            w->bound[i] = (w->bound[i] == B_TOUCHED || i == cur) ? B_FREE : level - 1;
      } else {
        w->bound[cur] = B_FREE;
      }
    }
  }
  if (stat) { stat[3] = (int64_t)(a->count - count0 + 1); stat[4] = (int64_t)(a->nodes - nodes0 + 1); }
  for (int32_t k = 0; k < nt; ++k) { w->cnt[w->touched[k]] = 0; w->posC[w->touched[k]] = -1; }
}

/* Enumerate the roots [root_begin, root_end) of the internal order (the
 * reference claims roots from V_size-1 downwards; the set of bicliques does
 * not depend on the order).  root_end <= 0 means all roots.  stats, if not
 * NULL, receives 5 int64 per internal root: |L|, |C|, sum of d(u) over L,
 * bicliques found under the root, pushes under the root. */
int orc_gmbe_range(int32_t nV, int32_t nU, const int32_t* row_off, const int32_t* col,
                   int32_t uvtrans, int32_t order, int32_t prune, int32_t threads,
                   int64_t root_begin, int64_t root_end, int64_t* stats, orc_result* out) {
  memset(out, 0, sizeof(*out));
  ograph g;
  ograph_build(nV, nU, row_off, col, uvtrans, order, &g);
  if (root_end <= 0 || root_end > g.nV) root_end = g.nV;
  if (root_begin < 0) root_begin = 0;
  int32_t maxdv = 0;
  for (int32_t v = 0; v < g.nV; ++v) if (deg_v(&g, v) > maxdv) maxdv = (int32_t)deg_v(&g, v);
  if (threads <= 0) threads = omp_get_max_threads();
  uint64_t cnt = 0, hash = 0, nonmax = 0, bytes = 0, nodes = 0;
  if (stats) memset(stats, 0, sizeof(int64_t) * 5 * (size_t)g.nV);
#pragma omp parallel num_threads(threads) reduction(+ : cnt, hash, nonmax, bytes, nodes)
  {
    gws w;
    size_t nv = (size_t)(g.nV > 0 ? g.nV : 1);
    w.cnt = (int32_t*)calloc(nv, sizeof(int32_t));
    w.posC = (int32_t*)malloc(nv * sizeof(int32_t));
    for (size_t i = 0; i < nv; ++i) w.posC[i] = -1;
    w.touched = (int32_t*)malloc(nv * sizeof(int32_t));
    w.Cv = (int32_t*)malloc(nv * sizeof(int32_t));
    w.ncnt = (int32_t*)malloc(nv * sizeof(int32_t));
    w.bound = (int32_t*)malloc(nv * sizeof(int32_t));
    w.stack = (int32_t*)malloc((nv + 2) * sizeof(int32_t));
    w.Llevel = (int32_t*)malloc(((size_t)maxdv + 1) * sizeof(int32_t));
    w.aoff = (int32_t*)malloc(((size_t)maxdv + 2) * sizeof(int32_t));
    w.aadj_cap = 1 << 16;
    w.aadj = (int32_t*)malloc(w.aadj_cap * sizeof(int32_t));
    gacc a = {0, 0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
    for (int64_t k = root_end - 1; k >= root_begin; --k) {
      gmbe_root(&g, (int32_t)k, prune, &w, &a, stats ? stats + 5 * k : NULL);
    }
    cnt += a.count;
    hash += a.hash;
    nonmax += a.non_max;
    bytes += a.bytes;
    nodes += a.nodes;
    free(w.cnt); free(w.posC); free(w.touched); free(w.Cv); free(w.ncnt); free(w.bound);
    free(w.stack); free(w.Llevel); free(w.aoff); free(w.aadj);
  }
  out->count = cnt;
  out->set_hash = hash;
  out->non_maximal = nonmax;
  out->alg_bytes = bytes;
  out->nodes = nodes;
  ograph_free(&g);
  return 0;
}

/* Stratified sample: roots at positions p = offset, offset+stride, ... counted
 * from the top of the internal order (the reference claims roots from
 * V_size-1 downwards, src/IterFinderGpu.cu:1008).  Used to time a bounded
 * share of a workload whose degree-sorted roots vary widely in cost. */
int orc_gmbe_strided(int32_t nV, int32_t nU, const int32_t* row_off, const int32_t* col,
                     int32_t uvtrans, int32_t order, int32_t prune, int32_t threads,
                     int64_t offset, int64_t stride, orc_result* out) {
  memset(out, 0, sizeof(*out));
  if (stride < 1 || offset < 0) return -1;
  ograph g;
  ograph_build(nV, nU, row_off, col, uvtrans, order, &g);
  int32_t maxdv = 0;
  for (int32_t v = 0; v < g.nV; ++v) if (deg_v(&g, v) > maxdv) maxdv = (int32_t)deg_v(&g, v);
  if (threads <= 0) threads = omp_get_max_threads();
  int64_t n = g.nV > offset ? (g.nV - offset + stride - 1) / stride : 0;
  uint64_t cnt = 0, hash = 0, nonmax = 0, bytes = 0, nodes = 0;
#pragma omp parallel num_threads(threads) reduction(+ : cnt, hash, nonmax, bytes, nodes)
  {
    gws w;
    size_t nv = (size_t)(g.nV > 0 ? g.nV : 1);
    w.cnt = (int32_t*)calloc(nv, sizeof(int32_t));
    w.posC = (int32_t*)malloc(nv * sizeof(int32_t));
    for (size_t i = 0; i < nv; ++i) w.posC[i] = -1;
    w.touched = (int32_t*)malloc(nv * sizeof(int32_t));
    w.Cv = (int32_t*)malloc(nv * sizeof(int32_t));
    w.ncnt = (int32_t*)malloc(nv * sizeof(int32_t));
    w.bound = (int32_t*)malloc(nv * sizeof(int32_t));
    w.stack = (int32_t*)malloc((nv + 2) * sizeof(int32_t));
    w.Llevel = (int32_t*)malloc(((size_t)maxdv + 1) * sizeof(int32_t));
    w.aoff = (int32_t*)malloc(((size_t)maxdv + 2) * sizeof(int32_t));
    w.aadj_cap = 1 << 16;
    w.aadj = (int32_t*)malloc(w.aadj_cap * sizeof(int32_t));
    gacc a = {0, 0, 0, 0, 0};
#pragma omp for schedule(dynamic, 1)
    for (int64_t k = 0; k < n; ++k) gmbe_root(&g, (int32_t)(g.nV - 1 - (offset + k * stride)), prune, &w, &a, NULL);
    cnt += a.count;
    hash += a.hash;
    nonmax += a.non_max;
    bytes += a.bytes;
    nodes += a.nodes;
    free(w.cnt); free(w.posC); free(w.touched); free(w.Cv); free(w.ncnt); free(w.bound);
    free(w.stack); free(w.Llevel); free(w.aoff); free(w.aadj);
  }
  out->count = cnt;
  out->set_hash = hash;
  out->non_maximal = nonmax;
  out->alg_bytes = bytes;
  out->nodes = nodes;
  ograph_free(&g);
  return 0;
}

int orc_gmbe(int32_t nV, int32_t nU, const int32_t* row_off, const int32_t* col, int32_t uvtrans,
             int32_t order, int32_t prune, int32_t threads, orc_result* out) {
  return orc_gmbe_range(nV, nU, row_off, col, uvtrans, order, prune, threads, 0, 0, NULL, out);
}

/* Internal-order permutation used by the oracle (for tests that compare
 * per-root behaviour): v_orig[i] = original id of internal root i. */
int orc_internal_order(int32_t nV, int32_t nU, const int32_t* row_off, const int32_t* col,
                       int32_t uvtrans, int32_t order, int32_t* v_orig_out, int32_t* nV_out) {
  ograph g;
  ograph_build(nV, nU, row_off, col, uvtrans, order, &g);
  memcpy(v_orig_out, g.v_orig, sizeof(int32_t) * (size_t)g.nV);
  *nV_out = g.nV;
  ograph_free(&g);
  return 0;
}
