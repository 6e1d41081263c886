/*
 * wtivo_oracle.c -- CPU oracle for the WTiVo graph-cut hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  See
 * wtivo_oracle.h for what each function restates and where.
 *
 * Build with strict IEEE double semantics (no FMA contraction, no fast
 * math): the capacity formula must round exactly like the reference's host
 * code (x86-64 SSE2 doubles, /fp:precise).
 */
#include "wtivo_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_INF_H 0xFFFFFFFFu

/* Face slot fi of a tet uses local vertices LUT[fi]; the neighbor in slot fi
 * is the tet opposite local vertex 3-fi (bindings.cpp:70,
 * native/core/wtivo_core.cpp:138). */
static const int FACE_LUT[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
static const int FACE_OPP[4] = {3, 2, 1, 0};

/* ------------------------------------------------------------------------ */
/* Capacity formula: bindings.cpp:65-98.                                     */
/* ------------------------------------------------------------------------ */
int orc_capacity(const double* V, uint64_t nv, const int32_t* tr, int fi,
                 uint8_t li, uint8_t lj, double fill_T, int32_t* cap)
{
    const int32_t a = tr[FACE_LUT[fi][0]];
    const int32_t b = tr[FACE_LUT[fi][1]];
    const int32_t c = tr[FACE_LUT[fi][2]];
    if (a < 0 || b < 0 || c < 0 || (uint64_t)a >= nv || (uint64_t)b >= nv ||
        (uint64_t)c >= nv)
        return ORC_ERR_BUILD;
    const double* p0 = V + (size_t)a * 3u;
    const double* p1 = V + (size_t)b * 3u;
    const double* p2 = V + (size_t)c * 3u;
    const double x1 = p1[0] - p0[0], y1 = p1[1] - p0[1], z1 = p1[2] - p0[2];
    const double x2 = p2[0] - p0[0], y2 = p2[1] - p0[1], z2 = p2[2] - p0[2];
    const double cx = y1 * z2 - z1 * y2;
    const double cy = z1 * x2 - x1 * z2;
    const double cz = x1 * y2 - y1 * x2;
    /* float(1e7 * 0.5 * |cross|): the constant product folds to 5e6. */
    const double s = sqrt(cx * cx + cy * cy + cz * cz);
    const float area_f = (float)(5.0e6 * s);
    const double area = (double)area_f;
    const double pen = (li != lj) ? area : area * (1.0 + fill_T);
    /* int64 truncation toward zero, then the [0, 2^30) check: values in
     * (-1, 0) truncate to 0 and pass; NaN/inf convert to INT64_MIN on x86-64
     * and fail, as does anything outside (-1, 2^30). */
    if (!(pen > -1.0 && pen < 1073741824.0)) return ORC_ERR_BUILD;
    const int64_t cap64 = (int64_t)pen;
    if (cap64 < 0 || cap64 >= 1073741824LL) return ORC_ERR_BUILD;
    *cap = (int32_t)cap64;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Classification + compaction: bindings.cpp:146-188.                        */
/* ------------------------------------------------------------------------ */
int orc_classify(const int32_t* nbrs, const uint8_t* labels, uint64_t N,
                 int32_t* full_to_free, uint32_t* free_old,
                 orc_build_info* info)
{
    memset(info, 0, sizeof(*info));
    info->n_full = N;
    if (N > 0xFFFFFFFFull) return ORC_ERR_ARG;
    uint64_t refs = 0;
    for (uint64_t i = 0; i < N; ++i) {
        int exterior = 0;
        for (int fi = 0; fi < 4; ++fi) {
            const int32_t j = nbrs[i * 4u + (uint64_t)fi];
            if (j < 0) exterior = 1;
            else {
                ++refs;
                if ((uint64_t)j >= N) return ORC_ERR_NBR_RANGE;
            }
        }
        if (labels[i] == 0u) { full_to_free[i] = -2; ++info->fixed_source; }
        else if (exterior) { full_to_free[i] = -3; ++info->fixed_sink; }
        else full_to_free[i] = -1;
    }
    info->full_refs = refs;
    if (refs & 1u) return ORC_ERR_REFS_ODD;
    uint64_t rid = 0;
    for (uint64_t i = 0; i < N; ++i) {
        if (full_to_free[i] == -1) {
            if (rid > 0x7FFFFFFFull) return ORC_ERR_TOO_MANY;
            full_to_free[i] = (int32_t)rid;
            free_old[rid] = (uint32_t)i;
            ++rid;
        }
    }
    info->free_n = rid;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Reduced ELL graph + t-links: bindings.cpp:227-314.                        */
/* ------------------------------------------------------------------------ */
int orc_build(const double* V, uint64_t nv, const int32_t* tets,
              const int32_t* nbrs, const uint8_t* labels, uint64_t N,
              double fill_T, const int32_t* full_to_free,
              orc_build_info* info, int32_t* nbr, uint32_t* res,
              int32_t* term)
{
    uint64_t free_refs = 0, terms = 0;
    int64_t base = 0;
    for (uint64_t i = 0; i < N; ++i) {
        const int32_t rr = full_to_free[i];
        if (rr < 0) continue;
        const uint64_t q = (uint64_t)rr;
        int64_t src = 0, snk = 0;
        for (int fi = 0; fi < 4; ++fi) {
            nbr[q * 4u + (uint64_t)fi] = -1;
            res[q * 4u + (uint64_t)fi] = 0u;
        }
        for (int fi = 0; fi < 4; ++fi) {
            const int32_t jj = nbrs[i * 4u + (uint64_t)fi];
            if (jj < 0 || (uint64_t)jj >= N) return ORC_ERR_BUILD;
            const int32_t m = full_to_free[jj];
            int32_t cap = 0;
            if (orc_capacity(V, nv, tets + i * 4u, fi, labels[i], labels[jj],
                             fill_T, &cap) != ORC_OK)
                return ORC_ERR_BUILD;
            if (m >= 0) {
                nbr[q * 4u + (uint64_t)fi] = m;
                res[q * 4u + (uint64_t)fi] = (uint32_t)cap;
                ++free_refs;
            } else if (m == -2) { src += cap; ++terms; }
            else if (m == -3) { snk += cap; ++terms; }
            else return ORC_ERR_BUILD;
        }
        base += (src < snk) ? src : snk;
        const int64_t diff = src - snk;
        if (diff < -2147483648LL || diff > 2147483647LL) return ORC_ERR_BUILD;
        term[q] = (int32_t)diff;
    }
    info->free_refs = free_refs;
    info->terminal_edges = terms;
    info->terminal_base_flow = base;
    if (free_refs & 1u) return ORC_ERR_FREE_REFS_ODD;
    return ORC_OK;
}

/* Slot of u in v's row (the reference searches it per push:
 * gpu_push_relabel_fast.cu:56-67). */
static int find_slot(const int32_t* nbr, uint32_t v, uint32_t u)
{
    for (int k = 0; k < 4; ++k)
        if (nbr[(uint64_t)v * 4u + (uint64_t)k] == (int32_t)u) return k;
    return -1;
}

int orc_reverse_slots(uint32_t F, const int32_t* nbr, uint8_t* rev)
{
    for (uint32_t v = 0; v < F; ++v) {
        for (int k = 0; k < 4; ++k) {
            const int32_t u = nbr[(uint64_t)v * 4u + (uint64_t)k];
            if (u < 0) { rev[(uint64_t)v * 4u + (uint64_t)k] = 255u; continue; }
            if ((uint32_t)u >= F) return ORC_ERR_ARG;
            const int rk = find_slot(nbr, (uint32_t)u, v);
            if (rk < 0) return ORC_ERR_NO_REVERSE;
            rev[(uint64_t)v * 4u + (uint64_t)k] = (uint8_t)rk;
        }
    }
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Sink-reachable set: the final residual BFS (.cu:551-562, :315-324).       */
/* ------------------------------------------------------------------------ */
int orc_sink_reachable(uint32_t F, const int32_t* nbr, const uint32_t* res,
                       const int32_t* term, uint8_t* partition)
{
    uint8_t* rev = (uint8_t*)malloc((size_t)F * 4u + 1u);
    uint32_t* queue = (uint32_t*)malloc((size_t)F * sizeof(uint32_t) + 4u);
    if (!rev || !queue) { free(rev); free(queue); return ORC_ERR_NO_MEM; }
    int rc = orc_reverse_slots(F, nbr, rev);
    if (rc != ORC_OK) { free(rev); free(queue); return rc; }
    uint64_t head = 0, tail = 0;
    for (uint32_t v = 0; v < F; ++v) {
        partition[v] = (term[v] < 0) ? 1u : 0u;
        if (partition[v]) queue[tail++] = v;
    }
    while (head < tail) {
        const uint32_t u = queue[head++];
        for (int k = 0; k < 4; ++k) {
            const int32_t v = nbr[(uint64_t)u * 4u + (uint64_t)k];
            if (v < 0 || partition[v]) continue;
            const uint8_t rk = rev[(uint64_t)u * 4u + (uint64_t)k];
            if (res[(uint64_t)v * 4u + rk] == 0u) continue; /* arc v->u */
            partition[v] = 1u;
            queue[tail++] = (uint32_t)v;
        }
    }
    free(rev);
    free(queue);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Boykov-Kolmogorov max flow on the ELL graph.                              */
/* Arcs are slots a = 4v+k; sister(a) is the reverse slot in the neighbor's  */
/* row.  Tree parents store the arc from a node toward its parent.           */
/* ------------------------------------------------------------------------ */
#define BK_NONE (-1)
#define BK_TERMINAL (-2)
#define BK_ORPHAN (-3)
#define BK_INF_D 0x7FFFFFFF

typedef struct {
    uint32_t F;
    const int32_t* head;   /* nbr */
    uint32_t* rc;          /* residual per arc */
    int64_t* tr;           /* + : source residual, - : sink residual */
    int64_t* sister;
    int64_t* parent;
    uint8_t* is_sink;
    uint8_t* inq;
    int64_t* ts;
    int32_t* dist;
    uint32_t* aq;          /* active FIFO (ring) */
    uint64_t aq_head, aq_count;
    uint32_t* orph;        /* orphan FIFO (ring) */
    uint64_t or_head, or_count;
    int64_t time;
} bk_state;

static void bk_set_active(bk_state* s, uint32_t i)
{
    if (s->inq[i]) return;
    s->inq[i] = 1u;
    s->aq[(s->aq_head + s->aq_count) % ((uint64_t)s->F + 1u)] = i;
    ++s->aq_count;
}

static int64_t bk_next_active(bk_state* s)
{
    while (s->aq_count) {
        const uint32_t i = s->aq[s->aq_head];
        s->aq_head = (s->aq_head + 1u) % ((uint64_t)s->F + 1u);
        --s->aq_count;
        s->inq[i] = 0u;
        if (s->parent[i] != BK_NONE) return (int64_t)i;
    }
    return -1;
}

static void bk_set_orphan(bk_state* s, uint32_t i)
{
    s->parent[i] = BK_ORPHAN;
    s->orph[(s->or_head + s->or_count) % ((uint64_t)s->F + 1u)] = i;
    ++s->or_count;
}

static void bk_augment(bk_state* s, int64_t middle, int64_t* flow)
{
    const int32_t* head = s->head;
    /* tail of middle = head of its sister */
    const uint32_t tail = (uint32_t)head[s->sister[middle]];
    int64_t b = s->rc[middle];
    uint32_t i = tail;
    while (s->parent[i] != BK_TERMINAL) {
        const int64_t pa = s->parent[i];
        const int64_t c = s->rc[s->sister[pa]];
        if (c < b) b = c;
        i = (uint32_t)head[pa];
    }
    if (s->tr[i] < b) b = s->tr[i];
    i = (uint32_t)head[middle];
    while (s->parent[i] != BK_TERMINAL) {
        const int64_t pa = s->parent[i];
        const int64_t c = s->rc[pa];
        if (c < b) b = c;
        i = (uint32_t)head[pa];
    }
    if (-s->tr[i] < b) b = -s->tr[i];

    s->rc[s->sister[middle]] += (uint32_t)b;
    s->rc[middle] -= (uint32_t)b;
    i = tail;
    while (s->parent[i] != BK_TERMINAL) {
        const int64_t pa = s->parent[i];
        s->rc[pa] += (uint32_t)b;
        s->rc[s->sister[pa]] -= (uint32_t)b;
        const uint32_t up = (uint32_t)head[pa];
        if (s->rc[s->sister[pa]] == 0u) bk_set_orphan(s, i);
        i = up;
    }
    s->tr[i] -= b;
    if (s->tr[i] == 0) bk_set_orphan(s, i);
    i = (uint32_t)head[middle];
    while (s->parent[i] != BK_TERMINAL) {
        const int64_t pa = s->parent[i];
        s->rc[s->sister[pa]] += (uint32_t)b;
        s->rc[pa] -= (uint32_t)b;
        const uint32_t up = (uint32_t)head[pa];
        if (s->rc[pa] == 0u) bk_set_orphan(s, i);
        i = up;
    }
    s->tr[i] += b;
    if (s->tr[i] == 0) bk_set_orphan(s, i);
    *flow += b;
}

/* Distance from j to its tree root, or BK_INF_D if the path reaches an
 * orphan; marks the path with the current time stamp. */
static int32_t bk_origin(bk_state* s, uint32_t j)
{
    int64_t d = 0;
    uint32_t jj = j;
    for (;;) {
        if (s->ts[jj] == s->time) { d += s->dist[jj]; break; }
        const int64_t a = s->parent[jj];
        ++d;
        if (a == BK_TERMINAL) { s->ts[jj] = s->time; s->dist[jj] = 1; break; }
        if (a == BK_ORPHAN) return BK_INF_D;
        jj = (uint32_t)s->head[a];
    }
    int64_t dd = d;
    for (jj = j; s->ts[jj] != s->time; jj = (uint32_t)s->head[s->parent[jj]]) {
        s->ts[jj] = s->time;
        s->dist[jj] = (int32_t)dd--;
    }
    return (int32_t)d;
}

static void bk_process_orphan(bk_state* s, uint32_t i)
{
    const int sink = s->is_sink[i];
    int64_t best = BK_NONE;
    int32_t dmin = BK_INF_D;
    for (int k = 0; k < 4; ++k) {
        const int64_t a0 = (int64_t)i * 4 + k;
        const int32_t j = s->head[a0];
        if (j < 0) continue;
        /* source tree: need residual j->i (sister); sink tree: i->j (a0) */
        const uint32_t c = sink ? s->rc[a0] : s->rc[s->sister[a0]];
        if (c == 0u) continue;
        if (s->parent[j] == BK_NONE || s->is_sink[j] != sink) continue;
        const int32_t d = bk_origin(s, (uint32_t)j);
        if (d < dmin) { dmin = d; best = a0; }
    }
    if (best != BK_NONE) {
        s->parent[i] = best;
        s->ts[i] = s->time;
        s->dist[i] = dmin + 1;
        return;
    }
    s->parent[i] = BK_NONE;
    for (int k = 0; k < 4; ++k) {
        const int64_t a0 = (int64_t)i * 4 + k;
        const int32_t j = s->head[a0];
        if (j < 0) continue;
        if (s->parent[j] == BK_NONE || s->is_sink[j] != sink) continue;
        const uint32_t c = sink ? s->rc[a0] : s->rc[s->sister[a0]];
        if (c) bk_set_active(s, (uint32_t)j);
        const int64_t pa = s->parent[j];
        if (pa != BK_TERMINAL && pa != BK_ORPHAN && s->head[pa] == (int32_t)i)
            bk_set_orphan(s, (uint32_t)j);
    }
}

int orc_maxflow_bk(uint32_t F, const int32_t* nbr, uint32_t* res,
                   int32_t* term, int64_t* raw_flow, uint8_t* partition)
{
    *raw_flow = 0;
    if (F == 0) return ORC_OK;
    bk_state s;
    memset(&s, 0, sizeof(s));
    s.F = F;
    s.head = nbr;
    s.rc = res;
    const size_t A = (size_t)F * 4u;
    uint8_t* rev = (uint8_t*)malloc(A);
    s.tr = (int64_t*)malloc((size_t)F * sizeof(int64_t));
    s.sister = (int64_t*)malloc(A * sizeof(int64_t));
    s.parent = (int64_t*)malloc((size_t)F * sizeof(int64_t));
    s.is_sink = (uint8_t*)calloc(F, 1);
    s.inq = (uint8_t*)calloc(F, 1);
    s.ts = (int64_t*)calloc(F, sizeof(int64_t));
    s.dist = (int32_t*)calloc(F, sizeof(int32_t));
    s.aq = (uint32_t*)malloc(((size_t)F + 1u) * sizeof(uint32_t));
    s.orph = (uint32_t*)malloc(((size_t)F + 1u) * sizeof(uint32_t));
    int rc = ORC_OK;
    if (!rev || !s.tr || !s.sister || !s.parent || !s.is_sink || !s.inq ||
        !s.ts || !s.dist || !s.aq || !s.orph) { rc = ORC_ERR_NO_MEM; goto done; }
    rc = orc_reverse_slots(F, nbr, rev);
    if (rc != ORC_OK) goto done;
    for (size_t a = 0; a < A; ++a)
        s.sister[a] = (nbr[a] < 0) ? -1 : (int64_t)nbr[a] * 4 + rev[a];

    for (uint32_t i = 0; i < F; ++i) {
        s.tr[i] = term[i];
        if (term[i] > 0) { s.parent[i] = BK_TERMINAL; s.is_sink[i] = 0; s.dist[i] = 1; bk_set_active(&s, i); }
        else if (term[i] < 0) { s.parent[i] = BK_TERMINAL; s.is_sink[i] = 1; s.dist[i] = 1; bk_set_active(&s, i); }
        else s.parent[i] = BK_NONE;
    }

    int64_t flow = 0;
    int64_t current = -1;
    for (;;) {
        int64_t i = current;
        if (i >= 0) {
            s.inq[i] = 0u;
            if (s.parent[i] == BK_NONE) i = -1;
        }
        if (i < 0) {
            i = bk_next_active(&s);
            if (i < 0) break;
        }
        const uint32_t u = (uint32_t)i;
        int64_t middle = -1;
        if (!s.is_sink[u]) {
            for (int k = 0; k < 4; ++k) {
                const int64_t a = (int64_t)u * 4 + k;
                const int32_t j = nbr[a];
                if (j < 0 || s.rc[a] == 0u) continue;
                if (s.parent[j] == BK_NONE) {
                    s.is_sink[j] = 0; s.parent[j] = s.sister[a];
                    s.ts[j] = s.ts[u]; s.dist[j] = s.dist[u] + 1;
                    bk_set_active(&s, (uint32_t)j);
                } else if (s.is_sink[j]) { middle = a; break; }
                else if (s.ts[j] <= s.ts[u] && s.dist[j] > s.dist[u]) {
                    s.parent[j] = s.sister[a];
                    s.ts[j] = s.ts[u]; s.dist[j] = s.dist[u] + 1;
                }
            }
        } else {
            for (int k = 0; k < 4; ++k) {
                const int64_t a = (int64_t)u * 4 + k;
                const int32_t j = nbr[a];
                if (j < 0) continue;
                const int64_t sa = s.sister[a];
                if (s.rc[sa] == 0u) continue;
                if (s.parent[j] == BK_NONE) {
                    s.is_sink[j] = 1; s.parent[j] = sa;
                    s.ts[j] = s.ts[u]; s.dist[j] = s.dist[u] + 1;
                    bk_set_active(&s, (uint32_t)j);
                } else if (!s.is_sink[j]) { middle = sa; break; }
                else if (s.ts[j] <= s.ts[u] && s.dist[j] > s.dist[u]) {
                    s.parent[j] = sa;
                    s.ts[j] = s.ts[u]; s.dist[j] = s.dist[u] + 1;
                }
            }
        }
        ++s.time;
        if (middle >= 0) {
            s.inq[u] = 1u; /* keep u out of the queue while it is current */
            current = (int64_t)u;
            bk_augment(&s, middle, &flow);
            while (s.or_count) {
                const uint32_t o = s.orph[s.or_head];
                s.or_head = (s.or_head + 1u) % ((uint64_t)F + 1u);
                --s.or_count;
                bk_process_orphan(&s, o);
            }
        } else {
            current = -1;
        }
    }
    for (uint32_t i = 0; i < F; ++i) term[i] = (int32_t)s.tr[i];
    *raw_flow = flow;
    if (partition) rc = orc_sink_reachable(F, nbr, res, term, partition);
done:
    free(rev); free(s.tr); free(s.sister); free(s.parent); free(s.is_sink);
    free(s.inq); free(s.ts); free(s.dist); free(s.aq); free(s.orph);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Sequential Phase-I push-relabel with the reference's rules.              */
/* ------------------------------------------------------------------------ */
/* Exact backward BFS distances to the sink (.cu:360-402); unreached nodes
 * get inf_h (.cu:141-147). */
static void pr_global_relabel(uint32_t F, const int32_t* nbr, const uint8_t* rev,
                              const uint32_t* res, const int32_t* term,
                              uint32_t* h, uint32_t* queue)
{
    const uint32_t inf_h = F + 1u;
    uint64_t head = 0, tail = 0;
    for (uint32_t v = 0; v < F; ++v) {
        h[v] = ORC_INF_H;
        if (term[v] < 0) { h[v] = 1u; queue[tail++] = v; }
    }
    while (head < tail) {
        const uint32_t u = queue[head++];
        for (int k = 0; k < 4; ++k) {
            const int32_t v = nbr[(uint64_t)u * 4u + (uint64_t)k];
            if (v < 0 || h[v] != ORC_INF_H) continue;
            const uint8_t rk = rev[(uint64_t)u * 4u + (uint64_t)k];
            if (res[(uint64_t)v * 4u + rk] == 0u) continue;
            h[v] = h[u] + 1u;
            queue[tail++] = (uint32_t)v;
        }
    }
    for (uint32_t v = 0; v < F; ++v) if (h[v] == ORC_INF_H) h[v] = inf_h;
}

int orc_maxflow_pr(uint32_t F, const int32_t* nbr, uint32_t* res,
                   int32_t* term, int64_t* excess, int local_steps,
                   int global_relabel_period, uint64_t max_rounds,
                   int64_t* raw_flow, uint8_t* partition,
                   uint64_t* rounds_out, uint64_t* relabels_out)
{
    *raw_flow = 0;
    if (rounds_out) *rounds_out = 0;
    if (relabels_out) *relabels_out = 0;
    if (F == 0) return ORC_OK;
    if (local_steps < 1) local_steps = 1;          /* .cu:421-422 */
    if (local_steps > 32) local_steps = 32;
    if (global_relabel_period < 0) global_relabel_period = 0;
    if (!max_rounds) max_rounds = 2000000ull;
    const uint32_t source_h = F, inf_h = F + 1u;
    uint64_t rounds = 0, relabels = 0, flow = 0;
    uint8_t* rev = (uint8_t*)malloc((size_t)F * 4u);
    uint32_t* h = (uint32_t*)malloc((size_t)F * 4u);
    uint32_t* cur = (uint32_t*)malloc((size_t)F * 4u);
    uint32_t* nxt = (uint32_t*)malloc((size_t)F * 4u);
    uint8_t* queued = (uint8_t*)calloc(F, 1);
    int rc = ORC_OK;
    if (!rev || !h || !cur || !nxt || !queued) { rc = ORC_ERR_NO_MEM; goto done; }
    rc = orc_reverse_slots(F, nbr, rev);
    if (rc != ORC_OK) goto done;

    for (uint32_t v = 0; v < F; ++v) excess[v] = term[v] > 0 ? term[v] : 0;
    int macro_period = 0;
    if (global_relabel_period > 0) {
        macro_period = (global_relabel_period + local_steps - 1) / local_steps;
        if (macro_period < 1) macro_period = 1;
    }
    uint64_t ncur = 0;
    for (;;) {
        /* exact relabel, then rebuild the active set (.cu:149-166) */
        pr_global_relabel(F, nbr, rev, res, term, h, cur);
        ++relabels;
        ncur = 0;
        memset(queued, 0, F);
        for (uint32_t v = 0; v < F; ++v)
            if (excess[v] > 0 && h[v] < source_h) { queued[v] = 1u; cur[ncur++] = v; }
        if (!ncur) break; /* maximum preflow: no excess can reach the sink */
        int since = 0;
        while (ncur) {
            if (rounds >= max_rounds) { rc = ORC_ERR_MAX_ROUNDS; goto done; }
            uint64_t nnext = 0;
            for (uint64_t qi = 0; qi < ncur; ++qi) {
                const uint32_t v = cur[qi];
                queued[v] = 0u;
                const uint64_t vb = (uint64_t)v * 4u;
                for (int step = 0; step < local_steps; ++step) {
                    int64_t ex = excess[v];
                    if (ex <= 0) break;
                    const uint32_t hv = h[v];
                    if (hv >= source_h) break;
                    int32_t tv = term[v];
                    if (tv < 0 && hv == 1u) {                /* .cu:220-236 */
                        const int64_t cap = -(int64_t)tv;
                        const int64_t d = ex < cap ? ex : cap;
                        term[v] = (int32_t)(tv + d);
                        excess[v] -= d;
                        flow += (uint64_t)d;
                        ex -= d;
                    }
                    for (int k = 0; k < 4 && ex > 0; ++k) {  /* .cu:238-269 */
                        const int32_t u = nbr[vb + (uint64_t)k];
                        if (u < 0) continue;
                        if (hv != h[u] + 1u) continue;
                        const uint32_t r = res[vb + (uint64_t)k];
                        if (!r) continue;
                        const int64_t d = ex < (int64_t)r ? ex : (int64_t)r;
                        res[vb + (uint64_t)k] -= (uint32_t)d;
                        res[(uint64_t)u * 4u + rev[vb + (uint64_t)k]] += (uint32_t)d;
                        excess[v] -= d;
                        const int64_t old_u = excess[u];
                        excess[u] += d;
                        ex -= d;
                        if (old_u == 0 && !queued[u]) { queued[u] = 1u; nxt[nnext++] = (uint32_t)u; }
                    }
                    ex = excess[v];
                    if (ex <= 0) break;
                    uint32_t min_h = ORC_INF_H;                /* .cu:274-289 */
                    tv = term[v];
                    if (tv < 0) min_h = 0u;
                    if (tv > 0 && source_h < min_h) min_h = source_h;
                    for (int k = 0; k < 4; ++k) {
                        const int32_t u = nbr[vb + (uint64_t)k];
                        if (u < 0 || res[vb + (uint64_t)k] == 0u) continue;
                        if (h[u] < min_h) min_h = h[u];
                    }
                    if (min_h == ORC_INF_H) { rc = ORC_ERR_INVARIANT; goto done; }
                    const uint32_t new_h = min_h + 1u;
                    if (new_h > hv) { h[v] = new_h; continue; }
                    break;
                }
                if (excess[v] > 0 && h[v] < source_h && !queued[v]) {
                    queued[v] = 1u;
                    nxt[nnext++] = v;
                }
            }
            ++rounds;
            uint32_t* t = cur; cur = nxt; nxt = t;
            ncur = nnext;
            ++since;
            if (macro_period > 0 && ncur && since >= macro_period) break;
        }
        (void)inf_h;
    }
    *raw_flow = (int64_t)flow;
    /* final residual BFS + partition (.cu:551-562) */
    for (uint32_t v = 0; v < F; ++v) partition[v] = (h[v] < inf_h) ? 1u : 0u;
done:
    if (rounds_out) *rounds_out = rounds;
    if (relabels_out) *relabels_out = relabels;
    free(rev); free(h); free(cur); free(nxt); free(queued);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Whole graph_cut_fast path (bindings.cpp:100-397).                         */
/* ------------------------------------------------------------------------ */
int orc_graph_cut(const double* V, uint64_t nv, const int32_t* tets,
                  const int32_t* nbrs, const uint8_t* labels, uint64_t N,
                  double fill_T, int solver, uint8_t* out_labels,
                  int64_t* stats)
{
    orc_build_info info;
    int32_t* f2f = (int32_t*)malloc((size_t)N * 4u + 4u);
    uint32_t* old = (uint32_t*)malloc((size_t)N * 4u + 4u);
    int32_t* nbr = NULL; uint32_t* res = NULL; int32_t* term = NULL;
    int64_t* excess = NULL; uint8_t* part = NULL;
    int rc;
    memset(stats, 0, 8 * sizeof(int64_t));
    if (!f2f || !old) { rc = ORC_ERR_NO_MEM; goto done; }
    rc = orc_classify(nbrs, labels, N, f2f, old, &info);
    if (rc != ORC_OK) goto done;
    memcpy(out_labels, labels, (size_t)N);
    stats[2] = (int64_t)(info.full_refs / 2u);
    stats[4] = (int64_t)info.fixed_source;
    stats[5] = (int64_t)info.fixed_sink;
    if (info.free_n == 0) goto done;
    {
        const size_t F = (size_t)info.free_n;
        nbr = (int32_t*)malloc(F * 16u);
        res = (uint32_t*)malloc(F * 16u);
        term = (int32_t*)malloc(F * 4u);
        excess = (int64_t*)malloc(F * 8u);
        part = (uint8_t*)malloc(F);
        if (!nbr || !res || !term || !excess || !part) { rc = ORC_ERR_NO_MEM; goto done; }
        rc = orc_build(V, nv, tets, nbrs, labels, N, fill_T, f2f, &info, nbr, res, term);
        if (rc != ORC_OK) goto done;
        int64_t raw = 0;
        if (solver == 0) rc = orc_maxflow_bk((uint32_t)F, nbr, res, term, &raw, part);
        else rc = orc_maxflow_pr((uint32_t)F, nbr, res, term, excess, 8, 1024, 0, &raw, part, NULL, NULL);
        if (rc != ORC_OK) goto done;
        for (size_t q = 0; q < F; ++q) out_labels[old[q]] = part[q] ? 1u : 0u;
        stats[0] = raw + info.terminal_base_flow;
        stats[1] = raw;
        stats[3] = (int64_t)(info.free_refs / 2u);
        stats[6] = (int64_t)info.terminal_edges;
        stats[7] = (int64_t)F;
    }
done:
    free(f2f); free(old); free(nbr); free(res); free(term); free(excess); free(part);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Cut-surface extraction: bindings.cpp:400-577.                             */
/* ------------------------------------------------------------------------ */
int orc_surface(const uint8_t* lp, const double* V, uint64_t nv,
                const int32_t* tets, const int32_t* nbrs, uint64_t N,
                uint64_t* n_faces, uint64_t* n_used,
                int32_t* out_faces, double* out_verts)
{
    uint64_t F = 0;
    for (uint64_t i = 0; i < N; ++i) {
        if (lp[i] != 0u) continue;
        for (int fi = 0; fi < 4; ++fi) {
            const int32_t j = nbrs[i * 4u + (uint64_t)fi];
            if (j < 0) ++F;
            else if ((uint64_t)j >= N) return ORC_ERR_NBR_RANGE;
            else if (lp[j] != 0u) ++F;
        }
    }
    int32_t* raw = (int32_t*)malloc((size_t)F * 12u + 4u);
    int32_t* remap = (int32_t*)malloc((size_t)nv * 4u + 4u);
    if (!raw || !remap) { free(raw); free(remap); return ORC_ERR_NO_MEM; }
    uint64_t pos = 0;
    for (uint64_t i = 0; i < N; ++i) {
        if (lp[i] != 0u) continue;
        const int32_t* tr = tets + i * 4u;
        for (int fi = 0; fi < 4; ++fi) {
            const int32_t j = nbrs[i * 4u + (uint64_t)fi];
            if (!(j < 0 || lp[j] != 0u)) continue;
            int32_t a0 = tr[FACE_LUT[fi][0]], b0 = tr[FACE_LUT[fi][1]];
            int32_t c0 = tr[FACE_LUT[fi][2]], fourth = tr[FACE_OPP[fi]];
            if (a0 < 0 || b0 < 0 || c0 < 0 || fourth < 0 || (uint64_t)a0 >= nv ||
                (uint64_t)b0 >= nv || (uint64_t)c0 >= nv || (uint64_t)fourth >= nv) {
                free(raw); free(remap); return ORC_ERR_BUILD;
            }
            int32_t t;
            if (a0 > b0) { t = a0; a0 = b0; b0 = t; }
            if (b0 > c0) { t = b0; b0 = c0; c0 = t; }
            if (a0 > b0) { t = a0; a0 = b0; b0 = t; }
            const double* v0 = V + (size_t)a0 * 3u;
            const double* v1 = V + (size_t)b0 * 3u;
            const double* v2 = V + (size_t)c0 * 3u;
            const double* vp = V + (size_t)fourth * 3u;
            const double x1 = v1[0] - v0[0], y1 = v1[1] - v0[1], z1 = v1[2] - v0[2];
            const double x2 = v2[0] - v0[0], y2 = v2[1] - v0[1], z2 = v2[2] - v0[2];
            const double cx = y1 * z2 - z1 * y2;
            const double cy = z1 * x2 - x1 * z2;
            const double cz = x1 * y2 - y1 * x2;
            const double px = vp[0] - v0[0], py = vp[1] - v0[1], pz = vp[2] - v0[2];
            const double vol = cx * px + cy * py + cz * pz;
            raw[3u * pos] = a0;
            raw[3u * pos + 1u] = (vol < 0.0) ? b0 : c0;
            raw[3u * pos + 2u] = (vol < 0.0) ? c0 : b0;
            ++pos;
        }
    }
    for (uint64_t i = 0; i < nv; ++i) remap[i] = -1;
    for (uint64_t i = 0; i < F * 3u; ++i) remap[raw[i]] = -2;
    uint64_t used = 0;
    for (uint64_t i = 0; i < nv; ++i) if (remap[i] == -2) remap[i] = (int32_t)used++;
    *n_faces = F;
    *n_used = used;
    if (out_faces && out_verts) {
        for (uint64_t i = 0; i < nv; ++i) {
            if (remap[i] >= 0) {
                const uint64_t ni = (uint64_t)remap[i];
                out_verts[3u * ni] = V[3u * i];
                out_verts[3u * ni + 1u] = V[3u * i + 1u];
                out_verts[3u * ni + 2u] = V[3u * i + 2u];
            }
        }
        for (uint64_t i = 0; i < F * 3u; ++i) out_faces[i] = remap[raw[i]];
    }
    free(raw);
    free(remap);
    return ORC_OK;
}

static int cmp_u64(const void* a, const void* b)
{
    const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return (x > y) - (x < y);
}

/* wtivo_core.cpp:418-447: edge keys, sort, runs of equal keys */
int orc_edge_audit(const int32_t* faces, uint64_t nf, uint64_t* bad_groups)
{
    if (!bad_groups || (nf && !faces)) return ORC_ERR_ARG;
    *bad_groups = 0;
    if (nf == 0) return ORC_OK;
    uint64_t* e = (uint64_t*)malloc(sizeof(uint64_t) * 3u * nf);
    if (!e) return ORC_ERR_NO_MEM;
    for (uint64_t i = 0; i < nf; ++i) {
        const int32_t a = faces[3u * i], b = faces[3u * i + 1u], c = faces[3u * i + 2u];
        if (a < 0 || b < 0 || c < 0) {
            free(e);
            return ORC_ERR_NEG_VERTEX;
        }
        const uint32_t ua = (uint32_t)a, ub = (uint32_t)b, uc = (uint32_t)c;
        e[3u * i] = ((uint64_t)(ua < ub ? ua : ub) << 32) | (ua < ub ? ub : ua);
        e[3u * i + 1u] = ((uint64_t)(ub < uc ? ub : uc) << 32) | (ub < uc ? uc : ub);
        e[3u * i + 2u] = ((uint64_t)(uc < ua ? uc : ua) << 32) | (uc < ua ? ua : uc);
    }
    qsort(e, 3u * nf, sizeof(uint64_t), cmp_u64);
    uint64_t bad = 0, p = 0;
    const uint64_t m = 3u * nf;
    while (p < m) {
        uint64_t q = p + 1u;
        while (q < m && e[q] == e[p]) ++q;
        if (q - p != 2u) ++bad;
        p = q;
    }
    free(e);
    *bad_groups = bad;
    return ORC_OK;
}

/* value of voxel (i,j,k): background outside the brick box or in an
 * inactive brick */
static float grid_value(const orc_brick_grid* g, int64_t i, int64_t j, int64_t k)
{
    i -= g->origin[0];
    j -= g->origin[1];
    k -= g->origin[2];
    if (i < 0 || j < 0 || k < 0) return g->background;
    const int64_t bx = i >> 3, by = j >> 3, bz = k >> 3;
    if (bx >= g->dims[0] || by >= g->dims[1] || bz >= g->dims[2]) return g->background;
    const int32_t b = g->table[(bx * g->dims[1] + by) * g->dims[2] + bz];
    if (b < 0) return g->background;
    return g->values[(size_t)b * 512u + (size_t)(((i & 7) * 8 + (j & 7)) * 8 + (k & 7))];
}

/* one lerp of BoxSampler::trilinearInterpolation: a + float((b - a) * w) */
static float box_lerp(float a, float b, double w)
{
    const float diff = b - a;
    const double temp = (double)diff * w;
    return a + (float)temp;
}

int orc_sample_tet_labels(const orc_brick_grid* g, const double* V, uint64_t nv,
                          const int32_t* tets, uint64_t nt, const double* bmin,
                          const double* bmax, double padding, double threshold,
                          uint8_t* labels, float* udf)
{
    if (!g || !bmin || !bmax || (nt && (!V || !tets || !labels)) || !(g->voxel_size > 0.0))
        return ORC_ERR_ARG;
    const double sx = bmax[0] - bmin[0], sy = bmax[1] - bmin[1], sz = bmax[2] - bmin[2];
    if (!(sx > 0 && sy > 0 && sz > 0)) return ORC_ERR_BBOX;         /* :1546-1547 */
    const double scale = 1.0 - 2.0 * padding;
    const double inv_h = 1.0 / g->voxel_size;   /* linear transform: index = world * (1/h) */
    for (uint64_t i = 0; i < nt; ++i) {
        double cx = 0.0, cy = 0.0, cz = 0.0;
        for (int q = 0; q < 4; ++q) {                               /* :1563-1570 */
            const int32_t vi = tets[4u * i + (uint64_t)q];
            if (vi < 0 || (uint64_t)vi >= nv) return ORC_ERR_TET_INDEX;
            cx += V[3u * (uint64_t)vi + 0u];
            cy += V[3u * (uint64_t)vi + 1u];
            cz += V[3u * (uint64_t)vi + 2u];
        }
        cx *= 0.25;
        cy *= 0.25;
        cz *= 0.25;
        const double nx = ((cx - bmin[0]) / sx) * scale + padding;  /* :1572-1574 */
        const double ny = ((cy - bmin[1]) / sy) * scale + padding;
        const double nz = ((cz - bmin[2]) / sz) * scale + padding;
        const double x = nx * inv_h, y = ny * inv_h, z = nz * inv_h;
        const double fx = floor(x), fy = floor(y), fz = floor(z);
        const int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
        const double u = x - fx, v = y - fy, w = z - fz;
        float d[2][2][2];
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                for (int c = 0; c < 2; ++c) d[a][b][c] = grid_value(g, ix + a, iy + b, iz + c);
        const float val = box_lerp(box_lerp(box_lerp(d[0][0][0], d[0][0][1], w),
                                            box_lerp(d[0][1][0], d[0][1][1], w), v),
                                   box_lerp(box_lerp(d[1][0][0], d[1][0][1], w),
                                            box_lerp(d[1][1][0], d[1][1][1], w), v),
                                   u);
        labels[i] = ((double)val <= threshold) ? 0u : 1u;             /* :1576 */
        if (udf) udf[i] = val;
    }
    return ORC_OK;
}
