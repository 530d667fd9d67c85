/*
 * CPU oracle for the TagMatch subset-matching path.  TEST INFRASTRUCTURE ONLY:
 * the tests, the smoke check and the bench's CPU-baseline leg use it as the
 * checker; the product never links or calls it.
 *
 * Pinned against the reference: tests compare it with the reference's own
 * sequential matcher (test_matcher.cc, built from the reference sources into
 * oracle/_ref by oracle/Makefile) and with the reference's CPU partitioner
 * (partitioning.cc, same recipe), and with the golden vectors under
 * tests/golden produced by those binaries.
 *
 * Filters and queries are 6 x uint32 words: bit p of the 192-bit filter is
 * bit (p % 32) of word p / 32 (bitvector.hh:210-212, test_io.cc:50-68).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define W 6

/* bitvector<192>::subset_of (bitvector.hh:282-296): f & ~q == 0 on every
 * block.  The 64-bit blocks are the word pairs (0,1), (2,3), (4,5). */
static inline int subset_of(const uint32_t *f, const uint32_t *q) {
    uint32_t acc = 0;
    for (int i = 0; i < W; ++i) acc |= f[i] & ~q[i];
    return acc == 0;
}

int oracle_subset_of(const uint32_t *f, const uint32_t *q) { return subset_of(f, q); }

/* bitvector<192>::operator< (bitvector.hh:389-397): in the first differing
 * 64-bit block, the lowest differing bit decides; the vector holding a 1
 * there is the greater one. */
int oracle_filter_less(const uint32_t *a, const uint32_t *b) {
    for (int blk = 0; blk < 3; ++blk) {
        uint64_t x = (uint64_t)a[2 * blk] | ((uint64_t)a[2 * blk + 1] << 32);
        uint64_t y = (uint64_t)b[2 * blk] | ((uint64_t)b[2 * blk + 1] << 32);
        if (x != y) {
            int pos = __builtin_ctzll(x ^ y);
            return (int)((y >> pos) & 1);
        }
    }
    return 0;
}

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

/* ------------------------------------------------------------------ */
/* Sequential matcher: test_matcher.cc:74-81 for each query, keys in   */
/* table order; match_unique sorts and de-duplicates each query's keys */
/* (tagmatch_query.hh:99-119).                                          */
/* ------------------------------------------------------------------ */
typedef struct {
    const uint32_t *filters; uint64_t n;
    const uint32_t *key_off; const uint32_t *keys;
    const uint32_t *queries; uint64_t q0, q1;
    int unique;
    uint64_t *counts;      /* pass 1 */
    const uint64_t *offs;  /* pass 2 */
    uint32_t *out;         /* pass 2 */
} job_t;

static uint64_t match_one(const job_t *j, uint64_t qi, uint32_t *dst) {
    const uint32_t *q = j->queries + qi * W;
    uint64_t c = 0;
    for (uint64_t f = 0; f < j->n; ++f) {
        if (subset_of(j->filters + f * W, q)) {
            uint32_t b = j->key_off[f], e = j->key_off[f + 1];
            if (dst) memcpy(dst + c, j->keys + b, (size_t)(e - b) * sizeof(uint32_t));
            c += e - b;
        }
    }
    return c;
}

static void *count_worker(void *arg) {
    job_t *j = (job_t *)arg;
    for (uint64_t qi = j->q0; qi < j->q1; ++qi) j->counts[qi] = match_one(j, qi, NULL);
    return NULL;
}

static void *fill_worker(void *arg) {
    job_t *j = (job_t *)arg;
    for (uint64_t qi = j->q0; qi < j->q1; ++qi) {
        uint32_t *dst = j->out + j->offs[qi];
        uint64_t c = match_one(j, qi, dst);
        if (j->unique && c > 1) {
            qsort(dst, (size_t)c, sizeof(uint32_t), cmp_u32);
            uint64_t u = 1;
            for (uint64_t k = 1; k < c; ++k) if (dst[k] != dst[u - 1]) dst[u++] = dst[k];
            for (uint64_t k = u; k < c; ++k) dst[k] = 0xFFFFFFFFu; /* tail unused */
            j->counts[qi] = u;
        } else {
            j->counts[qi] = c;
        }
    }
    return NULL;
}

static void run_jobs(job_t *base, int nthreads, uint64_t nq, void *(*fn)(void *)) {
    if (nthreads < 1) nthreads = 1;
    if ((uint64_t)nthreads > nq) nthreads = nq ? (int)nq : 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    job_t *jobs = (job_t *)malloc(sizeof(job_t) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        jobs[t] = *base;
        jobs[t].q0 = nq * t / nthreads;
        jobs[t].q1 = nq * (t + 1) / nthreads;
        pthread_create(&th[t], NULL, fn, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(jobs);
}

/* Pass 1: per-query key counts (before de-duplication). */
int oracle_count(const uint32_t *filters, uint64_t n, const uint32_t *key_off, const uint32_t *keys,
                 const uint32_t *queries, uint64_t nq, uint64_t *counts, int nthreads) {
    job_t j = {filters, n, key_off, keys, queries, 0, nq, 0, counts, NULL, NULL};
    run_jobs(&j, nthreads, nq, count_worker);
    return 0;
}

/* Pass 2: fill.  offs[i] = start of query i in out (from pass-1 counts);
 * counts[i] receives the final count (unique count when unique != 0), the
 * unique keys sorted ascending at out[offs[i]..]. */
int oracle_fill(const uint32_t *filters, uint64_t n, const uint32_t *key_off, const uint32_t *keys,
                const uint32_t *queries, uint64_t nq, int unique, const uint64_t *offs,
                uint32_t *out, uint64_t *counts, int nthreads) {
    job_t j = {filters, n, key_off, keys, queries, 0, nq, unique, counts, offs, out};
    run_jobs(&j, nthreads, nq, fill_worker);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Single pass per query with digests: the same work as test_matcher  */
/* (test_matcher.cc:74-81: one scan of the table per query, the keys  */
/* of every matching filter gathered), the keys reduced to a per-query */
/* (count, multiset hash) instead of printed.  The hash of a key k is  */
/* fin64(k + 0x9E3779B97F4A7C15) (the splitmix64 finalizer); a query's */
/* hash is the wrapping sum over its keys, so it does not depend on    */
/* key order.  unique != 0 sorts and de-duplicates first               */
/* (tagmatch_query.hh:99-119).                                          */
/* ------------------------------------------------------------------ */
static inline uint64_t fin64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct {
    job_t j;
    uint64_t *hashes;
} digest_job_t;

static void *digest_worker(void *arg) {
    digest_job_t *d = (digest_job_t *)arg;
    const job_t *j = &d->j;
    size_t cap = 1 << 16;
    uint32_t *buf = (uint32_t *)malloc(cap * sizeof(uint32_t));
    for (uint64_t qi = j->q0; qi < j->q1; ++qi) {
        const uint32_t *q = j->queries + qi * W;
        uint64_t c = 0;
        for (uint64_t f = 0; f < j->n; ++f) {
            if (subset_of(j->filters + f * W, q)) {
                uint32_t b = j->key_off[f], e = j->key_off[f + 1];
                if (c + (e - b) > cap) {
                    while (c + (e - b) > cap) cap *= 2;
                    buf = (uint32_t *)realloc(buf, cap * sizeof(uint32_t));
                }
                memcpy(buf + c, j->keys + b, (size_t)(e - b) * sizeof(uint32_t));
                c += e - b;
            }
        }
        if (j->unique && c > 1) {
            qsort(buf, (size_t)c, sizeof(uint32_t), cmp_u32);
            uint64_t u = 1;
            for (uint64_t k = 1; k < c; ++k) if (buf[k] != buf[u - 1]) buf[u++] = buf[k];
            c = u;
        }
        uint64_t h = 0;
        for (uint64_t k = 0; k < c; ++k) h += fin64((uint64_t)buf[k] + 0x9E3779B97F4A7C15ull);
        j->counts[qi] = c;
        d->hashes[qi] = h;
    }
    free(buf);
    return NULL;
}

int oracle_match_digest(const uint32_t *filters, uint64_t n, const uint32_t *key_off, const uint32_t *keys,
                        const uint32_t *queries, uint64_t nq, int unique, uint64_t *counts, uint64_t *hashes,
                        int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if ((uint64_t)nthreads > nq) nthreads = nq ? (int)nq : 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    digest_job_t *jobs = (digest_job_t *)malloc(sizeof(digest_job_t) * nthreads);
    for (int t = 0; t < nthreads; ++t) {
        job_t j = {filters, n, key_off, keys, queries, nq * t / nthreads, nq * (t + 1) / nthreads, unique, counts, NULL,
                   NULL};
        jobs[t].j = j;
        jobs[t].hashes = hashes;
        pthread_create(&th[t], NULL, digest_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    free(th); free(jobs);
    return 0;
}

/* ------------------------------------------------------------------ */
/* The reference's small-partition CPU backend (back_end.cc:496-517):  */
/* for a partition below the size threshold, every filter is tested    */
/* against every query routed to the partition on the CPU, and the     */
/* matching filter's keys are appended to the query's output.  Here    */
/* the partitions are split over threads; each thread reduces its      */
/* queries' keys to (count, multiset hash) as match_digest does, and   */
/* the per-thread sums are added at the end.                           */
/*   filters [n][6] grouped by partition (part_off[np + 1]), key CSR    */
/*   per filter; routed[route_off[p] .. route_off[p + 1]) the query     */
/*   indices routed to partition p.                                     */
/* ------------------------------------------------------------------ */
typedef struct {
    const uint32_t *filters, *part_off, *key_off, *keys, *queries, *route_off, *routed;
    uint64_t p0, p1, nq;
    uint64_t *counts, *hashes; /* per thread, nq each */
} backend_job_t;

static void *backend_worker(void *arg) {
    backend_job_t *j = (backend_job_t *)arg;
    for (uint64_t p = j->p0; p < j->p1; ++p) {
        for (uint32_t f = j->part_off[p]; f < j->part_off[p + 1]; ++f) {
            const uint32_t *fw = j->filters + (uint64_t)f * W;
            for (uint32_t r = j->route_off[p]; r < j->route_off[p + 1]; ++r) {
                const uint32_t qi = j->routed[r];
                if (subset_of(fw, j->queries + (uint64_t)qi * W)) {
                    for (uint32_t k = j->key_off[f]; k < j->key_off[f + 1]; ++k) {
                        j->hashes[qi] += fin64((uint64_t)j->keys[k] + 0x9E3779B97F4A7C15ull);
                        j->counts[qi] += 1;
                    }
                }
            }
        }
    }
    return NULL;
}

int oracle_cpu_backend(const uint32_t *filters, const uint32_t *part_off, uint64_t np, const uint32_t *key_off,
                       const uint32_t *keys, const uint32_t *queries, uint64_t nq, const uint32_t *route_off,
                       const uint32_t *routed, uint64_t *counts, uint64_t *hashes, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    if ((uint64_t)nthreads > np) nthreads = np ? (int)np : 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * nthreads);
    backend_job_t *jobs = (backend_job_t *)malloc(sizeof(backend_job_t) * nthreads);
    uint64_t *cnt = (uint64_t *)calloc((size_t)nthreads * (nq ? nq : 1), sizeof(uint64_t));
    uint64_t *hsh = (uint64_t *)calloc((size_t)nthreads * (nq ? nq : 1), sizeof(uint64_t));
    /* partitions dealt to threads by routed pair work, in contiguous runs */
    uint64_t total = 0;
    for (uint64_t p = 0; p < np; ++p)
        total += (uint64_t)(part_off[p + 1] - part_off[p]) * (route_off[p + 1] - route_off[p]);
    uint64_t p = 0, acc = 0;
    for (int t = 0; t < nthreads; ++t) {
        backend_job_t b = {filters, part_off, key_off, keys, queries, route_off, routed, p, p, nq,
                           cnt + (size_t)t * nq, hsh + (size_t)t * nq};
        const uint64_t goal = total * (uint64_t)(t + 1) / (uint64_t)nthreads;
        while (p < np && (acc < goal || t == nthreads - 1)) {
            acc += (uint64_t)(part_off[p + 1] - part_off[p]) * (route_off[p + 1] - route_off[p]);
            ++p;
        }
        b.p1 = p;
        jobs[t] = b;
        pthread_create(&th[t], NULL, backend_worker, &jobs[t]);
    }
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    for (uint64_t q = 0; q < nq; ++q) {
        uint64_t c = 0, h = 0;
        for (int t = 0; t < nthreads; ++t) {
            c += cnt[(size_t)t * nq + q];
            h += hsh[(size_t)t * nq + q];
        }
        counts[q] = c;
        hashes[q] = h;
    }
    free(cnt); free(hsh); free(th); free(jobs);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Balanced partitioning, restated from partitioning.cc.               */
/*                                                                     */
/* The reference runs a thread pool over a queue of candidates         */
/* (do_balanced_partitioning, :280-340); every branch of its loop is   */
/* equivalent to this recursion over contiguous ranges:                */
/*   node of size > max_p: split on balancing_pivot (:262-278): the    */
/*     first unused bit u, replaced only by a later bit (used or not)  */
/*     whose |freq - size/2| is strictly smaller; stable partition,    */
/*     zero side first (:133-148); both sides recurse, the one side    */
/*     gets the pivot in its mask, both get it in used_bits;           */
/*   leaf of size <= max_p: if its pivot mask is empty,                */
/*     nonzero_mask_partitioning (:230-250) peels the one side of the  */
/*     most frequent bit (first maximum) until all members share a     */
/*     bit; otherwise it is a partition.                               */
/*   The root with size <= max_p goes straight to the peeling step.    */
/* Partition masks are the AND of the members (:389-407).              */
/* Because the splits depend only on the members' frequencies, the     */
/* set of partitions is deterministic; only the reference's ids depend */
/* on thread order.  Here ids follow emission order.                   */
/*                                                                     */
/* The reference loops forever on an all-zero filter in the peeling    */
/* step; this restatement (like the product) closes a range whose      */
/* members are all zero as its own partition with an empty mask.       */
/* ------------------------------------------------------------------ */
typedef struct {
    uint32_t *idx;      /* permutation of filter indices */
    uint32_t *tmp;
    const uint32_t *f;
    uint32_t maxp;
    uint32_t *pb, *pe;  /* partition ranges (begin, end) */
    uint64_t np, cap;
    int overflow;
} part_ctx;

static inline int bit_of(const uint32_t *f, unsigned b) { return (f[b >> 5] >> (b & 31)) & 1; }

static void freqs(part_ctx *c, uint32_t b, uint32_t e, uint32_t *fr) {
    memset(fr, 0, 192 * sizeof(uint32_t));
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t *f = c->f + (uint64_t)c->idx[i] * W;
        for (int w = 0; w < W; ++w) {
            uint32_t x = f[w];
            while (x) { int t = __builtin_ctz(x); fr[w * 32 + t]++; x &= x - 1; }
        }
    }
}

static uint32_t split(part_ctx *c, uint32_t b, uint32_t e, unsigned pivot) {
    uint32_t z = b, o = 0;
    for (uint32_t i = b; i < e; ++i) {
        uint32_t id = c->idx[i];
        if (!bit_of(c->f + (uint64_t)id * W, pivot)) c->idx[z++] = id;
        else c->tmp[o++] = id;
    }
    memcpy(c->idx + z, c->tmp, (size_t)o * sizeof(uint32_t));
    return z;
}

static void emit(part_ctx *c, uint32_t b, uint32_t e) {
    if (c->np >= c->cap) { c->overflow = 1; c->np++; return; }
    c->pb[c->np] = b; c->pe[c->np] = e; c->np++;
}

static void peel(part_ctx *c, uint32_t b, uint32_t e) {
    uint32_t fr[192];
    for (;;) {
        freqs(c, b, e, fr);
        uint32_t mx = fr[0]; unsigned pv = 0;
        for (unsigned k = 1; k < 192; ++k) if (fr[k] > mx) { mx = fr[k]; pv = k; }
        if (mx == e - b || mx == 0) { emit(c, b, e); return; }
        uint32_t m = split(c, b, e, pv);
        emit(c, m, e);
        e = m;
    }
}

static void balance(part_ctx *c, uint32_t b, uint32_t e, const uint32_t *used_in, int mask_empty) {
    uint32_t size = e - b;
    if (size <= c->maxp) {
        if (mask_empty) peel(c, b, e); else emit(c, b, e);
        return;
    }
    uint32_t fr[192], used[W];
    memcpy(used, used_in, sizeof(used));
    freqs(c, b, e, fr);
    uint32_t half = size / 2;
    unsigned u = 0;
    while (u < 192 && bit_of(used, u)) ++u;
    unsigned pv = u;
    uint32_t md = fr[u] > half ? fr[u] - half : half - fr[u];
    for (unsigned k = u + 1; k < 192; ++k) {
        uint32_t d = fr[k] > half ? fr[k] - half : half - fr[k];
        if (d < md) { pv = k; if (d == 0) break; md = d; }
    }
    uint32_t m = split(c, b, e, pv);
    used[pv >> 5] |= 1u << (pv & 31);
    balance(c, b, m, used, mask_empty);
    balance(c, m, e, used, 0);
}

/* order: out permutation of filter indices (n), partitions listed as ranges
 * of it.  Returns the number of partitions, or -1 if cap is too small. */
int64_t oracle_partition(const uint32_t *filters, uint32_t n, uint32_t maxp, uint32_t *order,
                         uint32_t *part_begin, uint32_t *part_end, uint64_t cap) {
    if (maxp == 0) return -2;
    part_ctx c;
    c.idx = order; c.f = filters; c.maxp = maxp; c.pb = part_begin; c.pe = part_end;
    c.np = 0; c.cap = cap; c.overflow = 0;
    c.tmp = (uint32_t *)malloc(sizeof(uint32_t) * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    if (n > 0) {
        uint32_t used[W] = {0, 0, 0, 0, 0, 0};
        if (n > maxp) balance(&c, 0, n, used, 1); else peel(&c, 0, n);
    }
    free(c.tmp);
    return c.overflow ? -1 : (int64_t)c.np;
}
