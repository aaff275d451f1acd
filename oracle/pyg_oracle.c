/*
 * CPU oracle for the Pythia join / aggregation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, what the
 * reference's operators compute so that the CUDA path can be checked
 * bit-for-bit.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it; the product library never links or calls it.
 *
 * Parity pin: the restatement is itself checked against the reference
 * engine built from source (oracle/ref.mk -> oracle/_ref/executequery) on
 * committed golden fixtures (tests/golden/), and against the known answers
 * the reference's own unit tests assert (tests/test_oracle.py).
 *
 * Data model (reference util/buffer.h:134-357, schema.cpp): a relation is a
 * packed row-major array of fixed-width tuples; a column is (byte offset,
 * type) with type 4-byte signed int (CT_INTEGER) or 8-byte signed long
 * (CT_LONG).  Sums wrap modulo 2^width exactly like `CtLong +=` /
 * `CtInt +=` in operators/aggregatesum.cpp:81-105.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_INT32 1
#define ORC_INT64 2

typedef struct {
    const uint8_t* base;
    int64_t ntuples;
    int32_t tuple_bytes;
    int32_t ncols;
    int32_t col_offset[8];
    int32_t col_type[8];
} orc_rel;

static inline int colsize(const orc_rel* r, int c) { return r->col_type[c] == ORC_INT32 ? 4 : 8; }

static inline int64_t getcol(const orc_rel* r, int64_t i, int c)
{
    const uint8_t* p = r->base + (size_t)i * r->tuple_bytes + r->col_offset[c];
    if (r->col_type[c] == ORC_INT32) { int32_t v; memcpy(&v, p, 4); return v; }
    int64_t v; memcpy(&v, p, 8); return v;
}

/* ModuloValueHasher (hash.h:274-307): bucket = value & (2^k - 1), where the
 * bucket count is rounded up to a power of two by getlogarithm
 * (hash.cpp:49-59). */
static unsigned orc_getlogarithm(unsigned k)
{
    --k;
    for (unsigned i = 0; i < 32; ++i)
        if ((0x80000000u >> i) & k) return 32 - i;
    return 0;
}

/* ByteHasher FNV-1a over the key bytes (hash.h:158-201), folded to k bits. */
static unsigned orc_fnv(const uint8_t* p, int n, unsigned k)
{
    uint64_t h = 14695981039346656037ull;
    for (int i = 0; i < n; ++i) {
        h ^= (uint64_t)(int64_t)(int8_t)p[i];
        h += (h << 1) + (h << 4) + (h << 5) + (h << 7) + (h << 8) + (h << 40);
    }
    h = ((h >> k) ^ h) & ((1ull << k) - 1);
    return (unsigned)h;
}

/* Key bytes of tuple i over key columns: the reference compares keys column
 * by column with typed equality (comparator.cpp / conjunctionevaluator.cpp);
 * for int columns that is equality of the raw bytes. */
static int keyeq(const orc_rel* a, int64_t i, const int* ka, const orc_rel* b, int64_t j, const int* kb, int nk)
{
    for (int c = 0; c < nk; ++c)
        if (getcol(a, i, ka[c]) != getcol(b, j, kb[c])) return 0;
    return 1;
}

static unsigned hashkey(const orc_rel* r, int64_t i, const int* kc, int nk, unsigned logb, int bytes_hash)
{
    if (!bytes_hash) return (unsigned)((uint64_t)getcol(r, i, kc[0]) & ((1ull << logb) - 1));
    uint8_t buf[64]; int n = 0;
    for (int c = 0; c < nk; ++c) {
        int s = colsize(r, kc[c]);
        memcpy(buf + n, r->base + (size_t)i * r->tuple_bytes + r->col_offset[kc[c]], s);
        n += s;
    }
    return orc_fnv(buf, n, logb);
}

/* Chained bucket table (util/hashtable.h:44-299): each bucket holds a list
 * of tuple indices in insertion order.  Implemented as head/next arrays. */
typedef struct { int64_t* head; int64_t* next; unsigned logb; } orc_table;

static int table_build(orc_table* t, const orc_rel* R, const int* kc, int nk, unsigned buckets, int bytes_hash)
{
    t->logb = orc_getlogarithm(buckets ? buckets : 1);
    size_t nb = (size_t)1 << t->logb;
    t->head = (int64_t*)malloc(nb * sizeof(int64_t));
    t->next = (int64_t*)malloc((size_t)(R->ntuples > 0 ? R->ntuples : 1) * sizeof(int64_t));
    if (!t->head || !t->next) return -2;
    for (size_t b = 0; b < nb; ++b) t->head[b] = -1;
    /* HashJoinOp::buildFromPage (operators/join.cpp:838-884): hash each
     * build tuple, append it to its bucket.  Appending at the head reverses
     * in-bucket order, which only changes output order (unspecified). */
    for (int64_t i = 0; i < R->ntuples; ++i) {
        unsigned h = hashkey(R, i, kc, nk, t->logb, bytes_hash);
        t->next[i] = t->head[h];
        t->head[h] = i;
    }
    return 0;
}

static void table_free(orc_table* t) { free(t->head); free(t->next); }

/* Projection entry: side 0 = build ("B$i"), 1 = probe ("P$i")
 * (operators/join.cpp:142-183). */
typedef struct { int32_t side; int32_t col; } orc_proj;

/*
 * Hash join + fused aggregation: the plan hashjoin -> printer_tuplecount ->
 * aggregate_sum(fields=[]) per projected column.  Follows
 * HashJoinOp::getNext (operators/join.cpp:681-757): for every probe tuple,
 * walk its bucket and, for every build tuple with equal keys, produce the
 * projected output tuple; here each output column is summed (wrapping, as
 * aggregatesum.cpp:81-105) and the matches are counted.
 * sums[j] receives the wrapped sum of projected column j (int32 columns
 * wrap at 32 bits and are returned sign-extended).
 */
int orc_hashjoin_agg(const orc_rel* R, const int* rk, const orc_rel* S, const int* sk, int nk,
                     const orc_proj* proj, int nproj, unsigned buckets, int bytes_hash,
                     int64_t* out_count, int64_t* sums)
{
    orc_table t;
    int rc = table_build(&t, R, rk, nk, buckets, bytes_hash);
    if (rc) { table_free(&t); return rc; }
    uint64_t cnt = 0;
    uint64_t acc[16] = {0};
    for (int64_t j = 0; j < S->ntuples; ++j) {
        unsigned h = hashkey(S, j, sk, nk, t.logb, bytes_hash);
        for (int64_t i = t.head[h]; i >= 0; i = t.next[i]) {
            if (!keyeq(R, i, rk, S, j, sk, nk)) continue;
            ++cnt;
            for (int p = 0; p < nproj; ++p) {
                const orc_rel* src = proj[p].side ? S : R;
                int64_t row = proj[p].side ? j : i;
                acc[p] += (uint64_t)getcol(src, row, proj[p].col);
            }
        }
    }
    *out_count = (int64_t)cnt;
    for (int p = 0; p < nproj; ++p) {
        const orc_rel* src = proj[p].side ? S : R;
        if (src->col_type[proj[p].col] == ORC_INT32) sums[p] = (int64_t)(int32_t)(uint32_t)acc[p];
        else sums[p] = (int64_t)acc[p];
    }
    table_free(&t);
    return 0;
}

/* Materialising hash join: HashJoinOp::constructOutputTuple
 * (operators/join.cpp:648-679) writes the projected columns back to back in
 * projection order.  Returns the number of output tuples (or -1 if
 * out_capacity is too small; the count is still returned in *needed). */
int64_t orc_hashjoin_materialize(const orc_rel* R, const int* rk, const orc_rel* S, const int* sk, int nk,
                                 const orc_proj* proj, int nproj, unsigned buckets, int bytes_hash,
                                 uint8_t* out, int64_t out_capacity, int64_t* needed)
{
    orc_table t;
    if (table_build(&t, R, rk, nk, buckets, bytes_hash)) { table_free(&t); return -2; }
    int ob = 0;
    for (int p = 0; p < nproj; ++p) ob += colsize(proj[p].side ? S : R, proj[p].col);
    int64_t n = 0;
    for (int64_t j = 0; j < S->ntuples; ++j) {
        unsigned h = hashkey(S, j, sk, nk, t.logb, bytes_hash);
        for (int64_t i = t.head[h]; i >= 0; i = t.next[i]) {
            if (!keyeq(R, i, rk, S, j, sk, nk)) continue;
            if (n < out_capacity) {
                uint8_t* dst = out + (size_t)n * ob;
                for (int p = 0; p < nproj; ++p) {
                    const orc_rel* src = proj[p].side ? S : R;
                    int64_t row = proj[p].side ? j : i;
                    int s = colsize(src, proj[p].col);
                    memcpy(dst, src->base + (size_t)row * src->tuple_bytes + src->col_offset[proj[p].col], s);
                    dst += s;
                }
            }
            ++n;
        }
    }
    table_free(&t);
    *needed = n;
    return n <= out_capacity ? n : -1;
}

/*
 * Group-by aggregation: GenericAggregate::remember (operators/
 * genericaggregate.cpp:247-289) with AggregateSum / AggregateCount fold
 * (aggregatesum.cpp:53-105, aggregatecount.cpp:44-52).  Groups are kept in
 * a chained table; a new group copies the key columns and starts the fold,
 * an existing group folds.  flags bit0 = sum(sum_col), bit1 = count.
 * Output tuple = key columns packed, then the sum (type of sum_col) if
 * requested, then the count (int64) if requested, in first-seen order.
 * nk == 0 means no GROUP BY (the `alwayszero` hasher, :80-87): one group
 * when the input is non-empty.
 */
int64_t orc_groupby(const orc_rel* in, const int* kc, int nk, int flags, int sum_col,
                    unsigned buckets, int bytes_hash, uint8_t* out, int64_t out_capacity)
{
    unsigned logb = nk ? orc_getlogarithm(buckets ? buckets : 1) : 0;
    size_t nb = (size_t)1 << logb;
    int64_t* head = (int64_t*)malloc(nb * sizeof(int64_t));
    int64_t cap = in->ntuples > 0 ? in->ntuples : 1;
    int64_t* next = (int64_t*)malloc(cap * sizeof(int64_t));
    int64_t* rep = (int64_t*)malloc(cap * sizeof(int64_t)); /* group -> first input row */
    uint64_t* sum = (uint64_t*)calloc(cap, sizeof(uint64_t));
    uint64_t* cnt = (uint64_t*)calloc(cap, sizeof(uint64_t));
    if (!head || !next || !rep || !sum || !cnt) { free(head); free(next); free(rep); free(sum); free(cnt); return -2; }
    for (size_t b = 0; b < nb; ++b) head[b] = -1;
    int64_t ng = 0;
    for (int64_t i = 0; i < in->ntuples; ++i) {
        unsigned h = nk ? hashkey(in, i, kc, nk, logb, bytes_hash) : 0;
        int64_t g;
        for (g = head[h]; g >= 0; g = next[g])
            if (keyeq(in, rep[g], kc, in, i, kc, nk)) break;
        if (g < 0) { g = ng++; rep[g] = i; next[g] = head[h]; head[h] = g; }
        if (flags & 1) sum[g] += (uint64_t)getcol(in, i, sum_col);
        cnt[g] += 1;
    }
    int ob = 0;
    for (int c = 0; c < nk; ++c) ob += colsize(in, kc[c]);
    int sumsz = (flags & 1) ? colsize(in, sum_col) : 0;
    ob += sumsz + ((flags & 2) ? 8 : 0);
    if (out && ng <= out_capacity) {
        for (int64_t g = 0; g < ng; ++g) {
            uint8_t* dst = out + (size_t)g * ob;
            for (int c = 0; c < nk; ++c) {
                int s = colsize(in, kc[c]);
                memcpy(dst, in->base + (size_t)rep[g] * in->tuple_bytes + in->col_offset[kc[c]], s);
                dst += s;
            }
            if (flags & 1) {
                if (sumsz == 4) { uint32_t v = (uint32_t)sum[g]; memcpy(dst, &v, 4); }
                else memcpy(dst, &sum[g], 8);
                dst += sumsz;
            }
            if (flags & 2) memcpy(dst, &cnt[g], 8);
        }
    }
    free(head); free(next); free(rep); free(sum); free(cnt);
    return ng;
}

/* ExactRangeValueHasher (hash.h:452-487): bucketrange = (max-min+k)/k,
 * bucket = (value-min)/bucketrange with C truncating signed division. */
int orc_exactrange_bucket(int64_t v, int64_t mn, int64_t mx, unsigned k)
{
    int64_t br = (mx - mn + (int64_t)k) / (int64_t)k;
    return (int)(unsigned)((v - mn) / br);
}

int64_t orc_exactrange_min_for_bucket(unsigned b, int64_t mn, int64_t mx, unsigned k)
{
    if (b == k) return mx + 1;
    int64_t br = (mx - mn + (int64_t)k) / (int64_t)k;
    return (int64_t)b * br + mn;
}

/*
 * Partition: PartitionOp::scanStart (operators/partition.cpp:272-359):
 * histogram of bucket ids (copySourceIntoPageAndPopulateHistogram :166-200),
 * exclusive prefix sum, scatter in input order (repartition :249-270).
 * kind 0 = exactrange(mn, mx, fanout); kind 1 = explicit splitters
 * (fanout-1 ascending values; bucket = number of splitters <= key);
 * kind 2 = low bits of the key (radix, fanout a power of two).
 * Writes offsets[0..fanout] and the partitioned tuples.  Returns 0, or -1
 * if a key falls outside [0, fanout) under exactrange.
 */
int orc_partition(const orc_rel* in, int key_col, int kind, unsigned fanout, int64_t mn, int64_t mx,
                  const int64_t* splitters, uint8_t* out, int64_t* offsets)
{
    int64_t* hist = (int64_t*)calloc(fanout + 1, sizeof(int64_t));
    unsigned* bk = (unsigned*)malloc((size_t)(in->ntuples > 0 ? in->ntuples : 1) * sizeof(unsigned));
    if (!hist || !bk) { free(hist); free(bk); return -2; }
    for (int64_t i = 0; i < in->ntuples; ++i) {
        int64_t v = getcol(in, i, key_col);
        unsigned b;
        if (kind == 0) {
            b = (unsigned)orc_exactrange_bucket(v, mn, mx, fanout);
        } else if (kind == 1) {
            unsigned lo = 0, hi = fanout - 1; /* count splitters <= v */
            while (lo < hi) { unsigned m = (lo + hi) / 2; if (splitters[m] <= v) lo = m + 1; else hi = m; }
            b = lo;
        } else {
            b = (unsigned)((uint64_t)v & (uint64_t)(fanout - 1));
        }
        if (b >= fanout) { free(hist); free(bk); return -1; }
        bk[i] = b;
        hist[b]++;
    }
    offsets[0] = 0;
    for (unsigned b = 0; b < fanout; ++b) offsets[b + 1] = offsets[b] + hist[b];
    for (unsigned b = 0; b < fanout; ++b) hist[b] = offsets[b];
    for (int64_t i = 0; i < in->ntuples; ++i)
        memcpy(out + (size_t)(hist[bk[i]]++) * in->tuple_bytes, in->base + (size_t)i * in->tuple_bytes, in->tuple_bytes);
    free(hist); free(bk);
    return 0;
}

/* Sort: TupleBuffer::sort<KeyT> (util/buffer.inl:119-452) orders tuples by
 * the signed key at a column.  std::sort is unstable there; the oracle
 * sorts stably (a bottom-up merge sort on row indices), which is one of the
 * orders the reference may produce, so comparisons of sort output use the
 * key sequence plus the multiset of tuples. */
static const orc_rel* g_sort_rel;
static int g_sort_col;
static void msort(int64_t* a, int64_t* tmp, int64_t n)
{
    for (int64_t w = 1; w < n; w *= 2) {
        for (int64_t lo = 0; lo < n; lo += 2 * w) {
            int64_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            int64_t i = lo, j = mid, k = lo;
            while (i < mid && j < hi) {
                if (getcol(g_sort_rel, a[j], g_sort_col) < getcol(g_sort_rel, a[i], g_sort_col)) tmp[k++] = a[j++];
                else tmp[k++] = a[i++];
            }
            while (i < mid) tmp[k++] = a[i++];
            while (j < hi) tmp[k++] = a[j++];
        }
        memcpy(a, tmp, (size_t)n * sizeof(int64_t));
    }
}

int orc_sort(const orc_rel* in, int key_col, uint8_t* out)
{
    int64_t n = in->ntuples;
    int64_t* idx = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    int64_t* tmp = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    if (!idx || !tmp) { free(idx); free(tmp); return -2; }
    for (int64_t i = 0; i < n; ++i) idx[i] = i;
    g_sort_rel = in; g_sort_col = key_col;
    msort(idx, tmp, n);
    for (int64_t i = 0; i < n; ++i)
        memcpy(out + (size_t)i * in->tuple_bytes, in->base + (size_t)idx[i] * in->tuple_bytes, in->tuple_bytes);
    free(idx); free(tmp);
    return 0;
}

/*
 * MPSM sort-merge join (OldMPSMJoinOp, operators/join.cpp:1481-1617 over
 * SortMergeJoinOp::scanStart :1234-1292): both inputs sorted on the single
 * join key, then merged; equal-key runs produce their cross product (the
 * rewind of :1567-1572).  Output = projected columns packed, in
 * (build key, build position, probe position) order.  Aggregation variant:
 * count + sums of projected columns, as orc_hashjoin_agg.
 */
int64_t orc_mpsm_join(const orc_rel* R, int rk, const orc_rel* S, int sk,
                      const orc_proj* proj, int nproj, uint8_t* out, int64_t out_capacity,
                      int64_t* out_count, int64_t* sums)
{
    uint8_t* Rs = (uint8_t*)malloc((size_t)(R->ntuples > 0 ? R->ntuples : 1) * R->tuple_bytes);
    uint8_t* Ss = (uint8_t*)malloc((size_t)(S->ntuples > 0 ? S->ntuples : 1) * S->tuple_bytes);
    if (!Rs || !Ss) { free(Rs); free(Ss); return -2; }
    orc_sort(R, rk, Rs);
    orc_sort(S, sk, Ss);
    orc_rel r2 = *R; r2.base = Rs;
    orc_rel s2 = *S; s2.base = Ss;
    int ob = 0;
    for (int p = 0; p < nproj; ++p) ob += colsize(proj[p].side ? S : R, proj[p].col);
    uint64_t acc[16] = {0};
    int64_t n = 0, i = 0, j = 0;
    while (i < r2.ntuples && j < s2.ntuples) {
        int64_t a = getcol(&r2, i, rk), b = getcol(&s2, j, sk);
        if (a < b) { ++i; continue; }
        if (b < a) { ++j; continue; }
        int64_t i2 = i, j2 = j;
        while (i2 < r2.ntuples && getcol(&r2, i2, rk) == a) ++i2;
        while (j2 < s2.ntuples && getcol(&s2, j2, sk) == a) ++j2;
        for (int64_t x = i; x < i2; ++x)
            for (int64_t y = j; y < j2; ++y) {
                uint8_t* dst = (out && n < out_capacity) ? out + (size_t)n * ob : NULL;
                for (int p = 0; p < nproj; ++p) {
                    const orc_rel* src = proj[p].side ? &s2 : &r2;
                    int64_t row = proj[p].side ? y : x;
                    acc[p] += (uint64_t)getcol(src, row, proj[p].col);
                    if (dst) {
                        int s = colsize(src, proj[p].col);
                        memcpy(dst, src->base + (size_t)row * src->tuple_bytes + src->col_offset[proj[p].col], s);
                        dst += s;
                    }
                }
                ++n;
            }
        i = i2; j = j2;
    }
    if (out_count) *out_count = n;
    if (sums)
        for (int p = 0; p < nproj; ++p) {
            const orc_rel* src = proj[p].side ? S : R;
            sums[p] = src->col_type[proj[p].col] == ORC_INT32 ? (int64_t)(int32_t)(uint32_t)acc[p] : (int64_t)acc[p];
        }
    free(Rs); free(Ss);
    return n;
}

/* SortLimit (operators/sortlimit.cpp:32-120 init, :131-203 sortHelper,
 * :220-262 scanStart): a list of at most `limit` tuples kept in order.  A
 * tuple is "ahead of" another when it is lexicographically smaller over
 * the `by` columns (greater when asc == 0), the first column deciding
 * unless equal (the allpossible comparator chains, :56-75).  Each arriving
 * tuple walks the list from the head and goes before the first tuple it is
 * ahead of (after all tuples it ties with); when the list is full, the tail
 * drops off, and a tuple that is ahead of none is discarded.  Tuples arrive
 * in input order (the operator runs on thread 0 only, :224-228).  Output:
 * the list from the head, min(limit, n) tuples written to out; returns that
 * count.  The list is held as an index array (insertion by shifting). */
static int orc_ahead(const orc_rel* r, int64_t a, int64_t b, const int* by, int nby, int asc)
{
    for (int c = 0; c < nby; ++c) {
        const int64_t x = getcol(r, a, by[c]), y = getcol(r, b, by[c]);
        if (x == y) continue;
        return asc ? x < y : x > y;
    }
    return 0;
}

int64_t orc_sortlimit(const orc_rel* in, const int* by, int nby, int asc, int64_t limit, uint8_t* out)
{
    if (limit <= 0) return 0;
    int64_t* list = (int64_t*)malloc(sizeof(int64_t) * (size_t)(limit + 1));
    int64_t size = 0;
    for (int64_t i = 0; i < in->ntuples; ++i) {
        /* The list is ordered, so the walk's stopping point (the first
         * tuple this one is ahead of) is found by binary search, and a full
         * list whose tail this tuple is not ahead of rejects it at once. */
        if (size == limit && !orc_ahead(in, i, list[size - 1], by, nby, asc)) continue;
        int64_t lo = 0, hi = size;
        while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if (orc_ahead(in, i, list[mid], by, nby, asc)) hi = mid;
            else lo = mid + 1;
        }
        const int64_t pos = lo;
        memmove(list + pos + 1, list + pos, sizeof(int64_t) * (size_t)(size - pos));
        list[pos] = i;
        if (size < limit) ++size;                   /* else the tail dropped off */
    }
    for (int64_t j = 0; j < size; ++j)
        memcpy(out + (size_t)j * in->tuple_bytes, in->base + (size_t)list[j] * in->tuple_bytes, in->tuple_bytes);
    free(list);
    return size;
}
