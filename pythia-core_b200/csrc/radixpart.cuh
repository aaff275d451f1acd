// Hash partitioning of 16-byte (int64 key, int64 payload) tuples by the
// top bits of a multiplicative hash of the key, shared by the radix
// operators (join, group-by).
//
//   histogram   rj_hist_kernel counts the top `bits` bits of every tuple (or
//               of a strided sample) in shared memory.
//   layout      exact (dense partitions from a full histogram) or sampled
//               (regions sized from the sample with six standard deviations
//               of slack; a region that overflows is reported and the caller
//               redoes the side exactly).
//   passes      one tile pass (<= 9 bits) or two (coarse bits, then the rest
//               inside each coarse partition).  A CTA receives 2048-tuple
//               tiles by bulk copy into a two-deep shared-memory ring, groups
//               a tile by bin in shared memory and writes each bin's run
//               contiguously after one global reservation per (tile, bin).
//   packing     (callers that opt in) when the histogram's reading of the
//               relation shows that key - kbase and payload - pbase both
//               fit in 32 bits for some frame (kbase, pbase), the passes
//               write 8-byte words (key - kbase) | (payload - pbase) << 32
//               instead of 16-byte tuples: frame-of-reference encoding,
//               exact, and half the bytes of every intermediate write and
//               re-read.  A tuple outside the frame (possible when the
//               histogram read a sample) sets a flag and the relation is
//               redone with 16-byte intermediates.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "pyg_internal.cuh"

typedef struct pyg_cdf pyg_cdf;

namespace pyg {

#ifndef PYG_RJ_TILE
#define PYG_RJ_TILE 2048
#endif
#ifndef PYG_RJ_PT_THREADS16
#define PYG_RJ_PT_THREADS16 256
#endif
#ifndef PYG_RJ_PT_THREADS8
#define PYG_RJ_PT_THREADS8 512
#endif
constexpr int RJ_TILE = PYG_RJ_TILE;            // tuples per partition tile
constexpr int RJ_TILE8 = 4096;                  // packed words per partition tile (packed input)
// Partition CTA threads: passes over 16-byte tuples run 8 tuples per thread
// (fewer per-tile steps per tuple; measured 6.9 against 8.0 ms with 512
// threads on the 2^30-tuple probe side), passes over packed words 8 words
// per thread at 512 threads (4.99 against 5.73 ms with 256).
constexpr int RJ_PT_THREADS16 = PYG_RJ_PT_THREADS16;
constexpr int RJ_PT_THREADS8 = PYG_RJ_PT_THREADS8;
constexpr int RJ_MAX_LOCAL_BITS = 9;     // bins of one partition pass
constexpr int RJ_LMAX = 1 << RJ_MAX_LOCAL_BITS;
constexpr int RJ_SPLIT_MAX = 256;        // range mode: splitters per pass segment (<= 2^8 bins)
// Largest fine partition counts (log2); the histogram kernels keep up to
// 2^15 32-bit counters in shared memory.
constexpr int RJ_MAX_FINE_BITS = 16;   // hash mode (histograms run in halves above 2^15 bins)
constexpr int RJ_MAX_RANGE_BITS = 15;  // range mode (one 2^15-counter histogram)
#ifndef PYG_RJ_SAMPLE_LOG2
#define PYG_RJ_SAMPLE_LOG2 22
#endif
// Sampled layouts count every (n >> RJ_SAMPLE_LOG2)-th tuple (2^22 samples:
// at most 0.2 ms for two relations; regions get more slack than with a
// larger sample, which costs device memory, not traffic).
constexpr int RJ_SAMPLE_LOG2 = PYG_RJ_SAMPLE_LOG2;

// Partition bins computed by a learned CDF model instead of a search
// (range partitioning without splitters in the passes).  For a model with
// L leaves over keys (kmin, kmax) and 2^fbits bins:
//   x = (float)(k - kmin) * scale                     normalised key (the
//                                                     offset as unsigned)
//   r = a0 x + b0, l = clamp(floor(L r), 0, L - 1)     root line -> leaf
//   u = clamp(L r - l, 0, 1)                           leaf-local coordinate
//   g = clamp(A_l u + B_l, lo_l, hi_l)                 the leaf's line
//   g = min(g + (masses of the leaf's heavy keys below k), hi_l)
//   bin(k) = min(2^fbits - 1, trunc(g 2^fbits))
// with bin 0 for k <= kmin and the last bin for k >= kmax.  Every step is a
// correctly rounded fp32 operation that does not decrease when its input
// grows (A_l and the masses are >= 0), and hi_l <= lo_{l+1}, so bin(k)
// never decreases with k: the bins are key ranges, and their splitters
// (the first key of each bin, found by bisection over the same function)
// reproduce them exactly.  The model's accuracy only decides how even the
// bins are.
struct RJLeaf {
    float A, B;    // the leaf's line over u
    float lo, hi;  // its range of g
};
struct RJModel {
    const RJLeaf* leaf = nullptr;  // device, L leaves (null: no model)
    const int2* hinfo = nullptr;   // device, per leaf {first heavy key, count}; null without heavy keys
    const long long* hkey = nullptr;  // device, heavy keys ascending
    const float* hw = nullptr;        // device, their masses
    long long kmin = 0, kmax = 0;
    float scale = 0;
    float a0 = 0, b0 = 0;
    int L = 0;
    int fbits = 0;
};

__device__ __forceinline__ unsigned rj_model_bin(const RJModel& m, long long k)
{
    const unsigned last = (1u << m.fbits) - 1u;
    if (k <= m.kmin) return 0u;
    if (k >= m.kmax) return last;
    const float x = __fmul_rn(__ull2float_rn((unsigned long long)k - (unsigned long long)m.kmin), m.scale);
    const float lr = __fmul_rn(__fmaf_rn(m.a0, x, m.b0), (float)m.L);
    const float fl = floorf(lr);
    const int l = fl < 0.f ? 0 : (fl > (float)(m.L - 1) ? m.L - 1 : (int)fl);
    const float u = fminf(1.f, fmaxf(0.f, __fsub_rn(lr, (float)l)));
    const RJLeaf p = m.leaf[l];
    float g = fminf(p.hi, fmaxf(p.lo, __fmaf_rn(p.A, u, p.B)));
    if (m.hinfo) {
        const int2 hi = m.hinfo[l];
        for (int h = hi.x; h < hi.x + hi.y && m.hkey[h] < k; ++h) g = __fadd_rn(g, m.hw[h]);
        g = fminf(g, p.hi);
    }
    const float b = __fmul_rn(g, (float)(1u << m.fbits));
    return b >= (float)last ? last : (unsigned)b;
}

// Bins of a trained CDF model (cdf.cu): *out refers to device tables the
// model keeps until pyg_cdf_free.  model_splitters: the 2^fbits - 1
// splitters of those bins into host array out (bin(k) = number of
// splitters <= k).
int cdf_bin_model(pyg_ctx* ctx, const pyg_cdf* m, int fbits, RJModel* out);
int model_splitters(pyg_ctx* ctx, const RJModel& m, int64_t* out);

// The 64-bit code whose top fbits bits are the model's bin (the hash
// operators take their partition bits from the top of such a word).
__device__ __forceinline__ uint64_t rj_model_code(const RJModel& m, long long k)
{
    return (uint64_t)rj_model_bin(m, k) << (64 - m.fbits);
}

// Host-side layout of one relation's partitions.
struct RJLayout {
    bool sampled = false;
    // Packed (8-byte) intermediates and their frame: key = kbase + low 32
    // bits, payload = pbase + high 32 bits (64-bit wrap-around arithmetic).
    // Packed layouts start every region at an even word, so that each
    // region's tiles begin 16-byte aligned for bulk copies.
    bool packed = false;
    unsigned long long kbase = 0, pbase = 0;
    std::vector<unsigned long long> fstart;  // F + 1 fine region starts
    std::vector<unsigned long long> fcap;    // F fine region capacities (sampled)
    std::vector<unsigned long long> cstart;  // C + 1 coarse region starts
    std::vector<unsigned long long> ccap;    // C coarse region capacities (sampled)
    std::vector<unsigned long long> tiles2;  // C + 1 tile prefix of the second pass (exact)
    std::vector<unsigned long long> count;   // F tuples per fine partition, once known
    unsigned long long p1 = 0, p2 = 0;       // tuples in the pass-1 / pass-2 buffers
    unsigned long long tiles2_max = 0;       // upper bound of the second pass's tiles (sampled)
};

// Exact layout from exact per-fine-partition counts h (F = h.size()).
// pack: regions rounded up to an even number of words (packed layouts).
void layout_exact(const std::vector<unsigned long long>& h, int C, int sub, RJLayout& L, bool pack = false);
// Sampled layout from the counts sc of every step-th tuple: each region is
// sized with six standard deviations of slack.
void layout_sampled(const std::vector<unsigned long long>& sc, long long step, int C, int sub, RJLayout& L,
                    bool pack = false);
// Frame of a packed layout from the key and payload ranges seen by the
// histogram ([kmin, kmax], [pmin, pmax], signed).  exact: the ranges cover
// every tuple; else they come from a sample and must leave a margin of at
// least 2^30 on each side.  Offsets stay below 2^32 - 1.  key_base (when
// given) is a key frame shared with another relation (common_key_frame).
// Returns false when no frame fits.
bool pack_frame(long long kmin, long long kmax, long long pmin, long long pmax, bool exact, RJLayout& L,
                const unsigned long long* key_base = nullptr);
// One key frame covering two relations' key ranges mm = {kmin, kmax, ...},
// so that their packed words carry comparable 32-bit key offsets.
bool common_key_frame(const long long* mm0, bool exact0, const long long* mm1, bool exact1, unsigned long long* base);
// Bytes of one intermediate element of a layout.
inline int elem_bytes(const RJLayout& L) { return L.packed ? 8 : 16; }

// Device copy of one relation's partition metadata (u64 words).
struct RJSideDev {
    unsigned long long *fstart, *fcap, *cstart, *ccap, *cur1, *cur2, *tiles2, *whole, *wtiles;
    static size_t words(int F, int C) { return (size_t)(F + 1) + F + (C + 1) + C + C + F + (C + 1) + 4; }
    void carve(unsigned long long* m, int F, int C)
    {
        fstart = m;
        fcap = fstart + F + 1;
        cstart = fcap + F;
        ccap = cstart + C + 1;
        cur1 = ccap + C;
        cur2 = cur1 + C;
        tiles2 = cur2 + F;
        whole = tiles2 + C + 1;
        wtiles = whole + 2;
    }
};

// Copies a layout to the device and zeroes its cursors.
int upload_layout(pyg_ctx* ctx, const RJLayout& L, const RJSideDev& d, int F, int C, int64_t n);
// Histogram of the top FB hash bits of in[0], in[step], ... into hist
// (2^FB device words, zeroed here).  mm (optional, 4 words): receives the
// minimum and maximum key and payload of the tuples read, as signed
// {kmin, kmax, pmin, pmax}.
int hist_launch(pyg_ctx* ctx, const longlong2* in, int64_t n, int64_t step, int FB, unsigned long long* hist,
                long long* mm = nullptr, const RJModel* model = nullptr);
// Partition pass(es) of one relation into P1 (and P2 when two): *err is set
// if a tile's bulk copy never landed, *ovf if a sampled region overflowed,
// *frame if a tuple fell outside a packed layout's frame.  Afterwards
// d.cur2 holds the tuples written per fine partition.
// Range mode when csplit is set: pass 1 bins by the 2^CB - 1 coarse
// splitters, pass 2 by the fine splitters (F - 1, ascending; coarse
// splitter i = fine splitter (i + 1) * 2^(FB - CB) - 1).
int run_passes(pyg_ctx* ctx, const longlong2* in, int64_t n, const RJLayout& L, const RJSideDev& d, bool two, int FB,
               int CB, void* P1, void* P2, unsigned* err, unsigned* ovf, const long long* csplit = nullptr,
               const long long* fsplit = nullptr, unsigned* frame = nullptr, cudaEvent_t between = nullptr,
               const RJModel* model = nullptr);
// Device bytes of a layout's pass buffers (packed buffers get 16 bytes of
// tail so that the last tile's 16-byte-rounded copy stays inside).
inline size_t pass_bytes(const RJLayout& L, unsigned long long words)
{
    return (size_t)words * elem_bytes(L) + (L.packed ? 16 : 0);
}
// Histogram of range bins (see run_passes) of in[0], in[step], ...
int hist_launch_range(pyg_ctx* ctx, const longlong2* in, int64_t n, int64_t step, int CB, int sub,
                      const long long* csplit, const long long* fsplit, unsigned long long* hist);
// One relation for rp_partition_sides.  In: in, n, allow_sample, the
// splitters (range mode) and an optional event recorded after the
// relation's passes.  Out: the layout (counts included), the pass buffers
// (the caller frees them), the tuples its histogram read and whether a
// sampled region overflowed (then the relation was redone exactly).
struct RPSide {
    const longlong2* in = nullptr;
    int64_t n = 0;
    bool allow_sample = true;
    bool allow_pack = false;  // the caller reads packed intermediates (L.packed tells)
    const long long* csplit = nullptr;
    const long long* fsplit = nullptr;
    // Learned-model bins (rj_model_bin) instead of hash bits; model->fbits
    // must equal the partition bits.
    const RJModel* model = nullptr;
    cudaEvent_t begin = nullptr;  // recorded before the first pass (optional)
    cudaEvent_t mid = nullptr;    // between the two passes (optional)
    cudaEvent_t done = nullptr;
    RJLayout L;
    void* P1 = nullptr;
    void* P2 = nullptr;
    int64_t hist_tuples = 0;
    bool overflowed = false;
};

// Partitions one or two relations with the same bits: both histograms, one
// host round trip, both relations' passes (the second relation's layout is
// formed while the first one's passes run), one more round trip for the
// counts and flags, and an exact redo of a relation whose sampled region
// overflowed or whose packed frame missed a tuple (the redo is unpacked).
// flags: 4 device words per relation (bulk copy never landed, region
// overflow, frame miss, unused); hflags: as many pinned host words.
// hist_done (optional) is recorded after the histograms.
// share_key_frame: pack both relations with one key frame when their key
// ranges fit one (a redone relation gets its own frame).
int rp_partition_sides(pyg_ctx* ctx, RPSide* sd, int ns, int FB, bool two, unsigned* flags, unsigned* hflags,
                       cudaEvent_t hist_done, bool share_key_frame = false);

// Partitions one relation into 2^FB partitions (hash bits, or ranges when
// csplit is set; two passes when `two`): histogram (sampled when allowed
// and n >= 2^25), layout, passes, and an exact redo if a sampled region
// overflowed.  On success the partitions are in (two ? *P2 : *P1) at
// L.fstart with L.count tuples each; the caller frees *P1 and *P2.  flags:
// two device words (bulk copy never landed, region overflow); hflags: two
// pinned host words; both need 4 words (see rp_partition_sides).  hist_ms /
// hist_tuples (optional): the histogram's time and the tuples it read.
int rp_partition(pyg_ctx* ctx, const longlong2* in, int64_t n, int FB, bool two, bool allow_sample,
                 const long long* csplit, const long long* fsplit, RJLayout& L, void** P1, void** P2,
                 unsigned* flags, unsigned* hflags, float* hist_ms = nullptr, int64_t* hist_tuples = nullptr);

// Hash of the radix operators: multiplication by 2^64 / golden ratio
// (Fibonacci hashing) after three xor-shifts.  Bit j of the product depends
// on bits 0..j of the shifted key, so the top bits mix the whole key:
// partitions take the top `fb` bits and shared-memory tables the 32 bits
// below them.  Dense key ranges spread almost evenly over the partitions
// and over the slots of a partition's table (consecutive multiples of an
// irrational fraction; the xor-shifts permute aligned blocks of 2^16 keys
// onto themselves, so a dense range keeps this).  Without the xor-shifts,
// keys that are multiples of 2^16 or of a Fibonacci number (987, 1597, ...)
// see the product's weaker lower bits and pile into long probe chains
// (30-110 probes per insert at a third of the table instead of about 1.3);
// with these three shifts, strides, Fibonacci multiples and packed
// (a << s) | b keys stay at 1.0-2.1.
constexpr uint64_t kRjHashMul = 0x9E3779B97F4A7C15ULL;
__host__ __device__ __forceinline__ uint64_t rj_hash(uint64_t k)
{
    k ^= k >> 32;
    k ^= k >> 21;
    k ^= k >> 16;
    return k * kRjHashMul;
}

// Slot of key k in a shared-memory table of TS slots, for keys of one
// partition of 2^fb (fb = 0: one partition): multiply-high of the 32 hash
// bits below the partition bits.
__device__ __forceinline__ unsigned rj_slot(uint64_t k, int fb, unsigned TS)
{
    return __umulhi((unsigned)(rj_hash(k) >> (32 - fb)), TS);
}

}  // namespace pyg
