// Seeded synthetic relations for benchmarks and tests, generated on the
// device so full-size inputs (GBs) take milliseconds.
//
//  * Primary keys: 1 + pi(i), where pi is a bijection of [0, n): a 4-round
//    Feistel network on the smallest even bit width covering n, with cycle
//    walking for n not a power of four.
//  * Foreign keys: a rank r ~ Zipf(theta) over [1, nkeys] (uniform when
//    theta == 0) mapped to the key 1 + pi(r - 1), so the hot ranks land on
//    scattered keys of the primary relation.  Zipf variates use the
//    rejection-inversion method of Hoermann and Derflinger ("Rejection-
//    inversion to generate variates from monotone discrete distributions",
//    ACM TOMACS 6(3), 1996), which needs no CDF table.
#include "pyg_internal.cuh"

namespace pyg {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

struct Feistel {
    int half;          // bits per half
    uint64_t n;
    uint64_t keys[4];
};

__host__ __device__ __forceinline__ uint64_t feistel_once(const Feistel& f, uint64_t x)
{
    const uint64_t mask = (1ULL << f.half) - 1;
    uint64_t l = x >> f.half, r = x & mask;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        uint64_t t = l ^ (splitmix64(r ^ f.keys[i]) & mask);
        l = r;
        r = t;
    }
    return (l << f.half) | r;
}

__host__ __device__ __forceinline__ uint64_t permute(const Feistel& f, uint64_t x)
{
    do {
        x = feistel_once(f, x);
    } while (x >= f.n);
    return x;
}

static Feistel make_feistel(uint64_t n, uint64_t seed)
{
    Feistel f;
    int bits = 2;
    while (bits < 64 && (1ULL << bits) < n) ++bits;
    if (bits & 1) ++bits;
    f.half = bits / 2;
    f.n = n;
    for (int i = 0; i < 4; ++i) f.keys[i] = splitmix64(seed * 4 + i + 0x1234567ULL);
    return f;
}

__device__ __forceinline__ double u01(uint64_t x) { return (double)(splitmix64(x) >> 11) * 0x1.0p-53; }

// Zipf(s) over {1..N} by rejection-inversion.
struct ZipfRI {
    double s, hx1, hn, sq;
    uint64_t N;
};

__host__ __device__ __forceinline__ double expm1_over(double x) { return fabs(x) > 1e-8 ? expm1(x) / x : 1.0 + x * 0.5; }
__host__ __device__ __forceinline__ double log1p_over(double x) { return fabs(x) > 1e-8 ? log1p(x) / x : 1.0 - x * 0.5; }
// H(x) = integral of x^-s: (x^(1-s) - 1)/(1-s), log(x) when s == 1.
__host__ __device__ __forceinline__ double zH(double s, double x)
{
    double lx = log(x);
    return expm1_over((1.0 - s) * lx) * lx;
}
__host__ __device__ __forceinline__ double zh(double s, double x) { return exp(-s * log(x)); }
__host__ __device__ __forceinline__ double zHinv(double s, double y)
{
    double t = y * (1.0 - s);
    if (t < -1.0) t = -1.0;
    return exp(log1p_over(t) * y);
}

static ZipfRI make_zipf(double s, uint64_t N)
{
    ZipfRI z;
    z.s = s;
    z.N = N;
    z.hx1 = zH(s, 1.5) - 1.0;
    z.hn = zH(s, (double)N + 0.5);
    z.sq = 2.0 - zHinv(s, zH(s, 2.5) - zh(s, 2.0));
    return z;
}

__device__ __forceinline__ uint64_t zipf_sample(const ZipfRI& z, uint64_t stream)
{
    for (uint64_t tries = 0; tries < 64; ++tries) {
        double u = z.hn + u01(stream + tries * 0x632be59bd9b4e019ULL) * (z.hx1 - z.hn);
        double x = zHinv(z.s, u);
        double kf = floor(x + 0.5);
        if (kf < 1.0) kf = 1.0;
        if (kf > (double)z.N) kf = (double)z.N;
        if (kf - x <= z.sq || u >= zH(z.s, kf + 0.5) - zh(z.s, kf)) return (uint64_t)kf;
    }
    return 1;  // acceptance probability per try is high; this is unreachable in practice
}

__global__ void gen_pk_kernel(longlong2* __restrict__ out, int64_t n, int64_t mul, Feistel f)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        long long k = 1 + (long long)permute(f, (uint64_t)i);
        out[i] = make_longlong2(k, k * mul);
    }
}

__global__ void gen_fk_kernel(longlong2* __restrict__ out, int64_t n, int64_t nkeys, int uniform, ZipfRI z, Feistel f,
                              int64_t vmax, uint64_t seed)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t st = splitmix64(seed ^ ((uint64_t)i * 0xd1b54a32d192ed03ULL));
        uint64_t r;
        if (uniform) r = __umul64hi(splitmix64(st), (uint64_t)nkeys);
        else r = zipf_sample(z, st) - 1;
        long long fk = 1 + (long long)permute(f, r);
        long long v = (long long)__umul64hi(splitmix64(st ^ 0x5555555555555555ULL), (uint64_t)vmax);
        out[i] = make_longlong2(fk, v);
    }
}

}  // namespace pyg

using namespace pyg;

extern "C" {

int pyg_gen_pk(pyg_ctx* ctx, void* out, int64_t n, int64_t payload_mul, uint64_t seed)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n < 0 || (n > 0 && !out) || ((uintptr_t)out % 16)) {
        set_error("pyg_gen_pk: bad output");
        return PYG_ERR_ARG;
    }
    if (n == 0) return PYG_OK;
    Feistel f = make_feistel((uint64_t)n, seed);
    gen_pk_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>((longlong2*)out, n, payload_mul, f);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

int pyg_gen_fk(pyg_ctx* ctx, void* out, int64_t n, int64_t nkeys, double theta, uint64_t seed_keys, int64_t vmax,
               uint64_t seed)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n < 0 || nkeys < 1 || vmax < 1 || theta < 0 || (n > 0 && !out) || ((uintptr_t)out % 16)) {
        set_error("pyg_gen_fk: bad arguments");
        return PYG_ERR_ARG;
    }
    if (n == 0) return PYG_OK;
    Feistel f = make_feistel((uint64_t)nkeys, seed_keys);
    ZipfRI z = make_zipf(theta > 0 ? theta : 1.0, (uint64_t)nkeys);
    gen_fk_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>((longlong2*)out, n, nkeys, theta == 0.0, z, f,
                                                                        vmax, seed);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

}  // extern "C"
