// Learned CDF splitter: a two-level piecewise-linear model trained on the
// GPU with the library's own forward / backward kernels.
//
// Model (all formulas also in include/pyg_learned.h):
//   x = (key - lo) * scale                      normalised key in [0, 1]
//   r = a0 * x + b0                             root line (monotone: a0 >= 0)
//   l = clamp(floor(L * r), 0, L - 1)           leaf
//   u = clamp(L * r - l, 0, 1)                  leaf-local coordinate
//   cdf = ylo_l + (yhi_l - ylo_l) * clamp(a_l * u + b_l, 0, 1)
// The root is fitted to y_i = i / n of the sorted sample, then each leaf to
// its samples' targets normalised to the leaf's y range.  The root is the
// least-squares line (one pass of sums; it minimises the root's loss, so no
// steps follow), and so is each leaf to start with; the leaves then take
// `epochs` full-batch steps of projected Adam (slopes kept >= 0 so the
// model stays monotone) with the step size decayed to 1% over the epochs,
// through the forward and backward kernels.  Residual arithmetic is fp64;
// parameters are fp32.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/pyg_learned.h"
#include "primitives.cuh"
#include "radixpart.cuh"

struct pyg_cdf {
    int L = 0;
    double key_lo = 0, key_scale = 0;
    int64_t kmin = 0, kmax = 0;
    float a0 = 1, b0 = 0;
    std::vector<float> la, lb;      // leaf slope / intercept
    std::vector<double> ylo, yhi;   // leaf target range
    float* d_params = nullptr;      // device: a0, b0, then (a, b) per leaf
    double* d_yr = nullptr;         // device: (ylo, yhi) per leaf
    int64_t n_sample = 0, distinct = 0, f1 = 0;
    // Heavy keys: sample runs of at least n/4096 equal keys, kept as exact
    // point masses beside the linear leaves, which are fitted to the rest
    // of the sample (the continuous part C).  The model's CDF is
    //   F(k) = (1 - W) C(k) + sum of w_h over heavy keys h < k,
    // with w_h the share of the sample holding key h and W their total.
    std::vector<int64_t> heavy_key;
    std::vector<double> heavy_w, heavy_before;  // mass, mass of the heavy keys below it
    double wheavy = 0;
    int64_t* d_hkeys = nullptr;    // device copies for predict
    double* d_hbefore = nullptr;
    double* d_hw = nullptr;
    // Device tables of the model's own bins (pyg::cdf_bin_model), built on
    // first use: L leaves, then the heavy keys and their masses.
    mutable pyg::RJLeaf* d_bleaf = nullptr;
    mutable int2* d_bhinfo = nullptr;
    mutable long long* d_bhkey = nullptr;
    mutable float* d_bhw = nullptr;
};

namespace pyg {

constexpr int CDF_THREADS = 256;

struct LeafStat {
    unsigned long long lo, hi;  // first index, last index + 1 (lo = ~0 when empty)
};

__device__ __forceinline__ double norm_key(int64_t k, double lo, double scale)
{
    return (double)(float)(((double)k - lo) * scale);
}

// Root forward + backward over the sorted sample: acc[0] += e^2,
// acc[1] += e*x, acc[2] += e with e = a0*x + b0 - y.
__global__ void __launch_bounds__(CDF_THREADS) root_fwd_bwd_kernel(const int64_t* __restrict__ keys, int64_t n,
                                                                   double lo, double scale,
                                                                   const float* __restrict__ params,
                                                                   double* __restrict__ acc)
{
    const double a0 = params[0], b0 = params[1];
    double s0 = 0, s1 = 0, s2 = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x = norm_key(keys[i], lo, scale);
        double y = (double)i / (double)n;
        double e = a0 * x + b0 - y;
        s0 += e * e;
        s1 += e * x;
        s2 += e;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], s0);
        atomicAdd(&acc[1], s1);
        atomicAdd(&acc[2], s2);
    }
}

// Adam step on `count` parameters with gradient g[i] = gscale[i/2] * raw[i]
// (raw accumulated by a backward kernel); slopes (even i) projected to >= 0.
// Zeroes the raw gradient for the next epoch.
__global__ void adam_kernel(float* __restrict__ p, double* __restrict__ raw, const double* __restrict__ gscale,
                            float* __restrict__ m, float* __restrict__ v, int count, float lr, int t)
{
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        double gs = gscale[i >> 1];
        float g = (float)(raw[i] * gs);
        raw[i] = 0;
        if (gs == 0) continue;
        float mi = b1 * m[i] + (1 - b1) * g;
        float vi = b2 * v[i] + (1 - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        float mh = mi / (1 - powf(b1, (float)t));
        float vh = vi / (1 - powf(b2, (float)t));
        float q = p[i] - lr * mh / (sqrtf(vh) + eps);
        if ((i & 1) == 0 && q < 0) q = 0;
        p[i] = q;
    }
}

// Leaf of every sample and each leaf's index range.
__global__ void assign_kernel(const int64_t* __restrict__ keys, int64_t n, double lo, double scale,
                              const float* __restrict__ params, int L, int* __restrict__ leaf, double* __restrict__ u,
                              LeafStat* __restrict__ st)
{
    const double a0 = params[0], b0 = params[1];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x = norm_key(keys[i], lo, scale);
        double r = a0 * x + b0;
        double fl = floor(L * r);
        int l = fl < 0 ? 0 : (fl > L - 1 ? L - 1 : (int)fl);
        double uu = L * r - l;
        uu = uu < 0 ? 0 : (uu > 1 ? 1 : uu);
        leaf[i] = l;
        u[i] = uu;
        atomicMin(&st[l].lo, (unsigned long long)i);
        atomicMax(&st[l].hi, (unsigned long long)(i + 1));
    }
}

__global__ void leaf_range_kernel(const LeafStat* __restrict__ st, int64_t n, int L, double* __restrict__ yr,
                                  double* __restrict__ gscale)
{
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < L; l += gridDim.x * blockDim.x) {
        bool empty = st[l].lo == ~0ULL;
        double ylo = empty ? 0 : (double)st[l].lo / (double)n;
        double yhi = empty ? 0 : (double)st[l].hi / (double)n;
        yr[2 * l] = ylo;
        yr[2 * l + 1] = yhi;
        // d/dparam of (1/L) * mean over the leaf: (1/L) * 2 / n_l.
        gscale[1 + l] = empty ? 0 : 2.0 / ((double)(st[l].hi - st[l].lo) * (double)L);
    }
}

// Leaf forward: residual g_i = a_l u_i + b_l - t_i and loss sum per leaf.
__global__ void __launch_bounds__(CDF_THREADS) leaf_forward_kernel(int64_t n, const int* __restrict__ leaf,
                                                                   const double* __restrict__ u,
                                                                   const double* __restrict__ yr,
                                                                   const float* __restrict__ params,
                                                                   double* __restrict__ g, double* __restrict__ lsum)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int l = leaf[i];
        double y = (double)i / (double)n;
        double ylo = yr[2 * l], yhi = yr[2 * l + 1];
        double t = yhi > ylo ? (y - ylo) / (yhi - ylo) : 0.0;
        double e = (double)params[2 + 2 * l] * u[i] + (double)params[3 + 2 * l] - t;
        g[i] = e;
        if (lsum) atomicAdd(&lsum[l], e * e);
    }
}

// Leaf backward: raw[2l] += g u, raw[2l+1] += g (summed per leaf; samples
// are sorted so a warp is usually inside one leaf and reduces first).
__global__ void __launch_bounds__(CDF_THREADS) leaf_backward_kernel(int64_t n, const int* __restrict__ leaf,
                                                                    const double* __restrict__ u,
                                                                    const double* __restrict__ g,
                                                                    double* __restrict__ raw)
{
    const unsigned lane = threadIdx.x & 31;
    for (int64_t wb = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u); wb < n;
         wb += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = wb + lane;
        bool valid = i < n;
        int l = valid ? leaf[i] : -1;
        double ga = valid ? g[i] * u[i] : 0, gb = valid ? g[i] : 0;
        int l0 = __shfl_sync(0xffffffffu, l, 0);
        bool uniform = __all_sync(0xffffffffu, !valid || l == l0);
        if (uniform) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                ga += __shfl_xor_sync(0xffffffffu, ga, o);
                gb += __shfl_xor_sync(0xffffffffu, gb, o);
            }
            if (lane == 0) {
                atomicAdd(&raw[2 + 2 * l0], ga);
                atomicAdd(&raw[3 + 2 * l0], gb);
            }
        } else if (valid) {
            atomicAdd(&raw[2 + 2 * l], ga);
            atomicAdd(&raw[3 + 2 * l], gb);
        }
    }
}

// Closed-form start (the linear models of a recursive model index, Kraska
// et al., SIGMOD 2018, each fitted by least squares): root sums over the
// sorted sample, acc = {sum x, sum x^2, sum y, sum x y} with y = i / n.
__global__ void __launch_bounds__(CDF_THREADS) root_ls_kernel(const int64_t* __restrict__ keys, int64_t n, double lo,
                                                              double scale, double* __restrict__ acc)
{
    double sx = 0, sxx = 0, sy = 0, sxy = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = norm_key(keys[i], lo, scale), y = (double)i / (double)n;
        sx += x;
        sxx += x * x;
        sy += y;
        sxy += x * y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sxx += __shfl_xor_sync(0xffffffffu, sxx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sxy += __shfl_xor_sync(0xffffffffu, sxy, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], sx);
        atomicAdd(&acc[1], sxx);
        atomicAdd(&acc[2], sy);
        atomicAdd(&acc[3], sxy);
    }
}

// Least-squares line through c points from their sums; the slope is kept
// >= 0 (a monotone model), the intercept refitted when it is clamped.
__device__ __forceinline__ void ls_line(double c, double sx, double sxx, double sy, double sxy, float* a, float* b)
{
    if (c < 1) {
        *a = 1.f;
        *b = 0.f;
        return;
    }
    const double den = c * sxx - sx * sx;
    double s = den > 1e-12 * c * c ? (c * sxy - sx * sy) / den : 0.0;
    if (s < 0) s = 0;
    *a = (float)s;
    *b = (float)((sy - s * sx) / c);
}

__global__ void root_solve_kernel(const double* __restrict__ acc, int64_t n, float* __restrict__ params)
{
    ls_line((double)n, acc[0], acc[1], acc[2], acc[3], &params[0], &params[1]);
}

// Per-leaf least-squares sums of the leaf-local target t against u:
// s[5l .. 5l+4] = {count, sum u, sum u^2, sum t, sum u t}.
__global__ void __launch_bounds__(CDF_THREADS) leaf_ls_kernel(int64_t n, const int* __restrict__ leaf,
                                                              const double* __restrict__ u,
                                                              const double* __restrict__ yr, double* __restrict__ s)
{
    const unsigned lane = threadIdx.x & 31;
    for (int64_t wb = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u); wb < n;
         wb += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = wb + lane;
        const bool valid = i < n;
        const int l = valid ? leaf[i] : -1;
        double v[5] = {0, 0, 0, 0, 0};
        if (valid) {
            const double ylo = yr[2 * l], yhi = yr[2 * l + 1];
            const double t = yhi > ylo ? ((double)i / (double)n - ylo) / (yhi - ylo) : 0.0;
            const double uu = u[i];
            v[0] = 1;
            v[1] = uu;
            v[2] = uu * uu;
            v[3] = t;
            v[4] = uu * t;
        }
        const int l0 = __shfl_sync(0xffffffffu, l, 0);
        if (__all_sync(0xffffffffu, !valid || l == l0)) {
#pragma unroll
            for (int k = 0; k < 5; ++k)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
            if (lane == 0)
                for (int k = 0; k < 5; ++k) atomicAdd(&s[5 * l0 + k], v[k]);
        } else if (valid) {
            for (int k = 0; k < 5; ++k) atomicAdd(&s[5 * l + k], v[k]);
        }
    }
}

__global__ void leaf_solve_kernel(const double* __restrict__ s, int L, float* __restrict__ params)
{
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < L; l += gridDim.x * blockDim.x) {
        const double* q = s + 5 * l;
        ls_line(q[0], q[1], q[2], q[3], q[4], &params[2 + 2 * l], &params[3 + 2 * l]);
    }
}

__global__ void root_to_raw_kernel(const double* __restrict__ acc, double* __restrict__ raw)
{
    raw[0] = acc[1];
    raw[1] = acc[2];
}

// F(k) = (1 - W) C(k) + (mass of the heavy keys below k): C from the root
// and leaf of k, the heavy part by binary search over the nh heavy keys.
__global__ void predict_kernel(const int64_t* __restrict__ keys, int64_t n, double lo, double scale,
                               const float* __restrict__ params, const double* __restrict__ yr, int L,
                               const int64_t* __restrict__ hkeys, const double* __restrict__ hbefore,
                               const double* __restrict__ hw, int nh, double W, float* __restrict__ out)
{
    const double a0 = params[0], b0 = params[1];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = keys[i];
        double x = norm_key(k, lo, scale);
        double r = a0 * x + b0;
        double fl = floor(L * r);
        int l = fl < 0 ? 0 : (fl > L - 1 ? L - 1 : (int)fl);
        double uu = L * r - l;
        uu = uu < 0 ? 0 : (uu > 1 ? 1 : uu);
        double f = (double)params[2 + 2 * l] * uu + (double)params[3 + 2 * l];
        f = f < 0 ? 0 : (f > 1 ? 1 : f);
        const double c = yr[2 * l] + (yr[2 * l + 1] - yr[2 * l]) * f;
        int a = 0, b = nh;  // heavy keys < k: the first index with hkeys >= k
        while (a < b) {
            const int mid = (a + b) >> 1;
            if (hkeys[mid] < k) a = mid + 1;
            else b = mid;
        }
        const double below = a > 0 ? hbefore[a - 1] + hw[a - 1] : 0.0;
        out[i] = (float)((1.0 - W) * c + below);
    }
}

// Copies the sorted sample without its heavy runs [starts[r], ends[r]),
// r < nr, ascending: out[i - cum[j]] = k[i] for i outside every run, where
// j counts the runs starting at or before i and cum[j] is their length.
__global__ void drop_runs_kernel(const int64_t* __restrict__ k, int64_t n, const long long* __restrict__ starts,
                                 const long long* __restrict__ ends, const long long* __restrict__ cum, int nr,
                                 int64_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int a = 0, b = nr;
        while (a < b) {
            const int mid = (a + b) >> 1;
            if (starts[mid] <= i) a = mid + 1;
            else b = mid;
        }
        if (a > 0 && i < ends[a - 1]) continue;
        out[i - cum[a]] = k[i];
    }
}

__global__ void run_stats_kernel(const int64_t* __restrict__ k, int64_t n, unsigned long long* out)
{
    unsigned long long d = 0, f1 = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        bool start = i == 0 || k[i] != k[i - 1];
        bool end = i == n - 1 || k[i] != k[i + 1];
        d += start;
        f1 += start && end;
    }
    d = warp_sum_u64(d);
    f1 = warp_sum_u64(f1);
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&out[0], d);
        atomicAdd(&out[1], f1);
    }
}

// Runs of at least `thr` equal keys in the sorted sample: (key, first, end).
__global__ void heavy_runs_kernel(const int64_t* __restrict__ k, int64_t n, int64_t thr, longlong2* __restrict__ out,
                                  long long* __restrict__ ends, unsigned long long* count, int cap)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (i > 0 && k[i] == k[i - 1]) continue;
        if (i + thr - 1 >= n || k[i + thr - 1] != k[i]) continue;
        int64_t lo = i + thr - 1, hi = n;  // upper bound of k[i]
        while (lo < hi) {
            int64_t mid = lo + ((hi - lo) >> 1);
            if (k[mid] <= k[i]) lo = mid + 1;
            else hi = mid;
        }
        unsigned long long e = atomicAdd(count, 1ULL);
        if ((int)e < cap) {
            out[e] = make_longlong2(k[i], i);
            ends[e] = lo;
        }
    }
}

__global__ void to_signed_kernel(const uint64_t* __restrict__ in, int64_t n, int64_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = from_sortable(in[i]);
}

__global__ void to_sortable_kernel(const int64_t* __restrict__ in, int64_t n, uint64_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = to_sortable(in[i]);
}

// Sorted copy of n device keys into *sorted (device, caller frees).
int sort_keys(pyg_ctx* ctx, const int64_t* keys, int64_t n, int64_t** sorted)
{
    uint64_t* buf;
    int rc = dalloc(ctx, (void**)&buf, (size_t)2 * (n > 0 ? n : 1) * 8);
    if (rc) return rc;
    int g = grid_for(ctx, n, 256, 4, 8);
    if (n > 0) {
        to_sortable_kernel<<<g, 256, 0, ctx->stream>>>(keys, n, buf);
        PYG_LAUNCHED(ctx);
    }
    int b = 0, e = 0, alt = 0;
    if (!(rc = key_bit_range(ctx, buf, n, &b, &e))) rc = radix_sort_pairs(ctx, buf, nullptr, buf + n, nullptr, n, b, e, &alt);
    if (rc) {
        dfree(ctx, buf);
        return rc;
    }
    if ((rc = dalloc(ctx, (void**)sorted, (size_t)(n > 0 ? n : 1) * 8))) {
        dfree(ctx, buf);
        return rc;
    }
    if (n > 0) {
        to_signed_kernel<<<g, 256, 0, ctx->stream>>>(alt ? buf + n : buf, n, *sorted);
        PYG_LAUNCHED(ctx);
    }
    dfree(ctx, buf);
    return PYG_OK;
}

// Device workspace for one forward/backward pass over a sorted sample.
struct CdfWork {
    int* leaf = nullptr;
    double* u = nullptr;
    double* g = nullptr;
    double* raw = nullptr;     // 2 + 2L raw gradient sums
    double* gscale = nullptr;  // 1 + L gradient scales (root, leaves)
    double* acc = nullptr;     // root: e^2, e x, e ; then per-leaf loss sums (L)
    LeafStat* st = nullptr;
    double* ls = nullptr;      // least-squares sums: 4 (root), then 5 per leaf
    void release(pyg_ctx* ctx)
    {
        dfree(ctx, leaf); dfree(ctx, u); dfree(ctx, g); dfree(ctx, raw); dfree(ctx, gscale); dfree(ctx, acc);
        dfree(ctx, st); dfree(ctx, ls);
    }
    int alloc(pyg_ctx* ctx, int64_t n, int L)
    {
        int rc;
        if ((rc = dalloc(ctx, (void**)&leaf, (size_t)n * 4))) return rc;
        if ((rc = dalloc(ctx, (void**)&u, (size_t)n * 8))) return rc;
        if ((rc = dalloc(ctx, (void**)&g, (size_t)n * 8))) return rc;
        if ((rc = dalloc(ctx, (void**)&raw, (size_t)(2 + 2 * L) * 8))) return rc;
        if ((rc = dalloc(ctx, (void**)&gscale, (size_t)(1 + L) * 8))) return rc;
        if ((rc = dalloc(ctx, (void**)&acc, (size_t)(3 + L) * 8))) return rc;
        if ((rc = dalloc(ctx, (void**)&st, (size_t)L * sizeof(LeafStat)))) return rc;
        if ((rc = dalloc(ctx, (void**)&ls, (size_t)(4 + 5 * L) * 8))) return rc;
        PYG_CUDA(cudaMemsetAsync(raw, 0, (size_t)(2 + 2 * L) * 8, ctx->stream));
        PYG_CUDA(cudaMemsetAsync(ls, 0, (size_t)(4 + 5 * L) * 8, ctx->stream));
        return PYG_OK;
    }
};

// Assigns leaves with the current root and computes leaf target ranges and
// gradient scales.
static int cdf_assign(pyg_ctx* ctx, CdfWork& w, const int64_t* keys, int64_t n, int L, double lo, double scale,
                      const float* d_params, double* d_yr)
{
    PYG_CUDA(cudaMemsetAsync(w.st, 0xFF, (size_t)L * sizeof(LeafStat), ctx->stream));
    // hi must start at 0 for atomicMax: set every second word to zero.
    std::vector<LeafStat> init(L);
    for (auto& s : init) { s.lo = ~0ULL; s.hi = 0; }
    PYG_CUDA(cudaMemcpyAsync(w.st, init.data(), (size_t)L * sizeof(LeafStat), cudaMemcpyHostToDevice, ctx->stream));
    int gr = grid_for(ctx, n, CDF_THREADS, 4, 8);
    assign_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(keys, n, lo, scale, d_params, L, w.leaf, w.u, w.st);
    PYG_LAUNCHED(ctx);
    leaf_range_kernel<<<grid_for(ctx, L, 256, 1, 4), 256, 0, ctx->stream>>>(w.st, n, L, d_yr, w.gscale);
    PYG_LAUNCHED(ctx);
    return PYG_OK;  // `init` was staged by the (pageable) copy before it returned
}

// Packed key words of every step-th tuple (m of them).
__global__ void key_sample_kernel(const uint8_t* __restrict__ base, int64_t m, int64_t step, int32_t tb, KeySpec ks,
                                  int64_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int64_t)load_key(base + i * step * tb, ks);
}

}  // namespace pyg

using namespace pyg;

namespace pyg {

int estimate_distinct_keys(pyg_ctx* ctx, const uint8_t* base, int64_t n, int32_t tb, const KeySpec& ks,
                           int64_t* out)
{
    const int64_t m = n < CDF_ESTIMATE_SAMPLE ? n : CDF_ESTIMATE_SAMPLE;
    const int64_t step = n / m;
    int64_t* sample = nullptr;
    int rc = dalloc(ctx, (void**)&sample, (size_t)m * 8);
    if (rc) return rc;
    key_sample_kernel<<<grid_for(ctx, m, 256, 4, 4), 256, 0, ctx->stream>>>(base, m, step, tb, ks, sample);
    PYG_LAUNCHED(ctx);
    pyg_cdf_train_opts o;
    o.leaves = 64;
    o.epochs = 1;
    o.lr = 0.001f;
    o.seed = 1;
    pyg_cdf* model = nullptr;
    rc = pyg_cdf_train(ctx, sample, m, &o, &model);
    if (!rc) rc = pyg_cdf_estimate_distinct(ctx, model, n, out);
    pyg_cdf_free(ctx, model);
    dfree(ctx, sample);
    return rc;
}

}  // namespace pyg

extern "C" {

int pyg_cdf_train(pyg_ctx* ctx, const int64_t* sample_keys, int64_t n, const pyg_cdf_train_opts* opts, pyg_cdf** out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || !opts || n < 2 || !sample_keys || opts->leaves < 1 || opts->leaves > (1 << 20) || opts->epochs < 1) {
        set_error("pyg_cdf_train: need >= 2 sample keys, 1..2^20 leaves, >= 1 epoch");
        return PYG_ERR_ARG;
    }
    *out = nullptr;
    const int L = opts->leaves;
    int64_t* sorted = nullptr;
    if ((rc = sort_keys(ctx, sample_keys, n, &sorted))) return rc;
    pyg_cdf* m = new pyg_cdf();
    m->L = L;
    m->n_sample = n;
    CdfWork w;
    float* adam = nullptr;  // m and v for 2 + 2L params
    std::vector<long long> run_start, run_end;  // heavy runs in the sorted sample
    int64_t* cont = nullptr;                    // the sample without its heavy runs
    const int64_t* fit = sorted;                // what the root and leaves are fitted to
    int64_t nfit = n;
    do {
        if ((rc = w.alloc(ctx, n, L))) break;
        if ((rc = dalloc(ctx, (void**)&m->d_params, (size_t)(2 + 2 * L) * 4))) break;
        if ((rc = dalloc(ctx, (void**)&m->d_yr, (size_t)2 * L * 8))) break;
        if ((rc = dalloc(ctx, (void**)&adam, (size_t)2 * (2 + 2 * L) * 4))) break;
        // Sample statistics and heavy runs in one round trip: the end keys,
        // distinct / singleton counts, and up to `cap` heavy runs (start,
        // key, end) land in the pinned staging area together.
        const int cap = 4096;
        const int64_t thr = n / 4096 > 2 ? n / 4096 : 2;
        unsigned long long* dstat = ctx->dcounters + 80;  // [0..1] run stats, [2] heavy-run count
        longlong2* runs;
        long long* rend;
        if ((rc = dalloc(ctx, (void**)&runs, (size_t)cap * 24))) break;
        rend = (long long*)(runs + cap);
        PYG_CUDA(cudaMemsetAsync(dstat, 0, 24, ctx->stream));
        run_stats_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>(sorted, n, dstat);
        PYG_LAUNCHED(ctx);
        heavy_runs_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>(sorted, n, thr, runs, rend, dstat + 2,
                                                                              cap);
        PYG_LAUNCHED(ctx);
        unsigned char* stage = (unsigned char*)ctx->pinned + kPinnedScalarBytes;
        int64_t* hends = (int64_t*)stage;
        unsigned long long* hst = (unsigned long long*)(stage + 16);
        longlong2* hruns = (longlong2*)(stage + 64);
        long long* hrend = (long long*)(hruns + cap);
        PYG_CUDA(cudaMemcpyAsync(hends, sorted, 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(hends + 1, sorted + n - 1, 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(hst, dstat, 24, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(hruns, runs, (size_t)cap * 24, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        dfree(ctx, runs);
        m->kmin = hends[0];
        m->kmax = hends[1];
        m->distinct = (int64_t)hst[0];
        m->f1 = (int64_t)hst[1];
        {
            const int nh = (int)std::min<unsigned long long>(hst[2], (unsigned long long)cap);
            std::vector<longlong2> hr(hruns, hruns + nh);
            std::vector<long long> he(hrend, hrend + nh);
            std::vector<int> ord(nh);
            for (int i = 0; i < nh; ++i) ord[i] = i;
            std::sort(ord.begin(), ord.end(), [&](int a, int b) { return hr[a].x < hr[b].x; });
            double before = 0;
            for (int i : ord) {
                const double w = (double)(he[i] - hr[i].y) / (double)n;
                m->heavy_key.push_back(hr[i].x);
                m->heavy_w.push_back(w);
                m->heavy_before.push_back(before);
                run_start.push_back(hr[i].y);
                run_end.push_back(he[i]);
                before += w;
            }
            m->wheavy = before;
        }
        // The leaves are fitted to the sample without its heavy runs (they
        // are point masses of the model); the runs are ordered by key, so
        // also by position in the sorted sample.
        const int nh = (int)run_start.size();
        int64_t heavy_n = 0;
        for (int i = 0; i < nh; ++i) heavy_n += run_end[i] - run_start[i];
        if (nh > 0 && n - heavy_n >= 2) {
            std::vector<long long> cum(nh + 1, 0);
            for (int i = 0; i < nh; ++i) cum[i + 1] = cum[i] + (run_end[i] - run_start[i]);
            long long* runs = nullptr;
            if ((rc = dalloc(ctx, (void**)&runs, (size_t)(3 * nh + 1) * 8))) break;
            if ((rc = dalloc(ctx, (void**)&cont, (size_t)(n - heavy_n) * 8))) {
                dfree(ctx, runs);
                break;
            }
            PYG_CUDA(cudaMemcpyAsync(runs, run_start.data(), (size_t)nh * 8, cudaMemcpyHostToDevice, ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(runs + nh, run_end.data(), (size_t)nh * 8, cudaMemcpyHostToDevice, ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(runs + 2 * nh, cum.data(), (size_t)(nh + 1) * 8, cudaMemcpyHostToDevice,
                                     ctx->stream));
            drop_runs_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>(sorted, n, runs, runs + nh,
                                                                                   runs + 2 * nh, nh, cont);
            PYG_LAUNCHED(ctx);
            // Copies from pageable host memory are staged before the calls
            // return, so the host vectors may go; runs is freed in stream order.
            dfree(ctx, runs);
            fit = cont;
            nfit = n - heavy_n;
        }
        if (nh > 0) {
            if ((rc = dalloc(ctx, (void**)&m->d_hkeys, (size_t)nh * 8)) ||
                (rc = dalloc(ctx, (void**)&m->d_hbefore, (size_t)nh * 8)) ||
                (rc = dalloc(ctx, (void**)&m->d_hw, (size_t)nh * 8)))
                break;
            PYG_CUDA(cudaMemcpyAsync(m->d_hkeys, m->heavy_key.data(), (size_t)nh * 8, cudaMemcpyHostToDevice,
                                     ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(m->d_hbefore, m->heavy_before.data(), (size_t)nh * 8, cudaMemcpyHostToDevice,
                                     ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(m->d_hw, m->heavy_w.data(), (size_t)nh * 8, cudaMemcpyHostToDevice,
                                     ctx->stream));
        }
        m->key_lo = (double)m->kmin;
        m->key_scale = m->kmax > m->kmin ? 1.0 / ((double)m->kmax - (double)m->kmin) : 0.0;

        // Initial parameters: root y = x, leaves t = u.
        std::vector<float> p(2 + 2 * L);
        p[0] = 1.f;
        p[1] = 0.f;
        for (int l = 0; l < L; ++l) {
            p[2 + 2 * l] = 1.f;
            p[3 + 2 * l] = 0.f;
        }
        PYG_CUDA(cudaMemcpyAsync(m->d_params, p.data(), p.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
        PYG_CUDA(cudaMemsetAsync(adam, 0, (size_t)2 * (2 + 2 * L) * 4, ctx->stream));
        double root_scale = 2.0 / (double)nfit;
        PYG_CUDA(cudaMemcpyAsync(w.gscale, &root_scale, 8, cudaMemcpyHostToDevice, ctx->stream));
        int gr = grid_for(ctx, nfit, CDF_THREADS, 4, 8);
        const int E = opts->epochs;
        // Root: the least-squares line in one pass (the exact minimiser of
        // the root's squared loss, so no gradient steps follow).
        root_ls_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(fit, nfit, m->key_lo, m->key_scale, w.ls);
        root_solve_kernel<<<1, 1, 0, ctx->stream>>>(w.ls, nfit, m->d_params);
        ctx->launches += 2;
        PYG_CUDA(cudaGetLastError());
        if ((rc = cdf_assign(ctx, w, fit, nfit, L, m->key_lo, m->key_scale, m->d_params, m->d_yr))) break;
        // Leaves: least-squares lines from one pass of per-leaf sums, then
        // E epochs of forward (residuals), backward (per-leaf gradient
        // sums) and projected Adam, which keep the slopes >= 0.
        leaf_ls_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(nfit, w.leaf, w.u, m->d_yr, w.ls + 4);
        leaf_solve_kernel<<<grid_for(ctx, L, 256, 1, 4), 256, 0, ctx->stream>>>(w.ls + 4, L, m->d_params);
        ctx->launches += 2;
        PYG_CUDA(cudaGetLastError());
        int ga = grid_for(ctx, 2 + 2 * L, 256, 1, 4);
        for (int e = 1; e <= E; ++e) {
            float lr = opts->lr * powf(0.01f, (float)(e - 1) / (float)E);
            leaf_forward_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(nfit, w.leaf, w.u, m->d_yr, m->d_params, w.g,
                                                                      nullptr);
            leaf_backward_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(nfit, w.leaf, w.u, w.g, w.raw);
            // Root gradient entries are zero here; Adam skips scale-0 params.
            adam_kernel<<<ga, 256, 0, ctx->stream>>>(m->d_params + 2, w.raw + 2, w.gscale + 1, adam + 2,
                                                     adam + 2 + 2 * L + 2, 2 * L, lr, e);
            ctx->launches += 3;
        }
        PYG_CUDA(cudaGetLastError());
        // Host copies for splitter inversion.
        PYG_CUDA(cudaMemcpyAsync(p.data(), m->d_params, p.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
        std::vector<double> yr(2 * L);
        PYG_CUDA(cudaMemcpyAsync(yr.data(), m->d_yr, yr.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        m->a0 = p[0];
        m->b0 = p[1];
        m->la.resize(L);
        m->lb.resize(L);
        m->ylo.resize(L);
        m->yhi.resize(L);
        for (int l = 0; l < L; ++l) {
            m->la[l] = p[2 + 2 * l];
            m->lb[l] = p[3 + 2 * l];
            m->ylo[l] = yr[2 * l];
            m->yhi[l] = yr[2 * l + 1];
        }
        rc = PYG_OK;
    } while (0);
    w.release(ctx);
    dfree(ctx, adam);
    dfree(ctx, sorted);
    dfree(ctx, cont);
    if (rc) {
        pyg_cdf_free(ctx, m);
        return rc;
    }
    *out = m;
    return PYG_OK;
}

int pyg_cdf_free(pyg_ctx* ctx, pyg_cdf* m)
{
    if (!m) return PYG_OK;
    if (ctx) {
        dfree(ctx, m->d_params);
        dfree(ctx, m->d_yr);
        dfree(ctx, m->d_hkeys);
        dfree(ctx, m->d_hbefore);
        dfree(ctx, m->d_hw);
        dfree(ctx, m->d_bleaf);
    }
    delete m;
    return PYG_OK;
}

}  // extern "C"

namespace pyg {

// C(k), the continuous part of the model, on the host (the predict
// kernel's formula).
static double cdf_continuous(const pyg_cdf* m, int64_t k)
{
    const double x = (double)(float)(((double)k - m->key_lo) * m->key_scale);
    const double r = (double)m->a0 * x + (double)m->b0;
    const int L = m->L;
    const double fl = floor(L * r);
    const int l = fl < 0 ? 0 : (fl > L - 1 ? L - 1 : (int)fl);
    double uu = L * r - l;
    uu = uu < 0 ? 0 : (uu > 1 ? 1 : uu);
    double f = (double)m->la[l] * uu + (double)m->lb[l];
    f = f < 0 ? 0 : (f > 1 ? 1 : f);
    return m->ylo[l] + (m->yhi[l] - m->ylo[l]) * f;
}

// Inversion of C for the splitters: the non-empty leaves in order (their
// target ranges are ordered and disjoint) with the reciprocals the
// inversion needs, so that each splitter costs multiplications only.
struct CdfInverse {
    std::vector<int> leaf;
    std::vector<double> ylo, inv_span, slope, inv_slope, icpt;
    double inv_L = 0, inv_a0 = 0, b0 = 0, key_lo = 0, inv_scale = 0;
    bool usable = false;
    explicit CdfInverse(const pyg_cdf* m)
    {
        for (int l = 0; l < m->L; ++l) {
            if (!(m->yhi[l] > m->ylo[l])) continue;
            leaf.push_back(l);
            ylo.push_back(m->ylo[l]);
            inv_span.push_back(1.0 / (m->yhi[l] - m->ylo[l]));
            slope.push_back(m->la[l]);
            inv_slope.push_back(m->la[l] > 0 ? 1.0 / (double)m->la[l] : 0.0);
            icpt.push_back(m->lb[l]);
        }
        inv_L = 1.0 / (double)m->L;
        inv_a0 = m->a0 > 0 ? 1.0 / (double)m->a0 : 0.0;
        b0 = m->b0;
        key_lo = m->key_lo;
        inv_scale = m->key_scale != 0 ? 1.0 / m->key_scale : 0.0;
        usable = !leaf.empty() && m->key_scale != 0;
    }
};

// Splitter j of `fanout` (1 <= j < fanout) before the running maximum and
// the heavy-span fix-up that the host applies: the key at which the
// model's F reaches j / fanout -- the leaf whose target range holds the
// continuous part's value, its line inverted to a leaf coordinate, the
// root line inverted to a key; one thread per splitter -- and the heavy key
// whose span holds it (-1 if none).
struct SplitArgs {
    const double* ylo;        // non-empty leaves, in order
    const double* inv_span;
    const double* slope;
    const double* inv_slope;
    const double* icpt;
    const double* leaf;       // leaf index (exact in a double)
    int nleaf;
    const double* Fb;         // heavy spans [Fb, Fe) of F
    const double* Fe;
    const double* hbefore;
    const int64_t* hkey;
    int H;
    double W, cont, inv_L, inv_a0, b0, key_lo, inv_scale;
    int64_t kmin, kmax, past;
    int fanout;
    int64_t* out;             // fanout - 1 keys
    int* inside;              // fanout entries, index j
};

__global__ void cdf_split_kernel(SplitArgs a)
{
    for (int j = 1 + blockIdx.x * blockDim.x + threadIdx.x; j < a.fanout; j += gridDim.x * blockDim.x) {
        const double q = (double)j / (double)a.fanout;
        int lo = 0, hi = a.H;
        while (lo < hi) {  // first heavy key whose span ends after q
            const int mid = (lo + hi) >> 1;
            if (a.Fe[mid] <= q) lo = mid + 1;
            else hi = mid;
        }
        int64_t key;
        int in = -1;
        if (lo < a.H && q >= a.Fb[lo]) {
            key = a.hkey[lo];
            in = lo;
        } else {
            const double below = lo < a.H ? a.hbefore[lo] : a.W;
            const double c = a.cont > 1e-12 ? (q - below) / a.cont : 0.0;
            if (a.nleaf == 0) {
                key = a.past;
            } else {
                int l0 = 0, l1 = a.nleaf;  // last leaf with ylo <= c (the first if none)
                while (l0 + 1 < l1) {
                    const int mid = (l0 + l1) >> 1;
                    if (a.ylo[mid] <= c) l0 = mid;
                    else l1 = mid;
                }
                const double t = (c - a.ylo[l0]) * a.inv_span[l0];
                double uu = a.slope[l0] > 0 ? (t - a.icpt[l0]) * a.inv_slope[l0] : 0.0;
                uu = fmin(1.0, fmax(0.0, uu));
                const double r = (a.leaf[l0] + uu) * a.inv_L;
                const double x = (r - a.b0) * a.inv_a0;
                const double kf = a.key_lo + x * a.inv_scale;
                if (!(kf > (double)a.kmin)) key = a.kmin;
                else if (kf >= (double)a.kmax) key = a.past;
                else key = (int64_t)ceil(kf);
            }
            if (lo > 0) {
                const int64_t k = a.hkey[lo - 1];
                const int64_t floor_key = k == INT64_MAX ? INT64_MAX : k + 1;
                key = key < floor_key ? floor_key : key;
            }
            if (lo < a.H && key > a.hkey[lo]) key = a.hkey[lo];
        }
        a.out[j - 1] = key;
        a.inside[j] = in;
    }
}

// ---------------------------------------------------------------------------
// The model's own bins (rj_model_bin): partitions computed from the key by
// the model instead of searched among splitters.

// Normalisation of the model's bins: x = (float)(k - kmin) * scale.
static float bin_scale(const pyg_cdf* m)
{
    const double s = m->key_scale;
    return std::isfinite(s) && s > 0 ? (float)s : 0.f;
}

// Leaf of key k on the host, with the device's operations (correctly
// rounded fp32 steps give the same results on both sides).
static int bin_leaf_host(const pyg_cdf* m, int64_t k)
{
    const float x = (float)((unsigned long long)k - (unsigned long long)m->kmin) * bin_scale(m);
    const float lr = fmaf(m->a0, x, m->b0) * (float)m->L;
    const float fl = floorf(lr);
    return fl < 0.f ? 0 : (fl > (float)(m->L - 1) ? m->L - 1 : (int)fl);
}

int cdf_bin_model(pyg_ctx* ctx, const pyg_cdf* m, int fbits, RJModel* out)
{
    if (!m || m->L < 1 || fbits < 1 || fbits > 24) {
        set_error("cdf bins: no usable model for 2^%d bins", fbits);
        return PYG_ERR_ARG;
    }
    const int L = m->L, H = (int)m->heavy_key.size();
    if (!m->d_bleaf) {
        // Leaf l's line over u: g = base + span * clamp(slope u + icpt, 0,
        // 1), as A u + B clamped to [base, base + span]; its heavy keys
        // add their masses above that, capped at hi_l.  The heavy masses
        // below a leaf are part of its base, and lo_{l+1} >= hi_l keeps the
        // bins ordered across leaves.
        const double cont = 1.0 - m->wheavy;
        std::vector<RJLeaf> lv(L);
        std::vector<int2> hinfo(L);
        std::vector<float> hw(H);
        int h = 0;
        double below = 0.0;  // heavy mass of the leaves so far
        float prev_hi = 0.f;
        for (int l = 0; l < L; ++l) {
            RJLeaf& p = lv[l];
            const double ylo = m->ylo[l], yhi = m->yhi[l];
            const bool ok = std::isfinite(ylo) && std::isfinite(yhi) && yhi > ylo;
            const float base = std::max(prev_hi, (float)(cont * (ok ? ylo : 0.0) + below));
            const float span = ok ? (float)(cont * (yhi - ylo)) : 0.f;
            const float slope = std::isfinite(m->la[l]) ? std::max(0.f, m->la[l]) : 0.f;
            const float icpt = std::isfinite(m->lb[l]) ? m->lb[l] : 0.f;
            p.A = span * slope;
            p.B = base + span * icpt;
            p.lo = base;
            float top = base + span;
            hinfo[l].x = h;
            while (h < H && bin_leaf_host(m, m->heavy_key[h]) <= l) {
                hw[h] = (float)m->heavy_w[h];
                top = top + hw[h];
                below += m->heavy_w[h];
                ++h;
            }
            hinfo[l].y = h - hinfo[l].x;
            p.hi = std::max(top, base);
            prev_hi = p.hi;
        }
        char* buf = nullptr;
        const size_t bytes = (size_t)L * sizeof(RJLeaf) + (size_t)L * sizeof(int2) + (size_t)H * 8 + (size_t)H * 4 + 16;
        int rc = dalloc(ctx, (void**)&buf, bytes);
        if (rc) return rc;
        m->d_bleaf = (RJLeaf*)buf;
        m->d_bhinfo = (int2*)(m->d_bleaf + L);
        m->d_bhkey = (long long*)(m->d_bhinfo + L);
        m->d_bhw = (float*)(m->d_bhkey + H);
        if ((rc = stage_h2d(ctx, m->d_bleaf, lv.data(), (size_t)L * sizeof(RJLeaf)))) return rc;
        if (H) {
            if ((rc = stage_h2d(ctx, m->d_bhinfo, hinfo.data(), (size_t)L * sizeof(int2)))) return rc;
            if ((rc = stage_h2d(ctx, m->d_bhkey, m->heavy_key.data(), (size_t)H * 8))) return rc;
            if ((rc = stage_h2d(ctx, m->d_bhw, hw.data(), (size_t)H * 4))) return rc;
        }
    }
    RJModel r;
    r.leaf = m->d_bleaf;
    r.hinfo = H ? m->d_bhinfo : nullptr;
    r.hkey = m->d_bhkey;
    r.hw = m->d_bhw;
    r.kmin = m->kmin;
    r.kmax = m->kmax;
    // Bin 0 holds the keys <= kmin and the last bin those >= kmax; keep
    // kmin < kmax so that both ends exist.  A sample of one key value has
    // no scale: x = 0 for every key then (a constant is monotone too).
    if (r.kmax <= r.kmin) {
        if (r.kmin < INT64_MAX) r.kmax = r.kmin + 1;
        else r.kmin = r.kmax - 1;
    }
    r.scale = bin_scale(m);
    r.a0 = std::max(0.f, m->a0);
    r.b0 = m->b0;
    r.L = L;
    r.fbits = fbits;
    *out = r;
    return PYG_OK;
}

// Splitter j (1 <= j < 2^fbits) = the first key whose bin is >= j, by
// bisection over [kmin, kmax] (bin(kmin) = 0 < j <= bin(kmax)); since the
// bins never decrease with the key, bin(k) = number of splitters <= k.
__global__ void bin_splitters_kernel(RJModel m, int64_t* __restrict__ out)
{
    const int F = 1 << m.fbits;
    for (int j = 1 + blockIdx.x * blockDim.x + threadIdx.x; j < F; j += gridDim.x * blockDim.x) {
        // Keys as order-preserving unsigned words (sign bit flipped).
        unsigned long long lo = to_sortable(m.kmin), hi = to_sortable(m.kmax);
        while (hi - lo > 1) {
            const unsigned long long mid = lo + ((hi - lo) >> 1);
            if (rj_model_bin(m, from_sortable(mid)) >= (unsigned)j) hi = mid;
            else lo = mid;
        }
        out[j - 1] = from_sortable(hi);
    }
}

__global__ void model_bins_kernel(RJModel m, const int64_t* __restrict__ keys, int64_t n, uint32_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = rj_model_bin(m, keys[i]);
}

int model_splitters(pyg_ctx* ctx, const RJModel& m, int64_t* out)
{
    const int F = 1 << m.fbits;
    if (F < 2) return PYG_OK;
    int64_t* d = nullptr;
    int rc = dalloc(ctx, (void**)&d, (size_t)(F - 1) * 8);
    if (rc) return rc;
    bin_splitters_kernel<<<grid_for(ctx, F - 1, 128, 1, 8), 128, 0, ctx->stream>>>(m, d);
    cudaError_t e = cudaGetLastError();
    ctx->launches++;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d, (size_t)(F - 1) * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    dfree(ctx, d);
    return e == cudaSuccess ? PYG_OK : cuda_status(e, "model splitters");
}

}  // namespace pyg

extern "C" {

int pyg_cdf_splitters(pyg_ctx* ctx, const pyg_cdf* m, int32_t fanout, int64_t* out)
{
    if (fanout > 1) {
        const int rc0 = check_ctx(ctx);
        if (rc0) return rc0;
    }
    if (!m || fanout < 1 || (fanout > 1 && !out)) {
        set_error("pyg_cdf_splitters: bad arguments");
        return PYG_ERR_ARG;
    }
    const CdfInverse inv(m);
    const int64_t past = m->kmax == INT64_MAX ? INT64_MAX : m->kmax + 1;  // past the largest sample key
    // Heavy key h covers [Fb[h], Fb[h] + w_h) of F = (1 - W) C + heavy masses.
    const int H = (int)m->heavy_key.size();
    const double W = m->wheavy, cont = 1.0 - W;
    std::vector<double> Fb(H), Fe(H);
    for (int h = 0; h < H; ++h) {
        Fb[h] = cont * cdf_continuous(m, m->heavy_key[h]) + m->heavy_before[h];
        Fe[h] = Fb[h] + m->heavy_w[h];
        if (h > 0) {  // keep the spans ordered when the fit is off
            Fb[h] = std::max(Fb[h], Fe[h - 1]);
            Fe[h] = Fb[h] + m->heavy_w[h];
        }
    }
    std::vector<int> inside(fanout, -1);  // splitter j (1-based) falls in heavy key h's span
    if (!inv.usable) {
        for (int j = 1; j < fanout; ++j) out[j - 1] = past;
    } else {
        // One thread per splitter on the device: the model's leaf and heavy
        // tables go up in one copy, keys and span marks come back.
        const int n = (int)inv.ylo.size();
        std::vector<double> hd((size_t)6 * n + 3 * H);
        double* q = hd.data();
        for (int i = 0; i < n; ++i) {
            q[i] = inv.ylo[i];
            q[n + i] = inv.inv_span[i];
            q[2 * n + i] = inv.slope[i];
            q[3 * n + i] = inv.inv_slope[i];
            q[4 * n + i] = inv.icpt[i];
            q[5 * n + i] = (double)inv.leaf[i];
        }
        for (int h = 0; h < H; ++h) {
            q[6 * n + h] = Fb[h];
            q[6 * n + H + h] = Fe[h];
            q[6 * n + 2 * H + h] = m->heavy_before[h];
        }
        char* dbuf = nullptr;
        const size_t dbytes = hd.size() * 8 + (size_t)H * 8 + (size_t)(fanout - 1) * 8 + (size_t)fanout * 4;
        int rc = dalloc(ctx, (void**)&dbuf, dbytes);
        if (rc) return rc;
        double* dd = (double*)dbuf;
        int64_t* dk = (int64_t*)(dbuf + hd.size() * 8);
        int64_t* dout = dk + H;
        int* din = (int*)(dout + (fanout - 1));
        SplitArgs sa;
        sa.ylo = dd;
        sa.inv_span = dd + n;
        sa.slope = dd + 2 * n;
        sa.inv_slope = dd + 3 * n;
        sa.icpt = dd + 4 * n;
        sa.leaf = dd + 5 * n;
        sa.nleaf = n;
        sa.Fb = dd + 6 * n;
        sa.Fe = dd + 6 * n + H;
        sa.hbefore = dd + 6 * n + 2 * H;
        sa.hkey = dk;
        sa.H = H;
        sa.W = W;
        sa.cont = cont;
        sa.inv_L = inv.inv_L;
        sa.inv_a0 = inv.inv_a0;
        sa.b0 = inv.b0;
        sa.key_lo = inv.key_lo;
        sa.inv_scale = inv.inv_scale;
        sa.kmin = m->kmin;
        sa.kmax = m->kmax;
        sa.past = past;
        sa.fanout = fanout;
        sa.out = dout;
        sa.inside = din;
        cudaError_t e = cudaMemcpyAsync(dd, hd.data(), hd.size() * 8, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess && H)
            e = cudaMemcpyAsync(dk, m->heavy_key.data(), (size_t)H * 8, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) {
            cdf_split_kernel<<<grid_for(ctx, fanout, 256, 1, 4), 256, 0, ctx->stream>>>(sa);
            e = cudaGetLastError();
            ctx->launches++;
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out, dout, (size_t)(fanout - 1) * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(inside.data(), din, (size_t)fanout * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        dfree(ctx, dbuf);
        if (e != cudaSuccess) return cuda_status(e, "pyg_cdf_splitters");
        inside[0] = -1;
        // Running maximum: splitters never decrease.
        int64_t prev = m->kmin;
        for (int j = 1; j < fanout; ++j) {
            if (out[j - 1] < prev) out[j - 1] = prev;
            prev = out[j - 1];
        }
    }
    // A heavy key that takes two or more splitters gets a range of its own:
    // the last of them becomes key + 1 (exact quantiles do the same).
    for (int j = fanout - 1; j >= 1; --j) {
        const int h = inside[j];
        if (h < 0 || (j + 1 < fanout && inside[j + 1] == h)) continue;  // not the last of its span
        if (j - 1 >= 1 && inside[j - 1] == h) {
            const int64_t k = m->heavy_key[h];
            out[j - 1] = k == INT64_MAX ? k : k + 1;
            for (int t = j + 1; t < fanout && out[t - 1] < out[j - 1]; ++t) out[t - 1] = out[j - 1];
        }
    }
    return PYG_OK;
}

int pyg_cdf_predict(pyg_ctx* ctx, const pyg_cdf* m, const int64_t* keys, int64_t n, float* out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!m || n < 0 || (n > 0 && (!keys || !out))) {
        set_error("pyg_cdf_predict: bad arguments");
        return PYG_ERR_ARG;
    }
    if (n == 0) return PYG_OK;
    predict_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>(
        keys, n, m->key_lo, m->key_scale, m->d_params, m->d_yr, m->L, m->d_hkeys, m->d_hbefore, m->d_hw,
        (int)m->heavy_key.size(), m->wheavy, out);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

int pyg_cdf_bins(pyg_ctx* ctx, const pyg_cdf* m, int32_t fbits, const int64_t* keys, int64_t n, uint32_t* out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!m || n < 0 || (n > 0 && (!keys || !out))) {
        set_error("pyg_cdf_bins: bad arguments");
        return PYG_ERR_ARG;
    }
    RJModel bm;
    if ((rc = cdf_bin_model(ctx, m, fbits, &bm))) return rc;
    if (n == 0) return PYG_OK;
    model_bins_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>(bm, keys, n, out);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

int pyg_cdf_bin_splitters(pyg_ctx* ctx, const pyg_cdf* m, int32_t fbits, int64_t* out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!m || !out) {
        set_error("pyg_cdf_bin_splitters: bad arguments");
        return PYG_ERR_ARG;
    }
    RJModel bm;
    if ((rc = cdf_bin_model(ctx, m, fbits, &bm))) return rc;
    return model_splitters(ctx, bm, out);
}

int pyg_cdf_params(pyg_ctx* ctx, const pyg_cdf* m, float* params, int32_t cap, double* key_lo, double* key_scale)
{
    (void)ctx;
    if (!m || !params || cap < 2 + 2 * m->L) {
        set_error("pyg_cdf_params: need room for %d floats", m ? 2 + 2 * m->L : 0);
        return PYG_ERR_ARG;
    }
    params[0] = m->a0;
    params[1] = m->b0;
    for (int l = 0; l < m->L; ++l) {
        params[2 + 2 * l] = m->la[l];
        params[3 + 2 * l] = m->lb[l];
    }
    if (key_lo) *key_lo = m->key_lo;
    if (key_scale) *key_scale = m->key_scale;
    return PYG_OK;
}

int pyg_cdf_loss_grad(pyg_ctx* ctx, const int64_t* sorted_keys, int64_t n, int32_t L, const float* params_host,
                      double key_lo, double key_scale, double* loss, float* grad_host)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!sorted_keys || n < 1 || L < 1 || !params_host || !loss || !grad_host) {
        set_error("pyg_cdf_loss_grad: bad arguments");
        return PYG_ERR_ARG;
    }
    CdfWork w;
    float* dp = nullptr;
    double* dyr = nullptr;
    do {
        if ((rc = w.alloc(ctx, n, L))) break;
        if ((rc = dalloc(ctx, (void**)&dp, (size_t)(2 + 2 * L) * 4))) break;
        if ((rc = dalloc(ctx, (void**)&dyr, (size_t)2 * L * 8))) break;
        PYG_CUDA(cudaMemcpyAsync(dp, params_host, (size_t)(2 + 2 * L) * 4, cudaMemcpyHostToDevice, ctx->stream));
        PYG_CUDA(cudaMemsetAsync(w.acc, 0, (size_t)(3 + L) * 8, ctx->stream));
        int gr = grid_for(ctx, n, CDF_THREADS, 4, 8);
        root_fwd_bwd_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(sorted_keys, n, key_lo, key_scale, dp, w.acc);
        PYG_LAUNCHED(ctx);
        if ((rc = cdf_assign(ctx, w, sorted_keys, n, L, key_lo, key_scale, dp, dyr))) break;
        leaf_forward_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(n, w.leaf, w.u, dyr, dp, w.g, w.acc + 3);
        PYG_LAUNCHED(ctx);
        leaf_backward_kernel<<<gr, CDF_THREADS, 0, ctx->stream>>>(n, w.leaf, w.u, w.g, w.raw);
        PYG_LAUNCHED(ctx);
        std::vector<double> acc(3 + L), raw(2 + 2 * L), gs(1 + L);
        PYG_CUDA(cudaMemcpyAsync(acc.data(), w.acc, acc.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(raw.data(), w.raw, raw.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(gs.data(), w.gscale, gs.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        double total = acc[0] / (double)n;
        grad_host[0] = (float)(2.0 / n * acc[1]);
        grad_host[1] = (float)(2.0 / n * acc[2]);
        for (int l = 0; l < L; ++l) {
            // gs[1+l] = 2 / (n_l L); the leaf loss mean is (gs/2) * sum e^2.
            total += 0.5 * gs[1 + l] * acc[3 + l];
            grad_host[2 + 2 * l] = (float)(gs[1 + l] * raw[2 + 2 * l]);
            grad_host[3 + 2 * l] = (float)(gs[1 + l] * raw[3 + 2 * l]);
        }
        *loss = total;
        rc = PYG_OK;
    } while (0);
    w.release(ctx);
    dfree(ctx, dp);
    dfree(ctx, dyr);
    return rc;
}

__global__ void gather_quantiles_kernel(const int64_t* __restrict__ sorted, int64_t n, int fanout,
                                        int64_t* __restrict__ out)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x + 1; j < fanout; j += gridDim.x * blockDim.x) {
        int64_t idx = (int64_t)(((__int128)j * n + fanout - 1) / fanout);  // ceil(j n / F)
        int64_t last = sorted[n - 1];
        out[j - 1] = idx < n ? sorted[idx] : (last == INT64_MAX ? last : last + 1);
    }
}

int pyg_sampled_splitters(pyg_ctx* ctx, const int64_t* sample_keys, int64_t n, int32_t fanout, int64_t* out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!sample_keys || n < 1 || fanout < 1 || (fanout > 1 && !out)) {
        set_error("pyg_sampled_splitters: bad arguments");
        return PYG_ERR_ARG;
    }
    if (fanout == 1) return PYG_OK;
    int64_t* sorted = nullptr;
    if ((rc = sort_keys(ctx, sample_keys, n, &sorted))) return rc;
    int64_t* d;
    if ((rc = dalloc(ctx, (void**)&d, (size_t)(fanout - 1) * 8))) {
        dfree(ctx, sorted);
        return rc;
    }
    gather_quantiles_kernel<<<grid_for(ctx, fanout, 256, 1, 4), 256, 0, ctx->stream>>>(sorted, n, fanout, d);
    PYG_LAUNCHED(ctx);
    PYG_CUDA(cudaMemcpyAsync(out, d, (size_t)(fanout - 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    dfree(ctx, d);
    dfree(ctx, sorted);
    return PYG_OK;
}

int pyg_cdf_estimate_distinct(pyg_ctx* ctx, const pyg_cdf* m, int64_t population, int64_t* out)
{
    (void)ctx;
    if (!m || !out || population < 0) {
        set_error("pyg_cdf_estimate_distinct: bad arguments");
        return PYG_ERR_ARG;
    }
    // GEE (Charikar, Chaudhuri, Motwani, Narasayya, PODS 2000):
    // D = sqrt(N / n) * f1 + (d - f1).
    double r = m->n_sample > 0 ? sqrt((double)population / (double)m->n_sample) : 1.0;
    double est = r * (double)m->f1 + (double)(m->distinct - m->f1);
    if (est > (double)population) est = (double)population;
    if (est < (double)m->distinct) est = (double)m->distinct;
    *out = (int64_t)ceil(est);
    return PYG_OK;
}

}  // extern "C"
