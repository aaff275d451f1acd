/*
 * pyg_learned.h - learned CDF splitter of the B200 engine (libpyg.so).
 *
 * A two-level piecewise-linear model of a key sample's CDF: a root linear
 * model picks one of `leaves` linear leaves, each fitted to the keys routed
 * to it.  Keys that fill at least 1/4096 of the sample (heavy keys) are
 * exact point masses of the model; the root and leaves fit the rest, so
 *   F(k) = (1 - W) C(k) + (mass of the heavy keys below k),
 * with W the heavy keys' share of the sample.  It is trained on the GPU by
 * the library's own kernels (least-squares start, then projected Adam on
 * the squared CDF error through the forward / backward kernels) and used
 * to pick range partition splitters (the MPSM join) and to size hash
 * tables (its distinct-key estimate, for group-by without a group count).
 * It only moves partition boundaries: results stay exact.
 *
 * No reference counterpart: it replaces the equal-width range split of
 * ExactRangeValueHasher (hash.h:452-487, used by PartitionOp,
 * operators/partition.cpp:56-63, and by SortMergeJoinOp's
 * buildprepartitioned option, operators/join.cpp:1002-1009).
 */
#ifndef PYG_LEARNED_H
#define PYG_LEARNED_H

#include "pyg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pyg_cdf pyg_cdf;

typedef struct pyg_cdf_train_opts {
    int32_t leaves;              /* second-level linear leaves (e.g. 1024) */
    int32_t epochs;              /* full-batch gradient steps (leaves)    */
    float lr;                    /* Adam step size                        */
    uint64_t seed;
} pyg_cdf_train_opts;

/* Trains the model on n device int64 sample keys (any order): the root and
 * every leaf start from their least-squares lines (one pass of sums each),
 * then the leaves take `epochs` projected-Adam steps through the forward /
 * backward kernels.  A few epochs at a small step size fine-tune; the
 * least-squares start already holds most of the fit. */
int pyg_cdf_train(pyg_ctx* ctx, const int64_t* sample_keys, int64_t n, const pyg_cdf_train_opts* opts,
                  pyg_cdf** out);
int pyg_cdf_free(pyg_ctx* ctx, pyg_cdf* model);
/* fanout-1 non-decreasing splitters into host array out: bucket b holds
 * keys in [out[b-1], out[b]). */
int pyg_cdf_splitters(pyg_ctx* ctx, const pyg_cdf* model, int32_t fanout, int64_t* out);
/* Partition bins of n device keys computed by the model itself, without a
 * search: out[i] (device) in [0, 2^fbits), non-decreasing in the key (the
 * model's CDF scaled to 2^fbits bins, keys at or below the sample minimum
 * in bin 0, at or above its maximum in the last).  The MPSM join's learned
 * splitter partitions with these bins; fbits <= 24. */
int pyg_cdf_bins(pyg_ctx* ctx, const pyg_cdf* model, int32_t fbits, const int64_t* keys, int64_t n,
                 uint32_t* out);
/* The 2^fbits - 1 splitters of those bins into host array out: out[j - 1]
 * is the first key of bin j (bisection over the same device function), so
 * that bin(k) = number of splitters <= k, as a splitter search would
 * place k. */
int pyg_cdf_bin_splitters(pyg_ctx* ctx, const pyg_cdf* model, int32_t fbits, int64_t* out);
/* Predicted CDF in [0,1] for n device keys into device float array out. */
int pyg_cdf_predict(pyg_ctx* ctx, const pyg_cdf* model, const int64_t* keys, int64_t n, float* out);
/* Trained parameters to host: params[0..1] = root (slope, intercept) in
 * normalised key units, then per leaf (slope, intercept) of the leaf's
 * local fit; *key_lo / *key_scale normalise keys as x = (key - lo) * scale.
 * cap = number of floats params can hold (>= 2 + 2 * leaves). */
int pyg_cdf_params(pyg_ctx* ctx, const pyg_cdf* model, float* params, int32_t cap, double* key_lo,
                   double* key_scale);
/* One forward + backward evaluation on given parameters (host arrays) over
 * n sorted device keys: *loss and grad (2 + 2 * leaves floats) of
 *   L = mean_i (r(x_i) - y_i)^2 + (1/leaves) * sum_l mean_{i in l} (f_l(u_i) - t_i)^2
 * with r the root line, y_i = i / n, leaf l the root's bucket of x_i, u_i
 * the leaf-local coordinate and t_i the leaf-normalised target.  Lets a
 * test check the gradient kernels against a CPU computation. */
int pyg_cdf_loss_grad(pyg_ctx* ctx, const int64_t* sorted_keys, int64_t n, int32_t leaves,
                      const float* params_host, double key_lo, double key_scale, double* loss,
                      float* grad_host);
/* Splitters from the quantiles of a device key sample (the fallback, and
 * the yardstick for the learned splitters' imbalance). */
int pyg_sampled_splitters(pyg_ctx* ctx, const int64_t* sample_keys, int64_t n, int32_t fanout,
                          int64_t* out);
/* Distinct-key estimate for a population of `population` keys from the
 * model's sample (Charikar et al. GEE estimator over the sorted sample),
 * used to size hash tables. */
int pyg_cdf_estimate_distinct(pyg_ctx* ctx, const pyg_cdf* model, int64_t population, int64_t* out);

#ifdef __cplusplus
}
#endif
#endif /* PYG_LEARNED_H */
