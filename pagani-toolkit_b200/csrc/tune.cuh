// tune.cuh -- the launch-shape autotuner.
//
// A kernel family names its tunable choices (two integers, e.g. sources per
// batch and CTAs per SM) and a key that buckets the problem shape (GPU SM
// count, log2 of the node count and of the mean degree).  On the first
// problem of a bucket every candidate runs once on the real input, timed
// with CUDA events on the context stream, and the fastest is kept: in the
// process, and in a text cache file (PAGANI_TUNE_CACHE, default
// $XDG_CACHE_HOME or ~/.cache /pagani/tune.txt; one "key a b ms" line per
// entry) that later processes read.  PAGANI_TUNE=0 turns tuning off (the
// caller's default is used).  Tuning never runs while the stream is being
// captured into a CUDA graph.  Every candidate of a family computes the same
// result; only the time differs.
#pragma once
#include "pg_internal.cuh"
#include <functional>
#include <string>
#include <vector>

struct TuneChoice {
    int a, b;
};

std::string tune_key(const char* family, int64_t n, int64_t nnz);
// Returns the cached choice for `key`, or times every candidate with `run`
// (which enqueues the computation with that choice) and caches the fastest.
// *best holds the default on entry.
pg_status tune_pick(pg_ctx* ctx, const std::string& key, const std::vector<TuneChoice>& cands, TuneChoice* best,
                    const std::function<pg_status(const TuneChoice&)>& run);
