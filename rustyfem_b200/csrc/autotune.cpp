#include "autotune.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

namespace rfg {

namespace {

std::string cache_key(const Symbolic& S, Precision prec, bool use_tc, bool pair) {
    int dev = 0;
    cudaGetDevice(&dev);
    double w = S.work();
    uint64_t wb = 0;
    std::memcpy(&wb, &w, sizeof(wb));
    return std::to_string(dev) + ":" + std::to_string((int)prec) + ":" + std::to_string(use_tc ? 1 : 0) + ":" +
           std::to_string(pair ? 1 : 0) + ":" +
           std::to_string(S.n) + ":" + std::to_string(S.fronts.size()) + ":" + std::to_string(wb);
}

std::mutex g_mu;
std::map<std::string, TuneResult> g_cache;

}  // namespace

TuneResult autotune_cutover(const Symbolic& S, const std::function<std::unique_ptr<Engine>(Plan&&)>& make_engine,
                            const double* src, Precision prec, bool use_tc, const Tuning& base) {
    const std::string key = cache_key(S, prec, use_tc, base.pair_blocks);
    {
        std::lock_guard<std::mutex> lock(g_mu);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            TuneResult r = it->second;
            r.cached = true;
            return r;
        }
    }
    static const int64_t CANDIDATES[] = {128, 192, 256, 384, 512, 768, 1024, 1536};
    TuneResult res;
    std::vector<std::pair<int64_t, int64_t>> splits;  // (big tiles, small tiles) already measured
    double best = 1e300;
    std::vector<std::pair<int64_t, int>> cands;
    for (int64_t c : CANDIDATES) cands.push_back({c, TC_WIDE});
    if (use_tc && prec == PREC_MIXED)
        for (int64_t c : CANDIDATES) cands.push_back({c, 128});
    for (size_t ci = 0; ci < cands.size(); ci++) {
        Tuning t = base;
        t.big_min_rows = cands[ci].first;
        t.outer_tn = cands[ci].second;
        Plan P = build_plan(S, use_tc, t);
        if (ci == 0 || cands[ci].second != cands[ci - 1].second) splits.clear();
        std::pair<int64_t, int64_t> sp(P.big_tiles, P.small_tiles);
        if (std::find(splits.begin(), splits.end(), sp) != splits.end()) continue;
        splits.push_back(sp);
        double ms = 1e300;
        {
            std::unique_ptr<Engine> E = make_engine(std::move(P));
            if (E->factor(src, false) >= 0) return TuneResult();  // not positive definite: nothing to tune
            for (int rep = 0; rep < 2; rep++) {
                E->factor(src, false);
                ms = std::min(ms, E->last_factor.t_factor_ms);
            }
        }
        res.cutover.push_back(t.big_min_rows);
        res.tile_n.push_back(t.outer_tn);
        res.ms.push_back(ms);
        if (ms < best) {
            best = ms;
            res.best = t;
        }
    }
    std::lock_guard<std::mutex> lock(g_mu);
    g_cache[key] = res;
    return res;
}

}  // namespace rfg
