// Device plan construction (see plan.h).

#include "plan.h"
#include "par.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <thread>

namespace rfg {

namespace {

int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }
int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// first-fit allocator over one arena, used to place the update blocks; the free blocks
// are a vector sorted by offset (no node allocations; the scan is over contiguous memory)
struct Arena {
    std::vector<std::pair<int64_t, int64_t>> free_;  // (offset, size), by offset
    int64_t top = 0;
    int64_t alloc(int64_t size) {
        for (size_t i = 0; i < free_.size(); i++) {
            if (free_[i].second >= size) {
                const int64_t off = free_[i].first, rest = free_[i].second - size;
                if (rest > 0)
                    free_[i] = {off + size, rest};
                else
                    free_.erase(free_.begin() + i);
                return off;
            }
        }
        // grow: merge with a free block that ends at the top
        if (!free_.empty() && free_.back().first + free_.back().second == top) {
            const int64_t off = free_.back().first;
            free_.pop_back();
            top = off + size;
            return off;
        }
        const int64_t off = top;
        top += size;
        return off;
    }
    void release(int64_t off, int64_t size) {
        auto it = std::lower_bound(free_.begin(), free_.end(), std::make_pair(off, (int64_t)0));
        it = free_.insert(it, {off, size});
        auto nx = it + 1;
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = it - 1;
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

}  // namespace

Plan build_plan(const Symbolic& S, bool use_tc, const Tuning& tun) {
    Plan P;
    int64_t nt = (int64_t)S.fronts.size();
    HostTimer timer("build_plan");
    P.nfronts = nt;
    P.big_min_rows = tun.big_min_rows;
    P.outer_tn = tun.outer_tn == 128 ? 128 : TC_WIDE;
    P.n = S.n;
    P.work = S.work();
    P.rows.resize(S.rows.size());
    parallel_chunks((int64_t)S.rows.size(), (int64_t)1 << 20, [&](int64_t a, int64_t b) {
        std::copy(S.rows.begin() + a, S.rows.begin() + b, P.rows.begin() + a);
    });
    P.fronts.resize(nt);
    // levels
    std::vector<int64_t> level(nt, 0);
    int64_t nlev = 0;
    for (int64_t t = 0; t < nt; t++) {
        const SymFront& f = S.fronts[t];
        int64_t l = 0;
        for (int64_t c = 0; c < f.nchild; c++) l = std::max(l, level[S.children[f.child_off + c]] + 1);
        level[t] = l;
        nlev = std::max(nlev, l + 1);
    }
    P.nlevels = nlev;
    P.level_off.assign(nlev + 1, 0);
    for (int64_t t = 0; t < nt; t++) P.level_off[level[t] + 1]++;
    for (int64_t l = 0; l < nlev; l++) P.level_off[l + 1] += P.level_off[l];
    P.level_order.assign(nt, 0);
    {
        std::vector<int64_t> fill(P.level_off.begin(), P.level_off.end() - 1);
        for (int64_t t = 0; t < nt; t++) P.level_order[fill[level[t]]++] = t;
        for (int64_t l = 0; l < nlev; l++)
            std::stable_sort(P.level_order.begin() + P.level_off[l], P.level_order.begin() + P.level_off[l + 1],
                             [&](int64_t a, int64_t b) { return S.fronts[a].k > S.fronts[b].k; });
    }
    timer.lap("levels");
    // child rank
    std::vector<int64_t> rank(nt, 0);
    for (int64_t t = 0; t < nt; t++) {
        const SymFront& f = S.fronts[t];
        for (int64_t c = 0; c < f.nchild; c++) rank[S.children[f.child_off + c]] = c;
    }
    // descriptors and the panel arena (level order)
    int64_t poff = 0, vu = 0, emoff = 0, nblk = 0;
    for (int64_t l = 0; l < nlev; l++)
        for (int64_t i = P.level_off[l]; i < P.level_off[l + 1]; i++) {
            int64_t t = P.level_order[i];
            const SymFront& f = S.fronts[t];
            DFront& d = P.fronts[t];
            d.start = f.start;
            d.k = f.k;
            d.u = f.u;
            d.m = f.k + f.u;
            d.ldp = f.k > 0 ? round_up(f.k, 8) : 0;
            d.ldu = f.u > 0 ? round_up(f.u, 8) : 0;
            d.poff = poff;
            poff += round_up(d.m * d.ldp, 32);
            d.parent = f.parent;
            d.rows_off = f.rows_off;
            d.vuoff = vu;
            vu += f.u;
            d.blk_off = nblk;
            nblk += cdiv(f.k, NB);
        }
    P.panel_elems = poff;
    P.vu_rows = vu;
    P.nblocks = nblk;
    timer.lap("descriptors");
    // update arena with reuse: U_t lives from level(t) to level(parent(t))
    {
        Arena A;
        std::vector<std::vector<int64_t>> release_at(nlev + 1);
        for (int64_t l = 0; l < nlev; l++) {
            for (int64_t t : release_at[l]) A.release(P.fronts[t].uoff, round_up(P.fronts[t].u * P.fronts[t].ldu, 32));
            for (int64_t i = P.level_off[l]; i < P.level_off[l + 1]; i++) {
                int64_t t = P.level_order[i];
                DFront& d = P.fronts[t];
                int64_t sz = round_up(d.u * d.ldu, 32);
                d.uoff = sz > 0 ? A.alloc(sz) : 0;
                int64_t end = d.parent >= 0 ? level[d.parent] : l;
                if (sz > 0) release_at[end + 1].push_back(t);
            }
        }
        P.upd_elems = A.top;
        P.upd_peak_elems = A.top;
    }
    timer.lap("update arena");
    // maps of the later rows into the parent: per parent (in parallel), a table of the
    // local index of each of its later rows, read by all its children
    P.emap.assign(S.rows.size(), 0);
    for (int64_t t = 0; t < nt; t++) P.fronts[t].emap_off = P.fronts[t].rows_off;
    std::atomic<bool> missing{false};
    parallel_chunks(nt, 16, [&](int64_t a0, int64_t a1) {
        thread_local std::vector<int64_t> pos;
        if ((int64_t)pos.size() < S.n) pos.assign(S.n, 0);
        for (int64_t p = a0; p < a1; p++) {
            const SymFront& pf = S.fronts[p];
            if (pf.nchild == 0) continue;
            const int64_t* prow = S.rows.data() + pf.rows_off;
            for (int64_t x = 0; x < pf.u; x++) pos[prow[x]] = pf.k + x;
            for (int64_t ci = 0; ci < pf.nchild; ci++) {
                const DFront& d = P.fronts[S.children[pf.child_off + ci]];
                for (int64_t x = 0; x < d.u; x++) {
                    int64_t g = S.rows[d.rows_off + x];
                    int64_t loc;
                    if (g >= pf.start && g < pf.start + pf.k) {
                        loc = g - pf.start;
                    } else {
                        loc = pos[g];
                        // the table may hold another parent's entry: check it
                        if (loc < pf.k || loc >= pf.k + pf.u || prow[loc - pf.k] != g) {
                            missing = true;
                            loc = 0;
                        }
                    }
                    P.emap[d.rows_off + x] = (int32_t)loc;
                }
            }
        }
    });
    if (missing) throw std::runtime_error("internal: row missing in the parent front");
    (void)emoff;
    timer.lap("extend-add maps");
    // steps
    P.front_tc.assign(nt, 0);
    P.front_tc_inner.assign(nt, 0);
    P.step_off.assign(nlev + 1, 0);
    P.level_maxk.assign(nlev, 0);
    auto tri = [](int64_t nr, int64_t nc) { return nc * nr - nc * (nc - 1) / 2; };  // tiles (i, j), j <= i
    // 128×256 tiles of a lower-trapezoidal region of R rows and W ≤ R columns: column tile j
    // (columns 256j ..) takes the row tiles from its diagonal, cdiv(R, 128) − 2j of them
    auto wide_tiles = [](int64_t R, int64_t W) {
        const int64_t nc = cdiv(W, TC_WIDE), nr = cdiv(R, TC_TILE);
        return nc * nr - nc * (nc - 1);
    };
    auto lower_pairs = [](int64_t R, int64_t c0, int64_t c1) {
        // entries (r, c) with c in [c0, c1), r in [c, R) for a square region starting at 0
        double z = 0.0;
        for (int64_t c = c0; c < c1; c++) z += (double)(R - c);
        return z;
    };
    std::vector<char> pair_open(nt, 0);  // a front's last outer block passed only over a strip
    for (int64_t l = 0; l < nlev; l++) {
        int64_t lo = P.level_off[l], hi = P.level_off[l + 1];
        int64_t maxk = hi > lo ? S.fronts[P.level_order[lo]].k : 0;
        P.level_maxk[l] = maxk;
        int64_t nsteps = cdiv(maxk, NB);
        int64_t block_scr_off = 0, prev_scr_off = 0;
        for (int64_t s = 0; s < nsteps; s++) {
            DStep st{};
            st.level = l;
            st.s = s;
            st.fr_off = lo;
            int64_t nact = 0;
            while (lo + nact < hi && S.fronts[P.level_order[lo + nact]].k > s * NB) nact++;
            st.nact = nact;
            int64_t J0 = (s / KO) * NBO, J1 = J0 + NBO;
            if (s % KO == 0) {
                // scratch of the outer block: rows [J0, m) of every front active at its first step
                prev_scr_off = block_scr_off;
                block_scr_off = (int64_t)P.pre_scr.size();
                int64_t cs = 0;
                P.pre_scr.push_back(0);
                for (int64_t i = 0; i < nact; i++) {
                    cs += P.fronts[P.level_order[lo + i]].m - J0;
                    P.pre_scr.push_back(cs);
                }
                P.max_scr_rows = std::max(P.max_scr_rows, cs);
            }
            st.scr_off = block_scr_off;
            st.scr_off_prev = prev_scr_off;
            st.scr_rows = P.pre_scr[block_scr_off + nact];
            st.pre_off = (int64_t)P.pre_panel.size();
            int64_t cp = 0, ci = 0, co = 0;
            double fi = 0.0, fo = 0.0;
            st.out_lo = nact;
            for (int64_t i = 0; i < nact; i++) {
                const DFront& d = P.fronts[P.level_order[lo + i]];
                int64_t j1 = std::min<int64_t>((s + 1) * NB, d.k);
                int64_t J1e = std::min<int64_t>(J1, d.k);
                if ((j1 == J1e) && st.out_lo == nact) st.out_lo = i;
            }
            P.pre_panel.push_back(0);
            P.panel_mode.push_back(0);
            P.pre_inner.push_back(0);
            P.pre_inner_tc.push_back(0);
            P.pre_outer.push_back(0);
            P.pre_outer_tc.push_back(0);
            P.pre_outer_tc2.push_back(0);
            P.outer_mode.push_back(0);
            int64_t cot = 0, cot2 = 0, cit = 0;
            for (int64_t i = 0; i < nact; i++) {
                const DFront& d = P.fronts[P.level_order[lo + i]];
                int64_t j0 = s * NB;
                int64_t j1 = std::min<int64_t>((s + 1) * NB, d.k);
                int64_t jb = j1 - j0;
                int64_t J1e = std::min<int64_t>(J1, d.k);
                int64_t R = d.m - j1;
                cp += cdiv(R, PR);
                {
                    // what the panel writes for the inner update of this step and the outer
                    // update of this outer block (rows [J1e, m), decided as below)
                    const bool inner = J1e > j1, inner_tc = use_tc && R >= TC_INNER_MIN_ROWS && inner;
                    const int64_t Rob = d.m - J1e;
                    const bool outer_big = Rob >= tun.big_min_rows && (d.u == 0 || d.u >= TC_TILE);
                    const bool outer_tc = use_tc && Rob > 0 && outer_big;
                    uint8_t mode = 0;
                    if ((inner && !inner_tc) || (Rob > 0 && !outer_tc)) mode |= PANEL_SCR;
                    if (inner_tc || outer_tc) mode |= PANEL_SPLIT;
                    P.panel_mode[P.panel_mode.size() - 1] = mode;
                    P.panel_mode.push_back(0);
                }
                // inner: rows [j1, m), columns [j1, J1e); K = jb = NB whenever J1e > j1
                if (use_tc && R >= TC_INNER_MIN_ROWS && J1e > j1) {
                    P.front_tc_inner[P.level_order[lo + i]] = 1;
                    cit += tri(cdiv(R, TC_TILE), cdiv(J1e - j1, TC_TILE));
                } else {
                    ci += tri(cdiv(R, UT), cdiv(J1e - j1, UT));
                }
                fi += 2.0 * (double)jb * lower_pairs(R, 0, J1e - j1);
                // outer: rows [J1e, m), columns [J1e, k) and [k, m)
                if (i >= st.out_lo) {
                    int64_t Ro = d.m - J1e;
                    int64_t t = P.level_order[lo + i];
                    // 128-tiles for large trailing matrices whose update block is empty (a root) or
                    // fills whole tiles; the panel part is then either empty (k <= NBO) or at least
                    // NBO wide
                    const bool big = Ro >= tun.big_min_rows && (d.u == 0 || d.u >= TC_TILE);
                    // the kind of a tensor-core update: a block whose front has a next block that
                    // also ends with a tensor-core update passes only over the next block's columns
                    // (strip), and the next block passes over the rest with both blocks' pivots
                    uint8_t om = OUT_NONE;
                    if (big) {
                        om = OUT_FULL;
                        if (use_tc && tun.pair_blocks) {
                            const int64_t J1n = std::min<int64_t>(J1e + NBO, d.k);
                            if (pair_open[t]) {
                                om = OUT_PAIR;
                                pair_open[t] = 0;
                            } else if (J1e < d.k && d.m - J1n >= tun.big_min_rows) {
                                om = OUT_STRIP;
                                pair_open[t] = 1;
                            }
                        }
                    }
                    P.outer_mode[P.outer_mode.size() - 1] = om;
                    const int64_t Ws = std::min<int64_t>(NBO, d.k - J1e);  // the strip's columns
                    const int64_t Kp = (J1e - J0) + (om == OUT_PAIR ? NBO : 0);
                    if (big) {
                        P.front_tc[t] = use_tc ? 1 : 0;
                        if (om == OUT_STRIP) {
                            cot += tri(cdiv(Ro, TC_TILE), cdiv(Ws, TC_TILE));
                            cot2 += cdiv(Ro, TC_TILE);
                        } else {
                            cot += tri(cdiv(Ro, TC_TILE), cdiv(d.k - J1e, TC_TILE)) +
                                   cdiv(d.u, TC_TILE) * (cdiv(d.u, TC_TILE) + 1) / 2;
                            cot2 += wide_tiles(Ro, d.k - J1e) + wide_tiles(d.u, d.u);
                        }
                    } else {
                        co += tri(cdiv(Ro, UT), cdiv(d.k - J1e, UT)) + cdiv(d.u, UT) * (cdiv(d.u, UT) + 1) / 2;
                    }
                    // entries updated: the whole trailing lower triangle, or the strip's columns
                    const double ent = om == OUT_STRIP ? (double)Ws * (double)Ro - (double)Ws * (double)(Ws - 1) / 2.0
                                                       : (double)Ro * (double)(Ro + 1) / 2.0;
                    double f1 = 2.0 * (double)Kp * ent;
                    fo += f1;
                    if (big) {
                        P.outer_big_flops += f1;
                        // its least memory traffic: the updated entries read and written once
                        // (4-byte entries in the mixed path's fronts, 8 in FP64: counted in
                        // entries), the operand rows read once (rows × K values)
                        P.outer_big_entries += ent;
                        P.outer_big_opvals += (double)Ro * (double)Kp;
                    }
                }
                P.pre_panel.push_back(cp);
                P.pre_inner.push_back(ci);
                P.pre_inner_tc.push_back(cit);
                P.pre_outer.push_back(co);
                P.pre_outer_tc.push_back(cot);
                P.pre_outer_tc2.push_back(cot2);
                P.outer_mode.push_back(0);
            }
            st.n_panel = cp;
            st.n_inner = ci;
            st.n_inner_tc = cit;
            st.n_outer = co;
            st.n_outer_tc = cot;
            st.n_outer_tc2 = cot2;
            P.big_tiles += cot;
            P.small_tiles += co;
            st.inner_flops = fi;
            st.outer_flops = fo;
            P.inner_flops += fi;
            P.outer_flops += fo;
            P.max_nact = std::max(P.max_nact, nact);
            P.steps.push_back(st);
        }
        P.step_off[l + 1] = (int64_t)P.steps.size();
    }
    // solve steps
    P.wstep_off.assign(nlev + 1, 0);
    for (int64_t l = 0; l < nlev; l++) {
        const int64_t lo = P.level_off[l], hi = P.level_off[l + 1];
        const int64_t nws = cdiv(P.level_maxk[l], WS);
        for (int64_t S2 = 0; S2 < nws; S2++) {
            WStep w{};
            w.level = l;
            w.S = S2;
            w.fr_off = lo;
            while (lo + w.nact < hi && S.fronts[P.level_order[lo + w.nact]].k > S2 * WS) w.nact++;
            w.pre_off = (int64_t)P.pre_wrows.size();
            P.pre_wrows.push_back(0);
            P.pre_wpart.push_back(0);
            for (int64_t i = 0; i < w.nact; i++) {
                const DFront& d = P.fronts[P.level_order[lo + i]];
                const int64_t J1 = std::min<int64_t>((S2 + 1) * WS, d.k), wb = J1 - S2 * WS;
                const int64_t c = std::max<int64_t>(1, cdiv(d.m - J1, PR));
                w.n_rows += c;
                w.n_part += c * wb;
                P.pre_wrows.push_back(w.n_rows);
                P.pre_wpart.push_back(w.n_part);
            }
            P.max_wrows = std::max(P.max_wrows, w.n_rows);
            P.max_wpart = std::max(P.max_wpart, w.n_part);
            P.wsteps.push_back(w);
        }
        P.wstep_off[l + 1] = (int64_t)P.wsteps.size();
    }
    // solve chains: forward items by block position (the fronts of the level interleaved),
    // backward items by distance from the front's last block; the later rows' pieces
    {
        int64_t cf = tun.chain_fronts;
        if (cf < 0) {
            const char* e = std::getenv("RFG_SOLVE_CHAIN");
            cf = e ? std::atoll(e) : CHAIN_FRONTS;
        }
        P.level_chain.assign(nlev, 0);
        P.chain_blk.assign(nt, -1);
        P.chain_fwd_off.assign(nlev + 1, 0);
        P.chain_bwd_off.assign(nlev + 1, 0);
        P.chain_rows_off.assign(nlev + 1, 0);
        P.chain_cols_off.assign(nlev + 1, 0);
        for (int64_t l = 0; l < nlev; l++) {
            const int64_t lo = P.level_off[l], hi = P.level_off[l + 1];
            if (hi > lo && hi - lo <= cf) {
                P.level_chain[l] = 1;
                int64_t maxnb = 0;
                for (int64_t i = lo; i < hi; i++) {
                    const int64_t t = P.level_order[i], nb = cdiv(P.fronts[t].k, WS);
                    P.chain_blk[t] = P.chain_blocks;
                    for (int64_t b = 0; b < nb; b++) P.chain_bfront.push_back(t);
                    P.chain_blocks += nb;
                    maxnb = std::max(maxnb, nb);
                }
                for (int64_t b = 0; b < maxnb; b++)
                    for (int64_t i = lo; i < hi; i++) {
                        const int64_t t = P.level_order[i];
                        if (b < cdiv(P.fronts[t].k, WS)) P.chain_fwd.insert(P.chain_fwd.end(), {t, b});
                    }
                for (int64_t i = lo; i < hi; i++) {
                    const int64_t t = P.level_order[i];
                    if (P.fronts[t].u == 0) continue;
                    for (int64_t c = 0; c < cdiv(P.fronts[t].u, CHAIN_PIECE); c++) P.chain_rows.insert(P.chain_rows.end(), {t, c});
                    for (int64_t c = 0; c < cdiv(P.fronts[t].k, CHAIN_PIECE); c++) P.chain_cols.insert(P.chain_cols.end(), {t, c});
                }
                for (int64_t d = 0; d < maxnb; d++)
                    for (int64_t i = lo; i < hi; i++) {
                        const int64_t t = P.level_order[i], nb = cdiv(P.fronts[t].k, WS);
                        if (d < nb) P.chain_bwd.insert(P.chain_bwd.end(), {t, nb - 1 - d});
                    }
            }
            P.chain_fwd_off[l + 1] = (int64_t)P.chain_fwd.size() / 2;
            P.chain_bwd_off[l + 1] = (int64_t)P.chain_bwd.size() / 2;
            P.chain_rows_off[l + 1] = (int64_t)P.chain_rows.size() / 2;
            P.chain_cols_off[l + 1] = (int64_t)P.chain_cols.size() / 2;
            P.chain_colpart = std::max(P.chain_colpart, (P.chain_cols_off[l + 1] - P.chain_cols_off[l]) *
                                                            CHAIN_GROUPS * CHAIN_PIECE);
        }
    }
    timer.lap("steps");
    // extend-add lists
    P.xadd.assign(2 * nlev, DXadd{});
    for (int64_t l = 0; l < nlev; l++)
        for (int r = 0; r < 2; r++) {
            DXadd& x = P.xadd[2 * l + r];
            x.off = (int64_t)P.xadd_child.size();
            x.task_off = (int64_t)P.xadd_task.size() / 4;
            x.fpre_off = (int64_t)P.xadd_fpre.size();
            P.xadd_fpre.push_back(0);
            int64_t cnt = 0, fblk = 0;
            for (int64_t i = P.level_off[l]; i < P.level_off[l + 1]; i++) {
                const SymFront& f = S.fronts[P.level_order[i]];
                if (f.nchild <= r) continue;
                int64_t c = S.children[f.child_off + r];
                if (S.fronts[c].u == 0) continue;
                P.xadd_child.push_back(c);
                const int64_t uc = S.fronts[c].u;
                for (int64_t x0 = 0; x0 < uc; x0 += XR)
                    P.xadd_task.insert(P.xadd_task.end(), {c, P.level_order[i], x0, std::min<int64_t>(XR, uc - x0)});
                const int64_t T = cdiv(uc, XT);
                fblk += cdiv(T * (T + 1) / 2, 8);
                P.xadd_fpre.push_back(fblk);
                cnt++;
            }
            x.nchild = cnt;
            x.ntask = (int64_t)P.xadd_task.size() / 4 - x.task_off;
            x.nblk = cdiv(x.ntask, 8);
            x.fnblk = fblk;
        }
    if (std::any_of(S.fronts.begin(), S.fronts.end(), [](const SymFront& f) { return f.nchild > 2; }))
        throw std::runtime_error("internal: a front has more than two children");
    P.front_of_dof.assign(S.n, 0);
    for (int64_t t = 0; t < nt; t++)
        for (int64_t q = S.fronts[t].start; q < S.fronts[t].start + S.fronts[t].k; q++) P.front_of_dof[q] = t;
    timer.lap("extend-add lists");
    return P;
}

namespace {

struct LocalRows {
    std::vector<int64_t> pos;  // equation -> local row in the current front (valid for its rows)
    explicit LocalRows(int64_t n) : pos(n, 0) {}
    void set(const Symbolic& S, const DFront& d) {
        for (int64_t x = 0; x < d.u; x++) pos[S.rows[d.rows_off + x]] = d.k + x;
    }
    int64_t local(const DFront& d, int64_t g) const { return (g >= d.start && g < d.start + d.k) ? g - d.start : pos[g]; }
};

}  // namespace

Scatter scatter_from_lower(const Plan& P, const Symbolic& S, const std::vector<int64_t>& colptr,
                           const std::vector<int64_t>& rowidx) {
    Scatter X;
    LocalRows L(S.n);
    X.level_seg.assign(P.nlevels + 1, 0);
    X.front_seg.assign(P.nfronts + 1, 0);
    X.seg_ptr.push_back(0);
    for (int64_t l = 0; l < P.nlevels; l++) {
        for (int64_t i = P.level_off[l]; i < P.level_off[l + 1]; i++) {
            X.front_seg[i] = (int64_t)X.dst.size();
            const DFront& d = P.fronts[P.level_order[i]];
            L.set(S, d);
            for (int64_t c = d.start; c < d.start + d.k; c++)
                for (int64_t p = colptr[c]; p < colptr[c + 1]; p++) {
                    int64_t lr = L.local(d, rowidx[p]);
                    X.dst.push_back(d.poff + lr * d.ldp + (c - d.start));
                    X.src.push_back(p);
                    X.seg_ptr.push_back((int64_t)X.src.size());
                }
        }
        X.level_seg[l + 1] = (int64_t)X.dst.size();
    }
    X.front_seg[P.nfronts] = (int64_t)X.dst.size();
    return X;
}

namespace {

// general case: columns with unsorted or repeated rows (serial; duplicates summed in caller order)
Scatter scatter_from_caller_general(const Plan& P, const Symbolic& S, const int64_t* indptr, const int64_t* indices,
                                    const std::vector<int64_t>& eq, const std::vector<int64_t>& owner) {
    Scatter X;
    LocalRows L(S.n);
    X.level_seg.assign(P.nlevels + 1, 0);
    X.front_seg.assign(P.nfronts + 1, 0);
    X.seg_ptr.push_back(0);
    std::vector<std::pair<int64_t, int64_t>> col;  // (dst, p)
    for (int64_t l = 0; l < P.nlevels; l++) {
        for (int64_t i = P.level_off[l]; i < P.level_off[l + 1]; i++) {
            X.front_seg[i] = (int64_t)X.dst.size();
            const DFront& d = P.fronts[P.level_order[i]];
            L.set(S, d);
            for (int64_t q = d.start; q < d.start + d.k; q++) {
                int64_t c = owner[q];
                if (c < 0) continue;
                col.clear();
                for (int64_t p = indptr[c]; p < indptr[c + 1]; p++) {
                    int64_t qr = eq[indices[p]];
                    if (qr < 0 || qr < q) continue;
                    col.push_back({d.poff + L.local(d, qr) * d.ldp + (q - d.start), p});
                }
                std::stable_sort(col.begin(), col.end(), [](auto& a, auto& b) { return a.first < b.first; });
                size_t j = 0;
                while (j < col.size()) {
                    size_t e = j + 1;
                    while (e < col.size() && col[e].first == col[j].first) e++;
                    X.dst.push_back(col[j].first);
                    for (size_t q2 = j; q2 < e; q2++) X.src.push_back(col[q2].second);
                    X.seg_ptr.push_back((int64_t)X.src.size());
                    j = e;
                }
            }
        }
        X.level_seg[l + 1] = (int64_t)X.dst.size();
    }
    X.front_seg[P.nfronts] = (int64_t)X.dst.size();
    return X;
}

}  // namespace

Scatter scatter_from_caller(const Plan& P, const Symbolic& S, int64_t ncaller, const int64_t* indptr,
                            const int64_t* indices, const std::vector<int64_t>& eq) {
    HostTimer timer("scatter_from_caller");
    std::vector<int64_t> owner(S.n, -1);
    for (int64_t i = 0; i < ncaller; i++)
        if (eq[i] >= 0) owner[eq[i]] = i;
    int64_t nt = P.nfronts;
    // pass 1: entries per front (in level order); any unsorted or repeated row sends
    // the whole matrix through the general path
    std::vector<int64_t> cnt(nt + 1, 0);
    std::atomic<bool> disorder{false};
    parallel_chunks(nt, 1, [&](int64_t a, int64_t b) {
        for (int64_t j = a; j < b; j++) {
            const DFront& d = P.fronts[P.level_order[j]];
            int64_t z = 0;
            for (int64_t q = d.start; q < d.start + d.k; q++) {
                int64_t c = owner[q];
                if (c < 0) continue;
                int64_t prev = -1;
                for (int64_t p = indptr[c]; p < indptr[c + 1]; p++) {
                    int64_t r = indices[p];
                    if (r <= prev) disorder = true;
                    prev = r;
                    int64_t qr = eq[r];
                    if (qr >= 0 && qr >= q) z++;
                }
            }
            cnt[j + 1] = z;
        }
    });
    timer.lap("pass 1");
    if (disorder) return scatter_from_caller_general(P, S, indptr, indices, eq, owner);
    Scatter X;
    X.front_seg.assign(nt + 1, 0);
    for (int64_t j = 0; j < nt; j++) X.front_seg[j + 1] = X.front_seg[j] + cnt[j + 1];
    X.level_seg.assign(P.nlevels + 1, 0);
    for (int64_t l = 0; l <= P.nlevels; l++) X.level_seg[l] = X.front_seg[P.level_off[l]];
    int64_t total = X.front_seg[nt];
    X.dst.resize(total);
    X.src.resize(total);
    X.seg_ptr.clear();  // one source per segment
    timer.lap("allocation");
    // pass 2: destinations, per thread a local-row table
    parallel_chunks(nt, 1, [&](int64_t a, int64_t b) {
        thread_local std::vector<int64_t> pos;
        if ((int64_t)pos.size() < S.n) pos.assign(S.n, 0);
        for (int64_t j = a; j < b; j++) {
            const DFront& d = P.fronts[P.level_order[j]];
            for (int64_t x = 0; x < d.u; x++) pos[S.rows[d.rows_off + x]] = d.k + x;
            int64_t o = X.front_seg[j];
            for (int64_t q = d.start; q < d.start + d.k; q++) {
                int64_t c = owner[q];
                if (c < 0) continue;
                for (int64_t p = indptr[c]; p < indptr[c + 1]; p++) {
                    int64_t qr = eq[indices[p]];
                    if (qr < 0 || qr < q) continue;
                    int64_t lr = qr < d.start + d.k ? qr - d.start : pos[qr];
                    X.dst[o] = d.poff + lr * d.ldp + (q - d.start);
                    X.src[o] = p;
                    o++;
                }
            }
        }
    });
    return X;
}

}  // namespace rfg
