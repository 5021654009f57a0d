// Many independent H_eff plans merged into one plan (the batching form of the path).
//
// The reference splits the ket sectors of one H.psi across devices and host threads
// (solver/tasks.cpp:884-977) and runs one schedule per solve.  Here the work lists of N
// plans (N site problems, e.g. N independent small DMRG solves) are concatenated into the
// lists of one plan, so that one T-GEMM, one S-build and one split-K L.S launch sequence
// (per tile shape) applies every plan's H_eff at once.  The plans' vectors live in one
// arena (plan i's vector at offset xo[i]); T, S and the split-K partials get merged buffers
// of their own; the boundaries and coefficient blocks stay in the plans' buffers and are
// addressed from a common base (the lowest of the plans' buffer addresses), each job's
// offset shifted by its plan's distance from that base.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "heff.hpp"

namespace qcm {

namespace {

uint64_t round32(uint64_t n) { return (n + 31) / 32 * 32; }

// element distance of p from base (both double*, p >= base)
uint64_t dist(const double* p, const double* base) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p), b = reinterpret_cast<uintptr_t>(base);
    if (a < b || (a - b) % sizeof(double)) throw std::runtime_error("plan group: buffer below its base or misaligned");
    return uint64_t((a - b) / sizeof(double));
}

}  // namespace

std::unique_ptr<HeffPlan> merge_plans(const std::vector<HeffPlan*>& plans, std::vector<uint64_t>& xo, cudaStream_t s) {
    if (plans.empty()) throw std::runtime_error("plan group: no plans");
    auto g = std::make_unique<HeffPlan>();
    g->merged = true;
    g->stream = s;
    const double *bL = nullptr, *bR = nullptr, *bW = nullptr;
    for (const HeffPlan* p : plans) {
        if (!p || !p->L || !p->R || p->merged) throw std::runtime_error("plan group: a plan without boundaries, or a group");
        if (!p->d_W.get()) throw std::runtime_error("plan group: a plan without its coefficient blocks on the device");
        if (p->streamed()) throw std::runtime_error("plan group: a plan with streamed coefficient blocks");
        const double* l = p->L->data.get();
        const double* r = p->R->data.get();
        const double* w = p->d_W.get();
        bL = (!bL || l < bL) ? l : bL;
        bR = (!bR || r < bR) ? r : bR;
        bW = (!bW || w < bW) ? w : bW;
    }
    g->base_L = bL;
    g->base_R = bR;
    g->base_W = bW;
    {
        std::size_t nt = 0, nu = 0, nl = 0, ns = 0, nk = 0, ng = 0, no = 0;
        std::size_t ntt[N_SHAPES] = {}, nut[N_SHAPES] = {},not_[N_SHAPES] = {}, nki[N_SHAPES] = {};
        for (const HeffPlan* p : plans) {
            nt += p->tjobs.size(); nu += p->units.size(); nl += p->line_b1.size(); ns += p->slice_off.size();
            nk += p->klist.size(); ng += p->segs.size(); no += p->outs.size();
            for (int sh = 0; sh < N_SHAPES; ++sh) {
                ntt[sh] += p->ttiles[sh].size(); nut[sh] += p->utiles[sh].size();
                not_[sh] += p->otiles[sh].size(); nki[sh] += p->kitems[sh].size();
            }
        }
        g->tjobs.reserve(nt); g->units.reserve(nu); g->line_b1.reserve(nl); g->slice_off.reserve(ns);
        g->klist.reserve(nk); g->segs.reserve(ng); g->outs.reserve(no);
        for (int sh = 0; sh < N_SHAPES; ++sh) {
            g->ttiles[sh].reserve(ntt[sh]); g->utiles[sh].reserve(nut[sh]);
            g->otiles[sh].reserve(not_[sh]); g->kitems[sh].reserve(nki[sh]);
        }
    }
    xo.assign(plans.size(), 0);
    uint64_t xl = 0, tl = 0, sl = 0;
    uint64_t kl_items[N_SHAPES] = {};
    for (std::size_t i = 0; i < plans.size(); ++i) {
        const HeffPlan& p = *plans[i];
        xo[i] = xl;
        const uint64_t to = tl, so = sl;
        const uint64_t dL = dist(p.L->data.get(), bL), dR = dist(p.R->data.get(), bR), dW = dist(p.d_W.get(), bW);
        if (dW % 4) throw std::runtime_error("plan group: coefficient blocks not 16-byte aligned against their base");
        // T-GEMM jobs and their tiles
        const uint32_t j0 = uint32_t(g->tjobs.size());
        for (TJobD j : p.tjobs) {
            j.a_off += xl; j.b_off += dR; j.c_off += to;
            g->tjobs.push_back(j);
        }
        for (int sh = 0; sh < N_SHAPES; ++sh)
            for (TileD t : p.ttiles[sh]) { t.item += j0; g->ttiles[sh].push_back(t); }
        // S-build units, their lines, slices, k-step lists and tiles
        const uint32_t u0 = uint32_t(g->units.size()), l0 = uint32_t(g->line_b1.size()), s0 = uint32_t(g->slice_off.size());
        const uint32_t k0 = uint32_t(g->klist.size());
        for (UnitD u : p.units) {
            u.s_off += so; u.w_off += dW; u.line0 += l0; u.slice0 += s0;
            g->units.push_back(u);
        }
        g->line_b1.insert(g->line_b1.end(), p.line_b1.begin(), p.line_b1.end());
        for (uint64_t o : p.slice_off) g->slice_off.push_back(o + to);
        g->klist.insert(g->klist.end(), p.klist.begin(), p.klist.end());
        for (int sh = 0; sh < N_SHAPES; ++sh)
            for (TileD t : p.utiles[sh]) { t.item += u0; t.pad += k0; g->utiles[sh].push_back(t); }
        // L.S segments, output blocks, output tiles and split-K items
        const uint32_t sg0 = uint32_t(g->segs.size()), o0 = uint32_t(g->outs.size());
        for (SegD sg : p.segs) { sg.l_off += dL; sg.s_off += so; g->segs.push_back(sg); }
        for (OutD o : p.outs) { o.y_off += xl; o.seg_start += sg0; g->outs.push_back(o); }
        for (int sh = 0; sh < N_SHAPES; ++sh) {
            const uint32_t ot0 = uint32_t(g->otiles[sh].size());
            for (OTileD t : p.otiles[sh]) { t.out += o0; t.part0 += uint32_t(kl_items[sh]); g->otiles[sh].push_back(t); }
            for (KItemD k : p.kitems[sh]) { k.tile += ot0; k.seg += sg0; k.slot += uint32_t(kl_items[sh]); g->kitems[sh].push_back(k); }
            kl_items[sh] += p.kitems[sh].size();
        }
        g->flops += p.flops; g->flops_t += p.flops_t; g->flops_s += p.flops_s; g->flops_ls += p.flops_ls;
        g->flops_sexec += p.flops_sexec; g->flops_sdense += p.flops_sdense;
        g->n_alpha += p.n_alpha;
        xl += round32(p.x_len);
        tl += round32(p.t_len);
        sl += round32(p.s_len);
    }
    g->x_len = xl;
    g->t_len = tl;
    g->s_len = sl;
    uint64_t pl = 0;
    for (int sh = 0; sh < N_SHAPES; ++sh) pl = std::max<uint64_t>(pl, kl_items[sh] * shape_bm(sh) * shape_bn(sh));
    g->p_len = pl;
    static const bool tdbg = std::getenv("QCM_PLAN_TIMING") != nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    upload_merged(*g);
    if (tdbg) {
        const auto t1 = std::chrono::steady_clock::now();
        std::fprintf(stderr, "plan group: %zu plans, %zu T jobs, %zu units, %zu k-list words, upload %.4f s\n", plans.size(),
                     g->tjobs.size(), g->units.size(), g->klist.size(), std::chrono::duration<double>(t1 - t0).count());
    }
    return g;
}

}  // namespace qcm
