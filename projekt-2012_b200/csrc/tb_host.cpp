// tb_host.cpp -- host orchestration of stage 2 (the walker and, for pairs whose
// stores are kept on a coarser grid, the stage-1 recompute of each level-1 cell
// the path enters).  No sequence data is touched on the host.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "traceback.h"

namespace swb {
namespace tb {

int traceback(cudaStream_t st, int sms, const uint8_t *d_rows, int64_t m, const uint8_t *d_cols, int64_t n,
              const swb_scoring *sc, const Plan &plan, const int2 *d_srows, const int2 *d_scols, swb_result *out,
              const Scratch &scr, std::string &err, int32_t *launches) {
    const int kBR = block_rows(), kBC = block_cols();
    const int64_t ops_cap = m + n + 8;
    int32_t G = 0, T = 0;
    int64_t P1 = 0, P2 = 0;
    reference_geometry(m, n, &G, &T, &P1, &P2);
    const int32_t X = T > 0 ? 4 * T : 20;
    const int64_t xp_cap = m / X + 8;
    char *d_ops = (char *)scr.ensure(scr.owner, kScrOps, (size_t)ops_cap);
    int64_t *d_xps = (int64_t *)scr.ensure(scr.owner, kScrXps, sizeof(int64_t) * 4 * (size_t)xp_cap);
    int64_t *d_state = (int64_t *)scr.ensure(scr.owner, kScrState, sizeof(int64_t) * 16);
    if (!d_ops || !d_xps || !d_state) {
        err = "traceback buffers: out of device memory";
        return SWB_ENOMEM;
    }
    std::vector<int64_t> S(state_slots(), 0);
    S[slot_r()] = out->end_row;
    S[slot_c()] = out->end_col;
    S[slot_state()] = 0;

    WalkInputs w{};
    w.rows = d_rows;
    w.cols = d_cols;
    w.m = m;
    w.n = n;
    w.sc = *sc;
    w.score = out->score;
    w.xp_interval = X;
    w.ops = d_ops;
    w.ops_cap = ops_cap;
    w.xps = d_xps;
    w.xp_cap = xp_cap;
    w.dstate = d_state;
    int rc;
    if (!plan.level1) {
        w.srows = d_srows;
        w.scols = d_scols;
        w.rr0 = 0;
        w.cc0 = 0;
        w.rr1 = m;
        w.cc1 = n;
        w.rtop = nullptr;
        w.rleft = nullptr;
        w.rcorner = 0;
        if ((rc = walk_region(st, sms, w, S.data(), scr, err, launches)) != SWB_OK) return rc;
    } else {
        // level 1: walk level-1 cell after level-1 cell
        for (int guard = 0; guard < (1 << 24) && !S[slot_done()]; ++guard) {
            const int64_t r = S[slot_r()], c = S[slot_c()];
            if (r < 0 || c < 0) {
                err = "traceback left the matrix";
                return SWB_ECUDA;
            }
            const int64_t RR0 = (r / plan.kr) * plan.kr, CC0 = (c / plan.kc) * plan.kc;
            const int64_t mm = r - RR0 + 1, nn = c - CC0 + 1;
            const int64_t nsr2 = mm / kBR, nsc2 = nn / kBC;
            int2 *s2r = (int2 *)scr.ensure(scr.owner, kScrSrows2, sizeof(int2) * (size_t)std::max<int64_t>(1, nsr2 * nn));
            int2 *s2c = (int2 *)scr.ensure(scr.owner, kScrScols2, sizeof(int2) * (size_t)std::max<int64_t>(1, nsc2 * mm));
            Stage1Plan p1 = stage1_plan(mm, nn, sms, 16, false);
            const int64_t W = (int64_t)p1.blocks * p1.warps_per_block;
            int4 *hb = (int4 *)scr.ensure(scr.owner, kScrHbuf, sizeof(int4) * (size_t)nn);
            BestRec *wb = (BestRec *)scr.ensure(scr.owner, kScrWbest, sizeof(BestRec) * (size_t)W);
            BestRec *bb = (BestRec *)scr.ensure(scr.owner, kScrBest, sizeof(BestRec));
            int32_t *ee = (int32_t *)scr.ensure(scr.owner, kScrErr, 4 * sizeof(int32_t));
            if (!s2r || !s2c || !hb || !wb || !bb || !ee) {
                err = "level-1 recompute buffers: out of device memory";
                return SWB_ENOMEM;
            }
            Stage1Args a{};
            a.rows = d_rows + RR0;
            a.cols = d_cols + CC0;
            a.m = mm;
            a.n = nn;
            a.open = sc->gap_open;
            a.ext = sc->gap_extend;
            a.gx = std::max(sc->gap_open, sc->gap_extend);
            a.mt1 = sc->match - sc->gap_open;
            a.mm1 = sc->mismatch - sc->gap_open;
            a.hbuf = hb;
            a.srows = nsr2 > 0 ? s2r : nullptr;
            a.sr_every = 1;
            a.nsr = nsr2;
            a.scols = nsc2 > 0 ? s2c : nullptr;
            a.sc_every = kBC;
            a.nsc = nsc2;
            const int2 *top = RR0 > 0 ? d_srows + (RR0 / plan.kr - 1) * n + CC0 : nullptr;
            const int2 *left = CC0 > 0 ? d_scols + (CC0 / plan.kc - 1) * m + RR0 : nullptr;
            int32_t corner = 0;
            if (RR0 > 0 && CC0 > 0) {
                int2 cv;
                cudaError_t ce = scr.get(scr.owner, &cv, d_srows + (RR0 / plan.kr - 1) * n + CC0 - 1, sizeof cv);
                if (ce != cudaSuccess) {
                    err = std::string("level-1 corner: ") + cudaGetErrorString(ce);
                    return SWB_ECUDA;
                }
                corner = cv.x;
            }
            a.top = top;
            a.left = left;
            a.corner = corner;
            a.r_origin = RR0;
            a.c_origin = CC0;
            a.nstrips = p1.nstrips;
            a.wbest = wb;
            a.best = bb;
            a.err = ee;
            a.gbest = a.err + 2;
            a.trace = nullptr;
            a.tie.mode = kTieRowMajor;
            cudaError_t e;
            if ((e = cudaMemsetAsync(hb, 0xFF, sizeof(int4) * (size_t)nn, st)) != cudaSuccess ||
                (e = cudaMemsetAsync(ee, 0, 4 * sizeof(int32_t), st)) != cudaSuccess ||
                (e = stage1_launch(a, p1, st)) != cudaSuccess) {
                err = std::string("level-1 recompute: ") + cudaGetErrorString(e);
                return SWB_ECUDA;
            }
            *launches += 2;
            w.srows = s2r;
            w.scols = s2c;
            w.rr0 = RR0;
            w.cc0 = CC0;
            w.rr1 = RR0 + mm;
            w.cc1 = CC0 + nn;
            w.rtop = top;
            w.rleft = left;
            w.rcorner = corner;
            if ((rc = walk_region(st, sms, w, S.data(), scr, err, launches)) != SWB_OK) return rc;
        }
        if (!S[slot_done()]) {
            err = "traceback did not finish";
            return SWB_ECUDA;
        }
    }
    // results: ops and crosspoints come out end -> start
    const int64_t nops = S[slot_nops()], nxp = S[slot_nxp()];
    if (nops > ops_cap || nxp > xp_cap) {
        err = "traceback output larger than its buffers";
        return SWB_ECUDA;
    }
    out->ops = (char *)std::malloc((size_t)nops + 1);
    out->xpoints = (swb_xpoint *)std::malloc(sizeof(swb_xpoint) * (size_t)(nxp + 2));
    std::vector<int64_t> hx((size_t)(4 * nxp + 4));
    if (!out->ops || !out->xpoints) {
        err = "out of host memory";
        return SWB_ENOMEM;
    }
    cudaError_t e;
    if ((e = scr.get(scr.owner, out->ops, d_ops, (size_t)nops)) != cudaSuccess ||
        (e = scr.get(scr.owner, hx.data(), d_xps, sizeof(int64_t) * 4 * (size_t)nxp)) != cudaSuccess) {
        err = std::string("traceback copy: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    std::reverse(out->ops, out->ops + nops);
    out->ops[nops] = 0;
    out->n_ops = nops;
    out->start_row = S[slot_start_r()];
    out->start_col = S[slot_start_c()];
    // [start (score 0), crosspoints top -> bottom, end (best score)]
    int64_t k = 0;
    out->xpoints[k++] = swb_xpoint{0, 0, out->start_row, out->start_col};
    for (int64_t i = nxp - 1; i >= 0; --i) {
        const int64_t *d = hx.data() + 4 * i;
        out->xpoints[k++] = swb_xpoint{(int32_t)d[3], (int32_t)d[2], d[0], d[1]};
    }
    out->xpoints[k++] = swb_xpoint{0, out->score, out->end_row, out->end_col};
    out->n_xpoints = k;
    out->xpoint_interval = X;
    return SWB_OK;
}

}  // namespace tb
}  // namespace swb
