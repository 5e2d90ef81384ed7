// tb_host.cpp -- host orchestration of stage 2 (the walker and, for pairs whose
// stores are kept on a coarser grid, the stage-1 recompute of each level-1 cell
// the path enters).  No sequence data is touched on the host.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "batch.h"
#include "traceback.h"

namespace swb {
namespace tb {

// Level-1 cells recomputed per corridor round: about two waves of strips at 16
// warps per SM, and at most 8 GiB of their 512 x 256 stores.
int64_t level1_corridor_cells(const Plan &plan, int sms) {
    const int64_t strips_per_cell = (plan.kr + block_rows() - 1) / block_rows();
    const int64_t cell_store = level1_cell_store_bytes(plan);
    int64_t cap = std::max<int64_t>(3, (2LL * 16 * std::max(1, sms)) / strips_per_cell);
    return std::min<int64_t>(cap, std::max<int64_t>(3, (int64_t)(8ULL << 30) / std::max<int64_t>(1, cell_store)));
}

int64_t level1_cell_store_bytes(const Plan &plan) {
    return 8 * ((plan.kr / block_rows()) * plan.kc + (plan.kc / block_cols()) * plan.kr) + 16 * plan.kc;
}

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
        w.br = plan.br;
        w.srows = d_srows;
        w.scols = d_scols;
        w.rr0 = 0;
        w.cc0 = 0;
        w.rr1 = m;
        w.cc1 = n;
        w.rtop = nullptr;
        w.rleft = nullptr;
        if ((rc = walk_region(st, sms, w, S.data(), scr, err, launches)) != SWB_OK) return rc;
    } else {
        // level 1: rounds of a predicted corridor of level-1 cells, recomputed at
        // once by one batched launch that writes each cell's 512 x 256 stores,
        // then walked cell by cell
        const int64_t cap = level1_corridor_cells(plan, sms);
        std::vector<int64_t> cells;  // (RR0, CC0) pairs
        std::vector<BatchPair> bp;
        std::vector<int32_t> up;
        for (int round = 0; round < (1 << 24) && !S[slot_done()]; ++round) {
            const int64_t r = S[slot_r()], c = S[slot_c()];
            if (r < 0 || c < 0) {
                err = "traceback left the matrix";
                return SWB_ECUDA;
            }
            // corridor: the staircase of level-1 cells along the diagonal from (r, c),
            // with the cell above and the cell to the left of each as margin
            cells.clear();
            auto add = [&](int64_t bi, int64_t bj) {
                if (bi < 0 || bj < 0 || (int64_t)cells.size() / 2 >= cap) return;
                for (size_t q = cells.size() >= 16 ? cells.size() - 16 : 0; q < cells.size(); q += 2)
                    if (cells[q] == bi * plan.kr && cells[q + 1] == bj * plan.kc) return;
                cells.push_back(bi * plan.kr);
                cells.push_back(bj * plan.kc);
            };
            {
                int64_t rr = r, ccc = c, bi = r / plan.kr, bj = c / plan.kc;
                add(bi, bj);
                add(bi - 1, bj);
                add(bi, bj - 1);
                while ((int64_t)cells.size() / 2 < cap) {
                    const int64_t d = std::min(rr - bi * plan.kr + 1, ccc - bj * plan.kc + 1);
                    rr -= d;
                    ccc -= d;
                    if (rr < 0 || ccc < 0) break;
                    bi = rr / plan.kr;
                    bj = ccc / plan.kc;
                    add(bi, bj);
                    add(bi - 1, bj);
                    add(bi, bj - 1);
                }
            }
            const int64_t ncell = (int64_t)cells.size() / 2;
            // one batched launch: every cell is a sub-rectangle with its boundaries
            bp.assign((size_t)ncell, BatchPair{});
            up.clear();
            int64_t hb = 0, srn = 0, scn = 0;
            for (int64_t q = 0; q < ncell; ++q) {
                const int64_t RR0 = cells[2 * q], CC0 = cells[2 * q + 1];
                const int64_t mm = std::min(plan.kr, m - RR0), nn = std::min(plan.kc, n - CC0);
                BatchPair &d = bp[(size_t)q];
                d.row_off = RR0;
                d.col_off = CC0;
                d.m = (int32_t)mm;
                d.n = (int32_t)nn;
                d.nstrips = (int32_t)((mm + kBatchStripRows - 1) / kBatchStripRows);
                d.unit0 = d.ufirst = (int32_t)up.size();
                d.ucount = d.nstrips;
                d.slot = (int32_t)q;
                d.hbuf_off = hb;
                hb += nn;
                d.sr_every = 1;
                d.sc_every = kBC;
                d.sr_off = srn;
                d.sc_off = scn;
                srn += (mm / kBR) * nn;
                scn += (nn / kBC) * mm;
                d.tie.mode = kTieRowMajor;
                d.tie.G = d.tie.T = 1;
                d.tie.C = 1;
                d.top = RR0 > 0 ? d_srows + (RR0 / plan.kr - 1) * n + CC0 : nullptr;
                d.left = CC0 > 0 ? d_scols + (CC0 / plan.kc - 1) * m + RR0 : nullptr;
                for (int32_t u = 0; u < d.nstrips; ++u) up.push_back((int32_t)q);
            }
            BatchPair *dp = (BatchPair *)scr.ensure(scr.owner, kScrL1Pairs, sizeof(BatchPair) * bp.size());
            int32_t *du = (int32_t *)scr.ensure(scr.owner, kScrL1Units, sizeof(int32_t) * up.size());
            int4 *dh = (int4 *)scr.ensure(scr.owner, kScrL1Hbuf, sizeof(int4) * (size_t)std::max<int64_t>(1, hb));
            int32_t *dg = (int32_t *)scr.ensure(scr.owner, kScrL1Gbest, sizeof(int32_t) * (size_t)ncell);
            BestRec *dub = (BestRec *)scr.ensure(scr.owner, kScrL1Ubest, sizeof(BestRec) * up.size());
            BestRec *dpb = (BestRec *)scr.ensure(scr.owner, kScrL1Pbest, sizeof(BestRec) * (size_t)ncell);
            int32_t *dc = (int32_t *)scr.ensure(scr.owner, kScrL1Ctl, 4 * sizeof(int32_t));
            int2 *s2r = (int2 *)scr.ensure(scr.owner, kScrSrows2, sizeof(int2) * (size_t)std::max<int64_t>(1, srn));
            int2 *s2c = (int2 *)scr.ensure(scr.owner, kScrScols2, sizeof(int2) * (size_t)std::max<int64_t>(1, scn));
            if (!dp || !du || !dh || !dg || !dub || !dpb || !dc || !s2r || !s2c) {
                err = "level-1 recompute buffers: out of device memory";
                return SWB_ENOMEM;
            }
            BatchArgs ba{};
            ba.seq = d_rows;
            ba.cseq = d_cols;
            ba.open = sc->gap_open;
            ba.ext = sc->gap_extend;
            ba.gx = std::max(sc->gap_open, sc->gap_extend);
            ba.mt1 = sc->match - sc->gap_open;
            ba.mm1 = sc->mismatch - sc->gap_open;
            ba.pairs = dp;
            ba.unit_pair = du;
            ba.nunits = (int64_t)up.size();
            ba.hbuf = dh;
            ba.gbest = dg;
            ba.ubest = dub;
            ba.ctl = dc;
            ba.srows = s2r;
            ba.scols = s2c;
            cudaError_t e;
            if ((e = scr.put(scr.owner, dp, bp.data(), sizeof(BatchPair) * bp.size())) != cudaSuccess ||
                (e = scr.put(scr.owner, du, up.data(), sizeof(int32_t) * up.size())) != cudaSuccess ||
                (e = cudaMemsetAsync(dh, 0xFF, sizeof(int4) * (size_t)std::max<int64_t>(1, hb), st)) != cudaSuccess ||
                (e = cudaMemsetAsync(dg, 0, sizeof(int32_t) * (size_t)ncell, st)) != cudaSuccess ||
                (e = cudaMemsetAsync(dpb, 0, sizeof(BestRec) * (size_t)ncell, st)) != cudaSuccess ||
                (e = cudaMemsetAsync(dc, 0, 4 * sizeof(int32_t), st)) != cudaSuccess ||
                (e = batch_launch(ba, false, kBatchBounds, kBatchR, sms, 0, ncell, dpb, st)) != cudaSuccess) {
                err = std::string("level-1 recompute: ") + cudaGetErrorString(e);
                return SWB_ECUDA;
            }
            *launches += 2;
            int32_t ctl[4];
            if ((e = scr.get(scr.owner, ctl, dc, sizeof ctl)) != cudaSuccess) {
                err = std::string("level-1 recompute: ") + cudaGetErrorString(e);
                return SWB_ECUDA;
            }
            if (ctl[1] != 0) {
                err = "level-1 recompute: a bounded wait between strips ran out";
                return SWB_ETIMEOUT;
            }
            // walk cell after cell while the path stays in the corridor
            for (;;) {
                const int64_t rr = S[slot_r()], ccc = S[slot_c()];
                if (S[slot_done()] || rr < 0 || ccc < 0) break;
                const int64_t RR0 = (rr / plan.kr) * plan.kr, CC0 = (ccc / plan.kc) * plan.kc;
                int64_t q = -1;
                for (int64_t t = 0; t < ncell; ++t)
                    if (cells[2 * t] == RR0 && cells[2 * t + 1] == CC0) {
                        q = t;
                        break;
                    }
                if (q < 0) break;  // left the corridor: next round
                const BatchPair &d = bp[(size_t)q];
                w.srows = s2r + d.sr_off;
                w.scols = s2c + d.sc_off;
                w.rr0 = RR0;
                w.cc0 = CC0;
                w.rr1 = RR0 + d.m;
                w.cc1 = CC0 + d.n;
                w.rtop = d.top;
                w.rleft = d.left;
                if ((rc = walk_region(st, sms, w, S.data(), scr, err, launches)) != SWB_OK) return rc;
                if (S[slot_r()] == rr && S[slot_c()] == ccc && !S[slot_done()]) {
                    err = "traceback made no progress in a level-1 cell";
                    return SWB_ECUDA;
                }
            }
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
