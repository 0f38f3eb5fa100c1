// fvb_serve.cpp -- serving loop over the batched form (continuous batching).
//
// Requests become visible at their arrival time.  Between batch rounds the
// loop admits waiting requests -- in arrival order, or least estimated work
// first -- while the HBM budget, the instance slots and the cell cap allow,
// advances every admitted instance together for `steps_per_round` steps
// (one persistent launch per RK stage, graph replayed), then retires the
// instances that reached their t_end and frees their memory, so later
// arrivals join as room appears.  States never leave the device except the
// final state a request asks for (copied out as it retires).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <thread>
#include <vector>

#include "fvb_host.h"

using namespace fvb;
using clk = std::chrono::steady_clock;

extern "C" fvb_status fvb_serve_run(const fvb_serve_config *cfg, const fvb_request *reqs, int nreq,
                                    fvb_request_result *res, double *wall_seconds)
{
    NvtxRange nvtx_range("fvb_serve_run");
    if (!cfg || (!reqs && nreq) || (!res && nreq) || nreq < 0) return fail(FVB_ERR_INVALID, "bad argument");
    if ((cfg->policy != FVB_SERVE_FIFO && cfg->policy != FVB_SERVE_SHORTEST_FIRST) || !(cfg->max_cells >= 0.0))
        return fail(FVB_ERR_INVALID, "unknown admission policy %d or negative cell cap", cfg->policy);
    fvb_batch *b = nullptr;
    fvb_status st = fvb_batch_create(&cfg->batch, &b);
    if (st) return st;
    const int spr = cfg->steps_per_round > 0 ? cfg->steps_per_round : 8;
    std::vector<int> order(nreq);
    for (int i = 0; i < nreq; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int c) { return reqs[a].arrival < reqs[c].arrival; });
    for (int i = 0; i < nreq; ++i) {
        std::memset(&res[i], 0, sizeof res[i]);
        res[i].admitted = res[i].finished = -1.0;
    }
    std::vector<int> slot_req(65536, -1);
    std::deque<int> waiting;
    // the shortest-first key: cells x steps, steps ~ n t_end at a fixed CFL
    auto work = [&](int r) { const double n = reqs[r].desc.n; return n * n * n * reqs[r].desc.t_end; };
    const bool shortest = cfg->policy == FVB_SERVE_SHORTEST_FIRST;
    double live_cells = 0.0;
    size_t next = 0;
    int done = 0;
    const auto t0 = clk::now();
    auto now = [&] { return std::chrono::duration<double>(clk::now() - t0).count(); };
    std::vector<int> ids(4096);
    fvb_status result = FVB_OK;
    while (done < nreq) {
        double tnow = now();
        bool arrived = false;
        while (next < order.size() && reqs[order[next]].arrival <= tnow) {
            waiting.push_back(order[next++]);
            arrived = true;
        }
        if (shortest && arrived)
            std::stable_sort(waiting.begin(), waiting.end(), [&](int x, int y) { return work(x) < work(y); });
        // admission in the policy's order; a request that does not fit waits
        // (head of line) until an instance retires
        while (!waiting.empty()) {
            int r = waiting.front();
            const double cells = (double)reqs[r].desc.n * reqs[r].desc.n;
            if (cfg->max_cells > 0 && live_cells > 0 && live_cells + cells > cfg->max_cells) break;
            int id = -1;
            fvb_status a = fvb_batch_add(b, &reqs[r].desc, &id);
            if (a == FVB_ERR_NOMEM) {
                if (fvb_batch_active(b) == 0) {  // can never fit
                    res[r].status = FVB_ERR_NOMEM;
                    res[r].admitted = res[r].finished = now();
                    waiting.pop_front();
                    ++done;
                    continue;
                }
                break;
            }
            if (a) {
                res[r].status = a;
                res[r].admitted = res[r].finished = now();
                waiting.pop_front();
                ++done;
                continue;
            }
            slot_req[id] = r;
            res[r].admitted = now();
            live_cells += cells;
            waiting.pop_front();
        }
        if (fvb_batch_active(b) == 0) {
            if (next >= order.size() && waiting.empty()) break;
            if (next < order.size()) {
                double wait = reqs[order[next]].arrival - now();
                if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.01)));
            }
            continue;
        }
        st = fvb_batch_run(b, spr);
        int nd = 0;
        if (!st) st = fvb_batch_poll(b, ids.data(), (int)ids.size(), &nd);
        if (st) { result = st; break; }
        double tf = now();
        for (int k = 0; k < nd; ++k) {
            int id = ids[k], r = slot_req[id];
            if (r < 0) continue;
            fvb_stats s;
            if (fvb_batch_instance_stats(b, id, &s) == FVB_OK) {
                res[r].status = s.status;
                res[r].steps = s.steps;
                res[r].t = s.t;
            }
            if (reqs[r].out) {
                const fvb_status g =
                    fvb_batch_get_state(b, id, reqs[r].out, reqs[r].out_layout, reqs[r].out_dtype, 1);
                if (g) { result = g; break; }
                tf = now();
            }
            res[r].finished = tf;
            slot_req[id] = -1;
            live_cells -= (double)reqs[r].desc.n * reqs[r].desc.n;
            fvb_batch_remove(b, id);
            ++done;
        }
        if (result) break;
        if (cfg->max_seconds > 0 && now() > cfg->max_seconds) { result = fail(FVB_ERR_TIMEOUT, "serving run exceeded %.1f s", cfg->max_seconds); break; }
    }
    if (wall_seconds) *wall_seconds = now();
    fvb_batch_destroy(b);
    return result;
}
