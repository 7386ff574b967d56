// Shot server: continuous batching of RTM shots on one device.
//
// Two host threads.  The loader admits queued shots (first fit in arrival
// order, bounded by max_active and the HBM budget), builds each one's
// simulator (model upload, source, receivers, observed traces) on the
// simulator's own stream and hands it to the scheduler.  The scheduler runs
// rounds: every resident shot's next units (fused steps) go into one launch
// as parallel branches forked from and joined back into the server's stream,
// captured as a CUDA graph when use_graphs is set.  Round r+1 is planned,
// captured and issued behind round r while r runs, so the device does not
// wait for the host between rounds; shots that finish in round r are read
// back and released after it completes, while round r+1 runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <tuple>
#include <vector>

#include "tti_common.cuh"
#include "tti_internal.cuh"
#include "tti_shot.cuh"

namespace {

using namespace tti;

int rc_of(cudaError_t e)
{
    if (e == cudaSuccess) return TTI_OK;
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? TTI_ENOMEM : TTI_ELAUNCH;
}

struct Shot {
    int64_t ticket = 0;
    tti_shot_request req{};
    tti_shot_result res{};
    tti_sim* sim = nullptr;
    cudaEvent_t join = nullptr;
    double unit_ms = 1.0;  // estimated device time of one unit
    int64_t planned_left = 0;
};

// Per grid: device time of one fused forward, adjoint, imaging launch.
struct GridCost {
    float fwd_ms = 0, adj_ms = 0, img_ms = 0;
};

} // namespace

struct tti_server {
    tti_server_config cfg{};
    int device = 0;
    std::chrono::steady_clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Shot*> queue;        // submitted, not admitted
    std::vector<Shot*> ready;       // built by the loader, not yet scheduled
    std::map<int64_t, Shot*> done;  // finished, result not taken
    int64_t next_ticket = 1;
    int resident = 0;  // admitted (being built, ready or scheduled)
    int64_t used = 0;  // bytes reserved by resident shots
    bool stop = false;
    std::map<std::tuple<int, int, int>, GridCost> costs;
    tti_server_stats stats{};
    std::thread loader, scheduler, retirer;
    std::deque<std::pair<Shot*, int>> retire;  // finished on the device: read back and free
    bool scheduler_done = false;
    // The shots' device memory comes from a pool of the server's own that
    // keeps freed memory mapped, so a new shot reuses a finished one's pages
    // instead of mapping its stores afresh; when a shot's allocation fails
    // behind fragmented free chunks the pool is trimmed and the set-up
    // retried once.
    cudaMemPool_t pool = nullptr;
    // scheduler-owned
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr;
    cudaEvent_t round_start[2] = {}, round_end[2] = {};
    cudaGraphExec_t exec[2] = {};

    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

constexpr int64_t kMaxUnitsPerRound = 128;  // fused steps of one shot in one round

tti_sim_config shot_config(const tti_server* srv, const tti_shot_request& r, int ckpt)
{
    tti_sim_config c{};
    c.nx = r.nx;
    c.ny = r.ny;
    c.nz = r.nz;
    c.dx = r.dx;
    c.dy = r.dy;
    c.dz = r.dz;
    c.dt = r.dt;
    c.nt = r.nt;
    c.xcorr_step = r.xcorr_step;
    c.sponge_width = r.sponge_width;
    c.free_surface = r.free_surface;
    c.fused = 1;
    c.save_snapshots = 1;
    c.snap_precision = srv->cfg.snap_precision;
    c.scheme = srv->cfg.scheme;
    c.checkpoint_every = ckpt;
    c.use_graphs = 0;
    return c;
}

// Footprint of a shot with checkpoint segment K (0: none), including the
// receiver buffers and the transient buffers of the model upload.
int footprint(const tti_server* srv, const tti_shot_request& r, int ckpt, int64_t* out)
{
    tti_sim_config c = shot_config(srv, r, ckpt);
    int64_t b = 0;
    int rc = tti_sim_footprint_bytes(&c, &b);
    if (rc) return rc;
    const int64_t nvol = (int64_t)(32 * ((r.nx + 7) / 32 + 1)) * (r.ny + 8) * (r.nz + 8);
    b += (int64_t)r.nrec * (8 + 2 * 4 * (int64_t)r.nt);
    b += 8 * nvol * 4;  // set-up temporaries (seven parameter volumes and one dense array)
    *out = b;
    return TTI_OK;
}

// Checkpoint segment for a shot: none if it fits the budget with every
// snapshot kept, else the multiple of xcorr_step that minimises the
// footprint (checkpoints ~ nt/K, stored segment ~ K).
int choose_checkpoint(const tti_server* srv, const tti_shot_request& r, int64_t budget, int* ckpt, int64_t* bytes)
{
    int64_t b0 = 0;
    int rc = footprint(srv, r, 0, &b0);
    if (rc) return rc;
    if (b0 <= budget) {
        *ckpt = 0;
        *bytes = b0;
        return TTI_OK;
    }
    int best = 0;
    int64_t best_b = b0;
    for (int k = r.xcorr_step; k < r.nt; k += r.xcorr_step) {
        int64_t b = 0;
        if (footprint(srv, r, k, &b)) continue;
        if (b < best_b) {
            best_b = b;
            best = k;
        }
    }
    *ckpt = best;
    *bytes = best_b;
    return TTI_OK;
}

// The shot's simulator with its model, source, receivers and observed
// traces; *t_alloc: when its device memory was in place.
int setup_sim(tti_server* srv, Shot* sh, double* t_alloc)
{
    const tti_shot_request& r = sh->req;
    tti_sim_config c = shot_config(srv, r, sh->res.checkpoint_every);
    int rc = sim_create_in_pool(&c, srv->pool, &sh->sim);
    if (!rc) rc = rc_of(cudaStreamSynchronize(shot_stream(sh->sim)));
    *t_alloc = srv->now();
    if (!rc) rc = tti_sim_set_model(sh->sim, r.vp, r.eps, r.delta, r.vs, r.theta, r.phi, r.rho);
    if (!rc) rc = tti_sim_set_source(sh->sim, r.src_ix, r.src_iy, r.src_iz, r.wavelet, r.nt);
    if (!rc) rc = tti_sim_set_receivers(sh->sim, r.nrec, r.rec_ixyz);
    if (!rc) rc = shot_upload_observed(sh->sim, r.observed);
    if (!rc) rc = rc_of(cudaStreamSynchronize(shot_stream(sh->sim)));
    return rc;
}

int build_shot(tti_server* srv, Shot* sh)
{
    const tti_shot_request& r = sh->req;
    double t0 = srv->now(), t1 = t0;
    int rc = setup_sim(srv, sh, &t1);
    if (rc == TTI_ENOMEM && srv->pool) {  // free chunks too fragmented: return them and retry once
        if (sh->sim) {
            tti_sim_destroy(sh->sim);
            sh->sim = nullptr;
        }
        cudaMemPoolTrimTo(srv->pool, 0);
        cudaGetLastError();
        rc = setup_sim(srv, sh, &t1);
    }
    const double t2 = srv->now();
    // per-grid cost estimate: autotune on first sight, else a throughput model
    const auto key = std::make_tuple(r.nx, r.ny, r.nz);
    GridCost gc{};
    bool have = false;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        auto it = srv->costs.find(key);
        if (it != srv->costs.end()) {
            gc = it->second;
            have = true;
        }
    }
    if (!rc && !have) {
        if (srv->cfg.autotune) {
            tti_tune_report tr{};
            rc = tti_sim_autotune(sh->sim, 2, &tr);
            gc.fwd_ms = tr.ms[0];
            gc.adj_ms = tr.ms[1];
            gc.img_ms = tr.ms[2];
        } else {
            const double pts = (double)r.nx * r.ny * r.nz;
            gc.fwd_ms = (float)(pts / 2.3e7);  // ~23 Gpts/s forward, ~16 adjoint, ~20 imaging
            gc.adj_ms = (float)(pts / 1.6e7);
            gc.img_ms = (float)(pts / 2.0e7);
        }
        if (!rc) {
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->costs[key] = gc;
        }
    }
    sh->unit_ms = std::max(1e-3, (double)std::max(gc.fwd_ms, gc.adj_ms + gc.img_ms / std::max(1, r.xcorr_step)));
    {
        const double t3 = srv->now();
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stats.setup_alloc_ms += 1e3 * (t1 - t0);
        srv->stats.setup_model_ms += 1e3 * (t2 - t1);
        srv->stats.setup_tune_ms += 1e3 * (t3 - t2);
    }
    if (!rc) rc = shot_begin(sh->sim);
    if (!rc) rc = rc_of(cudaStreamSynchronize(shot_stream(sh->sim)));
    if (!rc) rc = rc_of(cudaEventCreateWithFlags(&sh->join, cudaEventDisableTiming));
    if (!rc) sh->planned_left = shot_units_left(sh->sim);
    return rc;
}

void finish_shot(tti_server* srv, Shot* sh, int status)
{
    sh->res.status = status;
    if (sh->sim) {
        if (!status && sh->req.image_vp) status = tti_sim_get_image(sh->sim, sh->req.image_vp, nullptr, 0);
        if (!status && sh->req.image_rho) status = tti_sim_get_image(sh->sim, nullptr, sh->req.image_rho, 0);
        if (!status && sh->req.traces && sh->req.nrec) status = shot_read_traces(sh->sim, sh->req.traces);
        sh->res.launches = tti_sim_launch_count(sh->sim);
        tti_sim_destroy(sh->sim);
        sh->sim = nullptr;
        sh->res.status = status;
    }
    if (sh->join) {
        cudaEventDestroy(sh->join);
        sh->join = nullptr;
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    sh->res.t_done = srv->now();
    srv->used -= sh->res.footprint;
    srv->resident -= 1;
    srv->done[sh->ticket] = sh;
    srv->cv.notify_all();
}

// Read-back and release of finished shots, off the scheduler thread so that
// the next round is issued while a result is being copied out.
void retirer_main(tti_server* srv)
{
    cudaSetDevice(srv->device);
    for (;;) {
        std::pair<Shot*, int> job{nullptr, 0};
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            while (srv->retire.empty() && !srv->scheduler_done) srv->cv.wait_for(lk, std::chrono::milliseconds(50));
            if (srv->retire.empty()) return;
            job = srv->retire.front();
            srv->retire.pop_front();
        }
        finish_shot(srv, job.first, job.second);
    }
}

void retire_later(tti_server* srv, Shot* sh, int status)
{
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->retire.push_back({sh, status});
    srv->cv.notify_all();
}

void loader_main(tti_server* srv)
{
    cudaSetDevice(srv->device);
    for (;;) {
        Shot* sh = nullptr;
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            for (;;) {
                if (srv->resident < srv->cfg.max_active) {
                    for (auto it = srv->queue.begin(); it != srv->queue.end(); ++it)
                        if ((*it)->res.footprint <= srv->cfg.hbm_budget - srv->used) {
                            sh = *it;
                            srv->queue.erase(it);
                            break;
                        }
                }
                if (sh) break;
                if (srv->stop && srv->queue.empty()) return;
                srv->cv.wait_for(lk, std::chrono::milliseconds(50));
            }
            srv->used += sh->res.footprint;
            srv->resident += 1;
            sh->res.t_admit = srv->now();
        }
        const double t_setup = srv->now();
        int rc = build_shot(srv, sh);
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->stats.setup_ms += 1e3 * (srv->now() - t_setup);
        }
        if (rc) {
            finish_shot(srv, sh, rc);
            continue;
        }
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->ready.push_back(sh);
        srv->stats.max_resident = std::max(srv->stats.max_resident, srv->resident);
        srv->cv.notify_all();
    }
}

// Enqueue (or capture into exec[slot]) one round on srv->main: each planned
// shot's units in its own branch, forked from and joined into srv->main.
int build_round(tti_server* srv, const std::vector<std::pair<Shot*, int64_t>>& plan, int slot)
{
    cudaStream_t m = srv->main;
    const bool graph = srv->cfg.use_graphs != 0;
    int rc = TTI_OK;
    if (!graph) cudaEventRecord(srv->round_start[slot], m);  // direct launches: the round starts here
    if (graph && (rc = rc_of(cudaStreamBeginCapture(m, cudaStreamCaptureModeThreadLocal)))) return rc;
    if (!rc) rc = rc_of(cudaEventRecord(srv->fork, m));
    for (auto& pu : plan) {
        if (rc) break;
        Shot* sh = pu.first;
        cudaStream_t st = shot_stream(sh->sim);
        rc = rc_of(cudaStreamWaitEvent(st, srv->fork, 0));
        int64_t got = 0;
        if (!rc) rc = shot_advance(sh->sim, st, pu.second, &got);
        sh->res.units += got;
        if (!rc) rc = rc_of(cudaEventRecord(sh->join, st));
        if (!rc) rc = rc_of(cudaStreamWaitEvent(m, sh->join, 0));
    }
    if (graph) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(m, &g);
        if (!rc) rc = rc_of(e);
        cudaGraphExec_t& ex = srv->exec[slot];
        if (!rc && ex) {
            cudaGraphExecUpdateResultInfo info{};
            if (cudaGraphExecUpdate(ex, g, &info) == cudaSuccess) {
                std::lock_guard<std::mutex> lk(srv->mu);
                srv->stats.graph_updates++;
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(ex);
                ex = nullptr;
            }
        }
        if (!rc && !ex) {
            rc = rc_of(cudaGraphInstantiate(&ex, g, 0));
            if (!rc) {
                std::lock_guard<std::mutex> lk(srv->mu);
                srv->stats.graph_instantiations++;
            } else {
                ex = nullptr;
            }
        }
        if (g) cudaGraphDestroy(g);
    }
    return rc;
}

void scheduler_main(tti_server* srv)
{
    cudaSetDevice(srv->device);
    std::vector<Shot*> active;
    std::vector<Shot*> inflight_finishing;
    bool inflight = false;
    int slot = 0;
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(srv->mu);
            for (;;) {
                for (Shot* s : srv->ready) active.push_back(s);
                srv->ready.clear();
                bool work = false;
                for (Shot* s : active) work = work || s->planned_left > 0;
                if (work || inflight) break;
                if (srv->stop && srv->queue.empty() && srv->resident == (int)active.size()) {
                    lk.unlock();
                    for (Shot* s : active) finish_shot(srv, s, TTI_OK);  // nothing left to run
                    return;
                }
                srv->cv.wait_for(lk, std::chrono::milliseconds(20));
            }
        }
        // plan: units per shot for about round_ms of device time
        std::vector<std::pair<Shot*, int64_t>> plan;
        std::vector<Shot*> finishing;
        for (Shot* s : active) {
            if (s->planned_left <= 0) continue;
            int64_t u = (int64_t)std::floor(srv->cfg.round_ms / s->unit_ms);
            // whole imaging periods, so that consecutive rounds of a shot have
            // the same launch pattern and the captured graph can be updated in
            // place instead of instantiated again
            const int64_t period = std::max(1, s->req.xcorr_step);
            // a small grid's round would otherwise hold thousands of launches
            // whose capture and update cost host time the device waits for
            u = std::min<int64_t>(u, kMaxUnitsPerRound);
            if (u >= period) u -= u % period;
            u = std::max<int64_t>(1, std::min(u, s->planned_left));
            plan.push_back({s, u});
            s->planned_left -= u;
            if (s->planned_left == 0) finishing.push_back(s);
        }
        // issue round r+1 behind the round in flight, so the device never
        // waits for the host between rounds
        int rc = TTI_OK;
        if (!plan.empty()) {
            const double t_build = srv->now();
            rc = build_round(srv, plan, slot);
            if (!rc && srv->cfg.use_graphs) {
                cudaEventRecord(srv->round_start[slot], srv->main);
                rc = rc_of(cudaGraphLaunch(srv->exec[slot], srv->main));
            }
            if (!rc) rc = rc_of(cudaEventRecord(srv->round_end[slot], srv->main));
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->stats.build_ms += 1e3 * (srv->now() - t_build);
        }
        // then wait for the round in flight and retire what it finished,
        // while round r+1 runs
        if (inflight) {
            cudaEventSynchronize(srv->round_end[slot ^ 1]);
            float ms = 0;
            if (cudaEventElapsedTime(&ms, srv->round_start[slot ^ 1], srv->round_end[slot ^ 1]) == cudaSuccess) {
                std::lock_guard<std::mutex> lk(srv->mu);
                srv->stats.busy_ms += ms;
            }
            // device gap between that round and the one just issued behind it
            if (!plan.empty() && !rc && cudaEventSynchronize(srv->round_start[slot]) == cudaSuccess &&
                cudaEventElapsedTime(&ms, srv->round_end[slot ^ 1], srv->round_start[slot]) == cudaSuccess) {
                std::lock_guard<std::mutex> lk(srv->mu);
                srv->stats.gap_ms += std::max(0.0f, ms);
            }
            cudaGetLastError();
            for (Shot* s : inflight_finishing) {
                active.erase(std::find(active.begin(), active.end(), s));
                retire_later(srv, s, shot_end(s->sim));
            }
            inflight_finishing.clear();
            inflight = false;
        }
        if (plan.empty()) continue;
        if (rc) {
            // the round could not be issued: fail its shots once the device is idle
            cudaStreamSynchronize(srv->main);
            for (auto& pu : plan) {
                active.erase(std::find(active.begin(), active.end(), pu.first));
                cudaStreamSynchronize(shot_stream(pu.first->sim));
                finish_shot(srv, pu.first, rc);
            }
            continue;
        }
        {
            std::lock_guard<std::mutex> lk(srv->mu);
            srv->stats.rounds++;
            srv->stats.max_batched = std::max(srv->stats.max_batched, (int)plan.size());
        }
        inflight = true;
        inflight_finishing = finishing;
        slot ^= 1;
    }
}

} // namespace

extern "C" {

int tti_server_create(const tti_server_config* cfg, tti_server** out)
{
    if (!cfg || !out) return TTI_EINVAL;
    *out = nullptr;
    if (cfg->max_active < 1 || !(cfg->round_ms > 0) || cfg->hbm_budget < 0 || cfg->snap_precision < 0 ||
        cfg->snap_precision > 2 || cfg->scheme < 0 || cfg->scheme > 1)
        return TTI_EINVAL;
    tti_server* srv = new (std::nothrow) tti_server();
    if (!srv) return TTI_ENOMEM;
    srv->cfg = *cfg;
    srv->t0 = std::chrono::steady_clock::now();
    int rc = rc_of(cudaGetDevice(&srv->device));
    if (!rc && srv->cfg.hbm_budget == 0) {
        size_t fr = 0, tot = 0;
        rc = rc_of(cudaMemGetInfo(&fr, &tot));
        const int64_t reserve = 2LL << 30;
        srv->cfg.hbm_budget = (int64_t)fr > reserve ? (int64_t)fr - reserve : 0;
    }

    if (!rc) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = srv->device;
        if (cudaMemPoolCreate(&srv->pool, &props) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        } else {
            srv->pool = nullptr;  // the default pool then
        }
        cudaGetLastError();
    }
    // kernel attributes and error words before any capture
    if (!rc) rc = prepare_fused_kernels();
    if (!rc) rc = rc_of(cudaStreamCreateWithFlags(&srv->main, cudaStreamNonBlocking));
    if (!rc) rc = rc_of(cudaEventCreateWithFlags(&srv->fork, cudaEventDisableTiming));
    for (int k = 0; k < 2 && !rc; ++k) {
        rc = rc_of(cudaEventCreate(&srv->round_start[k]));
        if (!rc) rc = rc_of(cudaEventCreate(&srv->round_end[k]));
    }
    if (rc) {
        if (srv->pool) cudaMemPoolDestroy(srv->pool);
        if (srv->main) cudaStreamDestroy(srv->main);
        if (srv->fork) cudaEventDestroy(srv->fork);
        for (int k = 0; k < 2; ++k) {
            if (srv->round_start[k]) cudaEventDestroy(srv->round_start[k]);
            if (srv->round_end[k]) cudaEventDestroy(srv->round_end[k]);
        }
        delete srv;
        return rc;
    }
    srv->loader = std::thread(loader_main, srv);
    srv->scheduler = std::thread(scheduler_main, srv);
    srv->retirer = std::thread(retirer_main, srv);
    *out = srv;
    return TTI_OK;
}

int tti_server_submit(tti_server* srv, const tti_shot_request* req, int64_t* ticket)
{
    if (!srv || !req || !ticket) return TTI_EINVAL;
    const tti_shot_request& r = *req;
    if (r.nx < 1 || r.ny < 1 || r.nz < 1 || r.nt < 1 || r.xcorr_step < 1 || !r.vp || !r.wavelet ||
        (r.nrec > 0 && !r.rec_ixyz) || r.nrec < 0)
        return TTI_EINVAL;
    Shot* sh = new (std::nothrow) Shot();
    if (!sh) return TTI_ENOMEM;
    sh->req = r;
    int ckpt = 0;
    int64_t bytes = 0;
    int rc = choose_checkpoint(srv, r, srv->cfg.hbm_budget, &ckpt, &bytes);
    if (!rc && bytes > srv->cfg.hbm_budget) rc = TTI_ENOMEM;  // cannot fit even alone
    if (rc) {
        delete sh;
        return rc;
    }
    sh->res.footprint = bytes;
    sh->res.checkpoint_every = ckpt;
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stop) {
        delete sh;
        return TTI_ESTATE;
    }
    sh->ticket = srv->next_ticket++;
    sh->res.t_submit = srv->now();
    srv->queue.push_back(sh);
    *ticket = sh->ticket;
    srv->cv.notify_all();
    return TTI_OK;
}

int tti_server_wait(tti_server* srv, int64_t ticket, double timeout_s, tti_shot_result* out)
{
    if (!srv || !out) return TTI_EINVAL;
    std::unique_lock<std::mutex> lk(srv->mu);
    if (ticket < 1 || ticket >= srv->next_ticket) return TTI_EINVAL;
    auto ready = [&] { return srv->done.count(ticket) > 0; };
    if (timeout_s < 0)
        srv->cv.wait(lk, ready);
    else if (!srv->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
        return TTI_ETIMEOUT;
    Shot* sh = srv->done[ticket];
    srv->done.erase(ticket);
    *out = sh->res;
    delete sh;
    return TTI_OK;
}

int tti_server_stats_get(tti_server* srv, tti_server_stats* out)
{
    if (!srv || !out) return TTI_EINVAL;
    std::lock_guard<std::mutex> lk(srv->mu);
    *out = srv->stats;
    return TTI_OK;
}

double tti_server_now(tti_server* srv) { return srv ? srv->now() : -1.0; }

int tti_server_destroy(tti_server* srv)
{
    if (!srv) return TTI_EINVAL;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
        srv->cv.notify_all();
    }
    srv->loader.join();
    srv->scheduler.join();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->scheduler_done = true;
        srv->cv.notify_all();
    }
    srv->retirer.join();
    for (auto& kv : srv->done) delete kv.second;
    for (int k = 0; k < 2; ++k)
        if (srv->exec[k]) cudaGraphExecDestroy(srv->exec[k]);
    cudaStreamSynchronize(srv->main);
    cudaStreamDestroy(srv->main);
    cudaEventDestroy(srv->fork);
    for (int k = 0; k < 2; ++k) {
        cudaEventDestroy(srv->round_start[k]);
        cudaEventDestroy(srv->round_end[k]);
    }
    if (srv->pool) cudaMemPoolDestroy(srv->pool);  // every shot's memory has been freed
    cudaGetLastError();
    delete srv;
    return TTI_OK;
}

} // extern "C"
