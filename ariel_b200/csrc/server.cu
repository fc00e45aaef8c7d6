// server.cu -- a request server that steps many scenes together (continuous batching).
//
// Requests (a scene and a number of steps) arrive at any time from any thread.  Host threads
// seed each arriving scene's particles while the device steps the live ones (seeding is the
// host half of FlipSim::Init, src/sim/flip.cpp:42-77).  A single worker thread owns the
// device: between two batch steps it retires the scenes that have run all their steps
// (copying their particles out) and admits prepared scenes, oldest first, while the device
// bytes of the new packed layout plus the persistent state of the old one fit the budget.
// Each membership change re-packs the live scenes into one particle / cell / face index
// space; scenes that stay are carried over by device copies of their persistent state
// (particles, pressure warm start, solid bins, frame counter), so their results do not depend
// on which other scenes share the launches.  Every stage of a batch step is one launch over
// all live scenes, replayed from a CUDA graph.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "sim.cuh"

using namespace ariel;
using namespace ariel::hostimpl;

namespace {

struct Request {
    int64_t id = 0;
    AsimSceneDesc desc{};
    int32_t nsteps = 0;
    int32_t state = ARIEL_REQ_QUEUED;
    ariel_status status = ARIEL_OK;
    int32_t steps_done = 0;  // steps queued on the device
    HostParticles hp;
    DeviceParticles dev;       // the same particles uploaded ahead of admission, when they fit
    long long staged_bytes = 0;
    long long np = 0, ns = 0, bytes = 0;
    double t_submit = -1, t_admit = -1, t_done = -1;
    std::vector<float> pos, vel;
    AsimStats stats{};
};

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double r = q * (double)(v.size() - 1);
    size_t lo = (size_t)r;
    size_t hi = std::min(lo + 1, v.size() - 1);
    double f = r - (double)lo;
    return v[lo] * (1.0 - f) + v[hi] * f;
}

}  // namespace

struct ariel_server {
    AsimParams prm{};
    AsimServerConfig cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    std::chrono::steady_clock::time_point t0;

    std::mutex mu;
    std::condition_variable cv_work;  // worker: ready requests or stop
    std::condition_variable cv_prep;  // preparers: queued requests or stop
    std::condition_variable cv_done;  // waiters: a request finished
    bool stopping = false;
    int64_t next_id = 1;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    std::deque<Request*> to_prepare;
    int preparing = 0;                  // being seeded by a host thread
    long long staged_total = 0;         // device bytes of uploaded, not yet admitted scenes
    std::map<int64_t, Request*> ready;  // prepared, waiting for device memory, oldest first
    std::vector<Request*> live;         // batch order
    ariel_sim* batch = nullptr;         // worker thread only

    // statistics (under mu)
    std::vector<double> step_ms;
    std::vector<double> latency_ms;
    int64_t batch_steps = 0, particle_steps = 0, submitted = 0, admitted = 0, finished = 0, failed = 0;
    int64_t relayouts = 0;
    double relayout_ms = 0, busy_ms = 0, relayout_wait_ms = 0, relayout_build_ms = 0, graph_build_ms = 0;
    int64_t staged = 0;
    long long in_use = 0, peak = 0;
    int max_live_seen = 0;
    ariel_status last_error = ARIEL_OK;

    std::thread worker;
    std::vector<std::thread> preparers;

    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

namespace {

long long bufs_bytes(const ariel_sim* s, bool keep_only) {
    long long b = 0;
    for (const auto& d : s->bufs)
        if (!keep_only || d.keep) b += (long long)d.bytes;
    return b;
}

void free_staged(ariel_server* S, Request* r, cudaStream_t st) {
    DeviceParticles& g = r->dev;
    if (!g.valid) return;
    for (void* p : {(void*)g.pos4, (void*)g.vel4, (void*)g.solid_pos, (void*)g.solid_start})
        if (p) cudaFreeAsync(p, st);
    g = DeviceParticles{};
    std::lock_guard<std::mutex> lk(S->mu);
    S->staged_total -= r->staged_bytes;
    r->staged_bytes = 0;
}

// Uploads a seeded scene into pool memory on the seeding thread's stream, so that admitting it
// later costs device copies only.  Returns false (and uploads nothing) when it does not fit.
bool stage(ariel_server* S, Request* r, cudaStream_t st) {
    const HostParticles& hp = r->hp;
    const long long n3 = (long long)r->desc.dim * r->desc.dim * r->desc.dim;
    const long long bytes = 32 * r->np + 16 * r->ns + (hp.solid_start.empty() ? 0 : 4 * (n3 + 1));
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->in_use + S->staged_total + bytes > S->cfg.hbm_budget_bytes) return false;
        S->staged_total += bytes;
        r->staged_bytes = bytes;
    }
    DeviceParticles g;
    g.np = r->np;
    g.ns = r->ns;
    bool ok = true;
    auto alloc = [&](void** p, size_t b) {
        if (ok && cudaMallocFromPoolAsync(p, b ? b : 16, S->pool, st) != cudaSuccess) ok = false;
    };
    alloc((void**)&g.pos4, 16 * (size_t)r->np);
    alloc((void**)&g.vel4, 16 * (size_t)r->np);
    if (r->ns > 0) alloc((void**)&g.solid_pos, 16 * (size_t)r->ns);
    if (!hp.solid_start.empty()) alloc((void**)&g.solid_start, 4 * hp.solid_start.size());
    if (ok && r->np > 0) {
        ok = cudaMemcpyAsync(g.pos4, hp.pos4.data(), 16 * (size_t)r->np, cudaMemcpyHostToDevice, st) == cudaSuccess &&
             cudaMemcpyAsync(g.vel4, hp.vel4.data(), 16 * (size_t)r->np, cudaMemcpyHostToDevice, st) == cudaSuccess;
    }
    if (ok && r->ns > 0)
        ok = cudaMemcpyAsync(g.solid_pos, hp.solid_pos.data(), 16 * (size_t)r->ns, cudaMemcpyHostToDevice, st) ==
             cudaSuccess;
    if (ok && g.solid_start)
        ok = cudaMemcpyAsync(g.solid_start, hp.solid_start.data(), 4 * hp.solid_start.size(), cudaMemcpyHostToDevice,
                             st) == cudaSuccess;
    if (cudaStreamSynchronize(st) != cudaSuccess) ok = false;
    g.valid = true;  // so that free_staged releases whatever was allocated
    r->dev = g;
    if (!ok) {
        cudaGetLastError();
        free_staged(S, r, st);
        cudaStreamSynchronize(st);
        return false;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->staged++;
    return true;
}

void prepare_main(ariel_server* S) {
    cudaSetDevice(S->device);
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            // at most max_ready scenes seeded ahead of admission (host and device memory)
            S->cv_prep.wait(lk, [&] {
                return S->stopping ||
                       (!S->to_prepare.empty() && (int)S->ready.size() + S->preparing < S->cfg.max_ready);
            });
            if (S->stopping) break;
            r = S->to_prepare.front();
            S->to_prepare.pop_front();
            S->preparing++;
        }
        HostParticles hp;
        NvtxRange range("server_seed");
        generate_particles(r->desc, hp);
        const long long np = (long long)hp.pos4.size(), ns = (long long)hp.solid_pos.size();
        const long long bytes = state_bytes({r->desc}, {np}, {ns}, S->prm);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            r->np = np;
            r->ns = ns;
            r->bytes = bytes;
            r->hp = std::move(hp);
        }
        const bool fits = bytes <= S->cfg.hbm_budget_bytes;
        // the host copy is kept until admission, so an upload can always be dropped again
        if (fits) stage(S, r, st);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->preparing--;
            if (!fits) {
                // can never fit, even alone
                r->state = ARIEL_REQ_FAILED;
                r->status = ARIEL_ERR_OOM;
                r->t_done = S->now_ms();
                r->hp = HostParticles{};
                S->failed++;
                S->cv_done.notify_all();
                continue;
            }
            r->state = ARIEL_REQ_READY;
            S->ready.emplace(r->id, r);
        }
        S->cv_work.notify_one();
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
}

// Moves the worker's step-time history into the server statistics.
void drain_step_times(ariel_server* S) {
    if (!S->batch) return;
    std::lock_guard<std::mutex> lk(S->mu);
    for (double t : S->batch->step_hist) {
        S->step_ms.push_back(t);
        S->busy_ms += t;
    }
    S->batch->step_hist.clear();
}

void fail_live(ariel_server* S, ariel_status st) {
    std::lock_guard<std::mutex> lk(S->mu);
    for (Request* r : S->live) {
        r->state = ARIEL_REQ_FAILED;
        r->status = st;
        r->t_done = S->now_ms();
        S->failed++;
    }
    S->live.clear();
    S->last_error = st;
    S->cv_done.notify_all();
}

// Copies out the finished scenes, then packs `keep` (a subset of live, in live order) and
// `add` into a new batch.  Called by the worker with no step in flight.
ariel_status relayout(ariel_server* S, const std::vector<Request*>& retire, const std::vector<Request*>& keep,
                      std::vector<Request*>& add) {
    NvtxRange range("server_repack");
    const double t_begin = S->now_ms();
    ariel_sim* old = S->batch;
    if (old) {
        if (cudaStreamSynchronize(S->stream) != cudaSuccess) return map_cuda_error(cudaGetLastError(), "batch step");
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->relayout_wait_ms += S->now_ms() - t_begin;
        }
        ariel_status st = collect_pending(old);
        if (st != ARIEL_OK) return st;
        drain_step_times(S);
        st = check_device_error(old);
        if (st != ARIEL_OK) return st;
        st = refresh_scene_table(old);
        if (st != ARIEL_OK) return st;
    }
    auto index_in_live = [&](Request* r) {
        for (size_t j = 0; j < S->live.size(); ++j)
            if (S->live[j] == r) return (int)j;
        return -1;
    };
    for (Request* r : retire) {
        const int j = index_in_live(r);
        AsimStats stats{};
        ariel_status st = ariel_stats(old, j, &stats);
        std::vector<float> pos, vel;
        if (st == ARIEL_OK && S->cfg.keep_results) {
            pos.resize(3 * (size_t)r->np);
            vel.resize(3 * (size_t)r->np);
            st = ariel_download_state(old, j, pos.data(), vel.data());
        }
        std::lock_guard<std::mutex> lk(S->mu);
        r->stats = stats;
        r->t_done = S->now_ms();
        if (st == ARIEL_OK) {
            r->pos.swap(pos);
            r->vel.swap(vel);
            r->state = ARIEL_REQ_DONE;
            S->finished++;
            S->latency_ms.push_back(r->t_done - r->t_submit);
        } else {
            r->state = ARIEL_REQ_FAILED;
            r->status = st;
            S->failed++;
        }
    }
    if (!retire.empty()) S->cv_done.notify_all();

    const int k = (int)(keep.size() + add.size());
    std::vector<DeviceParticles> staged(k);
    for (size_t a = 0; a < add.size(); ++a) staged[keep.size() + a] = add[a]->dev;
    std::vector<AsimSceneDesc> descs;
    std::vector<SceneDev> sh;
    std::vector<int64_t> frames;
    std::vector<int> src_idx;
    for (Request* r : keep) {
        const int j = index_in_live(r);
        descs.push_back(old->descs[j]);
        sh.push_back(old->sh[j]);
        frames.push_back(old->frames[j]);
        src_idx.push_back(j);
    }
    for (Request* r : add) {
        descs.push_back(r->desc);
        sh.push_back(make_scene(r->desc, S->prm));
        frames.push_back(0);
        src_idx.push_back(-1);
    }
    ariel_sim* s2 = nullptr;
    if (k > 0) {
        ariel_status st = new_sim(descs.data(), k, S->prm, S->stream, S->pool, &s2);
        if (st != ARIEL_OK) return st;
        s2->sh = sh;
        s2->frames = frames;
        if (old) free_scratch(old);
        std::vector<HostParticles> hp(k);
        for (size_t a = 0; a < add.size(); ++a) hp[keep.size() + a] = std::move(add[a]->hp);
        const double tb = S->now_ms();
        st = build_state(s2, hp, old, &src_idx, &staged);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->relayout_build_ms += S->now_ms() - tb;
        }
        if (st == ARIEL_OK) st = compute_max_density(s2);
        if (st == ARIEL_OK) st = sort_and_classify_init(s2);
        if (st == ARIEL_OK && cudaStreamSynchronize(S->stream) != cudaSuccess) st = map_cuda_error(cudaGetLastError());
        if (st != ARIEL_OK) {
            delete_sim(s2);
            return st;
        }
        s2->inited = true;
    }
    if (old) delete_sim(old);
    for (Request* r : add) {
        free_staged(S, r, S->stream);  // copied into the batch
        r->hp = HostParticles{};
    }
    S->batch = s2;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->live = keep;
        const double t = S->now_ms();
        for (Request* r : add) {
            r->state = ARIEL_REQ_RUNNING;
            r->t_admit = t;
            S->live.push_back(r);
            S->admitted++;
        }
        S->in_use = s2 ? bufs_bytes(s2, false) : 0;
        S->peak = std::max(S->peak, S->in_use);
        S->max_live_seen = std::max(S->max_live_seen, (int)S->live.size());
        S->relayouts++;
        S->relayout_ms += t - t_begin;
    }
    return ARIEL_OK;
}

void worker_main(ariel_server* S) {
    cudaSetDevice(S->device);
    for (;;) {
        std::vector<Request*> retire, keep, add;
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stopping || !S->live.empty() || !S->ready.empty(); });
            if (S->stopping) break;
            for (Request* r : S->live) (r->steps_done >= r->nsteps ? retire : keep).push_back(r);
            // admission, oldest first, while the new layout fits next to the old persistent state
            // and the scenes uploaded ahead
            const long long old_keep = (S->batch ? bufs_bytes(S->batch, true) : 0) + S->staged_total;
            std::vector<AsimSceneDesc> d;
            std::vector<long long> np, ns;
            for (Request* r : keep) {
                d.push_back(r->desc);
                np.push_back(r->np);
                ns.push_back(r->ns);
            }
            for (auto it = S->ready.begin(); it != S->ready.end();) {
                Request* r = it->second;
                if ((int)(keep.size() + add.size()) >= S->cfg.max_live) break;
                d.push_back(r->desc);
                np.push_back(r->np);
                ns.push_back(r->ns);
                if (state_bytes(d, np, ns, S->prm) + old_keep > S->cfg.hbm_budget_bytes) break;
                add.push_back(r);
                it = S->ready.erase(it);
            }
        }
        if (!add.empty()) S->cv_prep.notify_all();  // room for more seeding ahead
        if (add.empty() && retire.empty() && keep.empty() && !S->batch) {
            // Nothing runs and the oldest waiting scene does not fit next to the scenes uploaded
            // ahead: drop those uploads (their host copies remain) so that it can be admitted.
            std::vector<Request*> unstage;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                if (!S->ready.empty() && S->staged_total > 0)
                    for (auto& kv : S->ready)
                        if (kv.second->dev.valid) unstage.push_back(kv.second);
            }
            for (Request* r : unstage) free_staged(S, r, S->stream);
            if (!unstage.empty()) {
                cudaStreamSynchronize(S->stream);
                continue;
            }
        }
        if (!retire.empty() || !add.empty()) {
            ariel_status st = relayout(S, retire, keep, add);
            if (st != ARIEL_OK) {
                // the requests being admitted fail with the live ones
                {
                    std::lock_guard<std::mutex> lk(S->mu);
                    for (Request* r : add) S->live.push_back(r);
                }
                fail_live(S, st);
                if (S->batch) {
                    delete_sim(S->batch);
                    S->batch = nullptr;
                }
                continue;
            }
        }
        if (!S->batch) continue;
        const double g0 = S->batch->graph_ms;
        ariel_status st = step_async(S->batch);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            S->graph_build_ms += S->batch->graph_ms - g0;
        }
        if (st != ARIEL_OK) {
            fail_live(S, st);
            delete_sim(S->batch);
            S->batch = nullptr;
            continue;
        }
        drain_step_times(S);
        {
            std::lock_guard<std::mutex> lk(S->mu);
            for (Request* r : S->live) r->steps_done++;
            S->batch_steps++;
            S->particle_steps += S->batch->np;
        }
    }
    // stopping: unfinished requests are cancelled
    if (S->batch) {
        cudaStreamSynchronize(S->stream);
        collect_pending(S->batch);
        drain_step_times(S);
        delete_sim(S->batch);
        S->batch = nullptr;
    }
}

}  // namespace

extern "C" {

void ariel_server_config_default(AsimServerConfig* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->hbm_budget_bytes = 0;
    c->max_live = 32;
    c->prepare_threads = 4;
    c->keep_results = 1;
}

ariel_status ariel_server_create(const AsimParams* params, const AsimServerConfig* config, ariel_server** out) {
    if (!params || !config || !out) return ARIEL_ERR_INVALID_ARG;
    *out = nullptr;
    if (params->precision < 0 || params->precision > 2 || params->precond < 0 || params->precond > 1 ||
        params->stop_rule < 0 || params->stop_rule > 1)
        return ARIEL_ERR_INVALID_ARG;
    if (config->hbm_budget_bytes < 0 || config->max_live < 0 || config->max_live > kMaxScenes ||
        config->prepare_threads < 0 || config->prepare_threads > 64)
        return ARIEL_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return ARIEL_ERR_NO_DEVICE;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return ARIEL_ERR_NO_DEVICE;
    std::unique_ptr<ariel_server> S(new (std::nothrow) ariel_server());
    if (!S) return ARIEL_ERR_OOM;
    S->prm = *params;
    S->prm.timing = 1;  // per-step device times for the latency percentiles
    S->cfg = *config;
    if (S->cfg.max_live == 0) S->cfg.max_live = 32;
    if (S->cfg.prepare_threads == 0) S->cfg.prepare_threads = 4;
    if (S->cfg.max_ready <= 0) S->cfg.max_ready = 8;
    S->device = dev;
    if (S->cfg.hbm_budget_bytes == 0) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return map_cuda_error(cudaGetLastError(), "cudaMemGetInfo");
        S->cfg.hbm_budget_bytes = (int64_t)((double)fr * 0.85);
    }
    if (cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking) != cudaSuccess)
        return map_cuda_error(cudaGetLastError(), "cudaStreamCreate");
    // A pool that keeps what it has reserved: re-layouts free and allocate without returning
    // memory to the driver in between.
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&S->pool, &props) != cudaSuccess) {
        ariel_status st = map_cuda_error(cudaGetLastError(), "cudaMemPoolCreate");
        cudaStreamDestroy(S->stream);
        return st;
    }
    uint64_t keep_all = ~0ull;
    cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
    if (S->cfg.reserve_budget) {
        // grow the pool to the whole budget once; it keeps the memory after the free
        void* p = nullptr;
        if (cudaMallocFromPoolAsync(&p, (size_t)S->cfg.hbm_budget_bytes, S->pool, S->stream) == cudaSuccess) {
            cudaFreeAsync(p, S->stream);
            cudaStreamSynchronize(S->stream);
        } else {
            cudaGetLastError();
        }
    }
    S->t0 = std::chrono::steady_clock::now();
    ariel_server* raw = S.release();
    for (int i = 0; i < raw->cfg.prepare_threads; ++i) raw->preparers.emplace_back(prepare_main, raw);
    raw->worker = std::thread(worker_main, raw);
    *out = raw;
    return ARIEL_OK;
}

ariel_status ariel_server_submit(ariel_server* S, const AsimSceneDesc* desc, int32_t nsteps, int64_t* id) {
    if (!S || !desc || nsteps < 0) return ARIEL_ERR_INVALID_ARG;
    ariel_status st = validate(*desc);
    if (st != ARIEL_OK) return st;
    std::unique_ptr<Request> r(new (std::nothrow) Request());
    if (!r) return ARIEL_ERR_OOM;
    r->desc = *desc;
    r->nsteps = nsteps;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        if (S->stopping) return ARIEL_ERR_STATE;
        r->id = S->next_id++;
        r->t_submit = S->now_ms();
        if (id) *id = r->id;
        S->to_prepare.push_back(r.get());
        S->reqs.emplace(r->id, std::move(r));
        S->submitted++;
    }
    S->cv_prep.notify_one();
    return ARIEL_OK;
}

ariel_status ariel_server_poll(ariel_server* S, int64_t id, AsimRequestInfo* info) {
    if (!S || !info) return ARIEL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return ARIEL_ERR_INVALID_ARG;
    const Request& r = *it->second;
    std::memset(info, 0, sizeof(*info));
    info->state = r.state;
    info->status = r.status;
    info->nsteps = r.nsteps;
    info->steps_done = std::min(r.steps_done, r.nsteps);
    info->n_particles = r.np;
    info->state_bytes = r.bytes;
    info->submit_ms = r.t_submit;
    info->admit_ms = r.t_admit;
    info->done_ms = r.t_done;
    info->stats = r.stats;
    return ARIEL_OK;
}

ariel_status ariel_server_wait(ariel_server* S, int64_t id, double timeout_ms) {
    if (!S) return ARIEL_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return ARIEL_ERR_INVALID_ARG;
    Request* r = it->second.get();
    auto finished = [&] { return r->state == ARIEL_REQ_DONE || r->state == ARIEL_REQ_FAILED; };
    if (!S->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), finished))
        return ARIEL_ERR_PENDING;
    return r->state == ARIEL_REQ_DONE ? ARIEL_OK : r->status;
}

ariel_status ariel_server_drain(ariel_server* S, double timeout_ms) {
    if (!S) return ARIEL_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(S->mu);
    auto all_done = [&] { return S->finished + S->failed == S->submitted; };
    if (!S->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), all_done))
        return ARIEL_ERR_PENDING;
    return ARIEL_OK;
}

ariel_status ariel_server_fetch(ariel_server* S, int64_t id, float* pos, float* vel) {
    if (!S || !pos || !vel) return ARIEL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return ARIEL_ERR_INVALID_ARG;
    const Request& r = *it->second;
    if (r.state == ARIEL_REQ_FAILED) return r.status;
    if (r.state != ARIEL_REQ_DONE) return ARIEL_ERR_PENDING;
    if (!S->cfg.keep_results || r.pos.size() != 3 * (size_t)r.np) return ARIEL_ERR_STATE;
    std::memcpy(pos, r.pos.data(), r.pos.size() * sizeof(float));
    std::memcpy(vel, r.vel.data(), r.vel.size() * sizeof(float));
    return ARIEL_OK;
}

ariel_status ariel_server_release(ariel_server* S, int64_t id) {
    if (!S) return ARIEL_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return ARIEL_ERR_INVALID_ARG;
    const int st = it->second->state;
    if (st != ARIEL_REQ_DONE && st != ARIEL_REQ_FAILED) return ARIEL_ERR_PENDING;
    S->reqs.erase(it);
    return ARIEL_OK;
}

ariel_status ariel_server_stats(ariel_server* S, AsimServerStats* out) {
    if (!S || !out) return ARIEL_ERR_INVALID_ARG;
    std::vector<double> steps, lat;
    std::memset(out, 0, sizeof(*out));
    {
        std::lock_guard<std::mutex> lk(S->mu);
        steps = S->step_ms;
        lat = S->latency_ms;
        out->submitted = S->submitted;
        out->admitted = S->admitted;
        out->finished = S->finished;
        out->failed = S->failed;
        out->live = (int64_t)S->live.size();
        out->waiting = (int64_t)(S->to_prepare.size() + S->ready.size());
        out->batch_steps = S->batch_steps;
        out->particle_steps = S->particle_steps;
        out->busy_ms = S->busy_ms;
        out->relayouts = S->relayouts;
        out->relayout_ms = S->relayout_ms;
        out->hbm_budget_bytes = S->cfg.hbm_budget_bytes;
        out->hbm_in_use_bytes = S->in_use;
        out->hbm_peak_bytes = S->peak;
        out->max_live_seen = S->max_live_seen;
        out->last_error = S->last_error;
        out->relayout_wait_ms = S->relayout_wait_ms;
        out->relayout_build_ms = S->relayout_build_ms;
        out->graph_build_ms = S->graph_build_ms;
        out->staged = S->staged;
        out->timed_steps = (int64_t)steps.size();
    }
    out->wall_ms = S->now_ms();
    out->step_ms_p50 = percentile(steps, 0.50);
    out->step_ms_p99 = percentile(steps, 0.99);
    out->step_ms_max = steps.empty() ? 0.0 : *std::max_element(steps.begin(), steps.end());
    out->latency_ms_p50 = percentile(lat, 0.50);
    out->latency_ms_p99 = percentile(lat, 0.99);
    return ARIEL_OK;
}

ariel_status ariel_server_shutdown(ariel_server* S) {
    if (!S) return ARIEL_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    S->cv_prep.notify_all();
    if (S->worker.joinable()) S->worker.join();
    for (auto& t : S->preparers)
        if (t.joinable()) t.join();
    for (auto& kv : S->reqs) free_staged(S, kv.second.get(), S->stream);
    cudaStreamSynchronize(S->stream);
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (auto& kv : S->reqs) {
            Request* r = kv.second.get();
            if (r->state != ARIEL_REQ_DONE && r->state != ARIEL_REQ_FAILED) {
                r->state = ARIEL_REQ_FAILED;
                r->status = ARIEL_ERR_STATE;
            }
        }
    }
    S->cv_done.notify_all();
    cudaMemPoolDestroy(S->pool);
    cudaStreamDestroy(S->stream);
    delete S;
    return ARIEL_OK;
}

ariel_status ariel_state_bytes(const AsimSceneDesc* descs, int32_t k, const AsimParams* params, int64_t* bytes) {
    if (!descs || !params || !bytes || k < 1 || k > kMaxScenes) return ARIEL_ERR_INVALID_ARG;
    std::vector<AsimSceneDesc> d(descs, descs + k);
    std::vector<long long> np(k), ns(k);
    for (int i = 0; i < k; ++i) {
        ariel_status st = validate(d[i]);
        if (st != ARIEL_OK) return st;
        HostParticles hp;
        generate_particles(d[i], hp);
        np[i] = (long long)hp.pos4.size();
        ns[i] = (long long)hp.solid_pos.size();
    }
    *bytes = state_bytes(d, np, ns, *params);
    return ARIEL_OK;
}

}  // extern "C"
