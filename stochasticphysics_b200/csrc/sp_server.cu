// sp_server.cu — continuous batching of ensemble simulations on one GPU.
//
// Requests arrive through sp_server_submit at any time.  A scheduler thread
// admits queued requests while their device footprint (state, Philox
// counters are implicit, FP64 sample buffers, parameters) fits the memory
// budget, keeps every admitted ensemble's state on the device between chunks,
// and advances all of them chunk by chunk: admitted ensembles are grouped by
// kernel key (problem, anisotropy, solver, precision, noise mode) and each
// group runs ONE batched launch per chunk over a shared work list of particle
// tiles (step_kernel reads the tile -> ensemble map), captured once per group
// membership as a CUDA graph.  A request joins an idle group of its key; when
// its key's group is mid-round it starts a second group of that key at once.
// Groups run on separate streams so different kernels overlap on the device,
// each at its own pace: a group's round replays
// its chunk graph a few times, and when it ends (an event the scheduler polls)
// the group's finished ensembles are read back and freed, queued requests join,
// and its next round starts while the other groups' rounds are still running.
// One group's next chunk thus fills the SMs another's draining chunk frees, and
// no group waits for a slower one at a round boundary.
//
// Every particle's arithmetic, noise stream and per-warp reduction order are
// independent of which other ensembles share the launch, so a request's
// result is bit-identical alone and in any mix.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "sp_runtime.h"

namespace sp {

void launch_bump_targets(const EnsDev* e, int n_ens, cudaStream_t s);

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    sp_ensemble_desc desc{};
    std::vector<double> arrays;  // deep copy of every per-particle array and injected dW
    sp_provider_desc provider{};  // deep copy of a device-side provider, if any
    std::vector<sp_particle_template> templates;
    std::unique_ptr<Ensemble> ens;
    int state = SP_REQUEST_QUEUED;
    bool cancel = false;
    sp_status error = SP_OK;
    std::string message;
    uint64_t bytes = 0;
    unsigned long long chunks_per_round = 1;
    bool in_round = false;  // launched in the current round (not admitted during it)
    Clock::time_point t_submit, t_admit0, t_admit1, t_run_end, t_done;
    std::vector<double> mean, weight, time, field, weighted_sum;
    sp_stats stats{};
};

struct Group {
    int key = -1;  // kernel key of its members
    const KernelSet* ks = nullptr;
    std::vector<Request*> members;
    EnsDev* d_ens = nullptr;
    TileDesc* d_tiles = nullptr;
    int ntiles = 0, max_slots = 2, block = 128;
    unsigned long long max_chunk = 1;
    unsigned long long chunks_per_round = 1;  // the largest of its members'
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaEvent_t round_end = nullptr;  // recorded after the group's current round
    bool dirty = true;
    bool running = false;              // a round is in flight on `stream`
    unsigned long long round_launches = 0;  // chunk launches of the round in flight

    void release() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        if (d_ens) cudaFreeAsync(d_ens, stream);  // the context's pool, in stream order
        if (d_tiles) cudaFreeAsync(d_tiles, stream);
        gexec = nullptr; graph = nullptr; d_ens = nullptr; d_tiles = nullptr;
    }
};

}  // namespace sp

using namespace sp;

struct sp_server {
    sp_context* ctx = nullptr;
    sp_server_config cfg{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    uint64_t next_id = 1;
    uint64_t used_bytes = 0, budget = 0;
    std::deque<Request*> queue;
    std::vector<Request*> active;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
    std::vector<std::unique_ptr<Group>> groups;  // several may share a kernel key

    static int key_of(const sp_ensemble_desc& d) {
        return (((d.problem * kAnisoSlots + d.anisotropy) * kSolverSlots + solver_slot(d.solver, d.jacobian)) * 2 + d.precision) * 2 +
               (d.noise == SP_NOISE_INJECTED);
    }

    // Requests join and leave a group only between its rounds (a new request whose key's
    // group is mid-round starts a second group of that key, group_for), so the round bounds how long a
    // request that finishes or is cancelled mid-round waits to be read back: cfg.chunk_steps
    // steps, or else the tuned (throughput) chunk capped at kServeChunk steps, in whole
    // windows.  A round runs as chunk launches of at most kSliceSteps (whole windows where a
    // window fits): each launch ends with its CTAs draining, and with several groups in flight the others'
    // next launches fill the SMs so freed (two 65536-particle Brown+Neel ensembles run
    // 15 % faster in 1000-step launches than in 10000-step ones).
    static constexpr unsigned long long kServeChunk = 4000;
    static constexpr unsigned long long kSliceSteps = 1000;
    static unsigned long long whole_windows(unsigned long long steps, unsigned long long W) {
        return steps <= W ? W : steps / W * W;
    }
    LaunchConfig launch_for(const sp_ensemble_desc& d, unsigned long long* chunks_per_round = nullptr) const {
        LaunchConfig c = launch_config_for(ctx, d);
        const unsigned long long W = std::max<unsigned long long>(d.oversampling, 1);
        // no longer than the run itself, (K - 1) W steps: a configured round of 1e9 steps
        // would otherwise become 1e6 launches of which all but the first few do nothing
        // (K >= 1 is clamped here so an unvalidated description cannot underflow K - 1)
        const unsigned long long S = (std::max<unsigned long long>(d.number_of_steps / W, 1) - 1) * W;
        const unsigned long long round =
            std::min(cfg.chunk_steps ? cfg.chunk_steps : std::min(c.chunk, whole_windows(kServeChunk, W)),
                     std::max<unsigned long long>(S, 1));
        c.chunk = round <= kSliceSteps ? round : std::min(round, whole_windows(kSliceSteps, W));
        if (chunks_per_round) *chunks_per_round = std::max<unsigned long long>(1, round / c.chunk);
        return c;
    }

    void finish(Request* r, int state, sp_status err, const std::string& msg) {
        r->state = state;
        r->error = err;
        r->message = msg;
        r->t_done = Clock::now();
    }

    void retire(Request* r) {
        if (r->ens) {
            sp_result out{};
            r->mean.assign(r->ens->L.K * r->ens->L.OUT, 0.0);
            r->weight.assign(r->ens->L.OUT, 0.0);
            r->time.assign(r->ens->L.K, 0.0);
            r->field.assign(r->ens->L.K * 3, 0.0);
            r->weighted_sum.assign(r->ens->L.K * r->ens->L.OUT, 0.0);
            out.weighted_sum = r->weighted_sum.data();
            out.mean = r->mean.data();
            out.weight = r->weight.data();
            out.time = r->time.data();
            out.field = r->field.data();
            r->ens->read(&out, &r->stats);
            r->ens.reset();
            const auto ms = [](Clock::time_point a, Clock::time_point b) {
                return std::chrono::duration<double, std::milli>(b - a).count();
            };
            const Clock::time_point now = Clock::now();
            r->stats.queue_ms = ms(r->t_submit, r->t_admit0);
            r->stats.setup_ms = ms(r->t_admit0, r->t_admit1);
            r->stats.run_ms = ms(r->t_admit1, r->t_run_end);
            r->stats.readback_ms = ms(r->t_run_end, now);
        }
    }

    // The group a newly admitted request of kernel key `key` joins: an idle group of that
    // key (its next round starts at once); else, while the key has fewer running groups
    // than the cap, a group of its own (an idle empty group or a new one), so a
    // request arriving while its key's group is mid-round starts at once instead of
    // waiting for that round to end; else the key's running group with the fewest members,
    // joining at its next round.  The cap (sp_server_config.groups_per_kind, default
    // kGroupsPerKey) keeps a burst of arrivals batched in few launches.
    static constexpr int kGroupsPerKey = 2;
    Group& group_for(int key) {
        Group* empty = nullptr;
        Group* least_full = nullptr;
        int of_key = 0;
        for (auto& gp : groups) {
            if (gp->key == key && !gp->members.empty()) {
                if (!gp->running) return *gp;
                ++of_key;
                if (!least_full || gp->members.size() < least_full->members.size()) least_full = gp.get();
            } else if (!gp->running && gp->members.empty() && (!empty || gp->key == key)) {
                empty = gp.get();
            }
        }
        if (of_key >= (cfg.groups_per_kind > 0 ? cfg.groups_per_kind : kGroupsPerKey)) return *least_full;
        if (!empty) {
            groups.push_back(std::make_unique<Group>());
            empty = groups.back().get();
        }
        empty->key = key;
        empty->dirty = true;
        return *empty;
    }

    void admit_locked() {
        while (!queue.empty()) {
            Request* r = queue.front();
            if (r->cancel) {
                queue.pop_front();
                finish(r, SP_REQUEST_CANCELLED, SP_ERR_CANCELLED, "cancelled while queued");
                cv_done.notify_all();
                continue;
            }
            if (cfg.max_active > 0 && static_cast<int>(active.size()) >= cfg.max_active) break;
            if (used_bytes + r->bytes > budget) break;
            queue.pop_front();
            try {
                r->t_admit0 = Clock::now();
                r->ens = std::make_unique<Ensemble>(ctx, r->desc, launch_for(r->desc, &r->chunks_per_round), false, false);
                r->t_admit1 = Clock::now();
                r->ens->last_stream = nullptr;
                // the ensemble holds its inputs on the device now: drop the host copies
                std::vector<double>().swap(r->arrays);
                r->desc.particles = sp_particles{};
                r->desc.injected_dw = nullptr;
                r->state = SP_REQUEST_RUNNING;
                used_bytes += r->bytes;
                active.push_back(r);
                Group& g = group_for(key_of(r->desc));
                g.members.push_back(r);
                g.dirty = true;
            } catch (const Error& e) {
                finish(r, SP_REQUEST_FAILED, e.status, e.what());
                cv_done.notify_all();
            }
        }
    }

    void rebuild(Group& g) {
        g.release();
        if (g.members.empty()) return;
        if (!g.stream) check_cuda(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "group stream");
        g.ks = g.members.front()->ens->ks;
        std::vector<EnsDev> ens;
        std::vector<TileDesc> tiles;
        g.max_slots = 2;
        g.max_chunk = 1;
        g.chunks_per_round = 1;
        g.block = 32;
        for (Request* r : g.members) g.block = std::max(g.block, r->ens->block);
        for (size_t i = 0; i < g.members.size(); ++i) {
            Ensemble* e = g.members[i]->ens.get();
            ens.push_back(e->hdev);
            g.max_slots = std::max(g.max_slots, e->L.slots);
            g.max_chunk = std::max(g.max_chunk, e->L.chunk);
            g.chunks_per_round = std::max(g.chunks_per_round, g.members[i]->chunks_per_round);
            for (unsigned long long f = 0; f < e->L.n; f += g.block) tiles.push_back(TileDesc{static_cast<unsigned>(i), static_cast<unsigned>(f)});
        }
        g.ntiles = static_cast<int>(tiles.size());
        check_cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&g.d_ens), ens.size() * sizeof(EnsDev), ctx->pool,
                                           g.stream), "cudaMallocFromPoolAsync");
        check_cuda(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&g.d_tiles), tiles.size() * sizeof(TileDesc),
                                           ctx->pool, g.stream), "cudaMallocFromPoolAsync");
        check_cuda(cudaMemcpyAsync(g.d_ens, ens.data(), ens.size() * sizeof(EnsDev), cudaMemcpyHostToDevice, g.stream), "copy");
        // from pageable memory: each copy has taken its bytes when the call returns, and the
        // group's launches follow them on g.stream
        check_cuda(cudaMemcpyAsync(g.d_tiles, tiles.data(), tiles.size() * sizeof(TileDesc), cudaMemcpyHostToDevice, g.stream), "copy");
        const int n = static_cast<int>(ens.size());
        const int midpoint = g.members.front()->desc.solver == SP_SOLVER_IMPLICIT_MIDPOINT ? 1 : 0;
        cudaStream_t cs;
        check_cuda(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "capture stream");
        check_cuda(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
        launch_bump_targets(g.d_ens, n, cs);
        g.ks->field(g.d_ens, n, g.max_chunk, midpoint, cs);
        // one launch shape for the group: its largest tile, and the particles per thread
        // the first member was configured with where that tile allows it
        const int ppt = usable_ppt(*g.ks, g.members.front()->ens->launch.ppt, g.block);
        g.ks->step[ppt - 1](g.d_ens, g.d_tiles, g.ntiles, g.ntiles, g.block, cs);
        g.ks->reduce(g.d_ens, n, g.max_slots, 0, cs);
        launch_commit(g.d_ens, n, cs);
        const cudaError_t ce = cudaStreamEndCapture(cs, &g.graph);
        cudaStreamDestroy(cs);
        check_cuda(ce, "end capture");
        check_cuda(cudaGraphInstantiate(&g.gexec, g.graph, 0), "instantiate");
        g.dirty = false;
    }

    // waits for every round in flight (stop, or an error that fails every request)
    void drain() {
        for (auto& gp : groups) {
            if (gp->running && gp->stream) cudaStreamSynchronize(gp->stream);
            gp->running = false;
        }
    }

    // Polls until a running group ends its round (appended to `ended`), an idle group has
    // members to start, or the server stops; queued requests are admitted (uploaded) while
    // the rounds run.
    void wait_round(std::vector<Group*>& ended) {
        for (;;) {
            for (auto& gp : groups) {
                Group& g = *gp;
                if (!g.running) continue;
                const cudaError_t q = cudaEventQuery(g.round_end);
                if (q == cudaSuccess) ended.push_back(&g);
                else if (q != cudaErrorNotReady) check_cuda(q, "round");
            }
            if (!ended.empty()) return;
            {
                std::lock_guard<std::mutex> lk(mu);
                admit_locked();
                if (stop) return;
                for (const auto& gp : groups)
                    if (!gp->running && !gp->members.empty()) return;
            }
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }

    void run() {
        check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    admit_locked();
                    if (stop) {
                        drain();
                        return;
                    }
                    if (!active.empty()) break;
                    cv_work.wait(lk);
                }
            }
            std::vector<Group*> ended;
            try {
                // a round for every idle group with members: its chunk graph chunks_per_round
                // times on its own stream.  Groups that start together go longest first
                // (particle-steps of the round over the key's tuned rate; particle-steps alone
                // while any key is untuned), so the others' CTAs fill the SMs it leaves free
                // instead of it running alone at the end.
                std::vector<std::pair<double, Group*>> order;
                bool all_tuned = true;
                for (const auto& gp : groups)
                    if (!gp->running && !gp->members.empty() && tuned_rate(gp->members.front()->desc) <= 0.0)
                        all_tuned = false;
                for (auto& gp : groups) {
                    Group& g = *gp;
                    if (g.running || g.members.empty()) continue;
                    if (g.dirty) rebuild(g);
                    double work = 0.0;
                    for (Request* r : g.members) {
                        const Ensemble* e = r->ens.get();
                        work += static_cast<double>(e->L.n) *
                                static_cast<double>(std::min(g.chunks_per_round * e->L.chunk, e->L.S - e->steps_done));
                    }
                    order.emplace_back(all_tuned ? work / tuned_rate(g.members.front()->desc) : work, &g);
                }
                std::stable_sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
                unsigned long long launches = 0;
                for (auto& og : order) launches = std::max(launches, og.second->chunks_per_round);
                for (auto& og : order) {
                    Group& g = *og.second;
                    for (Request* r : g.members) r->in_round = true;
                    if (!g.round_end)
                        check_cuda(cudaEventCreateWithFlags(&g.round_end, cudaEventDisableTiming), "round event");
                    g.round_launches = g.chunks_per_round;
                    g.running = true;
                }
                for (unsigned long long j = 0; j < launches; ++j)
                    for (auto& og : order) {
                        Group& g = *og.second;
                        if (j >= g.chunks_per_round) continue;
                        check_cuda(cudaGraphLaunch(g.gexec, g.stream), "graph launch");
                        g_launch_count += 5;
                    }
                for (auto& og : order) check_cuda(cudaEventRecord(og.second->round_end, og.second->stream), "round event");
                wait_round(ended);
            } catch (const Error& e) {
                std::lock_guard<std::mutex> lk(mu);
                drain();
                for (Request* r : active) { r->ens.reset(); finish(r, SP_REQUEST_FAILED, e.status, e.what()); }
                active.clear();
                used_bytes = 0;
                for (auto& gp : groups) { gp->members.clear(); gp->release(); }
                cv_done.notify_all();
                continue;
            }
            // host mirror of the device counters of the groups whose round ended; retire
            // their finished or cancelled ensembles
            std::lock_guard<std::mutex> lk(mu);
            for (Group* g : ended) {
                g->running = false;
                const std::vector<Request*> members = g->members;  // retiring edits g->members
                for (Request* r : members) {
                    if (!r->in_round) continue;  // admitted during the round: joins the next one
                    r->in_round = false;
                    Ensemble* e = r->ens.get();
                    // each launch advances the ensemble by min(chunk, steps left) (bump, commit)
                    const unsigned long long nl = g->round_launches;
                    const unsigned long long step = std::min(nl * e->L.chunk, e->L.S - e->steps_done);
                    e->steps_done += step;
                    e->particle_steps += step * e->L.n;
                    e->launches += 5 * nl;
                    const bool done = e->steps_done >= e->L.S;
                    if (!done && !r->cancel) continue;
                    r->t_run_end = Clock::now();
                    try {
                        if (done) retire(r);
                        else r->ens.reset();
                        finish(r, done ? SP_REQUEST_DONE : SP_REQUEST_CANCELLED, done ? SP_OK : SP_ERR_CANCELLED,
                               done ? "" : "cancelled while running");
                    } catch (const Error& ex) {
                        r->ens.reset();
                        finish(r, SP_REQUEST_FAILED, ex.status, ex.what());
                    }
                    used_bytes -= r->bytes;
                    g->members.erase(std::find(g->members.begin(), g->members.end(), r));
                    g->dirty = true;
                    active.erase(std::find(active.begin(), active.end(), r));
                }
            }
            cv_done.notify_all();
        }
    }
};

namespace sp {
void copy_desc_arrays(const sp_ensemble_desc& in, Request& r) {
    const size_t n = in.n_particles;
    const bool brown = in.problem == SP_PROBLEM_BROWN_AND_NEEL || in.problem == SP_PROBLEM_BROWN_AND_NEEL_EULER_SPHERICAL;
    const int M = noise_dim(in.problem);
    const unsigned long long K = in.number_of_steps / in.oversampling;
    const size_t ndw = in.noise == SP_NOISE_INJECTED ? (K - 1) * in.oversampling * M * n : 0;
    const bool uc = in.anisotropy == SP_ANISOTROPY_UNIAXIAL_CUBIC;
    if (in.provider) {  // particles are drawn on the device: no arrays to keep
        r.desc = in;
        r.desc.particles = sp_particles{};
        r.desc.injected_dw = nullptr;
        r.provider = *in.provider;
        r.templates.assign(in.provider->templates, in.provider->templates + in.provider->n_templates);
        r.provider.templates = r.templates.data();
        r.desc.provider = &r.provider;
        return;
    }
    r.arrays.assign(n * (5 + (brown ? 2 : 0) + 6 + (uc ? 4 : 0)) + ndw, 0.0);
    double* p = r.arrays.data();
    auto put = [&](const double* src, size_t count) -> const double* {
        std::memcpy(p, src, count * 8);
        const double* at = p;
        p += count;
        return at;
    };
    r.desc = in;
    sp_particles& q = r.desc.particles;
    q.magnetic_radius = put(in.particles.magnetic_radius, n);
    q.saturation_magnetisation = put(in.particles.saturation_magnetisation, n);
    q.damping_constant = put(in.particles.damping_constant, n);
    q.gyromagnetic_ratio = put(in.particles.gyromagnetic_ratio, n);
    q.anisotropy_constant = put(in.particles.anisotropy_constant, n);
    if (brown) {
        q.hydrodynamic_radius = put(in.particles.hydrodynamic_radius, n);
        q.viscosity = put(in.particles.viscosity, n);
    } else {
        q.hydrodynamic_radius = nullptr;
        q.viscosity = nullptr;
    }
    q.orientation = put(in.particles.orientation, 3 * n);
    q.magnetisation = put(in.particles.magnetisation, 3 * n);
    q.cubic_constant = uc ? put(in.particles.cubic_constant, n) : nullptr;
    q.uniaxial_rotation = uc ? put(in.particles.uniaxial_rotation, 3 * n) : nullptr;
    r.desc.injected_dw = ndw ? put(in.injected_dw, ndw) : nullptr;
}
}  // namespace sp


extern "C" {

sp_status sp_server_create(sp_context* ctx, const sp_server_config* cfg, sp_server** out) {
    SP_GUARD_BEGIN
    if (!ctx || !out) return fail(SP_ERR_INVALID_ARG, "NULL argument");
    if (cfg && cfg->groups_per_kind < 0) return fail(SP_ERR_INVALID_ARG, "groups_per_kind must be >= 0");
    auto* s = new sp_server();
    s->ctx = ctx;
    if (cfg) s->cfg = *cfg;
    size_t free_b = 0, total_b = 0;
    check_cuda(cudaSetDevice(ctx->device), "cudaSetDevice");
    check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const uint64_t cap = static_cast<uint64_t>(0.9 * static_cast<double>(free_b));
    s->budget = s->cfg.memory_budget_bytes ? std::min<uint64_t>(s->cfg.memory_budget_bytes, cap) : cap;
    s->worker = std::thread([s] {
        try {
            s->run();
        } catch (...) {
        }
    });
    *out = s;
    return SP_OK;
    SP_GUARD_END
}

namespace {
// Validated deep copy of one description with its device footprint, or the refusal.
sp_status make_request(sp_server* s, const sp_ensemble_desc* desc, std::unique_ptr<Request>& out, std::string& why) {
    const sp_status st = validate_desc(desc, why);
    if (st != SP_OK) return st;
    auto r = std::make_unique<Request>();
    copy_desc_arrays(*desc, *r);
    r->bytes = layout_of(r->desc, s->launch_for(r->desc)).bytes;
    if (r->bytes > s->budget) {
        why = "request needs " + std::to_string(r->bytes) + " bytes; budget is " + std::to_string(s->budget);
        return SP_ERR_ADMISSION_REFUSED;
    }
    out = std::move(r);
    return SP_OK;
}
}  // namespace

sp_status sp_server_submit(sp_server* s, const sp_ensemble_desc* desc, uint64_t* id) {
    SP_GUARD_BEGIN
    if (!s || !id) return fail(SP_ERR_INVALID_ARG, "NULL argument");
    std::unique_ptr<Request> r;
    std::string why;
    const sp_status st = make_request(s, desc, r, why);
    if (st != SP_OK) return fail(st, why);
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    *id = r->id;
    s->queue.push_back(r.get());
    s->all[r->id] = std::move(r);
    s->cv_work.notify_one();
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_server_submit_many(sp_server* s, const sp_ensemble_desc* descs, int32_t n, uint64_t* ids) {
    SP_GUARD_BEGIN
    if (!s || !descs || !ids) return fail(SP_ERR_INVALID_ARG, "NULL argument");
    if (n < 1) return fail(SP_ERR_INVALID_ARG, "n must be >= 1");
    std::vector<std::unique_ptr<Request>> rs(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i) {
        std::string why;
        const sp_status st = make_request(s, &descs[i], rs[static_cast<size_t>(i)], why);
        if (st != SP_OK) return fail(st, "request " + std::to_string(i) + ": " + why);
    }
    const auto now = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    for (int32_t i = 0; i < n; ++i) {
        std::unique_ptr<Request>& r = rs[static_cast<size_t>(i)];
        r->t_submit = now;
        r->id = s->next_id++;
        ids[i] = r->id;
        s->queue.push_back(r.get());
        s->all[r->id] = std::move(r);
    }
    s->cv_work.notify_one();
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_server_poll(sp_server* s, uint64_t id, int32_t* state) {
    if (!s) return fail(SP_ERR_INVALID_ARG, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(SP_ERR_NOT_FOUND, "unknown request id");
    if (state) *state = it->second->state;
    return SP_OK;
}

sp_status sp_server_wait(sp_server* s, uint64_t id, double timeout_ms, sp_result* out, sp_stats* stats,
                         double* latency_ms) {
    SP_GUARD_BEGIN
    if (!s) return fail(SP_ERR_INVALID_ARG, "NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(SP_ERR_NOT_FOUND, "unknown request id");
    Request* r = it->second.get();
    auto terminal = [r] { return r->state >= SP_REQUEST_DONE; };
    if (timeout_ms < 0) s->cv_done.wait(lk, terminal);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), terminal))
        return fail(SP_ERR_NOT_READY, "request still running");
    if (r->state != SP_REQUEST_DONE) {
        const sp_status err = r->error;
        const std::string msg = r->message;
        s->all.erase(it);  // a failed or cancelled request is reported once
        return fail(err, msg);
    }
    if (out) {
        if (out->mean) std::memcpy(out->mean, r->mean.data(), r->mean.size() * 8);
        if (out->weight) std::memcpy(out->weight, r->weight.data(), r->weight.size() * 8);
        if (out->time) std::memcpy(out->time, r->time.data(), r->time.size() * 8);
        if (out->field) std::memcpy(out->field, r->field.data(), r->field.size() * 8);
        if (out->weighted_sum) std::memcpy(out->weighted_sum, r->weighted_sum.data(), r->weighted_sum.size() * 8);
        if (out->trajectories || out->final_state)
            return fail(SP_ERR_INVALID_ARG, "the server returns ensemble results only");
    }
    if (stats) *stats = r->stats;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    s->all.erase(it);  // results are handed over once; the id is forgotten
    return SP_OK;
    SP_GUARD_END
}

sp_status sp_server_cancel(sp_server* s, uint64_t id) {
    if (!s) return fail(SP_ERR_INVALID_ARG, "NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) return fail(SP_ERR_NOT_FOUND, "unknown request id");
    it->second->cancel = true;
    s->cv_work.notify_one();
    return SP_OK;
}

sp_status sp_server_destroy(sp_server* s) {
    SP_GUARD_BEGIN
    if (!s) return SP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    for (Request* r : s->active) r->ens.reset();
    for (auto& gp : s->groups) {
        gp->release();
        if (gp->round_end) cudaEventDestroy(gp->round_end);
        if (gp->stream) cudaStreamDestroy(gp->stream);
    }
    delete s;
    return SP_OK;
    SP_GUARD_END
}

}  // extern "C"
