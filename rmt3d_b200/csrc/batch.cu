// Batched form: many independent scenes stepped together.
//
// Every scene keeps its own device state and its own CUDA stream; a pool of
// host threads issues the scenes' steps so that the small kernels of many
// scenes overlap on the device (uneven grid sizes need no padding: each scene
// launches its own grids).  Scenes are assigned to threads by a greedy
// balance of cells.  An autotuner picks the multigrid schedule per grid size
// -- smoothing counts (v_down, v_up) and whether each solve runs as one
// thread-block-cluster launch or as per-phase launches -- by timing
// candidates on a probe scene.
#include <algorithm>
#include <array>
#include <cstdlib>
#include <atomic>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "host_common.h"
#include "rmt3d_gpu.h"

// knobs shared with scene.cu (defined there)
extern "C" int rmt3d_scene_set_schedule(rmt3d_scene *s, int v_down, int v_up, int coarse_pts);
extern "C" int rmt3d_scene_set_mg_launch(rmt3d_scene *s, int cluster);
extern "C" int rmt3d_scene_set_smoother(rmt3d_scene *s, int mode);
extern "C" int rmt3d_scene_set_coarse_cluster(rmt3d_scene *s, int pts);

struct rmt3d_batch {
    std::vector<rmt3d_scene *> scenes;
    std::vector<rmt3d_scene_desc> descs;
    std::vector<std::vector<int>> groups;  // scene indices per host thread
    std::vector<int> status;
    // grid shape, periodicity, precision and density form -> (v_down, v_up,
    // cluster launch, smoother mode)
    std::map<std::array<int, 8>, std::array<int, 6>> tuned;
    int nthreads = 1;
    // equally sized scenes stepped together: one graph per group, each
    // multigrid solve batched over the group's scenes
    std::vector<rmt3d::scene_group *> sg;
    std::vector<std::vector<int>> sg_members;
    bool sg_dirty = true;
    bool use_groups = true;
};

namespace {
// what a tuned schedule is keyed on: the scenes build_groups may put together
// share it (grid shape, periodicity, precision, density form)
std::array<int, 8> tune_key(const rmt3d_scene_desc &d) {
    return {d.sys_size[0], d.sys_size[1], d.sys_size[2], d.periodic[0], d.periodic[1], d.periodic[2],
            d.precision, d.var_den};
}

void drop_groups(rmt3d_batch *b) {
    for (auto *g : b->sg) rmt3d::group_destroy(g);
    b->sg.clear();
    b->sg_members.clear();
    b->sg_dirty = true;
}

// partition the scenes into groups that can share batched solves: same grid,
// periodicity, form and multigrid schedule
int build_groups(rmt3d_batch *b) {
    drop_groups(b);
    std::map<std::vector<double>, std::vector<int>> part;
    for (size_t i = 0; i < b->scenes.size(); i++) {
        const rmt3d_scene_desc &d = b->descs[i];
        int sch[5];
        rmt3d::scene_schedule(b->scenes[i], sch);
        std::vector<double> key = {(double)d.sys_size[0], (double)d.sys_size[1], (double)d.sys_size[2],
                                   (double)d.periodic[0], (double)d.periodic[1], (double)d.periodic[2],
                                   (double)d.precision, (double)d.var_den, (double)d.mg_exact, d.mixed_rtol,
                                   (double)sch[0], (double)sch[1], (double)sch[2], (double)sch[3], (double)sch[4]};
        part[key].push_back((int)i);
    }
    for (auto &kv : part) {
        std::vector<rmt3d_scene *> sc;
        for (int i : kv.second) sc.push_back(b->scenes[i]);
        rmt3d::scene_group *g = nullptr;
        int e = rmt3d::group_create(sc.data(), (int)sc.size(), &g);
        if (e) {
            drop_groups(b);
            return e;
        }
        b->sg.push_back(g);
        b->sg_members.push_back(kv.second);
    }
    b->sg_dirty = false;
    return 0;
}
}  // namespace

namespace {

long long cells(const rmt3d_scene_desc &d) { return (long long)d.sys_size[0] * d.sys_size[1] * d.sys_size[2]; }

// run fn(scene index) for every scene, each host thread over its group
template <typename F>
int for_all(rmt3d_batch *b, F fn) {
    std::vector<int> err(b->groups.size(), 0);
    std::vector<std::string> msg(b->groups.size());
    std::vector<std::thread> th;
    int dev = 0;
    cudaGetDevice(&dev);
    for (size_t t = 0; t < b->groups.size(); t++) {
        th.emplace_back([&, t]() {
            cudaSetDevice(dev);
            for (int i : b->groups[t]) {
                int e = fn(i);
                if (e && !err[t]) {
                    err[t] = e;
                    msg[t] = rmt3d_last_error();
                }
            }
        });
    }
    for (auto &x : th) x.join();
    for (size_t t = 0; t < err.size(); t++)
        if (err[t]) return rmt3d::fail(err[t], msg[t]);
    return RMT3D_OK;
}

}  // namespace

extern "C" int rmt3d_batch_create(const rmt3d_scene_desc *descs, int nscenes, int host_threads,
                                  rmt3d_batch **out) {
    if (!descs || !out || nscenes < 1) return rmt3d::fail(RMT3D_ERR_INVALID, "bad batch arguments");
    *out = nullptr;
    rmt3d_batch *b = new rmt3d_batch();
    b->descs.assign(descs, descs + nscenes);
    int dev = 0;
    cudaGetDevice(&dev);
    for (int i = 0; i < nscenes; i++) {
        rmt3d_scene *s = nullptr;
        int e = rmt3d_scene_create(&descs[i], nullptr, &s);
        if (e) {
            for (auto *x : b->scenes) rmt3d_scene_destroy(x);
            delete b;
            return e;
        }
        b->scenes.push_back(s);
    }
    b->status.assign(nscenes, 0);
    int nt = host_threads > 0 ? host_threads : (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, nscenes));
    b->nthreads = nt;
    b->groups.assign(nt, {});
    // greedy balance by cells, largest first
    std::vector<int> order(nscenes);
    for (int i = 0; i < nscenes; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int c) { return cells(descs[a]) > cells(descs[c]); });
    std::vector<long long> load(nt, 0);
    for (int i : order) {
        int t = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->groups[t].push_back(i);
        load[t] += cells(descs[i]);
    }
    *out = b;
    return RMT3D_OK;
}

extern "C" int rmt3d_batch_prepare(rmt3d_batch *b) {
    if (!b) return rmt3d::fail(RMT3D_ERR_INVALID, "null batch");
    drop_groups(b);
    return for_all(b, [&](int i) { return rmt3d_prepare(b->scenes[i]); });
}

// Each host thread queues all steps of its scenes (step-graph launches on
// the scenes' own streams) before waiting for any of them, so that every
// scene of the batch is in flight on the device at once.
extern "C" int rmt3d_batch_step(rmt3d_batch *b, int nsteps, int *status) {
    if (!b) return rmt3d::fail(RMT3D_ERR_INVALID, "null batch");
    {
        const char *e = getenv("RMT3D_GRAPH");
        if ((e && e[0] == '0') || (getenv("RMT3D_BATCH_GROUPS") && getenv("RMT3D_BATCH_GROUPS")[0] == '0'))
            b->use_groups = false;
    }
    if (b->use_groups) {
        if (b->sg_dirty) {
            int e = build_groups(b);
            if (e) return e;
        }
        int err = 0;
        std::string msg;
        for (auto *g : b->sg) {
            int e = rmt3d::group_launch(g, nsteps);
            if (e && !err) {
                err = e;
                msg = rmt3d_last_error();
            }
        }
        for (size_t k = 0; k < b->sg.size(); k++) {
            std::vector<int> st(b->sg_members[k].size(), 0);
            int e = rmt3d::group_finish(b->sg[k], st.data());
            if (e && !err) {
                err = e;
                msg = rmt3d_last_error();
            }
            for (size_t j = 0; j < st.size(); j++) b->status[b->sg_members[k][j]] = st[j];
        }
        if (status)
            for (size_t i = 0; i < b->status.size(); i++) status[i] = b->status[i];
        return err ? rmt3d::fail(err, msg) : RMT3D_OK;
    }
    std::vector<int> err(b->groups.size(), 0);
    std::vector<std::string> msg(b->groups.size());
    std::vector<std::thread> th;
    int dev = 0;
    cudaGetDevice(&dev);
    for (size_t t = 0; t < b->groups.size(); t++) {
        th.emplace_back([&, t]() {
            cudaSetDevice(dev);
            auto note = [&](int e) {
                if (e && !err[t]) {
                    err[t] = e;
                    msg[t] = rmt3d_last_error();
                }
            };
            for (int i : b->groups[t]) note(rmt3d::steps_launch(b->scenes[i], nsteps));
            for (int i : b->groups[t]) {
                int st = 0;
                note(rmt3d::steps_finish(b->scenes[i], &st));
                b->status[i] = st;
            }
        });
    }
    for (auto &x : th) x.join();
    if (status)
        for (size_t i = 0; i < b->status.size(); i++) status[i] = b->status[i];
    for (size_t t = 0; t < err.size(); t++)
        if (err[t]) return rmt3d::fail(err[t], msg[t]);
    return RMT3D_OK;
}

extern "C" int rmt3d_batch_size(rmt3d_batch *b, int *n) {
    if (!b || !n) return rmt3d::fail(RMT3D_ERR_INVALID, "null argument");
    *n = (int)b->scenes.size();
    return RMT3D_OK;
}

extern "C" int rmt3d_batch_scene(rmt3d_batch *b, int i, rmt3d_scene **out) {
    if (!b || !out || i < 0 || i >= (int)b->scenes.size()) return rmt3d::fail(RMT3D_ERR_INVALID, "bad scene index");
    *out = b->scenes[i];
    return RMT3D_OK;
}

// Autotune the multigrid schedule per kind of scene (grid shape,
// periodicity, precision and density form, the keys build_groups groups by):
// a probe copy of the first scene of each kind is set up, every candidate is
// stepped `probe_steps` times in each of three rounds, and the candidate with
// the least total time that ran without error is applied to every scene of
// that kind.  The candidates are
// the smoothing counts (v_down, v_up), each solve as one thread-block-cluster
// launch or as per-phase launches, and for the latter the smoother (one
// launch per colour pass, or one per whole sweep on shared-memory tiles) and
// the levels (none, up to 5000 or up to 40000 points) whose part of each
// V-cycle runs as one cluster launch.  With the fastest of those, the block
// shapes of the bulk stencil kernels are timed the same way
// (rmt3d_scene_set_block_shape).  tuned_out (optional, 7 ints per kind:
// cells, v_down, v_up, cluster launch, smoother, coarse cluster points,
// block shape) receives the choices.
extern "C" int rmt3d_batch_autotune(rmt3d_batch *b, int probe_steps, int *tuned_out, int max_out, int *n_out) {
    if (!b) return rmt3d::fail(RMT3D_ERR_INVALID, "null batch");
    if (probe_steps < 1) return rmt3d::fail(RMT3D_ERR_INVALID, "probe_steps < 1");
    drop_groups(b);
    static const int smooth[][2] = {{2, 2}, {1, 1}, {1, 2}, {2, 1}, {3, 3}};
    // (whole solve as one cluster launch, smoother: 0 colour passes, 1 tiled
    // sweeps, largest level of the coarse part run as one cluster launch)
    static const int launch[][3] = {{1, 0, 0}, {0, 0, 0}, {0, 1, 0}, {0, 0, 5000}, {0, 0, 40000}, {0, 1, 5000}};
    std::map<std::array<int, 8>, int> first;
    for (size_t i = 0; i < b->descs.size(); i++)
        if (!first.count(tune_key(b->descs[i]))) first[tune_key(b->descs[i])] = (int)i;
    int written = 0;
    for (auto &kv : first) {
        rmt3d_scene *probe = nullptr;
        int e = rmt3d_scene_create(&b->descs[kv.second], nullptr, &probe);
        if (e) return e;
        if ((e = rmt3d_prepare(probe))) {
            rmt3d_scene_destroy(probe);
            return e;
        }
        // The probe steps on through the search, and a flow's steps get
        // cheaper as it settles, so candidates are timed in rounds: every
        // round times each candidate still in the race for probe_steps steps,
        // in alternating order (forward, backward, forward), and a candidate's
        // time is its sum over the rounds.  After the first round candidates
        // slower than 1.5x the fastest leave the race.
        struct cand {
            int vd, vu, cl, sm, cc, bs;
            double t;
            bool ok;
        };
        auto race = [&](std::vector<cand> &cs) {
            for (int round = 0; round < 3; round++) {
                for (size_t q = 0; q < cs.size(); q++) {
                    cand &c = cs[round % 2 ? cs.size() - 1 - q : q];
                    if (!c.ok) continue;
                    if (rmt3d_scene_set_mg_launch(probe, c.cl) || rmt3d_scene_set_coarse_cluster(probe, c.cc) ||
                        rmt3d_scene_set_schedule(probe, c.vd, c.vu, 0) || rmt3d_scene_set_smoother(probe, c.sm) ||
                        rmt3d_scene_set_block_shape(probe, c.bs)) {
                        c.ok = false;  // e.g. clusters unavailable on this device
                        continue;
                    }
                    int st = 0;
                    // settle the cycle predictor, build the graph
                    if (rmt3d_run(probe, 1, &st) || rmt3d_sync(probe) || st) {
                        c.ok = false;
                        continue;
                    }
                    auto t0 = std::chrono::steady_clock::now();
                    const int er = rmt3d_run(probe, probe_steps, &st);
                    const int es = rmt3d_sync(probe);
                    if (er || es || st) {
                        c.ok = false;
                        continue;
                    }
                    c.t += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
                }
                if (round == 0) {
                    double tmin = 1e300;
                    for (auto &c : cs)
                        if (c.ok) tmin = std::min(tmin, c.t);
                    for (auto &c : cs)
                        if (c.ok && c.t > 1.5 * tmin) c.ok = false;
                }
            }
            int bi = -1;
            for (size_t q = 0; q < cs.size(); q++)
                if (cs[q].ok && (bi < 0 || cs[q].t < cs[bi].t)) bi = (int)q;
            return bi;
        };
        std::vector<cand> cs;
        for (auto &ln : launch)
            for (auto &c : smooth) cs.push_back({c[0], c[1], ln[0], ln[1], ln[2], 0, 0.0, true});
        int bi = race(cs);
        int bd = 2, bu = 2, bc = 0, bs = 0, bcc = 0, bb = 0;
        if (bi >= 0) {
            bd = cs[bi].vd, bu = cs[bi].vu, bc = cs[bi].cl, bs = cs[bi].sm, bcc = cs[bi].cc;
            // then the block shapes of the bulk kernels under that schedule
            std::vector<cand> shapes;
            for (int shape = 0; shape < RMT3D_BLOCK_SHAPES; shape++) shapes.push_back({bd, bu, bc, bs, bcc, shape, 0.0, true});
            const int si = race(shapes);
            if (si >= 0) bb = shapes[si].bs;
        }
        rmt3d_scene_destroy(probe);
        b->tuned[kv.first] = {bd, bu, bc, bs, bcc, bb};
        for (size_t i = 0; i < b->descs.size(); i++)
            if (tune_key(b->descs[i]) == kv.first) {
                if ((e = rmt3d_scene_set_schedule(b->scenes[i], bd, bu, 0))) return e;
                if ((e = rmt3d_scene_set_mg_launch(b->scenes[i], bc))) return e;
                if ((e = rmt3d_scene_set_smoother(b->scenes[i], bs))) return e;
                if ((e = rmt3d_scene_set_coarse_cluster(b->scenes[i], bcc))) return e;
                if ((e = rmt3d_scene_set_block_shape(b->scenes[i], bb))) return e;
            }
        if (tuned_out && written < max_out) {
            tuned_out[7 * written] = (int)cells(b->descs[kv.second]);
            tuned_out[7 * written + 1] = bd;
            tuned_out[7 * written + 2] = bu;
            tuned_out[7 * written + 3] = bc;
            tuned_out[7 * written + 4] = bs;
            tuned_out[7 * written + 5] = bcc;
            tuned_out[7 * written + 6] = bb;
        }
        written++;
    }
    if (n_out) *n_out = written;
    return RMT3D_OK;
}

// The smoother of every scene of the batch (rmt3d_scene_set_smoother); the
// groups are rebuilt at the next step.
extern "C" int rmt3d_batch_set_smoother(rmt3d_batch *b, int mode) {
    if (!b) return rmt3d::fail(RMT3D_ERR_INVALID, "null batch");
    drop_groups(b);
    for (auto *s : b->scenes) {
        const int e = rmt3d_scene_set_smoother(s, mode);
        if (e) return e;
    }
    return RMT3D_OK;
}

extern "C" int rmt3d_batch_destroy(rmt3d_batch *b) {
    if (!b) return RMT3D_OK;
    drop_groups(b);
    for (auto *s : b->scenes) rmt3d_scene_destroy(s);
    delete b;
    return RMT3D_OK;
}

// ---------------------------------------------------------------------------
// Serving loops with continuous batching: requests arrive over time and are
// admitted while others run, as slots and memory free up; their work
// overlaps on the device.
//
// rmt3d_serve (streams): each admitted request is a scene on its own stream,
// stepped by one of max_slots host workers; the workers' kernels overlap on
// the device.  A request is admitted when a worker is free and its device
// footprint fits the remaining HBM budget (the earliest arrived request that
// fits goes first).
//
// rmt3d_serve_grouped: a pool of set-up threads admits each arrived request,
// in arrival order, when its footprint fits the budget and fewer than
// max_slots requests are in the system, and sets its scene up while the
// running scenes keep stepping.  Scenes of the same kind (grid shape,
// periodicity, form, schedule) step together as one group graph -- each
// multigrid solve batched over the group -- in rounds of up to kServeRound
// steps.  Every kind's group runs its rounds on its own: the stepping thread
// polls the groups and, as soon as a round ends, lets finished requests leave
// (their memory returns to the budget), lets newly set-up requests of that
// kind join, and starts the next round.  A group is rebuilt only when its
// membership changes.
//
// Measured on the served workload's stream (mixed form, 100 steps per
// request) the stream form delivers more: the large grids fill the GPU on
// their own, and a group pays its rebuilds, its rounds and, in each batched
// solve, the cycles of its slowest member.
// ---------------------------------------------------------------------------
extern "C" int rmt3d_scene_checksum(rmt3d_scene *s, double out[4]);
extern "C" size_t rmt3d_scene_footprint(const rmt3d_scene_desc *d);

namespace {
double pct(std::vector<double> v, double q) {
    if (v.empty()) return 0;
    std::sort(v.begin(), v.end());
    double pos = q * (v.size() - 1);
    size_t lo = (size_t)pos, hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (pos - lo) * (v[hi] - v[lo]);
}

constexpr int kServeRound = 10;  // steps per round of the stepping thread

struct served {
    int id;
    rmt3d_scene *s;
    int left;   // steps still to run
    size_t fp;  // footprint held against the budget
};

// the kind of a scene: what a group's members must share
std::array<double, 15> serve_key(rmt3d_scene *s, const rmt3d_scene_desc &d) {
    int sch[5];
    rmt3d::scene_schedule(s, sch);
    return {(double)d.sys_size[0], (double)d.sys_size[1], (double)d.sys_size[2], (double)d.periodic[0],
            (double)d.periodic[1], (double)d.periodic[2], (double)d.precision, (double)d.var_den,
            (double)d.mg_exact, d.mixed_rtol, (double)sch[0], (double)sch[1], (double)sch[2], (double)sch[3],
            (double)sch[4]};
}
}  // namespace

extern "C" int rmt3d_serve_grouped(const rmt3d_request *reqs, int nreq, size_t hbm_budget, int max_slots,
                                   rmt3d_request_result *results, rmt3d_serve_summary *summary) {
    if (!reqs || nreq < 1 || !results || max_slots < 1) return rmt3d::fail(RMT3D_ERR_INVALID, "bad serve arguments");
    for (int i = 0; i < nreq; i++)
        if (rmt3d_scene_footprint(&reqs[i].desc) > hbm_budget)
            return rmt3d::fail(RMT3D_ERR_TOO_LARGE, "request " + std::to_string(i) + " exceeds the HBM budget");
    int dev = 0;
    cudaGetDevice(&dev);
    std::mutex mu;
    std::vector<char> taken(nreq, 0);
    size_t used = 0;
    int in_system = 0;  // admitted and not yet finished
    int finished = 0;
    std::vector<served> ready;  // set up, waiting for the next round
    std::atomic<int> first_err{0};
    std::string err_msg;
    std::vector<std::vector<double>> step_ms(nreq);
    for (int i = 0; i < nreq; i++) memset(&results[i], 0, sizeof(results[i]));
    const auto t0 = std::chrono::steady_clock::now();
    auto now_s = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    auto note_err = [&](int e) {
        if (e && !first_err.exchange(e)) {
            std::lock_guard<std::mutex> lk(mu);
            err_msg = rmt3d_last_error();
        }
    };
    // ---- set-up threads: admission by budget and slots, then set-up ----
    auto setup_worker = [&]() {
        cudaSetDevice(dev);
        while (!first_err) {
            int pick = -1;
            size_t fp = 0;
            {
                std::lock_guard<std::mutex> lk(mu);
                bool any_left = false;
                const double t = now_s();
                for (int i = 0; i < nreq; i++) {
                    if (taken[i]) continue;
                    any_left = true;
                    if (reqs[i].arrival_s > t) break;  // arrival order
                    const size_t f = rmt3d_scene_footprint(&reqs[i].desc);
                    if (in_system < max_slots && used + f <= hbm_budget) {
                        pick = i;
                        fp = f;
                    }
                    break;  // the earliest waiting request goes first
                }
                if (!any_left) return;
                if (pick >= 0) {
                    taken[pick] = 1;
                    used += fp;
                    in_system++;
                }
            }
            if (pick < 0) {
                std::this_thread::sleep_for(std::chrono::microseconds(200));
                continue;
            }
            results[pick].admit_s = now_s();
            rmt3d_scene *s = nullptr;
            int e = rmt3d_scene_create(&reqs[pick].desc, nullptr, &s);
            if (!e) e = rmt3d_prepare(s);
            if (e) {
                note_err(e);
                if (s) rmt3d_scene_destroy(s);
                return;
            }
            std::lock_guard<std::mutex> lk(mu);
            ready.push_back(served{pick, s, reqs[pick].steps, fp});
        }
    };
    std::vector<std::thread> th;
    const int nsetup = std::max(1, std::min(4, max_slots));
    for (int k = 0; k < nsetup; k++) th.emplace_back(setup_worker);

    // ---- the stepping thread (this one): each kind's group runs its rounds
    // on its own; the thread polls the groups and relaunches each one as soon
    // as its round ends, so small and large kinds do not wait for each other
    struct kind_group {
        std::vector<served> m;        // members of the running or next round
        std::vector<served> joining;  // set up, joining at the next round
        rmt3d::scene_group *g = nullptr;
        bool dirty = true, busy = false;
        int k = 0;  // steps of the round in flight
        std::chrono::steady_clock::time_point t_launch;
    };
    std::map<std::array<double, 15>, kind_group> kinds;
    long long cellsteps = 0;
    while (!first_err) {
        {
            std::lock_guard<std::mutex> lk(mu);
            if (finished >= nreq) break;
            for (auto &r : ready) kinds[serve_key(r.s, reqs[r.id].desc)].joining.push_back(r);
            ready.clear();
        }
        bool progress = false;
        for (auto &kv : kinds) {
            kind_group &kg = kv.second;
            if (kg.busy) {
                if (!rmt3d::group_done(kg.g)) continue;
                // the round ended: results of the members that are done
                progress = true;
                kg.busy = false;
                std::vector<int> st(kg.m.size(), 0);
                int e = rmt3d::group_finish(kg.g, st.data());
                const double ms =
                    1e3 * std::chrono::duration<double>(std::chrono::steady_clock::now() - kg.t_launch).count() / kg.k;
                std::vector<served> keep;
                for (size_t j = 0; j < kg.m.size(); j++) {
                    served &r = kg.m[j];
                    rmt3d_request_result &R = results[r.id];
                    for (int q = 0; q < kg.k; q++) step_ms[r.id].push_back(ms);
                    r.left -= kg.k;
                    if (r.left > 0 && st[j] == 0 && !e) {
                        keep.push_back(r);
                        continue;
                    }
                    R.steps_done = reqs[r.id].steps - std::max(r.left, 0);
                    R.status = e ? e : st[j];
                    if (rmt3d_scene_checksum(r.s, R.checksum) && !R.status) R.status = RMT3D_ERR_CUDA;
                    R.finish_s = now_s();
                    R.latency_s = R.finish_s - reqs[r.id].arrival_s;
                    R.step_p50_ms = pct(step_ms[r.id], 0.5);
                    R.step_p99_ms = pct(step_ms[r.id], 0.99);
                    cellsteps += (long long)R.steps_done * reqs[r.id].desc.sys_size[0] *
                                 reqs[r.id].desc.sys_size[1] * reqs[r.id].desc.sys_size[2];
                    kg.dirty = true;
                    if (kg.g) rmt3d::group_destroy(kg.g);  // before its member goes
                    kg.g = nullptr;
                    rmt3d_scene_destroy(r.s);
                    std::lock_guard<std::mutex> lk(mu);
                    used -= r.fp;
                    in_system--;
                    finished++;
                }
                kg.m.swap(keep);
                note_err(e);
                if (e) break;
            }
            // not busy: start the next round with the members and the joiners
            if (!kg.joining.empty()) {
                kg.m.insert(kg.m.end(), kg.joining.begin(), kg.joining.end());
                kg.joining.clear();
                kg.dirty = true;
            }
            if (kg.m.empty()) continue;
            if (kg.dirty) {
                if (kg.g) rmt3d::group_destroy(kg.g);
                kg.g = nullptr;
                std::vector<rmt3d_scene *> sc;
                for (auto &r : kg.m) sc.push_back(r.s);
                int e = rmt3d::group_create(sc.data(), (int)sc.size(), &kg.g);
                if (e) {
                    note_err(e);
                    break;
                }
                kg.dirty = false;
            }
            int k = kServeRound;
            for (auto &r : kg.m) k = std::min(k, r.left);
            kg.t_launch = std::chrono::steady_clock::now();
            int e = rmt3d::group_launch(kg.g, k);
            if (e) {
                note_err(e);
                break;
            }
            kg.k = k;
            kg.busy = true;
            progress = true;
        }
        if (!progress) std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
    // a failure can leave rounds in flight: wait for them before the scenes go
    for (auto &kv : kinds)
        if (kv.second.busy && kv.second.g) {
            std::vector<int> st(kv.second.m.size(), 0);
            rmt3d::group_finish(kv.second.g, st.data());
        }
    for (auto &x : th) x.join();
    for (auto &kv : kinds) {
        if (kv.second.g) rmt3d::group_destroy(kv.second.g);
        for (auto &r : kv.second.m) rmt3d_scene_destroy(r.s);
        for (auto &r : kv.second.joining) rmt3d_scene_destroy(r.s);
    }
    for (auto &r : ready) rmt3d_scene_destroy(r.s);
    const double wall = now_s();
    if (summary) {
        std::vector<double> lat, steps;
        for (int i = 0; i < nreq; i++) {
            lat.push_back(results[i].latency_s);
            steps.insert(steps.end(), step_ms[i].begin(), step_ms[i].end());
        }
        summary->wall_s = wall;
        summary->request_p50_s = pct(lat, 0.5);
        summary->request_p99_s = pct(lat, 0.99);
        summary->step_p50_ms = pct(steps, 0.5);
        summary->step_p99_ms = pct(steps, 0.99);
        summary->cellsteps_per_s = cellsteps / wall;
        summary->requests = nreq;
    }
    if (first_err) return rmt3d::fail(first_err, err_msg);
    return RMT3D_OK;
}

extern "C" int rmt3d_serve(const rmt3d_request *reqs, int nreq, size_t hbm_budget, int max_slots,
                           rmt3d_request_result *results, rmt3d_serve_summary *summary) {
    if (!reqs || nreq < 1 || !results || max_slots < 1) return rmt3d::fail(RMT3D_ERR_INVALID, "bad serve arguments");
    for (int i = 0; i < nreq; i++)
        if (rmt3d_scene_footprint(&reqs[i].desc) > hbm_budget)
            return rmt3d::fail(RMT3D_ERR_TOO_LARGE, "request " + std::to_string(i) + " exceeds the HBM budget");
    int dev = 0;
    cudaGetDevice(&dev);
    std::mutex mu;
    std::vector<char> taken(nreq, 0);
    size_t used = 0;
    int done = 0;
    std::atomic<int> first_err{0};
    std::string err_msg;
    std::vector<std::vector<double>> step_ms(nreq);
    const auto t0 = std::chrono::steady_clock::now();
    auto now_s = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    std::vector<long long> cellsteps(max_slots, 0);
    auto worker = [&](int slot) {
        cudaSetDevice(dev);
        while (true) {
            int pick = -1;
            size_t fp = 0;
            {
                std::lock_guard<std::mutex> lk(mu);
                if (done >= nreq || first_err) return;
                double t = now_s();
                // earliest arrived request that fits the free budget
                for (int i = 0; i < nreq; i++) {
                    if (taken[i] || reqs[i].arrival_s > t) continue;
                    size_t f = rmt3d_scene_footprint(&reqs[i].desc);
                    if (used + f <= hbm_budget) {
                        pick = i;
                        fp = f;
                        break;
                    }
                }
                if (pick >= 0) {
                    taken[pick] = 1;
                    used += fp;
                } else {
                    bool any_left = false;
                    for (int i = 0; i < nreq; i++)
                        if (!taken[i]) any_left = true;
                    if (!any_left) return;
                }
            }
            if (pick < 0) {
                std::this_thread::sleep_for(std::chrono::microseconds(200));
                continue;
            }
            rmt3d_request_result &R = results[pick];
            memset(&R, 0, sizeof(R));
            R.admit_s = now_s();
            rmt3d_scene *s = nullptr;
            int e = rmt3d_scene_create(&reqs[pick].desc, nullptr, &s);
            if (!e) e = rmt3d_prepare(s);
            int st = 0;
            for (int k = 0; !e && k < reqs[pick].steps && st == 0; k++) {
                auto a = std::chrono::steady_clock::now();
                e = rmt3d_step(s, 0, &st);
                if (!e) e = rmt3d_sync(s);
                step_ms[pick].push_back(
                    1e3 * std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count());
            }
            if (!e) e = rmt3d_scene_checksum(s, R.checksum);
            R.finish_s = now_s();
            R.latency_s = R.finish_s - reqs[pick].arrival_s;
            R.status = e ? e : st;
            R.steps_done = (int)step_ms[pick].size();
            R.step_p50_ms = pct(step_ms[pick], 0.5);
            R.step_p99_ms = pct(step_ms[pick], 0.99);
            cellsteps[slot] += (long long)R.steps_done * reqs[pick].desc.sys_size[0] * reqs[pick].desc.sys_size[1] *
                               reqs[pick].desc.sys_size[2];
            if (e && !first_err.exchange(e)) {
                std::lock_guard<std::mutex> lk(mu);
                err_msg = rmt3d_last_error();
            }
            rmt3d_scene_destroy(s);
            std::lock_guard<std::mutex> lk(mu);
            used -= fp;
            done++;
        }
    };
    std::vector<std::thread> th;
    for (int k = 0; k < max_slots; k++) th.emplace_back(worker, k);
    for (auto &x : th) x.join();
    const double wall = now_s();
    if (summary) {
        std::vector<double> lat, steps;
        long long cs = 0;
        for (int i = 0; i < nreq; i++) {
            lat.push_back(results[i].latency_s);
            steps.insert(steps.end(), step_ms[i].begin(), step_ms[i].end());
        }
        for (long long c : cellsteps) cs += c;
        summary->wall_s = wall;
        summary->request_p50_s = pct(lat, 0.5);
        summary->request_p99_s = pct(lat, 0.99);
        summary->step_p50_ms = pct(steps, 0.5);
        summary->step_p99_ms = pct(steps, 0.99);
        summary->cellsteps_per_s = cs / wall;
        summary->requests = nreq;
    }
    if (first_err) return rmt3d::fail(first_err, err_msg);
    return RMT3D_OK;
}
