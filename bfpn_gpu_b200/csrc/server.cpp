// Multi-beam batching and serving on top of the single-beam C ABI.
//
// The reference runs one beam per process (main.cu:344-348).  A treatment plan
// or a dose engine needs many independent beams, most too small to fill a
// B200 alone.  This layer keeps a thread-safe queue of beam requests and
// serves it two ways:
//
// - continuous batching: requests that a bundle can hold (mixed precision,
//   the eq15 step, square angular grids; bfpn_bundle_accepts) go to one
//   scheduler thread per device.  It admits them FIFO into bundles by shape
//   class -- each admission checks the beam's device footprint against the
//   free memory first -- and advances every bundle a time slice of depth
//   steps per round, the bundles of different classes on their own streams at
//   once.  Beams that arrive while others run join at the next round; a
//   finished beam's results are collected and its slot and memory freed at
//   once.  Results equal the beam run alone up to the order of the IDD
//   partial sums.
// - worker threads for everything else, each owning one solver context (its
//   own stream and CUDA graph) on one device, kept between requests of the
//   same shape (grid, flags, precision) with only the tables and the beam
//   reloaded; results equal a single-context run bit for bit.
//
// bfpn_server_submit copies the request's tables, so callers may free them at
// once.  Results stay with the server until bfpn_server_wait collects them.

#include "../../include/bfpn_capi.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <map>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

thread_local std::string g_server_error;

bfpn_status server_fail(bfpn_status s, const std::string& msg) {
    g_server_error = msg;
    return s;
}

struct Job {
    uint64_t ticket = 0;
    bfpn_grid grid{};
    bfpn_phys phys{};
    int32_t precision = BFPN_PREC_FP64;
    int32_t nsteps = 0;
    std::vector<double> mu, sigma;
    int32_t mu_rows = 0, sigma_rows = 0;
    // results
    bool done = false;
    bfpn_status status = BFPN_OK;
    std::string error;
    std::vector<double> idd, proxy;
    int32_t device = -1;
    bool bundled = false;  // served by a bundle scheduler
    Clock::time_point submitted, started, finished;
};

bool same_shape(const Job& a, const bfpn_grid& g, const bfpn_phys& p, int32_t prec) {
    return std::memcmp(&a.grid, &g, sizeof g) == 0 && a.phys.flags == p.flags && a.precision == prec &&
           a.phys.density == p.density && a.phys.energy_density == p.energy_density && a.phys.sig_E == p.sig_E &&
           a.phys.a_1 == p.a_1 && a.phys.a_2 == p.a_2 && a.phys.C_c == p.C_c && a.phys.beam_energy == p.beam_energy &&
           a.phys.material == p.material;
}

}  // namespace

struct bfpn_server {
    std::mutex mu;
    std::condition_variable cv_work;  // workers: a job was queued, or shutdown
    std::condition_variable cv_done;  // waiters: a job finished
    std::condition_variable cv_bundle;  // schedulers: a bundle job was queued, or shutdown
    std::deque<std::shared_ptr<Job>> queue;         // jobs for the context workers
    std::deque<std::shared_ptr<Job>> bundle_queue;  // jobs for the bundle schedulers
    std::unordered_map<uint64_t, std::shared_ptr<Job>> jobs;
    uint64_t next_ticket = 1;
    bool stopping = false;
    bool batching = true;
    std::vector<std::thread> workers;
    std::vector<std::thread> schedulers;
    std::vector<int> busy_per_device;     // context-worker jobs running, by position in `devices`
    std::vector<int> bundled_per_device;  // bundle jobs running, same index
    std::vector<int32_t> devices;
};

namespace {

// One request on this worker's device: (re)use the context, load, step, collect.
void run_job(bfpn_server* s, int dev_slot, Job& j, bfpn_ctx*& ctx, Job& ctx_shape) {
    const int32_t device = s->devices[dev_slot];
    auto fail = [&](bfpn_status st, const char* what) {
        j.status = st;
        j.error = std::string(what) + ": " + bfpn_last_error(ctx);
    };
    if (ctx && !same_shape(ctx_shape, j.grid, j.phys, j.precision)) {
        bfpn_destroy(ctx);
        ctx = nullptr;
    }
    if (!ctx) {
        // admission by footprint: wait while the beam does not fit in free
        // memory and other work on this device may still free some; then
        // create, and on OOM retry the same way (another worker may have
        // allocated in between); fail once nothing else runs
        uint64_t need = 0;
        if (bfpn_footprint_bytes(&j.grid, &j.phys, j.precision, &need) == BFPN_OK) {
            for (;;) {
                uint64_t free_b = 0;
                if (bfpn_device_memory(device, &free_b, nullptr) != BFPN_OK || need + (512ull << 20) <= free_b) break;
                std::unique_lock<std::mutex> lk(s->mu);
                const bool others = s->busy_per_device[dev_slot] > 1 || s->bundled_per_device[dev_slot] > 0;
                if (!others || s->stopping) break;  // let bfpn_create report it
                s->cv_done.wait_for(lk, std::chrono::milliseconds(50));
            }
        }
        for (;;) {
            bfpn_status st = bfpn_create(&j.grid, &j.phys, j.precision, device, &ctx);
            if (st == BFPN_OK) break;
            ctx = nullptr;
            if (st != BFPN_OOM) {
                j.status = st;
                j.error = std::string("create: ") + bfpn_last_error(nullptr);
                return;
            }
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->busy_per_device[dev_slot] <= 1 || s->stopping) {
                j.status = st;
                j.error = std::string("create: ") + bfpn_last_error(nullptr);
                return;
            }
            s->cv_done.wait_for(lk, std::chrono::milliseconds(50));
        }
        ctx_shape.grid = j.grid;
        ctx_shape.phys = j.phys;
        ctx_shape.precision = j.precision;
    }
    bfpn_status st = bfpn_load_tables(ctx, j.mu.data(), j.mu_rows, j.sigma.data(), j.sigma_rows);
    if (st != BFPN_OK) return fail(st, "load_tables");
    if ((st = bfpn_init_beam(ctx)) != BFPN_OK) return fail(st, "init_beam");
    j.idd.assign(static_cast<size_t>(j.nsteps), 0.0);
    j.proxy.assign(static_cast<size_t>(j.nsteps), 0.0);
    if ((st = bfpn_step(ctx, j.nsteps, j.idd.data(), j.proxy.data())) != BFPN_OK) return fail(st, "step");
    j.status = BFPN_OK;
}

void worker_main(bfpn_server* s, int dev_slot) {
    bfpn_ctx* ctx = nullptr;
    Job shape;
    for (;;) {
        std::shared_ptr<Job> j;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv_work.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
            if (s->queue.empty()) break;  // stopping and drained
            j = s->queue.front();
            s->queue.pop_front();
            s->busy_per_device[dev_slot]++;
            j->started = Clock::now();
            j->device = s->devices[dev_slot];
        }
        run_job(s, dev_slot, *j, ctx, shape);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            j->finished = Clock::now();
            j->done = true;
            s->busy_per_device[dev_slot]--;
        }
        s->cv_done.notify_all();
    }
    if (ctx) bfpn_destroy(ctx);
}

// ---- continuous batching ----------------------------------------------------

// Shape class of a bundle-eligible beam: kernels depend on the plane, the
// angular grid, the energy model and the clipping of psi^1.
std::string class_key(const Job& j) {
    const uint32_t fl = j.phys.flags & (BFPN_FLAG_EQ15_STRAGGLING | BFPN_FLAG_NO_SPATIAL_CLIPPING);
    return std::to_string(j.grid.Ny) + "x" + std::to_string(j.grid.Nz) + "/" + std::to_string(j.grid.Nmu) + "x" +
           std::to_string(j.grid.Nom) + "/" + std::to_string(fl);
}

constexpr int kBundleSlots = 64;
constexpr double kSliceMs = 40.0;  // target length of one round of bundle steps

struct LiveBundle {
    bfpn_bundle* b = nullptr;
    std::map<int, std::shared_ptr<Job>> slots;  // running jobs by slot
    double ms_per_step = 1.0;                     // running estimate (host clock, concurrent rounds)
};

void finish(bfpn_server* s, const std::shared_ptr<Job>& j, bfpn_status st, const std::string& err,
            int dev_slot = -1) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (dev_slot >= 0) s->bundled_per_device[dev_slot]--;  // a running bundle job ends
        j->status = st;
        if (st != BFPN_OK) j->error = err;
        j->finished = Clock::now();
        j->done = true;
    }
    s->cv_done.notify_all();
}

void scheduler_main(bfpn_server* s, int dev_slot) {
    const int32_t device = s->devices[dev_slot];
    std::map<std::string, LiveBundle> live;
    for (;;) {
        bool any_running = false;
        for (auto& kv : live) any_running = any_running || !kv.second.slots.empty();
        // 1. admit queued jobs FIFO while they fit (a job that does not fit waits at the head)
        for (;;) {
            std::shared_ptr<Job> j;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                if (!any_running)
                    s->cv_bundle.wait(lk, [&] { return s->stopping || !s->bundle_queue.empty(); });
                if (s->bundle_queue.empty()) {
                    if (s->stopping && !any_running) {
                        lk.unlock();
                        for (auto& kv : live) bfpn_bundle_destroy(kv.second.b);
                        return;
                    }
                    break;
                }
                j = s->bundle_queue.front();
                s->bundle_queue.pop_front();
            }
            LiveBundle& lb = live[class_key(*j)];
            bfpn_status st = BFPN_OK;
            if (!lb.b) st = bfpn_bundle_create(device, kBundleSlots, &lb.b);
            int32_t slot = -1;
            bfpn_beam beam{j->grid, j->phys, j->precision, j->nsteps, j->mu.data(), j->mu_rows, j->sigma.data(),
                           j->sigma_rows};
            if (st == BFPN_OK && static_cast<int>(lb.slots.size()) < kBundleSlots)
                st = bfpn_bundle_admit(lb.b, &beam, &slot);
            else if (st == BFPN_OK)
                st = BFPN_OOM;  // every slot taken: wait like a beam that does not fit
            if (st == BFPN_OK) {
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    j->started = Clock::now();
                    j->device = device;
                    s->bundled_per_device[dev_slot]++;
                }
                lb.slots[slot] = j;
                any_running = true;
                continue;
            }
            if (st == BFPN_OOM) {
                // wait for running beams -- bundled, or on this device's context workers -- to free memory
                std::unique_lock<std::mutex> lk(s->mu);
                if (any_running || s->busy_per_device[dev_slot] > 0) {
                    s->bundle_queue.push_front(j);
                    if (!any_running) s->cv_done.wait_for(lk, std::chrono::milliseconds(50));
                    break;
                }
            }
            if (st == BFPN_INVALID_ARG) {  // a bundle cannot hold it after all: a context worker serves it
                {
                    std::lock_guard<std::mutex> lk(s->mu);
                    j->bundled = false;
                    s->queue.push_back(j);
                }
                s->cv_work.notify_one();
                continue;
            }
            finish(s, j, st, std::string("bundle admit: ") + bfpn_bundle_last_error(lb.b));
        }
        if (!any_running) continue;
        // 2. one round: every bundle with running beams advances a time slice, concurrently
        const auto t0 = Clock::now();
        std::vector<std::pair<LiveBundle*, int>> stepped;
        for (auto& kv : live) {
            LiveBundle& lb = kv.second;
            if (lb.slots.empty()) continue;
            const int n = std::max(1, std::min(512, static_cast<int>(kSliceMs / std::max(lb.ms_per_step, 1e-3))));
            bfpn_status st = bfpn_bundle_step(lb.b, n);
            if (st != BFPN_OK) {
                const std::string err = std::string("bundle step: ") + bfpn_bundle_last_error(lb.b);
                for (auto& sj : lb.slots) finish(s, sj.second, st, err, dev_slot);
                lb.slots.clear();
                bfpn_bundle_destroy(lb.b);
                lb.b = nullptr;
                continue;
            }
            stepped.emplace_back(&lb, n);
        }
        // 3. wait, then collect the finished beams
        for (auto& [lb, n] : stepped) {
            bfpn_status st = bfpn_bundle_sync(lb->b);
            const double ms = ms_between(t0, Clock::now());
            lb->ms_per_step = 0.5 * lb->ms_per_step + 0.5 * ms / n;
            for (auto it = lb->slots.begin(); it != lb->slots.end();) {
                int32_t done = 0, total = 0;
                bfpn_bundle_slot(lb->b, it->first, &done, &total);
                if (st == BFPN_OK && done < total) {
                    ++it;
                    continue;
                }
                std::shared_ptr<Job> j = it->second;
                bfpn_status cs = st;
                if (cs == BFPN_OK) {
                    j->idd.assign(static_cast<size_t>(j->nsteps), 0.0);
                    j->proxy.assign(static_cast<size_t>(j->nsteps), 0.0);
                    cs = bfpn_bundle_collect(lb->b, it->first, j->idd.data(), j->proxy.data(), j->nsteps);
                }
                finish(s, j, cs, std::string("bundle: ") + bfpn_bundle_last_error(lb->b), dev_slot);
                it = lb->slots.erase(it);
            }
            if (st != BFPN_OK) {  // the bundle's state is suspect: drop it
                bfpn_bundle_destroy(lb->b);
                lb->b = nullptr;
            }
        }
        for (auto it = live.begin(); it != live.end();)
            it = (it->second.b == nullptr) ? live.erase(it) : std::next(it);
    }
}

}  // namespace

extern "C" {

const char* bfpn_server_last_error(void) { return g_server_error.c_str(); }

bfpn_status bfpn_server_set_batching(bfpn_server* s, int32_t on) {
    if (!s) return server_fail(BFPN_INVALID_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->next_ticket != 1) return server_fail(BFPN_NOT_READY, "set batching before the first submit");
    s->batching = on != 0;
    return BFPN_OK;
}

bfpn_status bfpn_server_create(const int32_t* devices, int32_t n_devices, int32_t workers_per_device,
                               bfpn_server** out) {
    if (!out) return server_fail(BFPN_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (n_devices < 0 || (n_devices > 0 && !devices) || workers_per_device < 1 || workers_per_device > 64)
        return server_fail(BFPN_INVALID_ARG, "need a device list (or none for device 0) and 1..64 workers per device");
    const int32_t ndev = bfpn_device_count();
    if (ndev <= 0) return server_fail(BFPN_NO_DEVICE, "no CUDA device available");
    std::vector<int32_t> devs = n_devices > 0 ? std::vector<int32_t>(devices, devices + n_devices)
                                              : std::vector<int32_t>{0};
    for (int32_t d : devs)
        if (d < 0 || d >= ndev) return server_fail(BFPN_INVALID_ARG, "device ordinal out of range");
    auto* s = new bfpn_server();
    s->devices = devs;
    s->busy_per_device.assign(devs.size(), 0);
    s->bundled_per_device.assign(devs.size(), 0);
    for (size_t k = 0; k < devs.size(); ++k) {
        for (int w = 0; w < workers_per_device; ++w) s->workers.emplace_back(worker_main, s, static_cast<int>(k));
        s->schedulers.emplace_back(scheduler_main, s, static_cast<int>(k));
    }
    *out = s;
    return BFPN_OK;
}

bfpn_status bfpn_server_submit(bfpn_server* s, const bfpn_beam* beam, uint64_t* ticket) {
    if (!s || !beam || !ticket) return server_fail(BFPN_INVALID_ARG, "null argument");
    if (beam->nsteps < 1) return server_fail(BFPN_INVALID_ARG, "nsteps must be >= 1");
    if ((!beam->mu && beam->mu_rows > 0) || !beam->sigma_c || beam->mu_rows < 0 || beam->sigma_rows < 1)
        return server_fail(BFPN_INVALID_ARG, "missing tables");
    if (beam->precision != BFPN_PREC_FP64 && beam->precision != BFPN_PREC_MIXED)
        return server_fail(BFPN_INVALID_ARG, "unknown precision");
    auto j = std::make_shared<Job>();
    j->grid = beam->grid;
    j->phys = beam->phys;
    j->precision = beam->precision;
    j->nsteps = beam->nsteps;
    j->mu_rows = beam->mu_rows;
    j->sigma_rows = beam->sigma_rows;
    j->mu.assign(beam->mu, beam->mu + 3 * static_cast<size_t>(beam->mu_rows));
    j->sigma.assign(beam->sigma_c, beam->sigma_c + beam->sigma_rows);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) return server_fail(BFPN_NOT_READY, "server is shutting down");
        j->ticket = s->next_ticket++;
        j->submitted = Clock::now();
        s->jobs[j->ticket] = j;
        j->bundled = s->batching && bfpn_bundle_accepts(beam) == BFPN_OK;
        (j->bundled ? s->bundle_queue : s->queue).push_back(j);
        *ticket = j->ticket;
    }
    if (j->bundled) s->cv_bundle.notify_all();
    else s->cv_work.notify_one();
    return BFPN_OK;
}

int32_t bfpn_server_poll(bfpn_server* s, uint64_t ticket) {
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return -1;
    return it->second->done ? 1 : 0;
}

bfpn_status bfpn_server_wait(bfpn_server* s, uint64_t ticket, double timeout_s, double* idd, double* proxy,
                             int32_t capacity, bfpn_beam_info* info) {
    if (!s) return server_fail(BFPN_INVALID_ARG, "null server");
    std::shared_ptr<Job> j;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->jobs.find(ticket);
        if (it == s->jobs.end()) return server_fail(BFPN_INVALID_ARG, "unknown ticket (or already collected)");
        j = it->second;
        auto ready = [&] { return j->done; };
        if (timeout_s < 0) {
            s->cv_done.wait(lk, ready);
        } else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
            return server_fail(BFPN_TIMEOUT, "beam not finished within the timeout");
        }
        if ((idd || proxy) && j->status == BFPN_OK && capacity < j->nsteps)
            return server_fail(BFPN_INVALID_ARG, "result arrays hold fewer than nsteps values");
        s->jobs.erase(it);
    }
    if (info) {
        info->steps = j->status == BFPN_OK ? j->nsteps : 0;
        info->device = j->device;
        info->queue_ms = ms_between(j->submitted, j->started);
        info->run_ms = ms_between(j->started, j->finished);
    }
    if (j->status != BFPN_OK) return server_fail(j->status, j->error);
    if (idd) std::copy(j->idd.begin(), j->idd.end(), idd);
    if (proxy) std::copy(j->proxy.begin(), j->proxy.end(), proxy);
    return BFPN_OK;
}

bfpn_status bfpn_server_destroy(bfpn_server* s) {
    if (!s) return BFPN_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
    }
    s->cv_work.notify_all();
    s->cv_bundle.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto& t : s->schedulers) t.join();
    delete s;
    return BFPN_OK;
}

bfpn_status bfpn_batch_run(const bfpn_beam* beams, int32_t n, const int32_t* devices, int32_t n_devices,
                           int32_t workers_per_device, double* const* idd_out, double* const* proxy_out,
                           bfpn_status* status_out) {
    if (n < 0 || (n > 0 && !beams)) return server_fail(BFPN_INVALID_ARG, "need n >= 0 beams");
    bfpn_server* s = nullptr;
    bfpn_status st = bfpn_server_create(devices, n_devices, workers_per_device, &s);
    if (st != BFPN_OK) return st;
    std::vector<uint64_t> tickets(static_cast<size_t>(n), 0);
    std::vector<bfpn_status> sub(static_cast<size_t>(n), BFPN_OK);
    for (int32_t i = 0; i < n; ++i) sub[i] = bfpn_server_submit(s, &beams[i], &tickets[i]);
    bfpn_status first = BFPN_OK;
    std::string first_msg;
    for (int32_t i = 0; i < n; ++i) {
        bfpn_status r = sub[i];
        if (r == BFPN_OK)
            r = bfpn_server_wait(s, tickets[i], -1.0, idd_out ? idd_out[i] : nullptr, proxy_out ? proxy_out[i] : nullptr,
                                 beams[i].nsteps, nullptr);
        if (status_out) status_out[i] = r;
        if (r != BFPN_OK && first == BFPN_OK) {
            first = r;
            first_msg = "beam " + std::to_string(i) + ": " + g_server_error;
        }
    }
    bfpn_server_destroy(s);
    if (first != BFPN_OK) return server_fail(first, first_msg);
    return BFPN_OK;
}

}  // extern "C"
