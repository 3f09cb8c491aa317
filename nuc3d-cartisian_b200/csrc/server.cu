// Served form of the solver: a request loop over one batch (nuc3d_serve_* in
// include/nuc3d_b200.h).
//
// One worker thread per server owns an Engine (the batched solver) and its
// stream.  Clients submit solve requests from any thread; the worker
//   1. admits queued requests in arrival order while the sum of the resident
//      solves' device bytes stays within the budget and a slot is free,
//      allocating each box and generating or uploading its initial state;
//   2. advances every resident solve together by one chunk of steps (the
//      batch's CUDA graph replayed), the chunk no longer than the shortest
//      remaining solve and sized to about chunk_ms of device time, so that
//      arrivals join within a chunk.  The step time of a new composition is
//      predicted from the last chunk's time per resident cell-step (the
//      first chunk of all is one step, to measure);
//   3. retires the solves whose step count is reached: final state to the
//      client's host buffer, device memory released, result posted.
// Solves therefore join and leave the running batch between chunks
// (continuous batching), and a solve's arithmetic never depends on the other
// boxes in the batch, so its result is the same alone and in the mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "engine.h"
#include "nuc3d_b200.h"
#include "op_kernels.h"

namespace nuc3d {

namespace {

using Clock = std::chrono::steady_clock;

struct Queued {
    long long ticket;
    nuc3d_solve_request req;
    long long bytes;
    double t_submit;
};

struct Resident {
    Queued q;
    int box = -1;
    long long remaining = 0;
    double t_admit = 0.0;
    double reynolds = 0.0;
};

void copy_error(nuc3d_solve_result &r, const char *msg) {
    std::strncpy(r.error, msg ? msg : "", sizeof r.error - 1);
    r.error[sizeof r.error - 1] = '\0';
}

}  // namespace

class Server {
public:
    explicit Server(const nuc3d_serve_config &c) : cfg_(c), t0_(Clock::now()) {}

    int start() {
        if (cudaGetDevice(&device_) != cudaSuccess)
            return set_last_error(NUC3D_ERR_CUDA, "no current CUDA device");
        if (cfg_.budget_bytes <= 0) {
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
                return set_last_error(NUC3D_ERR_CUDA, "cudaMemGetInfo failed");
            cfg_.budget_bytes = (long long)(0.9 * (double)free_b);
        }
        if (cfg_.max_resident <= 0) cfg_.max_resident = 256;
        if (cfg_.max_chunk_steps <= 0) cfg_.max_chunk_steps = 64;
        if (cfg_.chunk_ms <= 0.0) cfg_.chunk_ms = 20.0;
        std::unique_lock<std::mutex> lk(mu_);
        worker_ = std::thread([this] { run(); });
        started_cv_.wait(lk, [this] { return started_; });
        if (start_rc_ != NUC3D_OK) {
            lk.unlock();
            worker_.join();
            return set_last_error(start_rc_, start_err_.c_str());
        }
        return NUC3D_OK;
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        if (worker_.joinable()) worker_.join();
    }

    double now() const { return std::chrono::duration<double>(Clock::now() - t0_).count(); }

    int submit(const nuc3d_solve_request &r, long long *ticket) {
        nuc3d_box_desc d = r.desc;
        d.precision = cfg_.precision;
        std::string why;
        int rc = Engine::validate(d, &why);
        if (rc) return set_last_error(rc, why.c_str());
        if (r.nsteps < 0) return set_last_error(NUC3D_ERR_INVALID, "nsteps must be >= 0");
        if (!(r.cfl > 0.0)) return set_last_error(NUC3D_ERR_INVALID, "cfl must be > 0");
        if (r.init.kind == 0) {
            for (int e = 0; e < 5; ++e)
                if (!r.h_q0[e])
                    return set_last_error(NUC3D_ERR_INVALID, "initial state pointers missing");
        } else if (r.init.kind != NUC3D_INIT_TGV && r.init.kind != NUC3D_INIT_HIT) {
            return set_last_error(NUC3D_ERR_INVALID, "unknown initial state kind");
        }
        const long long bytes = Engine::box_bytes(d);
        if (bytes > cfg_.budget_bytes)
            return set_last_error(NUC3D_ERR_NOMEM, "solve needs more device memory than the budget");
        Queued q{0, r, bytes, now()};
        q.req.desc = d;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (stop_) return set_last_error(NUC3D_ERR_CANCELLED, "server is shutting down");
            q.ticket = next_ticket_++;
            queue_.push_back(q);
            outstanding_.insert(q.ticket);
            ++submitted_;
            *ticket = q.ticket;
        }
        cv_.notify_all();
        return NUC3D_OK;
    }

    int wait(long long ticket, double timeout_s, nuc3d_solve_result *out) {
        std::unique_lock<std::mutex> lk(mu_);
        if (ticket >= 0 && !outstanding_.count(ticket))
            return set_last_error(NUC3D_ERR_INVALID, "unknown or already collected ticket");
        if (ticket < 0 && outstanding_.empty())
            return set_last_error(NUC3D_ERR_INVALID, "no outstanding solve");
        auto ready = [&] { return ticket >= 0 ? done_.count(ticket) > 0 : !done_order_.empty(); };
        if (timeout_s < 0.0) {
            done_cv_.wait(lk, ready);
        } else if (!done_cv_.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
            return set_last_error(NUC3D_ERR_TIMEOUT, "solve not finished within the timeout");
        }
        long long t = ticket;
        if (t < 0) t = done_order_.front();
        done_order_.erase(std::find(done_order_.begin(), done_order_.end(), t));
        *out = done_[t];
        done_.erase(t);
        outstanding_.erase(t);
        return NUC3D_OK;
    }

    void info(nuc3d_serve_stats *o) {
        std::lock_guard<std::mutex> lk(mu_);
        *o = info_;
        o->submitted = submitted_;
        o->queued = (int)queue_.size();
        o->budget_bytes = cfg_.budget_bytes;
        o->now_s = now();
    }

private:
    void post(const Resident &r, int status, const char *err, Engine *eng) {
        nuc3d_solve_result res{};
        res.ticket = r.q.ticket;
        res.tag = r.q.req.tag;
        res.status = status;
        res.cells = (long long)r.q.req.desc.nx * r.q.req.desc.ny * r.q.req.desc.nz;
        res.t_submit = r.q.t_submit;
        res.t_admit = r.t_admit;
        res.reynolds = r.reynolds;
        res.sim_time = res.dt_last = res.res_last = 0.0;
        if (eng && r.box >= 0 && status == NUC3D_OK) {
            res.steps = eng->box_steps(r.box);
            res.sim_time = eng->time(r.box);
            eng->history(r.box, 1, &res.dt_last, &res.res_last);
        }
        if (err) copy_error(res, err);
        res.t_done = now();
        {
            std::lock_guard<std::mutex> lk(mu_);
            done_[res.ticket] = res;
            done_order_.push_back(res.ticket);
            if (status == NUC3D_OK) {
                ++info_.completed;
                info_.cell_updates += res.cells * res.steps;
            } else {
                ++info_.failed;
            }
        }
        done_cv_.notify_all();
    }

    // Allocates, initialises and activates one admitted solve.
    int admit(Engine &eng, Resident &r) {
        int id = -1;
        int rc = eng.add_box(r.q.req.desc, &id);
        if (rc) return rc;
        r.box = id;
        const nuc3d_solve_request &q = r.q.req;
        if (q.init.kind == 0) {
            rc = eng.set_state(id, q.h_q0, cudaMemcpyHostToDevice, true);
        } else {
            double inf[3];
            rc = eng.init_state(id, q.init, inf);
        }
        if (!rc) rc = eng.set_cfl(id, q.cfl);
        r.reynolds = eng.reynolds(id);
        r.remaining = q.nsteps;
        r.t_admit = now();
        return rc;
    }

    int retire(Engine &eng, Resident &r) {
        int rc = eng.sync_and_check(r.box);
        bool want = true;
        for (int e = 0; e < 5; ++e) want = want && r.q.req.h_q_out[e] != nullptr;
        if (!rc && want) rc = eng.get_state(r.box, r.q.req.h_q_out, cudaMemcpyDeviceToHost, true);
        return rc;
    }

    void run() {
        cudaSetDevice(device_);
        cudaStream_t st = nullptr;
        Engine *eng = nullptr;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
                start_rc_ = NUC3D_ERR_CUDA;
                start_err_ = "stream creation failed";
            } else {
                eng = new Engine(cfg_.precision, st);
            }
            started_ = true;
        }
        started_cv_.notify_all();
        if (!eng) return;
        std::vector<Resident> res;
        long long used = 0;
        // device milliseconds per resident cell and step, from the last chunk:
        // predicts the step time of any composition (0: nothing measured yet)
        double ms_per_cell_step = 0.0;
        for (;;) {
            std::vector<Queued> adm;
            bool stopping;
            {
                std::unique_lock<std::mutex> lk(mu_);
                if (res.empty()) cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
                stopping = stop_;
                while (!stopping && !queue_.empty() &&
                       (int)(res.size() + adm.size()) < cfg_.max_resident &&
                       used + queue_.front().bytes <= cfg_.budget_bytes) {
                    used += queue_.front().bytes;
                    adm.push_back(queue_.front());
                    queue_.pop_front();
                }
            }
            if (stopping) break;
            for (Queued &q : adm) {
                Resident r;
                r.q = q;
                int rc = admit(*eng, r);
                if (rc) {
                    post(r, rc, nuc3d_last_error(), nullptr);
                    if (r.box >= 0) eng->remove_box(r.box);
                    used -= q.bytes;
                    continue;
                }
                if (r.remaining == 0) {
                    rc = retire(*eng, r);
                    post(r, rc, rc ? nuc3d_last_error() : nullptr, eng);
                    eng->remove_box(r.box);
                    used -= q.bytes;
                    continue;
                }
                res.push_back(r);
            }
            if (!adm.empty()) {
                std::lock_guard<std::mutex> lk(mu_);
                info_.resident = (int)res.size();
                info_.resident_bytes = used;
                info_.peak_resident = std::max(info_.peak_resident, (int)res.size());
                info_.peak_resident_bytes = std::max(info_.peak_resident_bytes, used);
            }
            if (res.empty()) continue;
            long long chunk = cfg_.max_chunk_steps;
            double cells = 0.0;
            for (const Resident &r : res) {
                chunk = std::min(chunk, r.remaining);
                cells += (double)r.q.req.desc.nx * r.q.req.desc.ny * r.q.req.desc.nz;
            }
            if (ms_per_cell_step > 0.0)
                chunk = std::max(1LL, std::min(chunk, (long long)(cfg_.chunk_ms /
                                                                  (ms_per_cell_step * cells))));
            else
                chunk = 1;  // nothing measured yet
            const double t_a = now();
            int rc = eng->step((int)chunk);
            if (!rc) {
                const cudaError_t se = cudaStreamSynchronize(st);
                if (se != cudaSuccess) rc = set_last_error(NUC3D_ERR_CUDA, cudaGetErrorString(se));
            }
            const double dt_chunk = now() - t_a;
            if (rc) {
                // a failed step leaves every resident solve undefined
                const char *msg = nuc3d_last_error();
                for (Resident &r : res) {
                    post(r, rc, msg, nullptr);
                    eng->remove_box(r.box);
                }
                res.clear();
                used = 0;
            } else {
                ms_per_cell_step = 1e3 * dt_chunk / ((double)chunk * cells);
                std::vector<Resident> keep;
                for (Resident &r : res) {
                    r.remaining -= chunk;
                    if (r.remaining > 0) {
                        keep.push_back(r);
                        continue;
                    }
                    int rrc = retire(*eng, r);
                    post(r, rrc, rrc ? nuc3d_last_error() : nullptr, eng);
                    eng->remove_box(r.box);
                    used -= r.q.bytes;
                }
                res.swap(keep);
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                info_.batch_steps += chunk;
                info_.chunks += 1;
                info_.busy_s += dt_chunk;
                info_.resident = (int)res.size();
                info_.resident_bytes = used;
                info_.launches = eng->launches;
                info_.graph_captures = eng->graph_captures;
            }
        }
        // shutting down: cancel what is resident and queued
        for (Resident &r : res) post(r, NUC3D_ERR_CANCELLED, "server destroyed", nullptr);
        std::deque<Queued> rest;
        {
            std::lock_guard<std::mutex> lk(mu_);
            rest.swap(queue_);
        }
        for (Queued &q : rest) {
            Resident r;
            r.q = q;
            post(r, NUC3D_ERR_CANCELLED, "server destroyed", nullptr);
        }
        delete eng;
        cudaStreamDestroy(st);
    }

    nuc3d_serve_config cfg_;
    Clock::time_point t0_;
    int device_ = 0;
    std::thread worker_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_, started_cv_;
    bool started_ = false, stop_ = false;
    int start_rc_ = NUC3D_OK;
    std::string start_err_;
    std::deque<Queued> queue_;
    std::map<long long, nuc3d_solve_result> done_;
    std::deque<long long> done_order_;
    std::set<long long> outstanding_;
    long long next_ticket_ = 0, submitted_ = 0;
    nuc3d_serve_stats info_{};
};

}  // namespace nuc3d

struct nuc3d_server {
    nuc3d::Server *srv;
};

extern "C" {

void nuc3d_serve_config_default(nuc3d_serve_config *c) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->precision = NUC3D_MIXED;
    c->budget_bytes = 0;
    c->max_resident = 256;
    c->max_chunk_steps = 64;
    c->chunk_ms = 20.0;
}

int nuc3d_serve_create(const nuc3d_serve_config *cfg, nuc3d_server **out) {
    if (!cfg || !out) return nuc3d::set_last_error(NUC3D_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->precision != NUC3D_FP64 && cfg->precision != NUC3D_MIXED)
        return nuc3d::set_last_error(NUC3D_ERR_UNSUPPORTED, "unknown precision");
    auto *s = new (std::nothrow) nuc3d::Server(*cfg);
    auto *h = new (std::nothrow) nuc3d_server{s};
    if (!s || !h) {
        delete s;
        delete h;
        return nuc3d::set_last_error(NUC3D_ERR_NOMEM, "host allocation failed");
    }
    int rc = s->start();
    if (rc) {
        delete s;
        delete h;
        return rc;
    }
    *out = h;
    return NUC3D_OK;
}

int nuc3d_serve_destroy(nuc3d_server *s) {
    if (!s) return NUC3D_OK;
    delete s->srv;
    delete s;
    return NUC3D_OK;
}

int nuc3d_serve_submit(nuc3d_server *s, const nuc3d_solve_request *req, long long *ticket) {
    if (!s || !req || !ticket) return nuc3d::set_last_error(NUC3D_ERR_INVALID, "null argument");
    return s->srv->submit(*req, ticket);
}

int nuc3d_serve_wait(nuc3d_server *s, long long ticket, double timeout_s, nuc3d_solve_result *out) {
    if (!s || !out) return nuc3d::set_last_error(NUC3D_ERR_INVALID, "null argument");
    return s->srv->wait(ticket, timeout_s, out);
}

int nuc3d_serve_info(nuc3d_server *s, nuc3d_serve_stats *out) {
    if (!s || !out) return nuc3d::set_last_error(NUC3D_ERR_INVALID, "null argument");
    s->srv->info(out);
    return NUC3D_OK;
}

}  // extern "C"
