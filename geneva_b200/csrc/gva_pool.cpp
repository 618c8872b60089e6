// Host worker pool (gva_pool.h): a fixed set of threads, created on first
// use, taking indices of posted jobs from a shared list.
#include "gva_pool.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

namespace gva {
namespace {

struct Job {
    const std::function<void(unsigned)>* fn;
    unsigned n;
    std::atomic<unsigned> next{0};  // next index to hand out
    unsigned done = 0;              // indices finished (under the pool mutex)
    unsigned users = 0;             // workers holding the job (under the pool mutex)
};

class Pool {
public:
    Pool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        width_ = std::min(64u, hw);
        for (unsigned i = 0; i + 1 < width_; ++i) workers_.emplace_back([this]() { work(); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        for (auto& th : workers_) th.join();
    }
    unsigned width() const { return width_; }

    void run(unsigned n, const std::function<void(unsigned)>& fn) {
        if (n == 0) return;
        if (n == 1 || workers_.empty()) {
            for (unsigned t = 0; t < n; ++t) fn(t);
            return;
        }
        Job job;
        job.fn = &fn;
        job.n = n;
        {
            std::lock_guard<std::mutex> lk(mu_);
            jobs_.push_back(&job);
        }
        if (n - 1 >= workers_.size())
            cv_work_.notify_all();
        else
            for (unsigned i = 0; i + 1 < n; ++i) cv_work_.notify_one();
        unsigned mine = 0;
        for (unsigned t; (t = job.next.fetch_add(1)) < n;) {
            fn(t);
            ++mine;
        }
        std::unique_lock<std::mutex> lk(mu_);
        job.done += mine;
        drop(&job);
        cv_done_.wait(lk, [&]() { return job.done == job.n && job.users == 0; });
    }

private:
    // removes a job whose indices are all handed out from the list
    void drop(Job* j) {
        auto it = std::find(jobs_.begin(), jobs_.end(), j);
        if (it != jobs_.end()) jobs_.erase(it);
    }

    void work() {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_work_.wait(lk, [&]() { return stop_ || !jobs_.empty(); });
            if (stop_) return;
            Job* j = jobs_.front();
            if (j->next.load() >= j->n) {  // fully handed out: no longer offered
                drop(j);
                continue;
            }
            ++j->users;
            lk.unlock();
            unsigned mine = 0;
            for (unsigned t; (t = j->next.fetch_add(1)) < j->n;) {
                (*j->fn)(t);
                ++mine;
            }
            lk.lock();
            j->done += mine;
            --j->users;
            drop(j);
            if (j->done == j->n && j->users == 0) cv_done_.notify_all();
        }
    }

    unsigned width_ = 1;
    std::vector<std::thread> workers_;
    std::vector<Job*> jobs_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    bool stop_ = false;
};

Pool& pool() {
    static Pool p;
    return p;
}

// One background thread running deferred work in order.
class Deferred {
public:
    Deferred() : th_([this]() { work(); }) {}
    ~Deferred() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        th_.join();
    }
    void post(std::function<void()> fn) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            q_.push_back(std::move(fn));
        }
        cv_.notify_one();
    }

private:
    void work() {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            cv_.wait(lk, [&]() { return stop_ || !q_.empty(); });
            if (q_.empty()) return;  // stopping with nothing left
            std::function<void()> fn = std::move(q_.front());
            q_.pop_front();
            lk.unlock();
            fn();
            fn = nullptr;  // what it captured is released off the lock too
            lk.lock();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> q_;
    bool stop_ = false;
    std::thread th_;
};

}  // namespace

void pool_run(unsigned n, const std::function<void(unsigned)>& fn) { pool().run(n, fn); }

unsigned pool_width() { return pool().width(); }

void defer(std::function<void()> fn) {
    static Deferred d;
    d.post(std::move(fn));
}

}  // namespace gva
