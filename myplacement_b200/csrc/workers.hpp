// A fork-join helper for host-side loops: run(count, body) calls body(i) for
// every i in [0, count) on up to `threads` host threads (the caller's among
// them), handing out indices from a shared counter; the first exception a body
// throws is rethrown after every thread has stopped.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstddef>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

namespace mpgp {

class Workers {
public:
    explicit Workers(int threads) : threads_(std::max(1, threads)) {}

    // One per hardware thread, at most `cap`: a fork-join region costs a thread
    // start per helper, and large hosts have hundreds of hardware threads.
    static Workers all(unsigned cap) {
        return Workers(static_cast<int>(std::min(cap, std::max(1u, std::thread::hardware_concurrency()))));
    }

    [[nodiscard]] int threads() const { return threads_; }

    template <typename F>
    void run(std::size_t count, const F& body) const {
        const std::size_t helpers = std::min<std::size_t>(static_cast<std::size_t>(threads_), count);
        if (helpers <= 1) {
            for (std::size_t i = 0; i < count; ++i) body(i);
            return;
        }
        std::atomic<std::size_t> next{0};
        std::exception_ptr error;
        std::mutex lock;
        const auto work = [&] {
            try {
                for (std::size_t i; (i = next.fetch_add(1)) < count;) body(i);
            } catch (...) {
                const std::lock_guard<std::mutex> guard(lock);
                if (!error) error = std::current_exception();
                next.store(count);
            }
        };
        std::vector<std::thread> pool;
        pool.reserve(helpers - 1);
        try {
            for (std::size_t t = 1; t < helpers; ++t) pool.emplace_back(work);
        } catch (...) {
            next.store(count);
            for (std::thread& thread : pool) thread.join();
            throw;
        }
        work();
        for (std::thread& thread : pool) thread.join();
        if (error) std::rethrow_exception(error);
    }

    // body(begin, end) over [0, count) in blocks of `block`.
    template <typename F>
    void blocks(std::size_t count, std::size_t block, const F& body) const {
        run((count + block - 1) / block, [&](std::size_t b) { body(b * block, std::min(count, (b + 1) * block)); });
    }

private:
    int threads_;
};

}  // namespace mpgp
