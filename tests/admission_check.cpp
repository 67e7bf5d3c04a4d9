// CPU check of the request server's admission rule (uncertaintyte_b200/csrc/admission.h):
// a seeded simulation of workers taking requests of random sizes under a
// device-memory budget. The simulated workers hold two workspaces the way the
// server's do (a single request grows the context's, a pack the batch's; each
// keeps its memory after the run; a drop flag frees one before the run; a
// released idle worker loses both). Checked after every step:
//   * the bytes all workers really hold or use stay within the budget;
//   * each worker's commitment equals what it really holds or uses;
//   * every request is admitted once and all finish.
// Built with -fsanitize=address,undefined by tests/test_admission.py.
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <memory>
#include <random>
#include <set>
#include <vector>

#include "admission.h"

struct Request {
    long long id = 0;
    long long bytes = 0;
    bool small = false;
    int bypassed = 0;
};

struct Worker {
    long long committed = 0, ctx_held = 0, batch_held = 0;
    bool drop_ctx = false, drop_batch = false, busy = false, releasing = false, small_only = false;
    // simulation state: what the workspaces hold while running
    long long run_ctx = 0, run_batch = 0;
    std::vector<std::shared_ptr<Request>> running;
};

struct Server {
    std::deque<std::shared_ptr<Request>> pending;
    std::vector<std::unique_ptr<Worker>> workers;
    long long budget = 0;
};

static int fails = 0;
#define CHECK(c, ...)                        \
    do {                                     \
        if (!(c)) {                          \
            std::printf("FAIL: " __VA_ARGS__); \
            std::printf("\n");               \
            ++fails;                         \
        }                                    \
    } while (0)

static long long real_bytes(const Worker& w) {
    return w.busy ? w.run_ctx + w.run_batch : w.ctx_held + w.batch_held;
}

static void run_case(unsigned seed, int nworkers, long long budget, int nreq) {
    std::mt19937_64 rng(seed);
    Server s;
    s.budget = budget;
    for (int i = 0; i < nworkers; ++i) {
        s.workers.push_back(std::make_unique<Worker>());
        s.workers.back()->small_only = i < nworkers / 4;
    }
    const long long small_max = budget / 6;
    std::uniform_real_distribution<double> u(0.0, 1.0);
    long long next_id = 1, submitted = 0;
    std::set<long long> admitted, finished;
    for (int step = 0; step < 200000 && (long long)finished.size() < nreq; ++step) {
        const double a = u(rng);
        if (a < 0.35 && submitted < nreq) {  // a request arrives
            auto r = std::make_shared<Request>();
            r->id = next_id++;
            // sizes from a few KB to the whole budget, most of them small
            const double x = u(rng);
            r->bytes = x < 0.7 ? (long long)(1 + u(rng) * small_max) : (long long)(small_max + u(rng) * (budget - small_max));
            r->small = r->bytes <= small_max;
            s.pending.push_back(r);
            ++submitted;
        } else if (a < 0.75) {  // an idle worker looks for work
            Worker* w = s.workers[rng() % s.workers.size()].get();
            if (w->busy || w->releasing) continue;
            std::vector<Worker*> release;
            auto pack = unc_admission::pick(&s, w, release);
            for (Worker* v : release) {  // the picking worker frees their workspaces
                CHECK(!v->busy, "released a busy worker");
                v->releasing = false;
            }
            if (pack.empty()) continue;
            for (auto& r : pack) {
                CHECK(admitted.insert(r->id).second, "request %lld admitted twice", r->id);
                if (pack.size() > 1) CHECK(r->small, "a large request in a pack");
            }
            // the run: drop first, then grow the workspace of this kind
            long long ctx = w->drop_ctx ? 0 : w->ctx_held, batch = w->drop_batch ? 0 : w->batch_held;
            long long need = 0;
            for (auto& r : pack) need += r->bytes;
            if (pack.size() > 1) batch = std::max(batch, need);
            else ctx = std::max(ctx, need);
            w->run_ctx = ctx;
            w->run_batch = batch;
            w->busy = true;
            w->running = pack;
            CHECK(w->committed == ctx + batch, "commitment %lld != held %lld", w->committed, ctx + batch);
        } else {  // a busy worker finishes
            Worker* w = s.workers[rng() % s.workers.size()].get();
            if (!w->busy) continue;
            for (auto& r : w->running) finished.insert(r->id);
            w->running.clear();
            w->busy = false;
            unc_admission::settle(w, w->run_ctx, w->run_batch);
        }
        long long total = 0;
        for (auto& v : s.workers) total += real_bytes(*v);
        CHECK(total <= budget, "seed %u step %d: %lld bytes held, budget %lld", seed, step, total, budget);
        if (fails > 20) return;
    }
    CHECK((long long)finished.size() == nreq, "seed %u: %zu of %d requests finished", seed, finished.size(), nreq);
}

int main() {
    for (unsigned seed = 1; seed <= 40; ++seed)
        run_case(seed, 1 + (int)(seed % 8), (1LL << 30) * (1 + seed % 5), 300);
    if (fails) {
        std::printf("%d failures\n", fails);
        return 1;
    }
    std::printf("admission ok\n");
    return 0;
}
