// admission.h - the request server's admission rule (pure host code, no CUDA),
// shared by server.cu and the CPU test of the rule (tests/admission_check.cpp).
//
// A server holds `pending` (a deque of shared request pointers, oldest first),
// `workers` (unique worker pointers) and `budget` (device bytes). A request
// has `bytes` (its device footprint), `small` and `bypassed`; a worker has
// `committed` (device bytes held or promised), `ctx_held` and `batch_held`
// (what its two workspaces hold between runs), `drop_ctx`, `drop_batch`,
// `busy`, `releasing` and `small_only`. The server's lock is held by the
// caller of every function here.
#pragma once

#include <algorithm>
#include <memory>
#include <vector>

namespace unc_admission {

constexpr int kMaxBypass = 16;  // later requests may start ahead of a waiting one this many times
constexpr int kMaxPack = 64;    // small requests run together as one grouped batch

template <class Server, class Worker>
long long committed_except(const Server* s, const Worker* w) {
    long long t = 0;
    for (auto& v : s->workers)
        if (v.get() != w) t += v->committed;
    return t;
}

// Device bytes worker w holds while it runs `need` bytes of work as a single
// request (pack false: the context's workspace grows to it) or as a pack (the
// batch's grows), with the other workspace kept or freed first (drop_other).
template <class Worker>
long long holds(const Worker* w, long long need, bool pack, bool drop_other) {
    const long long same = pack ? w->batch_held : w->ctx_held, other = pack ? w->ctx_held : w->batch_held;
    return std::max(same, need) + (drop_other ? 0 : other);
}

// The requests worker `w` may start now (empty: none). A small request takes
// the small requests waiting behind it along (a pack) as long as their
// footprints fit. Idle workers whose workspaces must go to make room are
// returned in `release` (marked, their bytes no longer counted): the caller
// frees them after unlocking, before its own allocations, so that no CUDA call
// runs under the lock. w->drop_ctx / w->drop_batch tell the caller to free
// w's own workspace of the other kind before the run; w->committed becomes
// what w holds during the run.
template <class Server, class Worker>
auto pick(Server* s, Worker* w, std::vector<Worker*>& release) -> std::vector<typename decltype(s->pending)::value_type> {
    std::vector<typename decltype(s->pending)::value_type> pack;
    release.clear();
    if (w->releasing) return pack;
    for (size_t i = 0; i < s->pending.size(); ++i) {
        const auto r = s->pending[i];  // a copy: the queue slot is erased below
        if (w->small_only && !r->small) continue;  // not this worker's kind; no bypass counted
        // as a single request: this worker's batch workspace stays, unless freeing it makes room
        const long long others = committed_except(s, w);
        bool drop = false;
        bool fits = others + holds(w, r->bytes, false, false) <= s->budget;
        if (!fits && others + holds(w, r->bytes, false, true) <= s->budget) fits = drop = true;
        if (!fits) {
            // count idle workspaces (not this worker's) as released and look again
            long long idle = 0;
            for (auto& v : s->workers)
                if (v.get() != w && !v->busy && !v->releasing) idle += v->committed;
            fits = others - idle + holds(w, r->bytes, false, true) <= s->budget;
            if (fits) {
                drop = others - idle + holds(w, r->bytes, false, false) > s->budget;
                for (auto& v : s->workers)
                    if (v.get() != w && !v->busy && !v->releasing && v->committed > 0) {
                        v->releasing = true;
                        v->committed = v->ctx_held = v->batch_held = 0;
                        release.push_back(v.get());
                    }
            }
        }
        if (!fits) {
            if (r->bypassed >= kMaxBypass) break;  // the head waits for memory; nobody overtakes it any more
            continue;
        }
        for (size_t j = 0; j < i; ++j)
            if (!w->small_only || s->pending[j]->small) s->pending[j]->bypassed++;
        pack.push_back(r);
        s->pending.erase(s->pending.begin() + (long)i);
        long long sum = r->bytes;
        bool pdrop = false;  // the pack needs this worker's context workspace freed
        if (r->small) {
            for (size_t j = i; j < s->pending.size() && (int)pack.size() < kMaxPack;) {
                const auto q = s->pending[j];
                const long long base = committed_except(s, w);
                bool take = q->small && base + holds(w, sum + q->bytes, true, pdrop) <= s->budget;
                if (!take && q->small && !pdrop && base + holds(w, sum + q->bytes, true, true) <= s->budget)
                    take = pdrop = true;
                if (take) {
                    sum += q->bytes;
                    pack.push_back(q);
                    s->pending.erase(s->pending.begin() + (long)j);
                } else {
                    ++j;
                }
            }
        }
        const bool as_pack = pack.size() > 1;
        w->drop_ctx = as_pack && pdrop;
        w->drop_batch = !as_pack && drop;
        w->committed = as_pack ? holds(w, sum, true, pdrop) : holds(w, r->bytes, false, drop);
        return pack;
    }
    return pack;
}

// After a run: what the workspaces now hold (ctx_bytes, batch_bytes) becomes
// the worker's commitment.
template <class Worker>
void settle(Worker* w, long long ctx_bytes, long long batch_bytes) {
    w->ctx_held = ctx_bytes;
    w->batch_held = batch_bytes;
    w->committed = ctx_bytes + batch_bytes;
    w->drop_ctx = w->drop_batch = false;
}

}  // namespace unc_admission
