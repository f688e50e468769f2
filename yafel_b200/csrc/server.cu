// server.cu -- a continuous-batching solve server on one context.
//
// No reference counterpart: the reference solves one system per call.  Requests
// arrive with an estimate of the device bytes they need; the server admits them
// in arrival order while the admitted ones fit in its HBM budget (the head of
// the queue waits for room, so no request starves), the client builds each
// admitted system on the device (assembly, boundary conditions) and attaches
// it, and every attached system advances in the shared batch (batch.cu: one
// persistent launch per step of every iteration, PCG and BiCGSTAB together).
// A launch runs one block of iterations without blocking the host, which
// builds the next admitted systems meanwhile (yg_server_ready says, without
// blocking, whether the block is done; building on a second context of the
// device keeps the builds off the batch's stream); the following wait retires
// the systems that finished, whose results the client then reads and releases.
// Inside the batch, systems with a large matrix run their iteration SpMV as
// their own single-system launch (yg_server_set_solo_spmv_bytes).  Systems of
// at least `solo_rows` rows (when set; off by default) skip the batch instead
// and are solved one at a time by the single-system solvers, one per wait,
// before the wait for the block in flight (so the two overlap when the
// system's context has its own stream).
#include "internal.h"

#include <deque>
#include <unordered_map>
#include <vector>

namespace {

enum ReqState { RQ_QUEUED = 0, RQ_ADMITTED = 1, RQ_RUNNING = 2, RQ_DONE = 3 };

struct Request {
    uint64_t bytes = 0;  // estimate while queued / admitted, then the attached system's bytes
    int state = RQ_QUEUED;
    int32_t slot = -1;
    yg_solve_stats stats{};
    // a system solved alone
    yg_matrix A = nullptr;
    yg_vector b = nullptr, x = nullptr;
    int32_t method = 0;
    yg_solve_opts opts{};
};

uint64_t matrix_bytes(yg_matrix A) {
    const uint64_t b2 = (uint64_t)A->block * A->block;
    uint64_t n = (uint64_t)A->nnzb * (b2 * 8 + 4) + 4 * ((uint64_t)A->nbrows + 1) + 4 * (uint64_t)A->nbrows;
    if (A->d_val32) n += (uint64_t)A->nnzb * b2 * 4;
    return n;
}

}  // namespace

struct yg_server_t {
    yg_context ctx = nullptr;
    yg_batch batch = nullptr;
    uint64_t budget = 0, held = 0;
    int32_t capacity = 0, attached = 0;
    int64_t next_id = 0;
    bool in_flight = false;
    std::deque<int64_t> queue;
    std::unordered_map<int64_t, Request> reqs;
    std::vector<int64_t> slot_req;   // request of each batch slot, -1 when free
    std::vector<int64_t> finished;   // retired since the last yg_server_finished
    int64_t solo_rows = 0;           // 0: every system goes to the batch
    std::deque<int64_t> solo;        // attached systems solved alone, in order
};

using namespace yg;

extern "C" yg_status yg_server_create(yg_context ctx, uint64_t budget_bytes, int32_t max_active, yg_server *out) {
    if (!ctx || !out || max_active < 1 || budget_bytes == 0) return fail(YG_BAD_ARG, "yg_server_create: bad argument");
    auto *S = new yg_server_t();
    S->ctx = ctx;
    S->budget = budget_bytes;
    S->capacity = max_active;
    S->slot_req.assign(max_active, -1);
    yg_status st = yg_batch_create(ctx, max_active, &S->batch);
    if (st != YG_OK) {
        delete S;
        return st;
    }
    *out = S;
    return YG_OK;
}

extern "C" yg_status yg_server_destroy(yg_server S) {
    if (!S) return YG_OK;
    yg_batch_destroy(S->batch);
    delete S;
    return YG_OK;
}

extern "C" yg_status yg_server_submit(yg_server S, uint64_t bytes, int64_t *id) {
    if (!S || !id) return fail(YG_BAD_ARG, "yg_server_submit: NULL argument");
    if (bytes > S->budget)
        return fail(YG_OVER_BUDGET, "yg_server_submit: request needs %llu bytes, the budget is %llu",
                    (unsigned long long)bytes, (unsigned long long)S->budget);
    const int64_t r = S->next_id++;
    Request q;
    q.bytes = bytes;
    S->reqs[r] = q;
    S->queue.push_back(r);
    *id = r;
    return YG_OK;
}

extern "C" yg_status yg_server_admit(yg_server S, int64_t *id) {
    if (!S || !id) return fail(YG_BAD_ARG, "yg_server_admit: NULL argument");
    *id = -1;
    if (S->queue.empty()) return YG_OK;
    int admitted = 0;
    for (auto &kv : S->reqs)
        if (kv.second.state == RQ_ADMITTED) ++admitted;
    if (S->attached + admitted >= S->capacity) return YG_OK;  // no batch slot for it
    Request &q = S->reqs[S->queue.front()];
    if (S->held + q.bytes > S->budget) return YG_OK;  // the head waits for room
    *id = S->queue.front();
    S->queue.pop_front();
    q.state = RQ_ADMITTED;
    S->held += q.bytes;
    return YG_OK;
}

extern "C" yg_status yg_server_attach(yg_server S, int64_t id, yg_matrix A, yg_vector b, yg_vector x, int32_t method,
                                      const yg_solve_opts *opts) {
    if (!S || !A || !b || !x) return fail(YG_BAD_ARG, "yg_server_attach: NULL argument");
    auto it = S->reqs.find(id);
    if (it == S->reqs.end() || it->second.state != RQ_ADMITTED)
        return fail(YG_BAD_ARG, "yg_server_attach: request %lld is not admitted", (long long)id);
    if (S->in_flight) return fail(YG_BAD_ARG, "yg_server_attach: a block is in flight; attach after yg_server_wait");
    if (S->solo_rows > 0 && A->rows() >= S->solo_rows) {
        Request &q = it->second;
        const uint64_t actual = matrix_bytes(A) + 16 * (uint64_t)A->rows() + (uint64_t)yg_batch_work_bytes(A->rows(), method);
        S->held = S->held - q.bytes + actual;
        q.bytes = actual;
        q.state = RQ_RUNNING;
        q.A = A;
        q.b = b;
        q.x = x;
        q.method = method;
        q.opts = opts ? *opts : yg_solve_opts{YG_CRIT_RELRES, YG_PREC_FP64, 1e-10, 0, 0, 0};
        q.opts.criterion = YG_CRIT_RELRES;
        if (method == YG_METHOD_BICGSTAB) q.opts.precision = YG_PREC_FP64;  // the single-system BiCGSTAB is FP64
        S->solo.push_back(id);
        return YG_OK;
    }
    int32_t slot = -1;
    YG_TRY(yg_batch_add(S->batch, A, b, x, method, opts, &slot));
    Request &q = it->second;
    const uint64_t actual = matrix_bytes(A) + 16 * (uint64_t)A->rows() + (uint64_t)yg_batch_work_bytes(A->rows(), method);
    S->held = S->held - q.bytes + actual;
    q.bytes = actual;
    q.state = RQ_RUNNING;
    q.slot = slot;
    S->slot_req[slot] = id;
    ++S->attached;
    return YG_OK;
}

extern "C" yg_status yg_server_launch(yg_server S) {
    if (!S) return fail(YG_BAD_ARG, "yg_server_launch: NULL server");
    if (S->in_flight) return fail(YG_BAD_ARG, "yg_server_launch: a block is already in flight");
    if (S->attached == 0) return YG_OK;
    YG_TRY(yg_batch_launch(S->batch));
    S->in_flight = true;
    return YG_OK;
}

// One system of the solo queue solved alone by the single-system solvers (on
// its matrix's context: with the requests built on the server's second context
// this solve runs beside a block in flight on the batch's stream).
static yg_status solve_one_solo(yg_server S, int32_t *done) {
    if (S->solo.empty()) return YG_OK;
    const int64_t r = S->solo.front();
    S->solo.pop_front();
    Request &q = S->reqs[r];
    yg_precond M = nullptr;
    YG_TRY(yg_precond_create(q.A, YG_PRECOND_JACOBI, &M));
    yg_solve_stats st{};
    yg_status e = q.method == YG_METHOD_BICGSTAB ? yg_bicgstab(q.A, M, q.b, q.x, &q.opts, &st)
                                                  : yg_cg(q.A, M, q.b, q.x, &q.opts, &st);
    yg_precond_destroy(M);
    if (e != YG_OK && e != YG_NOT_CONVERGED && e != YG_BREAKDOWN && e != YG_NAN) return e;
    q.stats = st;
    q.state = RQ_DONE;
    q.A = nullptr;
    q.b = q.x = nullptr;
    S->finished.push_back(r);
    ++*done;
    return YG_OK;
}

extern "C" yg_status yg_server_wait(yg_server S, int32_t *n_finished) {
    if (!S) return fail(YG_BAD_ARG, "yg_server_wait: NULL server");
    int32_t done = 0;
    // one system solved alone per wait, while the block (if any) is still running
    YG_TRY(solve_one_solo(S, &done));
    if (S->in_flight) {
        S->in_flight = false;
        int32_t active = 0;
        YG_TRY(yg_batch_wait(S->batch, &active));
        for (int32_t s = 0; s < S->capacity; ++s) {
            const int64_t r = S->slot_req[s];
            if (r < 0 || batch_slot_running(S->batch, s)) continue;
            Request &q = S->reqs[r];
            batch_slot_stats(S->batch, s, &q.stats);
            YG_TRY(yg_batch_remove(S->batch, s));
            S->slot_req[s] = -1;
            q.slot = -1;
            q.state = RQ_DONE;
            --S->attached;
            S->finished.push_back(r);
            ++done;
        }
    }
    if (n_finished) *n_finished = done;
    return YG_OK;
}

extern "C" yg_status yg_server_ready(yg_server S, int32_t *ready) {
    if (!S || !ready) return fail(YG_BAD_ARG, "yg_server_ready: NULL argument");
    *ready = 1;
    if (!S->in_flight) return YG_OK;
    return yg_batch_ready(S->batch, ready);
}

extern "C" yg_status yg_server_set_solo_spmv_bytes(yg_server S, int64_t bytes) {
    if (!S) return fail(YG_BAD_ARG, "yg_server_set_solo_spmv_bytes: NULL server");
    return yg_batch_set_solo_bytes(S->batch, bytes);
}

extern "C" yg_status yg_server_set_solo_rows(yg_server S, int64_t rows) {
    if (!S || rows < 0) return fail(YG_BAD_ARG, "yg_server_set_solo_rows: bad argument");
    S->solo_rows = rows;
    return YG_OK;
}

extern "C" yg_status yg_server_finished(yg_server S, int64_t *ids, int32_t cap, int32_t *n) {
    if (!S || !n || (cap > 0 && !ids)) return fail(YG_BAD_ARG, "yg_server_finished: bad argument");
    const int32_t k = (int32_t)std::min<size_t>(S->finished.size(), (size_t)std::max(cap, 0));
    for (int32_t i = 0; i < k; ++i) ids[i] = S->finished[i];
    S->finished.erase(S->finished.begin(), S->finished.begin() + k);
    *n = k;
    return YG_OK;
}

extern "C" yg_status yg_server_poll(yg_server S, int64_t id, yg_solve_stats *stats) {
    if (!S || !stats) return fail(YG_BAD_ARG, "yg_server_poll: NULL argument");
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return fail(YG_BAD_ARG, "yg_server_poll: unknown request %lld", (long long)id);
    if (it->second.state == RQ_DONE) {
        *stats = it->second.stats;
    } else {
        *stats = yg_solve_stats{};
        stats->status = YG_RUNNING;
    }
    return YG_OK;
}

extern "C" yg_status yg_server_release(yg_server S, int64_t id) {
    if (!S) return fail(YG_BAD_ARG, "yg_server_release: NULL server");
    auto it = S->reqs.find(id);
    if (it == S->reqs.end() || it->second.state != RQ_DONE)
        return fail(YG_BAD_ARG, "yg_server_release: request %lld has not finished", (long long)id);
    S->held -= it->second.bytes;
    S->reqs.erase(it);
    return YG_OK;
}

extern "C" yg_status yg_server_info(yg_server S, int64_t *queued, int64_t *active, uint64_t *bytes_held) {
    if (!S) return fail(YG_BAD_ARG, "yg_server_info: NULL server");
    if (queued) *queued = (int64_t)S->queue.size();
    if (active) *active = S->attached + (int64_t)S->solo.size();
    if (bytes_held) *bytes_held = S->held;
    return YG_OK;
}

extern "C" yg_status yg_server_tune(yg_server S) {
    if (!S) return fail(YG_BAD_ARG, "yg_server_tune: NULL server");
    if (S->in_flight) return fail(YG_BAD_ARG, "yg_server_tune: a block is in flight; tune after yg_server_wait");
    if (S->attached == 0) return YG_OK;
    return yg_batch_tune(S->batch);
}
