// NxStereo.CudaNif: the NIF that NxStereo.CudaSegment calls, a thin layer
// over the C ABI of libnxs_b200 (include/nx_stereo_b200.h). It takes the
// very records the reference's NativeSegment sends its Port (configure, run;
// native/stereo_match/src/protocol.rs), decoded by port_records.h, and
// answers each run by a message to the caller, as NxStereo.Matcher does:
//
//   open(device)                                  -> {:ok, context} | {:error, reason}
//   configure(context, record)                    -> :ok | {:error, reason}
//   run(context, record, pid, ref, timeout_ms)    -> :ok | {:error, reason}
//       later, to pid: {ref, {:ok, outputs_record}} | {ref, {:error, reason}}
//   watch(context, owner, segment)                -> :ok
//   release(context, segment)                     -> :ok
//
// No call blocks a scheduler on the device: a configure allocates device
// memory (a dirty CPU call), a run only enqueues its copies and kernels. A
// thread of the context waits for the runs in the order sent and replies to
// each with the outputs record (tag 8 ...) or an error. A run without a reply
// within its timeout_ms fails with :timeout, and so does every run sent after
// it that is still waiting, as the Matcher fails every request waiting when a
// reply is late (lib/nx_stereo/matcher.ex:107-146); the device finishes them
// and their outputs are dropped. `watch` releases the segment once the owner
// process exits (matcher.ex:148-160).
#include <erl_nif.h>

#include <ctime>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../nx_stereo_b200/csrc/port_records.h"

namespace {

struct Pending {
    nxs_request *request;
    ErlNifPid pid;
    ErlNifEnv *env;  // holds the copy of the caller's ref
    ERL_NIF_TERM ref;
    uint64_t deadline_ns;  // CLOCK_MONOTONIC, the clock of nxs_request_done_ns
};

uint64_t monotonic_ns() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (uint64_t)t.tv_sec * 1000000000ull + (uint64_t)t.tv_nsec;
}

struct Context {
    nxs_context *context = nullptr;
    std::mutex lock;
    std::condition_variable wake;
    std::deque<Pending> pending;
    bool stopping = false;
    std::thread waiter;
};

struct ContextRef {  // the resource: a context's handle in Erlang terms
    Context *ctx;
};

struct Watch {  // the resource monitoring an owner: its segments
    Context *ctx;
    std::set<uint32_t> segments;
    std::mutex lock;
};

ErlNifResourceType *CONTEXT = nullptr, *WATCH = nullptr;
std::mutex watches_lock;
std::map<std::pair<Context *, std::string>, Watch *> watches;  // by context and owner pid

ERL_NIF_TERM atom(ErlNifEnv *env, const char *name) { return enif_make_atom(env, name); }

ERL_NIF_TERM text(ErlNifEnv *env, const std::string &s) {
    ERL_NIF_TERM term;
    unsigned char *data = enif_make_new_binary(env, s.size(), &term);
    std::memcpy(data, s.data(), s.size());
    return term;
}

ERL_NIF_TERM error(ErlNifEnv *env, ERL_NIF_TERM reason) {
    return enif_make_tuple2(env, atom(env, "error"), reason);
}

void reply(const Pending &p, ERL_NIF_TERM (*make)(ErlNifEnv *, void *), void *arg) {
    ErlNifEnv *msg = enif_alloc_env();
    ERL_NIF_TERM ref = enif_make_copy(msg, p.ref);
    ErlNifPid pid = p.pid;
    enif_send(nullptr, &pid, msg, enif_make_tuple2(msg, ref, make(msg, arg)));
    enif_free_env(msg);
}

ERL_NIF_TERM outputs_term(ErlNifEnv *env, void *arg) {
    auto *record = static_cast<std::vector<uint8_t> *>(arg);
    ERL_NIF_TERM bin;
    unsigned char *data = enif_make_new_binary(env, record->size(), &bin);
    std::memcpy(data, record->data(), record->size());
    return enif_make_tuple2(env, atom(env, "ok"), bin);
}

ERL_NIF_TERM error_term(ErlNifEnv *env, void *arg) {
    auto *reason = static_cast<std::string *>(arg);
    return error(env, *reason == ":timeout" ? atom(env, "timeout") : text(env, *reason));
}

// The context's waiter: the head run, until done or past its deadline. A run
// is late when the device finished it (its outputs on the host) after its
// deadline, or has not finished it by then, however soon the waiter looks:
// the reply's arrival against the deadline, as the Matcher's mailbox orders
// a Port reply and its deadline message.
void wait_for_runs(Context *c) {
    std::unique_lock<std::mutex> l(c->lock);
    for (;;) {
        c->wake.wait(l, [&] { return c->stopping || !c->pending.empty(); });
        if (c->pending.empty()) return;  // stopping with nothing left
        Pending head = c->pending.front();
        l.unlock();
        const uint64_t now = monotonic_ns();
        const long long left =
            head.deadline_ns > now ? (long long)((head.deadline_ns - now + 999999) / 1000000) : 0;
        char why[512] = "";
        nxs_status s = nxs_request_wait(head.request, left, why, sizeof why);
        if (s == NXS_OK && nxs_request_done_ns(head.request) > head.deadline_ns) s = NXS_TIMEOUT;
        l.lock();
        if (s == NXS_TIMEOUT) {
            // Late: fail it and every run behind it, then let the device finish them.
            std::deque<Pending> failed;
            failed.swap(c->pending);
            l.unlock();
            std::string reason = ":timeout";
            for (Pending &p : failed) {
                reply(p, error_term, &reason);
                nxs_request_free(p.request);  // waits for the device
                enif_free_env(p.env);
            }
            l.lock();
            continue;
        }
        c->pending.pop_front();
        l.unlock();
        std::vector<uint8_t> record;
        if (s == NXS_OK && nxs_port::outputs_record(head.request, &record)) {
            reply(head, outputs_term, &record);
        } else {
            std::string reason = why[0] ? why : "the run failed";
            reply(head, error_term, &reason);
        }
        nxs_request_free(head.request);
        enif_free_env(head.env);
        l.lock();
    }
}

void context_destructor(ErlNifEnv *, void *object) {
    Context *c = static_cast<ContextRef *>(object)->ctx;
    {  // owners still watched no longer release anything of this context
        std::lock_guard<std::mutex> g(watches_lock);
        for (auto it = watches.begin(); it != watches.end();) {
            if (it->first.first == c) {
                std::lock_guard<std::mutex> l(it->second->lock);
                it->second->ctx = nullptr;
                it = watches.erase(it);
            } else {
                ++it;
            }
        }
    }
    {
        std::lock_guard<std::mutex> l(c->lock);
        c->stopping = true;
    }
    c->wake.notify_all();
    if (c->waiter.joinable()) c->waiter.join();
    nxs_destroy(c->context);
    delete c;
}

void watch_down(ErlNifEnv *, void *object, ErlNifPid *, ErlNifMonitor *) {
    Watch *w = *static_cast<Watch **>(object);
    std::lock_guard<std::mutex> g(w->lock);
    if (w->ctx)
        for (uint32_t segment : w->segments) nxs_release(w->ctx->context, segment);
    w->segments.clear();
}

// The monitor's resource goes once its owner is down: so does its Watch.
void watch_destructor(ErlNifEnv *, void *object) {
    Watch *w = *static_cast<Watch **>(object);
    {
        std::lock_guard<std::mutex> g(watches_lock);
        for (auto it = watches.begin(); it != watches.end(); ++it)
            if (it->second == w) {
                watches.erase(it);
                break;
            }
    }
    delete w;
}

bool get_context(ErlNifEnv *env, ERL_NIF_TERM term, Context **out) {
    ContextRef *ref;
    if (!enif_get_resource(env, term, CONTEXT, reinterpret_cast<void **>(&ref))) return false;
    *out = ref->ctx;
    return true;
}

ERL_NIF_TERM open_nif(ErlNifEnv *env, int, const ERL_NIF_TERM argv[]) {
    int device;
    if (!enif_get_int(env, argv[0], &device)) return enif_make_badarg(env);
    char why[512] = "";
    nxs_context *handle = nullptr;
    if (nxs_create(device, &handle, why, sizeof why) != NXS_OK) return error(env, text(env, why));
    Context *c = new Context();
    c->context = handle;
    c->waiter = std::thread(wait_for_runs, c);
    auto *ref = static_cast<ContextRef *>(enif_alloc_resource(CONTEXT, sizeof(ContextRef)));
    ref->ctx = c;
    ERL_NIF_TERM term = enif_make_resource(env, ref);
    enif_release_resource(ref);
    return enif_make_tuple2(env, atom(env, "ok"), term);
}

ERL_NIF_TERM configure_nif(ErlNifEnv *env, int, const ERL_NIF_TERM argv[]) {
    Context *c;
    ErlNifBinary record;
    if (!get_context(env, argv[0], &c) || !enif_inspect_binary(env, argv[1], &record))
        return enif_make_badarg(env);
    nxs_port::Request q;
    std::string why;
    if (!nxs_port::parse(record.data, record.size, &q, &why)) return error(env, text(env, why));
    if (q.kind != nxs_port::kConfigure) return error(env, text(env, "not a configure record"));
    char buf[512] = "";
    if (nxs_configure(c->context, q.segment, &q.geometry, (uint32_t)q.members.size(),
                      q.members.data(), buf, sizeof buf) != NXS_OK) {
        nxs_release(c->context, q.segment);
        return error(env, enif_make_tuple2(env, atom(env, "configuration_refused"), text(env, buf)));
    }
    return atom(env, "ok");
}

ERL_NIF_TERM run_nif(ErlNifEnv *env, int, const ERL_NIF_TERM argv[]) {
    Context *c;
    ErlNifBinary record;
    ErlNifPid pid;
    unsigned int timeout_ms;
    if (!get_context(env, argv[0], &c) || !enif_inspect_binary(env, argv[1], &record) ||
        !enif_get_local_pid(env, argv[2], &pid) || !enif_get_uint(env, argv[4], &timeout_ms))
        return enif_make_badarg(env);
    nxs_port::Request q;
    std::string why;
    if (!nxs_port::parse(record.data, record.size, &q, &why)) return error(env, text(env, why));
    if (q.kind != nxs_port::kRun) return error(env, text(env, "not a run record"));
    char buf[512] = "";
    nxs_request *request = nullptr;
    // The entries are copied into the request before the call returns.
    const nxs_status s = nxs_run_async(c->context, q.segment, (uint32_t)q.params.size(),
                                       q.params.data(), (uint32_t)q.entries.size(),
                                       q.entries.data(), nullptr, nullptr, 0, &request, buf,
                                       sizeof buf);
    if (s == NXS_NO_SEGMENT)
        return error(env, text(env, "segment " + std::to_string(q.segment) + " is not configured"));
    if (s != NXS_OK) return error(env, text(env, buf));
    Pending p{request, pid, enif_alloc_env(), 0,
              monotonic_ns() + (uint64_t)timeout_ms * 1000000ull};
    p.ref = enif_make_copy(p.env, argv[3]);
    {
        std::lock_guard<std::mutex> l(c->lock);
        c->pending.push_back(p);
    }
    c->wake.notify_one();
    return atom(env, "ok");
}

ERL_NIF_TERM watch_nif(ErlNifEnv *env, int, const ERL_NIF_TERM argv[]) {
    Context *c;
    ErlNifPid owner;
    unsigned int segment;
    if (!get_context(env, argv[0], &c) || !enif_get_local_pid(env, argv[1], &owner) ||
        !enif_get_uint(env, argv[2], &segment))
        return enif_make_badarg(env);
    char key[64];
    enif_snprintf(key, sizeof key, "%T", argv[1]);
    std::lock_guard<std::mutex> g(watches_lock);
    Watch *&w = watches[{c, std::string(key)}];
    if (!w) {
        w = new Watch();
        w->ctx = c;
        auto *holder = static_cast<Watch **>(enif_alloc_resource(WATCH, sizeof(Watch *)));
        *holder = w;
        enif_monitor_process(env, holder, &owner, nullptr);
        enif_release_resource(holder);  // the monitor keeps it until the owner exits
    }
    std::lock_guard<std::mutex> l(w->lock);
    w->segments.insert(segment);
    return atom(env, "ok");
}

ERL_NIF_TERM release_nif(ErlNifEnv *env, int, const ERL_NIF_TERM argv[]) {
    Context *c;
    unsigned int segment;
    if (!get_context(env, argv[0], &c) || !enif_get_uint(env, argv[1], &segment))
        return enif_make_badarg(env);
    nxs_release(c->context, segment);
    return atom(env, "ok");
}

int load(ErlNifEnv *env, void **, ERL_NIF_TERM) {
    const ErlNifResourceFlags flags = ERL_NIF_RT_CREATE;
    CONTEXT = enif_open_resource_type(env, nullptr, "nx_stereo_cuda_context", context_destructor,
                                      flags, nullptr);
    ErlNifResourceTypeInit init{};
    init.dtor = watch_destructor;
    init.down = watch_down;
    WATCH = enif_open_resource_type_x(env, "nx_stereo_cuda_watch", &init, flags, nullptr);
    return CONTEXT && WATCH ? 0 : 1;
}

ErlNifFunc functions[] = {
    {"open", 1, open_nif, ERL_NIF_DIRTY_JOB_CPU_BOUND},
    {"configure", 2, configure_nif, ERL_NIF_DIRTY_JOB_CPU_BOUND},
    {"run", 5, run_nif, 0},
    {"watch", 3, watch_nif, 0},
    {"release", 2, release_nif, 0},
};

}  // namespace

ERL_NIF_INIT(Elixir.NxStereo.CudaNif, functions, load, nullptr, nullptr, nullptr)
