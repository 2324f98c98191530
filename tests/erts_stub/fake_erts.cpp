// A fake Erlang runtime for the NIF's tests (TEST INFRASTRUCTURE ONLY): terms
// live in one table for the process's life; enif_send queues each message's
// printed form for the test to read; monitors fire when the test says a
// process is down; resources are reference-counted and destructed at zero.
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "erl_nif.h"

struct nxs_fake_env {};
struct nxs_fake_resource_type {
    std::string name;
    ErlNifResourceDtor *dtor = nullptr;
    ErlNifResourceDown *down = nullptr;
};

namespace {
enum Kind { ATOM, INT, BINARY, TUPLE, PID, RESOURCE, REF };
struct Term {
    Kind kind;
    std::string text;  // atom name, binary bytes
    long long value = 0;
    std::vector<ERL_NIF_TERM> items;
    void *resource = nullptr;
};
struct Resource {
    nxs_fake_resource_type *type;
    int refs;
    alignas(16) unsigned char data[1];
};
std::mutex lock;
std::vector<Term> terms(1);  // term 0 is never handed out
std::deque<std::string> messages;
std::multimap<uint64_t, void *> monitors;  // pid -> resource object

ERL_NIF_TERM add(Term t) {
    std::lock_guard<std::mutex> g(lock);
    terms.push_back(std::move(t));
    return terms.size() - 1;
}
Term get(ERL_NIF_TERM t) {
    std::lock_guard<std::mutex> g(lock);
    return t < terms.size() ? terms[t] : Term{ATOM, "invalid"};
}
Resource *header(void *object) {
    return reinterpret_cast<Resource *>(static_cast<unsigned char *>(object) -
                                        offsetof(Resource, data));
}
std::string print(ERL_NIF_TERM t) {
    Term x = get(t);
    switch (x.kind) {
    case ATOM: return ":" + x.text;
    case INT: return std::to_string(x.value);
    case PID: return "#PID<" + std::to_string(x.value) + ">";
    case REF: return "#Ref<" + std::to_string(x.value) + ">";
    case RESOURCE: return "#Resource";
    case BINARY: {
        std::string hex = "<<";
        for (unsigned char c : x.text) {
            char b[4];
            snprintf(b, sizeof b, "%02x", c);
            hex += b;
        }
        return hex + ">>";
    }
    case TUPLE: {
        std::string s = "{";
        for (size_t i = 0; i < x.items.size(); ++i) s += (i ? ", " : "") + print(x.items[i]);
        return s + "}";
    }
    }
    return "?";
}
}  // namespace

extern "C" {
ERL_NIF_TERM enif_make_atom(ErlNifEnv *, const char *name) { return add(Term{ATOM, name}); }
unsigned char *enif_make_new_binary(ErlNifEnv *, size_t size, ERL_NIF_TERM *out) {
    *out = add(Term{BINARY, std::string(size, '\0')});
    std::lock_guard<std::mutex> g(lock);
    return reinterpret_cast<unsigned char *>(&terms[*out].text[0]);
}
ERL_NIF_TERM enif_make_tuple2(ErlNifEnv *, ERL_NIF_TERM a, ERL_NIF_TERM b) {
    Term t{TUPLE};
    t.items = {a, b};
    return add(t);
}
ERL_NIF_TERM enif_make_badarg(ErlNifEnv *) { return add(Term{ATOM, "badarg"}); }
ERL_NIF_TERM enif_make_copy(ErlNifEnv *, ERL_NIF_TERM t) { return t; }
ERL_NIF_TERM enif_make_resource(ErlNifEnv *, void *object) {
    Term t{RESOURCE};
    t.resource = object;
    header(object)->refs++;
    return add(t);
}
ErlNifEnv *enif_alloc_env(void) { return new nxs_fake_env(); }
void enif_free_env(ErlNifEnv *env) { delete env; }
int enif_send(ErlNifEnv *, const ErlNifPid *pid, ErlNifEnv *, ERL_NIF_TERM msg) {
    std::string text = "#PID<" + std::to_string(pid->id) + "> " + print(msg);
    std::lock_guard<std::mutex> g(lock);
    messages.push_back(text);
    return 1;
}
int enif_get_int(ErlNifEnv *, ERL_NIF_TERM t, int *out) {
    Term x = get(t);
    if (x.kind != INT) return 0;
    *out = (int)x.value;
    return 1;
}
int enif_get_uint(ErlNifEnv *, ERL_NIF_TERM t, unsigned *out) {
    Term x = get(t);
    if (x.kind != INT || x.value < 0) return 0;
    *out = (unsigned)x.value;
    return 1;
}
int enif_get_local_pid(ErlNifEnv *, ERL_NIF_TERM t, ErlNifPid *out) {
    Term x = get(t);
    if (x.kind != PID) return 0;
    out->id = (uint64_t)x.value;
    return 1;
}
int enif_inspect_binary(ErlNifEnv *, ERL_NIF_TERM t, ErlNifBinary *out) {
    std::lock_guard<std::mutex> g(lock);
    if (t >= terms.size() || terms[t].kind != BINARY) return 0;
    out->size = terms[t].text.size();
    out->data = reinterpret_cast<unsigned char *>(&terms[t].text[0]);
    return 1;
}
int enif_get_resource(ErlNifEnv *, ERL_NIF_TERM t, ErlNifResourceType *type, void **out) {
    Term x = get(t);
    if (x.kind != RESOURCE || header(x.resource)->type != type) return 0;
    *out = x.resource;
    return 1;
}
void *enif_alloc_resource(ErlNifResourceType *type, size_t size) {
    Resource *r = static_cast<Resource *>(calloc(1, sizeof(Resource) + size));
    r->type = type;
    r->refs = 1;
    return r->data;
}
void enif_release_resource(void *object) {
    Resource *r = header(object);
    if (--r->refs == 0) {
        if (r->type->dtor) r->type->dtor(nullptr, object);
        free(r);
    }
}
int enif_monitor_process(ErlNifEnv *, void *object, const ErlNifPid *pid, ErlNifMonitor *) {
    header(object)->refs++;
    std::lock_guard<std::mutex> g(lock);
    monitors.insert({pid->id, object});
    return 0;
}
int enif_snprintf(char *out, size_t size, const char *format, ...) {
    va_list args;
    va_start(args, format);
    int n;
    if (strcmp(format, "%T") == 0) n = snprintf(out, size, "%s", print(va_arg(args, ERL_NIF_TERM)).c_str());
    else n = vsnprintf(out, size, format, args);
    va_end(args);
    return n;
}
ErlNifResourceType *enif_open_resource_type(ErlNifEnv *, const char *, const char *name,
                                            ErlNifResourceDtor *dtor, ErlNifResourceFlags,
                                            ErlNifResourceFlags *) {
    auto *t = new nxs_fake_resource_type();
    t->name = name;
    t->dtor = dtor;
    return t;
}
ErlNifResourceType *enif_open_resource_type_x(ErlNifEnv *, const char *name,
                                              const ErlNifResourceTypeInit *init,
                                              ErlNifResourceFlags, ErlNifResourceFlags *) {
    auto *t = new nxs_fake_resource_type();
    t->name = name;
    t->dtor = init->dtor;
    t->down = init->down;
    return t;
}

// ---- the test's side
ERL_NIF_TERM fake_int(long long v) { Term t{INT}; t.value = v; return add(t); }
ERL_NIF_TERM fake_pid(long long v) { Term t{PID}; t.value = v; return add(t); }
ERL_NIF_TERM fake_ref(long long v) { Term t{REF}; t.value = v; return add(t); }
ERL_NIF_TERM fake_binary(const void *data, size_t size) {
    return add(Term{BINARY, std::string(static_cast<const char *>(data), size)});
}
// The printed form of a term (binaries in hex); returns the length written.
int fake_print(ERL_NIF_TERM t, char *out, int size) {
    return snprintf(out, (size_t)size, "%s", print(t).c_str());
}
// The oldest message not yet read, or an empty string.
int fake_next_message(char *out, int size) {
    std::string m;
    {
        std::lock_guard<std::mutex> g(lock);
        if (messages.empty()) return 0;
        m = messages.front();
        messages.pop_front();
    }
    return snprintf(out, (size_t)size, "%s", m.c_str());
}
// Process `pid` exits: its monitors' down callbacks run, then their references go.
void fake_process_down(long long pid) {
    std::vector<void *> fired;
    {
        std::lock_guard<std::mutex> g(lock);
        auto range = monitors.equal_range((uint64_t)pid);
        for (auto it = range.first; it != range.second; ++it) fired.push_back(it->second);
        monitors.erase(range.first, range.second);
    }
    for (void *object : fired) {
        ErlNifPid p{(uint64_t)pid};
        ErlNifMonitor m{0};
        if (header(object)->type->down) header(object)->type->down(nullptr, object, &p, &m);
        enif_release_resource(object);
    }
}
ErlNifEnv *fake_env(void) { static nxs_fake_env env; return &env; }
// Item `i` of a tuple term (0 when it is none).
ERL_NIF_TERM fake_tuple_item(ERL_NIF_TERM t, int i) {
    Term x = get(t);
    return x.kind == TUPLE && i >= 0 && (size_t)i < x.items.size() ? x.items[i] : 0;
}
}
