/* A stand-in for the part of Erlang/OTP's erl_nif.h that nif/nx_stereo_cuda_nif.cpp
 * uses, with the documented names and meanings, so that the NIF compiles and runs
 * here against tests/erts_stub/fake_erts.cpp (TEST INFRASTRUCTURE ONLY: a real
 * build uses the ERTS header, nif/Makefile). Terms are handles into the fake's
 * table; messages sent are queued for the test to read. */
#ifndef NXS_FAKE_ERL_NIF_H
#define NXS_FAKE_ERL_NIF_H
#include <stddef.h>
#include <stdint.h>

typedef uintptr_t ERL_NIF_TERM;
typedef struct nxs_fake_env ErlNifEnv;
typedef struct nxs_fake_resource_type ErlNifResourceType;
typedef struct { uint64_t id; } ErlNifPid;
typedef struct { uint64_t id; } ErlNifMonitor;
typedef struct { size_t size; unsigned char *data; } ErlNifBinary;
typedef enum { ERL_NIF_RT_CREATE = 1, ERL_NIF_RT_TAKEOVER = 2 } ErlNifResourceFlags;
typedef void ErlNifResourceDtor(ErlNifEnv *, void *);
typedef void ErlNifResourceStop(ErlNifEnv *, void *, int, int);
typedef void ErlNifResourceDown(ErlNifEnv *, void *, ErlNifPid *, ErlNifMonitor *);
typedef struct {
    ErlNifResourceDtor *dtor;
    ErlNifResourceStop *stop;
    ErlNifResourceDown *down;
    int members;
    void *dyncall;
} ErlNifResourceTypeInit;
typedef struct {
    const char *name;
    unsigned arity;
    ERL_NIF_TERM (*fptr)(ErlNifEnv *, int, const ERL_NIF_TERM[]);
    unsigned flags;
} ErlNifFunc;
#define ERL_NIF_DIRTY_JOB_CPU_BOUND 1
#define ERL_NIF_DIRTY_JOB_IO_BOUND 2
typedef struct {
    const char *name;
    int num_of_funcs;
    ErlNifFunc *funcs;
    int (*load)(ErlNifEnv *, void **, ERL_NIF_TERM);
} ErlNifEntry;

#ifdef __cplusplus
extern "C" {
#endif
ERL_NIF_TERM enif_make_atom(ErlNifEnv *, const char *);
unsigned char *enif_make_new_binary(ErlNifEnv *, size_t, ERL_NIF_TERM *);
ERL_NIF_TERM enif_make_tuple2(ErlNifEnv *, ERL_NIF_TERM, ERL_NIF_TERM);
ERL_NIF_TERM enif_make_badarg(ErlNifEnv *);
ERL_NIF_TERM enif_make_copy(ErlNifEnv *, ERL_NIF_TERM);
ERL_NIF_TERM enif_make_resource(ErlNifEnv *, void *);
ErlNifEnv *enif_alloc_env(void);
void enif_free_env(ErlNifEnv *);
int enif_send(ErlNifEnv *, const ErlNifPid *, ErlNifEnv *, ERL_NIF_TERM);
int enif_get_int(ErlNifEnv *, ERL_NIF_TERM, int *);
int enif_get_uint(ErlNifEnv *, ERL_NIF_TERM, unsigned *);
int enif_get_local_pid(ErlNifEnv *, ERL_NIF_TERM, ErlNifPid *);
int enif_inspect_binary(ErlNifEnv *, ERL_NIF_TERM, ErlNifBinary *);
int enif_get_resource(ErlNifEnv *, ERL_NIF_TERM, ErlNifResourceType *, void **);
void *enif_alloc_resource(ErlNifResourceType *, size_t);
void enif_release_resource(void *);
int enif_monitor_process(ErlNifEnv *, void *, const ErlNifPid *, ErlNifMonitor *);
int enif_snprintf(char *, size_t, const char *, ...);
ErlNifResourceType *enif_open_resource_type(ErlNifEnv *, const char *, const char *,
                                            ErlNifResourceDtor *, ErlNifResourceFlags,
                                            ErlNifResourceFlags *);
ErlNifResourceType *enif_open_resource_type_x(ErlNifEnv *, const char *,
                                              const ErlNifResourceTypeInit *,
                                              ErlNifResourceFlags, ErlNifResourceFlags *);
#ifdef __cplusplus
}
#endif

#define ERL_NIF_INIT(NAME, FUNCS, LOAD, RELOAD, UPGRADE, UNLOAD)                          \
    extern "C" ErlNifEntry *nif_init(void) {                                              \
        static ErlNifEntry entry = {#NAME, (int)(sizeof(FUNCS) / sizeof(FUNCS[0])), FUNCS,  \
                                    LOAD};                                                \
        return &entry;                                                                    \
    }
#endif
