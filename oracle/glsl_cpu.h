/*
 * GLSL compute-shader semantics on the CPU, for running the reference's own
 * shader sources as C++ (TEST INFRASTRUCTURE ONLY: the oracle's cross-check
 * against the reference; the product never includes it).
 *
 * oracle/build_ref.py rewrites each shader's declarations into the macros
 * below (buffer blocks become pointers the host binds, specialisation
 * constants become variables, `shared` arrays become statics of one
 * workgroup) and compiles it with this header. Each invocation of a
 * workgroup runs as a fiber (glsl_runtime.cpp); barrier() and the subgroup
 * operations are the points where the fibers meet: a subgroup operation
 * completes once every invocation of the subgroup that has not returned has
 * reached one, and barrier() once every invocation of the workgroup has.
 * Arithmetic follows GLSL's integer rules (32-bit wrap-around) and IEEE
 * single precision with every operation rounded on its own (the build uses
 * -ffp-contract=off), which GLSL permits and the reference's Nx evaluator
 * does.
 */
#ifndef NXS_GLSL_CPU_H
#define NXS_GLSL_CPU_H

/* No C library headers: the shaders' unqualified floor, abs, min ... must
 * find only the GLSL overloads below. */
#include <cstdint>

typedef unsigned int uint;

struct uvec2 {
    uint x, y;
    uvec2() : x(0), y(0) {}
    explicit uvec2(uint s) : x(s), y(s) {}
    uvec2(uint a, uint b) : x(a), y(b) {}
    uint &operator[](int i) { return i == 0 ? x : y; }
    uint operator[](int i) const { return i == 0 ? x : y; }
};
inline uvec2 operator+(uvec2 a, uvec2 b) { return uvec2(a.x + b.x, a.y + b.y); }
inline uvec2 operator-(uvec2 a, uvec2 b) { return uvec2(a.x - b.x, a.y - b.y); }
inline uvec2 operator^(uvec2 a, uvec2 b) { return uvec2(a.x ^ b.x, a.y ^ b.y); }
inline uvec2 operator&(uvec2 a, uvec2 b) { return uvec2(a.x & b.x, a.y & b.y); }
inline uvec2 operator|(uvec2 a, uvec2 b) { return uvec2(a.x | b.x, a.y | b.y); }
inline uvec2 &operator+=(uvec2 &a, uvec2 b) { return a = a + b; }

struct uvec3 {
    uint x, y, z;
    uvec3() : x(0), y(0), z(0) {}
    uvec3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
};

struct uvec4 {
    uint x, y, z, w;
    uvec4() : x(0), y(0), z(0), w(0) {}
    explicit uvec4(uint s) : x(s), y(s), z(s), w(s) {}
    uvec4(uint a, uint b, uint c, uint d) : x(a), y(b), z(c), w(d) {}
    uvec2 xy() const { return uvec2(x, y); }
    uvec2 zw() const { return uvec2(z, w); }
    uint &operator[](int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
    uint operator[](int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
};
inline uvec4 operator+(uvec4 a, uvec4 b) { return uvec4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline uvec4 &operator+=(uvec4 &a, uvec4 b) { return a = a + b; }

struct ivec2 {
    int x, y;
    ivec2() : x(0), y(0) {}
    explicit ivec2(int s) : x(s), y(s) {}
    ivec2(int a, int b) : x(a), y(b) {}
};

struct vec2 {
    float x, y;
    vec2() : x(0), y(0) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
    float &operator[](int i) { return i == 0 ? x : y; }
    float operator[](int i) const { return i == 0 ? x : y; }
};
struct vec3 {
    float x, y, z;
    vec3() : x(0), y(0), z(0) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct vec4 {
    float x, y, z, w;
    vec4() : x(0), y(0), z(0), w(0) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float &operator[](int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
    float operator[](int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
};
/* component-wise arithmetic, each component rounded on its own */
inline vec2 operator+(vec2 a, vec2 b) { return vec2(a.x + b.x, a.y + b.y); }
inline vec2 operator-(vec2 a, vec2 b) { return vec2(a.x - b.x, a.y - b.y); }
inline vec2 operator*(vec2 a, vec2 b) { return vec2(a.x * b.x, a.y * b.y); }
inline vec2 operator/(vec2 a, vec2 b) { return vec2(a.x / b.x, a.y / b.y); }
inline vec2 operator*(vec2 a, float b) { return vec2(a.x * b, a.y * b); }
inline vec2 operator*(float a, vec2 b) { return vec2(a * b.x, a * b.y); }
inline vec2 operator+(vec2 a, float b) { return vec2(a.x + b, a.y + b); }
inline vec2 operator-(vec2 a, float b) { return vec2(a.x - b, a.y - b); }
inline vec2 operator/(vec2 a, float b) { return vec2(a.x / b, a.y / b); }
inline vec4 operator+(vec4 a, vec4 b) { return vec4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline vec4 operator-(vec4 a, vec4 b) { return vec4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
inline vec4 operator*(vec4 a, vec4 b) { return vec4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
inline vec4 operator*(vec4 a, float b) { return vec4(a.x * b, a.y * b, a.z * b, a.w * b); }
inline vec4 operator*(float a, vec4 b) { return vec4(a * b.x, a * b.y, a * b.z, a * b.w); }

/* ---- built-in functions (GLSL 4.50 §8), the overloads the shaders use ---- */
inline int min(int a, int b) { return a < b ? a : b; }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline float min(float a, float b) { return b < a ? b : a; }
inline int max(int a, int b) { return a > b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline float max(float a, float b) { return a < b ? b : a; }
inline int clamp(int v, int lo, int hi) { return min(max(v, lo), hi); }
inline uint clamp(uint v, uint lo, uint hi) { return min(max(v, lo), hi); }
inline float clamp(float v, float lo, float hi) { return min(max(v, lo), hi); }
inline int abs(int v) { return v < 0 ? -v : v; }
inline float abs(float v) { return __builtin_fabsf(v); }
inline float floor(float v) { return __builtin_floorf(v); }
inline float ceil(float v) { return __builtin_ceilf(v); }
inline float trunc(float v) { return __builtin_truncf(v); }
inline float sqrt(float v) { return __builtin_sqrtf(v); }
inline float fract(float v) { return v - __builtin_floorf(v); }
inline int sign(int v) { return (v > 0) - (v < 0); }
inline float sign(float v) { return v > 0.0f ? 1.0f : (v < 0.0f ? -1.0f : 0.0f); }
inline bool isnan(float v) { return __builtin_isnan(v); }
inline bool isinf(float v) { return __builtin_isinf(v); }
inline int bitCount(uint v) { return __builtin_popcount(v); }
inline int bitCount(int v) { return __builtin_popcount((uint)v); }
inline int findLSB(uint v) { return v ? __builtin_ctz(v) : -1; }
inline int findMSB(uint v) { return v ? 31 - __builtin_clz(v) : -1; }
inline uint floatBitsToUint(float v) { uint u; __builtin_memcpy(&u, &v, 4); return u; }
inline int floatBitsToInt(float v) { int u; __builtin_memcpy(&u, &v, 4); return u; }
inline float uintBitsToFloat(uint u) { float v; __builtin_memcpy(&v, &u, 4); return v; }
inline float intBitsToFloat(int u) { float v; __builtin_memcpy(&v, &u, 4); return v; }
/* mix with a boolean selector picks y where a is true (GLSL 4.50 §8.3). */
inline float mix(float x, float y, bool a) { return a ? y : x; }
inline uint mix(uint x, uint y, bool a) { return a ? y : x; }
inline int mix(int x, int y, bool a) { return a ? y : x; }
/* mix with a float weight is x * (1 - a) + y * a, each operation rounded. */
inline float mix(float x, float y, float a) { return x * (1.0f - a) + y * a; }
inline uint bitfieldExtract(uint v, int offset, int bits) {
    return bits == 0 ? 0u : (v >> offset) & (bits == 32 ? 0xFFFFFFFFu : ((1u << bits) - 1u));
}

inline vec2 floor(vec2 v) { return vec2(floor(v.x), floor(v.y)); }
inline vec2 fract(vec2 v) { return vec2(fract(v.x), fract(v.y)); }
inline vec2 max(vec2 a, vec2 b) { return vec2(max(a.x, b.x), max(a.y, b.y)); }
inline vec2 min(vec2 a, vec2 b) { return vec2(min(a.x, b.x), min(a.y, b.y)); }
inline vec2 abs(vec2 v) { return vec2(abs(v.x), abs(v.y)); }
/* step(edge, x): 0 where x < edge, else 1 */
inline float step(float edge, float x) { return x < edge ? 0.0f : 1.0f; }
inline vec2 step(vec2 edge, vec2 x) { return vec2(step(edge.x, x.x), step(edge.y, x.y)); }
inline vec4 floor(vec4 v) { return vec4(floor(v.x), floor(v.y), floor(v.z), floor(v.w)); }
inline vec4 max(vec4 a, vec4 b) { return vec4(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z), max(a.w, b.w)); }
inline vec4 min(vec4 a, vec4 b) { return vec4(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z), min(a.w, b.w)); }

/* atomics on workgroup memory: fibers run one at a time, so a read-modify-write is atomic */
inline uint atomicMin(uint &mem, uint v) { uint old = mem; mem = min(old, v); return old; }
inline uint atomicMax(uint &mem, uint v) { uint old = mem; mem = max(old, v); return old; }
inline uint atomicAdd(uint &mem, uint v) { uint old = mem; mem = old + v; return old; }
inline int atomicAdd(int &mem, int v) { int old = mem; mem = (int)((uint)old + (uint)v); return old; }
inline uint atomicOr(uint &mem, uint v) { uint old = mem; mem = old | v; return old; }

/* ---- the invocation runtime (glsl_runtime.cpp) ---- */
struct nxs_invocation;
extern thread_local nxs_invocation *nxs_current;

enum nxs_sync { NXS_RUN = 0, NXS_SUBGROUP = 1, NXS_BARRIER = 2, NXS_DONE = 3 };
enum nxs_shuffle { NXS_UP = 0, NXS_DOWN = 1, NXS_XOR = 2, NXS_INDEX = 3 };

struct nxs_invocation {
    uvec3 local_id, group_id, global_id, groups, group_size;
    uint local_index, subgroup_size;
    uint subgroup_lane, subgroup;
    int state;       /* nxs_sync */
    int op;          /* nxs_shuffle, while state is NXS_SUBGROUP */
    uint operand;    /* the shuffle's delta, mask or index */
    unsigned char value[16], result[16];
    void *stack_pointer;
};

void nxs_yield();  /* back to the scheduler, which resumes this fiber once its sync point completes */

inline void barrier() {
    nxs_current->state = NXS_BARRIER;
    nxs_yield();
}
inline void memoryBarrierBuffer() {}
inline void memoryBarrierShared() {}
inline void memoryBarrier() {}
inline void groupMemoryBarrier() {}

template <typename T>
inline T nxs_subgroup(T v, int op, uint operand) {
    static_assert(sizeof(T) <= 16, "subgroup values of at most 16 bytes");
    nxs_invocation *me = nxs_current;
    __builtin_memcpy(me->value, &v, sizeof(T));
    me->op = op;
    me->operand = operand;
    me->state = NXS_SUBGROUP;
    nxs_yield();
    T r;
    __builtin_memcpy(&r, me->result, sizeof(T));
    return r;
}
template <typename T> inline T subgroupShuffleUp(T v, uint delta) { return nxs_subgroup(v, NXS_UP, delta); }
template <typename T> inline T subgroupShuffleDown(T v, uint delta) { return nxs_subgroup(v, NXS_DOWN, delta); }
template <typename T> inline T subgroupShuffleXor(T v, uint mask) { return nxs_subgroup(v, NXS_XOR, mask); }
template <typename T> inline T subgroupShuffle(T v, uint index) { return nxs_subgroup(v, NXS_INDEX, index); }

#define gl_LocalInvocationID (nxs_current->local_id)
#define gl_WorkGroupID (nxs_current->group_id)
#define gl_GlobalInvocationID (nxs_current->global_id)
#define gl_SubgroupInvocationID (nxs_current->subgroup_lane)
#define gl_SubgroupID (nxs_current->subgroup)
#define gl_SubgroupSize (nxs_current->subgroup_size)
#define gl_NumWorkGroups (nxs_current->groups)
#define gl_WorkGroupSize (nxs_current->group_size)
#define gl_LocalInvocationIndex (nxs_current->local_index)

/* A shader module as build_ref.py emits it: its entry point, its workgroup
 * size, and where its specialisation constants and buffers live. */
struct nxs_module {
    const char *name;
    void (*entry)();
    int local_size_x, local_size_y;
    int spec_count;
    int spec_id[8];
    void *spec[8];
    int spec_float[8]; /* the constant is a float (else an int) */
    int binding_count;
    int binding[12];
    void **buffer[12];
    long long (*shared_bytes)(); /* bytes its shared arrays need at the current constants */
};

/* Every workgroup of `groups` in turn, each as local_size_x x local_size_y
 * fibers (x fastest) in subgroups of `subgroup_size`. Returns 0, or -1 with a message in `error`. */
extern "C" int nxs_dispatch(const nxs_module *module, uvec3 groups, int subgroup_size, char *error,
                            int error_size);

/* Shared arrays: statics of at most NXS_SHARED_CAP elements each; the module's
 * shared_bytes() lets the dispatcher refuse constants that need more. */
#define NXS_SHARED_CAP 65536
#define NXS_SHARED(type, name, count) static type name[NXS_SHARED_CAP];

#endif
