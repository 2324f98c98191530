/*
 * The invocation scheduler behind glsl_cpu.h (TEST INFRASTRUCTURE ONLY).
 *
 * A workgroup's invocations run as fibers on the calling thread, each on its
 * own stack, switched by a few instructions of x86-64 assembly that save and
 * restore the callee-saved registers. The scheduler resumes every runnable
 * fiber until it reaches a sync point or returns; then it completes the sync
 * points that can complete: a barrier once every invocation of the workgroup
 * that has not returned waits at one, and the subgroup operations of a
 * subgroup once every invocation of it that has not returned waits at one
 * (each reads the value its source lane deposited; a source outside the
 * subgroup, or one that has returned, reads the caller's own value, a result
 * GLSL leaves undefined and the shaders discard). Anything else (a barrier
 * in divergent code, invocations of one subgroup waiting at a barrier and a
 * subgroup operation at once) is reported as an error, not guessed at.
 */
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "glsl_cpu.h"

thread_local nxs_invocation *nxs_current = nullptr;

extern "C" void nxs_switch(void **save, void *load);
extern "C" void nxs_fiber_entry();

// nxs_switch(save, load): push the callee-saved registers, store the stack
// pointer at *save, take `load` as the stack pointer, pop its registers and
// return on that stack. nxs_fiber_entry is where a new fiber's first switch
// returns to: r12 holds its invocation, r13 the function to run on it.
asm(R"(
    .text
    .globl nxs_switch
    .type nxs_switch, @function
nxs_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
    .size nxs_switch, .-nxs_switch

    .globl nxs_fiber_entry
    .type nxs_fiber_entry, @function
nxs_fiber_entry:
    subq $8, %rsp
    movq %r12, %rdi
    call *%r13
    ud2
    .size nxs_fiber_entry, .-nxs_fiber_entry
)");

namespace {

constexpr size_t kStackBytes = 256 * 1024;

struct Workgroup {
    std::vector<nxs_invocation> invocations;
    std::vector<char *> stacks;
    void *scheduler_sp = nullptr;
    void (*entry)() = nullptr;
};

thread_local Workgroup *current_group = nullptr;

void fiber_main(nxs_invocation *me) {
    current_group->entry();
    me->state = NXS_DONE;
    nxs_switch(&me->stack_pointer, current_group->scheduler_sp);
    std::abort();  // a finished fiber is never resumed
}

void start_fiber(nxs_invocation *inv, char *stack) {
    uintptr_t top = (reinterpret_cast<uintptr_t>(stack) + kStackBytes) & ~uintptr_t(15);
    void **sp = reinterpret_cast<void **>(top);
    *--sp = nullptr;                                          // alignment slot
    *--sp = reinterpret_cast<void *>(&nxs_fiber_entry);       // where the first switch returns
    *--sp = nullptr;                                          // rbp
    *--sp = nullptr;                                          // rbx
    *--sp = inv;                                              // r12: the invocation
    *--sp = reinterpret_cast<void *>(&fiber_main);            // r13: the function
    *--sp = nullptr;                                          // r14
    *--sp = nullptr;                                          // r15
    inv->stack_pointer = sp;
}

}  // namespace

void nxs_yield() {
    nxs_invocation *me = nxs_current;
    nxs_switch(&me->stack_pointer, current_group->scheduler_sp);
}

extern "C" int nxs_dispatch(const nxs_module *module, uvec3 groups, int subgroup_size, char *error,
                            int error_size) {
    auto fail = [&](const char *what) {
        std::snprintf(error, error_size, "%s: %s", module->name, what);
        return -1;
    };
    const int nx = module->local_size_x, n = module->local_size_x * module->local_size_y;
    if (n <= 0 || subgroup_size <= 0 || n % subgroup_size != 0) return fail("bad workgroup size");
    if (module->shared_bytes && module->shared_bytes() < 0)
        return fail("shared arrays exceed the emulator's capacity");
    Workgroup group;
    group.entry = module->entry;
    group.invocations.resize(n);
    group.stacks.resize(n);
    for (int i = 0; i < n; ++i) group.stacks[i] = static_cast<char *>(std::malloc(kStackBytes));
    Workgroup *saved_group = current_group;
    nxs_invocation *saved_current = nxs_current;
    current_group = &group;
    const int subgroups = n / subgroup_size;
    int status = 0;
    for (uint gz = 0; gz < groups.z && status == 0; ++gz)
        for (uint gy = 0; gy < groups.y && status == 0; ++gy)
            for (uint gx = 0; gx < groups.x && status == 0; ++gx) {
                for (int i = 0; i < n; ++i) {
                    nxs_invocation &inv = group.invocations[i];
                    std::memset(&inv, 0, sizeof(inv));
                    const uint lx = (uint)(i % nx), ly = (uint)(i / nx);
                    inv.local_id = uvec3(lx, ly, 0);
                    inv.local_index = (uint)i;
                    inv.groups = groups;
                    inv.group_size = uvec3((uint)nx, (uint)module->local_size_y, 1);
                    inv.subgroup_size = (uint)subgroup_size;
                    inv.group_id = uvec3(gx, gy, gz);
                    inv.global_id = uvec3(gx * (uint)nx + lx,
                                          gy * (uint)module->local_size_y + ly, gz);
                    inv.subgroup_lane = (uint)(i % subgroup_size);
                    inv.subgroup = (uint)(i / subgroup_size);
                    inv.state = NXS_RUN;
                    start_fiber(&inv, group.stacks[i]);
                }
                for (;;) {
                    for (int i = 0; i < n; ++i) {
                        nxs_invocation &inv = group.invocations[i];
                        if (inv.state != NXS_RUN) continue;
                        nxs_current = &inv;
                        nxs_switch(&group.scheduler_sp, inv.stack_pointer);
                    }
                    int done = 0, at_barrier = 0, at_subgroup = 0;
                    for (int i = 0; i < n; ++i) {
                        const int s = group.invocations[i].state;
                        done += s == NXS_DONE;
                        at_barrier += s == NXS_BARRIER;
                        at_subgroup += s == NXS_SUBGROUP;
                    }
                    if (done == n) break;
                    if (at_barrier > 0) {
                        if (at_barrier + done != n || at_subgroup > 0) {
                            status = fail("barrier() not reached by the whole workgroup");
                            break;
                        }
                        if (done > 0) {
                            status = fail("barrier() after some invocations returned");
                            break;
                        }
                        for (int i = 0; i < n; ++i) group.invocations[i].state = NXS_RUN;
                        continue;
                    }
                    // subgroup operations: each subgroup whose live invocations all wait
                    bool progressed = false;
                    for (int sg = 0; sg < subgroups; ++sg) {
                        nxs_invocation *base = &group.invocations[sg * subgroup_size];
                        int waiting = 0, live = 0;
                        for (int l = 0; l < subgroup_size; ++l) {
                            live += base[l].state != NXS_DONE;
                            waiting += base[l].state == NXS_SUBGROUP;
                        }
                        if (live == 0 || waiting != live) continue;
                        for (int l = 0; l < subgroup_size; ++l) {
                            nxs_invocation &inv = base[l];
                            if (inv.state != NXS_SUBGROUP) continue;
                            long src = -1;
                            if (inv.op == NXS_UP) src = (long)l - (long)inv.operand;
                            else if (inv.op == NXS_DOWN) src = (long)l + (long)inv.operand;
                            else if (inv.op == NXS_XOR) src = (long)(l ^ (int)inv.operand);
                            else src = (long)inv.operand;
                            const bool valid = src >= 0 && src < subgroup_size &&
                                               base[src].state == NXS_SUBGROUP;
                            std::memcpy(inv.result, valid ? base[src].value : inv.value, 16);
                        }
                        for (int l = 0; l < subgroup_size; ++l)
                            if (base[l].state == NXS_SUBGROUP) base[l].state = NXS_RUN;
                        progressed = true;
                    }
                    if (!progressed) {
                        status = fail("invocations wait at sync points that cannot complete");
                        break;
                    }
                }
            }
    for (int i = 0; i < n; ++i) std::free(group.stacks[i]);
    current_group = saved_group;
    nxs_current = saved_current;
    return status;
}
