// Runtime of the OpenCL C shim (clshim.h): kernel registry, NDRange launches and work-group
// barriers. Test infrastructure only; linked into every translated reference program under
// oracle/_ref/ by oracle/ref_build.py.
//
// Launch order: work-groups one after another in row-major group order (dimension 0 fastest), and
// inside a group the work-items in row-major local order. Without a barrier a work-item runs to
// completion before the next starts. With barriers (the kernel was registered as using one), every
// work-item of a group runs as a fiber on its own stack: the scheduler resumes the fibers in local
// order, each runs until its next barrier() or its end, and the rounds repeat until all have ended
// (OpenCL requires every work-item of a group to reach the same barriers).
#include <string.h>

#include <string>
#include <vector>

#include "clshim.h"

thread_local const clshim_item* clshim_current_item = nullptr;
thread_local const clshim_range* clshim_current_range = nullptr;

namespace {

struct kernel_entry {
    std::string name;
    clshim_entry entry;
    int arity;
    int uses_barrier;
};

std::vector<kernel_entry>& registry() {
    static std::vector<kernel_entry> kernels;
    return kernels;
}

thread_local std::string last_error;

// ---- fibers: a minimal x86-64 System V context switch -------------------------------------------
// clshim_swap(save, next): pushes the callee-saved registers, stores the stack pointer to *save,
// loads next as the stack pointer, pops the registers saved there and returns into that context.
extern "C" void clshim_swap(void** save, void* next);
extern "C" void clshim_fiber_trampoline();
asm(R"(
.text
.globl clshim_swap
.type clshim_swap,@function
clshim_swap:
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
.size clshim_swap, .-clshim_swap
.globl clshim_fiber_trampoline
.type clshim_fiber_trampoline,@function
clshim_fiber_trampoline:
    andq $-16, %rsp
    movq %rbx, %rdi
    call clshim_fiber_main@PLT
    ud2
.size clshim_fiber_trampoline, .-clshim_fiber_trampoline
)");

constexpr size_t kFiberStack = 256 * 1024;

struct fiber {
    void* sp = nullptr;
    std::vector<unsigned char> stack;
    clshim_item item{};
    bool done = false;
};

struct group_run {
    const kernel_entry* kernel = nullptr;
    void** argv = nullptr;
    std::vector<fiber>* fibers = nullptr;
    size_t current = 0;
    void* scheduler_sp = nullptr;
};
thread_local group_run* active_group = nullptr;

void prepare_fiber(fiber& f) {
    if (f.stack.size() != kFiberStack) f.stack.assign(kFiberStack, 0);
    uintptr_t top = reinterpret_cast<uintptr_t>(f.stack.data() + f.stack.size()) & ~uintptr_t(15);
    void** slots = reinterpret_cast<void**>(top - 64);
    // popped in the order r15, r14, r13, r12, rbx, rbp, then the return address
    slots[0] = nullptr;                                                // r15
    slots[1] = nullptr;                                                // r14
    slots[2] = nullptr;                                                // r13
    slots[3] = nullptr;                                                // r12
    slots[4] = &f;                                                     // rbx: the trampoline's argument
    slots[5] = nullptr;                                                // rbp
    slots[6] = reinterpret_cast<void*>(&clshim_fiber_trampoline);     // return address
    f.sp = slots;
    f.done = false;
}

}  // namespace

extern "C" void clshim_fiber_main(void* arg) {
    fiber* f = static_cast<fiber*>(arg);
    group_run* g = active_group;
    clshim_current_item = &f->item;
    g->kernel->entry(g->argv);
    f->done = true;
    clshim_swap(&f->sp, g->scheduler_sp);
    abort();  // a finished fiber is never resumed
}

void barrier(int) {
    group_run* g = active_group;
    if (g == nullptr) {
        fprintf(stderr, "clshim: barrier() in a kernel registered without barriers\n");
        abort();
    }
    fiber& f = (*g->fibers)[g->current];
    clshim_swap(&f.sp, g->scheduler_sp);
    clshim_current_item = &f.item;
}

void clshim_register(const char* name, clshim_entry entry, int arity, int uses_barrier) {
    registry().push_back(kernel_entry{name, entry, arity, uses_barrier});
}

extern "C" {

int clshim_kernel_count() { return (int)registry().size(); }
const char* clshim_kernel_name(int i) { return registry()[i].name.c_str(); }
int clshim_kernel_arity(int i) { return registry()[i].arity; }
const char* clshim_last_error() { return last_error.c_str(); }

}  // extern "C"

namespace {

// Runs groups [first, last) of the flattened group range on the calling thread. argv_in[i] points at
// argument i's storage; the thread copies every argument (at most 8 bytes each) so that its own
// __local buffers can replace the local-memory slots.
void run_groups(const kernel_entry& k, const clshim_range& range, const size_t* groups, void** argv_in,
                const long long* local_bytes, int nargs, size_t first, size_t last) {
    std::vector<uint64_t> slots(nargs > 0 ? nargs : 1);
    std::vector<void*> argv(nargs > 0 ? nargs : 1);
    std::vector<std::vector<unsigned char>> local_memory;
    for (int i = 0; i < nargs; ++i) {
        memcpy(&slots[i], argv_in[i], sizeof(uint64_t));
        if (local_bytes[i] > 0) {
            local_memory.emplace_back((size_t)local_bytes[i] + 64, 0);
            void* p = local_memory.back().data();
            memcpy(&slots[i], &p, sizeof(p));
        }
        argv[i] = &slots[i];
    }
    const size_t group_items = range.local_size[0] * range.local_size[1] * range.local_size[2];
    std::vector<fiber> fibers(k.uses_barrier ? group_items : 0);
    clshim_current_range = &range;
    clshim_item item{};
    for (size_t flat = first; flat < last; ++flat) {
        const size_t gid[3] = {flat % groups[0], (flat / groups[0]) % groups[1], flat / (groups[0] * groups[1])};
        for (auto& m : local_memory) memset(m.data(), 0, m.size());
        if (!k.uses_barrier) {
            for (size_t l2 = 0; l2 < range.local_size[2]; ++l2)
                for (size_t l1 = 0; l1 < range.local_size[1]; ++l1)
                    for (size_t l0 = 0; l0 < range.local_size[0]; ++l0) {
                        const size_t lid[3] = {l0, l1, l2};
                        for (int d = 0; d < 3; ++d) {
                            item.group_id[d] = gid[d];
                            item.local_id[d] = lid[d];
                            item.global_id[d] = gid[d] * range.local_size[d] + lid[d];
                        }
                        clshim_current_item = &item;
                        k.entry(argv.data());
                    }
            continue;
        }
        size_t n = 0;
        for (size_t l2 = 0; l2 < range.local_size[2]; ++l2)
            for (size_t l1 = 0; l1 < range.local_size[1]; ++l1)
                for (size_t l0 = 0; l0 < range.local_size[0]; ++l0, ++n) {
                    const size_t lid[3] = {l0, l1, l2};
                    fiber& f = fibers[n];
                    for (int d = 0; d < 3; ++d) {
                        f.item.group_id[d] = gid[d];
                        f.item.local_id[d] = lid[d];
                        f.item.global_id[d] = gid[d] * range.local_size[d] + lid[d];
                    }
                    prepare_fiber(f);
                }
        group_run run;
        run.kernel = &k;
        run.argv = argv.data();
        run.fibers = &fibers;
        active_group = &run;
        for (bool alive = true; alive;) {
            alive = false;
            for (size_t i = 0; i < fibers.size(); ++i) {
                if (fibers[i].done) continue;
                run.current = i;
                clshim_current_item = &fibers[i].item;
                clshim_swap(&run.scheduler_sp, fibers[i].sp);
                alive |= !fibers[i].done;
            }
        }
        active_group = nullptr;
    }
    clshim_current_item = nullptr;
    clshim_current_range = nullptr;
}

}  // namespace

extern "C" {

// Runs kernel `index` over an NDRange. argv[i] points at argument i's storage; local_bytes[i] > 0
// marks argument i as __local memory of that many bytes, which every work-group gets fresh.
// local_size may be null (the implementation picks the group size: one work-item per group).
// threads > 1 spreads the work-groups over that many threads; the caller passes it only for kernels
// whose work-groups write disjoint memory and use no atomics, whose results cannot depend on the
// order of the groups. Returns 0, or -1 with clshim_last_error() set.
int clshim_launch(int index, int dims, const size_t* global_size, const size_t* local_size, void** argv,
                  const long long* local_bytes, int nargs, int threads) {
    if (index < 0 || index >= (int)registry().size()) {
        last_error = "unknown kernel";
        return -1;
    }
    const kernel_entry& k = registry()[index];
    if (nargs != k.arity) {
        last_error = k.name + ": expected " + std::to_string(k.arity) + " arguments, got " + std::to_string(nargs);
        return -1;
    }
    if (dims < 1 || dims > 3) {
        last_error = "work_dim must be 1..3";
        return -1;
    }
    clshim_range range{};
    range.dims = dims;
    size_t groups[3] = {1, 1, 1};
    for (int d = 0; d < 3; ++d) {
        range.global_size[d] = d < dims ? global_size[d] : 1;
        range.local_size[d] = (d < dims && local_size != nullptr) ? local_size[d] : 1;
        if (range.local_size[d] == 0 || range.global_size[d] % range.local_size[d] != 0) {
            last_error = k.name + ": global size not a multiple of the local size";
            return -1;
        }
        groups[d] = range.global_size[d] / range.local_size[d];
    }
    const size_t total = groups[0] * groups[1] * groups[2];
    if (threads <= 1 || total < 2) {
        run_groups(k, range, groups, argv, local_bytes, nargs, 0, total);
        return 0;
    }
    const size_t chunk = 256;
    const long long chunks = (long long)((total + chunk - 1) / chunk);
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (long long c = 0; c < chunks; ++c) {
        const size_t first = (size_t)c * chunk;
        const size_t last = first + chunk < total ? first + chunk : total;
        run_groups(k, range, groups, argv, local_bytes, nargs, first, last);
    }
    return 0;
}

}  // extern "C"
