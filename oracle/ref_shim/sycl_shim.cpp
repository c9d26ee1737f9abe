// Runtime of the host SYCL subset (oracle/ref_shim/sycl/sycl.hpp).
//
// TEST INFRASTRUCTURE ONLY (see the header).
//
// run_range: a 1-d parallel_for, in index order on the calling thread, or
// over an OpenMP team of sycl_shim_set_threads() threads.
//
// run_nd_range: a 1-d nd_range parallel_for.  Each work item of a group is
// a fiber with its own small stack; the group's fibers run round robin, and
// a fiber that reaches item.barrier() switches back to the scheduler, so
// every item of the group reaches the barrier before any item passes it.
// Groups run one after another on each thread of the team, every thread
// with its own fibers (one contiguous block of stacks, so that a round over
// the group stays in cache) and its own work-group local memory.
// On x86-64 the switch is a few instructions that save the callee-saved
// registers and the stack pointer; elsewhere it falls back to ucontext.
#include <sycl/sycl.hpp>

#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#if !defined(__x86_64__)
#include <ucontext.h>
#endif

namespace {
int g_threads = 1;
}

void sycl_shim_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int sycl_shim_threads() { return g_threads; }

namespace sycl_shim {

void run_range(size_t n, const std::function<void(size_t)>& body) {
  if (g_threads <= 1 || n < 2048) {
    for (size_t i = 0; i < n; ++i) body(i);
    return;
  }
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 256)
  for (size_t i = 0; i < n; ++i) body(i);
}

#if defined(__x86_64__)
extern "C" void sycl_shim_switch(void** save_sp, void* load_sp);
// sycl_shim_switch(save, load): push the callee-saved registers, store the
// stack pointer in *save, load `load` as the stack pointer, pop the
// registers saved there and return into that context.
asm(R"(
    .text
    .p2align 4
    .globl sycl_shim_switch
    .type sycl_shim_switch, @function
sycl_shim_switch:
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
    .size sycl_shim_switch, .-sycl_shim_switch
    .section .note.GNU-stack,"",@progbits
    .text
)");
#endif

namespace {

constexpr size_t kStackBytes = 16 * 1024;

struct Fiber {
  char* stack = nullptr;
#if defined(__x86_64__)
  void* sp = nullptr;
#else
  ucontext_t ctx;
#endif
  size_t local = 0;
  bool done = false;
};

struct Group {
  std::vector<Fiber> fibers;
  std::vector<char> stacks;
#if defined(__x86_64__)
  void* sched_sp = nullptr;
#else
  ucontext_t sched_ctx;
#endif
  const std::function<void(size_t, size_t)>* body = nullptr;
  size_t group = 0;
  Fiber* current = nullptr;
};

thread_local Group* t_group = nullptr;

void to_scheduler() {
  Group* g = t_group;
  Fiber* f = g->current;
#if defined(__x86_64__)
  sycl_shim_switch(&f->sp, g->sched_sp);
#else
  swapcontext(&f->ctx, &g->sched_ctx);
#endif
}

[[noreturn]] void fiber_main() {
  for (;;) {
    Group* g = t_group;
    Fiber* f = g->current;
    (*g->body)(g->group, f->local);
    f->done = true;
    to_scheduler();
    // a finished fiber is resumed only after it is reset for a new item
  }
}

#if defined(__x86_64__)
void fiber_reset(Fiber& f) {
  // stack top, 16-byte aligned; a return address slot below it keeps the
  // SysV alignment at fiber_main's entry (rsp + 8 a multiple of 16)
  uintptr_t top = (reinterpret_cast<uintptr_t>(f.stack) + kStackBytes) & ~uintptr_t(15);
  void** sp = reinterpret_cast<void**>(top);
  *--sp = nullptr;                                       // fake return address of fiber_main
  *--sp = reinterpret_cast<void*>(&fiber_main);           // ret target of the first switch
  for (int i = 0; i < 6; ++i) *--sp = nullptr;           // rbp rbx r12 r13 r14 r15
  f.sp = sp;
}
#else
void fiber_reset(Fiber& f) {
  getcontext(&f.ctx);
  f.ctx.uc_stack.ss_sp = f.stack;
  f.ctx.uc_stack.ss_size = kStackBytes;
  f.ctx.uc_link = nullptr;
  makecontext(&f.ctx, reinterpret_cast<void (*)()>(&fiber_main), 0);
}
#endif

void resume(Group& g, Fiber& f) {
  g.current = &f;
#if defined(__x86_64__)
  sycl_shim_switch(&g.sched_sp, f.sp);
#else
  swapcontext(&g.sched_ctx, &f.ctx);
#endif
}

}  // namespace

void group_barrier() {
  if (!t_group || !t_group->current) {
    std::fprintf(stderr, "sycl shim: barrier outside an nd_range kernel\n");
    std::abort();
  }
  to_scheduler();
}

namespace {

void run_groups(size_t first, size_t last, size_t stride, size_t local,
                const std::function<void(size_t, size_t)>& body) {
  Group g;
  g.body = &body;
  g.fibers.resize(local);
  g.stacks.resize(local * kStackBytes + 64);
  char* base = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(g.stacks.data()) + 63) & ~uintptr_t(63));
  for (size_t l = 0; l < local; ++l) g.fibers[l].stack = base + l * kStackBytes;
  Group* saved = t_group;
  t_group = &g;
  for (size_t gi = first; gi < last; gi += stride) {
    g.group = gi;
    for (size_t l = 0; l < local; ++l) {
      g.fibers[l].local = l;
      g.fibers[l].done = false;
      fiber_reset(g.fibers[l]);
    }
    // every round runs each unfinished item up to its next barrier (or to
    // its end); rounds repeat until all items of the group have finished
    for (size_t guard = 0;; ++guard) {
      bool any = false;
      for (auto& f : g.fibers)
        if (!f.done) {
          resume(g, f);
          any = true;
        }
      if (!any) break;
      if (guard > (size_t(1) << 20)) {
        std::fprintf(stderr, "sycl shim: work group did not finish\n");
        std::abort();
      }
    }
  }
  t_group = saved;
}

}  // namespace

int current_thread() { return omp_in_parallel() ? omp_get_thread_num() : 0; }

void run_nd_range(size_t groups, size_t local, const std::function<void(size_t, size_t)>& body) {
  if (g_threads <= 1 || groups < 2) {
    run_groups(0, groups, 1, local, body);
    return;
  }
  const int team = static_cast<int>(std::min<size_t>(groups, static_cast<size_t>(g_threads)));
#pragma omp parallel num_threads(team)
  run_groups(static_cast<size_t>(omp_get_thread_num()), groups, static_cast<size_t>(omp_get_num_threads()), local,
             body);
}

}  // namespace sycl_shim
