// Runs the reference's OpenCL Barnes-Hut tree construction on the CPU:
// gen_mortons (include/Aster/kernels/morton_writer.cl.h:72-122), the bitonic
// sort (radix.cl.h:26-91) and build_tree (BHH_specific.cl.h:171-273), compiled
// from the reference's own kernel text (extract_cl.py) and launched with the
// ND-ranges, work-group sizes and argument order of BH_hyper's host code
// (src/solvers/full_GPU.cpp: make_mortons :97-112, sort_mortons :52-76,
// load_tree_kernel :312-338, buffer sizes :206-250, actual_msize :268-269).
// TEST INFRASTRUCTURE ONLY: the checker for the library's OpenCL-compatible
// build mode (compat_mode = 1), never part of the product.
//
// Work-groups: barrier-free kernels run their work-items one after another
// (work-items of one launch touch disjoint outputs, so the order does not
// change the result); a kernel with barriers runs each work-group's items as
// coroutines (ucontext), switching at every barrier, one group at a time.
#include <stdlib.h>
#include <ucontext.h>

#include <vector>

#include "cl_c_shim.h"

namespace clk_morton {
void gen_mortons(const uint N, const double* positions, ulong* mortons, const double* bd_arr, const int lower,
                 const int upper);
}
namespace clk_radix {
void Sort_BitonicMergesortStart(const ulong* inArray, ulong* outArray, const uint size);
void Sort_BitonicMergesortGlobal(ulong* data, const uint size, const uint k, const uint j);
}  // namespace clk_radix
namespace clk_tree {
void build_tree(const int N, const uint2* morton, int* left_nodes, int* right_nodes, double* node_pos,
                double* n_masses, const double* positions, const double* masses, int* parents, int* counters);
}

namespace clemu {
Item cur;

namespace {
ucontext_t g_sched;
std::vector<ucontext_t> g_items;
std::vector<int> g_state;  // 0 running, 1 waiting at a barrier, 2 finished
int g_item = -1;           // the work-item running, -1 outside a group
void (*g_body)(void*) = nullptr;
void* g_arg = nullptr;

void trampoline() {
    g_body(g_arg);
    g_state[g_item] = 2;  // uc_link returns to the scheduler
}

size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

// every work-item of [0, global) in order, groups of `local`
template <class F>
void run_flat(size_t global, size_t local, F f) {
    for (size_t g = 0; g < global; ++g) {
        cur = Item{g, g % local, g / local, local, global};
        f();
    }
}

// work-groups one at a time, each group's items as coroutines switching at barriers
template <class F>
void run_groups(size_t global, size_t local, F f) {
    const size_t stack = 1 << 16;
    std::vector<std::vector<char>> stacks(local, std::vector<char>(stack));
    g_items.assign(local, ucontext_t{});
    g_state.assign(local, 0);
    g_body = [](void* a) { (*static_cast<F*>(a))(); };
    g_arg = &f;
    for (size_t grp = 0; grp < global / local; ++grp) {
        for (size_t l = 0; l < local; ++l) {
            getcontext(&g_items[l]);
            g_items[l].uc_stack.ss_sp = stacks[l].data();
            g_items[l].uc_stack.ss_size = stack;
            g_items[l].uc_link = &g_sched;
            makecontext(&g_items[l], trampoline, 0);
            g_state[l] = 0;
        }
        for (;;) {
            size_t waiting = 0, finished = 0;
            for (size_t l = 0; l < local; ++l) {
                if (g_state[l] == 2) continue;
                g_state[l] = 0;
                g_item = (int)l;
                cur = Item{grp * local + l, l, grp, local, global};
                swapcontext(&g_sched, &g_items[l]);
            }
            for (size_t l = 0; l < local; ++l) (g_state[l] == 2 ? finished : waiting)++;
            if (finished == local) break;
            if (finished != 0) abort();  // some items passed a barrier the others never reach
            (void)waiting;
        }
        g_item = -1;
    }
}
}  // namespace

void barrier_wait() {
    if (g_item < 0) abort();  // a barrier in a kernel launched without group emulation
    g_state[g_item] = 1;
    swapcontext(&g_items[g_item], &g_sched);
}
}  // namespace clemu

// n bodies (positions xyz interleaved, masses), bounding half-sizes bd[3].
// Outputs: codes[i] the 30-bit code gen_mortons gives body i; sorted_codes and
// perm: the first n entries of the bitonic sort's output (code, body index);
// left, right, parent: 2n - 1 node links from build_tree (leaves 0..n-1,
// internal node i at n + i, root n, -1 none). Returns 0, or -1 for n < 2.
extern "C" int refcl_build(long n, const double* pos, const double* mass, const double* bd, uint32_t* codes,
                           uint32_t* sorted_codes, int32_t* perm, int32_t* left, int32_t* right, int32_t* parent) {
    using namespace clemu;
    if (n < 2) return -1;
    const size_t LOCAL_SIZE = 128;  // full_GPU.cpp:32
    uint msize = 128;
    while (msize < (uint)n) msize *= 2;
    // a fresh buffer: the entries past n read as zero (gen_mortons writes [0, n) only)
    std::vector<ulong> mortons(msize, 0), sorted(msize, 0);
    const int N = (int)n;
    run_flat(round_up((size_t)n, LOCAL_SIZE), LOCAL_SIZE,
             [&] { clk_morton::gen_mortons((uint)n, pos, mortons.data(), bd, 0, N); });
    for (long i = 0; i < n; ++i) codes[i] = (uint32_t)(mortons[i] & 0xffffffffu);
    run_groups(round_up(msize / 2, LOCAL_SIZE), LOCAL_SIZE,
               [&] { clk_radix::Sort_BitonicMergesortStart(mortons.data(), sorted.data(), msize); });
    for (uint blocksize = 2 * LOCAL_SIZE; blocksize <= msize; blocksize <<= 1)
        for (uint stride = blocksize / 2; stride > 0; stride >>= 1)
            run_flat(round_up(msize, LOCAL_SIZE), LOCAL_SIZE,
                     [&] { clk_radix::Sort_BitonicMergesortGlobal(sorted.data(), msize, blocksize, stride); });
    for (long i = 0; i < n; ++i) {
        sorted_codes[i] = (uint32_t)(sorted[i] & 0xffffffffu);
        perm[i] = (int32_t)(sorted[i] >> 32);
    }
    const size_t m = 2 * (size_t)n - 1;
    std::vector<int> l(m, -1), r(m, -1), par(m, 0), counters(m, 0);  // load_buffers: children start at -1
    std::vector<double> node_pos(3 * m, 0.0), n_masses(m, 0.0);
    run_flat(round_up((size_t)n, 64), 64, [&] {
        clk_tree::build_tree(N, reinterpret_cast<const uint2*>(sorted.data()), l.data(), r.data(), node_pos.data(),
                             n_masses.data(), pos, mass, par.data(), counters.data());
    });
    for (size_t i = 0; i < m; ++i) {
        left[i] = l[i];
        right[i] = r[i];
        parent[i] = par[i];
    }
    return 0;
}
