// qnd_sweep.cu — the persistent sweep kernel: the passes of many independent propagations
// (members: grids of different sizes, integrators, precisions of one kind) in one launch.
//
// Every member's run is a sequence of fused axis passes (its sandwich chains, recorded on the host
// with the arguments the per-pass launches would get). A pass consists of line groups (a CTA's
// share in qnd_pass_kernel); one group is one work item. The items are ordered by rounds: round r
// holds pass r of every member that has one, member by member; a pass's items hold gpi groups each
// (about 64 items per pass: fewer claims and waits per unit of work). Pass r of a member
// needs all groups of its pass r - 1, which come earlier in that order, so a CTA that claims an item
// (one atomic counter, in order) depends only on items already claimed by running CTAs: the launch
// makes progress whenever its CTAs are all resident (a cooperative launch, sized by occupancy).
//
// A member's groups done so far are counted in done[member]; pass r may start once the count
// reaches the groups of passes 0 .. r-1 (need). The wait is bounded: when it runs out, or when an
// abort flag is up, the CTA skips the item (still counting it done, so that no one waits on it) and
// raises the abort flag; the host then reports the error and resets the members' reduction counters.
// No member waits for another: they only share the CTAs.
#include "qnd_kernels.cuh"

#ifndef QND_SWEEP_FP64
#error "compile with -DQND_SWEEP_FP64=1 (FP64) or 0 (FP32)"
#endif

namespace qnd {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Waits (thread 0) until done >= need; false when the tries run out or the abort flag is up.
__device__ __forceinline__ bool sweep_wait(const unsigned* done, unsigned need, const int* abort_flag, int tries) {
    for (int i = 0; i < tries; ++i) {
        if (ld_acquire_u32(done) >= need) return true;
        if (*reinterpret_cast<const volatile int*>(abort_flag)) return false;
        __nanosleep(i < 64 ? 32 : 256);
    }
    return false;
}

template <typename R, int L, bool S, int KM>
__device__ __noinline__ void sweep_run(const SweepSlot& sl, long long g, unsigned char* smem) {
    pass_group<R, L, S ? 1 : 0, KM, 0>(*static_cast<const PassArgs<R>*>(sl.args), g, sl.ngroups, smem, [] {});
}

template <typename R, int L, bool S>
__device__ __forceinline__ void sweep_dispatch_mode(const SweepSlot& sl, long long g, unsigned char* smem) {
    switch (sl.kmode) {
    case PM_SANDWICH: sweep_run<R, L, S, PM_SANDWICH>(sl, g, smem); break;
    case PM_SANDWICH_RED: sweep_run<R, L, S, PM_SANDWICH_RED>(sl, g, smem); break;
    case PM_DOUBLE: sweep_run<R, L, S, PM_DOUBLE>(sl, g, smem); break;
    case PM_DOUBLE_RED: sweep_run<R, L, S, PM_DOUBLE_RED>(sl, g, smem); break;
    case PM_DOUBLE_RED_END: sweep_run<R, L, S, PM_DOUBLE_RED_END>(sl, g, smem); break;
    default: break;  // the host records only these modes
    }
}

template <typename R, int L>
__device__ __forceinline__ void sweep_dispatch_stride(const SweepSlot& sl, long long g, unsigned char* smem) {
    if (sl.strided) sweep_dispatch_mode<R, L, true>(sl, g, smem);
    else sweep_dispatch_mode<R, L, false>(sl, g, smem);
}

// The slot holding item, the last slot whose first item is <= item, searched forward from hint (the
// slot of this CTA's previous item: items are claimed in increasing order) by doubling steps, then
// bisection: a few loads where a search over all slots takes about fifteen dependent ones.
__device__ __forceinline__ int sweep_slot_of(const SweepArgs& sa, long long item, int hint) {
    int lo = hint, hi = sa.nslots - 1, step = 1;  // first[lo] <= item
    for (;;) {
        const int probe = lo + step;
        if (probe >= sa.nslots) break;  // the answer is in [lo, nslots - 1]
        if (sa.first[probe] <= item) {
            lo = probe;
            step <<= 1;
        } else {
            hi = probe - 1;  // the answer is in [lo, probe - 1]
            break;
        }
    }
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sa.first[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <typename R>
__global__ void __launch_bounds__(SWEEP_NT, 4) qnd_sweep_kernel(const __grid_constant__ SweepArgs sa) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ long long item_s;
    __shared__ int go_s, slot_s;
    const int t = threadIdx.x;
    if (t == 0) slot_s = 0;
    for (;;) {
        __syncthreads();  // the previous item is done with the shared memory
        if (t == 0) {
            const long long item = (long long)atomicAdd(sa.next, 1ull);
            item_s = item;
            if (item < sa.nitems) slot_s = sweep_slot_of(sa, item, slot_s);
        }
        __syncthreads();
        const long long item = item_s;
        if (item >= sa.nitems) break;
        const SweepSlot& sl = sa.slots[slot_s];
        const long long g0 = (item - sa.first[slot_s]) * sl.gpi;
        const long long g1 = g0 + sl.gpi < (long long)sl.ngroups ? g0 + sl.gpi : (long long)sl.ngroups;
        if (t == 0) {
            bool ok = sweep_wait(sa.done + sl.member, sl.need, sa.abort_flag, sa.wait_tries);
            if (!ok) atomicExch(sa.abort_flag, 1);
            go_s = ok ? 1 : 0;
        }
        __syncthreads();
        if (go_s) {
            for (long long g = g0; g < g1; ++g) {
                if (g > g0) __syncthreads();  // the previous group is done with the shared memory
                switch (sl.L) {
                case 128: sweep_dispatch_stride<R, 128>(sl, g, smem); break;
                case 256: sweep_dispatch_stride<R, 256>(sl, g, smem); break;
                case 512: sweep_dispatch_stride<R, 512>(sl, g, smem); break;
                case 1024: sweep_dispatch_stride<R, 1024>(sl, g, smem); break;
                default: break;  // the host records only these lengths
                }
            }
        }
        __syncthreads();  // every store of the item issued
        if (t == 0) {
            __threadfence();
            atomicAdd(sa.done + sl.member, unsigned(g1 - g0));
        }
    }
}

template <typename R> size_t sweep_smem_bytes() {
    size_t m = PassShape<R, 128>::SMEM;
    m = std::max(m, PassShape<R, 256>::SMEM);
    m = std::max(m, PassShape<R, 512>::SMEM);
    m = std::max(m, PassShape<R, 1024>::SMEM);
    return m;
}

template <typename R> cudaError_t launch_sweep(const SweepArgs& sa, cudaStream_t st, int num_sms, int* grid_out) {
    const size_t smem = sweep_smem_bytes<R>();
    const void* fn = reinterpret_cast<const void*>(&qnd_sweep_kernel<R>);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, SWEEP_NT, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    long long grid = (long long)per_sm * num_sms;
    if (grid > sa.nitems) grid = sa.nitems;
    if (grid < 1) grid = 1;
    *grid_out = int(grid);
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(unsigned(grid));
    lc.blockDim = dim3(SWEEP_NT);
    lc.dynamicSmemBytes = smem;
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // all CTAs resident, or the launch fails
    attr[0].val.cooperative = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    void* args[] = {const_cast<SweepArgs*>(&sa)};
    return cudaLaunchKernelExC(&lc, fn, args);
}

// one precision per compilation (-DQND_SWEEP_FP64=1 or 0): the kernel holds 32 pass bodies
#if QND_SWEEP_FP64
template cudaError_t launch_sweep<double>(const SweepArgs&, cudaStream_t, int, int*);
#else
template cudaError_t launch_sweep<float>(const SweepArgs&, cudaStream_t, int, int*);
#endif

}  // namespace qnd
