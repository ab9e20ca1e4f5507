// qnd_pass.cuh — the fused axis pass: every line of the N-D state along one axis
// is read once from HBM, transformed in registers/shared memory, combined with its
// phase tables and written once. All hot-path work is a sequence of these passes.
//
// State layout: row-major, axis 0 slowest (meshgrid.c:205-211). For the pass axis
// with length L and stride S (the product of the later axes' lengths) the lines are
// lam = o*S + s, element m of line lam sits at flat = o*L*S + m*S + s. A CTA owns G
// lines: for the contiguous axis (S = 1) G whole rows; for a strided axis G
// neighbouring s values, so every global access is a run of G consecutive values.
//
// Modes
//   PM_SANDWICH  psi <- epi(x) . IFFT[ spec(k) . FFT[ pro(x) . psi ] ]   (+ reductions)
//                The split-operator kernel/potential sub-steps: one read, one write.
//   PM_DOUBLE    psi <- epi . IFFT spec2 FFT [ mid(x) . IFFT spec FFT [ pro . psi ] ]: two kinetic
//                sandwiches along the same axis with the r-space factor between them, still one
//                read and one write (consecutive sandwiches alternate their axis order so that
//                the last axis of one is the first axis of the next).
//
// Full-grid tables (pro/mid/epi factors, WK_GRID weights) are stored LINE-MAJOR for the pass
// axis: entry lam*L + m for element m of line lam. Reads are then coalesced on every axis; for
// the contiguous axis this is the natural layout.
//   PM_FFT_FWD / PM_FFT_INV   psi <- scale . (I)FFT[psi]   (representation changes)
//   PM_SPECRED   reductions of |FFT psi|^2 weighted by k-space tables; no write
//   PM_APPLY     u = IFFT[spec . FFT psi] (+ V psi) (+ dst); optional store into dst and
//                reductions of |u|^2 or Re(conj(partner) u)   (energy moments, Lz)
//   PM_ROUNDTRIP psi <- FFT[ mid(x) . scale . IFFT[psi] ]: the closing inverse transform of one
//                sandwich and the opening transform of the next on the strided virtual axis of a
//                long 1-D axis, with the r-space factors between (tables in natural order)
//
// Reductions are FP64 and deterministic: per-CTA partial sums, then the last CTA
// to finish (ticket counter) adds the partials in a fixed order.
#pragma once

#include <cuda.h>  // CUtensorMap (the type only; maps are encoded on the host)

#include "qnd_fft.cuh"

namespace qnd {

constexpr int MAX_RED = 8;
constexpr int MAX_DIM = 6;  // grid dimensions (the reference reads DIMENSION from its parameters)

enum : int {
    PM_SANDWICH = 0,
    PM_FFT_FWD = 1,
    PM_FFT_INV = 2,
    PM_SPECRED = 3,
    PM_APPLY = 4,
    PM_DOUBLE = 5,
    PM_ROUNDTRIP = 6,
    PM_SANDWICH_RED = 7,  // PM_SANDWICH / PM_DOUBLE with fused reductions: separate instantiations, so that
    PM_DOUBLE_RED = 8,    // the passes without reductions (most of a chain) keep their registers for the FFT;
    PM_DOUBLE_RED_END = 9,  // PM_DOUBLE_RED reduces between its sandwiches (a step boundary), _END after both
    PM_NMODES = 10
};
// The transform structure of a mode (the reducing variants share their base mode's) and whether the
// mode can carry reductions at all.
__host__ __device__ constexpr int pass_base_mode(int m) {
    return m == PM_SANDWICH_RED ? PM_SANDWICH : ((m == PM_DOUBLE_RED || m == PM_DOUBLE_RED_END) ? PM_DOUBLE : m);
}
__host__ __device__ constexpr bool pass_mode_reduces(int m) {
    return m == PM_SANDWICH_RED || m == PM_DOUBLE_RED || m == PM_DOUBLE_RED_END || m == PM_SPECRED || m == PM_APPLY;
}
// |v|^2 w, Re(conj(partner) v) w, or (element-wise grid reductions only) Im(conj(partner) v) w and
// the count of elements with a non-finite part
enum : int { RK_ABS2 = 0, RK_BILIN = 1, RK_BILIN_IM = 2, RK_NONFINITE = 3 };
enum : int { WK_ONE = 0, WK_AXIS = 1, WK_GRID = 2 }; // weight 1, table[idx_axis], line-major table

struct RedDesc {
    int n;                       // accumulators in use (0: no reduction)
    int accumulate;              // out[k] += result instead of out[k] = result
    int kind[MAX_RED];
    int wkind[MAX_RED];
    int waxis[MAX_RED];
    // WK_AXIS: the weight axis' log2 stride and index mask (set by the host from waxis, so that the
    // pass kernels index no parameter array by a run-time value)
    int wshift[MAX_RED];
    long long wmask[MAX_RED];
    const double* wtab[MAX_RED];
    double scale[MAX_RED];
    double* partials;            // [gridDim.x][MAX_RED] scratch
    unsigned int* counter;       // must be 0 at launch; the last CTA resets it
    double* out;                 // final values
};

template <typename R> struct PassArgs {
    using V = cplx_t<R>;
    V* psi;
    V* dst;
    const V* partner;
    const V* tw;
    int axis;                    // the pass axis (its index along a line is m)
    int log2S;
    long long nlines;
    int dim;
    int shift[MAX_DIM];
    long long nmask[MAX_DIM];
    const R* pro_real;
    const V* pro_cplx;
    const double* pro_scale_dev;
    const V* spec;
    int spec_full;               // spec is a full-grid table in line-major order (one row per line),
                                 // not one row shared by every line (the long-axis four-step pass)
    const V* spec2;              // PM_DOUBLE: the second sandwich's spectral factors
    const R* mid_real;           // PM_DOUBLE: r-space factors between the two sandwiches
    const V* mid_cplx;
    const V* mid_ax_cplx[MAX_DIM];
    const R* mid_ax_real[MAX_DIM];  // PM_DOUBLE: per-axis real factors between the sandwiches (step mask)
    int red_at_mid;                 // PM_DOUBLE: reduce the state between the sandwiches, not at the end
    const R* epi_real;
    const V* epi_cplx;
    const V* ax_cplx[MAX_DIM];   // per-axis factors (laser phases, step mask) applied ...
    const R* ax_real[MAX_DIM];
    int ax_in_prologue;          // complex factors before the forward transform (1) or after the inverse
                                 // (0); real factors (the step mask) always after the inverse
    R scale;
    int apply_acc;
    unsigned seed;               // FP32: the random stream of the stochastic rounding (one per launch)
    const double* apply_vtab;
    RedDesc red;
    // strided passes: the state as a 3-D tensor {contiguous sub-index, pass axis, outer} for TMA box
    // loads of a CTA's G lines, read by the SK = 2 instantiations (use_tma records the host's choice);
    // err: set when a wait for those loads runs out
    int use_tma;
    int* err;
    int tma_wait_tries;          // tries of the bounded wait for those loads before the CTA gives up
    int red_lm;                  // grid reductions: full-grid weights in the line-major order of `axis`
    CUtensorMap tmap;
};

// Threads-per-line, values-per-thread and lines-per-CTA for a line length.
//   E = 16 values per thread in registers (L itself up to 16 points; 32 values per thread, one
//   warp per 1024-point line, measured slower: WIDE). T = L/E threads per line; a CTA of NT = T*G
//   threads owns G lines. Lines along a strided axis are staged through shared memory, by
//   per-thread cp.async copies or by TMA boxes (the kernel's SK), so that the global accesses run
//   over G neighbouring lines; the stage buffer is then the exchange space.
//
// Shape variants VAR (the tile-shape autotuner picks one per geometry by timing, shape_choice in
// qnd_engine.cu): 0 the default, 1 half the lines per CTA (smaller CTAs, more of them per SM),
// 2 twice the lines per CTA (256-thread CTAs), 3 seven lines per CTA at L = 1024 (448 threads, one
// CTA per SM: a 1024-line pass then runs as 147 CTAs, 7 lines on every SM, where 2-line CTAs leave
// some SMs 8 lines and others 6). Variants exist for the two-sandwich and sandwich passes of lines
// of 256 to 2048 points; VALID says whether a variant differs from the default.
constexpr int NSHAPES = 4;
template <typename R, int L, int VAR = 0> struct PassShape {
    // FP64, L >= 1024: 32 values per thread (two radix-32 stages at L = 1024), one CTA per line, a
    // single warp per line at L = 1024 (warp-synchronous exchanges). Otherwise 16 values per thread
    // and 128-thread CTAs holding several lines.
    static constexpr bool WIDE = false;  // 32 values per thread for long FP64 lines: measured slower (too few warps per SM)
    static constexpr int E = L <= 16 ? L : (WIDE ? 32 : 16);
    static constexpr int T = L / E;
    static constexpr int G0 = WIDE ? 1 : (T >= 128 ? 1 : 128 / T);
    static constexpr int G = VAR == 1 ? (G0 > 1 ? G0 / 2 : 1) : (VAR == 2 ? 2 * G0 : (VAR == 3 ? 7 : G0));
    static constexpr bool VALID =
        VAR == 0 || (VAR == 3 ? (L == 1024 && T == 64)
                              : (L >= 256 && L <= 2048 && (VAR == 1 ? G0 > 1 : (T > 32 ? G <= 15 : true))));
    static constexpr int NT = T * G;
    static constexpr bool EXCHANGE = FFTPlan<L, E>::NSTAGE > 1;
    static constexpr int SLOTS = sizeof(R) == 8 ? 8 : 16;  // element slots per bank cycle (16 B / 8 B values)
    // line stride: the G lines touched in one bank cycle of the staging copy land on distinct slots
    static constexpr int LS_TARGET = G >= SLOTS ? 1 : SLOTS / G;
    static constexpr int LINE_RAW = FFTPlan<L, E>::SMEM_LINE;
    static constexpr int LS = LINE_RAW + ((LS_TARGET - LINE_RAW % SLOTS) % SLOTS + SLOTS) % SLOTS;
    // stage twiddle entries: FP64 plans keep one base per butterfly position (pow_twiddles)
    static constexpr int TW_ENTRIES = sizeof(R) == 8 ? FFTPlan<L, E>::twb_size() : FFTPlan<L, E>::tw_size();
    static constexpr int TWN_RAW = (TW_ENTRIES + 1) & ~1;
    // stage twiddles in shared memory when they are small and shared by several lines of the CTA;
    // otherwise read them through L1 (one copy per SM instead of one per CTA)
    static constexpr bool TW_SMEM = G > 1 && size_t(TWN_RAW) * sizeof(cplx_t<R>) <= 16 * 1024;
    // the line buffers start on a 128-byte boundary (TMA box destinations)
    static constexpr int TWN = TW_SMEM ? ((TWN_RAW * int(sizeof(cplx_t<R>)) + 127) / 128 * 128) / int(sizeof(cplx_t<R>)) : 0;
    // the 7-line shape (one CTA per SM, shared memory to spare) keeps the spectral rows of both
    // sandwiches in shared memory: read by 7 lines each, once per CTA from L2
    static constexpr bool SPEC_SMEM = VAR == 3;
    static constexpr int SPECN = SPEC_SMEM ? 2 * L : 0;
    static constexpr size_t SMEM = sizeof(cplx_t<R>) * (size_t(TWN) + size_t(G) * LS + size_t(SPECN));
    // 128-thread CTAs: <= 128 registers (4 CTAs per SM) when shared memory allows; one-line CTAs
    // of L >= 1024 keep their registers (the SM holds as many lines as its register file allows)
    static constexpr int MINB_DEFAULT =
        WIDE ? 1 : (SMEM <= 54 * 1024 ? 4 : (SMEM <= 72 * 1024 ? 3 : (SMEM <= 110 * 1024 ? 2 : 1)));
    // variants: as many CTAs as 128 registers a thread and the shared memory allow
    static constexpr int MINB_REGS = 65536 / (NT * 128) > 0 ? 65536 / (NT * 128) : 1;
    static constexpr int MINB_SMEM = int((227 * 1024) / (SMEM > 0 ? SMEM : 1)) > 0 ? int((227 * 1024) / (SMEM > 0 ? SMEM : 1)) : 1;
    static constexpr int MINB = VAR == 0 ? MINB_DEFAULT : (MINB_REGS < MINB_SMEM ? MINB_REGS : MINB_SMEM);
};

// Barrier over the threads of one line: a named barrier when a line spans whole warps,
// a warp barrier when several lines share a warp.
template <int T> struct LineSync {
    int id;
    __device__ __forceinline__ void operator()() const {
        if constexpr (T > 32) {
            asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(T) : "memory");
        } else {
            __syncwarp();
        }
    }
};

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename V> __device__ __forceinline__ void cp_async_elem(V* smem_dst, const V* gsrc) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    if constexpr (sizeof(V) == 16) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
    } else {
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
    }
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

// ---- TMA box loads completing on an mbarrier (strided passes)
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int x, int y, int z) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(smem_u32(src)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// shared memory of the committed bulk stores read (the CTA may then leave; the writes complete
// before the grid does)
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// generic-proxy writes to shared memory visible to the bulk-copy (async) proxy
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Waits for phase `phase` of the barrier at most `limit` tries; false when they run out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, int limit) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename R, typename V>
__device__ __forceinline__ void accumulate_red(const RedDesc& rd, double* acc, V v, const V* partner, long long flat,
                                               long long lflat, const int* shift, const long long* nmask) {
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) {
        if (k >= rd.n) break;
        double val;
        if (rd.kind[k] == RK_ABS2) {
            val = double(v.x) * double(v.x) + double(v.y) * double(v.y);
        } else if (rd.kind[k] == RK_BILIN) {
            V p = partner[flat];
            val = double(p.x) * double(v.x) + double(p.y) * double(v.y);
        } else if (rd.kind[k] == RK_NONFINITE) {
            val = (isfinite(double(v.x)) && isfinite(double(v.y))) ? 0.0 : 1.0;
        } else {
            V p = partner[flat];
            val = double(p.x) * double(v.y) - double(p.y) * double(v.x);
        }
        const int wk = rd.wkind[k];
        if (wk == WK_AXIS) {
            const int ax = rd.waxis[k];
            val *= rd.wtab[k][(flat >> shift[ax]) & nmask[ax]];
        } else if (wk == WK_GRID) {
            val *= rd.wtab[k][lflat];
        }
        acc[k] += val;
    }
}

// Reductions over the E values a thread holds of one line (m = tid + u*T), accumulator-outer: for
// each accumulator the weights are either a per-line scalar (weight 1, or a weight along another
// axis) or a row read with stride T (a weight along the pass axis, or the line's row of a line-major
// full-grid table), so one loop serves both; |v|^2 is recomputed per accumulator (two FMAs) rather
// than held in E extra FP64 registers.
template <typename R, int E, int T>
__device__ __forceinline__ void accumulate_line(const RedDesc& rd, double* acc, const cplx_t<R>* v,
                                                const cplx_t<R>* partner, long long base, int log2S, long long lbase,
                                                int tid, int axis, const int* shift, const long long* nmask) {
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) {
        if (k >= rd.n) break;
        double sum = 0.0;
        const int wk = rd.wkind[k];
        const double* __restrict__ wt = rd.wtab[k];
        if (rd.kind[k] == RK_ABS2) {
            const double* __restrict__ row = nullptr;  // stride-T weights of this line
            double wl = 1.0;                           // or one weight for the whole line
            if (wk == WK_GRID) {
                row = wt + lbase + tid;
            } else if (wk == WK_AXIS) {
                if (rd.waxis[k] == axis) row = wt + tid;
                else wl = __ldg(wt + ((base >> rd.wshift[k]) & rd.wmask[k]));
            }
            if (row) {
#pragma unroll
                for (int u = 0; u < E; ++u) {
                    const double x = v[u].x, y = v[u].y;
                    sum = fma(fma(x, x, y * y), __ldg(row + u * T), sum);
                }
            } else {
#pragma unroll
                for (int u = 0; u < E; ++u) {
                    const double x = v[u].x, y = v[u].y;
                    sum += fma(x, x, y * y);
                }
                sum *= wl;
            }
        } else {
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const int m = tid + u * T;
                const long long flat = base + ((long long)m << log2S);
                const cplx_t<R> p = partner[flat];
                double val = double(p.x) * double(v[u].x) + double(p.y) * double(v[u].y);
                if (wk == WK_AXIS) val *= __ldg(wt + ((flat >> rd.wshift[k]) & rd.wmask[k]));
                else if (wk == WK_GRID) val *= __ldg(wt + lbase + m);
                sum += val;
            }
        }
        acc[k] += sum;
    }
}

// Warm L2 with the line-major rows a pass will read later (a full-grid table), one 128-byte
// line per request.
template <int L, int T, typename X> __device__ __forceinline__ void prefetch_row_l2(const X* row, int tid) {
    constexpr int BYTES = L * int(sizeof(X));
    constexpr int NLINES = (BYTES + 127) / 128;
    const char* p = reinterpret_cast<const char*>(row);
#pragma unroll
    for (int q = tid; q < NLINES; q += T) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + 128 * q));
}

// Block reduction of acc[0..n) into partials, then the last CTA sums the partials in order.
// blk / nblk: this CTA's group and the number of groups (the grid, or a persistent kernel's groups
// of one pass).
template <int NT>
__device__ __forceinline__ void finish_red(const RedDesc& rd, double* acc, unsigned blk, unsigned nblk) {
    constexpr int NW = NT / 32 > 0 ? NT / 32 : 1;
    __shared__ double red_s[NW][MAX_RED];
    __shared__ int is_last;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) {
        if (k >= rd.n) break;
        double s = warp_sum(acc[k]);
        if (lane == 0) red_s[wid][k] = s;
    }
    __syncthreads();
    if (t < rd.n) {
        double s = 0.0;
        for (int w = 0; w < NW; ++w) s += red_s[w][t];
        rd.partials[(long long)blk * MAX_RED + t] = s;
    }
    __threadfence();
    __syncthreads();
    if (t == 0) is_last = (atomicAdd(rd.counter, 1u) == nblk - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // every accumulator in one sweep over the partials (one round of L2 loads, one barrier): the
    // last CTA's tail is the critical path of the pass. Per accumulator the order of the sums is
    // the same as one accumulator at a time (thread-strided partials, warp sum, warps in order).
    double s[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) s[k] = 0.0;
    for (unsigned b = t; b < nblk; b += NT) {
        const double* pb = rd.partials + (long long)b * MAX_RED;
#pragma unroll
        for (int k = 0; k < MAX_RED; ++k)
            if (k < rd.n) s[k] += __ldcg(pb + k);
    }
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) {
        if (k >= rd.n) break;
        const double ws = warp_sum(s[k]);
        if (lane == 0) red_s[wid][k] = ws;
    }
    __syncthreads();
    if (t < rd.n) {
        double tot = 0.0;
        for (int w = 0; w < NW; ++w) tot += red_s[w][t];
        tot *= rd.scale[t];
        rd.out[t] = rd.accumulate ? rd.out[t] + tot : tot;
    }
    if (t == 0) *rd.counter = 0u;
}
template <int NT> __device__ __forceinline__ void finish_red(const RedDesc& rd, double* acc) {
    finish_red<NT>(rd, acc, blockIdx.x, gridDim.x);
}

// Point-wise r-space factors on the E values a thread holds of one line: a full-grid table
// (line-major: entry lbase + m), per-axis complex factors (the pass axis per element, the other
// axes once per line), per-axis real factors and a scalar.
// NAT: every table is indexed by the element's natural point index base + (m << log2S) instead of
// the line-major lbase + m and the position m along the pass axis (the strided virtual axis of a
// long 1-D axis, whose tables are in natural order).
template <typename R, int E, int T, bool NAT = false>
__device__ __forceinline__ void apply_factors(cplx_t<R>* v, int tid, long long base, long long lbase,
                                              const R* __restrict__ tr, const cplx_t<R>* __restrict__ tc,
                                              const cplx_t<R>* const* axc, const R* const* axr, int axis, int dim,
                                              const int* shift, const long long* nmask, const double* scale_dev,
                                              uint32_t key, int log2S = 0) {
    using V = cplx_t<R>;
    V lf = fone<V>();
    R lr = R(1);
    bool use_lf = false, use_lr = false;
    // the pass axis' tables picked by a compile-time index (no run-time indexing of the argument
    // arrays, which would copy them to local memory)
    const V* __restrict__ pc = nullptr;
    const R* __restrict__ pr = nullptr;
#pragma unroll
    for (int k = 0; k < MAX_DIM; ++k) {
        if (k >= dim) break;  // the grid's axes only (a 2-D pass runs two turns of the six)
        if (k == axis) {
            if (axc) pc = axc[k];
            if (axr) pr = axr[k];
            continue;
        }
        const long long ik = (base >> shift[k]) & nmask[k];
        if (axc && axc[k]) { lf = fcompose(lf, axc[k][ik]); use_lf = true; }
        if (axr && axr[k]) { lr *= axr[k][ik]; use_lr = true; }
    }
    if (scale_dev) { lr *= R(*scale_dev); use_lr = true; }
    if constexpr (sizeof(R) == 8) {
#pragma unroll
        for (int u = 0; u < E; ++u) {
            const int m = tid + u * T;
            const long long gi = NAT ? base + ((long long)m << log2S) : lbase + m;  // full-grid tables
            const long long ai = NAT ? gi : (long long)m;                           // pass-axis tables
            V x = v[u];
            if (tr) x = cscale(x, tr[gi]);
            if (tc) x = fmul(x, tc[gi]);
            if (pc) x = fmul(x, __ldg(pc + ai));
            if (pr) x = cscale(x, __ldg(pr + ai));
            if (use_lf) x = fmul(x, lf);
            if (use_lr) x = cscale(x, lr);
            v[u] = x;
        }
    } else {
        // FP32: the per-axis laser phases near the origin, where the state lives, are rotations by
        // angles ~1e-4 and take the dithered product (fmul_dither): along the pass axis the elements
        // around the axis centre (u = E/2 - 1, E/2; a compile-time choice after unrolling), and the
        // whole line when the factor of the other axes is a small rotation (a line-uniform branch).
        // The potential tables rotate by h V, far from small where the state is.
        const bool lf_small = use_lf && lf.y != 0.0f && fabsf(lf.y) < 2e-3f;
        if (lf_small) {
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const int m = tid + u * T;
                const long long gi = NAT ? base + ((long long)m << log2S) : lbase + m;
                const long long ai = NAT ? gi : (long long)m;
                V x = v[u];
                if (tr) x = cscale(x, tr[gi]);
                if (tc) x = fmul(x, tc[gi]);
                if (pc) x = (u == E / 2 - 1 || u == E / 2) ? fmul_dither(x, __ldg(pc + ai), mix32(key + uint32_t(m)))
                                                          : fmul(x, __ldg(pc + ai));
                if (pr) x = cscale(x, __ldg(pr + ai));
                x = fmul_dither(x, lf, mix32((key ^ 0x85ebca6bu) + uint32_t(m)));
                if (use_lr) x = cscale(x, lr);
                v[u] = x;
            }
        } else {
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const int m = tid + u * T;
                const long long gi = NAT ? base + ((long long)m << log2S) : lbase + m;
                const long long ai = NAT ? gi : (long long)m;
                V x = v[u];
                if (tr) x = cscale(x, tr[gi]);
                if (tc) x = fmul(x, tc[gi]);
                if (pc) x = (u == E / 2 - 1 || u == E / 2) ? fmul_dither(x, __ldg(pc + ai), mix32(key + uint32_t(m)))
                                                          : fmul(x, __ldg(pc + ai));
                if (pr) x = cscale(x, __ldg(pr + ai));
                if (use_lf) x = fmul(x, lf);
                if (use_lr) x = cscale(x, lr);
                v[u] = x;
            }
        }
    }
}

// One CTA's share of a pass: line group g of ngroups (the CTA's G lines), with the dynamic shared
// memory smem_raw. `wait` runs after the prologue (twiddles to shared memory, read-only tables to
// L2), before the state is touched: the wait for the previous pass (programmatic dependent launch
// in qnd_pass_kernel, the pass's dependency counter in the persistent sweep kernel).
// SK: 0 a contiguous axis, 1 a strided axis staged by per-thread cp.async copies, 2 a strided axis
// staged by TMA boxes (separate instantiations: each staging gets its own register allocation).
template <typename R, int L, int SK, int KMODE, int VAR = 0, typename Wait>
__device__ __forceinline__ void pass_group(const PassArgs<R>& a, long long g, unsigned ngroups,
                                           unsigned char* smem_raw, Wait wait) {
    constexpr bool STRIDED = SK != 0;
    constexpr bool TMA = SK == 2;
    constexpr int MODE = pass_base_mode(KMODE);
    constexpr bool HAS_RED = pass_mode_reduces(KMODE);
    // two-sandwich passes: reductions between the sandwiches, or after both (compile-time)
    constexpr bool RED_MID = KMODE == PM_DOUBLE_RED, RED_END = KMODE == PM_DOUBLE_RED_END;
    using V = cplx_t<R>;
    using SH = PassShape<R, L, VAR>;
    constexpr int E = SH::E, T = SH::T, G = SH::G, NT = SH::NT, LS = SH::LS;
    constexpr bool TWS = SH::TW_SMEM;
    V* tw_s = reinterpret_cast<V*>(smem_raw);   // [TWN] stage twiddles (when they fit)
    V* lines = tw_s + SH::TWN;                   // [G][LS]
    V* spec_s = lines + G * LS;                  // [2][L] spectral rows (SPEC_SMEM)

    const int t = threadIdx.x;
    const int w = t / T;  // line within the CTA (the threads of a line are consecutive)
    const int tid = t % T;
    const LineSync<T> lsync{1 + w};
    V* line = lines + w * LS;

    const long long nlines = a.nlines;
    const int log2S = a.log2S;
    const long long smask = (1ll << log2S) - 1;
    auto line_base = [&](long long lam) { return (((lam >> log2S) * L) << log2S) + (lam & smask); };
    const long long lam = g * G + w;
    const bool active = lam < nlines;
    const long long base = line_base(active ? lam : 0);
    const long long lbase = (active ? lam : 0) * L;  // line-major table offset of this line
    // stochastic-rounding stream of this line: two spectral multiplies of L elements per line
    const uint32_t key0 = mix32(a.seed) + uint32_t(lbase) * 2u;

    const V* tw = a.tw;
    if constexpr (TWS) {
        for (int i = t; i < SH::TW_ENTRIES; i += NT) tw_s[i] = a.tw[i];
        tw = tw_s;
    }
    // spectral rows to shared memory (read-only tables: before the wait for the previous pass);
    // visible after the CTA barrier that precedes the first transform
    const bool spec_row = a.spec && !a.spec_full;
    if constexpr (SH::SPEC_SMEM && (MODE == PM_DOUBLE || MODE == PM_SANDWICH)) {
        if (spec_row)
            for (int i = t; i < L; i += NT) spec_s[i] = __ldg(a.spec + i);
        if (MODE == PM_DOUBLE && a.spec2)
            for (int i = t; i < L; i += NT) spec_s[L + i] = __ldg(a.spec2 + i);
    }

    if constexpr (MODE == PM_DOUBLE || MODE == PM_SANDWICH) {
        // the read-only tables: start their journey to L2 now, before the wait for the previous
        // pass (which writes only the state), so that it overlaps that pass's tail
        if (active) {
            if (a.pro_cplx) prefetch_row_l2<L, T>(a.pro_cplx + lbase, tid);
            if (a.mid_cplx) prefetch_row_l2<L, T>(a.mid_cplx + lbase, tid);
            if (a.mid_real) prefetch_row_l2<L, T>(a.mid_real + lbase, tid);
            if (a.epi_cplx) prefetch_row_l2<L, T>(a.epi_cplx + lbase, tid);
            if (a.epi_real) prefetch_row_l2<L, T>(a.epi_real + lbase, tid);
            if constexpr (HAS_RED)
                for (int k = 0; k < a.red.n; ++k)
                    if (a.red.wkind[k] == WK_GRID) prefetch_row_l2<L, T>(a.red.wtab[k] + lbase, tid);
        }
    }

    wait();

    V v[E];
    if constexpr (STRIDED) {
        if constexpr (TMA) {
            // the CTA's G lines as L/BOXL boxes {G lines, BOXL rows} in [row][line] order, loaded by TMA
            // (the host enables this only when every group lies inside one slab of lines and the boxes
            // meet the 16-byte rules; a partial last group reads the fill value past the last line)
            __shared__ __align__(8) uint64_t tma_bar;
            __shared__ int tma_gave_up;
            constexpr int BOXL = L < 256 ? L : 256;
            const long long lam0 = g * G;
            if (t == 0) {
                mbar_init(&tma_bar, 1);
                mbar_init_fence();
                tma_gave_up = 0;
            }
            __syncthreads();
            if (t == 0) {
                mbar_expect_tx(&tma_bar, uint32_t(G * L * sizeof(V)));
                const int x = int(lam0 & smask) * int(sizeof(V) / sizeof(uint64_t));
                const int z = int(lam0 >> log2S);
#pragma unroll 1
                for (int c = 0; c < L / BOXL; ++c) tma_load_3d(lines + c * BOXL * G, &a.tmap, x, c * BOXL, z, &tma_bar);
            }
            if (!mbar_wait_bounded(&tma_bar, 0, a.tma_wait_tries)) tma_gave_up = 1;
            __syncthreads();
            if (tma_gave_up) {
                // The CTA's lines did not arrive in time (one decision for the whole CTA). Give the
                // copies in flight a second bounded wait so that none lands after the CTA has left,
                // raise the error flag, and leave the state untouched: no transform, no store. The CTA
                // still takes its ticket in the grid reduction (with nothing), so that the last CTA
                // finishes it and resets the counter.
                mbar_wait_bounded(&tma_bar, 0, 1 << 20);
                if (t == 0 && a.err) atomicExch(a.err, 1);
                if (HAS_RED && (MODE == PM_SPECRED || a.red.n)) {
                    double none[MAX_RED];
#pragma unroll
                    for (int k = 0; k < MAX_RED; ++k) none[k] = 0.0;
                    finish_red<NT>(a.red, none, unsigned(g), ngroups);
                }
                return;
            }
#pragma unroll
            for (int u = 0; u < E; ++u) v[u] = lines[(tid + u * T) * G + w];
            __syncthreads();  // every line has read its inputs before the exchanges reuse the buffer
        } else {
            // stage the CTA's G neighbouring lines: consecutive threads -> consecutive addresses
#pragma unroll 4
            for (int e = t; e < G * L; e += NT) {
                const int wl = e % G, m = e / G;
                const long long l2 = g * G + wl;
                if (l2 < nlines)
                    cp_async_elem(lines + wl * LS + spad<E>(m), a.psi + line_base(l2) + ((long long)m << log2S));
            }
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
#pragma unroll
            for (int u = 0; u < E; ++u) v[u] = active ? line[spad<E>(tid + u * T)] : V{R(0), R(0)};
        }
    } else {
        const V* __restrict__ src = a.psi;
#pragma unroll
        for (int u = 0; u < E; ++u) v[u] = active ? src[base + tid + u * T] : V{R(0), R(0)};
        if constexpr (TWS) __syncthreads();  // twiddles visible
    }

    constexpr bool PROPAGATE = MODE == PM_SANDWICH || MODE == PM_DOUBLE;
    if constexpr (PROPAGATE) {
        if (active && (a.pro_real || a.pro_cplx || a.pro_scale_dev || a.ax_in_prologue))
            apply_factors<R, E, T>(v, tid, base, lbase, a.pro_real, a.pro_cplx, a.ax_in_prologue ? a.ax_cplx : nullptr,
                                   nullptr, a.axis, a.dim, a.shift, a.nmask, a.pro_scale_dev, key0 ^ 0x51ed270bu);
    }
    if constexpr (STRIDED) {
        if constexpr (!TMA) lsync();  // staged inputs read before the exchanges reuse the buffer
    }

    double acc[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;

    if constexpr (MODE == PM_FFT_INV || MODE == PM_ROUNDTRIP) {
        fft_line_stages<L, E, +1, 0, TWS>(v, tid, line, tw, lsync);
    } else if constexpr (MODE != PM_DOUBLE) {
        fft_line_stages<L, E, -1, 0, TWS>(v, tid, line, tw, lsync);
    }

    bool store_out = false;  // write v back to psi at the end
    if constexpr (MODE == PM_FFT_FWD || MODE == PM_FFT_INV) {
#pragma unroll
        for (int u = 0; u < E; ++u) v[u] = cscale(v[u], a.scale);
        store_out = true;
    } else if constexpr (MODE == PM_ROUNDTRIP) {
#pragma unroll
        for (int u = 0; u < E; ++u) v[u] = cscale(v[u], a.scale);
        if (active)
            apply_factors<R, E, T, true>(v, tid, base, lbase, a.mid_real, a.mid_cplx, a.mid_ax_cplx, a.mid_ax_real,
                                         a.axis, a.dim, a.shift, a.nmask, nullptr, key0 ^ 0x2545f491u, log2S);
        fft_line_stages<L, E, -1, 0, TWS>(v, tid, line, tw, lsync);
        store_out = true;
    } else if constexpr (MODE == PM_SPECRED) {
        if (active) accumulate_line<R, E, T>(a.red, acc, v, a.partner, base, log2S, lbase, tid, a.axis, a.shift, a.nmask);
    } else if constexpr (MODE == PM_DOUBLE) {
        // The two sandwiches along the same axis as two turns of one loop, the r-space factor (and
        // the reductions of a step boundary) after the first: the code of each transform direction
        // exists once, so that the pass fits the instruction cache of the SM. The reducing variant
        // (one pass per step) is unrolled: its accumulators would otherwise stay live in the loop.
        constexpr int TURNS_UNROLLED = HAS_RED ? 2 : 1;
#pragma unroll TURNS_UNROLLED
        for (int half = 0; half < 2; ++half) {
            fft_line_stages<L, E, -1, 0, TWS>(v, tid, line, tw, lsync);
            const V* __restrict__ sp = half ? a.spec2 : (a.spec ? a.spec + (a.spec_full ? lbase : 0ll) : nullptr);
            if (sp) {
                const uint32_t kh = key0 + uint32_t(half * L);
                if (SH::SPEC_SMEM && (half || spec_row)) {
                    const V* sps = spec_s + (half ? L : 0);
#pragma unroll
                    for (int u = 0; u < E; ++u)
                        v[u] = fmul_spec<L>(v[u], sps[tid + u * T], kh + uint32_t(tid + u * T), u == 0 || u == E - 1);
                } else {
#pragma unroll
                    for (int u = 0; u < E; ++u)
                        v[u] = fmul_spec<L>(v[u], __ldg(sp + tid + u * T), kh + uint32_t(tid + u * T),
                                            u == 0 || u == E - 1);
                }
            }
            fft_line_stages<L, E, +1, 0, TWS>(v, tid, line, tw, lsync);
            if (half == 0) {
                if (active) {
                    apply_factors<R, E, T>(v, tid, base, lbase, a.mid_real, a.mid_cplx, a.mid_ax_cplx, a.mid_ax_real,
                                           a.axis, a.dim, a.shift, a.nmask, nullptr, key0 ^ 0x2545f491u);
                    // a step boundary inside the pass: observables of the state between the two steps
                    if (RED_MID && a.red.n)
                        accumulate_line<R, E, T>(a.red, acc, v, a.partner, base, log2S, lbase, tid, a.axis, a.shift,
                                                 a.nmask);
                }
                // finish those reductions here, so that no accumulator stays live through the second sandwich
                if constexpr (HAS_RED) {
                    if (RED_MID && a.red.n) finish_red<NT>(a.red, acc, unsigned(g), ngroups);
                    // zero again whichever branch ran (the end reductions start from zero either way):
                    // the compiler then holds no accumulator across the second sandwich
#pragma unroll
                    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;
                }
            }
        }
        if (active) {
            if (a.epi_real || a.epi_cplx || !a.ax_in_prologue)
                apply_factors<R, E, T>(v, tid, base, lbase, a.epi_real, a.epi_cplx, a.ax_in_prologue ? nullptr : a.ax_cplx,
                                       a.ax_real, a.axis, a.dim, a.shift, a.nmask, nullptr, key0 ^ 0x68e31da4u);
            else
                apply_factors<R, E, T>(v, tid, base, lbase, nullptr, nullptr, nullptr, a.ax_real, a.axis, a.dim,
                                       a.shift, a.nmask, nullptr, key0 ^ 0x68e31da4u);
            // the end of a chain of 1-D sandwich pairs: reductions of the final state
            if (RED_END && a.red.n)
                accumulate_line<R, E, T>(a.red, acc, v, a.partner, base, log2S, lbase, tid, a.axis, a.shift, a.nmask);
        }
        store_out = true;
    } else {
        // SANDWICH / APPLY: spectral multiply, inverse transform
        if (a.spec) {
            const V* __restrict__ sp = a.spec + (a.spec_full ? lbase : 0ll);
            if (SH::SPEC_SMEM && MODE == PM_SANDWICH && spec_row) {
#pragma unroll
                for (int u = 0; u < E; ++u)
                    v[u] = fmul_spec<L>(v[u], spec_s[tid + u * T], key0 + uint32_t(tid + u * T), u == 0 || u == E - 1);
            } else {
#pragma unroll
                for (int u = 0; u < E; ++u)
                    v[u] = fmul_spec<L>(v[u], __ldg(sp + tid + u * T), key0 + uint32_t(tid + u * T),
                                        u == 0 || u == E - 1);
            }
        }
        fft_line_stages<L, E, +1, 0, TWS>(v, tid, line, tw, lsync);
        if (active) {
            if constexpr (PROPAGATE) {
                if (a.epi_real || a.epi_cplx || !a.ax_in_prologue)
                    apply_factors<R, E, T>(v, tid, base, lbase, a.epi_real, a.epi_cplx,
                                           a.ax_in_prologue ? nullptr : a.ax_cplx, a.ax_real, a.axis, a.dim, a.shift,
                                           a.nmask, nullptr, key0 ^ 0x68e31da4u);
                else
                    apply_factors<R, E, T>(v, tid, base, lbase, nullptr, nullptr, nullptr, a.ax_real, a.axis, a.dim,
                                           a.shift, a.nmask, nullptr, key0 ^ 0x68e31da4u);
                if (HAS_RED && a.red.n && !a.red_at_mid)
                    accumulate_line<R, E, T>(a.red, acc, v, a.partner, base, log2S, lbase, tid, a.axis, a.shift, a.nmask);
            } else {  // PM_APPLY
#pragma unroll
                for (int u = 0; u < E; ++u) {
                    const long long flat = base + ((long long)(tid + u * T) << log2S);
                    V x = v[u];
                    if (a.apply_vtab) {
                        const V p = a.psi[flat];
                        const R vv = R(a.apply_vtab[flat]);
                        x = cadd(x, cscale(p, vv));
                    }
                    if (a.apply_acc) x = cadd(x, a.dst[flat]);
                    v[u] = x;
                }
                if (a.red.n)
                    accumulate_line<R, E, T>(a.red, acc, v, a.partner, base, log2S, lbase, tid, a.axis, a.shift, a.nmask);
                if (a.dst) {
#pragma unroll
                    for (int u = 0; u < E; ++u) a.dst[base + ((long long)(tid + u * T) << log2S)] = v[u];
                }
            }
        }
        store_out = PROPAGATE;
    }

    if (store_out) {
        if constexpr (STRIDED) {
            if (TMA && g * G + G > nlines) {
                // the last group of a pass whose line count G does not divide: its boxes were loaded
                // with the missing lines filled in, and its lines go back by plain stores (a box store
                // would reach past the tensor)
                if (active) {
#pragma unroll
                    for (int u = 0; u < E; ++u) a.psi[base + ((long long)(tid + u * T) << log2S)] = v[u];
                }
            } else if constexpr (TMA) {
                // the G lines back in [row][line] order, then one thread stores the boxes
                constexpr int BOXL = L < 256 ? L : 256;
                __syncthreads();  // every line is done with its exchange buffer
#pragma unroll
                for (int u = 0; u < E; ++u) lines[(tid + u * T) * G + w] = v[u];
                fence_proxy_async_smem();
                __syncthreads();
                if (t == 0) {
                    const long long lam0 = g * G;
                    const int x = int(lam0 & smask) * int(sizeof(V) / sizeof(uint64_t));
                    const int z = int(lam0 >> log2S);
#pragma unroll 1
                    for (int c = 0; c < L / BOXL; ++c) tma_store_3d(&a.tmap, lines + c * BOXL * G, x, c * BOXL, z);
                    bulk_commit();
                    bulk_wait_read_all();
                }
            } else {
                // park the line in shared memory, then a coalesced copy-out over the G lines
                lsync();
#pragma unroll
                for (int u = 0; u < E; ++u) line[spad<E>(tid + u * T)] = v[u];
                __syncthreads();
#pragma unroll 4
                for (int e = t; e < G * L; e += NT) {
                    const int wl = e % G, m = e / G;
                    const long long l2 = g * G + wl;
                    if (l2 < nlines) a.psi[line_base(l2) + ((long long)m << log2S)] = lines[wl * LS + spad<E>(m)];
                }
            }
        } else if (active) {
            V* __restrict__ out = a.psi;
#pragma unroll
            for (int u = 0; u < E; ++u) out[base + tid + u * T] = v[u];
        }
    }
    if constexpr (HAS_RED)
        if (MODE == PM_SPECRED || (a.red.n && (MODE == PM_DOUBLE ? RED_END : !a.red_at_mid)))
            finish_red<NT>(a.red, acc, unsigned(g), ngroups);
}

template <typename R, int L, int SK, int KMODE, int VAR = 0>
__global__ void __launch_bounds__(PassShape<R, L, VAR>::NT, PassShape<R, L, VAR>::MINB)
    qnd_pass_kernel(const __grid_constant__ PassArgs<R> a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    pass_group<R, L, SK, KMODE, VAR>(a, blockIdx.x, gridDim.x, smem_raw, [] {
        pdl_wait();
        pdl_launch_dependents();
    });
}

// Element-wise reductions over a whole state in r-space (no transform): norm, dipole,
// acceleration, potential energy of an arbitrary state.
template <typename R>
__global__ void __launch_bounds__(256) qnd_grid_reduce_kernel(const __grid_constant__ PassArgs<R> a, long long n) {
    using V = cplx_t<R>;
    double acc[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;
    const int sa = a.shift[a.axis];
    const long long L = a.nmask[a.axis] + 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long li = i;  // the index of element i in the weights' order
        if (a.red_lm) {
            const long long q = (i >> sa) & a.nmask[a.axis];
            li = ((((i >> sa) / L) << sa) | (i & ((1ll << sa) - 1))) * L + q;
        }
        accumulate_red<R>(a.red, acc, a.psi[i], a.partner, i, li, a.shift, a.nmask);
    }
    finish_red<256>(a.red, acc);
}

}  // namespace qnd
