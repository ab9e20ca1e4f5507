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
//   PM_FFT_FWD / PM_FFT_INV   psi <- scale . (I)FFT[psi]   (representation changes)
//   PM_SPECRED   reductions of |FFT psi|^2 weighted by k-space tables; no write
//   PM_APPLY     u = IFFT[spec . FFT psi] (+ V psi) (+ dst); optional store into dst and
//                reductions of |u|^2 or Re(conj(partner) u)   (energy moments, Lz)
//
// Reductions are FP64 and deterministic: per-CTA partial sums, then the last CTA
// to finish (ticket counter) adds the partials in a fixed order.
#pragma once

#include "qnd_fft.cuh"

namespace qnd {

constexpr int MAX_RED = 8;
constexpr int MAX_DIM = 3;

enum : int { PM_SANDWICH = 0, PM_FFT_FWD = 1, PM_FFT_INV = 2, PM_SPECRED = 3, PM_APPLY = 4, PM_NMODES = 5 };
enum : int { RK_ABS2 = 0, RK_BILIN = 1 };          // |v|^2 * w   or   Re(conj(partner) * v) * w
enum : int { WK_ONE = 0, WK_AXIS = 1, WK_GRID = 2 }; // weight 1, table[idx_axis], table[flat]

struct RedDesc {
    int n;                       // accumulators in use (0: no reduction)
    int accumulate;              // out[k] += result instead of out[k] = result
    int kind[MAX_RED];
    int wkind[MAX_RED];
    int waxis[MAX_RED];
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
    const R* epi_real;
    const V* epi_cplx;
    const V* ax_cplx[MAX_DIM];   // per-axis factors (laser phases, step mask) applied ...
    const R* ax_real[MAX_DIM];
    int ax_in_prologue;          // complex factors before the forward transform (1) or after the inverse
                                 // (0); real factors (the step mask) always after the inverse
    R scale;
    int apply_acc;
    const double* apply_vtab;
    RedDesc red;
};

// Threads-per-line, values-per-thread and lines-per-CTA for a line length.
//   E values per thread in registers: 32 for L >= 1024 (two radix-32 stages, one warp per line
//   at L = 1024), else 16. T = L/E threads per line; a CTA of NT = T*G threads owns G lines.
//   Lines along a strided axis are staged through shared memory with cp.async so that the
//   global accesses run over G neighbouring lines; the stage buffer is then the exchange space.
template <typename R, int L> struct PassShape {
    static constexpr int E = L <= 16 ? L : 16;
    static constexpr int T = L / E;
    static constexpr int G = T >= 128 ? 1 : 128 / T;
    static constexpr int NT = T * G;
    static constexpr bool EXCHANGE = FFTPlan<L, E>::NSTAGE > 1;
    static constexpr int SLOTS = sizeof(R) == 8 ? 8 : 16;  // element slots per bank cycle (16 B / 8 B values)
    // line stride: the G lines touched in one bank cycle of the staging copy land on distinct slots
    static constexpr int LS_TARGET = G >= SLOTS ? 1 : SLOTS / G;
    static constexpr int LINE_RAW = FFTPlan<L, E>::SMEM_LINE;
    static constexpr int LS = LINE_RAW + ((LS_TARGET - LINE_RAW % SLOTS) % SLOTS + SLOTS) % SLOTS;
    static constexpr int TWN_RAW = (FFTPlan<L, E>::tw_size() + 1) & ~1;
    static constexpr bool TW_SMEM = size_t(TWN_RAW) * sizeof(cplx_t<R>) <= 16 * 1024;  // stage twiddles in smem
    static constexpr int TWN = TW_SMEM ? TWN_RAW : 0;
    static constexpr size_t SMEM = sizeof(cplx_t<R>) * (size_t(TWN) + size_t(G) * LS);
    // 128 threads per CTA and <= 128 registers per thread: 4 CTAs (16 warps) per SM when shared memory allows
    static constexpr int MINB = SMEM <= 54 * 1024 ? 4 : (SMEM <= 72 * 1024 ? 3 : (SMEM <= 110 * 1024 ? 2 : 1));
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
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <typename R, typename V>
__device__ __forceinline__ void accumulate_red(const RedDesc& rd, double* acc, V v, const V* partner, long long flat,
                                               const int* shift, const long long* nmask) {
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) {
        if (k >= rd.n) break;
        double val;
        if (rd.kind[k] == RK_ABS2) {
            val = double(v.x) * double(v.x) + double(v.y) * double(v.y);
        } else {
            V p = partner[flat];
            val = double(p.x) * double(v.x) + double(p.y) * double(v.y);
        }
        const int wk = rd.wkind[k];
        if (wk == WK_AXIS) {
            const int ax = rd.waxis[k];
            val *= rd.wtab[k][(flat >> shift[ax]) & nmask[ax]];
        } else if (wk == WK_GRID) {
            val *= rd.wtab[k][flat];
        }
        acc[k] += val;
    }
}

// Block reduction of acc[0..n) into partials, then the last CTA sums the partials in order.
template <int NT>
__device__ __forceinline__ void finish_red(const RedDesc& rd, double* acc) {
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
        rd.partials[(long long)blockIdx.x * MAX_RED + t] = s;
    }
    __threadfence();
    __syncthreads();
    if (t == 0) is_last = (atomicAdd(rd.counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    for (int k = 0; k < rd.n; ++k) {
        double s = 0.0;
        for (unsigned b = t; b < gridDim.x; b += NT) s += __ldcg(rd.partials + (long long)b * MAX_RED + k);
        s = warp_sum(s);
        if (lane == 0) red_s[wid][k] = s;
        __syncthreads();
        if (t == 0) {
            double tot = 0.0;
            for (int w = 0; w < NW; ++w) tot += red_s[w][k];
            tot *= rd.scale[k];
            rd.out[k] = rd.accumulate ? rd.out[k] + tot : tot;
        }
        __syncthreads();
    }
    if (t == 0) *rd.counter = 0u;
}

template <typename R, int L, bool STRIDED, int MODE>
__global__ void __launch_bounds__(PassShape<R, L>::NT, PassShape<R, L>::MINB)
    qnd_pass_kernel(const __grid_constant__ PassArgs<R> a) {
    using V = cplx_t<R>;
    using SH = PassShape<R, L>;
    constexpr int E = SH::E, T = SH::T, G = SH::G, NT = SH::NT, LS = SH::LS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tw_s = reinterpret_cast<V*>(smem_raw);   // [TWN] stage twiddles (when they fit)
    V* lines = tw_s + SH::TWN;                   // [G][LS]

    const int t = threadIdx.x;
    const int w = t / T;  // line within the CTA (the threads of a line are consecutive)
    const int tid = t % T;
    const LineSync<T> lsync{1 + w};
    V* line = lines + w * LS;

    const long long nlines = a.nlines;
    const int log2S = a.log2S;
    const long long smask = (1ll << log2S) - 1;
    auto line_base = [&](long long lam) { return (((lam >> log2S) * L) << log2S) + (lam & smask); };
    const long long g = blockIdx.x;
    const long long lam = g * G + w;
    const bool active = lam < nlines;
    const long long base = line_base(active ? lam : 0);
    const V* tw = a.tw;
    if constexpr (SH::TW_SMEM) {
        for (int i = t; i < FFTPlan<L, E>::tw_size(); i += NT) tw_s[i] = a.tw[i];
        tw = tw_s;
    }

    pdl_wait();
    pdl_launch_dependents();

    V v[E];
    if constexpr (STRIDED) {
        // stage the CTA's G neighbouring lines: consecutive threads -> consecutive addresses
#pragma unroll 4
        for (int e = t; e < G * L; e += NT) {
            const int wl = e % G, m = e / G;
            const long long l2 = g * G + wl;
            if (l2 < nlines) cp_async_elem(lines + wl * LS + spad<E>(m), a.psi + line_base(l2) + ((long long)m << log2S));
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
#pragma unroll
        for (int u = 0; u < E; ++u) v[u] = active ? line[spad<E>(tid + u * T)] : V{R(0), R(0)};
    } else {
        const V* __restrict__ src = a.psi;
#pragma unroll
        for (int u = 0; u < E; ++u) v[u] = active ? src[base + tid + u * T] : V{R(0), R(0)};
        if constexpr (SH::TW_SMEM) __syncthreads();  // twiddles visible
    }

    if constexpr (MODE == PM_SANDWICH) {
        if (active && (a.pro_real || a.pro_cplx || a.pro_scale_dev || a.ax_in_prologue)) {
            const R sc = a.pro_scale_dev ? R(*a.pro_scale_dev) : R(1);
            const R* __restrict__ pr = a.pro_real;
            const V* __restrict__ pc = a.pro_cplx;
            const V* __restrict__ axc = a.ax_in_prologue ? a.ax_cplx[a.axis] : nullptr;
            V lf = V{R(1), R(0)};
            R lr = R(1);
            bool use_lf = false, use_lr = false;
            if (a.ax_in_prologue) {
#pragma unroll
                for (int k = 0; k < MAX_DIM; ++k) {
                    if (k >= a.dim || k == a.axis) continue;
                    const long long ik = (base >> a.shift[k]) & a.nmask[k];
                    if (a.ax_cplx[k]) { lf = cmul(lf, a.ax_cplx[k][ik]); use_lf = true; }
                }
            }
            if (a.pro_scale_dev) { lr *= sc; use_lr = true; }
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const int m = tid + u * T;
                const long long flat = base + ((long long)m << log2S);
                V x = v[u];
                if (pr) x = cscale(x, pr[flat]);
                if (pc) x = cmul(x, pc[flat]);
                if (axc) x = cmul(x, __ldg(axc + m));
                if (use_lf) x = cmul(x, lf);
                if (use_lr) x = cscale(x, lr);
                v[u] = x;
            }
        }
    }
    if constexpr (STRIDED) lsync();  // staged inputs read before the exchanges reuse the buffer

    double acc[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;

    if constexpr (MODE == PM_FFT_INV) {
        fft_line_stages<L, E, +1, 0, SH::TW_SMEM>(v, tid, line, tw, lsync);
    } else {
        fft_line_stages<L, E, -1, 0, SH::TW_SMEM>(v, tid, line, tw, lsync);
    }

    bool store_out = false;  // write v back to psi at the end
    if constexpr (MODE == PM_FFT_FWD || MODE == PM_FFT_INV) {
#pragma unroll
        for (int u = 0; u < E; ++u) v[u] = cscale(v[u], a.scale);
        store_out = true;
    } else if constexpr (MODE == PM_SPECRED) {
        if (active) {
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const long long flat = base + ((long long)(tid + u * T) << log2S);
                accumulate_red<R>(a.red, acc, v[u], a.partner, flat, a.shift, a.nmask);
            }
        }
    } else {
        // SANDWICH and APPLY: spectral multiply, inverse transform
        if (a.spec) {
            const V* __restrict__ sp = a.spec;
#pragma unroll
            for (int u = 0; u < E; ++u) v[u] = cmul(v[u], __ldg(sp + tid + u * T));
        }
        fft_line_stages<L, E, +1, 0, SH::TW_SMEM>(v, tid, line, tw, lsync);
        if (active) {
            if constexpr (MODE == PM_SANDWICH) {
                const R* __restrict__ er = a.epi_real;
                const V* __restrict__ ec = a.epi_cplx;
                const V* __restrict__ axc = a.ax_in_prologue ? nullptr : a.ax_cplx[a.axis];
                const R* __restrict__ axr = a.ax_real[a.axis];
                V lf = V{R(1), R(0)};
                R lr = R(1);
                bool use_lf = false, use_lr = false;
#pragma unroll
                for (int k = 0; k < MAX_DIM; ++k) {
                    if (k >= a.dim || k == a.axis) continue;
                    const long long ik = (base >> a.shift[k]) & a.nmask[k];
                    if (a.ax_cplx[k] && !a.ax_in_prologue) { lf = cmul(lf, a.ax_cplx[k][ik]); use_lf = true; }
                    if (a.ax_real[k]) { lr *= a.ax_real[k][ik]; use_lr = true; }
                }
#pragma unroll
                for (int u = 0; u < E; ++u) {
                    const int m = tid + u * T;
                    const long long flat = base + ((long long)m << log2S);
                    V x = v[u];
                    if (er) x = cscale(x, er[flat]);
                    if (ec) x = cmul(x, ec[flat]);
                    if (axc) x = cmul(x, __ldg(axc + m));
                    if (axr) x = cscale(x, __ldg(axr + m));
                    if (use_lf) x = cmul(x, lf);
                    if (use_lr) x = cscale(x, lr);
                    v[u] = x;
                }
                if (a.red.n) {
#pragma unroll
                    for (int u = 0; u < E; ++u) {
                        const long long flat = base + ((long long)(tid + u * T) << log2S);
                        accumulate_red<R>(a.red, acc, v[u], a.partner, flat, a.shift, a.nmask);
                    }
                }
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
                if (a.red.n) {
#pragma unroll
                    for (int u = 0; u < E; ++u) {
                        const long long flat = base + ((long long)(tid + u * T) << log2S);
                        accumulate_red<R>(a.red, acc, v[u], a.partner, flat, a.shift, a.nmask);
                    }
                }
                if (a.dst) {
#pragma unroll
                    for (int u = 0; u < E; ++u) a.dst[base + ((long long)(tid + u * T) << log2S)] = v[u];
                }
            }
        }
        store_out = MODE == PM_SANDWICH;
    }

    if (store_out) {
        if constexpr (STRIDED) {
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
        } else if (active) {
            V* __restrict__ out = a.psi;
#pragma unroll
            for (int u = 0; u < E; ++u) out[base + tid + u * T] = v[u];
        }
    }
    if (MODE == PM_SPECRED || a.red.n) finish_red<NT>(a.red, acc);
}

// Element-wise reductions over a whole state in r-space (no transform): norm, dipole,
// acceleration, potential energy of an arbitrary state.
template <typename R>
__global__ void __launch_bounds__(256) qnd_grid_reduce_kernel(const __grid_constant__ PassArgs<R> a, long long n) {
    using V = cplx_t<R>;
    double acc[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        accumulate_red<R>(a.red, acc, a.psi[i], a.partner, i, a.shift, a.nmask);
    finish_red<256>(a.red, acc);
}

}  // namespace qnd
