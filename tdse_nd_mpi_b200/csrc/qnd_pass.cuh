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
    const V* ax_cplx[MAX_DIM];
    const R* ax_real[MAX_DIM];
    R scale;
    int apply_acc;
    const double* apply_vtab;
    RedDesc red;
};

// Threads-per-line, values-per-thread and lines-per-CTA for a line length.
template <typename R, int L> struct PassShape {
    static constexpr int E = L < 16 ? L : 16;
    static constexpr int T = L / E;
    static constexpr int G = T >= 256 ? 1 : 256 / T;
    static constexpr int NT = T * G;
    static constexpr bool EXCHANGE = FFTPlan<L, E>::NSTAGE > 1;
    static constexpr int LINE_PAD = sizeof(R) == 8 ? 2 : 4;  // line stride = 2 (mod 8) x16B / 4 (mod 16) x8B
    static constexpr int LS = EXCHANGE ? FFTPlan<L, E>::SMEM_LINE + LINE_PAD : 0;
    static constexpr int TWN = (FFTPlan<L, E>::tw_size() + 1) & ~1;
    static constexpr size_t SMEM = sizeof(cplx_t<R>) * (size_t(TWN) + size_t(G) * LS);
    static constexpr int MINB = SMEM * 2 <= 200 * 1024 ? 2 : 1;  // two CTAs per SM when shared memory allows
};

struct CtaSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

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
    }
    __syncthreads();
    if (t < rd.n) {
        double s = 0.0;
        for (int w = 0; w < NW; ++w) s += red_s[w][t];
        s *= rd.scale[t];
        rd.out[t] = rd.accumulate ? rd.out[t] + s : s;
    }
    if (t == 0) *rd.counter = 0u;
}

template <typename R, int L, bool STRIDED, int MODE>
__global__ void __launch_bounds__(PassShape<R, L>::NT, PassShape<R, L>::MINB) qnd_pass_kernel(const __grid_constant__ PassArgs<R> a) {
    using V = cplx_t<R>;
    using SH = PassShape<R, L>;
    constexpr int E = SH::E, T = SH::T, G = SH::G, NT = SH::NT;
    using P = FFTPlan<L, E>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* tw_s = reinterpret_cast<V*>(smem_raw);
    V* lines = tw_s + SH::TWN;

    const int t = threadIdx.x;
    const int w = STRIDED ? (t % G) : (t / T);
    const int tid = STRIDED ? (t / G) : (t % T);
    V* line = lines + w * SH::LS;
    const long long lam = (long long)blockIdx.x * G + w;
    const bool active = lam < a.nlines;
    const long long smask = (1ll << a.log2S) - 1;
    const long long base = (((lam >> a.log2S) * L) << a.log2S) + (lam & smask);

    for (int i = t; i < P::tw_size(); i += NT) tw_s[i] = a.tw[i];

    V v[E];
#pragma unroll
    for (int u = 0; u < E; ++u) {
        const long long flat = base + ((long long)(tid + u * T) << a.log2S);
        v[u] = active ? a.psi[flat] : V{R(0), R(0)};
    }

    if constexpr (MODE == PM_SANDWICH) {
        if (active && (a.pro_real || a.pro_cplx || a.pro_scale_dev)) {
            const R sc = a.pro_scale_dev ? R(*a.pro_scale_dev) : R(1);
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const long long flat = base + ((long long)(tid + u * T) << a.log2S);
                V x = v[u];
                if (a.pro_real) x = cscale(x, a.pro_real[flat]);
                if (a.pro_cplx) x = cmul(x, a.pro_cplx[flat]);
                if (a.pro_scale_dev) x = cscale(x, sc);
                v[u] = x;
            }
        }
    }
    __syncthreads();  // twiddles visible

    CtaSync sync;
    if constexpr (MODE == PM_FFT_INV) {
        fft_line_stages<L, E, +1, 0>(v, tid, line, tw_s, sync);
    } else {
        fft_line_stages<L, E, -1, 0>(v, tid, line, tw_s, sync);
    }

    double acc[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;

    if constexpr (MODE == PM_FFT_FWD || MODE == PM_FFT_INV) {
        if (active) {
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const long long flat = base + ((long long)(tid + u * T) << a.log2S);
                a.psi[flat] = cscale(v[u], a.scale);
            }
        }
        return;
    } else if constexpr (MODE == PM_SPECRED) {
        if (active) {
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const long long flat = base + ((long long)(tid + u * T) << a.log2S);
                accumulate_red<R>(a.red, acc, v[u], a.partner, flat, a.shift, a.nmask);
            }
        }
        finish_red<NT>(a.red, acc);
        return;
    } else {
        // SANDWICH and APPLY: spectral multiply then the inverse transform
        if (a.spec) {
#pragma unroll
            for (int u = 0; u < E; ++u) v[u] = cmul(v[u], a.spec[tid + u * T]);
        }
        fft_line_stages<L, E, +1, 0>(v, tid, line, tw_s, sync);
        if (active) {
#pragma unroll
            for (int u = 0; u < E; ++u) {
                const long long flat = base + ((long long)(tid + u * T) << a.log2S);
                V x = v[u];
                if constexpr (MODE == PM_SANDWICH) {
                    if (a.epi_real) x = cscale(x, a.epi_real[flat]);
                    if (a.epi_cplx) x = cmul(x, a.epi_cplx[flat]);
#pragma unroll
                    for (int k = 0; k < MAX_DIM; ++k) {
                        if (k >= a.dim) break;
                        const long long ik = (flat >> a.shift[k]) & a.nmask[k];
                        if (a.ax_cplx[k]) x = cmul(x, a.ax_cplx[k][ik]);
                        if (a.ax_real[k]) x = cscale(x, a.ax_real[k][ik]);
                    }
                    if (a.red.n) accumulate_red<R>(a.red, acc, x, a.partner, flat, a.shift, a.nmask);
                    a.psi[flat] = x;
                } else {  // PM_APPLY
                    if (a.apply_vtab) {
                        const V p = a.psi[flat];
                        const R vv = R(a.apply_vtab[flat]);
                        x = cadd(x, cscale(p, vv));
                    }
                    if (a.apply_acc) x = cadd(x, a.dst[flat]);
                    if (a.red.n) accumulate_red<R>(a.red, acc, x, a.partner, flat, a.shift, a.nmask);
                    if (a.dst) a.dst[flat] = x;
                }
            }
        }
        if (a.red.n) finish_red<NT>(a.red, acc);
    }
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
