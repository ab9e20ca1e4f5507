// qnd_fft.cuh — in-CTA power-of-two FFT building blocks for sm_100a.
//
// A line of L complex values is spread over T = L/E threads, E values per
// thread in registers. The transform is a Stockham autosort FFT (the
// formulation of Govindaraju et al., "High Performance Discrete Fourier
// Transforms on Graphics Processors", SC'08): stage k with radix R and span Ns
// reads x[j + r*L/R], twiddles by W_{Ns*R}^{(j mod Ns)*r}, does an R-point DFT in
// registers and writes to (j/Ns)*Ns*R + (j mod Ns) + r*Ns. Between stages data is
// exchanged through shared memory with a padded layout (one 16-element pad per
// 16 values) that keeps the exchanges free of bank conflicts.
//
// Two facts make the fused passes cheap:
//  * the first stage reads x[tid + r*T] and the last stage writes
//    x[tid + r*T]: global loads/stores are coalesced straight to/from registers;
//  * the last forward stage and the first inverse stage hold the same elements
//    in the same registers, so a spectral multiply between them needs no
//    shared-memory round trip.
//
// Sign convention is FFTW's: forward exp(-2*pi*i*k*n/L), inverse exp(+...), both
// unnormalised (the reference's plans, meshgrid.c:166-167).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

namespace qnd {

template <typename R> struct cvec;
template <> struct cvec<double> { using T = double2; };
template <> struct cvec<float> { using T = float2; };
template <typename R> using cplx_t = typename cvec<R>::T;

template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return V{a.x + b.x, a.y + b.y}; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return V{a.x - b.x, a.y - b.y}; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
    return V{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
// a * conj(b)
template <typename V> __device__ __forceinline__ V cmulc(V a, V b) {
    return V{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
}
template <typename V, typename S> __device__ __forceinline__ V cscale(V a, S s) { return V{a.x * s, a.y * s}; }

// Stored complex factors. FP64 tables hold the factor w itself. FP32 tables hold d = w - 1 (for the
// spectral tables, d = w N_axis - 1, the 1/N_axis applied as an exact power-of-two scaling): then
// x w = x + x d. A near-unit factor (a small phase: the entries that a smooth state weights most)
// rounded as d keeps its magnitude exact to a few units in the last place of d rather than of 1,
// which removes the systematic FP32 norm drift that rounding w itself leaves (about 1e-7 per BM4
// step). The product costs the same four fused multiply-adds as cmul.
template <typename V> __device__ __forceinline__ V fmul(V x, V f) {
    if constexpr (sizeof(x.x) == 8) {
        return cmul(x, f);
    } else {
        return V{fmaf(x.x, f.x, fmaf(-x.y, f.y, x.x)), fmaf(x.x, f.y, fmaf(x.y, f.x, x.y))};
    }
}
// The factor of a product of two stored factors, in the same representation.
template <typename V> __device__ __forceinline__ V fcompose(V f, V g) {
    if constexpr (sizeof(f.x) == 8) {
        return cmul(f, g);
    } else {
        return cadd(cadd(f, g), cmul(f, g));
    }
}
// The stored representation of the factor 1.
template <typename V> __device__ __forceinline__ V fone() {
    if constexpr (sizeof(V{}.x) == 8) return V{1.0, 0.0};
    else return V{0.0f, 0.0f};
}
// 32 well-mixed bits from a counter (an integer hash: xor-shift / multiply rounds).
__device__ __forceinline__ uint32_t mix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}

// A uniform dither in [-1/2, 1/2) units in the last place of t (16 random bits); 0 for |t| below
// 2^-102, where it no longer matters.
__device__ __forceinline__ float dither_ulp(float t, uint32_t r16) {
    // branch-free (a select), so that the table loads around it stay batched
    const uint32_t eb = __float_as_uint(t) & 0x7f800000u;
    const float ulp = __uint_as_float(eb > (24u << 23) ? eb - (23u << 23) : 0u);
    return (float(r16) * (1.0f / 65536.0f) - 0.5f) * ulp;
}

// FP32 x (1 + d) with the second-order parts (x d_re: for a rotation by a small angle a,
// d_re = cos a - 1 ~ -a^2/2) added under a dither of one unit in the last place. A rotation by an
// angle below ~3e-4 changes the magnitude by less than half a unit in the last place, so nearest
// rounding would drop that change at every application; the dithered sum keeps it on average (an
// unbiased rounding), leaving a zero-mean error in place of a systematic drift of the norm.
__device__ __forceinline__ float2 fmul_dither(float2 x, float2 d, uint32_t h) {
    const float tr = fmaf(-x.y, d.y, x.x);
    const float ti = fmaf(x.x, d.y, x.y);
    return float2{tr + fmaf(x.x, d.x, dither_ulp(tr, h & 0xffffu)), ti + fmaf(x.y, d.x, dither_ulp(ti, h >> 16))};
}

// Multiply by a stored spectral factor of an axis of length L. In FP32 the entries of the lowest
// momenta (|k| < L/E, `low`; after unrolling a compile-time choice) take the dithered product:
// their spectral phases, which dominate a smooth state, are rotations by angles below 3e-4 for the
// usual time steps. `key` identifies the element and the call.
template <int L, typename V> __device__ __forceinline__ V fmul_spec(V x, V f, uint32_t key, bool low) {
    if constexpr (sizeof(x.x) == 8) {
        return cmul(x, f);
    } else {
        return cscale(low ? fmul_dither(x, f, mix32(key)) : fmul(x, f), 1.0f / float(L));
    }
}

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }

// Correctly rounded cos(k*pi/16), k = 0..8 (exact mathematical constants; sin(k*pi/16) = cos((8-k)*pi/16)).
__host__ __device__ constexpr double cos_pi16(int k) {
    return k == 0 ? 1.0
         : k == 1 ? 0.9807852804032304
         : k == 2 ? 0.9238795325112867
         : k == 3 ? 0.8314696123025452
         : k == 4 ? 0.7071067811865476
         : k == 5 ? 0.5555702330196022
         : k == 6 ? 0.3826834323650898
         : k == 7 ? 0.19509032201612828
         : 0.0;
}

// Multiply a by exp(SIGN * 2*pi*i*K/N) for N <= 32, with the trivial angles special-cased.
template <int N, int K, int SIGN, typename V> __device__ __forceinline__ V twiddle_const(V a) {
    using S = decltype(a.x);
    static_assert(32 % N == 0, "twiddle_const handles N <= 32");
    constexpr int k = ((K % N) + N) % N;
    constexpr int e = k * (32 / N);  // angle in units of 2*pi/32
    if constexpr (e == 0) {
        return a;
    } else if constexpr (e == 16) {
        return V{-a.x, -a.y};
    } else if constexpr (e == 8 || e == 24) {
        // exp(+-i*pi/2) = +-i ; (x+iy)*i = -y+ix
        constexpr int s = (e == 8 ? 1 : -1) * SIGN;
        if constexpr (s > 0) return V{-a.y, a.x};
        else return V{a.y, -a.x};
    } else {
        constexpr int r = e % 8, quad = e / 8;
        constexpr double c0 = cos_pi16(r), s0 = cos_pi16(8 - r);
        // rotate (c0, s0) by quad * pi/2
        constexpr double c = quad == 0 ? c0 : (quad == 1 ? -s0 : (quad == 2 ? -c0 : s0));
        constexpr double sn = quad == 0 ? s0 : (quad == 1 ? c0 : (quad == 2 ? -s0 : -c0));
        if constexpr (sizeof(S) == 4) {
            // A float pair (cos, sin) has |w|^2 != 1 by a fixed amount, and since the same constants
            // are used in every butterfly that bias would accumulate into a steady drift of the norm.
            // Apply each constant as hi + lo (double-float) so the product is accurate to well below
            // float rounding; the remaining error is the unbiased rounding of the result.
            constexpr float chi = float(c), clo = float(c - double(float(c)));
            constexpr double sd = SIGN * sn;
            constexpr float shi = float(sd), slo = float(sd - double(float(sd)));
            const float re = __fmaf_rn(a.x, chi, __fmaf_rn(-a.y, shi, a.x * clo - a.y * slo));
            const float im = __fmaf_rn(a.x, shi, __fmaf_rn(a.y, chi, a.x * slo + a.y * clo));
            return V{re, im};
        } else {
            const S cw = S(c), sw = S(SIGN * sn);
            return V{a.x * cw - a.y * sw, a.x * sw + a.y * cw};
        }
    }
}

// In-register R-point DFT (natural order in and out), radix-2 decimation in time.
template <int R, int SIGN> struct RegDFT {
    template <typename V, int... K>
    __device__ __forceinline__ static void combine(V* v, const V* e, const V* o, std::integer_sequence<int, K...>) {
        ((void)([&] {
             V t = twiddle_const<R, K, SIGN>(o[K]);
             v[K] = cadd(e[K], t);
             v[K + R / 2] = csub(e[K], t);
         }()),
         ...);
    }
    template <typename V> __device__ __forceinline__ static void run(V* v) {
        V e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; ++i) {
            e[i] = v[2 * i];
            o[i] = v[2 * i + 1];
        }
        RegDFT<R / 2, SIGN>::run(e);
        RegDFT<R / 2, SIGN>::run(o);
        combine(v, e, o, std::make_integer_sequence<int, R / 2>{});
    }
};
template <int SIGN> struct RegDFT<1, SIGN> {
    template <typename V> __device__ __forceinline__ static void run(V*) {}
};
template <int SIGN> struct RegDFT<2, SIGN> {
    template <typename V> __device__ __forceinline__ static void run(V* v) {
        V a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

// Shared-memory index with one pad slot per E values (E = values per thread): the first stage
// writes E*tid + r, which the pad spreads over consecutive banks.
template <int E> __device__ __forceinline__ int spad(int i) { return i + (i >> ilog2(E)); }

// Compile-time description of the stage sequence for a length-L line with E values per thread.
template <int L, int E> struct FFTPlan {
    static constexpr int T = L / E;                        // threads per line
    static constexpr int LOGL = ilog2(L);
    static constexpr int LOGE = ilog2(E);
    static constexpr int NSTAGE = (LOGL + LOGE - 1) / LOGE; // ceil(LOGL / LOGE)
    __host__ __device__ static constexpr int radix(int st) {
        return st < NSTAGE - 1 ? E : (1 << (LOGL - LOGE * (NSTAGE - 1)));
    }
    __host__ __device__ static constexpr int span(int st) { return st == 0 ? 1 : span(st - 1) * radix(st - 1); }
    // Offset of stage st's twiddles in the per-plan table ([j mod Ns][r-1] layout).
    __host__ __device__ static constexpr int tw_offset(int st) {
        return st <= 1 ? 0 : tw_offset(st - 1) + span(st - 1) * (radix(st - 1) - 1);
    }
    __host__ __device__ static constexpr int tw_size() { return tw_offset(NSTAGE) ; }
    // FP64 plans store one base twiddle per butterfly position, W_{Ns R}^{jm} for jm < Ns, and form
    // its powers in registers (pow_twiddles): stage st's bases start at twb_offset(st)
    __host__ __device__ static constexpr int twb_offset(int st) {
        return st <= 1 ? 0 : twb_offset(st - 1) + span(st - 1);
    }
    __host__ __device__ static constexpr int twb_size() { return twb_offset(NSTAGE); }
    static constexpr int SMEM_LINE = L + L / E;  // padded values per line (before line padding)
};

// Multiply u[1..R-1] by w^1 .. w^(R-1) with w the base twiddle of the butterfly (FP64 plans). The
// powers are formed as w^(4k + j) = w^(4k) w^j from w, w^2, w^3 and the running w^(4k) (w^4, w^8 =
// (w^4)^2, w^12 = w^8 w^4): at most four rounded products deep, about four units in the last place,
// against one shared-memory load per twiddle in the table form. Trades shared-memory bandwidth, the
// bound of the transform's exchanges, for FP64 multiplies.
template <int R, typename V> __device__ __forceinline__ void pow_twiddles(V* u, V w) {
    if constexpr (R >= 2) u[1] = cmul(u[1], w);
    if constexpr (R >= 4) {
        const V w2 = cmul(w, w);
        const V w3 = cmul(w2, w);
        u[2] = cmul(u[2], w2);
        u[3] = cmul(u[3], w3);
        const V w4 = cmul(w2, w2);
        V w4k = w4;
#pragma unroll
        for (int k = 1; k < R / 4; ++k) {
            u[4 * k] = cmul(u[4 * k], w4k);
            u[4 * k + 1] = cmul(u[4 * k + 1], cmul(w4k, w));
            u[4 * k + 2] = cmul(u[4 * k + 2], cmul(w4k, w2));
            u[4 * k + 3] = cmul(u[4 * k + 3], cmul(w4k, w3));
            if (k + 1 < R / 4) w4k = (k == 1) ? cmul(w4, w4) : cmul(w4k, w4);
        }
    }
}

// One Stockham stage on the thread's E registers (B = E/R butterflies, j = tid + b*T).
// Input registers hold x[j + r*L/R] for butterfly b at v[b*R + r]; output registers hold
// the butterfly outputs in the same slots. Twiddles come from smem table tw (forward sign).
// TWS: the twiddle table lives in shared memory (plain loads) rather than global memory
// (read-only cache loads; never use those on a shared-memory address).
template <int L, int E, int ST, int SIGN, bool TWS, typename V>
__device__ __forceinline__ void fft_stage_regs(V* v, int tid, const V* __restrict__ tw) {
    using P = FFTPlan<L, E>;
    constexpr int R = P::radix(ST);
    constexpr int Ns = P::span(ST);
    constexpr int B = E / R;
#pragma unroll
    for (int b = 0; b < B; ++b) {
        V* u = v + b * R;
        if constexpr (Ns > 1) {
            const int j = tid + b * P::T;
            const int jm = j & (Ns - 1);
            if constexpr (sizeof(u[0].x) == 8) {
                const V* t = tw + P::twb_offset(ST) + jm;
                V w;
                if constexpr (TWS) w = *t;
                else w = __ldg(t);
                if constexpr (SIGN > 0) w.y = -w.y;
                pow_twiddles<R>(u, w);
            } else {
                const V* t = tw + P::tw_offset(ST) + jm * (R - 1);
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    V w;
                    if constexpr (TWS) w = t[r - 1];
                    else w = __ldg(t + r - 1);
                    if constexpr (SIGN > 0) w.y = -w.y;
                    u[r] = fmul(u[r], w);
                }
            }
        }
        RegDFT<R, SIGN>::run(u);
    }
}

// Register slot of element index (tid + u*T) held after the LAST stage (position j + r*Ns_last,
// j = tid + b*T): u = b + r*B_last. Loading order before the FIRST stage is slot b*R0 + r for
// element j + r*L/R0 with j = tid + b*T, i.e. u = b + r*B_0. For the first stage R0 = E, B_0 = 1.
template <int L, int E> struct SlotMap {
    using P = FFTPlan<L, E>;
    static constexpr int RL = P::radix(P::NSTAGE - 1);
    static constexpr int BL = E / RL;
    // slot holding element tid + u*T after the last stage
    __host__ __device__ static constexpr int last_slot(int u) { return (u % BL) * RL + (u / BL); }
};

// Full FFT of one line held in registers: on entry v[u] = x[tid + u*T], on exit
// v[u] = X[tid + u*T] (both in natural slots). `line` is this line's padded smem
// buffer; `sync` is the CTA barrier (all lines of a CTA transform in lockstep).
// Call as fft_line_stages<L, E, SIGN, 0, TWS>(...).
template <int L, int E, int SIGN, int ST, bool TWS, typename V, typename Sync>
__device__ __forceinline__ void fft_line_stages(V* v, int tid, V* line, const V* __restrict__ tw, Sync sync) {
    using P = FFTPlan<L, E>;
    constexpr int T = P::T;
    constexpr int R = P::radix(ST);
    constexpr int Ns = P::span(ST);
    constexpr int B = E / R;
    fft_stage_regs<L, E, ST, SIGN, TWS>(v, tid, tw);
    if constexpr (ST + 1 < P::NSTAGE) {
        // Exchange: store the outputs of stage ST, load the inputs of stage ST+1. Every stride used
        // here (Ns for the stores, L/R2 for the loads) is 1 with an E-aligned base (first stage) or a
        // multiple of E, so spad(base + r*step) = spad(base) + r*(step + step/E): one padded base per
        // butterfly and compile-time offsets after it.
        constexpr int R2 = P::radix(ST + 1);
        constexpr int B2 = E / R2;
        constexpr int SP = Ns == 1 ? 1 : Ns + Ns / E;                 // padded store stride
        constexpr int LP = (L / R2) + (L / R2) / E;                   // padded load stride
        static_assert(Ns == 1 || Ns % E == 0, "stage spans are multiples of E");
        static_assert((L / R2) % E == 0, "load strides are multiples of E");
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int j = tid + b * T;
            V* p = line + spad<E>((j / Ns) * Ns * R + (j & (Ns - 1)));
#pragma unroll
            for (int r = 0; r < R; ++r) p[r * SP] = v[b * R + r];
        }
        sync();
#pragma unroll
        for (int b = 0; b < B2; ++b) {
            const V* p = line + spad<E>(tid + b * T);
#pragma unroll
            for (int r = 0; r < R2; ++r) v[b * R2 + r] = p[r * LP];
        }
        sync();
        fft_line_stages<L, E, SIGN, ST + 1, TWS>(v, tid, line, tw, sync);
    } else {
        // last stage: outputs at positions j + r*Ns (j = tid + b*T < Ns); reorder registers to
        // natural slots v[u] = X[tid + u*T].
        V tmp[E];
#pragma unroll
        for (int u = 0; u < E; ++u) tmp[u] = v[SlotMap<L, E>::last_slot(u)];
#pragma unroll
        for (int u = 0; u < E; ++u) v[u] = tmp[u];
    }
}

}  // namespace qnd
