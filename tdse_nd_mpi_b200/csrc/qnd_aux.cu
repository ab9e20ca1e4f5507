// qnd_aux.cu — small kernels around the passes: Gram-Schmidt projections
// (QuantumND_imag.c:265-311), r-space reductions, scaling, per-step field tables.
#include "qnd_kernels.cuh"

namespace qnd {

// ---- Gram-Schmidt ---------------------------------------------------------------

// c_k = sum conj(states[k]) * psi  for k in [k0, k0+nk): accumulators (re, im) pairs.
template <typename R> __global__ void __launch_bounds__(256) gs_dot_kernel(const __grid_constant__ GSArgs<R> a) {
    using V = cplx_t<R>;
    double acc[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        const V v = a.psi[i];
#pragma unroll
        for (int q = 0; q < MAX_RED / 2; ++q) {
            if (q >= a.nk) break;
            const V p = a.states[a.k0 + q][i];
            acc[2 * q] += double(p.x) * double(v.x) + double(p.y) * double(v.y);
            acc[2 * q + 1] += double(p.x) * double(v.y) - double(p.y) * double(v.x);
        }
    }
    finish_red<256>(a.red, acc);
}

// psi <- psi - sum_k c_k states[k]; accumulate |psi|^2.
template <typename R> __global__ void __launch_bounds__(256) gs_axpy_kernel(const __grid_constant__ GSArgs<R> a) {
    using V = cplx_t<R>;
    double acc[MAX_RED];
#pragma unroll
    for (int k = 0; k < MAX_RED; ++k) acc[k] = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        V v = a.psi[i];
        for (int k = 0; k < a.j; ++k) {
            const V p = a.states[k][i];
            const R cr = R(a.coef[2 * k]), ci = R(a.coef[2 * k + 1]);
            v.x -= cr * p.x - ci * p.y;
            v.y -= cr * p.y + ci * p.x;
        }
        a.psi[i] = v;
        acc[0] += double(v.x) * double(v.x) + double(v.y) * double(v.y);
    }
    finish_red<256>(a.red, acc);
}

__global__ void gs_finalize_kernel(const double* norm2, double tol, double* scale, int* flag) {
    const double n2 = *norm2;
    if (n2 < tol || !(n2 == n2)) {
        *flag = 1;
        *scale = 1.0;
    } else {
        *scale = 1.0 / sqrt(n2);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) scale_kernel(cplx_t<R>* psi, long long n, const double* scale_dev) {
    const R s = R(*scale_dev);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        cplx_t<R> v = psi[i];
        psi[i] = cplx_t<R>{v.x * s, v.y * s};
    }
}

template <typename R> void launch_gs_dot(const GSArgs<R>& a, cudaStream_t st, int nblocks) {
    gs_dot_kernel<R><<<nblocks, 256, 0, st>>>(a);
}
template <typename R> void launch_gs_axpy(const GSArgs<R>& a, cudaStream_t st, int nblocks) {
    gs_axpy_kernel<R><<<nblocks, 256, 0, st>>>(a);
}
template <typename R> void launch_grid_reduce(const PassArgs<R>& a, long long n, cudaStream_t st, int nblocks) {
    qnd_grid_reduce_kernel<R><<<nblocks, 256, 0, st>>>(a, n);
}
template <typename R> void launch_scale(cplx_t<R>* psi, long long n, const double* scale_dev, cudaStream_t st) {
    long long nb = (n + 255) / 256;
    if (nb > 148 * 8) nb = 148 * 8;
    scale_kernel<R><<<(int)nb, 256, 0, st>>>(psi, n, scale_dev);
}
void launch_gs_finalize(const double* norm2, double tol, double* scale, int* flag, cudaStream_t st) {
    gs_finalize_kernel<<<1, 1, 0, st>>>(norm2, tol, scale, flag);
}

// ---- per-step field tables ------------------------------------------------------

template <typename R>
__global__ void __launch_bounds__(256) field_tables_kernel(const __grid_constant__ FieldTableArgs a, cplx_t<R>* out) {
    const long long total = (long long)a.nsteps * a.s * a.ntot;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
        const long long blk = i / a.ntot;
        const int pos = int(i - blk * a.ntot);
        const int ia = int(blk % a.s);
        int ax = 0;
        while (ax + 1 < a.dim && pos >= a.off[ax + 1]) ++ax;
        const double f = a.field[blk * a.dim + ax];
        const double x = a.axes[pos];
        const double h = (blk / a.s) >= a.conj_from ? -a.h[ia] : a.h[ia];  // conj: the phase negated
        double theta, mag;
        if (a.velocity) {
            theta = h * (.5 * x * x + (x + .5 * f) * f);
            mag = 1.0 / double(a.nr[ax]);
        } else {
            theta = h * (x * f);
            mag = 1.0;
        }
        if constexpr (sizeof(R) == 4) {
            // FP32 factors are stored as d = e^{-i theta} - 1 (the velocity tables' 1/N is applied
            // as the spectral scaling): cos - 1 = -2 sin^2(theta/2)
            double sh, ch;
            sincos(0.5 * theta, &sh, &ch);
            out[i] = cplx_t<R>{R(-2.0 * sh * sh), R(-2.0 * sh * ch)};
        } else {
            double sn, cs;
            sincos(theta, &sn, &cs);
            out[i] = cplx_t<R>{R(mag * cs), R(-mag * sn)};
        }
    }
}

template <typename R> void launch_field_tables(const FieldTableArgs& a, cplx_t<R>* out, cudaStream_t st) {
    const long long total = (long long)a.nsteps * a.s * a.ntot;
    long long nb = (total + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    if (nb < 1) nb = 1;
    field_tables_kernel<R><<<(int)nb, 256, 0, st>>>(a, out);
}

template <typename R>
__global__ void axis_table_kernel(int mode, const double* p, int N, double alpha, void* out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        const double w = p[k] + alpha;
        if (mode == 0) {
            static_cast<double*>(out)[k] = w;
        } else {
            // a spectral factor: FP32 tables hold w N - 1 (see fmul_spec)
            static_cast<cplx_t<R>*>(out)[k] = sizeof(R) == 8 ? cplx_t<R>{R(w / double(N)), R(0)}
                                                             : cplx_t<R>{R(w - 1.0), R(0)};
        }
    }
}

template <typename R> void launch_axis_table(int mode, const double* p, int N, double alpha, void* out, cudaStream_t st) {
    axis_table_kernel<R><<<(N + 255) / 256, 256, 0, st>>>(mode, p, N, alpha, out);
}

// ---- final photoelectron spectra (io_functions.c:136-287) -------------------------

// out = f(|r|) in, f = sin^2(pi/2 (|r| - rmin)/(rmax - rmin)) between rmin and rmax, 1 beyond, 0 inside
// (io_functions.c:159-167).
template <typename R>
__global__ void __launch_bounds__(256) radial_mask_kernel(const __grid_constant__ SpectraArgs a, const cplx_t<R>* in,
                                                          cplx_t<R>* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        double r2 = 0.0;
        for (int j = 0; j < a.dim; ++j) {
            const double x = a.r[a.axoff[j] + ((i >> a.shift[j]) & a.nmask[j])];
            r2 += x * x;
        }
        const double radius = sqrt(r2);
        double f = 0.0;
        if (radius >= a.rmin && radius <= a.rmax) {
            const double sn = sin(0.5 * 3.14159265358979323846 * (radius - a.rmin) / (a.rmax - a.rmin));
            f = sn * sn;
        } else if (radius > a.rmax) {
            f = 1.0;
        }
        const cplx_t<R> v = in[i];
        out[i] = cplx_t<R>{R(double(v.x) * f), R(double(v.y) * f)};
    }
}

// Energy distribution: block b sums, for every energy bin, the Gaussian-weighted densities of its
// PED_CHUNK elements (those with every |p_j| <= pr_max_j); a second kernel adds the blocks' partial
// sums in block order (deterministic) and applies the normalisation (io_functions.c:192-199). Bins
// further than 39 sigma from an element's kinetic energy get exp(...) < 1e-330, which is zero.
template <typename R>
__global__ void __launch_bounds__(256) ped_partial_kernel(const __grid_constant__ SpectraArgs a, const cplx_t<R>* psi,
                                                          double* partials) {
    __shared__ double w_s[PED_CHUNK], k_s[PED_CHUNK];
    const long long i0 = (long long)blockIdx.x * PED_CHUNK;
    for (int c = threadIdx.x; c < PED_CHUNK; c += blockDim.x) {
        const long long i = i0 + c;
        double w = 0.0, kin = 0.0;
        if (i < a.n) {
            bool keep = true;
            for (int j = 0; j < a.dim; ++j) {
                const long long ij = (i >> a.shift[j]) & a.nmask[j];
                if (a.rank[a.axoff[j] + ij] < 0) keep = false;
                const double pj = a.p[a.axoff[j] + ij];
                kin += .5 * pj * pj;
            }
            if (keep) {
                const cplx_t<R> v = psi[i];
                const double m = sqrt(double(v.x) * double(v.x) + double(v.y) * double(v.y));
                w = m * m;
            }
        }
        w_s[c] = w;
        k_s[c] = kin;
    }
    __syncthreads();
    const double inv2s2 = .5 / (a.sigma * a.sigma), reach = 39.0 * a.sigma;
    for (int j = threadIdx.x; j < a.ne; j += blockDim.x) {
        const double e = j * a.de;
        double s = 0.0;
        for (int c = 0; c < PED_CHUNK; ++c) {
            const double d = k_s[c] - e;
            if (w_s[c] != 0.0 && fabs(d) <= reach) s += w_s[c] * exp(-d * d * inv2s2);
        }
        partials[(long long)blockIdx.x * a.ne + j] = s;
    }
}

__global__ void ped_final_kernel(const __grid_constant__ SpectraArgs a, const double* partials, int nblocks, double* out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < a.ne; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblocks; ++b) s += partials[(long long)b * a.ne + j];
        out[j] = s * a.norm;
    }
}

// Momentum distribution: (|psi~|^2, arg psi~) of the kept momenta, packed in flat order
// (io_functions.c:266-274); the kept set is a product of per-axis sets, so an element's place in the
// packed array follows from its per-axis ranks.
template <typename R>
__global__ void __launch_bounds__(256) pmd_kernel(const __grid_constant__ SpectraArgs a, const cplx_t<R>* psi,
                                                  double* out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        long long q = 0;
        bool keep = true;
        for (int j = 0; j < a.dim; ++j) {
            const int rk = a.rank[a.axoff[j] + ((i >> a.shift[j]) & a.nmask[j])];
            if (rk < 0) keep = false;
            q += (long long)rk * a.stride[j];
        }
        if (!keep) continue;
        const cplx_t<R> v = psi[i];
        const double re = v.x, im = v.y;
        const double m = sqrt(re * re + im * im);
        out[2 * q] = m * m;
        out[2 * q + 1] = atan2(im, re);
    }
}

template <typename R>
void launch_radial_mask(const SpectraArgs& a, const cplx_t<R>* in, cplx_t<R>* out, cudaStream_t st) {
    long long nb = (a.n + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    radial_mask_kernel<R><<<(int)nb, 256, 0, st>>>(a, in, out);
}
template <typename R>
void launch_ped(const SpectraArgs& a, const cplx_t<R>* psi_p, double* partials, double* out, cudaStream_t st) {
    const int nb = int((a.n + PED_CHUNK - 1) / PED_CHUNK);
    ped_partial_kernel<R><<<nb, 256, 0, st>>>(a, psi_p, partials);
    ped_final_kernel<<<(a.ne + 255) / 256, 256, 0, st>>>(a, partials, nb, out);
}
template <typename R> void launch_pmd(const SpectraArgs& a, const cplx_t<R>* psi_p, double* out, cudaStream_t st) {
    long long nb = (a.n + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    pmd_kernel<R><<<(int)nb, 256, 0, st>>>(a, psi_p, out);
}

// ---- laser field samples (integrators.c:74-101, parameters.c:899-949) -------------

// E(t) and A(t) summed over the modes: envelope f(ts) and its derivative df, ts = t - delay,
// A = F0 f (cos, xi sin)(w ts + cep) / w, E = -dA/dt (parameters.c:911-946).
__device__ void field_at(const FieldSampleArgs& a, double t, double* A, double* E) {
    const double pi = 3.14159265358979323846;
    for (int j = 0; j < a.dim; ++j) A[j] = E[j] = 0.0;
    for (int m = 0; m < a.nmodes; ++m) {
        const FieldMode& md = a.mode[m];
        const double w = md.w, ts = t - md.delay, tau = md.tau;
        double f = 0.0, df = 0.0;
        if (md.env == ENV_CONSTANT) {
            f = 1.0;
        } else if (md.env == ENV_TRAPZ) {
            const double tr = 2. * 2. * pi / w;
            const double up = (ts >= 0. && ts <= tr) ? 1. : 0., flat = (ts > tr && ts < tau - tr) ? 1. : 0.,
                         down = (ts >= tau - tr && ts <= tau) ? 1. : 0.;
            const double s1 = sin(.5 * pi * ts / tr), s2 = sin(.5 * pi * (ts - tau) / tr);
            f = pow(s1, 4) * up + flat + pow(s2, 4) * down;
            df = pi / tr * (pow(s1, 2) * sin(pi * ts / tr) * up + pow(s2, 2) * sin(pi * (ts - tau) / tr) * down);
        } else {
            const double on = (ts >= 0. && ts <= tau) ? 1. : 0.;
            const double sn = sin(pi * ts / tau);
            if (md.env == ENV_COS2) {
                f = pow(sn, 2) * on;
                df = pi * sin(2. * pi * ts / tau) / tau * on;
            } else {
                f = pow(sn, 4) * on;
                df = 4. * pi * cos(pi * ts / tau) * pow(sn, 3) / tau * on;
            }
        }
        double sp, cp;
        sincos(w * ts + md.cep, &sp, &cp);
        E[0] += -md.F0 * (df * cp - f * w * sp) / w;
        A[0] += md.F0 * f * cp / w;
        if (a.dim >= 2) {
            E[1] += -md.F0 * md.xi * (df * sp + f * w * cp) / w;
            A[1] += md.F0 * md.xi * f * sp / w;
        }
    }
}

// One thread per (step i, slot j): j < s the sub-step samples, j == s the step-start alpha.
__global__ void __launch_bounds__(256) field_samples_kernel(const __grid_constant__ FieldSampleArgs a, double* E,
                                                            double* A, double* alpha) {
    const long long total = a.nsteps * (a.s + 1);
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
        const long long i = q / (a.s + 1);
        const int j = int(q - i * (a.s + 1));
        double av[MAX_DIM], ev[MAX_DIM];
        if (j == a.s) {
            if (!alpha) continue;
            field_at(a, __dmul_rn(double(i), a.dt), av, ev);
            for (int k = 0; k < a.dim; ++k) alpha[i * a.dim + k] = av[k];
            continue;
        }
        if (!E && !A) continue;
        // the sub-step time accumulated as in integrators.c:90-99
        double t = __dadd_rn(__dmul_rn(double(i), a.dt), a.as[0]);
        for (int jj = 0; jj < j; ++jj) t = __dadd_rn(t, __dadd_rn(a.as[2 * jj + 1], a.as[2 * jj + 2]));
        field_at(a, t, av, ev);
        const long long o = (i * a.s + j) * a.dim;
        for (int k = 0; k < a.dim; ++k) {
            if (E) E[o + k] = ev[k];
            if (A) A[o + k] = av[k];
        }
    }
}

void launch_field_samples(const FieldSampleArgs& a, double* E, double* A, double* alpha, cudaStream_t st) {
    const long long total = a.nsteps * (a.s + 1);
    long long nb = (total + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    if (nb < 1) nb = 1;
    field_samples_kernel<<<int(nb), 256, 0, st>>>(a, E, A, alpha);
}

// ---- initial state: centring + superposition (io_functions.c:292-459) -------------

template <typename R>
__global__ void __launch_bounds__(256) embed_kernel(const __grid_constant__ EmbedArgs a, const double2* src,
                                                    cplx_t<R>* psi) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n_src; i += (long long)gridDim.x * blockDim.x) {
        long long idx = i, dst = 0, mult = 1;
        bool ok = true;
        for (int j = a.dim - 1; j >= 0; --j) {
            const long long ij = idx % a.nr_src[j] + a.off[j];
            idx /= a.nr_src[j];
            if (ij < 0 || ij >= a.nr[j]) ok = false;
            dst += ij * mult;
            mult *= a.nr[j];
        }
        if (!ok) continue;
        const double2 v = src[i];
        // c * v rounded per operation (no contraction), as a C99 complex product
        const double re = __dsub_rn(__dmul_rn(a.cr, v.x), __dmul_rn(a.ci, v.y));
        const double im = __dadd_rn(__dmul_rn(a.cr, v.y), __dmul_rn(a.ci, v.x));
        const cplx_t<R> p = psi[dst];
        psi[dst] = cplx_t<R>{R(__dadd_rn(double(p.x), re)), R(__dadd_rn(double(p.y), im))};
    }
}

template <typename R> void launch_embed(const EmbedArgs& a, const double2* src, cplx_t<R>* psi, cudaStream_t st) {
    long long nb = (a.n_src + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    if (nb < 1) nb = 1;
    embed_kernel<R><<<int(nb), 256, 0, st>>>(a, src, psi);
}

// ---- axes longer than one pass: the four-step pieces (qnd_engine.cu, long_fft) -------

template <typename R>
__global__ void __launch_bounds__(256) long_twiddle_kernel(long long n, cplx_t<R>* psi, const cplx_t<R>* w, int conj) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        cplx_t<R> f = w[i];
        if (conj) f.y = -f.y;  // conj(w) and, for FP32 tables, conj(w - 1) = conj(w) - 1
        psi[i] = fmul(psi[i], f);
    }
}

template <typename R>
__global__ void __launch_bounds__(256) long_transpose_kernel(LongArgs a, const cplx_t<R>* in, cplx_t<R>* out,
                                                             int to_natural) {
    const long long m2 = (1ll << a.log2n2) - 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        const long long k = (i >> a.log2n2) + ((i & m2) << a.log2n1);  // slot i holds natural index k
        if (to_natural) out[k] = in[i];
        else out[i] = in[k];
    }
}

template <typename R>
__global__ void __launch_bounds__(256) point_factors_kernel(long long n, cplx_t<R>* psi, const R* tr,
                                                            const cplx_t<R>* tc, const cplx_t<R>* pc, const R* pr,
                                                            const double* scale_dev) {
    const R sc = scale_dev ? R(*scale_dev) : R(1);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        cplx_t<R> x = psi[i];
        if (tr) x = cscale(x, tr[i]);
        if (tc) x = fmul(x, tc[i]);
        if (pc) x = fmul(x, pc[i]);
        if (pr) x = cscale(x, pr[i]);
        if (scale_dev) x = cscale(x, sc);
        psi[i] = x;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) add_potential_kernel(long long n, cplx_t<R>* dst, const cplx_t<R>* src,
                                                            const double* vtab) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = cadd(dst[i], cscale(src[i], R(vtab[i])));
}

template <typename R>
__global__ void __launch_bounds__(256) axis_factors_kernel(const __grid_constant__ AxisFactorArgs a, cplx_t<R>* psi) {
    using V = cplx_t<R>;
    const int sa = a.shift[a.axis];
    const long long smask = (1ll << sa) - 1;
    const R sc = a.scale_dev ? R(*a.scale_dev) : R(1);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        const long long q = (i >> sa) & a.nmask[a.axis];
        V x = psi[i];
        if (a.tr || a.tc) {
            const long long lam = ((i >> (sa + a.log2L)) << sa) | (i & smask);
            const long long lm = (lam << a.log2L) + q;
            if (a.tr) x = cscale(x, static_cast<const R*>(a.tr)[lm]);
            if (a.tc) x = fmul(x, static_cast<const V*>(a.tc)[lm]);
        }
        for (int k = 0; k < a.dim; ++k) {
            const long long ik = (i >> a.shift[k]) & a.nmask[k];
            if (a.axc[k]) x = fmul(x, static_cast<const V*>(a.axc[k])[ik]);
            if (a.axr[k]) x = cscale(x, static_cast<const R*>(a.axr[k])[ik]);
        }
        if (a.spec) {
            V f = static_cast<const V*>(a.spec)[q];
            if (a.spec_conj) f.y = -f.y;  // conj(w), and for FP32 tables conj(w - 1) = conj(w) - 1
            x = fmul(x, f);
            if (a.spec_scale != 1.0) x = cscale(x, R(a.spec_scale));
        }
        if (a.scale_dev) x = cscale(x, sc);
        psi[i] = x;
    }
}

template <typename R>
__global__ void __launch_bounds__(256) axis_permute_kernel(AxisPermArgs a, const cplx_t<R>* in, cplx_t<R>* out,
                                                           int to_natural) {
    const long long nm = (1ll << a.log2N) - 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += (long long)gridDim.x * blockDim.x) {
        const long long q = (i >> a.shift) & nm;
        long long src;
        if (to_natural) {  // q is the frequency k1 + n1 k2, held at slot k1 n2 + k2
            src = ((q & ((1ll << a.log2n1) - 1)) << a.log2n2) + (q >> a.log2n1);
        } else {           // q is the slot k1 n2 + k2, holding frequency k1 + n1 k2
            src = (q >> a.log2n2) + ((q & ((1ll << a.log2n2) - 1)) << a.log2n1);
        }
        out[i] = in[i + (src - q) * (1ll << a.shift)];
    }
}

template <typename R>
__global__ void __launch_bounds__(256) apply_combine_kernel(long long n, cplx_t<R>* dst, const cplx_t<R>* tmp,
                                                            const cplx_t<R>* src, const double* vtab, int acc) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        cplx_t<R> x = tmp[i];
        if (vtab) x = cadd(x, cscale(src[i], R(vtab[i])));
        if (acc) x = cadd(x, dst[i]);
        dst[i] = x;
    }
}

struct MaskArgs {
    int dim;
    int shift[MAX_DIM];
    long long nmask[MAX_DIM];
    const void* mask[MAX_DIM];
};

template <typename R>
__global__ void __launch_bounds__(256) apply_masks_kernel(long long n, cplx_t<R>* psi, const __grid_constant__ MaskArgs a) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        cplx_t<R> x = psi[i];
        for (int j = 0; j < a.dim; ++j)
            if (a.mask[j]) x = cscale(x, static_cast<const R*>(a.mask[j])[(i >> a.shift[j]) & a.nmask[j]]);
        psi[i] = x;
    }
}

static int elementwise_blocks(long long n) {
    long long nb = (n + 255) / 256;
    if (nb > 148 * 16) nb = 148 * 16;
    return int(nb < 1 ? 1 : nb);
}
template <typename R> void launch_long_twiddle(const LongArgs& a, cplx_t<R>* psi, const cplx_t<R>* w, int conj,
                                               cudaStream_t st) {
    long_twiddle_kernel<R><<<elementwise_blocks(a.n), 256, 0, st>>>(a.n, psi, w, conj);
}
template <typename R> void launch_long_transpose(const LongArgs& a, const cplx_t<R>* in, cplx_t<R>* out, int to_natural,
                                                 cudaStream_t st) {
    long_transpose_kernel<R><<<elementwise_blocks(a.n), 256, 0, st>>>(a, in, out, to_natural);
}
template <typename R> void launch_point_factors(long long n, cplx_t<R>* psi, const R* tr, const cplx_t<R>* tc,
                                                const cplx_t<R>* pc, const R* pr, const double* scale_dev,
                                                cudaStream_t st) {
    point_factors_kernel<R><<<elementwise_blocks(n), 256, 0, st>>>(n, psi, tr, tc, pc, pr, scale_dev);
}
template <typename R> void launch_apply_masks(long long n, cplx_t<R>* psi, int dim, const int* shift,
                                              const long long* nmask, const R* const* masks, cudaStream_t st) {
    MaskArgs a{};
    a.dim = dim;
    for (int j = 0; j < dim; ++j) {
        a.shift[j] = shift[j];
        a.nmask[j] = nmask[j];
        a.mask[j] = masks[j];
    }
    apply_masks_kernel<R><<<elementwise_blocks(n), 256, 0, st>>>(n, psi, a);
}
template <typename R> void launch_add_potential(long long n, cplx_t<R>* dst, const cplx_t<R>* src, const double* vtab,
                                                cudaStream_t st) {
    add_potential_kernel<R><<<elementwise_blocks(n), 256, 0, st>>>(n, dst, src, vtab);
}

template <typename R> void launch_axis_factors(const AxisFactorArgs& a, cplx_t<R>* psi, cudaStream_t st) {
    axis_factors_kernel<R><<<elementwise_blocks(a.n), 256, 0, st>>>(a, psi);
}
template <typename R> void launch_axis_permute(const AxisPermArgs& a, const cplx_t<R>* in, cplx_t<R>* out,
                                               int to_natural, cudaStream_t st) {
    axis_permute_kernel<R><<<elementwise_blocks(a.n), 256, 0, st>>>(a, in, out, to_natural);
}
template <typename R> void launch_apply_combine(long long n, cplx_t<R>* dst, const cplx_t<R>* tmp,
                                               const cplx_t<R>* src, const double* vtab, int acc, cudaStream_t st) {
    apply_combine_kernel<R><<<elementwise_blocks(n), 256, 0, st>>>(n, dst, tmp, src, vtab, acc);
}

#define QND_INST(R)                                                                               \
    template void launch_gs_dot<R>(const GSArgs<R>&, cudaStream_t, int);                          \
    template void launch_gs_axpy<R>(const GSArgs<R>&, cudaStream_t, int);                         \
    template void launch_grid_reduce<R>(const PassArgs<R>&, long long, cudaStream_t, int);        \
    template void launch_scale<R>(cplx_t<R>*, long long, const double*, cudaStream_t);            \
    template void launch_field_tables<R>(const FieldTableArgs&, cplx_t<R>*, cudaStream_t);        \
    template void launch_axis_table<R>(int, const double*, int, double, void*, cudaStream_t);             \
    template void launch_radial_mask<R>(const SpectraArgs&, const cplx_t<R>*, cplx_t<R>*, cudaStream_t);  \
    template void launch_ped<R>(const SpectraArgs&, const cplx_t<R>*, double*, double*, cudaStream_t);    \
    template void launch_pmd<R>(const SpectraArgs&, const cplx_t<R>*, double*, cudaStream_t);             \
    template void launch_long_twiddle<R>(const LongArgs&, cplx_t<R>*, const cplx_t<R>*, int, cudaStream_t); \
    template void launch_long_transpose<R>(const LongArgs&, const cplx_t<R>*, cplx_t<R>*, int, cudaStream_t); \
    template void launch_point_factors<R>(long long, cplx_t<R>*, const R*, const cplx_t<R>*, const cplx_t<R>*, \
                                          const R*, const double*, cudaStream_t);                          \
    template void launch_add_potential<R>(long long, cplx_t<R>*, const cplx_t<R>*, const double*, cudaStream_t); \
    template void launch_embed<R>(const EmbedArgs&, const double2*, cplx_t<R>*, cudaStream_t);                \
    template void launch_apply_masks<R>(long long, cplx_t<R>*, int, const int*, const long long*, const R* const*, \
                                        cudaStream_t);                                                      \
    template void launch_axis_factors<R>(const AxisFactorArgs&, cplx_t<R>*, cudaStream_t);                   \
    template void launch_axis_permute<R>(const AxisPermArgs&, const cplx_t<R>*, cplx_t<R>*, int, cudaStream_t); \
    template void launch_apply_combine<R>(long long, cplx_t<R>*, const cplx_t<R>*, const cplx_t<R>*, const double*, \
                                          int, cudaStream_t);
QND_INST(double)
QND_INST(float)
#undef QND_INST

}  // namespace qnd
