// qnd_engine.cu — host side of libqnd_b200.so: context, tables, pass schedules and
// the extern "C" API declared in include/qnd.h.
//
// Representation: the engine keeps every state in r-space. A split-operator
// sub-step of the reference, e.g. for the length gauge (integrators.c:170-194)
//     psi_p <- K(b) F [ V(h) B K(a) psi_p ] / N
// is, with chi = B psi_p / sqrt(N), the r-space product
//     chi <- S(b) V(h) S(a) chi,   S(c) = B K(c) F / N.
// The kinetic factor is separable (K = sum_j p_j^2/2), so S(c) = prod_j S_j(c): one
// "sandwich" pass per axis (FFT along j, multiply by exp(-i c p_j^2/2)/N_j, inverse
// FFT along j). Consecutive S(b) S(a') merge into S(b + a'), and V(h) -- the only
// non-separable factor -- is applied in the epilogue of the last pass of each
// sandwich. One sub-step therefore costs one read and one write of the state per
// axis, and the observables at step boundaries (QuantumND_real.c:197-212) come out
// of the last pass's fused reductions without the reference's extra transforms.
#include <cuda.h>
#include <dlfcn.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <atomic>
#include <map>
#include <set>
#include <tuple>
#include <type_traits>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/qnd.h"
#include "qnd_kernels.cuh"

namespace qnd {

static thread_local std::string g_err;

struct Error {
    int code;
    std::string msg;
};

static std::string fmt(const char* f, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

#define QND_FAIL(code, ...) throw ::qnd::Error{code, ::qnd::fmt(__VA_ARGS__)}
#define QND_CK(x)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) QND_FAIL(QND_ECUDA, "%s: %s", #x, cudaGetErrorString(e_));           \
    } while (0)

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void ensure(size_t b) {
        if (b <= bytes && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        // fault injection for the tests: QND_FAIL_ALLOC_ABOVE=<bytes> makes every larger request fail
        // here, on the host, as an out-of-memory would
        if (const char* lim = std::getenv("QND_FAIL_ALLOC_ABOVE"))
            if (b > size_t(std::strtoull(lim, nullptr, 10)))
                QND_FAIL(QND_ENOMEM, "cudaMalloc(%zu bytes): refused by QND_FAIL_ALLOC_ABOVE=%s", b, lim);
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e != cudaSuccess) {
            cudaGetLastError();
            QND_FAIL(QND_ENOMEM, "cudaMalloc(%zu bytes): %s", b, cudaGetErrorString(e));
        }
        bytes = b;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

static PassKernelInfo lookup_pass(bool fp64, int L, bool strided, int mode, int var = 0, bool tma = false) {
#define QND_CASE(LL)                                                                                              \
    case LL:                                                                                                      \
        return fp64 ? pass_kernel_info<double, LL>(strided, mode, var, tma)                                       \
                    : pass_kernel_info<float, LL>(strided, mode, var, tma);
    switch (L) {
        QND_CASE(2) QND_CASE(4) QND_CASE(8) QND_CASE(16) QND_CASE(32) QND_CASE(64) QND_CASE(128) QND_CASE(256)
        QND_CASE(512) QND_CASE(1024) QND_CASE(2048) QND_CASE(4096)
    default: QND_FAIL(QND_EUNSUPPORTED, "axis length %d: this build supports powers of two from 2 to 4096", L);
    }
#undef QND_CASE
}

enum ObsKind { OB_ZERO, OB_NORM, OB_DIPOLE_R, OB_ACCEL, OB_DIPOLE_V, OB_ENERGY, OB_LZ };

struct ObsItem {
    ObsKind kind;
    int offset, width;
};

static const double MAX_EXP_ARG = 700.;  // integrators.h:12
static const int64_t LONG_AXIS_MAX = int64_t(1) << 24;  // longest 1-D axis (four-step transform)

}  // namespace qnd

using namespace qnd;

namespace qnd {
struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    std::vector<int64_t> launches;  // kernels one replay launches, per context it spans
    uint64_t last_use = 0;
};
constexpr size_t MAX_GRAPHS = 8;
static std::atomic<uint64_t> g_ctx_serial{0};
}  // namespace qnd

// One pass of a member's run, recorded for the persistent sweep kernel: the pass kernel it would
// launch (line length, stride, mode), its line groups, and its PassArgs<R> as bytes.
struct RecordedPass {
    int L = 0, strided = 0, kmode = 0;
    unsigned ngroups = 0;
    std::vector<unsigned char> args;
};

struct qnd_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool fp64 = true;
    int dim = 0;
    int64_t nr[MAX_DIM] = {1, 1, 1, 1, 1, 1};
    double dr[MAX_DIM] = {};
    int64_t n = 0;
    int lognr[MAX_DIM] = {};
    int shift[MAX_DIM] = {};
    std::string integrator;
    double dt = 0;
    int s = 0;
    double as[20] = {0};
    double dNr = 1, dNp = 1;
    int axoff[MAX_DIM] = {};
    int axtot = 0;

    std::vector<double> r[MAX_DIM], p[MAX_DIM];
    std::vector<double> vpot, vcap;
    std::vector<double> gradv[MAX_DIM];
    std::vector<double> mask[MAX_DIM];
    uint64_t table_epoch = 0;  // bumps when V / Vcap change; invalidates r-space tables

    DevBuf tw[MAX_DIM];
    DevBuf r_dev, p_dev;  // concatenated axes (double)
    DevBuf gradv_dev[MAX_DIM];                // natural layout
    DevBuf gradv_lm[MAX_DIM][MAX_DIM];        // [component][pass axis] line-major copies
    DevBuf mask_dev[MAX_DIM];
    DevBuf vpot_dev;      // double, for the energy operator
    std::map<std::tuple<int, int, double, double>, std::unique_ptr<DevBuf>> spec_cache;
    std::map<std::tuple<int, double, double, uint64_t>, std::unique_ptr<DevBuf>> rtab_cache;

    DevBuf partials, counter, obs_dev, scal;  // reduction scratch; scal: [0]=gs norm2 [1]=gs scale [2..] coefs
    DevBuf gs_flag;
    DevBuf field_dev, field_tab, wtab_dev[MAX_DIM], spec_tmp[MAX_DIM];
    DevBuf scratch_a, scratch_b;
    // qnd_run_length_sweep: while recorder is set, launch_pass records each pass (kind and arguments)
    // there instead of launching it; field_view, when set, is where the chain reads its per-step field
    // tables (a segment's tables live side by side in sweep_field)
    std::vector<RecordedPass>* recorder = nullptr;
    const void* field_view = nullptr;
    DevBuf sweep_field, sweep_buf;
    DevBuf spec_rank, spec_partials, spec_out;  // final spectra: per-axis ranks, partial sums, results
    DevBuf field_out, embed_src;                // qnd_field_samples host-output staging; qnd_state_embed source
    DevBuf err_flag;                            // set by a kernel whose bounded wait ran out
    DevBuf tune_buf;                            // scratch state of the staging autotuner
    DevBuf shape_buf;                           // scratch state of the shape autotuner (its own: the
                                                // staging tuner frees tune_buf inside its launches)
    DevBuf finite_slot;                         // QND_CHECK_FINITE: the non-finite count
    std::map<std::tuple<const void*, int, int>, CUtensorMap> tmaps;  // strided-pass TMA views of states

    // A 1-D axis longer than one pass handles: N = n1 n2 (n1 >= 16, n2 <= 4096) as a virtual
    // n1 x n2 grid transformed in four steps (long_fft). tw_long[v]: the stage twiddles of the
    // length-n1 (v = 0) and length-n2 (v = 1) passes; twf_long / twc_long: the four-step twiddle
    // W_N^{k1 m} and its conjugate at slot k1 n2 + m; p_slot: the momentum of each k-space slot
    // (slot k1 n2 + k2 holds frequency k1 + n1 k2).
    bool long1d = false;
    int64_t n1 = 0, n2 = 0;
    int lg1 = 0, lg2 = 0;
    DevBuf tw_long[2], twf_long, twc_long, p_slot_dev, long_tmp;
    // Axes longer than 4096 points on grids of several dimensions (emulate_long_pass): per axis the
    // virtual lengths n1 n2, their pass twiddles, the four-step twiddles and their conjugates (at
    // slot k1 n2 + m, as for the 1-D long axis); two scratch states for permutations and copies.
    struct LongAxis {
        bool on = false;
        int64_t n1 = 0, n2 = 0;
        int lg1 = 0, lg2 = 0;
        DevBuf tw[2], twf, twc;
    } lax[MAX_DIM];
    DevBuf lax_perm, lax_tmp;
    std::vector<double> p_slot;
    std::vector<char> host_tmp;

    int num_sms = 148;
    bool pdl = true;  // programmatic dependent launch between passes
    bool profiling = false;
    int64_t kernels_launched = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_pairs;
    std::vector<cudaEvent_t> event_pool;

    // Chunk-wide sandwich chains captured in CUDA graphs and replayed for the later chunks of the
    // same shape (run_chunk_graph): the executable graphs by what they captured (key; at most
    // MAX_GRAPHS, least recently used first out), and the keys already run directly once (their
    // tables exist). config_epoch bumps with every setter that changes what a chain reads; serial
    // tells this context from any earlier one at the same addresses.
    std::map<std::string, GraphEntry> graphs;
    std::set<std::string> warm_keys;
    uint64_t graph_clock = 0;
    uint64_t config_epoch = 0;
    uint64_t serial = 0;

    size_t elem() const { return fp64 ? 16 : 8; }
    size_t rsize() const { return fp64 ? 8 : 4; }
};

namespace qnd {

// ---------------------------------------------------------------- tables --

// Rounds n stored FP32 factors d (interleaved doubles; the factor is 1 + d, see fmul in
// qnd_fft.cuh) to float pairs so that the squared magnitudes |1 + d|^2 of the rounded values add up
// to those of the exact ones along the array: each value takes, among the 5 x 5 neighbourhood of its
// nearest-rounded parts, the pair that brings the running sum of magnitude errors closest to zero
// (ties: the nearer pair). Every contiguous run of entries then carries a magnitude error bounded
// by two single-entry errors in total, so the FFT stage twiddles and the phase tables applied at
// every step leave no systematic drift of the norm. Each part stays within two units in the last
// place.
// QND_F32_TABLES selects another rounding for experiments: "nearest" (each part to nearest) or
// "magnitude" (per entry the candidate pair whose |1 + d|^2 is closest, no running sum).
static void round_pairs_f32_balanced(const double* v, size_t n, float* out) {
    const char* mode = std::getenv("QND_F32_TABLES");
    const bool nearest = mode && !std::strcmp(mode, "nearest");
    const bool per_entry = mode && !std::strcmp(mode, "magnitude");
    if (nearest) {
        for (size_t i = 0; i < 2 * n; ++i) out[i] = float(v[i]);
        return;
    }
    double run = 0.0;
    for (size_t i = 0; i < n; ++i) {
        if (per_entry) run = 0.0;
        const double re = v[2 * i], im = v[2 * i + 1];
        // |1 + x|^2 - |1 + d|^2 = (xr - dr)(2 + xr + dr) + (xi - di)(xi + di)
        auto merr = [&](double xr, double xi) { return (xr - re) * (2.0 + xr + re) + (xi - im) * (xi + im); };
        float rs[5], is[5];
        rs[2] = float(re);
        is[2] = float(im);
        rs[1] = std::nextafter(rs[2], -INFINITY);
        rs[0] = std::nextafter(rs[1], -INFINITY);
        rs[3] = std::nextafter(rs[2], INFINITY);
        rs[4] = std::nextafter(rs[3], INFINITY);
        is[1] = std::nextafter(is[2], -INFINITY);
        is[0] = std::nextafter(is[1], -INFINITY);
        is[3] = std::nextafter(is[2], INFINITY);
        is[4] = std::nextafter(is[3], INFINITY);
        float br = rs[2], bi = is[2];
        double be = std::fabs(run + merr(br, bi)), bd = 1e300;
        for (int a = 0; a < 5; ++a)
            for (int q = 0; q < 5; ++q) {
                const double xr = rs[a], xi = is[q];
                const double e = std::fabs(run + merr(xr, xi));
                const double d = (xr - re) * (xr - re) + (xi - im) * (xi - im);
                if (e < be || (e == be && d < bd)) {
                    be = e;
                    bd = d;
                    br = rs[a];
                    bi = is[q];
                }
            }
        run += merr(br, bi);
        out[2 * i] = br;
        out[2 * i + 1] = bi;
    }
}

// Stage twiddles of HostPlan(L), exp(-2 pi i jm r / (Ns R)) in long double: FP64 plans one base per
// butterfly position (r = 1; the kernel forms the powers, pow_twiddles), FP32 plans every r in the
// [j mod Ns][r-1] layout.
static void build_twiddles(qnd_ctx* c, int L, DevBuf& dst) {
    HostPlan pl(L, lookup_pass(c->fp64, L, false, PM_SANDWICH).E);
    const int entries = c->fp64 ? pl.twb_size : pl.tw_size;
    std::vector<double> tw(2 * size_t(entries > 0 ? entries : 1));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    size_t o = 0;
    for (int st = 1; st < pl.nstage; ++st) {
        const int R = pl.radix[st], Ns = pl.span[st];
        for (int jm = 0; jm < Ns; ++jm)
            for (int r = 1; r < (c->fp64 ? 2 : R); ++r) {
                long double ang = two_pi * (long double)(jm * r) / (long double)(Ns * R);
                if (c->fp64) {
                    tw[2 * o] = (double)cosl(ang);
                } else {  // stored as w - 1 (cos - 1 = -2 sin^2(ang/2))
                    const long double sh = sinl(ang / 2);
                    tw[2 * o] = (double)(-2 * sh * sh);
                }
                tw[2 * o + 1] = (double)(-sinl(ang));
                ++o;
            }
    }
    const size_t cnt = size_t(entries > 0 ? entries : 1);
    dst.ensure(cnt * c->elem());
    if (c->fp64) {
        QND_CK(cudaMemcpyAsync(dst.p, tw.data(), cnt * 16, cudaMemcpyHostToDevice, c->stream));
    } else {
        std::vector<float> f(2 * cnt);
        round_pairs_f32_balanced(tw.data(), cnt, f.data());
        QND_CK(cudaMemcpyAsync(dst.p, f.data(), cnt * 8, cudaMemcpyHostToDevice, c->stream));
    }
}

// Upload n stored complex factors given as interleaved doubles: the factors w themselves for FP64
// contexts, d = w - 1 (spectral tables: w N_axis - 1) for FP32 contexts.
static void upload_cplx(qnd_ctx* c, DevBuf& dst, const std::vector<double>& v) {
    const size_t n = v.size() / 2;
    dst.ensure(n * c->elem());
    if (c->fp64) {
        QND_CK(cudaMemcpyAsync(dst.p, v.data(), n * 16, cudaMemcpyHostToDevice, c->stream));
    } else {
        std::vector<float> f(2 * n);
        for (size_t i = 0; i < 2 * n; ++i)
            if (std::isinf(float(v[i])) && !std::isinf(v[i]))
                QND_FAIL(QND_EUNSUPPORTED, "a phase/decay factor exceeds the FP32 range: use QND_FP64 for this case");
        round_pairs_f32_balanced(v.data(), n, f.data());
        QND_CK(cudaMemcpyAsync(dst.p, f.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
    }
}

static void upload_real(qnd_ctx* c, DevBuf& dst, const std::vector<double>& v) {
    const size_t n = v.size();
    dst.ensure(n * c->rsize());
    if (c->fp64) {
        QND_CK(cudaMemcpyAsync(dst.p, v.data(), n * 8, cudaMemcpyHostToDevice, c->stream));
    } else {
        std::vector<float> f(n);
        for (size_t i = 0; i < n; ++i) {
            f[i] = float(v[i]);
            if (std::isinf(f[i]) && !std::isinf(v[i]))
                QND_FAIL(QND_EUNSUPPORTED, "a decay factor exceeds the FP32 range: use QND_FP64 for this case");
        }
        QND_CK(cudaMemcpyAsync(dst.p, f.data(), n * 4, cudaMemcpyHostToDevice, c->stream));
    }
}

// Every upload is ordered on the context's stream: a synchronous cudaMemcpy from pageable memory may
// return before its DMA lands, and the kernels that read the table run on the context's stream.
static void upload_f64(qnd_ctx* c, DevBuf& dst, const std::vector<double>& v) {
    dst.ensure(v.size() * 8);
    QND_CK(cudaMemcpyAsync(dst.p, v.data(), v.size() * 8, cudaMemcpyHostToDevice, c->stream));
}

enum SpecKind { SP_LENGTH = 0, SP_IMAG = 1, SP_KIN = 2 };

// Per-axis spectral factor tables (include the 1/N_axis of the inverse transform):
//   SP_LENGTH: exp(-i c p^2/2)/N     (integrators.c:177, :192 factorised over axes)
//   SP_IMAG:   exp(-c p^2/2)/N       (integrators.c:151-153; clamp checked up front)
//   SP_KIN:    (p^2/2)/N             (the kinetic operator of calculate_observables.c:165)
static const void* spec_table(qnd_ctx* c, int kind, int ax, double coef) {
    auto key = std::make_tuple(kind, ax, coef, 0.0);
    auto it = c->spec_cache.find(key);
    if (it != c->spec_cache.end()) return it->second->p;
    const int N = int(c->nr[ax]);
    // a long axis: slot order, and the 1/N of the inverse transform split as 1/n2 here (FP64; FP32
    // tables are scaled by 1/n2 in the pass) and 1/n1 in the closing length-n1 pass
    const double Nn = c->long1d ? double(c->n2) : double(N);
    std::vector<double> v(2 * size_t(N));
    for (int k = 0; k < N; ++k) {
        const double pk = c->long1d ? c->p_slot[k] : c->p[ax][k];
        const double kin = .5 * pk * pk;
        double re, im;
        if (kind == SP_LENGTH) {
            const double th = coef * kin;
            if (c->fp64) {
                re = std::cos(th) / Nn;
            } else {
                const double sh = std::sin(th / 2);
                re = -2 * sh * sh;
            }
            im = c->fp64 ? -std::sin(th) / Nn : -std::sin(th);
        } else if (kind == SP_IMAG) {
            re = c->fp64 ? std::exp(-coef * kin) / Nn : std::expm1(-coef * kin);
            im = 0;
        } else {
            re = c->fp64 ? kin / Nn : kin - 1.0;
            im = 0;
        }
        v[2 * k] = re;
        v[2 * k + 1] = im;
    }
    auto buf = std::make_unique<DevBuf>();
    upload_cplx(c, *buf, v);
    const void* ptr = buf->p;
    c->spec_cache[key] = std::move(buf);
    return ptr;
}

enum RtabKind { RT_IMAG = 0, RT_LENGTH = 1, RT_VEL = 2, RT_LENGTH_ADJ = 3, RT_VEL_ADJ = 4 };
static const double NO_COEF = 1e300;  // marks "no second factor"

static inline double clamped_exp(double arg) { return std::exp(arg > MAX_EXP_ARG ? MAX_EXP_ARG : arg); }

// Full-grid r-space factor tables.
//   RT_IMAG   (a[, b]):  exp(min(700, -a V)) [* exp(min(700, -b V))]           real (integrators.c:143-160)
//   RT_LENGTH (h):       exp(min(700, -h Vcap)) exp(-i h V)                      complex (integrators.c:186-188)
//   RT_VEL    (a[, b]):  exp(min(700,-a Vcap)) exp(-i a V) [* same with b]       complex (integrators.c:209-229)
//   RT_LENGTH_ADJ (h), RT_VEL_ADJ (a[, b]): the complex conjugates (the adjoints of those factors)
// Reorder a full-grid array (comps values per point) to line-major order for axis ax: entry
// lam*L + m holds point m of line lam (the order in which a pass along ax visits the grid).
static std::vector<double> line_major(const qnd_ctx* c, const std::vector<double>& nat, int comps, int ax) {
    if (ax == c->dim - 1) return nat;
    const int64_t L = c->nr[ax];
    const int log2S = c->shift[ax];
    const int64_t S = int64_t(1) << log2S, nlines = c->n / L;
    std::vector<double> out(nat.size());
    for (int64_t lam = 0; lam < nlines; ++lam) {
        const int64_t base = ((lam >> log2S) * L << log2S) + (lam & (S - 1));
        for (int64_t m = 0; m < L; ++m) {
            const int64_t src = (base + (m << log2S)) * comps, dst = (lam * L + m) * comps;
            for (int q = 0; q < comps; ++q) out[dst + q] = nat[src + q];
        }
    }
    return out;
}

static const void* rtab(qnd_ctx* c, int kind, double a, double b, int ax);

// Full-grid tables in the natural layout (the contiguous axis' line-major layout).
static const void* rtab(qnd_ctx* c, int kind, double a, double b) { return rtab(c, kind, a, b, c->dim - 1); }

// d = w - 1 for w = exp(x) e^{-i th} (x = the clamped CAP exponent), computed without cancellation:
// Re d = (e^x - 1) cos th + (cos th - 1), Im d = -e^x sin th.
static void unit_factor_d(double x, double th, double* dr, double* di) {
    const double em1 = x > MAX_EXP_ARG ? std::exp(MAX_EXP_ARG) - 1.0 : std::expm1(x);
    const double sh = std::sin(th / 2);
    *dr = em1 * std::cos(th) - 2 * sh * sh;
    *di = -(em1 + 1.0) * std::sin(th);
}

static const void* rtab(qnd_ctx* c, int kind, double a, double b, int ax) {
    auto key = std::make_tuple(kind * 8 + ax, a, b, c->table_epoch);
    auto it = c->rtab_cache.find(key);
    if (it != c->rtab_cache.end()) return it->second->p;
    if (c->vpot.empty()) QND_FAIL(QND_EINVAL, "no potential set: call qnd_set_potential_named or qnd_set_potential");
    const size_t n = size_t(c->n);
    auto buf = std::make_unique<DevBuf>();
    if (kind == RT_IMAG) {
        std::vector<double> v(n);
        for (size_t i = 0; i < n; ++i) {
            double f = clamped_exp(-a * c->vpot[i]);
            if (b != NO_COEF) f *= clamped_exp(-b * c->vpot[i]);
            v[i] = f;
        }
        upload_real(c, *buf, line_major(c, v, 1, ax));
    } else {
        std::vector<double> v(2 * n);
        for (size_t i = 0; i < n; ++i) {
            const double vc = c->vcap.empty() ? 0.0 : c->vcap[i];
            double re, im;
            if (c->fp64) {
                if (kind == RT_LENGTH || kind == RT_LENGTH_ADJ) {
                    const double m = clamped_exp(-a * vc), th = a * c->vpot[i];
                    re = m * std::cos(th);
                    im = -m * std::sin(th);
                } else {
                    const double m1 = clamped_exp(-a * vc), th1 = a * c->vpot[i];
                    re = m1 * std::cos(th1);
                    im = -m1 * std::sin(th1);
                    if (b != NO_COEF) {
                        const double m2 = clamped_exp(-b * vc), th2 = b * c->vpot[i];
                        const double r2 = m2 * std::cos(th2), i2 = -m2 * std::sin(th2);
                        const double nr_ = re * r2 - im * i2, ni = re * i2 + im * r2;
                        re = nr_;
                        im = ni;
                    }
                }
            } else {
                // FP32 factors are stored as d = w - 1 (one factor, or the product of two)
                double dr, di;
                unit_factor_d(-a * vc, a * c->vpot[i], &dr, &di);
                if ((kind == RT_VEL || kind == RT_VEL_ADJ) && b != NO_COEF) {
                    double er, ei;
                    unit_factor_d(-b * vc, b * c->vpot[i], &er, &ei);
                    const double pr = dr * er - di * ei, pi = dr * ei + di * er;
                    dr = dr + er + pr;
                    di = di + ei + pi;
                }
                re = dr;
                im = di;
            }
            v[2 * i] = re;
            // conj(w), and for FP32 conj(w - 1) = conj(w) - 1
            v[2 * i + 1] = (kind == RT_LENGTH_ADJ || kind == RT_VEL_ADJ) ? -im : im;
        }
        upload_cplx(c, *buf, line_major(c, v, 2, ax));
    }
    const void* ptr = buf->p;
    c->rtab_cache[key] = std::move(buf);
    return ptr;
}

static void invalidate_rtabs(qnd_ctx* c) {
    c->rtab_cache.clear();
    c->table_epoch++;
}

// ---------------------------------------------------------------- passes --

struct PassSpec {
    int axis = 0;
    int mode = PM_SANDWICH;
    void* psi = nullptr;
    void* dst = nullptr;
    const void* partner = nullptr;
    const void* pro_real = nullptr;
    const void* pro_cplx = nullptr;
    const double* pro_scale = nullptr;
    const void* spec = nullptr;
    const void* spec2 = nullptr;
    const void* mid_real = nullptr;
    const void* mid_cplx = nullptr;
    const void* mid_ax_cplx[MAX_DIM] = {};
    const void* mid_ax_real[MAX_DIM] = {};
    int red_at_mid = 0;
    const void* epi_real = nullptr;
    const void* epi_cplx = nullptr;
    const void* ax_cplx[MAX_DIM] = {};
    const void* ax_real[MAX_DIM] = {};
    int ax_in_prologue = 0;
    double scale = 1.0;
    int apply_acc = 0;
    const double* apply_vtab = nullptr;
    RedDesc red{};
    int spec_full = 0;           // spec: a full-grid table in line-major order
    int force_staging = -1;      // strided passes: -1 the tuned staging, 0 per-thread copies, 1 TMA boxes
    int force_shape = -1;        // -1 the tuned shape variant (shape_choice), else that variant
    // a pass over a virtual axis of a long 1-D axis: its length, log2 stride and stage twiddles
    int vL = 0, vlog2S = 0;
    const void* vtw = nullptr;
};

static void ensure_red_scratch(qnd_ctx* c, long long blocks) {
    const size_t need = size_t(blocks) * MAX_RED * sizeof(double);
    if (c->partials.bytes < need) c->partials.ensure(need);
    if (!c->counter.p) {
        c->counter.ensure(64);
        QND_CK(cudaMemsetAsync(c->counter.p, 0, 64, c->stream));
    }
}

// Tries of the bounded wait of a strided pass for its TMA box loads (2^20). QND_TMA_WAIT_TRIES
// overrides it, read at every launch: a host-side way to make the wait run out (0 tries) and check
// that path (the CTAs then leave the state untouched and the next synchronising call reports it).
static int tma_wait_tries() {
    const char* e = std::getenv("QND_TMA_WAIT_TRIES");
    if (!e || !*e) return 1 << 20;
    const long v = std::strtol(e, nullptr, 10);
    return v < 0 ? 0 : (v > (1 << 20) ? (1 << 20) : int(v));
}

// The log2 stride and index mask of each axis-weighted reduction's axis (RedDesc wshift / wmask).
static void set_red_axes(const qnd_ctx* c, RedDesc& rd) {
    for (int k = 0; k < rd.n && k < MAX_RED; ++k) {
        const int wax = rd.waxis[k] >= 0 && rd.waxis[k] < c->dim ? rd.waxis[k] : 0;
        rd.wshift[k] = c->shift[wax];
        rd.wmask[k] = c->nr[wax] - 1;
    }
}

template <typename R> static void fill_args(qnd_ctx* c, const PassSpec& ps, PassArgs<R>& a) {
    using V = cplx_t<R>;
    std::memset(&a, 0, sizeof a);
    a.psi = static_cast<V*>(ps.psi);
    a.dst = static_cast<V*>(ps.dst);
    a.axis = ps.axis;
    a.partner = static_cast<const V*>(ps.partner);
    a.dim = c->dim;
    for (int k = 0; k < MAX_DIM; ++k) {
        a.shift[k] = c->shift[k];
        a.nmask[k] = c->nr[k] - 1;
    }
    a.pro_real = static_cast<const R*>(ps.pro_real);
    a.pro_cplx = static_cast<const V*>(ps.pro_cplx);
    a.pro_scale_dev = ps.pro_scale;
    a.spec = static_cast<const V*>(ps.spec);
    a.spec_full = ps.spec_full;
    a.spec2 = static_cast<const V*>(ps.spec2);
    a.mid_real = static_cast<const R*>(ps.mid_real);
    a.mid_cplx = static_cast<const V*>(ps.mid_cplx);
    for (int k = 0; k < MAX_DIM; ++k) {
        a.mid_ax_cplx[k] = static_cast<const V*>(ps.mid_ax_cplx[k]);
        a.mid_ax_real[k] = static_cast<const R*>(ps.mid_ax_real[k]);
    }
    a.red_at_mid = ps.red_at_mid;
    a.epi_real = static_cast<const R*>(ps.epi_real);
    a.epi_cplx = static_cast<const V*>(ps.epi_cplx);
    for (int k = 0; k < MAX_DIM; ++k) {
        a.ax_cplx[k] = static_cast<const V*>(ps.ax_cplx[k]);
        a.ax_real[k] = static_cast<const R*>(ps.ax_real[k]);
    }
    a.ax_in_prologue = ps.ax_in_prologue;
    a.scale = R(ps.scale);
    a.apply_acc = ps.apply_acc;
    a.apply_vtab = ps.apply_vtab;
    a.seed = uint32_t(c->kernels_launched) * 0x9e3779b9u + 0x632be5abu;
    a.red = ps.red;
    set_red_axes(c, a.red);
    a.err = c->err_flag.as<int>();
    a.tma_wait_tries = tma_wait_tries();
}

struct LaunchCfg {
    int blocks_per_sm = 0;
};

// cuTensorMapEncodeTiled from the driver, found at run time (the library links only the runtime).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn tensor_map_encoder() {
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {  // looked up once, thread-safe
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<EncodeTiledFn>(p);
        cudaGetLastError();
        return nullptr;
    }();
    return fn;
}

// The TMA view of a state for a strided pass along an axis of L points with stride S = 2^log2S:
// a 3-D tensor {S (contiguous sub-index), L, n / (S L)} of complex values (FP64: pairs of doubles;
// FP32: one 8-byte element each) whose boxes {G lines, min(L, 256) rows, 1} are a CTA's lines. False
// (per-thread staging) unless the boxes obey the rules of the copy engine: a 16-byte aligned base,
// 16-byte box rows and x offsets (G complex values a multiple of 16 bytes), and full groups of G
// lines that share their outer index (G <= S, every group complete).
static bool strided_tma_map(qnd_ctx* c, const void* psi, int L, int log2S, int G, CUtensorMap* map) {
    if (std::getenv("QND_NO_TMA")) return false;
    const int64_t S = int64_t(1) << log2S;
    const size_t ce = c->elem();
    // boxes of G neighbouring lines: every group inside one slab of S lines (G divides S, or the pass
    // has a single slab; a last group with fewer lines loads past the last line, which reads the fill
    // value, and stores its lines without boxes)
    const int64_t slabs = c->n / (S * L);
    if (reinterpret_cast<uintptr_t>(psi) % 16 || S < G || (size_t(G) * ce) % 16 || (S % G && slabs != 1)) return false;
    const auto key = std::make_tuple(psi, L * 64 + G, log2S);  // G <= 32 lines per box
    auto it = c->tmaps.find(key);
    if (it != c->tmaps.end()) {
        *map = it->second;
        return true;
    }
    EncodeTiledFn enc = tensor_map_encoder();
    if (!enc) return false;
    const int boxl = L < 256 ? L : 256;
    cuuint64_t dims[3] = {cuuint64_t(c->fp64 ? 2 * S : S), cuuint64_t(L), cuuint64_t(c->n / (S * L))};
    cuuint64_t strides[2] = {cuuint64_t(S) * ce, cuuint64_t(S) * cuuint64_t(L) * ce};
    cuuint32_t box[3] = {cuuint32_t(c->fp64 ? 2 * G : G), cuuint32_t(boxl), 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUtensorMap m;
    const CUresult r = enc(&m, c->fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_UINT64, 3,
                           const_cast<void*>(psi), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    if (c->tmaps.size() >= 64) c->tmaps.clear();
    c->tmaps[key] = m;
    *map = m;
    return true;
}

static void launch_pass(qnd_ctx* c, const PassSpec& ps);

// Staging autotuner. A strided pass can stage its CTA's lines by per-thread cp.async copies or by
// TMA box loads; both move the same values into the same registers, so the choice changes the time
// and never the results. Per (device, precision, points, line length, stride) the first eligible
// launch outside a stream capture times a forward-transform pass along that geometry with each
// staging (one warm-up and three timed launches each, on a zeroed scratch state, untimed by the
// launch counters) and keeps TMA only if it is at least 2% faster. Until then, and with QND_TUNE=0,
// lines of 1024 points and more use TMA (measured faster there, slower at 256).
struct StagingKey {
    int device, fp64;
    long long n;
    int L, log2S;
    bool operator<(const StagingKey& o) const {
        return std::tie(device, fp64, n, L, log2S) < std::tie(o.device, o.fp64, o.n, o.L, o.log2S);
    }
};
static std::mutex g_staging_mu;
static std::map<StagingKey, int> g_staging;

static int staging_choice(qnd_ctx* c, const PassSpec& ps, int L, int log2S) {
    const StagingKey key{c->device, int(c->fp64), c->n, L, log2S};
    {
        std::lock_guard<std::mutex> lk(g_staging_mu);
        auto it = g_staging.find(key);
        if (it != g_staging.end()) return it->second;
    }
    const int fallback = L >= 1024 ? 1 : 0;
    const char* tune = std::getenv("QND_TUNE");
    if ((tune && !std::atoi(tune)) || c->profiling) return fallback;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    QND_CK(cudaStreamIsCapturing(c->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return fallback;
    c->tune_buf.ensure(size_t(c->n) * c->elem());
    QND_CK(cudaMemsetAsync(c->tune_buf.p, 0, size_t(c->n) * c->elem(), c->stream));
    CUtensorMap probe;
    const PassKernelInfo info = lookup_pass(c->fp64, L, true, PM_FFT_FWD);
    int choice = 0;
    if (strided_tma_map(c, c->tune_buf.p, L, log2S, info.G, &probe)) {
        PassSpec t;
        t.axis = ps.axis;
        t.mode = PM_FFT_FWD;
        t.psi = c->tune_buf.p;
        t.vL = ps.vL;
        t.vlog2S = ps.vlog2S;
        t.vtw = ps.vtw;
        const int64_t k0 = c->kernels_launched;
        cudaEvent_t e0, e1;
        QND_CK(cudaEventCreate(&e0));
        QND_CK(cudaEventCreate(&e1));
        float ms[2] = {0.f, 0.f};
        for (int mode = 0; mode < 2; ++mode) {
            t.force_staging = mode;
            launch_pass(c, t);
            QND_CK(cudaEventRecord(e0, c->stream));
            for (int r = 0; r < 3; ++r) launch_pass(c, t);
            QND_CK(cudaEventRecord(e1, c->stream));
            QND_CK(cudaEventSynchronize(e1));
            QND_CK(cudaEventElapsedTime(&ms[mode], e0, e1));
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c->kernels_launched = k0;
        choice = ms[1] < 0.98f * ms[0] ? 1 : 0;
    }
    c->tune_buf.reset();  // a one-time measurement: give the scratch state back
    std::lock_guard<std::mutex> lk(g_staging_mu);
    g_staging[key] = choice;
    return choice;
}

// Reads and clears the error flag that a kernel sets when a bounded wait ran out.
static void check_device_error(qnd_ctx* c) {
    if (!c->err_flag.p) return;
    int flag = 0;
    QND_CK(cudaMemcpyAsync(&flag, c->err_flag.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    QND_CK(cudaStreamSynchronize(c->stream));
    if (flag) {
        QND_CK(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), c->stream));
        QND_FAIL(QND_ECUDA, "a pass kernel's wait for its TMA box loads ran out; the CTAs concerned left their "
                            "lines untransformed (results of that call are invalid)");
    }
}

// Tile-shape autotuner. The sandwich and two-sandwich passes of lines of 256 to 2048 points are
// built in up to NSHAPES shapes (PassShape: the default, half and twice the lines per CTA, and seven
// lines per CTA at L = 1024). Per (device,
// precision, points, line length, stride, pass kind) the first launch outside a stream capture times
// the pass itself with each shape (its reductions left out) on a zeroed scratch state: one warm-up
// and three launches each, untimed by the launch counters. A variant replaces the default only when
// it is at least 2% faster. Every line is transformed the same way in every shape, so a pass without
// reductions gives the same bits in each; the shape changes only how the partial sums of a reduction
// are grouped (the CTA count), a rounding-level difference. The choice holds for the whole process,
// so repeated runs agree bit for bit. The committed tuning table (load_shape_table) answers first,
// so that the choice does not depend on one measurement. QND_SHAPE=<v> forces a variant where it
// exists; QND_TUNE=0 keeps the table's choice or the default; QND_TUNE_LOG=<file> appends every
// measurement to that file (the table's source).
struct ShapeKey {
    int device, fp64;
    long long n;
    int L, log2S, mode;
    bool operator<(const ShapeKey& o) const {
        return std::tie(device, fp64, n, L, log2S, mode) < std::tie(o.device, o.fp64, o.n, o.L, o.log2S, o.mode);
    }
};
static std::mutex g_shape_mu;
static std::map<ShapeKey, int> g_shape;

// The committed tuning table (shape_table.tsv beside the library, written from QND_TUNE_LOG
// measurements on a B200): geometries found there take its choice without a measurement, on every
// device of that name. Lines: precision, n=, L=, log2S=, pass kind, ms=..., choice=.
static std::map<std::tuple<int, long long, int, int, int>, int> g_shape_table;
static std::string g_shape_table_device;
static void load_shape_table() {
    static bool loaded = false;
    if (loaded) return;
    loaded = true;
    Dl_info info{};
    if (!dladdr(reinterpret_cast<void*>(&load_shape_table), &info) || !info.dli_fname) return;
    std::string path = info.dli_fname;
    const size_t slash = path.rfind('/');
    path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/shape_table.tsv";
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return;
    char line[512];
    while (std::fgets(line, sizeof line, f)) {
        if (line[0] == '#') {
            const char* k = std::strstr(line, "device=");
            if (k) {
                g_shape_table_device = k + 7;
                while (!g_shape_table_device.empty() &&
                       (g_shape_table_device.back() == '\n' || g_shape_table_device.back() == '\r'))
                    g_shape_table_device.pop_back();
            }
            continue;
        }
        char prec[8] = {0}, kind[16] = {0};
        long long n = 0;
        int L = 0, log2S = 0, choice = 0;
        const char* c = std::strstr(line, "choice=");
        if (!c || std::sscanf(line, "%7s n=%lld L=%d log2S=%d %15s", prec, &n, &L, &log2S, kind) != 5) continue;
        choice = std::atoi(c + 7);
        const int mode = !std::strcmp(kind, "double") ? PM_DOUBLE : PM_SANDWICH;
        g_shape_table[std::make_tuple(!std::strcmp(prec, "fp64") ? 1 : 0, n, L, log2S, mode)] = choice;
    }
    std::fclose(f);
}

static int shape_choice(qnd_ctx* c, const PassSpec& ps, int L, int log2S, int kmode) {
    const int mode = pass_base_mode(kmode);
    if (ps.vL || (mode != PM_SANDWICH && mode != PM_DOUBLE) || L < 256 || L > 2048) return 0;
    const bool strided = log2S > 0;
    if (const char* f = std::getenv("QND_SHAPE")) {
        const int v = std::atoi(f);
        if (v > 0 && v < NSHAPES && lookup_pass(c->fp64, L, strided, kmode, v).fn) return v;
        return 0;
    }
    const ShapeKey key{c->device, int(c->fp64), c->n, L, log2S, mode};
    {
        std::lock_guard<std::mutex> lk(g_shape_mu);
        auto it = g_shape.find(key);
        if (it != g_shape.end()) return it->second;
        load_shape_table();
        auto tt = g_shape_table.find(std::make_tuple(int(c->fp64), (long long)c->n, L, log2S, mode));
        if (tt != g_shape_table.end()) {
            cudaDeviceProp prop{};
            if (cudaGetDeviceProperties(&prop, c->device) == cudaSuccess && g_shape_table_device == prop.name &&
                tt->second >= 0 && tt->second < NSHAPES && lookup_pass(c->fp64, L, strided, mode, tt->second).fn) {
                g_shape[key] = tt->second;
                return tt->second;
            }
        }
    }
    const char* tune = std::getenv("QND_TUNE");
    if ((tune && !std::atoi(tune)) || c->profiling) return 0;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    QND_CK(cudaStreamIsCapturing(c->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return 0;
    if (strided) staging_choice(c, ps, L, log2S);  // settled first: its measurement has its own scratch
    c->shape_buf.ensure(size_t(c->n) * c->elem());
    QND_CK(cudaMemsetAsync(c->shape_buf.p, 0, size_t(c->n) * c->elem(), c->stream));
    PassSpec t = ps;
    t.mode = mode;
    t.red = RedDesc{};
    t.red_at_mid = 0;
    t.psi = c->shape_buf.p;
    const int64_t k0 = c->kernels_launched;
    cudaEvent_t e0, e1;
    QND_CK(cudaEventCreate(&e0));
    QND_CK(cudaEventCreate(&e1));
    float ms[NSHAPES];
    int choice = 0;
    for (int v = 0; v < NSHAPES; ++v) {
        ms[v] = -1.f;
        if (!lookup_pass(c->fp64, L, strided, mode, v).fn) continue;
        t.force_shape = v;
        launch_pass(c, t);
        QND_CK(cudaEventRecord(e0, c->stream));
        for (int r = 0; r < 3; ++r) launch_pass(c, t);
        QND_CK(cudaEventRecord(e1, c->stream));
        QND_CK(cudaEventSynchronize(e1));
        QND_CK(cudaEventElapsedTime(&ms[v], e0, e1));
        if (v > 0 && ms[v] < 0.98f * ms[choice]) choice = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->kernels_launched = k0;
    c->shape_buf.reset();  // after the event wait above: no launch reads it any more
    if (const char* logf = std::getenv("QND_TUNE_LOG")) {
        if (FILE* f = std::fopen(logf, "a")) {
            std::fprintf(f, "%s\tn=%lld\tL=%d\tlog2S=%d\t%s\tms=", c->fp64 ? "fp64" : "fp32", (long long)c->n, L,
                         log2S, mode == PM_DOUBLE ? "double" : "sandwich");
            for (int v = 0; v < NSHAPES; ++v) std::fprintf(f, v ? ",%.4f" : "%.4f", ms[v]);
            std::fprintf(f, "\tchoice=%d\n", choice);
            std::fclose(f);
        }
    }
    std::lock_guard<std::mutex> lk(g_shape_mu);
    g_shape[key] = choice;
    return choice;
}

static void emulate_long_pass(qnd_ctx* c, const PassSpec& ps);

// Launch one fused axis pass: persistent grid (at most the resident CTAs), programmatic
// dependent launch so the pass's prologue overlaps the tail of the previous kernel.
static void launch_pass(qnd_ctx* c, const PassSpec& ps) {
    const int ax = ps.axis;
    if (!ps.vL && c->lax[ax].on) {
        if (c->recorder)
            QND_FAIL(QND_EUNSUPPORTED, "qnd_run_length_sweep: an axis of %lld points is outside the sweep kernel "
                                       "(axis lengths 128 to 1024)", (long long)c->nr[ax]);
        emulate_long_pass(c, ps);  // an axis longer than one pass holds (several dimensions)
        return;
    }
    const int L = ps.vL ? ps.vL : int(c->nr[ax]);
    const int log2S = ps.vL ? ps.vlog2S : c->shift[ax];
    const void* tw = ps.vL ? ps.vtw : c->tw[ax].p;
    const bool strided = log2S > 0;
    // passes that reduce run the instantiation that carries the reduction code; the others keep its
    // registers for the transform
    int kmode = ps.mode;
    if (ps.red.n && ps.mode == PM_SANDWICH) kmode = PM_SANDWICH_RED;
    if (ps.red.n && ps.mode == PM_DOUBLE) kmode = ps.red_at_mid ? PM_DOUBLE_RED : PM_DOUBLE_RED_END;
    // the shape variant: the default while recording (the sweep kernel holds the default shapes)
    const int var = c->recorder ? 0 : (ps.force_shape >= 0 ? ps.force_shape : shape_choice(c, ps, L, log2S, kmode));
    const PassKernelInfo info = lookup_pass(c->fp64, L, strided, kmode, var);
    if (!info.fn) QND_FAIL(QND_EINVAL, "internal: no pass kernel for L=%d, mode %d, shape %d", L, kmode, var);
    if (var != 0 && info.E != lookup_pass(c->fp64, L, strided, kmode, 0).E)
        QND_FAIL(QND_EINVAL, "internal: shape %d of L=%d has its own FFT plan", var, L);  // every shape shares the plan
    const long long nlines = c->n / L;
    const long long ngroups = (nlines + info.G - 1) / info.G;
    if (c->recorder) {
        // qnd_run_length_sweep: the arguments this launch would get (per-thread staging: the sweep
        // kernel takes its arguments from device memory), kept for the persistent kernel
        if (!sweep_length_ok(L) || ps.vL || (kmode != PM_SANDWICH && kmode != PM_SANDWICH_RED && kmode != PM_DOUBLE &&
                                             kmode != PM_DOUBLE_RED && kmode != PM_DOUBLE_RED_END))
            QND_FAIL(QND_EUNSUPPORTED, "qnd_run_length_sweep: a pass of line length %d, mode %d is outside the "
                                       "sweep kernel (axis lengths 128 to 1024)", L, kmode);
        RecordedPass rp;
        rp.L = L;
        rp.strided = strided ? 1 : 0;
        rp.kmode = kmode;
        rp.ngroups = unsigned(std::max<long long>(1, ngroups));
        RedDesc red = ps.red;
        if (red.n) {
            ensure_red_scratch(c, rp.ngroups);
            red.partials = c->partials.as<double>();
            red.counter = c->counter.as<unsigned int>();
        }
        auto record = [&](auto& a) {
            using A = std::remove_reference_t<decltype(a)>;
            a.red = red;
            set_red_axes(c, a.red);
            a.log2S = log2S;
            a.nlines = nlines;
            a.use_tma = 0;
            rp.args.resize(sizeof(A));
            std::memcpy(rp.args.data(), &a, sizeof(A));
        };
        if (c->fp64) {
            PassArgs<double> a;
            fill_args<double>(c, ps, a);
            a.tw = static_cast<const double2*>(tw);
            record(a);
        } else {
            PassArgs<float> a;
            fill_args<float>(c, ps, a);
            a.tw = static_cast<const float2*>(tw);
            record(a);
        }
        c->recorder->push_back(std::move(rp));
        c->kernels_launched++;
        return;
    }
    const int staging = !strided ? 0 : ps.force_staging >= 0 ? ps.force_staging : staging_choice(c, ps, L, log2S);
    // TMA box staging: the tensor map first, then the instantiation compiled for it
    CUtensorMap tmap{};
    const bool use_tma = strided && staging && strided_tma_map(c, ps.psi, L, log2S, info.G, &tmap);
    const PassKernelInfo kinfo = use_tma ? lookup_pass(c->fp64, L, strided, kmode, var, true) : info;
    if (!kinfo.fn) QND_FAIL(QND_EINVAL, "internal: no TMA pass kernel for L=%d, mode %d, shape %d", L, kmode, var);
    // per (kernel, device), shared by the contexts of every host thread
    static std::map<std::pair<const void*, int>, LaunchCfg> configured;
    static std::mutex configured_mu;
    {
        std::lock_guard<std::mutex> lk(configured_mu);
        auto cfg_key = std::make_pair(kinfo.fn, c->device);
        if (configured.find(cfg_key) == configured.end()) {
            QND_CK(cudaFuncSetAttribute(kinfo.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kinfo.smem)));
            LaunchCfg cfg;
            QND_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cfg.blocks_per_sm, kinfo.fn, kinfo.nt, kinfo.smem));
            if (cfg.blocks_per_sm < 1) QND_FAIL(QND_ECUDA, "pass kernel for L=%d does not fit on an SM", L);
            configured.emplace(cfg_key, cfg);
        }
    }
    const long long blocks = std::max<long long>(1, ngroups);
    RedDesc red = ps.red;
    if (red.n) {
        ensure_red_scratch(c, blocks);
        red.partials = c->partials.as<double>();
        red.counter = c->counter.as<unsigned int>();
    }
    std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
    if (c->profiling) {
        for (cudaEvent_t* e : {&ev.first, &ev.second}) {
            if (c->event_pool.empty()) {
                QND_CK(cudaEventCreate(e));
            } else {
                *e = c->event_pool.back();
                c->event_pool.pop_back();
            }
        }
        QND_CK(cudaEventRecord(ev.first, c->stream));
    }
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(unsigned(blocks));
    lc.blockDim = dim3(unsigned(kinfo.nt));
    lc.dynamicSmemBytes = kinfo.smem;
    lc.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = c->pdl ? 1 : 0;
    lc.attrs = attr;
    lc.numAttrs = 1;
    if (c->fp64) {
        PassArgs<double> a;
        fill_args<double>(c, ps, a);
        a.red = red;
        set_red_axes(c, a.red);
        a.tw = static_cast<const double2*>(tw);
        a.log2S = log2S;
        a.nlines = nlines;
        a.use_tma = use_tma ? 1 : 0;
        if (use_tma) a.tmap = tmap;
        void* args[] = {&a};
        QND_CK(cudaLaunchKernelExC(&lc, kinfo.fn, args));
    } else {
        PassArgs<float> a;
        fill_args<float>(c, ps, a);
        a.red = red;
        set_red_axes(c, a.red);
        a.tw = static_cast<const float2*>(tw);
        a.log2S = log2S;
        a.nlines = nlines;
        a.use_tma = use_tma ? 1 : 0;
        if (use_tma) a.tmap = tmap;
        void* args[] = {&a};
        QND_CK(cudaLaunchKernelExC(&lc, kinfo.fn, args));
    }
    c->kernels_launched++;
    if (c->profiling) {
        QND_CK(cudaEventRecord(ev.second, c->stream));
        c->prof_pairs.push_back(ev);
    }
}

static int reduce_blocks(qnd_ctx* c) {
    long long nb = (c->n + 255) / 256;
    if (nb > 148 * 4) nb = 148 * 4;
    return int(nb < 1 ? 1 : nb);
}

// Element-wise r-space reductions of psi.
// lm_axis >= 0: the full-grid weights are in the line-major order of that axis (a pass's layout).
static void grid_reduce(qnd_ctx* c, const void* psi, const RedDesc& rd_in, const void* partner = nullptr,
                        int lm_axis = -1) {
    RedDesc rd = rd_in;
    const int nb = reduce_blocks(c);
    ensure_red_scratch(c, nb);
    rd.partials = c->partials.as<double>();
    rd.counter = c->counter.as<unsigned int>();
    PassSpec ps;
    ps.psi = const_cast<void*>(psi);
    ps.partner = partner;
    ps.red = rd;
    ps.axis = lm_axis >= 0 ? lm_axis : 0;
    if (c->fp64) {
        PassArgs<double> a;
        fill_args<double>(c, ps, a);
        a.red_lm = lm_axis >= 0;
        launch_grid_reduce<double>(a, c->n, c->stream, nb);
    } else {
        PassArgs<float> a;
        fill_args<float>(c, ps, a);
        a.red_lm = lm_axis >= 0;
        launch_grid_reduce<float>(a, c->n, c->stream, nb);
    }
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

// Debug scan (QND_CHECK_FINITE=1): the count of state elements with a NaN or Inf part, read back
// after the call's work; QND_ENONFINITE names the call when there are any.
static void check_finite(qnd_ctx* c, const void* psi, const char* what) {
    const char* e = std::getenv("QND_CHECK_FINITE");
    if (!e || !std::atoi(e)) return;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    QND_CK(cudaStreamIsCapturing(c->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return;  // no read-back inside a capture
    c->finite_slot.ensure(sizeof(double));
    double* slot = c->finite_slot.as<double>();
    RedDesc rd{};
    rd.n = 1;
    rd.kind[0] = RK_NONFINITE;
    rd.wkind[0] = WK_ONE;
    rd.scale[0] = 1.0;
    rd.out = slot;
    grid_reduce(c, psi, rd);
    double bad = 0.0;
    QND_CK(cudaMemcpyAsync(&bad, slot, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    QND_CK(cudaStreamSynchronize(c->stream));
    if (bad > 0.0) QND_FAIL(QND_ENONFINITE, "%s: %.0f state elements hold NaN or Inf", what, bad);
}

// Axes in pass order: the contiguous axis first, axis 0 last (the last pass carries the epilogue).
static std::vector<int> pass_order(const qnd_ctx* c) {
    std::vector<int> o;
    for (int k = c->dim - 1; k >= 0; --k) o.push_back(k);
    return o;
}

// ---------------------------------------------------------------- long axes of N-D grids --
//
// On a grid of two or more dimensions, an axis j of N > 4096 points (N = n1 n2) is transformed in
// four steps in natural order: the length-n1 pass along the virtual axis of stride n2 S_j, the
// twiddles W_N^{k1 m} (element-wise along j), the length-n2 pass along the virtual axis of stride
// S_j, and a permutation from the slot order (slot k1 n2 + k2 holds frequency k1 + n1 k2) to
// natural order; the inverse runs the other way. A pass along j (any mode) is then emulated from
// these transforms and element-wise kernels that apply its factors in natural order (its full-grid
// tables are read in their line-major order for j) and reduce it. Every operation built on passes
// (sandwich chains, imaginary time, the velocity gauge, k-space observables, spectra, adjoints)
// takes such axes unchanged; the cost is more launches and memory passes than a fused pass.

static PassSpec lax_pass(qnd_ctx* c, int ax, int v, int mode, void* psi, double scale) {
    const auto& la = c->lax[ax];
    PassSpec ps;
    ps.axis = ax;
    ps.mode = mode;
    ps.psi = psi;
    ps.scale = scale;
    ps.vL = int(v == 0 ? la.n1 : la.n2);
    ps.vlog2S = v == 0 ? la.lg2 + c->shift[ax] : c->shift[ax];
    ps.vtw = la.tw[v].p;
    return ps;
}

// Element-wise factors along axis ax (see AxisFactorArgs); any pointer may be null.
static void lax_factors(qnd_ctx* c, void* psi, int ax, const void* tr, const void* tc, const void* const* axc,
                        const void* const* axr, const void* spec, int spec_conj, double spec_scale,
                        const double* scale_dev) {
    if (!tr && !tc && !spec && !scale_dev) {
        bool any = false;
        for (int k = 0; k < c->dim; ++k) any = any || (axc && axc[k]) || (axr && axr[k]);
        if (!any) return;
    }
    AxisFactorArgs a{};
    a.n = c->n;
    a.dim = c->dim;
    a.axis = ax;
    a.log2L = c->lognr[ax];
    for (int k = 0; k < MAX_DIM; ++k) {
        a.shift[k] = c->shift[k];
        a.nmask[k] = c->nr[k] - 1;
        a.axc[k] = axc ? axc[k] : nullptr;
        a.axr[k] = axr ? axr[k] : nullptr;
    }
    a.tr = tr;
    a.tc = tc;
    a.spec = spec;
    a.spec_conj = spec_conj;
    a.spec_scale = spec_scale;
    a.scale_dev = scale_dev;
    if (c->fp64) launch_axis_factors<double>(a, static_cast<double2*>(psi), c->stream);
    else launch_axis_factors<float>(a, static_cast<float2*>(psi), c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

static void lax_permute(qnd_ctx* c, void* psi, int ax, bool to_natural) {
    const auto& la = c->lax[ax];
    c->lax_perm.ensure(size_t(c->n) * c->elem());
    AxisPermArgs a{};
    a.n = c->n;
    a.shift = c->shift[ax];
    a.log2N = c->lognr[ax];
    a.log2n1 = la.lg1;
    a.log2n2 = la.lg2;
    if (c->fp64)
        launch_axis_permute<double>(a, static_cast<const double2*>(psi), c->lax_perm.as<double2>(), to_natural, c->stream);
    else
        launch_axis_permute<float>(a, static_cast<const float2*>(psi), c->lax_perm.as<float2>(), to_natural, c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
    QND_CK(cudaMemcpyAsync(psi, c->lax_perm.p, size_t(c->n) * c->elem(), cudaMemcpyDeviceToDevice, c->stream));
}

// Unnormalised transform along axis ax (times scale), natural order in and out.
static void lax_fft(qnd_ctx* c, void* psi, int ax, bool forward, double scale) {
    const auto& la = c->lax[ax];
    if (forward) {
        launch_pass(c, lax_pass(c, ax, 0, PM_FFT_FWD, psi, 1.0));
        lax_factors(c, psi, ax, nullptr, nullptr, nullptr, nullptr, la.twf.p, 0, 1.0, nullptr);
        launch_pass(c, lax_pass(c, ax, 1, PM_FFT_FWD, psi, scale));
        lax_permute(c, psi, ax, true);
    } else {
        lax_permute(c, psi, ax, false);
        launch_pass(c, lax_pass(c, ax, 1, PM_FFT_INV, psi, 1.0));
        lax_factors(c, psi, ax, nullptr, nullptr, nullptr, nullptr, la.twc.p, 0, 1.0, nullptr);
        launch_pass(c, lax_pass(c, ax, 0, PM_FFT_INV, psi, scale));
    }
}

static void emulate_long_pass(qnd_ctx* c, const PassSpec& ps) {
    const int ax = ps.axis;
    const int mode = ps.mode;
    if (ps.spec_full) QND_FAIL(QND_EINVAL, "internal: a full-grid spectral table along a long axis");
    // FP32 spectral tables hold d = w N_axis - 1; the 1/N_axis is applied as a scaling
    const double sscale = c->fp64 ? 1.0 : 1.0 / double(c->nr[ax]);
    void* psi = ps.psi;
    auto sandwich = [&](void* buf, const void* spec) {
        lax_fft(c, buf, ax, true, 1.0);
        lax_factors(c, buf, ax, nullptr, nullptr, nullptr, nullptr, spec, 0, spec ? sscale : 1.0, nullptr);
        lax_fft(c, buf, ax, false, 1.0);
    };
    auto reduce = [&](const void* buf) {
        if (ps.red.n) grid_reduce(c, buf, ps.red, ps.partner, ax);
    };
    if (mode == PM_FFT_FWD || mode == PM_FFT_INV) {
        lax_fft(c, psi, ax, mode == PM_FFT_FWD, ps.scale);
        return;
    }
    if (mode == PM_SANDWICH || mode == PM_DOUBLE) {
        lax_factors(c, psi, ax, ps.pro_real, ps.pro_cplx, ps.ax_in_prologue ? ps.ax_cplx : nullptr, nullptr, nullptr, 0,
                    1.0, ps.pro_scale);
        sandwich(psi, ps.spec);
        if (mode == PM_DOUBLE) {
            lax_factors(c, psi, ax, ps.mid_real, ps.mid_cplx, ps.mid_ax_cplx, ps.mid_ax_real, nullptr, 0, 1.0, nullptr);
            if (ps.red_at_mid) reduce(psi);
            sandwich(psi, ps.spec2);
        }
        lax_factors(c, psi, ax, ps.epi_real, ps.epi_cplx, ps.ax_in_prologue ? nullptr : ps.ax_cplx, ps.ax_real, nullptr, 0,
                    1.0, nullptr);
        if (!ps.red_at_mid) reduce(psi);
        return;
    }
    if (mode == PM_APPLY || mode == PM_SPECRED) {
        // on a copy: the pass's state is not modified
        c->lax_tmp.ensure(size_t(c->n) * c->elem());
        void* tmp = c->lax_tmp.p;
        QND_CK(cudaMemcpyAsync(tmp, psi, size_t(c->n) * c->elem(), cudaMemcpyDeviceToDevice, c->stream));
        if (mode == PM_SPECRED) {
            lax_fft(c, tmp, ax, true, 1.0);
            reduce(tmp);
            return;
        }
        sandwich(tmp, ps.spec);
        if (ps.apply_vtab || ps.apply_acc) {
            if (ps.apply_acc && !ps.dst) QND_FAIL(QND_EINVAL, "internal: an accumulating apply pass without dst");
            void* out = ps.apply_acc ? ps.dst : tmp;
            if (c->fp64)
                launch_apply_combine<double>(c->n, static_cast<double2*>(out), static_cast<const double2*>(tmp),
                                             static_cast<const double2*>(psi), ps.apply_vtab, ps.apply_acc, c->stream);
            else
                launch_apply_combine<float>(c->n, static_cast<float2*>(out), static_cast<const float2*>(tmp),
                                            static_cast<const float2*>(psi), ps.apply_vtab, ps.apply_acc, c->stream);
            c->kernels_launched++;
            QND_CK(cudaGetLastError());
            if (ps.apply_acc) {
                reduce(ps.dst);
                return;
            }
        }
        if (ps.dst) QND_CK(cudaMemcpyAsync(ps.dst, tmp, size_t(c->n) * c->elem(), cudaMemcpyDeviceToDevice, c->stream));
        reduce(ps.dst ? ps.dst : tmp);
        return;
    }
    QND_FAIL(QND_EUNSUPPORTED, "internal: pass mode %d along an axis longer than 4096 points", mode);
}

// ---------------------------------------------------------------- long axes --
//
// A 1-D axis of N = n1 n2 points (n2 = min(4096, N / 16), n1 = N / n2) is transformed in four
// steps over the virtual n1 x n2 grid in which point n1_ n2 + n2_ sits (natural order):
//   F[k1 + n1 k2] = sum_{n2_} W_{n2}^{n2_ k2} W_N^{n2_ k1} sum_{n1_} W_{n1}^{n1_ k1} psi[n1_ n2 + n2_]
// i.e. length-n1 transforms along the strided virtual axis, the twiddles W_N^{k1 n2_}, then
// length-n2 transforms along the contiguous one; the spectrum lands in slot order (slot k1 n2 + k2
// holds frequency k1 + n1 k2), where every k-space table of the axis is stored. A kinetic sandwich
// F^-1 K F is three passes: length-n1 forward; one length-n2 sandwich pass with the twiddles as its
// prologue, the slot-order table K as its spectral factor and the conjugate twiddles as its
// epilogue; length-n1 inverse carrying the last 1/n1. The r-space work between sandwiches (factor
// tables, laser phases, the mask, reductions) runs as element-wise kernels in natural order.

static PassSpec long_pass(qnd_ctx* c, int v, int mode, void* psi, double scale) {
    PassSpec ps;
    ps.axis = 0;
    ps.mode = mode;
    ps.psi = psi;
    ps.scale = scale;
    ps.vL = int(v == 0 ? c->n1 : c->n2);
    ps.vlog2S = v == 0 ? c->lg2 : 0;
    ps.vtw = c->tw_long[v].p;
    return ps;
}

static LongArgs long_args(const qnd_ctx* c) {
    LongArgs a{};
    a.n = c->n;
    a.log2n1 = c->lg1;
    a.log2n2 = c->lg2;
    return a;
}

static void long_twiddle(qnd_ctx* c, void* psi, bool conj) {
    if (c->fp64)
        launch_long_twiddle<double>(long_args(c), static_cast<double2*>(psi), c->twf_long.as<double2>(), conj, c->stream);
    else
        launch_long_twiddle<float>(long_args(c), static_cast<float2*>(psi), c->twf_long.as<float2>(), conj, c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

// Unnormalised transform (times s1 s2): forward from natural order into slot order, inverse back.
static void long_fft(qnd_ctx* c, void* psi, bool forward, double s1, double s2) {
    if (forward) {
        launch_pass(c, long_pass(c, 0, PM_FFT_FWD, psi, s1));
        long_twiddle(c, psi, false);
        launch_pass(c, long_pass(c, 1, PM_FFT_FWD, psi, s2));
    } else {
        launch_pass(c, long_pass(c, 1, PM_FFT_INV, psi, s2));
        long_twiddle(c, psi, true);
        launch_pass(c, long_pass(c, 0, PM_FFT_INV, psi, s1));
    }
}

// psi <- F^-1 spec F psi for a slot-order spectral table (1/N included as described above).
static void long_sandwich(qnd_ctx* c, void* psi, const void* spec) {
    launch_pass(c, long_pass(c, 0, PM_FFT_FWD, psi, 1.0));
    PassSpec ps = long_pass(c, 1, PM_SANDWICH, psi, 1.0);
    ps.pro_cplx = c->twf_long.p;
    ps.spec = spec;
    ps.spec_full = 1;
    ps.epi_cplx = c->twc_long.p;
    launch_pass(c, ps);
    launch_pass(c, long_pass(c, 0, PM_FFT_INV, psi, 1.0 / double(c->n1)));
}

// Slot order <-> natural order, through the context's long-axis scratch state.
static void long_reorder(qnd_ctx* c, void* psi, bool to_natural) {
    c->long_tmp.ensure(size_t(c->n) * c->elem());
    if (c->fp64)
        launch_long_transpose<double>(long_args(c), static_cast<const double2*>(psi), c->long_tmp.as<double2>(),
                                      to_natural, c->stream);
    else
        launch_long_transpose<float>(long_args(c), static_cast<const float2*>(psi), c->long_tmp.as<float2>(),
                                     to_natural, c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
    QND_CK(cudaMemcpyAsync(psi, c->long_tmp.p, size_t(c->n) * c->elem(), cudaMemcpyDeviceToDevice, c->stream));
}

static void long_point(qnd_ctx* c, void* psi, const void* treal, const void* tcplx, const void* pcplx, const void* preal,
                       const double* scale_dev) {
    if (!treal && !tcplx && !pcplx && !preal && !scale_dev) return;
    if (c->fp64)
        launch_point_factors<double>(c->n, static_cast<double2*>(psi), static_cast<const double*>(treal),
                                     static_cast<const double2*>(tcplx), static_cast<const double2*>(pcplx),
                                     static_cast<const double*>(preal), scale_dev, c->stream);
    else
        launch_point_factors<float>(c->n, static_cast<float2*>(psi), static_cast<const float*>(treal),
                                    static_cast<const float2*>(tcplx), static_cast<const float2*>(pcplx),
                                    static_cast<const float*>(preal), scale_dev, c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

// dst = H src = F^-1 (p^2/2) F src + V src (the kinetic operator of calculate_observables.c:165).
static void long_apply_h(qnd_ctx* c, const void* src, void* dst, const void* kin_spec, const double* vpot) {
    QND_CK(cudaMemcpyAsync(dst, src, size_t(c->n) * c->elem(), cudaMemcpyDeviceToDevice, c->stream));
    long_sandwich(c, dst, kin_spec);
    if (c->fp64)
        launch_add_potential<double>(c->n, static_cast<double2*>(dst), static_cast<const double2*>(src), vpot, c->stream);
    else
        launch_add_potential<float>(c->n, static_cast<float2*>(dst), static_cast<const float2*>(src), vpot, c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

// ---------------------------------------------------------------- observables --

static std::vector<ObsItem> parse_obs(qnd_ctx* c, int nobs, const char* const* names, int* nvalues) {
    std::vector<ObsItem> items;
    int off = 0;
    for (int k = 0; k < nobs; ++k) {
        const char* nm = names[k] ? names[k] : "";
        ObsItem it{OB_ZERO, off, 0};
        if (!strcmp(nm, "norm")) it = {OB_NORM, off, 1};
        else if (!strcmp(nm, "dipole_r")) it = {OB_DIPOLE_R, off, c->dim};
        else if (!strcmp(nm, "accel")) it = {OB_ACCEL, off, c->dim};
        else if (!strcmp(nm, "dipole_v")) it = {OB_DIPOLE_V, off, c->dim};
        else if (!strcmp(nm, "energy")) it = {OB_ENERGY, off, 1};
        else if (!strcmp(nm, "Lz")) it = {OB_LZ, off, 1};
        if (it.kind == OB_ACCEL)
            for (int j = 0; j < c->dim; ++j)
                if (!c->gradv_dev[j].p) QND_FAIL(QND_EINVAL, "observable 'accel' needs qnd_set_gradv for every axis");
        off += it.width;
        items.push_back(it);
    }
    if (nvalues) *nvalues = off;
    return items;
}

static bool all_rspace(const std::vector<ObsItem>& items) {
    for (auto& it : items)
        if (it.kind == OB_DIPOLE_V || it.kind == OB_ENERGY || it.kind == OB_LZ) return false;
    return true;
}

// Reductions of |psi|^2 for the r-space observables, writing into row (the contiguous
// outputs must be adjacent: r-space items are emitted in one descriptor per contiguous run).
// dV/dx_j laid out line-major for pass axis ax (the natural array when ax is the last axis).
static const double* gradv_layout(qnd_ctx* c, int j, int ax) {
    if (ax == c->dim - 1) return c->gradv_dev[j].as<double>();
    DevBuf& b = c->gradv_lm[j][ax];
    if (!b.p) upload_f64(c, b, line_major(c, c->gradv[j], 1, ax));
    return b.as<double>();
}

// lm_axis: the pass axis whose line-major order the fused reduction visits (dim-1: natural).
static std::vector<RedDesc> rspace_red(qnd_ctx* c, const std::vector<ObsItem>& items, double* row, int lm_axis) {
    std::vector<RedDesc> out;
    RedDesc cur{};
    int cur_off = -1;
    auto flush = [&]() {
        if (cur.n) out.push_back(cur);
        cur = RedDesc{};
        cur_off = -1;
    };
    auto add = [&](int off, int kind, int wkind, int waxis, const double* wtab, double scale) {
        if (cur.n == MAX_RED || (cur.n && cur_off + cur.n != off)) flush();
        if (!cur.n) {
            cur_off = off;
            cur.out = row + off;
        }
        cur.kind[cur.n] = kind;
        cur.wkind[cur.n] = wkind;
        cur.waxis[cur.n] = waxis;
        cur.wtab[cur.n] = wtab;
        cur.scale[cur.n] = scale;
        cur.n++;
    };
    for (auto& it : items) {
        if (it.kind == OB_NORM) add(it.offset, RK_ABS2, WK_ONE, 0, nullptr, c->dNr);
        else if (it.kind == OB_DIPOLE_R)
            for (int j = 0; j < c->dim; ++j) add(it.offset + j, RK_ABS2, WK_AXIS, j, c->r_dev.as<double>() + c->axoff[j], c->dNr);
        else if (it.kind == OB_ACCEL)
            for (int j = 0; j < c->dim; ++j) add(it.offset + j, RK_ABS2, WK_GRID, 0, gradv_layout(c, j, lm_axis), -c->dNr);
    }
    flush();
    return out;
}

static void ensure_scratch_state(qnd_ctx* c, DevBuf& b) { b.ensure(size_t(c->n) * c->elem()); }

static void ensure_vpot_dev(qnd_ctx* c) {
    if (c->vpot.empty()) QND_FAIL(QND_EINVAL, "no potential set");
    if (!c->vpot_dev.p) upload_f64(c, c->vpot_dev, c->vpot);
}

// out[m-1] = Re <psi | H^m | psi> dNr for m = 1..nmom (calculate_observables.c:146-175), written to dev.
static void energy_moments(qnd_ctx* c, const void* psi, int nmom, double* out_dev) {
    ensure_vpot_dev(c);
    ensure_scratch_state(c, c->scratch_a);
    if (nmom > 1) ensure_scratch_state(c, c->scratch_b);
    const void* src = psi;
    auto order = pass_order(c);
    for (int m = 1; m <= nmom; ++m) {
        void* dst = (m % 2) ? c->scratch_a.p : c->scratch_b.p;
        if (c->long1d) {
            long_apply_h(c, src, dst, spec_table(c, SP_KIN, 0, 0.0), c->vpot_dev.as<double>());
            RedDesc rd{};
            rd.n = 1;
            rd.kind[0] = RK_BILIN;
            rd.wkind[0] = WK_ONE;
            rd.scale[0] = c->dNr;
            rd.out = out_dev + (m - 1);
            grid_reduce(c, dst, rd, psi);
            src = dst;
            continue;
        }
        for (size_t q = 0; q < order.size(); ++q) {
            const int ax = order[q];
            PassSpec ps;
            ps.axis = ax;
            ps.mode = PM_APPLY;
            ps.psi = const_cast<void*>(src);
            ps.dst = dst;
            ps.spec = spec_table(c, SP_KIN, ax, 0.0);
            if (q == 0) ps.apply_vtab = c->vpot_dev.as<double>();
            else ps.apply_acc = 1;
            if (q + 1 == order.size()) {
                ps.partner = psi;
                ps.red.n = 1;
                ps.red.kind[0] = RK_BILIN;
                ps.red.wkind[0] = WK_ONE;
                ps.red.scale[0] = c->dNr;
                ps.red.out = out_dev + (m - 1);
            }
            launch_pass(c, ps);
        }
        src = dst;
    }
}

// Evaluate observables of an r-space psi into the device row (calculate_observables.c:119-140).
static void eval_obs(qnd_ctx* c, const void* psi, const std::vector<ObsItem>& items, const double* alpha,
                     double* row_dev) {
    for (auto& rd : rspace_red(c, items, row_dev, c->dim - 1)) grid_reduce(c, psi, rd);
    for (auto& it : items) {
        if (it.kind == OB_DIPOLE_V) {
            // sum_k |psi~|^2 (p_j + alpha_j) dNp fft_scaling = (dNp/N_j) sum |F_j psi|^2 (p_j + alpha_j)
            if (c->long1d) {
                // |F psi|^2 in slot order, weighted by the slot momenta
                c->long_tmp.ensure(size_t(c->n) * c->elem());
                QND_CK(cudaMemcpyAsync(c->long_tmp.p, psi, size_t(c->n) * c->elem(), cudaMemcpyDeviceToDevice,
                                       c->stream));
                long_fft(c, c->long_tmp.p, true, 1.0, 1.0);
                c->wtab_dev[0].ensure(size_t(c->n) * 8);
                launch_axis_table<double>(0, c->p_slot_dev.as<double>(), int(c->n), alpha[0], c->wtab_dev[0].p,
                                          c->stream);
                c->kernels_launched++;
                RedDesc rd{};
                rd.n = 1;
                rd.kind[0] = RK_ABS2;
                rd.wkind[0] = WK_AXIS;
                rd.waxis[0] = 0;
                rd.wtab[0] = c->wtab_dev[0].as<double>();
                rd.scale[0] = c->dNp / double(c->n);
                rd.out = row_dev + it.offset;
                grid_reduce(c, c->long_tmp.p, rd);
                continue;
            }
            for (int j = 0; j < c->dim; ++j) {
                c->wtab_dev[j].ensure(size_t(c->nr[j]) * 8);
                if (c->fp64)
                    launch_axis_table<double>(0, c->p_dev.as<double>() + c->axoff[j], int(c->nr[j]), alpha[j],
                                              c->wtab_dev[j].p, c->stream);
                else
                    launch_axis_table<float>(0, c->p_dev.as<double>() + c->axoff[j], int(c->nr[j]), alpha[j],
                                             c->wtab_dev[j].p, c->stream);
                c->kernels_launched++;
                PassSpec ps;
                ps.axis = j;
                ps.mode = PM_SPECRED;
                ps.psi = const_cast<void*>(psi);
                ps.red.n = 1;
                ps.red.kind[0] = RK_ABS2;
                ps.red.wkind[0] = WK_AXIS;
                ps.red.waxis[0] = j;
                ps.red.wtab[0] = c->wtab_dev[j].as<double>();
                ps.red.scale[0] = c->dNp / double(c->nr[j]);
                ps.red.out = row_dev + it.offset + j;
                launch_pass(c, ps);
            }
        } else if (it.kind == OB_ENERGY) {
            energy_moments(c, psi, 1, row_dev + it.offset);
        } else if (it.kind == OB_LZ) {
            if (c->dim <= 1) {
                QND_CK(cudaMemsetAsync(row_dev + it.offset, 0, sizeof(double), c->stream));
                continue;
            }
            // Lz = Re sum conj(psi) [x T'_y psi - y T'_x psi] dNr, T'_j = F_j^-1 (p_j + A_j) F_j / N_j
            for (int q = 0; q < 2; ++q) {
                const int opax = q == 0 ? 1 : 0, wax = q == 0 ? 0 : 1;
                c->spec_tmp[opax].ensure(size_t(c->nr[opax]) * c->elem());
                if (c->fp64)
                    launch_axis_table<double>(1, c->p_dev.as<double>() + c->axoff[opax], int(c->nr[opax]),
                                              alpha[opax], c->spec_tmp[opax].p, c->stream);
                else
                    launch_axis_table<float>(1, c->p_dev.as<double>() + c->axoff[opax], int(c->nr[opax]),
                                             alpha[opax], c->spec_tmp[opax].p, c->stream);
                c->kernels_launched++;
                PassSpec ps;
                ps.axis = opax;
                ps.mode = PM_APPLY;
                ps.psi = const_cast<void*>(psi);
                ps.spec = c->spec_tmp[opax].p;
                ps.partner = psi;
                ps.red.n = 1;
                ps.red.kind[0] = RK_BILIN;
                ps.red.wkind[0] = WK_AXIS;
                ps.red.waxis[0] = wax;
                ps.red.wtab[0] = c->r_dev.as<double>() + c->axoff[wax];
                ps.red.scale[0] = q == 0 ? c->dNr : -c->dNr;
                ps.red.accumulate = q;
                ps.red.out = row_dev + it.offset;
                launch_pass(c, ps);
            }
        } else if (it.kind == OB_ZERO && it.width) {
            QND_CK(cudaMemsetAsync(row_dev + it.offset, 0, it.width * sizeof(double), c->stream));
        }
    }
}

// ---------------------------------------------------------------- steps --

static void check_imag_clamp(qnd_ctx* c) {
    // The per-axis factorisation of exp(min(700, -c Kin)) is exact unless the clamp engages.
    double kmax = 0;
    for (int j = 0; j < c->dim; ++j) {
        double m = 0;
        for (double pk : c->p[j]) m = std::max(m, .5 * pk * pk);
        kmax += m;
    }
    for (int ia = 0; ia < c->s; ++ia) {
        const double h = c->as[2 * ia] + c->as[2 * ia + 1];
        if (-h * kmax > MAX_EXP_ARG)
            QND_FAIL(QND_EUNSUPPORTED,
                     "imaginary-time kinetic factor reaches the exp(700) clamp (dt too large for this grid)");
    }
}

// Per-step field tables (laser phases / velocity-gauge kinetic phases) for a chunk of steps
// from field samples already on the device.
static void build_field_tables(qnd_ctx* c, const double* field_dev, int64_t nsteps, bool velocity,
                               int conj_from = 1 << 30, void* out = nullptr) {
    FieldTableArgs fa{};
    fa.conj_from = conj_from;
    fa.field = field_dev;
    // velocity tables of a long axis: slot order (k-space tables), the 1/n2 of its sandwich pass
    fa.axes = velocity ? (c->long1d ? c->p_slot_dev.as<double>() : c->p_dev.as<double>()) : c->r_dev.as<double>();
    fa.nsteps = int(nsteps);
    fa.s = c->s;
    fa.dim = c->dim;
    for (int j = 0; j < c->dim; ++j) {
        fa.nr[j] = int(c->long1d ? c->n2 : c->nr[j]);
        fa.off[j] = c->axoff[j];
    }
    fa.ntot = c->axtot;
    for (int ia = 0; ia < c->s; ++ia) fa.h[ia] = c->as[2 * ia] + c->as[2 * ia + 1];
    fa.velocity = velocity ? 1 : 0;
    if (!out) {
        c->field_tab.ensure(size_t(nsteps) * c->s * c->axtot * c->elem());
        out = c->field_tab.p;
    }
    if (c->fp64) launch_field_tables<double>(fa, static_cast<double2*>(out), c->stream);
    else launch_field_tables<float>(fa, static_cast<float2*>(out), c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

static void upload_field_chunk(qnd_ctx* c, const double* host, int64_t nsteps, bool velocity, int conj_from = 1 << 30) {
    const size_t nval = size_t(nsteps) * c->s * c->dim;
    c->field_dev.ensure(nval * 8);
    QND_CK(cudaMemcpyAsync(c->field_dev.p, host, nval * 8, cudaMemcpyHostToDevice, c->stream));
    build_field_tables(c, c->field_dev.as<double>(), nsteps, velocity, conj_from);
}

static const void* field_slice(qnd_ctx* c, int64_t st, int ia, int ax) {
    const size_t idx = (size_t(st) * c->s + ia) * c->axtot + c->axoff[ax];
    const void* base = c->field_view ? c->field_view : c->field_tab.p;
    return static_cast<const char*>(base) + idx * c->elem();
}

static bool has_mask(const qnd_ctx* c) {
    for (int j = 0; j < c->dim; ++j)
        if (c->mask_dev[j].p) return true;
    return false;
}

// ---------------------------------------------------------------- sandwich chains --

struct Factor {
    int kind = -1;        // RT_IMAG (real table), RT_LENGTH / RT_VEL (complex), -1: none
    double a = 0.0, b = NO_COEF;
    int laser_ia = -1;    // length gauge: per-axis laser phases of sub-step laser_ia
};

// A kinetic sandwich: exp(-i coef p_j^2/2)/N_j (SP_LENGTH), exp(-coef p_j^2/2)/N_j (SP_IMAG), or
// the velocity-gauge k-space phases of sub-step ia of chunk step lst (KV_FIELD).
constexpr int KV_FIELD = 100;
struct ChainK {
    int kind = SP_LENGTH;
    double coef = 0.0;
    int64_t lst = 0;
    int ia = 0;
};

// Point-wise r-space work between two sandwiches (or after the last one): a factor (a full-grid
// table and/or the laser phases of chunk step lst), the step mask, then reductions of the state.
struct ChainMid {
    Factor f;
    int64_t lst = 0;
    bool mask = false;
    const RedDesc* red = nullptr;
    bool empty() const { return f.kind < 0 && f.laser_ia < 0 && !mask && !red; }
};

static void set_factor(qnd_ctx* c, const Factor& f, int ax, int64_t lst, const void** treal, const void** tcplx,
                       const void** axc) {
    if (f.kind >= 0) {
        const void* p = rtab(c, f.kind, f.a, f.b, ax);
        if (f.kind == RT_IMAG) *treal = p;
        else *tcplx = p;
    }
    if (f.laser_ia >= 0 && axc)
        for (int j = 0; j < c->dim; ++j) axc[j] = field_slice(c, lst, f.laser_ia, j);
}

static const void* chain_spec(qnd_ctx* c, const ChainK& k, int ax) {
    if (k.kind == KV_FIELD) return field_slice(c, k.lst, k.ia, ax);
    return spec_table(c, k.kind, ax, k.coef);
}

// Axis of the pass that ends sandwich i of a chain (it carries the factor after sandwich i).
static int sandwich_last_axis(const qnd_ctx* c, int64_t i) {
    if (c->dim == 1) return 0;
    return (i % 2 == 0) ? 0 : c->dim - 1;
}

// Axis of the chain's last pass (the one that carries the final factor, mask and reductions).
static int chain_final_axis(const qnd_ctx* c, int NK) { return sandwich_last_axis(c, NK - 1); }

// Run a chain of kinetic sandwiches K_0 .. K_{NK-1} with M[i] between K_i and K_{i+1}, `pre` (and
// the device scalar pre_scale) before K_0 and `post` after K_{NK-1}. Consecutive sandwiches run
// their axes in opposite orders, so the last axis of K_i is the first axis of K_{i+1}: those two
// axis passes and M[i] fuse into one PM_DOUBLE pass. A chain of NK sandwiches costs NK + 1 passes
// in 2-D (2 NK + 1 in 3-D) instead of d NK; in 1-D the sandwiches pair up two per pass, and a
// factor between pairs moves into the next pass's prologue (1-D chains carry no mask or
// reductions between sandwiches).
static void run_chain(qnd_ctx* c, void* psi, const std::vector<ChainK>& K, const std::vector<ChainMid>& M,
                      const Factor& pre, int64_t pre_lst, const double* pre_scale, const ChainMid& post) {
    const int d = c->dim;
    const int64_t NK = int64_t(K.size());
    if (NK == 0 || int64_t(M.size()) != NK - 1) QND_FAIL(QND_EINVAL, "internal: malformed sandwich chain");
    if (c->long1d) {
        // four-step sandwiches: length-n1 forward, the length-n2 sandwich pass (twiddles, slot-order
        // k-space table, conjugate twiddles), then either one length-n1 roundtrip pass (inverse,
        // the r-space factors in natural order, forward of the next sandwich; FP32) or the
        // length-n1 inverse and element-wise work in natural order (FP64, reductions, chain end)
        auto point = [&](const Factor& f, int64_t lst, bool mask, const double* scale_dev) {
            const void *tr = nullptr, *tc = nullptr;
            const void* axc[MAX_DIM] = {};
            set_factor(c, f, 0, lst, &tr, &tc, axc);
            long_point(c, psi, tr, tc, axc[0], mask ? c->mask_dev[0].p : nullptr, scale_dev);
        };
        point(pre, pre_lst, false, pre_scale);
        launch_pass(c, long_pass(c, 0, PM_FFT_FWD, psi, 1.0));
        for (int64_t i = 0; i < NK; ++i) {
            PassSpec ps = long_pass(c, 1, PM_SANDWICH, psi, 1.0);
            ps.pro_cplx = c->twf_long.p;
            ps.spec = chain_spec(c, K[i], 0);
            ps.spec_full = 1;
            ps.epi_cplx = c->twc_long.p;
            launch_pass(c, ps);
            const bool last = i + 1 == NK;
            const ChainMid& m = last ? post : M[i];
            // the roundtrip gathers its natural-order tables across the strided virtual axis:
            // measured 13% faster per step in FP32 at 262144 points, 4% slower in FP64 (where the
            // separate coalesced element-wise kernel wins)
            if (!last && !m.red && !c->fp64) {
                PassSpec r = long_pass(c, 0, PM_ROUNDTRIP, psi, 1.0 / double(c->n1));
                set_factor(c, m.f, 0, m.lst, &r.mid_real, &r.mid_cplx, r.mid_ax_cplx);
                if (m.mask) r.mid_ax_real[0] = c->mask_dev[0].p;
                launch_pass(c, r);
                continue;
            }
            launch_pass(c, long_pass(c, 0, PM_FFT_INV, psi, 1.0 / double(c->n1)));
            point(m.f, m.lst, m.mask, nullptr);
            if (m.red) grid_reduce(c, psi, *m.red);
            if (!last) launch_pass(c, long_pass(c, 0, PM_FFT_FWD, psi, 1.0));
        }
        return;
    }
    auto finish = [&](PassSpec& ps) {
        // laser phases after the chain go in the last pass's epilogue (its prologue must have none)
        const bool lasers = post.f.laser_ia >= 0;
        if (lasers && ps.ax_in_prologue) QND_FAIL(QND_EINVAL, "internal: laser phases on both sides of one pass");
        set_factor(c, post.f, ps.axis, post.lst, &ps.epi_real, &ps.epi_cplx, lasers ? ps.ax_cplx : nullptr);
        if (post.mask)
            for (int j = 0; j < d; ++j) ps.ax_real[j] = c->mask_dev[j].p;
        if (post.red) ps.red = *post.red;
    };
    if (d == 1) {
        int64_t i = 0;
        while (i < NK) {
            PassSpec ps;
            ps.axis = 0;
            ps.psi = psi;
            ps.spec = chain_spec(c, K[i], 0);
            if (i == 0) {
                set_factor(c, pre, 0, pre_lst, &ps.pro_real, &ps.pro_cplx, ps.ax_cplx);
                if (pre.laser_ia >= 0) ps.ax_in_prologue = 1;
                ps.pro_scale = pre_scale;
            } else {
                const ChainMid& b = M[i - 1];
                if (b.mask || b.red) QND_FAIL(QND_EINVAL, "internal: 1-D chain with a mask or reduction inside");
                set_factor(c, b.f, 0, b.lst, &ps.pro_real, &ps.pro_cplx, ps.ax_cplx);
                if (b.f.laser_ia >= 0) ps.ax_in_prologue = 1;
            }
            if (i + 1 < NK) {
                const ChainMid& m = M[i];
                if (m.mask || m.red) QND_FAIL(QND_EINVAL, "internal: 1-D chain with a mask or reduction inside");
                ps.mode = PM_DOUBLE;
                set_factor(c, m.f, 0, m.lst, &ps.mid_real, &ps.mid_cplx, ps.mid_ax_cplx);
                ps.spec2 = chain_spec(c, K[i + 1], 0);
                i += 2;
            } else {
                i += 1;
            }
            if (i >= NK) finish(ps);
            launch_pass(c, ps);
        }
        return;
    }
    for (int64_t i = 0; i < NK; ++i) {
        for (int q = (i > 0 ? 1 : 0); q < d; ++q) {
            const int ax = (i % 2 == 0) ? d - 1 - q : q;
            PassSpec ps;
            ps.axis = ax;
            ps.psi = psi;
            ps.spec = chain_spec(c, K[i], ax);
            if (i == 0 && q == 0) {
                set_factor(c, pre, ax, pre_lst, &ps.pro_real, &ps.pro_cplx, ps.ax_cplx);
                if (pre.laser_ia >= 0) ps.ax_in_prologue = 1;
                ps.pro_scale = pre_scale;
            }
            if (q == d - 1 && i + 1 < NK) {
                const ChainMid& m = M[i];
                ps.mode = PM_DOUBLE;
                set_factor(c, m.f, ax, m.lst, &ps.mid_real, &ps.mid_cplx, ps.mid_ax_cplx);
                if (m.mask)
                    for (int j = 0; j < d; ++j) ps.mid_ax_real[j] = c->mask_dev[j].p;
                if (m.red) {
                    ps.red = *m.red;
                    ps.red_at_mid = 1;
                }
                ps.spec2 = chain_spec(c, K[i + 1], ax);
            }
            if (q == d - 1 && i + 1 == NK) finish(ps);
            launch_pass(c, ps);
        }
    }
}

// Reductions after step k of a multi-step chain, with full-grid weights laid out line-major for
// pass axis `axis` (the pass that carries them); at most one descriptor.
using RedFn = std::function<std::vector<RedDesc>(int64_t k, int axis)>;

// Integration_step_imag x nsteps on an r-space psi (integrators.c:135-163): per step V(a_0) K(h_0)
// V(a_1)V(a_2) K(h_1) ... K(h_{s-1}) V(a_{2s-1}); between steps V(a_{2s-1})V(a_0) is one factor.
// pro_scale (device scalar, may be null) multiplies psi first (the deferred Gram-Schmidt
// normalisation).
static void imag_steps(qnd_ctx* c, void* psi, int64_t nsteps, const double* pro_scale) {
    check_imag_clamp(c);
    if (nsteps <= 0) return;
    const int s = c->s;
    std::vector<ChainK> K;
    std::vector<ChainMid> M;
    for (int64_t st = 0; st < nsteps; ++st)
        for (int i = 0; i < s; ++i) {
            if (i > 0 || st > 0) {
                ChainMid m;
                m.f.kind = RT_IMAG;
                m.f.a = i > 0 ? c->as[2 * i - 1] : c->as[2 * s - 1];
                m.f.b = c->as[2 * i];
                M.push_back(m);
            }
            ChainK k;
            k.kind = SP_IMAG;
            k.coef = c->as[2 * i] + c->as[2 * i + 1];
            K.push_back(k);
        }
    Factor pre;
    ChainMid post;
    pre.kind = post.f.kind = RT_IMAG;
    pre.a = c->as[0];
    post.f.a = c->as[2 * s - 1];
    run_chain(c, psi, K, M, pre, 0, pro_scale, post);
}

// Length-gauge steps lst0 .. lst0+n-1 of the current field chunk in r-space (integrators.c:170-194
// rewritten in r-space): per step K(a_0) V(h_0) K(a_1 + a_2) V(h_1) ... V(h_{s-1}) K(a_{2s-1}); after
// each step the step mask and the reductions red_fn(k, .) (of psi(t_{k+1})). A step boundary with
// nothing on it merges K(a_{2s-1}) with the next step's K(a_0).
static void length_steps(qnd_ctx* c, void* psi, int64_t lst0, int64_t n, const RedFn& red_fn, bool masked) {
    if (n <= 0) return;
    if (c->dim == 1 && !c->long1d && n > 1 && (masked || red_fn)) {
        // 1-D chains carry boundary work only at their end
        for (int64_t k = 0; k < n; ++k)
            length_steps(c, psi, lst0 + k, 1, red_fn ? RedFn([&](int64_t, int ax) { return red_fn(k, ax); }) : RedFn(),
                         masked);
        return;
    }
    const int s = c->s;
    auto kc = [&](int i) {
        if (i == 0) return c->as[0];
        if (i == s) return c->as[2 * s - 1];
        return c->as[2 * i - 1] + c->as[2 * i];
    };
    std::vector<ChainK> K;
    std::vector<ChainMid> M;
    std::vector<std::vector<RedDesc>> reds;
    reds.reserve(size_t(n) + 1);
    auto reductions = [&](int64_t k) -> const RedDesc* {
        if (!red_fn) return nullptr;
        reds.push_back(red_fn(k, sandwich_last_axis(c, int64_t(K.size()) - 1)));
        if (reds.back().size() > 1) QND_FAIL(QND_EINVAL, "internal: more than one reduction descriptor in a chain");
        return reds.back().empty() ? nullptr : &reds.back()[0];
    };
    for (int64_t k = 0; k < n; ++k) {
        const int64_t lst = lst0 + k;
        for (int i = 0; i <= s; ++i) {
            ChainK kk;
            kk.kind = SP_LENGTH;
            kk.coef = kc(i);
            if (i == 0 && k > 0) {
                ChainMid b;
                b.lst = lst - 1;
                b.mask = masked;
                b.red = reductions(k - 1);
                if (b.empty()) {
                    K.back().coef += kk.coef;
                    continue;
                }
                M.push_back(b);
            } else if (i > 0) {
                ChainMid m;
                m.f.kind = RT_LENGTH;
                m.f.a = c->as[2 * (i - 1)] + c->as[2 * (i - 1) + 1];
                m.f.laser_ia = i - 1;
                m.lst = lst;
                M.push_back(m);
            }
            K.push_back(kk);
        }
    }
    ChainMid post;
    post.lst = lst0 + n - 1;
    post.mask = masked;
    post.red = reductions(n - 1);
    run_chain(c, psi, K, M, Factor{}, lst0, nullptr, post);
}

// Velocity-gauge steps lst0 .. lst0+n-1 in r-space (integrators.c:201-232); between steps the
// factors V(a_{2s-1}) V(a_0) merge into one. The step mask and the reductions `fin` apply after the
// last step only.
static void velocity_steps(qnd_ctx* c, void* psi, int64_t lst0, int64_t n, const RedDesc* fin, bool masked) {
    if (n <= 0) return;
    const int s = c->s;
    std::vector<ChainK> K;
    std::vector<ChainMid> M;
    for (int64_t k = 0; k < n; ++k)
        for (int i = 0; i < s; ++i) {
            if (i > 0 || k > 0) {
                ChainMid m;
                m.f.kind = RT_VEL;
                m.f.a = i > 0 ? c->as[2 * i - 1] : c->as[2 * s - 1];
                m.f.b = c->as[2 * i];
                M.push_back(m);
            }
            ChainK kk;
            kk.kind = KV_FIELD;
            kk.lst = lst0 + k;
            kk.ia = i;
            K.push_back(kk);
        }
    Factor pre;
    ChainMid post;
    pre.kind = post.f.kind = RT_VEL;
    pre.a = c->as[0];
    post.f.a = c->as[2 * s - 1];
    post.lst = lst0 + n - 1;
    post.mask = masked;
    post.red = fin;
    run_chain(c, psi, K, M, pre, lst0, nullptr, post);
}

static void unitary_fft(qnd_ctx* c, void* psi, bool forward) {
    if (c->long1d) {
        const double s1 = 1.0 / std::sqrt(double(c->n1)), s2 = 1.0 / std::sqrt(double(c->n2));
        if (forward) {
            long_fft(c, psi, true, s1, s2);
            long_reorder(c, psi, true);
        } else {
            long_reorder(c, psi, false);
            long_fft(c, psi, false, s1, s2);
        }
        return;
    }
    for (int ax : pass_order(c)) {
        PassSpec ps;
        ps.axis = ax;
        ps.mode = forward ? PM_FFT_FWD : PM_FFT_INV;
        ps.psi = psi;
        ps.scale = 1.0 / std::sqrt(double(c->nr[ax]));
        launch_pass(c, ps);
    }
}

static const int64_t CHUNK = 128;

// Steps per field chunk: CHUNK, or fewer where the chunk's per-step tables (s sub-steps x all axis
// points) would pass 1 GiB (long 1-D axes).
static int64_t chunk_steps(const qnd_ctx* c) {
    const size_t per_step = size_t(c->s) * size_t(c->axtot) * c->elem();
    const int64_t fit = int64_t((size_t(1) << 30) / std::max<size_t>(per_step, 1));
    return std::max<int64_t>(1, std::min<int64_t>(CHUNK, fit));
}

// The context's graph for key, or null; a hit counts as a use.
static GraphEntry* find_graph(qnd_ctx* c, const std::string& key) {
    auto it = c->graphs.find(key);
    if (it == c->graphs.end()) return nullptr;
    it->second.last_use = ++c->graph_clock;
    return &it->second;
}

// Keep an instantiated graph under key; past MAX_GRAPHS the least recently used one goes (after the
// device is idle, so that no launch of it is in flight).
static GraphEntry* keep_graph(qnd_ctx* c, const std::string& key, cudaGraphExec_t ex, std::vector<int64_t> launches) {
    if (c->graphs.size() >= MAX_GRAPHS) {
        auto lru = c->graphs.begin();
        for (auto it = c->graphs.begin(); it != c->graphs.end(); ++it)
            if (it->second.last_use < lru->second.last_use) lru = it;
        QND_CK(cudaDeviceSynchronize());
        cudaGraphExecDestroy(lru->second.exec);
        c->graphs.erase(lru);
    }
    GraphEntry& e = c->graphs[key];
    e.exec = ex;
    e.launches = std::move(launches);
    e.last_use = ++c->graph_clock;
    return &e;
}

// First sight of key: run directly and remember it; true if it had been seen before.
static bool seen_before(qnd_ctx* c, const std::string& key) {
    if (c->warm_keys.count(key)) return true;
    if (c->warm_keys.size() >= 64) c->warm_keys.clear();
    c->warm_keys.insert(key);
    return false;
}

// Run a chunk-wide chain (body) through a CUDA graph. The first run of a key goes directly (it
// builds the tables the chain reads); the second captures it; later runs replay the graph, so the
// host enqueues one graph launch per chunk instead of ~7 kernels per step and the device does not
// wait on a slow host. The graphs stay with the context (a few keys: a run's full and last chunks,
// repeated calls), so a later call of the same shape replays from its first chunk. Direct runs
// when profiling (per-launch events), when the caller is already capturing the stream, or with
// QND_NO_GRAPH set.
static void run_chunk_graph(qnd_ctx* c, const std::string& key, const std::function<void()>& body) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    QND_CK(cudaStreamIsCapturing(c->stream, &cs));
    if (c->profiling || cs != cudaStreamCaptureStatusNone || std::getenv("QND_NO_GRAPH")) {
        body();
        return;
    }
    if (GraphEntry* ge = find_graph(c, key)) {
        QND_CK(cudaGraphLaunch(ge->exec, c->stream));
        c->kernels_launched += ge->launches[0];
        return;
    }
    if (!seen_before(c, key)) {
        body();
        return;
    }
    const int64_t k0 = c->kernels_launched;
    QND_CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t g = nullptr;
    try {
        body();
    } catch (...) {
        cudaStreamEndCapture(c->stream, &g);
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        c->kernels_launched = k0;
        throw;
    }
    QND_CK(cudaStreamEndCapture(c->stream, &g));
    cudaGraphExec_t ex = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        QND_FAIL(QND_ECUDA, "cudaGraphInstantiate of a step chain: %s", cudaGetErrorString(e));
    }
    keep_graph(c, key, ex, {c->kernels_launched - k0});
    QND_CK(cudaGraphLaunch(ex, c->stream));
}

// What a length-gauge chunk chain captures (see run_chunk_graph).
static std::string chain_key(qnd_ctx* c, const void* psi, int64_t ch, int nobs, const char* const* names,
                             const double* rows, bool masked) {
    std::string k = fmt("L|%llu|%p|%lld|%p|%d|%p|%p|%p|%llu|%llu|%d|", (unsigned long long)c->serial, psi,
                        (long long)ch, (const void*)rows, int(masked), c->field_tab.p, c->partials.p, c->counter.p,
                        (unsigned long long)c->table_epoch, (unsigned long long)c->config_epoch, int(c->pdl));
    for (int q = 0; q < nobs; ++q) {
        k += names[q] ? names[q] : "";
        k += ',';
    }
    return k;
}

// Real-time driver loop (QuantumND_real.c:168-229) for either gauge.
static void run_realtime(qnd_ctx* c, void* psi, const double* field_host, const double* alpha_host, int64_t nsteps,
                         int nobs, const char* const* names, double* obs_host, bool velocity) {
    int nv = 0;
    auto items = parse_obs(c, nobs, names, &nv);
    const bool fused = all_rspace(items) && !velocity;  // velocity obs use A(t) -> evaluate per step
    const bool fused_v = all_rspace(items) && velocity;
    const bool masked = has_mask(c);
    const int64_t ch_max = std::min<int64_t>(chunk_steps(c), std::max<int64_t>(nsteps, 1));
    if (nv > 0) {
        c->obs_dev.ensure(size_t(ch_max + 1) * nv * sizeof(double));
        QND_CK(cudaMemsetAsync(c->obs_dev.p, 0, size_t(ch_max + 1) * nv * sizeof(double), c->stream));
    }
    std::vector<double> zero_alpha(MAX_DIM, 0.0);
    double* rows = c->obs_dev.as<double>();
    // length gauge whose observables are r-space reductions of one descriptor: chunk-wide chains
    const bool chain = !velocity && (nv == 0 || (fused && rspace_red(c, items, rows, 0).size() <= 1));
    for (int64_t c0 = 0; c0 < nsteps; c0 += ch_max) {
        const int64_t ch = std::min(ch_max, nsteps - c0);
        if (nv > 0 && c0 == 0) {
            const double* al = velocity ? alpha_host : zero_alpha.data();
            eval_obs(c, psi, items, al, rows);
        }
        upload_field_chunk(c, field_host + size_t(c0) * c->s * c->dim, ch, velocity);
        if (chain) {
            // the whole chunk is one sandwich chain; the observables of each step come out of the
            // pass that straddles the step boundary
            RedFn rf;
            if (nv > 0) rf = [&](int64_t k, int ax) { return rspace_red(c, items, rows + size_t(k + 1) * nv, ax); };
            run_chunk_graph(c, chain_key(c, psi, ch, nobs, names, rows, masked),
                            [&]() { length_steps(c, psi, 0, ch, rf, masked); });
        } else {
            for (int64_t k = 0; k < ch; ++k) {
                const int64_t gst = c0 + k;
                double* row = rows + size_t(k + 1) * nv;
                std::vector<RedDesc> fin;
                const int NK = velocity ? c->s : c->s + 1;
                if (nv > 0 && (fused || fused_v)) fin = rspace_red(c, items, row, chain_final_axis(c, NK));
                const RedDesc* f0 = fin.empty() ? nullptr : &fin[0];
                if (velocity) {
                    velocity_steps(c, psi, k, 1, f0, masked);
                } else {
                    RedFn rf;
                    if (f0) rf = [&](int64_t, int) { return std::vector<RedDesc>{*f0}; };
                    length_steps(c, psi, k, 1, rf, masked);
                }
                if (fin.size() > 1) {  // outputs beyond the first descriptor: a read of the final state
                    auto nat = rspace_red(c, items, row, c->dim - 1);
                    for (size_t q = 1; q < nat.size(); ++q) grid_reduce(c, psi, nat[q]);
                }
                if (nv > 0 && !(fused || fused_v) && gst + 1 < nsteps) {
                    const double* al = velocity ? alpha_host + size_t(gst + 1) * c->dim : zero_alpha.data();
                    eval_obs(c, psi, items, al, row);
                }
            }
        }
        if (nv > 0) {
            // rows[0] holds obs(psi(t_c0)); rows[k+1] obs after step c0+k
            const int64_t first = c0;  // host row index of rows[0]
            const int64_t cnt = std::min<int64_t>(ch, nsteps - first);
            QND_CK(cudaMemcpyAsync(obs_host + size_t(first) * nv, rows, size_t(cnt) * nv * sizeof(double),
                                   cudaMemcpyDeviceToHost, c->stream));
            QND_CK(cudaStreamSynchronize(c->stream));
            // carry the last row (obs after the chunk) to the front for the next chunk
            QND_CK(cudaMemcpyAsync(rows, rows + size_t(ch) * nv, nv * sizeof(double), cudaMemcpyDeviceToDevice,
                                   c->stream));
        }
    }
    QND_CK(cudaGetLastError());
    check_device_error(c);  // a wait that ran out in this call is reported by this call
}

// ---------------------------------------------------------------- adjoint --
//
// Gradient of J = dNr sum_x w(x) |psi_T(x)|^2 with respect to every field sample of a real-time
// run (an extension: the reference has no adjoint). With the adjoint state lambda = dJ/dconj(psi)
// (lambda_T = dNr w psi_T), every operator O of the run maps lambda <- O^dagger lambda going
// backward, and an operator that depends on a sample F contributes 2 Re <lambda', dO/dF psi> with
// psi' = O psi and lambda' the adjoint state at the same point.
//
// Length gauge (integrators.c:170-194 in r-space): a step is
//   psi <- M K(a_{2s-1}) D_{s-1} K(c_{s-1}) ... D_0 K(c_0) psi,  c_0 = a_0, c_i = a_{2i-1} + a_{2i},
// with the kinetic sandwiches K(c) (unitary), the step mask M (real, diagonal) and the potential
// factors D_i = exp(-h_i Vcap) exp(-i h_i (V + x.E[k][i])), h_i = a_{2i} + a_{2i+1}, so
//   dJ/dE[k][i][j] = 2 h_i sum_x x_j Im(conj(lambda') psi')   (just after D_i).
// Adjoints: K(-c) for K(c), M for M, RT_LENGTH_ADJ times the laser phases of -E for D_i.
//
// Velocity gauge (integrators.c:201-232): a step is
//   psi <- M V(a_{2s-1}) P_{s-1} V(a_{2s-3}) V(a_{2s-2}) ... V(a_1) V(a_2) P_0 V(a_0) psi,
// with the r-space factors V(a) = exp(-a Vcap) exp(-i a V) and the kinetic sandwiches
// P_i = F^-1 exp(-i h_i sum_j (p_j^2/2 + (p_j + A_j/2) A_j)) F of the samples A[k][i], so
// (Parseval, unitary transforms of both states)
//   dJ/dA[k][i][j] = 2 h_i sum_k (p_j + A[k][i][j]) Im(conj(lambda~') psi~')   (just after P_i).
// Adjoints: V(a) -> RT_VEL_ADJ, P_i -> the sandwich with the conjugate phase tables.
//
// The forward states are kept every `every` steps; a segment's step-start states are recomputed
// from its checkpoint, and a step's sub-step states from its start.

// psi <- M psi for the step masks set on the axes.
static void apply_step_masks(qnd_ctx* c, void* psi) {
    if (c->fp64) {
        const double* m[MAX_DIM];
        for (int j = 0; j < MAX_DIM; ++j) m[j] = c->mask_dev[j].as<double>();
        long long nm[MAX_DIM];
        for (int j = 0; j < MAX_DIM; ++j) nm[j] = c->nr[j] - 1;
        launch_apply_masks<double>(c->n, static_cast<double2*>(psi), c->dim, c->shift, nm, m, c->stream);
    } else {
        const float* m[MAX_DIM];
        for (int j = 0; j < MAX_DIM; ++j) m[j] = c->mask_dev[j].as<float>();
        long long nm[MAX_DIM];
        for (int j = 0; j < MAX_DIM; ++j) nm[j] = c->nr[j] - 1;
        launch_apply_masks<float>(c->n, static_cast<float2*>(psi), c->dim, c->shift, nm, m, c->stream);
    }
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

// psi <- t psi for a full-grid complex table in natural order (any dimension).
static void apply_table(qnd_ctx* c, void* psi, const void* table) {
    if (c->fp64)
        launch_point_factors<double>(c->n, static_cast<double2*>(psi), nullptr, static_cast<const double2*>(table),
                                     nullptr, nullptr, nullptr, c->stream);
    else
        launch_point_factors<float>(c->n, static_cast<float2*>(psi), nullptr, static_cast<const float2*>(table),
                                    nullptr, nullptr, nullptr, c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

static void copy_state(qnd_ctx* c, void* dst, const void* src) {
    QND_CK(cudaMemcpyAsync(dst, src, size_t(c->n) * c->elem(), cudaMemcpyDeviceToDevice, c->stream));
}

// Steps k0 .. k0+n-1 of the run's field samples (host [nsteps][s][dim]) on an r-space psi.
static void steps_span(qnd_ctx* c, void* psi, const double* F, int64_t k0, int64_t n, bool masked, bool velocity) {
    const int64_t chunk = chunk_steps(c);
    for (int64_t q = 0; q < n; q += chunk) {
        const int64_t ch = std::min(chunk, n - q);
        upload_field_chunk(c, F + size_t(k0 + q) * c->s * c->dim, ch, velocity);
        if (!velocity) length_steps(c, psi, 0, ch, RedFn(), masked);
        else if (!masked) velocity_steps(c, psi, 0, ch, nullptr, false);
        else  // a velocity chain masks after its last step only: one chain per step
            for (int64_t k = 0; k < ch; ++k) velocity_steps(c, psi, k, 1, nullptr, true);
    }
}

// One member of qnd_run_length_batch: its context, observables, mask and staged rows.
struct SweepMember {
    qnd_ctx* c = nullptr;
    std::vector<ObsItem> items;
    int nv = 0;
    bool masked = false;
    double* stage = nullptr;
};

static void adjoint_run(qnd_ctx* c, const void* psi0, const double* F, int64_t nsteps, const double* w_host,
                        int64_t every, double* J_out, double* grad_host, void* psiT, bool velocity) {
    const int s = c->s, d = c->dim;
    const size_t sb = size_t(c->n) * c->elem();
    const int64_t K = std::max<int64_t>(1, std::min(every, nsteps));
    const int64_t nck = (nsteps + K - 1) / K;
    const bool masked = has_mask(c);
    DevBuf ck, seg, sub, work, lam, wgrid, wscaled, out, tl, tp;
    ck.ensure(size_t(nck) * sb);
    seg.ensure(size_t(K) * sb);
    sub.ensure(size_t(s) * sb);
    work.ensure(sb);
    lam.ensure(sb);
    if (velocity) {
        tl.ensure(sb);
        tp.ensure(sb);
    }
    out.ensure((size_t(nsteps) * s * d + 1) * sizeof(double));
    auto at = [&](DevBuf& b, int64_t k) { return static_cast<void*>(static_cast<char*>(b.p) + size_t(k) * sb); };
    // the weight: FP64 for J, and dNr w in the state's precision for lambda_T
    std::vector<double> w(w_host, w_host + c->n), wl(size_t(c->n));
    for (size_t i = 0; i < wl.size(); ++i) wl[i] = c->dNr * w[i];
    upload_f64(c, wgrid, w);
    upload_real(c, wscaled, wl);

    // forward, keeping the checkpoints
    copy_state(c, work.p, psi0);
    for (int64_t q = 0; q < nck; ++q) {
        copy_state(c, at(ck, q), work.p);
        steps_span(c, work.p, F, q * K, std::min(K, nsteps - q * K), masked, velocity);
    }
    if (psiT) copy_state(c, psiT, work.p);
    double* grad_dev = out.as<double>();
    double* J_dev = grad_dev + size_t(nsteps) * s * d;
    RedDesc rj{};
    rj.n = 1;
    rj.kind[0] = RK_ABS2;
    rj.wkind[0] = WK_GRID;
    rj.wtab[0] = wgrid.as<double>();
    rj.scale[0] = c->dNr;
    rj.out = J_dev;
    grid_reduce(c, work.p, rj);
    copy_state(c, lam.p, work.p);
    if (c->fp64)
        launch_point_factors<double>(c->n, lam.as<double2>(), wscaled.as<double>(), nullptr, nullptr, nullptr, nullptr,
                                     c->stream);
    else
        launch_point_factors<float>(c->n, lam.as<float2>(), wscaled.as<float>(), nullptr, nullptr, nullptr, nullptr,
                                    c->stream);
    c->kernels_launched++;

    auto kin = [&](double coef) {
        ChainK k;
        k.kind = SP_LENGTH;
        k.coef = coef;
        return std::vector<ChainK>{k};
    };
    auto kvel = [&](int64_t lst, int ia) {
        ChainK k;
        k.kind = KV_FIELD;
        k.lst = lst;
        k.ia = ia;
        return std::vector<ChainK>{k};
    };
    auto cst = [&](int i) { return i == 0 ? c->as[0] : c->as[2 * i - 1] + c->as[2 * i]; };
    auto hst = [&](int i) { return c->as[2 * i] + c->as[2 * i + 1]; };
    // velocity gauge: the r-space factor before sandwich i (V(a_0), then V(a_{2i-1}) V(a_{2i}))
    auto vpre = [&](int i, int kind) {
        Factor f;
        f.kind = kind;
        f.a = i == 0 ? c->as[0] : c->as[2 * i - 1];
        f.b = i == 0 ? NO_COEF : c->as[2 * i];
        return f;
    };
    std::vector<double> fe(size_t(2) * s * d);
    // backward, segment by segment
    for (int64_t q = nck - 1; q >= 0; --q) {
        const int64_t k0 = q * K, kn = std::min(K, nsteps - k0);
        copy_state(c, work.p, at(ck, q));
        for (int64_t k = 0; k < kn; ++k) {
            copy_state(c, at(seg, k), work.p);
            if (k + 1 < kn) steps_span(c, work.p, F, k0 + k, 1, masked, velocity);
        }
        for (int64_t k = kn - 1; k >= 0; --k) {
            const int64_t kk = k0 + k;
            const double* Fk = F + size_t(kk) * s * d;
            // field tables of this step: slot 0 forward; slot 1 the adjoint's (length: the laser
            // phases of -E; velocity: the conjugate k-space phases)
            for (int q2 = 0; q2 < s * d; ++q2) {
                fe[q2] = Fk[q2];
                fe[s * d + q2] = velocity ? Fk[q2] : -Fk[q2];
            }
            upload_field_chunk(c, fe.data(), 2, velocity, velocity ? 1 : (1 << 30));
            // the states just after each parameter-dependent operator
            copy_state(c, work.p, at(seg, k));
            for (int i = 0; i < s; ++i) {
                if (velocity) {
                    run_chain(c, work.p, kvel(0, i), {}, vpre(i, RT_VEL), 0, nullptr, ChainMid{});
                } else {
                    ChainMid post;
                    post.f.kind = RT_LENGTH;
                    post.f.a = hst(i);
                    post.f.laser_ia = i;
                    post.lst = 0;
                    run_chain(c, work.p, kin(cst(i)), {}, Factor{}, 0, nullptr, post);
                }
                copy_state(c, at(sub, i), work.p);
            }
            // lambda back through the step's last operators: M, then K(a_{2s-1}) or V(a_{2s-1})
            if (masked) apply_step_masks(c, lam.p);
            if (velocity) apply_table(c, lam.p, rtab(c, RT_VEL_ADJ, c->as[2 * s - 1], NO_COEF));
            else run_chain(c, lam.p, kin(-c->as[2 * s - 1]), {}, Factor{}, 0, nullptr, ChainMid{});
            for (int i = s - 1; i >= 0; --i) {
                RedDesc rg{};
                rg.n = d;
                const void* pr = at(sub, i);
                const void* pl = lam.p;
                if (velocity) {
                    // unitary transforms of both states, weights p_j + A_j
                    copy_state(c, tl.p, lam.p);
                    copy_state(c, tp.p, at(sub, i));
                    unitary_fft(c, tl.p, true);
                    unitary_fft(c, tp.p, true);
                    pr = tp.p;
                    pl = tl.p;
                    for (int j = 0; j < d; ++j) {
                        c->wtab_dev[j].ensure(size_t(c->nr[j]) * 8);
                        launch_axis_table<double>(0, c->p_dev.as<double>() + c->axoff[j], int(c->nr[j]),
                                                  Fk[size_t(i) * d + j], c->wtab_dev[j].p, c->stream);
                        c->kernels_launched++;
                    }
                }
                for (int j = 0; j < d; ++j) {
                    rg.kind[j] = RK_BILIN_IM;
                    rg.wkind[j] = WK_AXIS;
                    rg.waxis[j] = j;
                    rg.wtab[j] = velocity ? c->wtab_dev[j].as<double>() : c->r_dev.as<double>() + c->axoff[j];
                    rg.scale[j] = 2.0 * hst(i);
                }
                rg.out = grad_dev + (size_t(kk) * s + i) * d;
                grid_reduce(c, pr, rg, pl);
                if (velocity) {
                    ChainMid post;
                    post.f = vpre(i, RT_VEL_ADJ);
                    run_chain(c, lam.p, kvel(1, i), {}, Factor{}, 0, nullptr, post);
                } else {
                    Factor adj;
                    adj.kind = RT_LENGTH_ADJ;
                    adj.a = hst(i);
                    adj.laser_ia = i;
                    run_chain(c, lam.p, kin(-cst(i)), {}, adj, 1, nullptr, ChainMid{});
                }
            }
        }
    }
    QND_CK(cudaMemcpyAsync(grad_host, grad_dev, size_t(nsteps) * s * d * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream));
    double J = 0.0;
    QND_CK(cudaMemcpyAsync(&J, J_dev, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    QND_CK(cudaStreamSynchronize(c->stream));
    check_device_error(c);
    if (J_out) *J_out = J;
}

// ---------------------------------------------------------------- Gram-Schmidt --

// v = psi_j - sum_k <psi_k|psi_j> psi_k; norm2 = ||v||^2 dNr into scal[0]; scale 1/sqrt(norm2) into
// scal[1]; the flag is raised when norm2 < 1e-12 (QuantumND_imag.c:280-304). The normalisation itself
// is left to the caller (scale kernel or the next step's prologue).
static void gs_project(qnd_ctx* c, void* const* states, int j) {
    if (j >= GS_MAXK) QND_FAIL(QND_EUNSUPPORTED, "Gram-Schmidt against %d states (max %d)", j, GS_MAXK - 1);
    c->scal.ensure(sizeof(double) * (2 + 2 * GS_MAXK));
    if (!c->gs_flag.p) {
        c->gs_flag.ensure(sizeof(int));
        QND_CK(cudaMemsetAsync(c->gs_flag.p, 0, sizeof(int), c->stream));
    }
    double* scal = c->scal.as<double>();
    const int nb = reduce_blocks(c);
    ensure_red_scratch(c, nb);
    auto run = [&](auto tag) {
        using R = decltype(tag);
        GSArgs<R> g;
        std::memset(&g, 0, sizeof g);
        g.psi = static_cast<cplx_t<R>*>(states[j]);
        for (int k = 0; k < j; ++k) g.states[k] = static_cast<const cplx_t<R>*>(states[k]);
        g.n = c->n;
        g.red.partials = c->partials.as<double>();
        g.red.counter = c->counter.as<unsigned int>();
        for (int k0 = 0; k0 < j; k0 += MAX_RED / 2) {
            g.k0 = k0;
            g.nk = std::min(MAX_RED / 2, j - k0);
            g.red.n = 2 * g.nk;
            for (int q = 0; q < g.red.n; ++q) {
                g.red.kind[q] = RK_ABS2;
                g.red.wkind[q] = WK_ONE;
                g.red.scale[q] = c->dNr;
            }
            g.red.out = scal + 2 + 2 * k0;
            launch_gs_dot<R>(g, c->stream, nb);
            c->kernels_launched++;
        }
        g.j = j;
        g.coef = scal + 2;
        g.red.n = 1;
        g.red.scale[0] = c->dNr;
        g.red.out = scal;
        launch_gs_axpy<R>(g, c->stream, nb);
        c->kernels_launched++;
    };
    if (c->fp64) run(double{});
    else run(float{});
    QND_CK(cudaGetLastError());
    launch_gs_finalize(scal, 1.e-12, scal + 1, c->gs_flag.as<int>(), c->stream);
    c->kernels_launched++;
}

static void check_gs_flag(qnd_ctx* c, int j) {
    int flag = 0;
    QND_CK(cudaMemcpyAsync(&flag, c->gs_flag.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    QND_CK(cudaStreamSynchronize(c->stream));
    if (flag) {
        QND_CK(cudaMemsetAsync(c->gs_flag.p, 0, sizeof(int), c->stream));
        QND_FAIL(QND_ENORM, "Wavefunction norm decayed to zero during Gram-Schmidt for state %d (norm < 1e-12)", j);
    }
}

static void scale_state(qnd_ctx* c, void* psi, const double* scale_dev) {
    if (c->fp64) launch_scale<double>(static_cast<double2*>(psi), c->n, scale_dev, c->stream);
    else launch_scale<float>(static_cast<float2*>(psi), c->n, scale_dev, c->stream);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

// ---------------------------------------------------------------- context --

static void set_device(qnd_ctx* c) { QND_CK(cudaSetDevice(c->device)); }

// The four-step twiddles of an axis of N = n1 n2 points: W_N^{k1 m} at slot k1 n2 + m, and their
// conjugates (FP32: stored as w - 1).
static void build_four_step_twiddles(qnd_ctx* c, int64_t N, int64_t n1, int64_t n2, DevBuf& twf, DevBuf& twc) {
    std::vector<double> w(2 * size_t(N)), wc(2 * size_t(N));
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int64_t k1 = 0; k1 < n1; ++k1)
        for (int64_t m = 0; m < n2; ++m) {
            const int64_t i = k1 * n2 + m;
            const long double ang = two_pi * (long double)((k1 * m) & (N - 1)) / (long double)N;
            const double sn = (double)sinl(ang);
            double re;
            if (c->fp64) {
                re = (double)cosl(ang);
            } else {
                const long double sh = sinl(ang / 2);
                re = (double)(-2 * sh * sh);
            }
            w[2 * i] = re;
            w[2 * i + 1] = -sn;
            wc[2 * i] = re;
            wc[2 * i + 1] = sn;
        }
    upload_cplx(c, twf, w);
    upload_cplx(c, twc, wc);
}

// An axis longer than 4096 points on a grid of several dimensions (emulate_long_pass): the virtual
// lengths (n2 = min(4096, N / 16), n1 = N / n2), their pass twiddles, the four-step twiddles.
static void build_long_axis_nd(qnd_ctx* c, int ax) {
    auto& la = c->lax[ax];
    const int64_t N = c->nr[ax];
    la.on = true;
    la.lg1 = std::max(4, c->lognr[ax] - 12);
    la.lg2 = c->lognr[ax] - la.lg1;
    la.n1 = int64_t(1) << la.lg1;
    la.n2 = int64_t(1) << la.lg2;
    build_twiddles(c, int(la.n1), la.tw[0]);
    build_twiddles(c, int(la.n2), la.tw[1]);
    build_four_step_twiddles(c, N, la.n1, la.n2, la.twf, la.twc);
}

// The tables of a long 1-D axis (see long_fft): pass twiddles for both virtual lengths, the
// four-step twiddles W_N^{k1 n2} and their conjugates (FP32: stored as w - 1), slot momenta.
static void build_long_axis(qnd_ctx* c) {
    const int64_t N = c->nr[0];
    c->long1d = true;
    c->lg1 = std::max(4, c->lognr[0] - 12);  // n1 >= 16: the strided passes keep 16 values per thread
    c->lg2 = c->lognr[0] - c->lg1;
    c->n1 = int64_t(1) << c->lg1;
    c->n2 = int64_t(1) << c->lg2;
    build_twiddles(c, int(c->n1), c->tw_long[0]);
    build_twiddles(c, int(c->n2), c->tw_long[1]);
    build_four_step_twiddles(c, N, c->n1, c->n2, c->twf_long, c->twc_long);
    c->p_slot.resize(size_t(N));
    for (int64_t i = 0; i < N; ++i) c->p_slot[i] = c->p[0][(i >> c->lg2) + ((i & (c->n2 - 1)) << c->lg1)];
    upload_f64(c, c->p_slot_dev, c->p_slot);
}

static void build_context(qnd_ctx* c, int dim, const int64_t* nr, const double* dr, const char* integrator,
                          double dt, int precision) {
    if (dim < 1 || dim > MAX_DIM) QND_FAIL(QND_EINVAL, "dimension %d not in 1..%d", dim, MAX_DIM);
    if (precision != QND_FP64 && precision != QND_MIXED) QND_FAIL(QND_EINVAL, "unknown precision %d", precision);
    c->fp64 = precision == QND_FP64;
    c->dim = dim;
    c->n = 1;
    // one pass handles an axis of up to 4096 points; longer axes (up to 2^24 points) take four steps
    const int64_t nmax = LONG_AXIS_MAX;
    for (int j = 0; j < dim; ++j) {
        if (nr[j] < 2 || nr[j] > nmax || (nr[j] & (nr[j] - 1)))
            QND_FAIL(nr[j] > nmax ? QND_EUNSUPPORTED : QND_EINVAL,
                     "NR[%d]=%lld: must be a power of 2 between 2 and %lld", j, (long long)nr[j], (long long)nmax);
        if (!(dr[j] > 0)) QND_FAIL(QND_EINVAL, "DR[%d] must be positive", j);
        c->nr[j] = nr[j];
        c->dr[j] = dr[j];
        c->n *= nr[j];
        int l = 0;
        while ((int64_t(1) << l) < nr[j]) ++l;
        c->lognr[j] = l;
    }
    for (int j = 0; j < dim; ++j) {
        int sh = 0;
        for (int k = j + 1; k < dim; ++k) sh += c->lognr[k];
        c->shift[j] = sh;
    }
    // integrator coefficients (integrators.c:22-64)
    static const double verlet[] = {.5};
    static const double bm4[] = {.0792036964311957, .1303114101821663, .2228614958676077,
                                 -.3667132690474257, .3246481886897062, .1096884778767498};
    static const double bm6[] = {.050262764400392, .098553683500650, .314960616927694, -.447346482695478,
                                 .492426372489876, -.425118767797691, .237063913978122, .195602488600053,
                                 .346358189850727, -.362762779254345};
    static const double rkn4[] = {.082984406417405, .162314550766866, .233995250731502,
                                  .370877414979578, -.409933719901926, .059762097006575};
    const double* base = nullptr;
    if (!integrator) QND_FAIL(QND_EINVAL, "integrator name is NULL");
    if (!strcmp(integrator, "Verlet")) { base = verlet; c->s = 1; }
    else if (!strcmp(integrator, "BM4")) { base = bm4; c->s = 6; }
    else if (!strcmp(integrator, "BM6")) { base = bm6; c->s = 10; }
    else if (!strcmp(integrator, "RKN4")) { base = rkn4; c->s = 6; }
    else QND_FAIL(QND_EINVAL, "Unknown integrator: %s", integrator);
    double as[20];
    for (int j = 0; j < c->s; ++j) as[j] = base[j];
    for (int j = 0; j < c->s; ++j) as[c->s + j] = as[c->s - 1 - j];
    for (int j = 0; j < 2 * c->s; ++j) c->as[j] = as[j] * dt;
    c->integrator = integrator;
    c->dt = dt;
    // grid (meshgrid.c:22-28, 75-89)
    c->dNr = 1.;
    c->dNp = 1.;
    int off = 0;
    for (int j = 0; j < dim; ++j) {
        c->dNr *= dr[j];
        c->dNp *= 2. * M_PI / (double)(dr[j] * nr[j]);
        const int64_t N = nr[j];
        const double L = dr[j] * N, dp = 2. * M_PI / L;
        c->r[j].resize(N);
        c->p[j].resize(N);
        for (int64_t i = 0; i < N; ++i) {
            c->r[j][i] = -.5 * L + i * dr[j];
            c->p[j][i] = i < N / 2 ? i * dp : (i - N) * dp;
        }
        c->axoff[j] = off;
        off += int(N);
    }
    c->axtot = off;
    QND_CK(cudaGetDevice(&c->device));
    QND_CK(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device));
    if (const char* e = getenv("QND_PDL")) c->pdl = atoi(e) != 0;
    QND_CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
    std::vector<double> rall, pall;
    for (int j = 0; j < dim; ++j) {
        rall.insert(rall.end(), c->r[j].begin(), c->r[j].end());
        pall.insert(pall.end(), c->p[j].begin(), c->p[j].end());
    }
    c->err_flag.ensure(sizeof(int));
    QND_CK(cudaMemsetAsync(c->err_flag.p, 0, sizeof(int), c->stream));
    upload_f64(c, c->r_dev, rall);
    upload_f64(c, c->p_dev, pall);
    if (dim == 1 && nr[0] > 4096) {
        build_long_axis(c);
        return;
    }
    bool any_long = false;
    for (int j = 0; j < dim; ++j) {
        if (c->nr[j] > 4096) {
            build_long_axis_nd(c, j);
            any_long = true;
        } else {
            build_twiddles(c, int(c->nr[j]), c->tw[j]);
        }
    }
    if (any_long) {
        // the scratch states of the emulated passes, allocated up front (not inside a graph capture)
        c->lax_perm.ensure(size_t(c->n) * c->elem());
        c->lax_tmp.ensure(size_t(c->n) * c->elem());
    }
}

// Named potentials as functions of |r| (meshgrid.c:137-153) and their radial derivative dV/dr.
static bool named_potential(const char* name, double r, double* v) {
    const double r2 = r * r;
    if (!strcmp(name, "H_1D")) *v = -1. / (double)sqrt(r2 + 2.);
    else if (!strcmp(name, "H_3D")) *v = -1. / (double)sqrt(r2 + 1e-4);
    else if (!strcmp(name, "H_2D")) *v = -1. / (double)sqrt(r2 + .7396);
    else if (!strcmp(name, "Ne_2D")) *v = -(1. + 9. * exp(-r2)) / (double)sqrt(r2 + 2.88172);
    else if (!strcmp(name, "Ar_2D")) *v = -(1. + 17. * exp(-r2)) / (double)sqrt(r2 + .91205);
    else if (!strcmp(name, "Kr_2D")) *v = -(1. + 35. * exp(-r2)) / (double)sqrt(r2 + .7875);
    else if (!strcmp(name, "Xe_2D")) *v = -(1. + 53. * exp(-r2)) / (double)sqrt(r2 + .52592);
    else if (!strcmp(name, "Ne_short_2D")) *v = -2.7459 * exp(-.5 * r2 / 1.96);
    else return false;
    return true;
}

}  // namespace qnd

// ================================================================ C API ==

#define QND_API_BEGIN try {
#define QND_API_END                                                   \
    return QND_OK;                                                    \
    }                                                                 \
    catch (const ::qnd::Error& e) {                                   \
        ::qnd::g_err = e.msg;                                         \
        return e.code;                                                \
    }                                                                 \
    catch (const std::exception& e) {                                 \
        ::qnd::g_err = e.what();                                      \
        return QND_EINVAL;                                            \
    }

#define QND_NEED(ptr)                                                  \
    if (!(ptr)) QND_FAIL(QND_EINVAL, "%s: %s is NULL", __func__, #ptr)

extern "C" {

const char* qnd_version(void) { return "qnd_b200 0.1 (sm_100a)"; }
const char* qnd_last_error(void) { return qnd::g_err.c_str(); }

int qnd_ctx_create(int dim, const int64_t* nr, const double* dr, const char* integrator, double dt, int precision,
                   qnd_ctx** out) {
    QND_API_BEGIN
    QND_NEED(out);
    QND_NEED(nr);
    QND_NEED(dr);
    *out = nullptr;
    auto c = std::make_unique<qnd_ctx>();
    c->serial = ++g_ctx_serial;
    build_context(c.get(), dim, nr, dr, integrator, dt, precision);
    *out = c.release();
    QND_API_END
}

int qnd_ctx_destroy(qnd_ctx* ctx) {
    QND_API_BEGIN
    if (!ctx) return QND_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& pr : ctx->prof_pairs) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    for (auto e : ctx->event_pool) cudaEventDestroy(e);
    for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second.exec);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    QND_API_END
}

int qnd_ctx_set_stream(qnd_ctx* ctx, void* stream) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->config_epoch++;
    set_device(ctx);
    QND_CK(cudaStreamSynchronize(ctx->stream));
    if (stream) {
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        ctx->stream = static_cast<cudaStream_t>(stream);
        ctx->own_stream = false;
    } else if (!ctx->own_stream) {
        QND_CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->own_stream = true;
    }
    QND_API_END
}

int qnd_ctx_info(qnd_ctx* ctx, int64_t* n_total, int* s_integrator, double* as_scaled, double* dNr, double* dNp) {
    QND_API_BEGIN
    QND_NEED(ctx);
    if (n_total) *n_total = ctx->n;
    if (s_integrator) *s_integrator = ctx->s;
    if (as_scaled)
        for (int j = 0; j < 2 * ctx->s; ++j) as_scaled[j] = ctx->as[j];
    if (dNr) *dNr = ctx->dNr;
    if (dNp) *dNp = ctx->dNp;
    QND_API_END
}

int qnd_state_bytes(qnd_ctx* ctx, int64_t* bytes) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(bytes);
    *bytes = int64_t(ctx->n) * int64_t(ctx->elem());
    QND_API_END
}

int qnd_set_potential_named(qnd_ctx* ctx, const char* name) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->config_epoch++;
    QND_NEED(name);
    double probe;
    if (!named_potential(name, 0.0, &probe)) QND_FAIL(QND_EINVAL, "Unknown potential: %s", name);
    std::vector<double> v(size_t(ctx->n));
    int64_t idx[MAX_DIM];
    for (int64_t i = 0; i < ctx->n; ++i) {
        int64_t rem = i;
        for (int j = ctx->dim - 1; j >= 0; --j) {
            idx[j] = rem % ctx->nr[j];
            rem /= ctx->nr[j];
        }
        double r = 0.;
        for (int j = 0; j < ctx->dim; ++j) {
            const double x = ctx->r[j][idx[j]];
            r += x * x;
        }
        r = sqrt(r);
        named_potential(name, r, &v[size_t(i)]);
    }
    ctx->vpot.swap(v);
    ctx->vpot_dev.reset();
    invalidate_rtabs(ctx);
    QND_API_END
}

int qnd_set_potential(qnd_ctx* ctx, const double* vpot_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->config_epoch++;
    QND_NEED(vpot_host);
    ctx->vpot.assign(vpot_host, vpot_host + ctx->n);
    ctx->vpot_dev.reset();
    invalidate_rtabs(ctx);
    QND_API_END
}

int qnd_set_cap(qnd_ctx* ctx, double strength, double length) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->config_epoch++;
    std::vector<double> v(size_t(ctx->n), 0.0);
    int64_t idx[MAX_DIM];
    for (int64_t i = 0; i < ctx->n; ++i) {
        int64_t rem = i;
        for (int j = ctx->dim - 1; j >= 0; --j) {
            idx[j] = rem % ctx->nr[j];
            rem /= ctx->nr[j];
        }
        double acc = 0.;
        for (int j = 0; j < ctx->dim; ++j) {
            const double x = ctx->r[j][idx[j]];
            const double L = .5 * ctx->nr[j] * ctx->dr[j] - length;
            if (fabs(x) >= L) acc += strength * (fabs(x) - L) * (fabs(x) - L);
        }
        v[size_t(i)] = acc;
    }
    ctx->vcap.swap(v);
    invalidate_rtabs(ctx);
    QND_API_END
}

int qnd_set_vcap(qnd_ctx* ctx, const double* vcap_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->config_epoch++;
    if (vcap_host) ctx->vcap.assign(vcap_host, vcap_host + ctx->n);
    else ctx->vcap.clear();
    invalidate_rtabs(ctx);
    QND_API_END
}

int qnd_set_gradv(qnd_ctx* ctx, int axis, const double* gradv_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->config_epoch++;
    if (axis < 0 || axis >= ctx->dim) QND_FAIL(QND_EINVAL, "axis %d out of range", axis);
    set_device(ctx);
    if (!gradv_host) {
        ctx->gradv[axis].clear();
        ctx->gradv_dev[axis].reset();
        for (int k = 0; k < MAX_DIM; ++k) ctx->gradv_lm[axis][k].reset();
    } else {
        ctx->gradv[axis].assign(gradv_host, gradv_host + ctx->n);
        upload_f64(ctx, ctx->gradv_dev[axis], ctx->gradv[axis]);
        for (int k = 0; k < MAX_DIM; ++k) ctx->gradv_lm[axis][k].reset();
    }
    QND_API_END
}

int qnd_set_mask_axis(qnd_ctx* ctx, int axis, const double* mask_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->config_epoch++;
    if (axis < 0 || axis >= ctx->dim) QND_FAIL(QND_EINVAL, "axis %d out of range", axis);
    set_device(ctx);
    if (!mask_host) {
        ctx->mask[axis].clear();
        ctx->mask_dev[axis].reset();
    } else {
        ctx->mask[axis].assign(mask_host, mask_host + ctx->nr[axis]);
        upload_real(ctx, ctx->mask_dev[axis], ctx->mask[axis]);
    }
    QND_API_END
}

int qnd_state_alloc(qnd_ctx* ctx, int64_t nstates, void** psi_dev) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    if (nstates < 1) QND_FAIL(QND_EINVAL, "nstates must be >= 1");
    set_device(ctx);
    void* p = nullptr;
    const size_t bytes = size_t(nstates) * size_t(ctx->n) * ctx->elem();
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        QND_FAIL(QND_ENOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    QND_CK(cudaMemsetAsync(p, 0, bytes, ctx->stream));
    *psi_dev = p;
    QND_API_END
}

int qnd_state_free(qnd_ctx* ctx, void* psi_dev) {
    QND_API_BEGIN
    QND_NEED(ctx);
    set_device(ctx);
    QND_CK(cudaStreamSynchronize(ctx->stream));
    if (psi_dev) QND_CK(cudaFree(psi_dev));
    QND_API_END
}

int qnd_state_upload(qnd_ctx* ctx, void* psi_dev, const double* host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    QND_NEED(host);
    set_device(ctx);
    if (ctx->fp64) {
        QND_CK(cudaMemcpyAsync(psi_dev, host, size_t(ctx->n) * 16, cudaMemcpyHostToDevice, ctx->stream));
    } else {
        ctx->host_tmp.resize(size_t(ctx->n) * 8);
        float* f = reinterpret_cast<float*>(ctx->host_tmp.data());
        QND_CK(cudaStreamSynchronize(ctx->stream));
        for (int64_t i = 0; i < 2 * ctx->n; ++i) f[i] = float(host[i]);
        QND_CK(cudaMemcpyAsync(psi_dev, f, size_t(ctx->n) * 8, cudaMemcpyHostToDevice, ctx->stream));
    }
    QND_CK(cudaStreamSynchronize(ctx->stream));
    QND_API_END
}

int qnd_state_download(qnd_ctx* ctx, double* host, const void* psi_dev) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    QND_NEED(host);
    set_device(ctx);
    if (ctx->fp64) {
        QND_CK(cudaMemcpyAsync(host, psi_dev, size_t(ctx->n) * 16, cudaMemcpyDeviceToHost, ctx->stream));
        QND_CK(cudaStreamSynchronize(ctx->stream));
    } else {
        ctx->host_tmp.resize(size_t(ctx->n) * 8);
        float* f = reinterpret_cast<float*>(ctx->host_tmp.data());
        QND_CK(cudaMemcpyAsync(f, psi_dev, size_t(ctx->n) * 8, cudaMemcpyDeviceToHost, ctx->stream));
        QND_CK(cudaStreamSynchronize(ctx->stream));
        for (int64_t i = 0; i < 2 * ctx->n; ++i) host[i] = double(f[i]);
    }
    check_device_error(ctx);
    QND_API_END
}

int qnd_synchronize(qnd_ctx* ctx) {
    QND_API_BEGIN
    QND_NEED(ctx);
    set_device(ctx);
    QND_CK(cudaStreamSynchronize(ctx->stream));
    QND_CK(cudaGetLastError());
    check_device_error(ctx);
    QND_API_END
}

int qnd_step_imag(qnd_ctx* ctx, void* psi_dev, int64_t nsteps) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    set_device(ctx);
    imag_steps(ctx, psi_dev, nsteps, nullptr);
    QND_CK(cudaGetLastError());
    check_finite(ctx, psi_dev, "qnd_step_imag");
    QND_API_END
}

int qnd_to_p(qnd_ctx* ctx, void* psi_dev) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    set_device(ctx);
    unitary_fft(ctx, psi_dev, true);
    QND_API_END
}

int qnd_to_r(qnd_ctx* ctx, void* psi_dev) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    set_device(ctx);
    unitary_fft(ctx, psi_dev, false);
    QND_API_END
}

int qnd_step_length(qnd_ctx* ctx, void* psi_p_dev, const double* E_host, int64_t nsteps) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_p_dev);
    if (nsteps <= 0) return QND_OK;
    QND_NEED(E_host);
    set_device(ctx);
    unitary_fft(ctx, psi_p_dev, false);
    const int64_t chunk = chunk_steps(ctx);
    for (int64_t c0 = 0; c0 < nsteps; c0 += chunk) {
        const int64_t ch = std::min(chunk, nsteps - c0);
        upload_field_chunk(ctx, E_host + size_t(c0) * ctx->s * ctx->dim, ch, false);
        length_steps(ctx, psi_p_dev, 0, ch, RedFn(), false);
    }
    unitary_fft(ctx, psi_p_dev, true);
    QND_CK(cudaGetLastError());
    check_finite(ctx, psi_p_dev, "qnd_step_length");
    QND_API_END
}

int qnd_step_velocity(qnd_ctx* ctx, void* psi_dev, const double* A_host, int64_t nsteps) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    if (nsteps <= 0) return QND_OK;
    QND_NEED(A_host);
    set_device(ctx);
    const int64_t chunk = chunk_steps(ctx);
    for (int64_t c0 = 0; c0 < nsteps; c0 += chunk) {
        const int64_t ch = std::min(chunk, nsteps - c0);
        upload_field_chunk(ctx, A_host + size_t(c0) * ctx->s * ctx->dim, ch, true);
        velocity_steps(ctx, psi_dev, 0, ch, nullptr, false);
    }
    QND_CK(cudaGetLastError());
    check_finite(ctx, psi_dev, "qnd_step_velocity");
    QND_API_END
}

int qnd_run_length(qnd_ctx* ctx, void* psi_r_dev, const double* E_host, int64_t nsteps, int nobs,
                   const char* const* names, double* obs_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_r_dev);
    if (nsteps <= 0) return QND_OK;
    QND_NEED(E_host);
    if (nobs > 0) QND_NEED(names);
    set_device(ctx);
    int nv = 0;
    parse_obs(ctx, nobs, names, &nv);
    if (nv > 0) QND_NEED(obs_host);
    run_realtime(ctx, psi_r_dev, E_host, nullptr, nsteps, nobs, names, obs_host, false);
    check_finite(ctx, psi_r_dev, "qnd_run_length");
    QND_API_END
}

int qnd_run_velocity(qnd_ctx* ctx, void* psi_r_dev, const double* A_host, const double* alpha_host, int64_t nsteps,
                     int nobs, const char* const* names, double* obs_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_r_dev);
    if (nsteps <= 0) return QND_OK;
    QND_NEED(A_host);
    if (nobs > 0) QND_NEED(names);
    set_device(ctx);
    int nv = 0;
    parse_obs(ctx, nobs, names, &nv);
    if (nv > 0) {
        QND_NEED(obs_host);
        QND_NEED(alpha_host);
    }
    run_realtime(ctx, psi_r_dev, A_host, alpha_host, nsteps, nobs, names, obs_host, true);
    check_finite(ctx, psi_r_dev, "qnd_run_velocity");
    QND_API_END
}

int qnd_gram_schmidt(qnd_ctx* ctx, void* const* states_dev, int j, double* norm2_out) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(states_dev);
    if (j < 0) QND_FAIL(QND_EINVAL, "state index %d < 0", j);
    for (int k = 0; k <= j; ++k) QND_NEED(states_dev[k]);
    set_device(ctx);
    gs_project(ctx, states_dev, j);
    if (norm2_out) {
        QND_CK(cudaMemcpyAsync(norm2_out, ctx->scal.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    check_gs_flag(ctx, j);
    scale_state(ctx, states_dev[j], ctx->scal.as<double>() + 1);
    QND_CK(cudaStreamSynchronize(ctx->stream));
    QND_API_END
}

int qnd_imag_propagate(qnd_ctx* ctx, void* const* states_dev, int j, int64_t nsteps) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(states_dev);
    if (j < 0) QND_FAIL(QND_EINVAL, "state index %d < 0", j);
    for (int k = 0; k <= j; ++k) QND_NEED(states_dev[k]);
    if (nsteps <= 0) return QND_OK;
    set_device(ctx);
    // the first step, then blocks of up to CHUNK steps {step with the deferred normalisation,
    // Gram-Schmidt}, each replayed from a CUDA graph once its shape has been seen (run_chunk_graph);
    // the norm-collapse flag is read after every block
    imag_steps(ctx, states_dev[j], 1, nullptr);
    gs_project(ctx, states_dev, j);
    const double* pending = ctx->scal.as<double>() + 1;
    for (int64_t st = 1; st < nsteps; st += CHUNK) {
        const int64_t n = std::min(CHUNK, nsteps - st);
        std::string key = fmt("I|%llu|%d|%lld|%p|%p|%p|%p|%llu|%llu|%d|", (unsigned long long)ctx->serial, j,
                              (long long)n, ctx->scal.p, ctx->gs_flag.p, ctx->partials.p, ctx->counter.p,
                              (unsigned long long)ctx->table_epoch, (unsigned long long)ctx->config_epoch,
                              int(ctx->pdl));
        for (int k = 0; k <= j; ++k) key += fmt("%p,", states_dev[k]);
        run_chunk_graph(ctx, key, [&]() {
            for (int64_t q = 0; q < n; ++q) {
                imag_steps(ctx, states_dev[j], 1, pending);
                gs_project(ctx, states_dev, j);
            }
        });
        check_gs_flag(ctx, j);
    }
    scale_state(ctx, states_dev[j], pending);
    check_gs_flag(ctx, j);
    check_finite(ctx, states_dev[j], "qnd_imag_propagate");
    QND_API_END
}

int qnd_run_length_dev(qnd_ctx* ctx, void* psi_r_dev, const double* E_dev, int64_t nsteps, int nobs,
                       const char* const* names, double* obs_dev) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_r_dev);
    if (nsteps <= 0) return QND_OK;
    QND_NEED(E_dev);
    if (nobs > 0) QND_NEED(names);
    set_device(ctx);
    int nv = 0;
    auto items = parse_obs(ctx, nobs, names, &nv);
    if (nv > 0) QND_NEED(obs_dev);
    const bool fused = all_rspace(items);
    const bool masked = has_mask(ctx);
    const double zero[MAX_DIM] = {};
    // observables that are r-space reductions of one descriptor: chunk-wide chains
    const bool chain = nv == 0 || (fused && rspace_red(ctx, items, obs_dev, 0).size() <= 1);
    const int64_t chunk = chunk_steps(ctx);
    for (int64_t c0 = 0; c0 < nsteps; c0 += chunk) {
        const int64_t ch = std::min(chunk, nsteps - c0);
        build_field_tables(ctx, E_dev + size_t(c0) * ctx->s * ctx->dim, ch, false);
        if (chain) {
            // rows are staged in the context's buffer (fixed addresses, so that a captured chain
            // replays for every chunk), then copied to obs_dev
            double* stage = nullptr;
            if (nv > 0) {
                ctx->obs_dev.ensure(size_t(chunk) * nv * sizeof(double));
                stage = ctx->obs_dev.as<double>();
            }
            RedFn rf;
            if (nv > 0) rf = [&](int64_t k, int ax) { return rspace_red(ctx, items, stage + size_t(k) * nv, ax); };
            run_chunk_graph(ctx, chain_key(ctx, psi_r_dev, ch, nobs, names, stage, masked),
                            [&]() { length_steps(ctx, psi_r_dev, 0, ch, rf, masked); });
            if (nv > 0)
                QND_CK(cudaMemcpyAsync(obs_dev + size_t(c0) * nv, stage, size_t(ch) * nv * sizeof(double),
                                       cudaMemcpyDeviceToDevice, ctx->stream));
            continue;
        }
        for (int64_t k = 0; k < ch; ++k) {
            double* row = nv > 0 ? obs_dev + size_t(c0 + k) * nv : nullptr;
            std::vector<RedDesc> fin;
            if (nv > 0 && fused) fin = rspace_red(ctx, items, row, chain_final_axis(ctx, ctx->s + 1));
            RedFn rf;
            if (!fin.empty()) rf = [&](int64_t, int) { return std::vector<RedDesc>{fin[0]}; };
            length_steps(ctx, psi_r_dev, k, 1, rf, masked);
            if (fin.size() > 1) {
                auto nat = rspace_red(ctx, items, row, ctx->dim - 1);
                for (size_t q = 1; q < nat.size(); ++q) grid_reduce(ctx, psi_r_dev, nat[q]);
            }
            if (nv > 0 && !fused) eval_obs(ctx, psi_r_dev, items, zero, row);
        }
    }
    QND_CK(cudaGetLastError());
    check_finite(ctx, psi_r_dev, "qnd_run_length_dev");
    QND_API_END
}

int qnd_ctx_set_profiling(qnd_ctx* ctx, int enable) {
    QND_API_BEGIN
    QND_NEED(ctx);
    ctx->profiling = enable != 0;
    QND_API_END
}

int qnd_ctx_get_profile(qnd_ctx* ctx, int64_t* kernels_launched, int64_t* passes_timed, double* pass_ms_total,
                        int reset) {
    QND_API_BEGIN
    QND_NEED(ctx);
    set_device(ctx);
    QND_CK(cudaStreamSynchronize(ctx->stream));
    double total = 0;
    for (auto& pr : ctx->prof_pairs) {
        float ms = 0;
        QND_CK(cudaEventElapsedTime(&ms, pr.first, pr.second));
        total += ms;
    }
    if (kernels_launched) *kernels_launched = ctx->kernels_launched;
    if (passes_timed) *passes_timed = int64_t(ctx->prof_pairs.size());
    if (pass_ms_total) *pass_ms_total = total;
    if (reset) {
        for (auto& pr : ctx->prof_pairs) {
            ctx->event_pool.push_back(pr.first);
            ctx->event_pool.push_back(pr.second);
        }
        ctx->prof_pairs.clear();
        ctx->kernels_launched = 0;
    }
    QND_API_END
}

int qnd_observable_count(qnd_ctx* ctx, int nobs, const char* const* names, int* nvalues) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(nvalues);
    if (nobs > 0) QND_NEED(names);
    int nv = 0;
    for (int k = 0; k < nobs; ++k) {
        const char* nm = names[k] ? names[k] : "";
        if (!strcmp(nm, "norm") || !strcmp(nm, "energy") || !strcmp(nm, "Lz")) nv += 1;
        else if (!strcmp(nm, "dipole_r") || !strcmp(nm, "dipole_v") || !strcmp(nm, "accel")) nv += ctx->dim;
    }
    *nvalues = nv;
    QND_API_END
}

int qnd_observables(qnd_ctx* ctx, const void* psi_r_dev, int nobs, const char* const* names, const double* alpha,
                    double* out_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_r_dev);
    if (nobs > 0) QND_NEED(names);
    set_device(ctx);
    int nv = 0;
    auto items = parse_obs(ctx, nobs, names, &nv);
    if (nv == 0) return QND_OK;
    QND_NEED(out_host);
    double zero[MAX_DIM] = {};
    ctx->obs_dev.ensure(size_t(nv) * sizeof(double) * 2);
    eval_obs(ctx, psi_r_dev, items, alpha ? alpha : zero, ctx->obs_dev.as<double>());
    QND_CK(cudaMemcpyAsync(out_host, ctx->obs_dev.p, nv * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QND_CK(cudaStreamSynchronize(ctx->stream));
    QND_API_END
}

int qnd_energies(qnd_ctx* ctx, const void* psi_r_dev, int n, double* out_host) {
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_r_dev);
    if (n <= 0) return QND_OK;
    QND_NEED(out_host);
    set_device(ctx);
    ctx->obs_dev.ensure(size_t(n) * sizeof(double) * 2);
    energy_moments(ctx, psi_r_dev, n, ctx->obs_dev.as<double>());
    QND_CK(cudaMemcpyAsync(out_host, ctx->obs_dev.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QND_CK(cudaStreamSynchronize(ctx->stream));
    QND_API_END
}

int qnd_final_spectra(qnd_ctx* ctx, const void* psi_r_dev, double r_mask_min, double r_mask_max, const double* pr_max,
                      double de, int ne, double* ped_host, int64_t* npr_host, double* pmd_host) {
    using namespace qnd;
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_r_dev);
    QND_NEED(pr_max);
    if (ped_host && (ne <= 0 || !(de > 0.0))) QND_FAIL(QND_EINVAL, "qnd_final_spectra: the PED needs NE > 0 and DE > 0");
    if (!(r_mask_max > r_mask_min)) QND_FAIL(QND_EINVAL, "qnd_final_spectra: R_MASK needs Rmin < Rmax");
    set_device(ctx);
    const int d = ctx->dim;
    // kept momenta per axis (|p| <= pr_max, io_functions.c:191, :218-225) and their ranks
    std::vector<int> rank(size_t(ctx->axtot), -1);
    int64_t npr[MAX_DIM] = {};
    for (int j = 0; j < d; ++j)
        for (int k = 0; k < int(ctx->nr[j]); ++k)
            if (std::fabs(ctx->p[j][k]) <= pr_max[j]) rank[ctx->axoff[j] + k] = int(npr[j]++);
    if (npr_host)
        for (int j = 0; j < d; ++j) npr_host[j] = npr[j];
    if (!ped_host && !pmd_host) return QND_OK;
    ctx->spec_rank.ensure(rank.size() * sizeof(int));
    QND_CK(cudaMemcpyAsync(ctx->spec_rank.p, rank.data(), rank.size() * sizeof(int), cudaMemcpyHostToDevice,
                           ctx->stream));
    SpectraArgs a{};
    a.r = ctx->r_dev.as<double>();
    a.p = ctx->p_dev.as<double>();
    a.rank = ctx->spec_rank.as<int>();
    a.dim = d;
    a.n = ctx->n;
    long long stride = 1;
    for (int j = d - 1; j >= 0; --j) {
        a.stride[j] = stride;
        stride *= npr[j];
    }
    for (int j = 0; j < d; ++j) {
        a.axoff[j] = ctx->axoff[j];
        a.shift[j] = ctx->shift[j];
        a.nmask[j] = ctx->nr[j] - 1;
    }
    a.rmin = r_mask_min;
    a.rmax = r_mask_max;
    a.de = de;
    a.sigma = de;
    a.ne = ne;
    a.norm = 1.0 / std::pow(2.0 * M_PI * de * de, .5 * d);
    // the masked state, in the unitary p-representation (io_functions.c:158-170)
    ensure_scratch_state(ctx, ctx->scratch_a);
    void* q = ctx->scratch_a.p;
    if (ctx->fp64)
        launch_radial_mask<double>(a, static_cast<const double2*>(psi_r_dev), static_cast<double2*>(q), ctx->stream);
    else
        launch_radial_mask<float>(a, static_cast<const float2*>(psi_r_dev), static_cast<float2*>(q), ctx->stream);
    ctx->kernels_launched++;
    QND_CK(cudaGetLastError());
    unitary_fft(ctx, q, true);
    if (ped_host) {
        const size_t nb = size_t((ctx->n + PED_CHUNK - 1) / PED_CHUNK);
        ctx->spec_partials.ensure(nb * size_t(ne) * sizeof(double));
        ctx->spec_out.ensure(size_t(ne) * sizeof(double));
        if (ctx->fp64)
            launch_ped<double>(a, static_cast<const double2*>(q), ctx->spec_partials.as<double>(),
                               ctx->spec_out.as<double>(), ctx->stream);
        else
            launch_ped<float>(a, static_cast<const float2*>(q), ctx->spec_partials.as<double>(),
                              ctx->spec_out.as<double>(), ctx->stream);
        ctx->kernels_launched += 2;
        QND_CK(cudaGetLastError());
        QND_CK(cudaMemcpyAsync(ped_host, ctx->spec_out.p, size_t(ne) * sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream));
        QND_CK(cudaStreamSynchronize(ctx->stream));
    }
    if (pmd_host && stride > 0) {
        ctx->spec_out.ensure(size_t(stride) * 2 * sizeof(double));
        if (ctx->fp64)
            launch_pmd<double>(a, static_cast<const double2*>(q), ctx->spec_out.as<double>(), ctx->stream);
        else
            launch_pmd<float>(a, static_cast<const float2*>(q), ctx->spec_out.as<double>(), ctx->stream);
        ctx->kernels_launched++;
        QND_CK(cudaGetLastError());
        QND_CK(cudaMemcpyAsync(pmd_host, ctx->spec_out.p, size_t(stride) * 2 * sizeof(double), cudaMemcpyDeviceToHost,
                               ctx->stream));
        QND_CK(cudaStreamSynchronize(ctx->stream));
    }
    QND_API_END
}

int qnd_run_length_batch(int count, qnd_ctx* const* ctxs, void* const* psi_r_dev, const double* const* E_dev,
                         int64_t nsteps, int nobs, const char* const* names, double* const* obs_dev) {
    using namespace qnd;
    QND_API_BEGIN
    if (count < 1) QND_FAIL(QND_EINVAL, "qnd_run_length_batch: count %d < 1", count);
    QND_NEED(ctxs);
    QND_NEED(psi_r_dev);
    QND_NEED(E_dev);
    if (nobs > 0) QND_NEED(names);
    for (int i = 0; i < count; ++i) {
        QND_NEED(ctxs[i]);
        QND_NEED(psi_r_dev[i]);
        QND_NEED(E_dev[i]);
        if (ctxs[i]->device != ctxs[0]->device) QND_FAIL(QND_EINVAL, "qnd_run_length_batch: members on different devices");
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == ctxs[i]) QND_FAIL(QND_EINVAL, "qnd_run_length_batch: a context appears twice");
    }
    if (nsteps <= 0) return QND_OK;
    set_device(ctxs[0]);
    std::vector<SweepMember> ms(static_cast<size_t>(count));
    bool one_graph = true;
    int64_t chunk = CHUNK;
    for (int i = 0; i < count; ++i) {
        SweepMember& m = ms[i];
        m.c = ctxs[i];
        m.items = parse_obs(m.c, nobs, names, &m.nv);
        if (m.nv > 0) QND_NEED(obs_dev);
        if (m.nv > 0 && obs_dev) QND_NEED(obs_dev[i]);
        m.masked = has_mask(m.c);
        std::vector<double> probe(size_t(m.nv) + 1);  // only the descriptor count is wanted here
        if (m.nv > 0 && !(all_rspace(m.items) && rspace_red(m.c, m.items, probe.data(), 0).size() <= 1))
            one_graph = false;
        chunk = std::min(chunk, chunk_steps(m.c));
    }
    if (!one_graph) {
        // observables beyond one fused descriptor: each member's own device loop
        for (int i = 0; i < count; ++i) {
            const int rc = qnd_run_length_dev(ctxs[i], psi_r_dev[i], E_dev[i], nsteps, nobs, names,
                                              ms[i].nv ? obs_dev[i] : nullptr);
            if (rc != QND_OK) return rc;
        }
        return QND_OK;
    }
    for (SweepMember& m : ms)
        if (m.nv > 0) {
            m.c->obs_dev.ensure(size_t(chunk) * m.nv * sizeof(double));
            m.stage = m.c->obs_dev.as<double>();
        }
    // a root stream forks to every member's stream and joins them again: the members' chains of one
    // chunk are the parallel branches of one graph
    struct Res {
        cudaStream_t root = nullptr;
        cudaEvent_t fork = nullptr;
        std::vector<cudaEvent_t> join;
        ~Res() {
            if (root) cudaStreamSynchronize(root);
            if (fork) cudaEventDestroy(fork);
            for (cudaEvent_t e : join)
                if (e) cudaEventDestroy(e);
            if (root) cudaStreamDestroy(root);
        }
    } r;
    QND_CK(cudaStreamCreateWithFlags(&r.root, cudaStreamNonBlocking));
    QND_CK(cudaEventCreateWithFlags(&r.fork, cudaEventDisableTiming));
    r.join.assign(size_t(count), nullptr);
    for (auto& e : r.join) QND_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    auto fork_members = [&]() {
        QND_CK(cudaEventRecord(r.fork, r.root));
        for (SweepMember& m : ms) QND_CK(cudaStreamWaitEvent(m.c->stream, r.fork, 0));
    };
    auto join_members = [&]() {
        for (int i = 0; i < count; ++i) {
            QND_CK(cudaEventRecord(r.join[i], ms[i].c->stream));
            QND_CK(cudaStreamWaitEvent(r.root, r.join[i], 0));
        }
    };
    auto chains = [&](int64_t ch) {
        for (SweepMember& m : ms) {
            RedFn rf;
            if (m.nv > 0) {
                SweepMember* mp = &m;
                rf = [mp](int64_t k, int ax) { return rspace_red(mp->c, mp->items, mp->stage + size_t(k) * mp->nv, ax); };
            }
            length_steps(m.c, psi_r_dev[&m - ms.data()], 0, ch, rf, m.masked);
        }
    };
    // the sweep's graphs live in the first member's context, keyed by every member's chain
    qnd_ctx* home = ms[0].c;
    const bool no_graph = std::getenv("QND_NO_GRAPH") != nullptr;
    for (int64_t c0 = 0; c0 < nsteps; c0 += chunk) {
        const int64_t ch = std::min(chunk, nsteps - c0);
        for (int i = 0; i < count; ++i)
            build_field_tables(ms[i].c, E_dev[i] + size_t(c0) * ms[i].c->s * ms[i].c->dim, ch, false);
        join_members();  // the root waits for every member's tables (and its earlier work)
        std::string key = fmt("B%d|%lld|", count, (long long)ch);
        for (int i = 0; i < count; ++i)
            key += chain_key(ms[i].c, psi_r_dev[i], ch, nobs, names, ms[i].stage, ms[i].masked) + "#";
        GraphEntry* ge = no_graph ? nullptr : find_graph(home, key);
        if (ge) {
            QND_CK(cudaGraphLaunch(ge->exec, r.root));
            // the launch counters advance as for direct launches (they seed the FP32 dithering)
            for (int i = 0; i < count; ++i) ms[i].c->kernels_launched += ge->launches[i];
        } else if (no_graph || !seen_before(home, key)) {
            // first chunk of this shape: direct launches (they build the tables the chains read)
            fork_members();
            chains(ch);
            join_members();
        } else {
            std::vector<int64_t> launches(static_cast<size_t>(count));
            for (int i = 0; i < count; ++i) launches[i] = ms[i].c->kernels_launched;
            QND_CK(cudaStreamBeginCapture(r.root, cudaStreamCaptureModeThreadLocal));
            cudaGraph_t g = nullptr;
            try {
                fork_members();
                chains(ch);
                join_members();
            } catch (...) {
                cudaStreamEndCapture(r.root, &g);
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                throw;
            }
            QND_CK(cudaStreamEndCapture(r.root, &g));
            for (int i = 0; i < count; ++i) launches[i] = ms[i].c->kernels_launched - launches[i];
            cudaGraphExec_t ex = nullptr;
            const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                cudaGetLastError();
                QND_FAIL(QND_ECUDA, "cudaGraphInstantiate of a batch chunk: %s", cudaGetErrorString(e));
            }
            keep_graph(home, key, ex, std::move(launches));
            QND_CK(cudaGraphLaunch(ex, r.root));
        }
        // each member's rows of this chunk to the caller, after the chunk
        fork_members();
        for (int i = 0; i < count; ++i)
            if (ms[i].nv > 0)
                QND_CK(cudaMemcpyAsync(obs_dev[i] + size_t(c0) * ms[i].nv, ms[i].stage,
                                       size_t(ch) * ms[i].nv * sizeof(double), cudaMemcpyDeviceToDevice,
                                       ms[i].c->stream));
    }
    join_members();
    QND_CK(cudaGetLastError());
    QND_API_END
}

// qnd_run_length_sweep: every member's passes recorded (the chains qnd_run_length_dev would launch,
// chunk by chunk, with the same arguments), then run by the persistent sweep kernel (qnd_sweep.cu) in
// one launch per segment of SWEEP_SEGMENT steps. Segments keep the recorded arguments and the field
// tables of all their chunks in device memory at once.
static const int64_t SWEEP_SEGMENT = 512;

int qnd_run_length_sweep(int count, qnd_ctx* const* ctxs, void* const* psi_r_dev, const double* const* E_dev,
                         int64_t nsteps, int nobs, const char* const* names, double* const* obs_dev) {
    using namespace qnd;
    QND_API_BEGIN
    if (count < 1) QND_FAIL(QND_EINVAL, "qnd_run_length_sweep: count %d < 1", count);
    QND_NEED(ctxs);
    QND_NEED(psi_r_dev);
    QND_NEED(E_dev);
    if (nobs > 0) QND_NEED(names);
    for (int i = 0; i < count; ++i) {
        QND_NEED(ctxs[i]);
        QND_NEED(psi_r_dev[i]);
        QND_NEED(E_dev[i]);
        qnd_ctx* c = ctxs[i];
        if (c->device != ctxs[0]->device) QND_FAIL(QND_EINVAL, "qnd_run_length_sweep: members on different devices");
        if (c->fp64 != ctxs[0]->fp64)
            QND_FAIL(QND_EUNSUPPORTED, "qnd_run_length_sweep: members of both precisions (one kernel per precision)");
        if (c->long1d) QND_FAIL(QND_EUNSUPPORTED, "qnd_run_length_sweep: a 1-D axis longer than 4096 points");
        for (int j = 0; j < c->dim; ++j)
            if (!sweep_length_ok(c->nr[j]))
                QND_FAIL(QND_EUNSUPPORTED, "qnd_run_length_sweep: axis length %lld (the sweep kernel takes 128 to 1024)",
                         (long long)c->nr[j]);
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == c) QND_FAIL(QND_EINVAL, "qnd_run_length_sweep: a context appears twice");
    }
    if (nsteps <= 0) return QND_OK;
    set_device(ctxs[0]);
    std::vector<SweepMember> ms(static_cast<size_t>(count));
    for (int i = 0; i < count; ++i) {
        SweepMember& m = ms[i];
        m.c = ctxs[i];
        m.items = parse_obs(m.c, nobs, names, &m.nv);
        if (m.nv > 0) {
            QND_NEED(obs_dev);
            QND_NEED(obs_dev[i]);
        }
        m.masked = has_mask(m.c);
        std::vector<double> probe(size_t(m.nv) + 1);
        if (m.nv > 0 && !(all_rspace(m.items) && rspace_red(m.c, m.items, probe.data(), 0).size() <= 1))
            QND_FAIL(QND_EUNSUPPORTED, "qnd_run_length_sweep: observables beyond one fused reduction descriptor");
    }
    qnd_ctx* home = ctxs[0];
    const size_t argsz = (size_t(home->fp64 ? sizeof(PassArgs<double>) : sizeof(PassArgs<float>)) + 127) / 128 * 128;
    struct Ev {
        std::vector<cudaEvent_t> e;
        ~Ev() {
            for (cudaEvent_t x : e)
                if (x) cudaEventDestroy(x);
        }
    } ev;
    ev.e.assign(size_t(count) + 1, nullptr);
    for (auto& x : ev.e) QND_CK(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    int failed = 0;
    for (int64_t s0 = 0; s0 < nsteps && !failed; s0 += SWEEP_SEGMENT) {
        const int64_t seg = std::min(SWEEP_SEGMENT, nsteps - s0);
        // record every member's chains for this segment (their field tables built on their streams)
        std::vector<std::vector<RecordedPass>> rec(static_cast<size_t>(count));
        for (int i = 0; i < count; ++i) {
            SweepMember& m = ms[i];
            qnd_ctx* c = m.c;
            const int64_t chunk = chunk_steps(c);
            const size_t per_step = size_t(c->s) * c->axtot * c->elem();
            c->sweep_field.ensure(size_t(seg) * per_step);
            for (int64_t c0 = 0; c0 < seg; c0 += chunk) {
                const int64_t ch = std::min(chunk, seg - c0);
                void* tabs = static_cast<char*>(c->sweep_field.p) + size_t(c0) * per_step;
                build_field_tables(c, E_dev[i] + size_t(s0 + c0) * c->s * c->dim, ch, false, 1 << 30, tabs);
                RedFn rf;
                if (m.nv > 0) {
                    double* rows = obs_dev[i] + size_t(s0 + c0) * m.nv;
                    SweepMember* mp = &m;
                    rf = [mp, rows](int64_t k, int ax) { return rspace_red(mp->c, mp->items, rows + size_t(k) * mp->nv, ax); };
                }
                c->recorder = &rec[i];
                c->field_view = tabs;
                try {
                    length_steps(c, psi_r_dev[i], 0, ch, rf, m.masked);
                } catch (...) {
                    c->recorder = nullptr;
                    c->field_view = nullptr;
                    throw;
                }
                c->recorder = nullptr;
                c->field_view = nullptr;
            }
        }
        // slots in round order, items (line groups) numbered through them
        size_t npass = 0, maxp = 0;
        for (auto& r : rec) {
            npass += r.size();
            maxp = std::max(maxp, r.size());
        }
        std::vector<unsigned> need(size_t(count), 0);
        std::vector<SweepSlot> slots;
        std::vector<long long> first;
        std::vector<unsigned char> blob(npass * argsz);
        slots.reserve(npass);
        first.reserve(npass);
        long long nitems = 0;
        size_t nb = 0;
        std::vector<size_t> blob_off;
        blob_off.reserve(npass);
        for (size_t r = 0; r < maxp; ++r)
            for (int i = 0; i < count; ++i) {
                if (r >= rec[i].size()) continue;
                const RecordedPass& p = rec[i][r];
                std::memcpy(blob.data() + nb, p.args.data(), p.args.size());
                SweepSlot sl{};
                sl.ngroups = p.ngroups;
                // about 64 work items per pass (measured: items of a fixed size of about 16384 points,
                // fewer for the small members' passes, ran the 96-member sweep 10% slower)
                sl.gpi = std::max(1u, p.ngroups / 64u);
                sl.need = need[i];
                sl.member = i;
                sl.L = p.L;
                sl.strided = p.strided;
                sl.kmode = p.kmode;
                slots.push_back(sl);
                blob_off.push_back(nb);
                first.push_back(nitems);
                nitems += (p.ngroups + sl.gpi - 1) / sl.gpi;
                need[i] += p.ngroups;
                nb += argsz;
            }
        // device layout: [args blob][slots][first][done (count) | next | abort]
        const size_t o_slots = (nb + 255) / 256 * 256;
        const size_t o_first = (o_slots + slots.size() * sizeof(SweepSlot) + 255) / 256 * 256;
        const size_t o_ctl = (o_first + first.size() * sizeof(long long) + 255) / 256 * 256;
        const size_t ctl_bytes = (size_t(count) * sizeof(unsigned) + 15) / 16 * 16 + 16 + 16;
        home->sweep_buf.ensure(o_ctl + ctl_bytes);
        char* dbuf = static_cast<char*>(home->sweep_buf.p);
        for (size_t q = 0; q < slots.size(); ++q) slots[q].args = dbuf + blob_off[q];
        // every member's earlier work (state, tables) before the sweep's stream reads it
        for (int i = 0; i < count; ++i) {
            QND_CK(cudaEventRecord(ev.e[i], ms[i].c->stream));
            QND_CK(cudaStreamWaitEvent(home->stream, ev.e[i], 0));
        }
        QND_CK(cudaMemcpyAsync(dbuf, blob.data(), nb, cudaMemcpyHostToDevice, home->stream));
        QND_CK(cudaMemcpyAsync(dbuf + o_slots, slots.data(), slots.size() * sizeof(SweepSlot), cudaMemcpyHostToDevice,
                               home->stream));
        QND_CK(cudaMemcpyAsync(dbuf + o_first, first.data(), first.size() * sizeof(long long), cudaMemcpyHostToDevice,
                               home->stream));
        QND_CK(cudaMemsetAsync(dbuf + o_ctl, 0, ctl_bytes, home->stream));
        SweepArgs sa{};
        sa.slots = reinterpret_cast<const SweepSlot*>(dbuf + o_slots);
        sa.first = reinterpret_cast<const long long*>(dbuf + o_first);
        sa.nslots = int(slots.size());
        sa.nitems = nitems;
        sa.done = reinterpret_cast<unsigned*>(dbuf + o_ctl);
        const size_t o_next = (size_t(count) * sizeof(unsigned) + 15) / 16 * 16;
        sa.next = reinterpret_cast<unsigned long long*>(dbuf + o_ctl + o_next);
        sa.abort_flag = reinterpret_cast<int*>(dbuf + o_ctl + o_next + 16);
        sa.wait_tries = 1 << 22;  // ~1 s of polling per item before the launch gives up
        int grid = 0;
        const cudaError_t le = home->fp64 ? launch_sweep<double>(sa, home->stream, home->num_sms, &grid)
                                          : launch_sweep<float>(sa, home->stream, home->num_sms, &grid);
        if (le != cudaSuccess) {
            cudaGetLastError();
            QND_FAIL(QND_ECUDA, "qnd_run_length_sweep: launch of the sweep kernel: %s", cudaGetErrorString(le));
        }
        // the members' later work after the sweep; the blob and tables are reused by the next segment
        QND_CK(cudaEventRecord(ev.e[count], home->stream));
        for (int i = 0; i < count; ++i) QND_CK(cudaStreamWaitEvent(ms[i].c->stream, ev.e[count], 0));
        QND_CK(cudaMemcpyAsync(&failed, sa.abort_flag, sizeof(int), cudaMemcpyDeviceToHost, home->stream));
        QND_CK(cudaStreamSynchronize(home->stream));
    }
    if (failed) {
        // a wait ran out: the skipped groups' reductions never finished; clear their ticket counters
        for (SweepMember& m : ms)
            if (m.c->counter.p) QND_CK(cudaMemsetAsync(m.c->counter.p, 0, m.c->counter.bytes, m.c->stream));
        for (SweepMember& m : ms) QND_CK(cudaStreamSynchronize(m.c->stream));
        QND_FAIL(QND_ECUDA, "qnd_run_length_sweep: a wait for a member's previous pass ran out; results are invalid");
    }
    QND_CK(cudaGetLastError());
    QND_API_END
}

int qnd_adjoint_length(qnd_ctx* ctx, const void* psi0_dev, const double* E_host, int64_t nsteps, const double* w_host,
                       int64_t checkpoint, double* J_out, double* grad_host, void* psiT_dev) {
    using namespace qnd;
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi0_dev);
    QND_NEED(w_host);
    if (nsteps < 1) QND_FAIL(QND_EINVAL, "qnd_adjoint_length: nsteps %lld < 1", (long long)nsteps);
    QND_NEED(E_host);
    QND_NEED(grad_host);
    if (checkpoint < 1) QND_FAIL(QND_EINVAL, "qnd_adjoint_length: checkpoint interval %lld < 1", (long long)checkpoint);
    set_device(ctx);
    adjoint_run(ctx, psi0_dev, E_host, nsteps, w_host, checkpoint, J_out, grad_host, psiT_dev, false);
    QND_API_END
}

int qnd_adjoint_velocity(qnd_ctx* ctx, const void* psi0_dev, const double* A_host, int64_t nsteps,
                         const double* w_host, int64_t checkpoint, double* J_out, double* grad_host, void* psiT_dev) {
    using namespace qnd;
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi0_dev);
    QND_NEED(w_host);
    if (nsteps < 1) QND_FAIL(QND_EINVAL, "qnd_adjoint_velocity: nsteps %lld < 1", (long long)nsteps);
    QND_NEED(A_host);
    QND_NEED(grad_host);
    if (checkpoint < 1) QND_FAIL(QND_EINVAL, "qnd_adjoint_velocity: checkpoint interval %lld < 1", (long long)checkpoint);
    set_device(ctx);
    adjoint_run(ctx, psi0_dev, A_host, nsteps, w_host, checkpoint, J_out, grad_host, psiT_dev, true);
    QND_API_END
}

int qnd_field_samples(qnd_ctx* ctx, int nmodes, const qnd_laser_mode* modes, int64_t nsteps, double* E_out,
                      double* A_out, double* alpha_out, int on_device) {
    using namespace qnd;
    QND_API_BEGIN
    QND_NEED(ctx);
    if (nmodes < 0 || nmodes > MAX_MODES) QND_FAIL(QND_EUNSUPPORTED, "%d laser modes: this build takes 0 to %d", nmodes, MAX_MODES);
    if (nmodes > 0) QND_NEED(modes);
    if (nsteps < 0) QND_FAIL(QND_EINVAL, "nsteps %lld < 0", (long long)nsteps);
    if (nsteps == 0 || (!E_out && !A_out && !alpha_out)) return QND_OK;
    set_device(ctx);
    FieldSampleArgs a{};
    for (int m = 0; m < nmodes; ++m) {
        const qnd_laser_mode& md = modes[m];
        if (md.envelope < QND_ENV_CONSTANT || md.envelope > QND_ENV_COS4)
            QND_FAIL(QND_EINVAL, "Unknown envelope code %d (mode %d)", md.envelope, m);
        a.mode[m] = FieldMode{md.frequency, md.amplitude, md.ellipticity, md.cep, md.delay, md.duration, md.envelope};
    }
    a.nmodes = nmodes;
    a.dim = ctx->dim;
    a.s = ctx->s;
    a.nsteps = nsteps;
    a.dt = ctx->dt;
    for (int k = 0; k < 2 * ctx->s; ++k) a.as[k] = ctx->as[k];
    const size_t nsub = size_t(nsteps) * ctx->s * ctx->dim, nal = size_t(nsteps) * ctx->dim;
    if (on_device) {
        launch_field_samples(a, E_out, A_out, alpha_out, ctx->stream);
        ctx->kernels_launched++;
        QND_CK(cudaGetLastError());
        return QND_OK;
    }
    ctx->field_out.ensure((2 * nsub + nal) * sizeof(double));
    double* dE = ctx->field_out.as<double>();
    double* dA = dE + nsub;
    double* dal = dA + nsub;
    launch_field_samples(a, E_out ? dE : nullptr, A_out ? dA : nullptr, alpha_out ? dal : nullptr, ctx->stream);
    ctx->kernels_launched++;
    QND_CK(cudaGetLastError());
    if (E_out) QND_CK(cudaMemcpyAsync(E_out, dE, nsub * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (A_out) QND_CK(cudaMemcpyAsync(A_out, dA, nsub * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    if (alpha_out) QND_CK(cudaMemcpyAsync(alpha_out, dal, nal * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    QND_CK(cudaStreamSynchronize(ctx->stream));
    QND_API_END
}

int qnd_state_embed(qnd_ctx* ctx, void* psi_dev, const double* src_host, const int64_t* nr_src, double coeff_re,
                    double coeff_im, int accumulate) {
    using namespace qnd;
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_dev);
    QND_NEED(src_host);
    QND_NEED(nr_src);
    EmbedArgs a{};
    a.dim = ctx->dim;
    a.n_src = 1;
    for (int j = 0; j < ctx->dim; ++j) {
        if (nr_src[j] < 1) QND_FAIL(QND_EINVAL, "source grid NR[%d]=%lld < 1", j, (long long)nr_src[j]);
        a.nr_src[j] = nr_src[j];
        a.nr[j] = ctx->nr[j];
        a.off[j] = (ctx->nr[j] - nr_src[j]) / 2;  // C division, as io_functions.c's centring offset
        a.n_src *= nr_src[j];
    }
    a.cr = coeff_re;
    a.ci = coeff_im;
    set_device(ctx);
    if (!accumulate) QND_CK(cudaMemsetAsync(psi_dev, 0, size_t(ctx->n) * ctx->elem(), ctx->stream));
    ctx->embed_src.ensure(size_t(a.n_src) * 16);
    QND_CK(cudaMemcpyAsync(ctx->embed_src.p, src_host, size_t(a.n_src) * 16, cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->fp64)
        launch_embed<double>(a, ctx->embed_src.as<double2>(), static_cast<double2*>(psi_dev), ctx->stream);
    else
        launch_embed<float>(a, ctx->embed_src.as<double2>(), static_cast<float2*>(psi_dev), ctx->stream);
    ctx->kernels_launched++;
    QND_CK(cudaGetLastError());
    QND_CK(cudaStreamSynchronize(ctx->stream));  // the caller may release src_host on return
    QND_API_END
}

}  // extern "C"

// ============================================== r-space observables, no allocation ==
//
// qnd_observables_rspace_noalloc evaluates the r-space observables of qnd_observables
// ("norm", "dipole_r", "accel") with the same grid-reduction kernel and the same CTA count,
// so it adds the same partial sums in the same order. It differs in three ways:
//  - the reduction scratch is a fixed device array in this file, not the context's
//    growable buffers;
//  - the values go to a caller device buffer, not through a host copy;
//  - it allocates no device, pinned or host memory and does not synchronise.
//
// It serves callers that must not call cudaMalloc or cudaFree:
//  - A monitor that samples a state between the steps of a device-resident loop. Growing a
//    buffer frees the old one, and cudaFree synchronises the whole device, stalling the
//    propagation and every other stream.
//  - A process whose device memory is already reserved by another allocator's pool. There a
//    new cudaMalloc fails.
//
// The first call on a device does a one-time set-up with that device current: it resolves
// the scratch array's address and zeroes its ticket counter, which synchronises the context's
// stream once. Make that first call before any stream capture.
//
// All calls on one device share the one scratch array. Calls whose launches can overlap
// (different streams without ordering between them) race on it and give wrong sums.
// Serialise them.

namespace qnd {

constexpr int NOALLOC_MAX_BLOCKS = 148 * 4;   // CTAs of one grid reduction (the cap of reduce_blocks)
constexpr int NOALLOC_MAX_VALUES = 64;        // observable values per call
constexpr size_t NOALLOC_PARTIALS = size_t(NOALLOC_MAX_BLOCKS) * MAX_RED;  // doubles
constexpr size_t NOALLOC_COUNTER_SLOT = 32;   // doubles (256 bytes) holding the ticket counter word
constexpr int NOALLOC_MAX_DEVICES = 64;

// Reduction scratch: [NOALLOC_MAX_BLOCKS][MAX_RED] partial sums (37,888 bytes), then the
// ticket counter (one 32-bit word in a 256-byte slot): 38,144 bytes per device.
//  - The counter word must be zero when a reduction starts. Static device storage is zero at
//    module load, the set-up zeroes it again, and the last CTA of every reduction resets it.
//  - The partial sums need no initial value: each CTA writes its own slot before it takes a
//    ticket.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_PARTIALS + NOALLOC_COUNTER_SLOT];

static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[NOALLOC_MAX_DEVICES];  // per device, filled by the set-up

// Address of this device's scratch array; the set-up runs once per device, c->device current.
static double* noalloc_scratch(qnd_ctx* c) {
    if (c->device < 0 || c->device >= NOALLOC_MAX_DEVICES)
        QND_FAIL(QND_EUNSUPPORTED, "qnd_observables_rspace_noalloc: device %d is beyond the %d devices it tracks",
                 c->device, NOALLOC_MAX_DEVICES);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    double*& p = g_noalloc_ptr[c->device];
    if (!p) {
        void* q = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&q, g_noalloc_scratch);
        if (e != cudaSuccess || !q) {
            cudaGetLastError();
            QND_FAIL(QND_ECUDA, "qnd_observables_rspace_noalloc: cudaGetSymbolAddress of the scratch array on device %d: %s",
                     c->device, cudaGetErrorString(e));
        }
        double* base = static_cast<double*>(q);
        QND_CK(cudaMemsetAsync(base + NOALLOC_PARTIALS, 0, NOALLOC_COUNTER_SLOT * sizeof(double), c->stream));
        QND_CK(cudaStreamSynchronize(c->stream));
        p = base;
    }
    return p;
}

template <typename R>
static void noalloc_launch(qnd_ctx* c, const void* psi, const RedDesc& rd, double* scratch, int nblocks) {
    PassSpec ps;
    ps.psi = const_cast<void*>(psi);
    ps.red = rd;
    PassArgs<R> a;
    fill_args<R>(c, ps, a);
    a.red.partials = scratch;
    a.red.counter = reinterpret_cast<unsigned int*>(scratch + NOALLOC_PARTIALS);
    launch_grid_reduce<R>(a, c->n, c->stream, nblocks);
    c->kernels_launched++;
    QND_CK(cudaGetLastError());
}

}  // namespace qnd

extern "C" int qnd_observables_rspace_noalloc(qnd_ctx* ctx, const void* psi_r_dev, int nobs, const char* const* names,
                                              double* out_dev) {
    using namespace qnd;
    QND_API_BEGIN
    QND_NEED(ctx);
    QND_NEED(psi_r_dev);
    if (nobs < 0) QND_FAIL(QND_EINVAL, "qnd_observables_rspace_noalloc: nobs = %d", nobs);
    if (nobs > 0) QND_NEED(names);
    // Values per name, in qnd_observables' row layout; the k-space observables need transform
    // passes whose tables and scratch states the context allocates on first use.
    int nv = 0;
    for (int k = 0; k < nobs; ++k) {
        const char* nm = names[k] ? names[k] : "";
        if (!strcmp(nm, "norm")) nv += 1;
        else if (!strcmp(nm, "dipole_r")) nv += ctx->dim;
        else if (!strcmp(nm, "accel")) {
            for (int j = 0; j < ctx->dim; ++j)
                if (!ctx->gradv_dev[j].p) QND_FAIL(QND_EINVAL, "observable 'accel' needs qnd_set_gradv for every axis");
            nv += ctx->dim;
        } else if (!strcmp(nm, "dipole_v") || !strcmp(nm, "energy") || !strcmp(nm, "Lz"))
            QND_FAIL(QND_EUNSUPPORTED,
                     "qnd_observables_rspace_noalloc: '%s' needs k-space passes; only norm, dipole_r and accel are "
                     "evaluated without allocation (use qnd_observables)", nm);
    }
    if (nv > NOALLOC_MAX_VALUES)
        QND_FAIL(QND_EINVAL, "qnd_observables_rspace_noalloc: %d observable values requested, at most %d per call", nv,
                 NOALLOC_MAX_VALUES);
    if (nv == 0) return QND_OK;
    QND_NEED(out_dev);
    const int nblocks = reduce_blocks(ctx);
    if (nblocks > NOALLOC_MAX_BLOCKS)
        QND_FAIL(QND_EUNSUPPORTED,
                 "qnd_observables_rspace_noalloc: the reduction needs %d CTAs x %d partial sums of scratch, the static "
                 "array holds %d CTAs", nblocks, MAX_RED, NOALLOC_MAX_BLOCKS);
    set_device(ctx);
    double* scratch = noalloc_scratch(ctx);
    // Contiguous runs of at most MAX_RED values per launch, in row order.
    RedDesc cur{};
    int off = 0;
    auto flush = [&]() {
        if (!cur.n) return;
        if (ctx->fp64) noalloc_launch<double>(ctx, psi_r_dev, cur, scratch, nblocks);
        else noalloc_launch<float>(ctx, psi_r_dev, cur, scratch, nblocks);
        cur = RedDesc{};
    };
    auto add = [&](int wkind, int waxis, const double* wtab, double scale) {
        if (cur.n == MAX_RED) flush();
        if (!cur.n) cur.out = out_dev + off;
        cur.kind[cur.n] = RK_ABS2;
        cur.wkind[cur.n] = wkind;
        cur.waxis[cur.n] = waxis;
        cur.wtab[cur.n] = wtab;
        cur.scale[cur.n] = scale;
        cur.n++;
        off++;
    };
    for (int k = 0; k < nobs; ++k) {
        const char* nm = names[k] ? names[k] : "";
        if (!strcmp(nm, "norm")) add(WK_ONE, 0, nullptr, ctx->dNr);
        else if (!strcmp(nm, "dipole_r"))
            for (int j = 0; j < ctx->dim; ++j) add(WK_AXIS, j, ctx->r_dev.as<double>() + ctx->axoff[j], ctx->dNr);
        else if (!strcmp(nm, "accel"))
            for (int j = 0; j < ctx->dim; ++j) add(WK_GRID, 0, ctx->gradv_dev[j].as<double>(), -ctx->dNr);
    }
    flush();
    QND_API_END
}
