// qnd_kernels.cuh — kernel registry and auxiliary kernels shared by the engine.
#pragma once

#include "qnd_pass.cuh"

namespace qnd {

struct PassKernelInfo {
    const void* fn;
    int nt;       // threads per CTA
    size_t smem;  // dynamic shared memory bytes
    int G;        // lines per CTA
    int tw_size;  // twiddle entries expected in the plan table
    int E;        // values per thread (fixes the stage structure of the twiddle table)
};

// Defined once per line length in qnd_pass_inst.cu (compiled with -DQND_L=...). var: the shape
// variant (PassShape); fn is null where a variant does not exist.
// tma: the strided instantiation that stages its lines by TMA boxes (the host has a tensor map for it)
template <typename R, int L> PassKernelInfo pass_kernel_info(bool strided, int mode, int var = 0, bool tma = false);

// Host-side copy of the FFTPlan stage structure for a runtime line length.
struct HostPlan {
    int L, E, T, nstage;
    int radix[16], span[16];
    int tw_size;   // table form (FP32): R - 1 twiddles per butterfly position
    int twb_size;  // base form (FP64): one twiddle per butterfly position
    HostPlan(int L_, int E_) : L(L_) {
        E = E_;
        T = L / E;
        int logl = 0, loge = 0;
        while ((1 << logl) < L) ++logl;
        while ((1 << loge) < E) ++loge;
        nstage = loge ? (logl + loge - 1) / loge : 1;
        int ns = 1;
        tw_size = 0;
        twb_size = 0;
        for (int st = 0; st < nstage; ++st) {
            radix[st] = st < nstage - 1 ? E : (1 << (logl - loge * (nstage - 1)));
            span[st] = ns;
            if (st >= 1) tw_size += ns * (radix[st] - 1);
            if (st >= 1) twb_size += ns;
            ns *= radix[st];
        }
    }
};

constexpr int GS_MAXK = 32;  // states a Gram-Schmidt call can orthogonalise against

template <typename R> struct GSArgs {
    using V = cplx_t<R>;
    V* psi;                   // state being orthonormalised
    const V* states[GS_MAXK]; // previous states
    int k0, nk;               // dot kernel: states[k0 .. k0+nk) (nk <= MAX_RED/2)
    int j;                    // axpy kernel: subtract states[0..j)
    const double* coef;       // [2*j] (re, im) projection coefficients
    long long n;
    RedDesc red;
};

template <typename R> void launch_gs_dot(const GSArgs<R>& a, cudaStream_t st, int nblocks);
template <typename R> void launch_gs_axpy(const GSArgs<R>& a, cudaStream_t st, int nblocks);
template <typename R> void launch_grid_reduce(const PassArgs<R>& a, long long n, cudaStream_t st, int nblocks);
template <typename R> void launch_scale(cplx_t<R>* psi, long long n, const double* scale_dev, cudaStream_t st);
void launch_gs_finalize(const double* norm2, double tol, double* scale, int* flag, cudaStream_t st);

// Per-step field tables for a chunk of steps; each (step, stage) block holds sum_j N_j values,
// axis j at offset off[j].
//  length:   out = exp(-i h_ia r_j[i] E[step][ia][j])                     (r-space, per axis)
//  velocity: out = exp(-i h_ia (p_j^2/2 + (p_j + A_j/2) A_j)) / N_j        (k-space, per axis)
struct FieldTableArgs {
    const double* field;  // [nsteps][s][dim]
    const double* axes;   // concatenated r (length) or p (velocity) axes
    int nsteps, s, dim;
    int nr[MAX_DIM], off[MAX_DIM], ntot;
    double h[32];
    int velocity;
    int conj_from;        // steps from this one on get the conjugate factors (adjoint sweeps)
};
template <typename R> void launch_field_tables(const FieldTableArgs& a, cplx_t<R>* out, cudaStream_t st);

// Laser field samples at the integrator's sub-step times (Initialize_field_vectors,
// integrators.c:74-101) from the modes of Field_vectors (parameters.c:899-949).
constexpr int MAX_MODES = 16;
enum : int { ENV_CONSTANT = 0, ENV_TRAPZ = 1, ENV_COS2 = 2, ENV_COS4 = 3 };
struct FieldMode {
    double w, F0, xi, cep, delay, tau;
    int env;
};
struct FieldSampleArgs {
    FieldMode mode[MAX_MODES];
    int nmodes, dim, s;
    long long nsteps;
    double dt;
    double as[20];
};
// E, A: [nsteps][s][dim] at the sub-step times; alpha: [nsteps][dim] = A(i dt). Any may be null.
void launch_field_samples(const FieldSampleArgs& a, double* E, double* A, double* alpha, cudaStream_t st);

// The centring + superposition of Read_wavefunction_MPI (io_functions.c:292-459):
// psi[i + off] (+)= c src[i] over the source grid, points outside psi's grid dropped.
struct EmbedArgs {
    long long n_src;
    int dim;
    long long nr_src[MAX_DIM], nr[MAX_DIM], off[MAX_DIM];
    double cr, ci;
};
template <typename R> void launch_embed(const EmbedArgs& a, const double2* src, cplx_t<R>* psi, cudaStream_t st);

// Per-axis tables that depend on a runtime shift alpha:
//   mode 0: w[k] = p[k] + alpha (double)            dipole_v weights
//   mode 1: spec[k] = (p[k] + alpha) / N (complex)   Lz operator
template <typename R> void launch_axis_table(int mode, const double* p, int N, double alpha, void* out, cudaStream_t st);

// Final photoelectron spectra (Write_final_observables, io_functions.c:136-287).
struct SpectraArgs {
    const double* r;      // concatenated r axes
    const double* p;      // concatenated p axes (FFT order)
    const int* rank;      // concatenated per-axis rank among the kept momenta (|p| <= pr_max), -1 if not kept
    int axoff[MAX_DIM];
    int shift[MAX_DIM];
    long long nmask[MAX_DIM];
    long long stride[MAX_DIM];  // strides of the packed PMD array
    int dim;
    long long n;
    double rmin, rmax;    // sin^2 mask between rmin and rmax, 1 beyond (R_MASK)
    double de, sigma, norm;
    int ne;
};
constexpr int PED_CHUNK = 256;  // elements per block of the energy-distribution partial sums
template <typename R>
void launch_radial_mask(const SpectraArgs& a, const cplx_t<R>* in, cplx_t<R>* out, cudaStream_t st);
template <typename R>
void launch_ped(const SpectraArgs& a, const cplx_t<R>* psi_p, double* partials, double* out, cudaStream_t st);
template <typename R> void launch_pmd(const SpectraArgs& a, const cplx_t<R>* psi_p, double* out, cudaStream_t st);

// Axes longer than one pass handles (1-D, N = N1 N2): the four-step transform over the virtual
// N1 x N2 grid (index n1 N2 + n2), see long_fft in qnd_engine.cu. Slot k1 N2 + k2 of its output
// holds frequency k1 + N1 k2.
struct LongArgs {
    long long n;          // N
    int log2n1, log2n2;
};
// psi[k1 N2 + n2] times the stored twiddle w[k1 N2 + n2] (W_N^{k1 n2}), or its conjugate
template <typename R> void launch_long_twiddle(const LongArgs& a, cplx_t<R>* psi, const cplx_t<R>* w, int conj,
                                               cudaStream_t st);
// to_natural: out[k1 + N1 k2] = in[k1 N2 + k2]; otherwise the inverse permutation
template <typename R> void launch_long_transpose(const LongArgs& a, const cplx_t<R>* in, cplx_t<R>* out, int to_natural,
                                                 cudaStream_t st);
// Point-wise factors of a 1-D state in natural order: real table, complex table, per-axis complex
// table, real per-axis table (the mask), device scalar; any may be null.
template <typename R> void launch_point_factors(long long n, cplx_t<R>* psi, const R* tr, const cplx_t<R>* tc,
                                                const cplx_t<R>* pc, const R* pr, const double* scale_dev,
                                                cudaStream_t st);
// psi *= prod_j mask_j[index along axis j] over the axes whose mask is set (natural layout)
template <typename R> void launch_apply_masks(long long n, cplx_t<R>* psi, int dim, const int* shift,
                                              const long long* nmask, const R* const* masks, cudaStream_t st);
// dst += vtab * src (H psi = T psi + V psi)
template <typename R> void launch_add_potential(long long n, cplx_t<R>* dst, const cplx_t<R>* src, const double* vtab,
                                                cudaStream_t st);

// ---- passes along an axis longer than one pass holds, on a grid of several dimensions
// (emulate_long_pass in qnd_engine.cu): element-wise work along that axis in natural order.
// psi *= tr[lm] * tc[lm] * prod_k axc[k][i_k] * prod_k axr[k][i_k] * spec[i_axis] * spec_scale * *scale_dev,
// every table optional; lm is the element's index in the line-major order of the axis (the layout of
// the pass's full-grid tables), i_k its index along axis k.
struct AxisFactorArgs {
    long long n;
    int dim, axis, log2L;
    int shift[MAX_DIM];
    long long nmask[MAX_DIM];
    const void* tr;
    const void* tc;
    const void* axc[MAX_DIM];
    const void* axr[MAX_DIM];
    const void* spec;
    int spec_conj;
    double spec_scale;
    const double* scale_dev;
};
template <typename R> void launch_axis_factors(const AxisFactorArgs& a, cplx_t<R>* psi, cudaStream_t st);
// The four-step order along an axis of N = n1 n2 points at stride 2^shift (slot k1 n2 + k2 holds
// frequency k1 + n1 k2): out = in reordered to natural order (to_natural) or back to slot order.
struct AxisPermArgs {
    long long n;
    int shift, log2N, log2n1, log2n2;
};
template <typename R> void launch_axis_permute(const AxisPermArgs& a, const cplx_t<R>* in, cplx_t<R>* out,
                                               int to_natural, cudaStream_t st);
// dst = tmp + vtab * src (vtab may be null) + dst (when acc)
template <typename R> void launch_apply_combine(long long n, cplx_t<R>* dst, const cplx_t<R>* tmp,
                                               const cplx_t<R>* src, const double* vtab, int acc, cudaStream_t st);

// ---- the persistent sweep kernel (qnd_sweep.cu): recorded passes of many members in one launch
constexpr int SWEEP_NT = 128;  // threads per CTA: every line length it takes has 128-thread pass CTAs
// One recorded pass of one member: its arguments (PassArgs<R> in device memory), its line groups,
// and the groups of the member's earlier passes that must be done before it starts.
struct SweepSlot {
    const void* args;
    unsigned ngroups;
    unsigned need;      // groups of the member's earlier passes that must be done before this one
    unsigned gpi;       // line groups per work item (the last item of the pass may hold fewer)
    int member;
    int L, strided, kmode;
};
struct SweepArgs {
    const SweepSlot* slots;      // in round order: pass r of every member, member by member
    const long long* first;      // [nslots] the first work item of each slot
    int nslots;
    long long nitems;
    unsigned long long* next;    // item counter, zero at launch
    unsigned* done;              // [members] groups done, zero at launch
    int* abort_flag;             // raised when a wait runs out; zero at launch
    int wait_tries;
};
// Line lengths the sweep kernel is built for (every axis of every member).
constexpr bool sweep_length_ok(long long L) { return L == 128 || L == 256 || L == 512 || L == 1024; }
// Cooperative launch over every resident CTA slot (at most one per item); the grid size goes to grid_out.
template <typename R> cudaError_t launch_sweep(const SweepArgs& sa, cudaStream_t st, int num_sms, int* grid_out);

}  // namespace qnd
