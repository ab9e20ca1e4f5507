// qnd_pass_inst.cu — instantiates the fused axis-pass kernels for one line length.
// The build compiles this file once per supported length with -DQND_L=<L>.
#include "qnd_kernels.cuh"

#ifndef QND_L
#error "compile with -DQND_L=<line length>"
#endif

namespace qnd {

// A shape variant of the sandwich / two-sandwich passes (null where the variant is the default).
// sk: 0 contiguous, 1 strided with per-thread staging, 2 strided with TMA box staging
#define QND_SK(R, L, M, VAR) \
    (sk == 2 ? (const void*)&qnd_pass_kernel<R, L, 2, M, VAR> \
             : sk == 1 ? (const void*)&qnd_pass_kernel<R, L, 1, M, VAR> : (const void*)&qnd_pass_kernel<R, L, 0, M, VAR>)

template <typename R, int L, int VAR> static PassKernelInfo variant_info(int sk, int mode) {
    using SH = PassShape<R, L, VAR>;
    const void* fn = nullptr;
    if constexpr (SH::VALID) {
#define QND_PICKV(M) QND_SK(R, L, M, VAR)
        switch (mode) {
        case PM_SANDWICH: fn = QND_PICKV(PM_SANDWICH); break;
        case PM_DOUBLE: fn = QND_PICKV(PM_DOUBLE); break;
        case PM_SANDWICH_RED: fn = QND_PICKV(PM_SANDWICH_RED); break;
        case PM_DOUBLE_RED: fn = QND_PICKV(PM_DOUBLE_RED); break;
        case PM_DOUBLE_RED_END: fn = QND_PICKV(PM_DOUBLE_RED_END); break;
        default: fn = nullptr;
        }
#undef QND_PICKV
    }
    return PassKernelInfo{fn, SH::NT, SH::SMEM, SH::G, SH::TW_ENTRIES, SH::E};
}

template <typename R, int L> PassKernelInfo pass_kernel_info(bool strided, int mode, int var, bool tma) {
    const int sk = strided ? (tma ? 2 : 1) : 0;
    if (var == 1) return variant_info<R, L, 1>(sk, mode);
    if (var == 2) return variant_info<R, L, 2>(sk, mode);
    if (var == 3) return variant_info<R, L, 3>(sk, mode);
    using SH = PassShape<R, L>;
    const void* fn = nullptr;
#define QND_PICK(M) QND_SK(R, L, M, 0)
    switch (mode) {
    case PM_SANDWICH: fn = QND_PICK(PM_SANDWICH); break;
    case PM_FFT_FWD: fn = QND_PICK(PM_FFT_FWD); break;
    case PM_FFT_INV: fn = QND_PICK(PM_FFT_INV); break;
    case PM_SPECRED: fn = QND_PICK(PM_SPECRED); break;
    case PM_APPLY: fn = QND_PICK(PM_APPLY); break;
    case PM_DOUBLE: fn = QND_PICK(PM_DOUBLE); break;
    case PM_ROUNDTRIP: fn = QND_PICK(PM_ROUNDTRIP); break;
    case PM_SANDWICH_RED: fn = QND_PICK(PM_SANDWICH_RED); break;
    case PM_DOUBLE_RED: fn = QND_PICK(PM_DOUBLE_RED); break;
    case PM_DOUBLE_RED_END: fn = QND_PICK(PM_DOUBLE_RED_END); break;
    default: fn = nullptr;
    }
#undef QND_PICK
    return PassKernelInfo{fn, SH::NT, SH::SMEM, SH::G, SH::TW_ENTRIES, SH::E};
}

template PassKernelInfo pass_kernel_info<double, QND_L>(bool, int, int, bool);
template PassKernelInfo pass_kernel_info<float, QND_L>(bool, int, int, bool);

}  // namespace qnd
