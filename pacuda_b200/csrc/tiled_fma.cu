// The on-chip executor in f64 with multiply-adds contracted (PACUDA_B200_KERNEL_F64_FMA): the
// same source as the f64 kind, compiled in this file with -fmad=true, so that the compiler fuses
// a product and the sum it feeds into one DFMA (one rounding instead of two). Its values differ
// from the reference's f64 arithmetic in the last bits (about 1e-15 relative per operation); the
// plan's structure, order of operations and everything else are the f64 kind's.
#include "tiled.cuh"

namespace pacuda {

// a kind of its own (so that its kernels are not the -fmad=false f64 kind's instantiations)
struct KindF64Fma : Kind<double, double, double, double> {};

const void *tiled_fma_kernel(bool abi) {
    return abi ? (const void *)run_tiled<KindF64Fma, true> : (const void *)run_tiled<KindF64Fma, false>;
}

}  // namespace pacuda
