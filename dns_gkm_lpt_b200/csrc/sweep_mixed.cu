// Mixed-precision form of the sweeps (north-star precision pattern): WENO
// reconstruction and the gas-kinetic flux in single precision on
// non-dimensional values, the BGK time coefficients in double (their
// 1 - exp(-dt/tau) differences cancel), the state, the flux differences and the
// update in FP64, exactly as the FP64 sweeps accumulate them.
//
// Compiled with fast single-precision math (-use_fast_math: approximate
// division, square root and exp, denormals flushed); the FP64 arithmetic of
// this file is unaffected by that flag.
#include "sweep_impl.cuh"

namespace gkm {
namespace {

template <int DIR>
cudaError_t launch_one_mixed(const SweepArgs& a, int nseg, cudaStream_t s)
{
    dim3 grid((a.fc.n + kTB - 1) / kTB, (a.fc.n + kTA - 1) / kTA, nseg);
    dim3 block(kTB, kTA);
    sweep_kernel<DIR, float><<<grid, block, sweep_detail::sweep_smem_bytes<float>(), s>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_sweep_mixed(int dir, const SweepArgs& a, int nseg, cudaStream_t s)
{
    if (dir == 0) return launch_one_mixed<0>(a, nseg, s);
    if (dir == 1) return launch_one_mixed<1>(a, nseg, s);
    return launch_one_mixed<2>(a, nseg, s);
}

}  // namespace gkm
