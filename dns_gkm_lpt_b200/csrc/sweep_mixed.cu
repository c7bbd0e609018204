// Mixed-precision form of the sweeps (the precision pattern beside the FP64 drop-in): WENO
// reconstruction and the gas-kinetic flux in single precision on
// non-dimensional values, the BGK time coefficients in double (their
// 1 - exp(-dt/tau) differences cancel), the state, the flux differences and the
// update in FP64, exactly as the FP64 sweeps accumulate them.
//
// Compiled with fast single-precision math (-use_fast_math: approximate
// division, square root and exp, denormals flushed; the FP64 arithmetic of
// this file is unaffected by that flag) and with the flux's two half-Maxwellian
// sides as one loop body (-DGKM_UNROLL_SIDES=0), the faster code shape for
// the single-precision flux.
#include "sweep_impl.cuh"

namespace gkm {
namespace {

template <int DIR>
cudaError_t launch_one_mixed(const SweepArgs& a, int nseg, cudaStream_t s)
{
    using Tile = SweepTile32a;
    dim3 grid((a.fc.n + Tile::TB - 1) / Tile::TB, (a.fc.n + Tile::TA - 1) / Tile::TA, nseg);
    dim3 block(Tile::TB, Tile::TA);
    launch_form<DIR, float, Tile>(a, grid, block, s);
    return cudaGetLastError();
}

}  // namespace

cudaError_t sweep_mixed_prepare()
{
    using Tile = SweepTile32a;
    cudaError_t e = set_form_smem<0, float, Tile>();
    if (e == cudaSuccess) e = set_form_smem<1, float, Tile>();
    if (e == cudaSuccess) e = set_form_smem<2, float, Tile>();
    if (e == cudaSuccess) e = set_ensemble_smem<float, Tile>();
    return e;
}

cudaError_t launch_ensemble_sweep32(int dir, int variant, const MemberDev* mem, const long long* off,
                                    const long long* order, int nm, int parity, unsigned long long* next,
                                    cudaStream_t s)
{
    (void)variant;
    return launch_ensemble_sweep_t<float, SweepTile32a>(dir, mem, off, order, nm, parity, next, s);
}

cudaError_t launch_sweep_mixed_rows(int dir, int variant, SweepArgs a, int j0, int j1, cudaStream_t s)
{
    (void)variant;
    return launch_sweep_rows_t<float, SweepTile32a>(dir, a, j0, j1, s);
}

cudaError_t launch_sweep_mixed(int dir, int variant, const SweepArgs& a, int nseg, cudaStream_t s)
{
    (void)variant;   // one window for the single-precision sweeps
    if (dir == 0) return launch_one_mixed<0>(a, nseg, s);
    if (dir == 1) return launch_one_mixed<1>(a, nseg, s);
    return launch_one_mixed<2>(a, nseg, s);
}

}  // namespace gkm
