// mcg_bs.cu -- Black--Scholes path kernel (FP64, compiled with -fmad=false).
//
// Single-terminal products take the exact lognormal step and the pathwise
// adjoint of pathwise_aad_single_terminal
// (crates/pricing/src/engine/processes/black_scholes.rs:757-793), evaluated
// at the base point and the six bumped points of pathwise_values (:417-472):
// spot bumps reuse the base exponential bit for bit, only the two volatility
// bumps need their own.  Multi-observation products follow the cumulative
// Brownian motion of path_observations_from_normals (:297-331) with streaming
// payoffs and the continuous-barrier bridge (:94-293).
#include "mcg_bs_tile.cuh"

namespace mcg {

// Single-terminal kernel (European/Digital at expiry), price-only or risk.
template <bool kRisk>
__global__ void __launch_bounds__(kThreads) bs_terminal_kernel(const DevicePlan P, uint64_t unit_begin,
                                                               StatRecord* partials, uint32_t mask,
                                                               ErrorWord* err, int detail) {
    __shared__ Stat s_red[4 * kComponents];
    (void)err;
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < unit_begin + (detail ? 1 : P.units) && point < P.units;
    StatRecord* tile_out = partials + (static_cast<size_t>(scramble) * gridDim.x + blockIdx.x) * P.product_count * kComponents;
    bs_terminal_tile<kRisk>(P, s_red, scramble, point, valid, tile_out, mask);
}

// Multi-observation kernel, price and barrier diagnostics (NP products; EV
// evolutions: 2 with the antithetic mate).  Several products or evolutions
// run at 5 CTAs per SM (96 registers; left free they took 118-248 registers:
// four antithetic products at 2^20 x 252 ran 13.0 against 10.8 ms).
template <int NP, int EV>
__global__ void __launch_bounds__(kThreads, (NP == 1 && EV == 1) ? 1 : 5) bs_path_kernel(const DevicePlan P, uint64_t unit_begin,
                                                           StatRecord* partials, uint32_t mask,
                                                           ErrorWord* err, int detail) {
    __shared__ Stat s_red[4 * kComponents];
    __shared__ double s_z[z_batch<1>() * kThreads];                 // batched normals [k][thread]
    __shared__ uint16_t s_zlist[(kThreads / 32) * 32 * z_batch<1>()];  // tail lists, per warp
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < unit_begin + (detail ? 1 : P.units) && point < P.units;
    StatRecord* tile_out = partials + (static_cast<size_t>(scramble) * gridDim.x + blockIdx.x) * P.product_count * kComponents;
    bs_path_tile<NP, EV>(P, s_red, scramble, point, valid, tile_out, mask, err, detail, nullptr, s_z, s_zlist);
}

cudaError_t launch_bs_path_risk(const DevicePlan& P, uint64_t unit_begin, uint64_t units, uint32_t scrambles,
                                StatRecord* partials, uint32_t mask, ErrorWord* err, int detail,
                                cudaStream_t stream);

cudaError_t launch_bs_path(const DevicePlan& P, bool single_terminal, uint64_t unit_begin, uint64_t units,
                           uint32_t scrambles, StatRecord* partials, uint32_t mask, ErrorWord* err,
                           int detail, cudaStream_t stream) {
    const dim3 grid(static_cast<unsigned>((units + kThreads - 1) / kThreads), scrambles);
    if (single_terminal) {
        if (P.risk)
            bs_terminal_kernel<true><<<grid, kThreads, 0, stream>>>(P, unit_begin, partials, mask, err, detail);
        else
            bs_terminal_kernel<false><<<grid, kThreads, 0, stream>>>(P, unit_begin, partials, mask, err, detail);
        return cudaGetLastError();
    }
    if (P.risk) return launch_bs_path_risk(P, unit_begin, units, scrambles, partials, mask, err, detail, stream);
    const int np = static_cast<int>(P.product_count);
    auto go = [&](auto kernel) {
        kernel<<<grid, kThreads, 0, stream>>>(P, unit_begin, partials, mask, err, detail);
        return cudaGetLastError();
    };
    const bool anti = P.antithetic != 0;
    if (np == 1) return anti ? go(bs_path_kernel<1, 2>) : go(bs_path_kernel<1, 1>);
    if (np == 2) return anti ? go(bs_path_kernel<2, 2>) : go(bs_path_kernel<2, 1>);
    if (np <= 4) return anti ? go(bs_path_kernel<4, 2>) : go(bs_path_kernel<4, 1>);
    return cudaErrorNotSupported;
}

}  // namespace mcg
