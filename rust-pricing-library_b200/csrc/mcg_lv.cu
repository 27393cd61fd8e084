// mcg_lv.cu -- local-volatility Log-Euler path kernel (FP64).
//
// Compiled with -fmad=false: every a*b+c of the reference's arithmetic rounds
// twice, as Rust evaluates it.
//
// Per unit: normals (Philox or scrambled Sobol) -> time-ordered Brownian-bridge
// program -> Log-Euler steps on the forward-normalised state
//   x = ln(f / F_i),  v = bilinear(t_i, x),  f <- f * (F_{i+1}/F_i) * exp(-v dt/2 + sqrt(v) sqrt(dt) z)
// (crates/pricing/src/engine/processes/local_vol.rs:459-619) for up to three
// spot runtimes (base, S-h, S+h for CRN Delta/Gamma,
// crates/pricing/src/engine/risk/pathwise_local_vol.rs:332-355) and both
// antithetic signs, with streaming payoffs and the continuous-barrier bridge
// (crates/pricing/src/engine/processes/local_vol_valuation.rs:251-434).
#include "mcg_lv_tile.cuh"

namespace mcg {

template <int E, int NP>
__global__ void __launch_bounds__(kThreads) lv_path_kernel(const DevicePlan P, uint64_t unit_begin,
                                                           StatRecord* partials, uint32_t mask,
                                                           ErrorWord* err, int detail) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = static_cast<int>(P.nx);
    const size_t nv = static_cast<size_t>(P.nt) * P.nx;
    double* s_v = reinterpret_cast<double*>(smem_raw);
    double* s_x = s_v + nv;
    long long* s_xk = reinterpret_cast<long long*>(s_x + nx);
    double* s_w = reinterpret_cast<double*>(s_xk + nx);  // bridge slots [slot][thread]
    Stat* s_red = reinterpret_cast<Stat*>(s_w + static_cast<size_t>(P.slot_count) * kThreads);
    for (size_t i = threadIdx.x; i < nv; i += kThreads) s_v[i] = P.grid_v[i];
    for (int i = threadIdx.x; i < nx; i += kThreads) {
        s_x[i] = P.grid_x[i];
        s_xk[i] = total_key(P.grid_x[i]);
    }
    __syncthreads();
    const GridView g{s_v, s_x, s_xk, nx};
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < unit_begin + (detail ? 1 : P.units) && point < P.units;
    StatRecord* tile_out = partials + (static_cast<size_t>(scramble) * gridDim.x + blockIdx.x) * P.product_count * kComponents;
    lv_tile<E, NP>(P, g, s_w, s_red, scramble, point, valid, tile_out, mask, err, detail);
}


template __global__ void lv_path_kernel<1, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<1, 2>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<1, 4>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<2, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<2, 2>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<3, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<3, 2>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);
template __global__ void lv_path_kernel<6, 1>(const DevicePlan, uint64_t, StatRecord*, uint32_t, ErrorWord*, int);

// Launch helper: picks the instantiation for (evolutions, products).
cudaError_t launch_lv_path(const DevicePlan& P, uint64_t unit_begin, uint64_t units, uint32_t scrambles,
                           StatRecord* partials, uint32_t mask, ErrorWord* err, int detail,
                           cudaStream_t stream, int& evolutions_out) {
    const int pairs = P.antithetic ? 2 : 1;
    const int per = P.lv_bumps ? 3 : 1;
    const int E = pairs * per;
    evolutions_out = E;
    const int np = static_cast<int>(P.product_count);
    const size_t smem = (static_cast<size_t>(P.nt) * P.nx + 2 * P.nx) * sizeof(double) +
                        static_cast<size_t>(P.slot_count) * kThreads * sizeof(double) +
                        4 * kComponents * sizeof(Stat);
    const dim3 grid(static_cast<unsigned>((units + kThreads - 1) / kThreads), scrambles);
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<grid, kThreads, smem, stream>>>(P, unit_begin, partials, mask, err, detail);
        return cudaGetLastError();
    };
    if (E == 1 && np == 1) return go(lv_path_kernel<1, 1>);
    if (E == 1 && np == 2) return go(lv_path_kernel<1, 2>);
    if (E == 1 && np <= 4) return go(lv_path_kernel<1, 4>);
    if (E == 2 && np == 1) return go(lv_path_kernel<2, 1>);
    if (E == 2 && np == 2) return go(lv_path_kernel<2, 2>);
    if (E == 3 && np == 1) return go(lv_path_kernel<3, 1>);
    if (E == 3 && np == 2) return go(lv_path_kernel<3, 2>);
    if (E == 6 && np == 1) return go(lv_path_kernel<6, 1>);
    return cudaErrorNotSupported;
}

}  // namespace mcg
