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

// Occupancy: one evolution with at most two discrete products runs two paths
// per thread (Q = 2: two tiles per CTA, their dependency chains interleaved
// and the per-step record, grid rows, product dispatch and Sobol direction
// rows shared) at 5 CTAs of 128 threads per SM (96 registers); one path per
// thread runs 7 CTAs, 5 with a continuous barrier; the multi-evolution
// (antithetic, CRN) and four-product kernels are held to 5 CTAs as well
// (96 registers, some spilled to L1): left free they took 150-240 registers
// and 1-3 CTAs, and ran 1.1-1.6x slower (CRN Delta/Gamma under a smoothed
// continuous barrier, 2^20 x 252: 86.2 -> 54.0 ms).  The grid values are
// read through L1 (24.8 KB for 31 x 100), so shared memory holds only the x
// nodes, the bridge slots and the batched normals.
template <int E, int NP, int RQ, int CB, int Q>
__global__ void __launch_bounds__(kThreads, (E == 1 && NP <= 2) ? (Q == 2 ? 5 : (CB == 0 ? 7 : 5)) : 5)
    lv_path_kernel(const DevicePlan P, uint64_t unit_begin, StatRecord* partials, uint32_t mask, ErrorWord* err,
                   int detail) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = static_cast<int>(P.nx);
    double2* s_b = reinterpret_cast<double2*>(smem_raw);  // cell bounds {x[c], x[c+1]}
    double* s_w = reinterpret_cast<double*>(s_b + nx);    // bridge slots [q][slot][thread]
    Stat* s_red = reinterpret_cast<Stat*>(s_w + static_cast<size_t>(Q) * P.slot_count * kThreads);
    double* s_z = reinterpret_cast<double*>(s_red + 4 * kComponents);       // batched normals [k][q][thread]
    uint16_t* s_zlist = reinterpret_cast<uint16_t*>(s_z + z_batch<Q>() * Q * kThreads);  // tail lists, per warp
    for (int i = threadIdx.x; i + 1 < nx; i += kThreads) s_b[i] = make_double2(P.grid_x[i], P.grid_x[i + 1]);
    __syncthreads();
    // cell records through L1, bounds in shared memory
    const GridView g{nullptr, nullptr, nullptr, nx, s_b, P.grid_cells, P.grid_x[0], P.grid_x[nx - 1]};
    const uint32_t scramble = blockIdx.y;
    const size_t rec = static_cast<size_t>(P.product_count) * kComponents;
    if constexpr (Q == 1) {
        const uint64_t point = unit_begin + static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
        const bool valid = point < unit_begin + (detail ? 1 : P.units) && point < P.units;
        StatRecord* tile_out = partials + (static_cast<size_t>(scramble) * gridDim.x + blockIdx.x) * rec;
        lv_tile<E, NP, RQ, CB>(P, g, s_w, s_red, scramble, point, valid, tile_out, mask, err, detail,
                               (unit_begin & 31u) == 0, s_z, s_zlist);
    } else {
        // The whole plan from unit 0: CTA b holds tiles 2b and 2b + 1.
        const uint64_t tiles = (P.units + kThreads - 1) / kThreads;
        const uint64_t tile = static_cast<uint64_t>(blockIdx.x) * Q;
        const uint64_t point = tile * kThreads + threadIdx.x;
        StatRecord* base = partials + static_cast<size_t>(scramble) * tiles * rec;
        StatRecord* second = tile + 1 < tiles ? base + (tile + 1) * rec : nullptr;
        lv_tile<E, NP, RQ, CB, Q>(P, g, s_w, s_red, scramble, point, point < P.units, base + tile * rec, mask, err,
                                  detail, true, s_z, s_zlist, point + kThreads < P.units, second);
    }
}


// Early-exercise path store under local volatility: the Log-Euler paths of
// lv_tile on the base runtime (both antithetic signs, E = pairs), their state
// at every exercise date written date-major, spots[d * paths + unit * E + e]
// (write_local_vol_lsm_trajectory, crates/pricing/src/engine/mc/early_exercise.rs:389-450;
// the observation's post-dividend spot is 0 * S0 + 1 * state).  `domain` is
// the Philox RandomDomain (Valuation 0, LsmTrain 1) of pseudo paths.
template <int E>
__global__ void __launch_bounds__(kThreads) lsm_lv_spots_kernel(const DevicePlan P, uint32_t domain,
                                                                double* spots, uint64_t paths, ErrorWord* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nx = static_cast<int>(P.nx);
    const size_t nv = static_cast<size_t>(P.nt) * P.nx;
    double* s_v = reinterpret_cast<double*>(smem_raw);
    double* s_x = s_v + nv;
    long long* s_xk = reinterpret_cast<long long*>(s_x + nx);
    double* s_w = reinterpret_cast<double*>(s_xk + nx);
    for (size_t i = threadIdx.x; i < nv; i += kThreads) s_v[i] = P.grid_v[i];
    for (int i = threadIdx.x; i < nx; i += kThreads) {
        s_x[i] = P.grid_x[i];
        s_xk[i] = total_key(P.grid_x[i]);
    }
    __syncthreads();
    const GridView g{s_v, s_x, s_xk, nx};
    const uint32_t scramble = blockIdx.y;
    const uint64_t point = static_cast<uint64_t>(blockIdx.x) * kThreads + threadIdx.x;
    const bool valid = point < P.units;
    const uint64_t local = valid ? point : 0;
    NormalSource ns;
    ns.rqmc = P.engine == MCG_ENGINE_RQMC;
    ns.seed = P.seed;
    ns.unit = local;
    ns.gray = static_cast<uint32_t>(local ^ (local >> 1));
    ns.dirs = P.scr_dirs ? P.scr_dirs + static_cast<size_t>(scramble) * P.dimension * 32u : nullptr;
    ns.shift = P.scr_shift ? P.scr_shift + static_cast<size_t>(scramble) * P.dimension : nullptr;
    ns.cached_block = 0xffffffffu;
    ns.domain = domain;
    const uint64_t unit = static_cast<uint64_t>(scramble) * P.units + local;
    double f[E];
    int hint[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
        f[e] = P.spot_variant[0];
        hint[e] = 0;
    }
    int fail_code = 0;
    uint32_t fail_step = 0;
    double fail_value = 0.0;
    double* w = s_w + threadIdx.x;
    for (uint32_t oi = 0; oi < P.op_count; ++oi) {
        const Op op = P.ops[oi];
        if (op.kind == kOpZero) {
            w[op.out * kThreads] = 0.0;
            continue;
        }
        if (op.kind == kOpTerminal) {
            w[op.out * kThreads] = op.sd * ns.normal(op.rank);
            continue;
        }
        if (op.kind == kOpInterior) {
            const double z = ns.normal(op.rank);
            w[op.out * kThreads] = op.wl * w[op.left * kThreads] + op.wr * w[op.right * kThreads] + op.sd * z;
            continue;
        }
        const uint32_t s = static_cast<uint32_t>(op.step);
        const double shock = op.kind == kOpStep ? (w[op.right * kThreads] - w[op.left * kThreads]) * P.inv_sqrt_dt[s]
                                                : ns.normal(op.rank);
        const int tc = P.time_cell[s];
        const double tw = P.time_weight[s];
        const double dt = P.dt[s];
        const double sq = P.sqrt_dt[s];
        const int32_t obs = P.obs_of_node[s + 1];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const double z = e == 0 ? shock : -shock;
            const double x = log(f[e] / P.fwd[s]);
            const double v = interp_variance(g, tc, tw, x, hint[e]);
            f[e] *= P.ratio[s] * exp(-0.5 * v * dt + sqrt(v) * sq * z);
            if (!(isfinite(f[e]) && f[e] > 0.0) && !fail_code) {
                fail_code = MCG_ERR_NON_FINITE_STATE;
                fail_step = s + 1;
                fail_value = f[e];
            }
            if (obs >= 0 && valid) spots[static_cast<size_t>(obs) * paths + unit * E + e] = 0.0 * P.spot + 1.0 * f[e];
        }
    }
    if (valid && fail_code) report_error(err, unit, fail_code, fail_step, fail_value, false);
}

template __global__ void lsm_lv_spots_kernel<1>(const DevicePlan, uint32_t, double*, uint64_t, ErrorWord*);
template __global__ void lsm_lv_spots_kernel<2>(const DevicePlan, uint32_t, double*, uint64_t, ErrorWord*);

cudaError_t launch_lsm_lv_spots(const DevicePlan& P, uint32_t domain, double* spots, uint64_t paths, ErrorWord* err,
                                cudaStream_t stream) {
    const size_t smem = (static_cast<size_t>(P.nt) * P.nx + 2 * P.nx) * sizeof(double) +
                        static_cast<size_t>(P.slot_count) * kThreads * sizeof(double);
    const dim3 grid(static_cast<unsigned>((P.units + kThreads - 1) / kThreads), P.scramble_count);
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<grid, kThreads, smem, stream>>>(P, domain, spots, paths, err);
        return cudaGetLastError();
    };
    return P.antithetic ? go(lsm_lv_spots_kernel<2>) : go(lsm_lv_spots_kernel<1>);
}

// Shared memory of a path-kernel launch with Q paths per thread.
size_t lv_path_smem(const DevicePlan& P, int Q) {
    return (2 * static_cast<size_t>(P.nx)) * sizeof(double) +
           static_cast<size_t>(Q) * P.slot_count * kThreads * sizeof(double) + 4 * kComponents * sizeof(Stat) +
           static_cast<size_t>(Q == 2 ? z_batch<2>() : z_batch<1>()) * Q * kThreads * sizeof(double) +
           (kThreads / 32) * 32 * (Q == 2 ? z_batch<2>() : z_batch<1>()) * Q * sizeof(uint16_t);
}

// Launch helper: picks the instantiation for (evolutions, products).  A whole
// plan evaluated from unit 0 with one evolution runs two paths per thread;
// a re-run of one unit (detail) and the multi-evolution kernels one.
cudaError_t launch_lv_path(const DevicePlan& P, uint64_t unit_begin, uint64_t units, uint32_t scrambles,
                           StatRecord* partials, uint32_t mask, ErrorWord* err, int detail,
                           cudaStream_t stream, int& evolutions_out) {
    const int pairs = P.antithetic ? 2 : 1;
    const int per = P.lv_bumps ? 3 : 1;
    const int E = pairs * per;
    evolutions_out = E;
    const int np = static_cast<int>(P.product_count);
    bool cb = false;
    for (int k = 0; k < np; ++k) cb |= P.products[k].kind == MCG_PRODUCT_CONTINUOUS_BARRIER;
    // Two paths per thread pay for discrete products (B200: 87.4 -> 75.8 ms on the
    // 2^24-path local-vol workload); a continuous barrier's bridge state makes
    // the pair too large (25.0 -> 32.6 ms), so those kernels keep one, and so
    // do plans with discrete dividends (their observation coordinates are
    // compiled out of the two-path kernels, which otherwise spill).
    const bool two = E == 1 && np <= 2 && !cb && !P.dividends && !detail && unit_begin == 0 && units == P.units;
    const int Q = two ? 2 : 1;
    const size_t smem = lv_path_smem(P, Q);
    const dim3 grid(static_cast<unsigned>((units + kThreads * Q - 1) / (kThreads * Q)), scrambles);
    auto go = [&](auto kernel) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        kernel<<<grid, kThreads, smem, stream>>>(P, unit_begin, partials, mask, err, detail);
        return cudaGetLastError();
    };
    const bool rq = P.engine == MCG_ENGINE_RQMC;
    const bool smooth = cb && P.smoothing > 0.0;
    // (evolutions, products, paths per thread) x (engine, continuous barrier:
    // none, exact or smoothed) instantiations
#define MCG_LV_PICK(EE, NN, QQ)                                                       \
    do {                                                                              \
        if (rq && smooth) return go(lv_path_kernel<EE, NN, 1, 2, QQ>);                \
        if (rq && cb) return go(lv_path_kernel<EE, NN, 1, 1, QQ>);                    \
        if (rq) return go(lv_path_kernel<EE, NN, 1, 0, QQ>);                          \
        if (smooth) return go(lv_path_kernel<EE, NN, 0, 2, QQ>);                      \
        if (cb) return go(lv_path_kernel<EE, NN, 0, 1, QQ>);                          \
        return go(lv_path_kernel<EE, NN, 0, 0, QQ>);                                  \
    } while (0)
    if (two && np == 1) {
        if (rq) return go(lv_path_kernel<1, 1, 1, 0, 2>);
        return go(lv_path_kernel<1, 1, 0, 0, 2>);
    }
    if (two && np == 2) {
        if (rq) return go(lv_path_kernel<1, 2, 1, 0, 2>);
        return go(lv_path_kernel<1, 2, 0, 0, 2>);
    }
    if (E == 1 && np == 1) MCG_LV_PICK(1, 1, 1);
    if (E == 1 && np == 2) MCG_LV_PICK(1, 2, 1);
    if (E == 1 && np <= 4) MCG_LV_PICK(1, 4, 1);
    if (E == 2 && np == 1) MCG_LV_PICK(2, 1, 1);
    if (E == 2 && np == 2) MCG_LV_PICK(2, 2, 1);
    if (E == 3 && np == 1) MCG_LV_PICK(3, 1, 1);
    if (E == 3 && np == 2) MCG_LV_PICK(3, 2, 1);
    if (E == 6 && np == 1) MCG_LV_PICK(6, 1, 1);
#undef MCG_LV_PICK
    return cudaErrorNotSupported;
}

}  // namespace mcg
