// mcg_surface.cuh -- implied-variance surfaces and their Dupire local
// variance, evaluated once per grid node (mcg_setup.cu kernels).
//
// Total variance w(t, k) and its derivatives w_k, w_kk, w_t
// (ImpliedVarianceSurface::total_variance_derivatives) for
//   * standard SSVI (crates/pricing/src/market/ssvi.rs:410-479): theta(t) from
//     the PCHIP curve (crates/pricing/src/market/pchip.rs:111-176), phi(theta)
//     power-law or Heston-like (ssvi.rs:121-176);
//   * eSSVI (crates/pricing/src/market/essvi.rs:192-396): (theta, psi, rho psi)
//     linear in time between slices, scaled by t / t_0 before the first,
//     theta extended by the terminal slope after the last.
// The local variance is w_t over the Durrleman density factor
// (ssvi.rs:226-273), floored and capped as classify_local_variance
// (crates/pricing/src/market/local_variance.rs:607-627).
//
// Compiled with -fmad=false: every a*b+c rounds twice, as the reference's
// Rust arithmetic does.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mcg.h"

namespace mcg {

struct Surface {
    int32_t kind;
    // SSVI theta curve: knots, values, PCHIP derivatives, long-end slope
    const double* t;
    const double* v;
    const double* d;
    uint32_t n;
    double slope;
    double rho, eta, gamma, lambda;
    // eSSVI slices
    const double* st;
    const double* stheta;
    const double* spsi;
    const double* srho_psi;
    uint32_t slices;
};

struct TotalVariance {
    double w, wk, wkk, wt;
};

// ThetaPchip::evaluate (pchip.rs:111-176): value and time derivative.
__device__ __forceinline__ int64_t surface_time_key(double x) {
    const int64_t b = __double_as_longlong(x);
    return b ^ static_cast<int64_t>(static_cast<uint64_t>(b >> 63) >> 1);
}

__device__ inline void pchip_theta(const Surface& c, double time, double& theta, double& deriv) {
    if (time == 0.0) time = 0.0;
    if (time < c.t[0]) {
        deriv = c.v[0] / c.t[0];
        theta = time * deriv;
        return;
    }
    const int64_t key = surface_time_key(time);
    uint32_t lo = 0, hi = c.n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (surface_time_key(c.t[mid]) < key) lo = mid + 1; else hi = mid;
    }
    if (lo < c.n && surface_time_key(c.t[lo]) == key) {
        theta = c.v[lo];
        deriv = c.d[lo];
        return;
    }
    if (lo < c.n) {
        const uint32_t r = lo, l = lo - 1;
        const double width = c.t[r] - c.t[l];
        const double sc = (time - c.t[l]) / width;
        const double sc2 = sc * sc;
        const double sc3 = sc2 * sc;
        const double h00 = 2.0 * sc3 - 3.0 * sc2 + 1.0;
        const double h10 = sc3 - 2.0 * sc2 + sc;
        const double h01 = -2.0 * sc3 + 3.0 * sc2;
        const double h11 = sc3 - sc2;
        theta = h00 * c.v[l] + h10 * width * c.d[l] + h01 * c.v[r] + h11 * width * c.d[r];
        const double d00 = (6.0 * sc2 - 6.0 * sc) / width;
        const double d10 = 3.0 * sc2 - 4.0 * sc + 1.0;
        const double d01 = (-6.0 * sc2 + 6.0 * sc) / width;
        const double d11 = 3.0 * sc2 - 2.0 * sc;
        deriv = d00 * c.v[l] + d10 * c.d[l] + d01 * c.v[r] + d11 * c.d[r];
        return;
    }
    const uint32_t last = c.n - 1;
    theta = c.v[last] + c.slope * (time - c.t[last]);
    deriv = c.slope;
}

// PhiSpec::evaluate (ssvi.rs:121-176): phi(theta) and d phi / d theta.
__device__ inline void ssvi_phi(const Surface& c, double theta, double& phi, double& dphi) {
    if (c.kind == MCG_SURFACE_SSVI_POWER_LAW) {
        phi = c.eta / (pow(theta, c.gamma) * pow(1.0 + theta, 1.0 - c.gamma));
        dphi = -phi * (c.gamma / theta + (1.0 - c.gamma) / (1.0 + theta));
        return;
    }
    const double lambda = c.lambda;
    const double z = lambda * theta;
    if (fabs(z) <= 1.0e-4) {
        // the series of (z - 1 + e^-z) / z^2 and of its z-derivative, in Horner form
        phi = 0.5 + z * (-1.0 / 6.0 +
                         z * (1.0 / 24.0 + z * (-1.0 / 120.0 + z * (1.0 / 720.0 + z * (-1.0 / 5040.0 + z / 40320.0)))));
        const double by_z =
            -1.0 / 6.0 + z * (1.0 / 12.0 + z * (-1.0 / 40.0 + z * (1.0 / 180.0 + z * (-1.0 / 1008.0 + z / 6720.0))));
        dphi = lambda * by_z;
        return;
    }
    const double e = exp(-z);
    phi = (z - 1.0 + e) / (z * z);
    dphi = lambda * (2.0 - z - (z + 2.0) * e) / (z * z * z);
}

// eSSVI parameters at `time` (EssviSurface::parameters, essvi.rs:192-240 with
// interpolate/long_parameters, :299-340): theta, psi, rho psi and their time
// derivatives.
struct EssviParams {
    double theta, psi, rho_psi, dtheta, dpsi, drho_psi;
};

__device__ inline EssviParams essvi_params(const Surface& c, double time) {
    const uint32_t n = c.slices;
    if (time < c.st[0]) {
        const double inv = 1.0 / c.st[0];
        const double scale = time * inv;
        return {scale * c.stheta[0], scale * c.spsi[0], scale * c.srho_psi[0],
                c.stheta[0] * inv,   c.spsi[0] * inv,   c.srho_psi[0] * inv};
    }
    uint32_t lo = 0, hi = n;  // first slice with time >= `time`
    while (lo < hi) {
        const uint32_t mid = (lo + hi) / 2;
        if (c.st[mid] < time) lo = mid + 1; else hi = mid;
    }
    uint32_t left, right;
    if (lo < n && c.st[lo] == time) {
        if (lo + 1 >= n) lo = n;  // the last slice: long end
        left = lo < n ? lo : n - 1;
        right = left + 1;
    } else {
        left = lo - 1;
        right = lo;
    }
    if (lo >= n) {
        const uint32_t last = n - 1;
        return {c.stheta[last] + c.slope * (time - c.st[last]), c.spsi[last], c.srho_psi[last], c.slope, 0.0, 0.0};
    }
    const double width = c.st[right] - c.st[left];
    const double weight = (time - c.st[left]) / width;
    return {c.stheta[left] + weight * (c.stheta[right] - c.stheta[left]),
            c.spsi[left] + weight * (c.spsi[right] - c.spsi[left]),
            c.srho_psi[left] + weight * (c.srho_psi[right] - c.srho_psi[left]),
            (c.stheta[right] - c.stheta[left]) / width,
            (c.spsi[right] - c.spsi[left]) / width,
            (c.srho_psi[right] - c.srho_psi[left]) / width};
}

// Total variance derivatives at (time, k); false where the reference's
// surface reports a non-finite or non-positive value.
__device__ inline bool surface_total_variance(const Surface& c, double time, double k, TotalVariance& out) {
    if (c.kind == MCG_SURFACE_ESSVI) {
        // evaluate_total_variance, essvi.rs:342-396
        const EssviParams p = essvi_params(c, time);
        const double phi = p.psi / p.theta;
        const double rho = p.rho_psi / p.psi;
        const double rho_d = (p.drho_psi * p.psi - p.rho_psi * p.dpsi) / (p.psi * p.psi);
        const double phi_d = (p.dpsi * p.theta - p.psi * p.dtheta) / (p.theta * p.theta);
        const double y = phi * k;
        const double y_d = k * phi_d;
        const double a = y + rho;
        const double q = sqrt(a * a + 1.0 - rho * rho);
        const double q_d = (a * (y_d + rho_d) - rho * rho_d) / q;
        const double shape = 1.0 + rho * y + q;
        const double shape_d = rho_d * y + rho * y_d + q_d;
        out.w = p.theta * shape / 2.0;
        out.wk = p.theta * phi * (rho + a / q) / 2.0;
        out.wkk = p.theta * phi * phi * (1.0 - rho * rho) / (2.0 * q * q * q);
        out.wt = p.dtheta * shape / 2.0 + p.theta * shape_d / 2.0;
    } else {
        // StandardSsvi::total_variance_derivatives, ssvi.rs:410-479
        double theta, dtheta, phi, dphi;
        pchip_theta(c, time, theta, dtheta);
        ssvi_phi(c, theta, phi, dphi);
        const double rho = c.rho;
        const double y = phi * k;
        const double a = y + rho;
        const double q = sqrt(a * a + 1.0 - rho * rho);
        const double shape = 1.0 + rho * y + q;
        const double common = rho + a / q;
        out.w = theta * shape / 2.0;
        out.wk = theta * phi * common / 2.0;
        out.wkk = theta * phi * phi * (1.0 - rho * rho) / (2.0 * q * q * q);
        const double partial = shape / 2.0 + theta * k * dphi * common / 2.0;
        out.wt = partial * dtheta;
    }
    return isfinite(out.w) && isfinite(out.wk) && isfinite(out.wkk) && isfinite(out.wt) && out.w > 0.0;
}

cudaError_t launch_surface_grid(const Surface& s, const double* tn, uint32_t nt, const double* xn, uint32_t nx,
                                double floor, double cap, double* out, uint32_t* counters, cudaStream_t stream);
cudaError_t launch_surface_eval(const Surface& s, const double* times, const double* ks, uint32_t count,
                                double* out, uint32_t* failures, cudaStream_t stream);

}  // namespace mcg
